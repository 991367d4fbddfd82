"""picomax_b200: B200 (sm_100a) implementation of PicoMax's EPM band solve and
chi(q, w) local-field accumulation behind the reference's own CLI and files.

The compute path is the in-tree shared library ``lib/libpicomax_b200.so``
(C-ABI in ``include/picomax.h``); this package binds it with ctypes and adds
the torch autograd wrapper. There is no CPU implementation of the GPU stages.
"""
from ._capi import (  # noqa: F401
    KGRID_TIME_REVERSAL, KGRID_LITTLE_GROUP_Q,
    PREC_FP64, PREC_MIXED, SWITCH_BAND, SWITCH_EPSIJ, SWITCH_EPSLL, SWITCH_EPSXYZ, CLI_PATH, LIB_PATH, Context,
    PicomaxError, Problem, load, run_main, PMX_OK, PMX_ERR_INVALID, PMX_ERR_CUDA, PMX_ERR_NOCONV, PMX_ERR_TIMEOUT,
    PMX_ERR_NO_DEVICE, PMX_ERR_UNSUPPORTED, PMX_ERR_LIMIT, PMX_ERR_IO, write_npz)
from .kgrid import gamma_grid, make_kfile, write_kfile  # noqa: F401
from . import dat  # noqa: F401
