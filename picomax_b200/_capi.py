"""ctypes binding of the picomax B200 C-ABI (include/picomax.h).

The shared library is built in-tree by ``picomax_b200/csrc/Makefile`` into
``picomax_b200/lib/libpicomax_b200.so``. There is no CPU implementation of the
two GPU stages: if the library is missing this module raises, and the stage
functions return ``PMX_ERR_NO_DEVICE`` when no CUDA device is visible.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_size_t, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpicomax_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "picomax")

PMX_OK = 0
PMX_ERR_INVALID = 1
PMX_ERR_CUDA = 2
PMX_ERR_NOCONV = 3
PMX_ERR_TIMEOUT = 4
PMX_ERR_NO_DEVICE = 5
PMX_ERR_UNSUPPORTED = 6
PMX_ERR_LIMIT = 7
PMX_ERR_IO = 8

SWITCH_NONE, SWITCH_BAND, SWITCH_EPSIJ, SWITCH_EPSLL, SWITCH_EPSXYZ = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1

# Every entry point declared in include/picomax.h.
EXPORTS = (
    "pmx_problem_create", "pmx_problem_destroy", "pmx_problem_get_info", "pmx_problem_gvectors",
    "pmx_problem_loci", "pmx_problem_kpoints", "pmx_problem_qpoints", "pmx_problem_dump",
    "pmx_problem_write_gpt", "pmx_ctx_create", "pmx_ctx_destroy", "pmx_ctx_last_error",
    "pmx_ctx_stage_times", "pmx_ctx_kernel_launches", "pmx_hamiltonian", "pmx_heev_batched",
    "pmx_ref_energy", "pmx_band", "pmx_chi", "pmx_kk", "pmx_main", "pmx_ctx_stream",
    "pmx_ctx_transfer_bytes", "pmx_ctx_degenerate_cuts", "pmx_chi_device", "pmx_chi_epsm",
    "pmx_eps_macroscopic", "pmx_ctx_kernel_time", "pmx_ctx_set_autotune", "pmx_ctx_set_schedule", "pmx_ctx_tuning", "pmx_ctx_mixed_mmas",
    "pmx_ctx_overlap_error",
    "pmx_heev_batched_noalloc",
    "pmx_problem_params",
    "pmx_problem_set_params",
    "pmx_band_vjp",
    "pmx_epsm_vjp", "pmx_ctx_set_wait_limit", "pmx_ctx_set_fault", "pmx_eels",
    "pmx_band_batch",
    "pmx_chi_batch",
    "pmx_ctx_occupation_ties",
    "pmx_problem_symmetry",
    "pmx_kgrid_reduce",
    "pmx_ctx_set_overlap_mode",
    "pmx_write_npz",
)

KGRID_TIME_REVERSAL, KGRID_LITTLE_GROUP_Q = 1, 2


class ProblemInfo(ctypes.Structure):
    _fields_ = [
        ("npw", c_int), ("nh", c_int), ("soc", c_int), ("neps", c_int), ("nband", c_int),
        ("nvalence", c_int), ("nk", c_int), ("nq", c_int), ("nfreq", c_int), ("natom", c_int),
        ("sw", c_int), ("debug", c_int), ("kk", c_int), ("delta", c_int), ("epsilon", c_double),
        ("dfreq", c_double), ("a", c_double), ("gcut", c_double), ("bz_volume", c_double),
        ("chi_values", c_longlong),
    ]


class PicomaxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Loads the in-tree shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C picomax_b200/csrc`")
    lib = ctypes.CDLL(LIB_PATH)
    dp, ip = POINTER(c_double), POINTER(c_int)
    sig = {
        "pmx_problem_create": (c_int, [c_int, POINTER(c_char_p), POINTER(c_void_p)]),
        "pmx_problem_destroy": (None, [c_void_p]),
        "pmx_problem_get_info": (c_int, [c_void_p, POINTER(ProblemInfo)]),
        "pmx_problem_gvectors": (c_int, [c_void_p, dp, ip]),
        "pmx_problem_loci": (c_int, [c_void_p, ip]),
        "pmx_problem_kpoints": (c_int, [c_void_p, dp, dp]),
        "pmx_problem_qpoints": (c_int, [c_void_p, dp]),
        "pmx_problem_dump": (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_size_t)]),
        "pmx_problem_write_gpt": (c_int, [c_void_p]),
        "pmx_write_npz": (c_int, [c_char_p, c_int, POINTER(c_char_p), POINTER(dp), ip, POINTER(c_longlong)]),
        "pmx_ctx_create": (c_int, [c_int, POINTER(c_void_p)]),
        "pmx_ctx_destroy": (None, [c_void_p]),
        "pmx_ctx_last_error": (c_char_p, [c_void_p]),
        "pmx_ctx_stage_times": (c_int, [c_void_p, dp]),
        "pmx_ctx_kernel_launches": (c_longlong, [c_void_p]),
        "pmx_hamiltonian": (c_int, [c_void_p, c_void_p, dp, c_int, dp]),
        "pmx_heev_batched": (c_int, [c_void_p, c_int, c_int, dp, c_int, dp, dp]),
        "pmx_ref_energy": (c_int, [c_void_p, c_void_p, dp]),
        "pmx_band": (c_int, [c_void_p, c_void_p, dp]),
        "pmx_chi": (c_int, [c_void_p, c_void_p, c_int, c_int, dp, dp]),
        "pmx_kk": (c_int, [c_void_p, c_int, c_int, c_double, dp, dp]),
        "pmx_main": (c_int, [c_int, POINTER(c_char_p)]),
        "pmx_ctx_stream": (c_void_p, [c_void_p]),
        "pmx_ctx_transfer_bytes": (c_int, [c_void_p, POINTER(c_longlong), POINTER(c_longlong)]),
        "pmx_ctx_degenerate_cuts": (c_int, [c_void_p]),
        "pmx_ctx_occupation_ties": (c_int, [c_void_p]),
        "pmx_chi_device": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
        "pmx_chi_epsm": (c_int, [c_void_p, c_void_p, c_int, c_int, dp, dp, dp]),
        "pmx_eps_macroscopic": (c_int, [c_void_p, c_int, c_int, c_int, dp, dp, dp]),
        "pmx_ctx_kernel_time": (c_int, [c_void_p, c_char_p, dp, POINTER(c_longlong)]),
        "pmx_ctx_set_autotune": (c_int, [c_void_p, c_int]),
        "pmx_ctx_set_schedule": (c_int, [c_void_p, c_int]),
        "pmx_ctx_mixed_mmas": (c_int, [c_void_p, POINTER(c_longlong)]),
        "pmx_ctx_overlap_error": (c_int, [c_void_p, dp, dp]),
        "pmx_heev_batched_noalloc": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
        "pmx_problem_params": (c_int, [c_void_p, dp, ip]),
        "pmx_problem_set_params": (c_int, [c_void_p, dp, c_int]),
        "pmx_band_vjp": (c_int, [c_void_p, c_void_p, dp, dp]),
        "pmx_epsm_vjp": (c_int, [c_void_p, c_void_p, dp, dp, dp, dp]),
        "pmx_ctx_set_wait_limit": (c_int, [c_void_p, c_longlong]),
        "pmx_ctx_set_fault": (c_int, [c_void_p, c_int]),
        "pmx_eels": (c_int, [c_void_p, c_int, c_int, c_double, c_double, dp, dp, dp]),
        "pmx_band_batch": (c_int, [c_void_p, c_int, POINTER(c_void_p), POINTER(dp)]),
        "pmx_chi_batch": (c_int, [c_void_p, c_int, POINTER(c_void_p), c_int, c_int, POINTER(dp), POINTER(dp),
                                  POINTER(dp)]),
        "pmx_ctx_tuning": (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_size_t)]),
        "pmx_problem_symmetry": (c_int, [c_void_p, c_int, ip, ip]),
        "pmx_kgrid_reduce": (c_int, [c_void_p, c_void_p, ip, c_int, ip, ip, ip]),
        "pmx_ctx_set_overlap_mode": (c_int, [c_void_p, c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int))


def _argv(args) -> tuple:
    toks = ["picomax"] + [str(a) for a in args]
    arr = (c_char_p * len(toks))(*[t.encode() for t in toks])
    return len(toks), arr


class Problem:
    """A parsed picomax invocation (argv without the program name)."""

    def __init__(self, args):
        lib = load()
        self._lib = lib
        self.args = list(args)
        argc, argv = _argv(self.args)
        h = c_void_p()
        st = lib.pmx_problem_create(argc, argv, ctypes.byref(h))
        if st != PMX_OK:
            raise PicomaxError(st, "pmx_problem_create rejected the options")
        self.handle = h
        info = ProblemInfo()
        lib.pmx_problem_get_info(h, ctypes.byref(info))
        self.info = info

    def close(self):
        if getattr(self, "handle", None):
            self._lib.pmx_problem_destroy(self.handle)
            self.handle = None

    __del__ = close

    def gvectors(self):
        n = self.info.npw
        G = np.zeros((n, 3), np.float64)
        H = np.zeros((n, 3), np.int32)
        self._lib.pmx_problem_gvectors(self.handle, _dptr(G), _iptr(H))
        return G, H

    def loci(self):
        L = np.zeros((self.info.neps, self.info.npw), np.int32)
        self._lib.pmx_problem_loci(self.handle, _iptr(L))
        return L

    def kpoints(self):
        K = np.zeros((self.info.nk, 3), np.float64)
        W = np.zeros(self.info.nk, np.float64)
        self._lib.pmx_problem_kpoints(self.handle, _dptr(K), _dptr(W))
        return K, W

    def symmetry_ops(self, flags: int = KGRID_TIME_REVERSAL) -> np.ndarray:
        """Point-group operations [nops, 3, 3] (integer, reciprocal basis; identity first)."""
        n = c_int()
        st = self._lib.pmx_problem_symmetry(self.handle, int(flags), ctypes.byref(n), None)
        if st != PMX_OK:
            raise PicomaxError(st, "pmx_problem_symmetry failed")
        ops = np.zeros((n.value, 9), np.int32)
        self._lib.pmx_problem_symmetry(self.handle, int(flags), ctypes.byref(n), _iptr(ops))
        return ops.reshape(-1, 3, 3)

    def qpoints(self):
        Q = np.zeros((self.info.nq, 3), np.float64)
        if self.info.nq:
            self._lib.pmx_problem_qpoints(self.handle, _dptr(Q))
        return Q

    def params(self) -> np.ndarray:
        """Form factors and SOC parameters (Ry) in the order of pmx_problem_params."""
        n = c_int()
        self._lib.pmx_problem_params(self.handle, None, ctypes.byref(n))
        v = np.zeros(n.value, np.float64)
        self._lib.pmx_problem_params(self.handle, _dptr(v), ctypes.byref(n))
        return v

    def set_params(self, values):
        v = np.ascontiguousarray(values, np.float64)
        st = self._lib.pmx_problem_set_params(self.handle, _dptr(v), len(v))
        if st != PMX_OK:
            raise PicomaxError(st, "pmx_problem_set_params: wrong parameter count")

    def dump(self) -> str:
        need = c_size_t()
        self._lib.pmx_problem_dump(self.handle, None, 0, ctypes.byref(need))
        buf = ctypes.create_string_buffer(need.value)
        self._lib.pmx_problem_dump(self.handle, buf, need.value, ctypes.byref(need))
        return buf.value.decode()


class Context:
    """Device context (one CUDA stream and its workspaces) on `device`."""

    def __init__(self, device: int = 0):
        lib = load()
        self._lib = lib
        h = c_void_p()
        st = lib.pmx_ctx_create(device, ctypes.byref(h))
        if st != PMX_OK:
            raise PicomaxError(st, "pmx_ctx_create failed (a CUDA device is required)")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self._lib.pmx_ctx_destroy(self.handle)
            self.handle = None

    __del__ = close

    def _check(self, st, what):
        if st != PMX_OK:
            raise PicomaxError(st, f"{what}: {self._lib.pmx_ctx_last_error(self.handle).decode()}")

    def stage_times(self):
        ms = np.zeros(5, np.float64)
        self._lib.pmx_ctx_stage_times(self.handle, _dptr(ms))
        return ms

    def kernel_launches(self) -> int:
        return int(self._lib.pmx_ctx_kernel_launches(self.handle))

    def hamiltonian(self, prob: Problem, kpts) -> np.ndarray:
        k = np.ascontiguousarray(kpts, np.float64).reshape(-1, 3)
        nh = prob.info.nh
        out = np.zeros((len(k), nh, nh, 2), np.float64)
        self._check(self._lib.pmx_hamiltonian(self.handle, prob.handle, _dptr(k), len(k), _dptr(out)), "hamiltonian")
        # stored column-major: out[k][col][row]
        return (out[..., 0] + 1j * out[..., 1]).transpose(0, 2, 1)

    def heev(self, A, nev: int, vectors: bool = True):
        """Lowest `nev` eigenpairs of Hermitian matrices A [batch, n, n]."""
        A = np.asarray(A, np.complex128)
        b, n, _ = A.shape
        colmajor = np.ascontiguousarray(A.transpose(0, 2, 1))
        buf = np.ascontiguousarray(np.stack([colmajor.real, colmajor.imag], -1))
        w = np.zeros((b, nev), np.float64)
        z = np.zeros((b, nev, n, 2), np.float64) if vectors else None
        st = self._lib.pmx_heev_batched(self.handle, n, b, _dptr(buf), nev, _dptr(w),
                                        _dptr(z) if vectors else None)
        self._check(st, "heev_batched")
        if not vectors:
            return w, None
        zc = z[..., 0] + 1j * z[..., 1]  # [b][nev][n]
        return w, zc.transpose(0, 2, 1)

    def ref_energy(self, prob: Problem) -> float:
        off = c_double()
        self._check(self._lib.pmx_ref_energy(self.handle, prob.handle, ctypes.byref(off)), "ref_energy")
        return off.value

    def band(self, prob: Problem) -> np.ndarray:
        out = np.zeros((prob.info.nq, prob.info.nband), np.float64)
        self._check(self._lib.pmx_band(self.handle, prob.handle, _dptr(out)), "band")
        return out

    def chi(self, prob: Problem, switch: int, precision: int = PREC_FP64):
        n = prob.info.chi_values
        re = np.zeros(n, np.float64)
        im = np.zeros(n, np.float64)
        self._check(self._lib.pmx_chi(self.handle, prob.handle, switch, precision, _dptr(re), _dptr(im)), "chi")
        return re, im

    def stream(self) -> int:
        return int(self._lib.pmx_ctx_stream(self.handle) or 0)

    def transfer_bytes(self):
        a, b = c_longlong(), c_longlong()
        self._lib.pmx_ctx_transfer_bytes(self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def kernel_time(self, family: str):
        """(device ms, launches) of one kernel family since the context was created."""
        ms, n = c_double(), c_longlong()
        self._lib.pmx_ctx_kernel_time(self.handle, family.encode(), ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def overlap_error(self):
        """(max ||M32|^2 - |M|^2|, max |M|^2) of the last mixed-precision chi call."""
        a, b = c_double(), c_double()
        self._lib.pmx_ctx_overlap_error(self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def set_autotune(self, on: bool):
        self._lib.pmx_ctx_set_autotune(self.handle, 1 if on else 0)

    def mixed_mmas(self) -> int:
        """tcgen05 MMA instructions (M128 N256 K16) of the mixed contractions so far."""
        v = c_longlong()
        self._check(self._lib.pmx_ctx_mixed_mmas(self.handle, ctypes.byref(v)), "mixed_mmas")
        return int(v.value)

    def set_wait_limit(self, ns: int):
        """Limit (ns) of the mixed contraction's bounded device waits (0: 2 s)."""
        self._check(self._lib.pmx_ctx_set_wait_limit(self.handle, int(ns)), "set_wait_limit")

    def set_fault(self, fault: int):
        """Test hooks: 1 = the mixed contraction's producers withhold one arrival
        (its wait runs out), 2 = the eigenvalue bisection stops after one round,
        3 = the two-stage bulge chase's second sweep waits for progress that
        never comes (its wait runs out), 4 = the tensor-core overlaps leave
        their first chunk uncommitted (a wait runs out); 0 = normal operation."""
        self._check(self._lib.pmx_ctx_set_fault(self.handle, int(fault)), "set_fault")

    def set_overlap_mode(self, mode: int):
        """Overlaps of the mixed path: 3 tensor cores (split TF32), 0 FP64
        rounded to FP32, 1 (default) the faster of the two for the problem
        (tensor cores without spin-orbit coupling), 2 both with the error
        reported by overlap_error."""
        self._check(self._lib.pmx_ctx_set_overlap_mode(self.handle, int(mode)), "set_overlap_mode")

    def set_schedule(self, schedule: int):
        """Fix the eigensolver schedule for later batches (-1: autotuner)."""
        self._check(self._lib.pmx_ctx_set_schedule(self.handle, schedule), "set_schedule")

    def tuning(self) -> dict:
        import json
        need = c_size_t()
        self._lib.pmx_ctx_tuning(self.handle, None, 0, ctypes.byref(need))
        buf = ctypes.create_string_buffer(need.value)
        self._lib.pmx_ctx_tuning(self.handle, buf, need.value, ctypes.byref(need))
        return json.loads(buf.value.decode())

    def degenerate_cuts(self) -> int:
        return int(self._lib.pmx_ctx_degenerate_cuts(self.handle))

    def occupation_ties(self) -> int:
        return int(self._lib.pmx_ctx_occupation_ties(self.handle))

    def chi_epsm(self, prob: Problem, switch: int, precision: int = PREC_FP64, chi: bool = True):
        """(re, im, eps_M); chi=False: eps_M only (re, im None; chi stays on the device)."""
        n = prob.info.chi_values
        re = np.zeros(n, np.float64) if chi else None
        im = np.zeros(n, np.float64) if chi else None
        eps = np.zeros((prob.info.nq, prob.info.nfreq, 2), np.float64)
        self._check(self._lib.pmx_chi_epsm(self.handle, prob.handle, switch, precision,
                                           _dptr(re) if chi else None, _dptr(im) if chi else None, _dptr(eps)),
                    "chi_epsm")
        return re, im, eps[..., 0] + 1j * eps[..., 1]

    def band_batch(self, probs):
        """pmx_band of several problems in merged launches: list of [nq][nband]."""
        outs = [np.zeros((p.info.nq, p.info.nband), np.float64) for p in probs]
        ph = (c_void_p * len(probs))(*[p.handle for p in probs])
        op = (POINTER(c_double) * len(probs))(*[_dptr(o) for o in outs])
        self._check(self._lib.pmx_band_batch(self.handle, len(probs), ph, op), "band_batch")
        return outs

    def chi_batch(self, probs, switch: int, precision: int = PREC_FP64, epsm: bool = False, chi: bool = True):
        """pmx_chi(_epsm) of several problems: list of (re, im[, eps_M]);
        chi=False (with epsm): eps_M only, re and im None."""
        n = len(probs)
        if not chi and not epsm:
            raise ValueError("chi=False needs epsm=True")
        res = [np.zeros(p.info.chi_values, np.float64) if chi else None for p in probs]
        ims = [np.zeros(p.info.chi_values, np.float64) if chi else None for p in probs]
        eps = [np.zeros((p.info.nq, p.info.nfreq, 2), np.float64) for p in probs] if epsm else None
        ph = (c_void_p * n)(*[p.handle for p in probs])
        rp = (POINTER(c_double) * n)(*[_dptr(x) for x in res]) if chi else None
        ip = (POINTER(c_double) * n)(*[_dptr(x) for x in ims]) if chi else None
        ep = (POINTER(c_double) * n)(*[_dptr(x) for x in eps]) if epsm else None
        self._check(self._lib.pmx_chi_batch(self.handle, n, ph, switch, precision, rp, ip, ep), "chi_batch")
        if epsm:
            return [(r, i, e[..., 0] + 1j * e[..., 1]) for r, i, e in zip(res, ims, eps)]
        return list(zip(res, ims))

    def band_vjp(self, prob: Problem, dE) -> np.ndarray:
        """dL/dparams from dL/d eband [nq][nband]."""
        dE = np.ascontiguousarray(dE, np.float64).reshape(prob.info.nq, prob.info.nband)
        g = np.zeros(len(prob.params()), np.float64)
        self._check(self._lib.pmx_band_vjp(self.handle, prob.handle, _dptr(dE), _dptr(g)), "band_vjp")
        return g

    def epsm_vjp(self, prob: Problem, deps, chi=None) -> np.ndarray:
        """dL/dparams from dL/d eps_M ([nq][nf] complex: dL/dRe + 1j dL/dIm);
        chi = (re, im) of a FP64 epsLL chi call on the same parameters, or None."""
        deps = np.asarray(deps, np.complex128).reshape(prob.info.nq, prob.info.nfreq)
        d = np.ascontiguousarray(np.stack([deps.real, deps.imag], -1))
        g = np.zeros(len(prob.params()), np.float64)
        if chi is None:
            st = self._lib.pmx_epsm_vjp(self.handle, prob.handle, None, None, _dptr(d), _dptr(g))
        else:
            re = np.ascontiguousarray(chi[0], np.float64)
            im = np.ascontiguousarray(chi[1], np.float64)
            st = self._lib.pmx_epsm_vjp(self.handle, prob.handle, _dptr(re), _dptr(im), _dptr(d), _dptr(g))
        self._check(st, "epsm_vjp")
        return g

    def chi_device(self, prob: Problem, switch: int, precision: int, re_ptr: int, im_ptr: int, epsm_ptr: int = 0):
        """pmx_chi_device on caller-owned device buffers (raw pointers, e.g. torch .data_ptr())."""
        st = self._lib.pmx_chi_device(self.handle, prob.handle, switch, precision, c_void_p(re_ptr),
                                      c_void_p(im_ptr), c_void_p(epsm_ptr) if epsm_ptr else None)
        self._check(st, "chi_device")

    def kgrid_reduce(self, problem, n, flags: int = KGRID_TIME_REVERSAL):
        """Irreducible points of the Gamma-centred grid n = (n1, n2, n3) of the
        problem's reciprocal basis: grid indices [nirr, 3] and orbit sizes [nirr]."""
        nn = np.ascontiguousarray(n, np.int32)
        cnt = c_int()
        self._check(self._lib.pmx_kgrid_reduce(self.handle, problem.handle, _iptr(nn), int(flags),
                                               ctypes.byref(cnt), None, None), "kgrid_reduce")
        idx = np.zeros((cnt.value, 3), np.int32)
        w = np.zeros(cnt.value, np.int32)
        self._check(self._lib.pmx_kgrid_reduce(self.handle, problem.handle, _iptr(nn), int(flags),
                                               ctypes.byref(cnt), _iptr(idx), _iptr(w)), "kgrid_reduce")
        return idx, w

    def eels(self, epsm, dfreq: float, wmin: float = 0.0):
        """Loss function -Im(1/eps_M) [nq, nf] and plasmon peaks [nq, 2] (eV,
        height) from eps_M [nq, nf] (complex)."""
        e = np.asarray(epsm, np.complex128)
        e = e.reshape(-1, e.shape[-1])
        nq, nf = e.shape
        buf = np.ascontiguousarray(np.stack([e.real, e.imag], -1))
        loss = np.zeros((nq, nf), np.float64)
        peak = np.zeros((nq, 2), np.float64)
        self._check(self._lib.pmx_eels(self.handle, nq, nf, float(dfreq), float(wmin), _dptr(buf), _dptr(loss),
                                       _dptr(peak)), "eels")
        return loss, peak

    def eps_macroscopic(self, neps: int, chi_re, chi_im):
        """eps_M [nq, nf] from the LL block [nq, npairs, nf] of a chi spectrum."""
        chi_re = np.ascontiguousarray(chi_re, np.float64)
        chi_im = np.ascontiguousarray(chi_im, np.float64)
        nq, _, nf = chi_re.shape
        out = np.zeros((nq, nf, 2), np.float64)
        self._check(self._lib.pmx_eps_macroscopic(self.handle, neps, nq, nf, _dptr(chi_re), _dptr(chi_im),
                                                  _dptr(out)), "eps_macroscopic")
        return out[..., 0] + 1j * out[..., 1]

    def kk(self, re, im, dfreq: float):
        re = np.ascontiguousarray(re, np.float64).copy()
        im = np.ascontiguousarray(im, np.float64).copy()
        rows, nf = re.shape
        self._check(self._lib.pmx_kk(self.handle, rows, nf, dfreq, _dptr(re), _dptr(im)), "kk")
        return re, im


def write_npz(path: str, arrays: dict) -> None:
    """pmx_write_npz: float64 arrays (C order) into an uncompressed .npz."""
    lib = load()
    items = [(k, np.require(np.asarray(v, np.float64), requirements="C")) for k, v in arrays.items()]
    n = len(items)
    names = (c_char_p * n)(*[k.encode() for k, _ in items])
    data = (POINTER(c_double) * n)(*[_dptr(a) for _, a in items])
    nd = np.array([a.ndim for _, a in items], np.int32)
    shp = np.array([d for _, a in items for d in a.shape] or [0], np.int64)
    st = lib.pmx_write_npz(path.encode(), n, names, data, _iptr(nd),
                           shp.ctypes.data_as(POINTER(c_longlong)))
    if st != PMX_OK:
        raise PicomaxError(st, "pmx_write_npz")


def run_main(args) -> int:
    """Runs the whole picomax program in-process (pmx_main)."""
    lib = load()
    argc, argv = _argv(args)
    return int(lib.pmx_main(argc, argv))
