import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def ctx():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import picomax_b200 as pm
    c = pm.Context(0)
    yield c
    c.close()


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    return {k: d[k] for k in d.files}


def golden_args(g, tmpdir):
    """argv of a golden case with its k-point file rewritten under tmpdir."""
    from picomax_b200.kgrid import write_kfile
    args = [str(a) for a in g["argv"]]
    if "kpts" in g:
        kf = os.path.join(str(tmpdir), "kpts.txt")
        write_kfile(kf, g["kpts"], np.ones(len(g["kpts"])))
        args += ["-kpoint", "0", "-kpointfile", kf]
    return args


def arg_value(args, flag, default=None):
    return args[args.index(flag) + 1] if flag in args else default
