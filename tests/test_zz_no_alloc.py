"""pmx_heev_batched_noalloc (caller-owned device buffers, fixed scratch array)
against pmx_heev_batched on the same matrices, two calls in a row.

Named to be collected last, so that it also runs after every other GPU test
has used the library on the same device."""
import ctypes

import numpy as np
import pytest

from test_gpu_parity import _random_hermitian

pytestmark = pytest.mark.gpu


def _noalloc(lib, A, nev, vectors=True):
    import torch
    b, n, _ = A.shape
    colmajor = np.ascontiguousarray(A.transpose(0, 2, 1))
    dA = torch.from_numpy(np.ascontiguousarray(np.stack([colmajor.real, colmajor.imag], -1))).cuda()
    dw = torch.zeros((b, nev), dtype=torch.float64, device="cuda")
    dz = torch.zeros((b, nev, n, 2), dtype=torch.float64, device="cuda") if vectors else None
    dinfo = torch.full((b,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.pmx_heev_batched_noalloc(ctypes.c_void_p(stream), n, b, ctypes.c_void_p(dA.data_ptr()), nev,
                                      ctypes.c_void_p(dw.data_ptr()),
                                      ctypes.c_void_p(dz.data_ptr()) if vectors else None,
                                      ctypes.c_void_p(dinfo.data_ptr()))
    torch.cuda.synchronize()
    assert st == 0
    assert (dinfo.cpu().numpy() == 0).all()
    w = dw.cpu().numpy()
    if not vectors:
        return w, None
    z = dz.cpu().numpy()
    return w, (z[..., 0] + 1j * z[..., 1]).transpose(0, 2, 1)


def _check(ctx, A, nev):
    from picomax_b200 import _capi
    w0, Z0 = ctx.heev(A, nev)
    w1, Z1 = _noalloc(_capi.load(), A, nev)
    n = A.shape[1]
    for b in range(A.shape[0]):
        scale = np.max(np.abs(np.linalg.eigvalsh(A[b])))
        assert np.max(np.abs(w1[b] - w0[b])) < 1e-12 * scale * n
        # same subspace and residual as the context path (vectors agree up to
        # the basis inside degenerate sets)
        R = A[b] @ Z1[b] - Z1[b] * w1[b]
        assert np.max(np.linalg.norm(R, axis=0)) < 1e-10 * scale
        assert np.max(np.abs(Z1[b].conj().T @ Z1[b] - np.eye(nev))) < 1e-10
        P0 = Z0[b] @ Z0[b].conj().T
        P1 = Z1[b] @ Z1[b].conj().T
        assert np.max(np.abs(P1 - P0)) < 1e-10


def test_noalloc_matches_context_path_two_calls(ctx):
    rng = np.random.default_rng(2024)
    # first call: global-memory eigensolver path (n above the shared-memory resident size)
    A1 = np.stack([_random_hermitian(rng, 226) for _ in range(6)])
    _check(ctx, A1, 16)
    # second call: smaller, degenerate, shared-memory resident path; the
    # scratch array still holds the first call's contents
    A2 = np.stack([_random_hermitian(rng, 120, degenerate=True) for _ in range(4)])
    _check(ctx, A2, 16)


def test_noalloc_rejects_sizes_beyond_limit(ctx):
    from picomax_b200 import _capi
    lib = _capi.load()
    d = ctypes.c_void_p(16)  # never dereferenced: the size checks come first
    assert lib.pmx_heev_batched_noalloc(None, 833, 1, d, 8, d, d, d) == _capi.PMX_ERR_LIMIT
    assert lib.pmx_heev_batched_noalloc(None, 64, 1025, d, 8, d, None, d) == _capi.PMX_ERR_LIMIT
    # 4 n nev batch doubles of inverse-iteration vectors above the scratch
    assert lib.pmx_heev_batched_noalloc(None, 832, 1000, d, 512, d, d, d) == _capi.PMX_ERR_LIMIT
    assert lib.pmx_heev_batched_noalloc(None, 64, 2, d, 65, d, d, d) == _capi.PMX_ERR_INVALID


def test_noalloc_values_only_and_largest_sizes(ctx):
    """Eigenvalues only (no vectors: the scratch array is not touched), then the
    largest matrices the entry point takes (n 800, partial sums next to the
    scratch limit in shared memory), two calls in a row."""
    from picomax_b200 import _capi
    rng = np.random.default_rng(7)
    A = np.stack([_random_hermitian(rng, 226) for _ in range(3)])
    w0, _ = ctx.heev(A, 12, vectors=False)
    w1, _ = _noalloc(_capi.load(), A, 12, vectors=False)
    scale = max(np.max(np.abs(np.linalg.eigvalsh(a))) for a in A)
    assert np.max(np.abs(w1 - w0)) < 1e-12 * scale * 226
    B = np.stack([_random_hermitian(rng, 800) for _ in range(2)])
    _check(ctx, B, 16)
