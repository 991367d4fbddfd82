"""Gamma-centred uniform k-point files in the reference's kpointfile format.

Format read by import_kpt (src/pmx_basis.cpp:200-245): line 1 = number of
points of the full grid (the weight normaliser), line 2 = number of listed
points, then ``kx ky kz w`` per point in units of 2 pi / a (Cartesian).

The grids are Gamma-centred N1 x N2 x N3 Monkhorst-Pack meshes of the
reciprocal basis of the preset (src/pmx_io.cpp:126-209); every index is folded
into (-N/2, N/2] and the point is then moved into the first Brillouin zone
with the zone tests and the 27 lattice shifts of generate_kpt_fcc/_hex
(src/pmx_basis.cpp:655-690, :384-396). Results of the reference depend on
which zone image a boundary point takes, so the same file must be given to
every implementation that is compared.
"""
from __future__ import annotations

import math

import numpy as np


def reciprocal(crystal: str, f: float = math.sqrt(8.0 / 3.0)) -> np.ndarray:
    s3 = math.sqrt(3.0)
    if crystal in ("zb", "rs"):
        return np.array([[-1, 1, 1], [1, -1, 1], [1, 1, -1]], np.float64)
    if crystal in ("wz", "te"):
        return np.array([[1, -1 / s3, 0], [1, 1 / s3, 0], [0, 0, 1.0 / f]], np.float64)
    raise ValueError(f"no 3D reciprocal basis for crystal {crystal!r}")


def _in_bz(crystal: str, k, f: float) -> bool:
    tol = 1e-6
    x, y, z = abs(k[0]), abs(k[1]), abs(k[2])
    if crystal in ("zb", "rs"):
        return not (x > 1 + tol or y > 1 + tol or z > 1 + tol or x + y + z > 1.5 + tol)
    s3 = math.sqrt(3.0)
    return not (z > 0.5 / f + tol or y > 1 / s3 + tol or x + y / s3 > 1 / s3 + tol)


def _fold_point(crystal: str, b: np.ndarray, i, n, f: float) -> np.ndarray:
    """Cartesian k of grid index i (indices folded into (-N/2, N/2], then the
    point moved into the first zone with the 27 lattice shifts)."""
    j = [ii if ii <= nn // 2 else ii - nn for ii, nn in zip(i, n)]
    k = (j[0] / n[0]) * b[0] + (j[1] / n[1]) * b[1] + (j[2] / n[2]) * b[2]
    if not _in_bz(crystal, k, f):
        for s1 in (-1, 0, 1):
            for s2 in (-1, 0, 1):
                for s3_ in (-1, 0, 1):
                    kk = k + s1 * b[0] + s2 * b[1] + s3_ * b[2]
                    if _in_bz(crystal, kk, f):
                        return kk
    return k


def gamma_grid(crystal: str, n1: int, n2: int, n3: int, f: float = math.sqrt(8.0 / 3.0)):
    """Returns (K [N,3], W [N]) of the folded Gamma-centred grid, first index fastest."""
    b = reciprocal(crystal, f)
    pts = [_fold_point(crystal, b, (i1, i2, i3), (n1, n2, n3), f)
           for i3 in range(n3) for i2 in range(n2) for i1 in range(n1)]
    K = np.array(pts, np.float64)
    return K, np.ones(len(K), np.float64)


def ibz_grid(ctx, problem, crystal: str, n1: int, n2: int, n3: int, f: float = math.sqrt(8.0 / 3.0),
             flags: int = 1):
    """Irreducible wedge of the Gamma-centred grid under the problem's point
    group (with time reversal by default; flags as pmx_kgrid_reduce), reduced
    on the device: (K [nirr, 3] folded like gamma_grid, W [nirr] orbit sizes,
    N = n1 n2 n3 for the kpointfile's first line)."""
    idx, w = ctx.kgrid_reduce(problem, (n1, n2, n3), flags)
    b = reciprocal(crystal, f)
    K = np.array([_fold_point(crystal, b, tuple(int(x) for x in i), (n1, n2, n3), f) for i in idx], np.float64)
    return K.reshape(-1, 3), w.astype(np.float64), n1 * n2 * n3


def write_kfile(path: str, K, W, ntotal: int | None = None) -> None:
    K = np.asarray(K, np.float64)
    W = np.asarray(W, np.float64)
    with open(path, "w") as fh:
        fh.write(f"{len(K) if ntotal is None else ntotal}\n{len(K)}\n")
        for k, w in zip(K, W):
            fh.write(f"{float(k[0])!r} {float(k[1])!r} {float(k[2])!r} {float(w)!r}\n")


def make_kfile(path: str, crystal: str, n1: int, n2: int, n3: int, f: float = math.sqrt(8.0 / 3.0)) -> int:
    K, W = gamma_grid(crystal, n1, n2, n3, f)
    write_kfile(path, K, W)
    return len(K)
