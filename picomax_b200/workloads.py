"""The benchmark workloads as picomax argv, with seeded synthetic form factors.

Each workload is the restatement of one benchmark configuration as concrete
options; form factors that the configuration only describes ("drawn from a
seed within +-0.3 Ry") are drawn here from fixed numpy seeds, so every run and
every implementation sees identical inputs. k-point files are Gamma-centred
uniform grids written by picomax_b200.kgrid (same file for every
implementation compared).
"""
from __future__ import annotations

import math
import os

import numpy as np

from .kgrid import make_kfile

SI_VG = "3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08"


def _fmt(xs):
    return ",".join(f"{float(x):.6f}" for x in xs)


def gaas_form_factors(seed: int = 1965):
    """V_S, V_A ~ U(-0.3, 0.3) Ry on |G|^2 = 3, 4, 8, 11 (2 pi/a)^2; per-atom
    V = V_S +- V_A; SOC: lambda_S ~ U(0.002, 0.01) Ry (uniform over |G|^2),
    lambda_A ~ U(0, 0.005) Ry per shell."""
    r = np.random.default_rng(seed)
    vs = r.uniform(-0.3, 0.3, 4)
    va = r.uniform(-0.3, 0.3, 4)
    lam_s = r.uniform(0.002, 0.01)
    lam_a = r.uniform(0.0, 0.005, 4)
    vg = "3,4,8,11," + _fmt(vs + va) + "," + _fmt(vs - va)
    soc = ["-use_uniform_us_so", "-uniform_us_so_val", f"{lam_s:.6f}",
           "-ua_so", ",".join(f"{g}:{x:.6f}" for g, x in zip((3, 4, 8, 11), lam_a))]
    return vg, soc


def wz_form_factors(seed: int = 1967, f: float = 1.626):
    """Per-atom V ~ U(-0.3, 0.3) Ry on the first five |G|^2 shells of the
    wurtzite reciprocal lattice (cation pair = atoms 1, 2; anion pair = 3, 4)."""
    s3 = math.sqrt(3.0)
    b = np.array([[1, -1 / s3, 0], [1, 1 / s3, 0], [0, 0, 1.0 / f]])
    r3 = np.arange(-3, 4)
    hkl = np.array(np.meshgrid(r3, r3, r3, indexing="ij")).reshape(3, -1).T
    g2 = np.unique(np.round(((hkl @ b) ** 2).sum(1), 6))
    keys = g2[1:6]
    r = np.random.default_rng(seed)
    vc = r.uniform(-0.3, 0.3, 5)
    van = r.uniform(-0.3, 0.3, 5)
    vg = _fmt(keys) + "," + ",".join([_fmt(vc), _fmt(vc), _fmt(van), _fmt(van)])
    return vg


def te_shells(f: float = 1.33):
    """The first 8 |G|^2 shells ((2 pi/a)^2) of the trigonal Te lattice."""
    s3 = math.sqrt(3.0)
    b = np.array([[1, -1 / s3, 0], [1, 1 / s3, 0], [0, 0, 1.0 / f]])
    r3 = np.arange(-3, 4)
    hkl = np.array(np.meshgrid(r3, r3, r3, indexing="ij")).reshape(3, -1).T
    g2 = np.unique(np.round(((hkl @ b) ** 2).sum(1), 6))
    return g2[1:9]


def te_params(seed: int = 1969):
    """The 10 free parameters of trigonal Te (Ry): 8 form factors (the same
    for the 3 atoms) ~ U(-0.3, 0.3), lambda_S ~ U(0.002, 0.01) (uniform over
    |G|^2) and lambda_A ~ U(0, 0.005) (on the first 4 shells). The default
    seed gives an insulator on the 10x10x8 grid (no state within 0.9 eV of
    the reference energy), so occupations do not change under small steps."""
    r = np.random.default_rng(seed)
    v = r.uniform(-0.3, 0.3, 8)
    return np.concatenate([v, [r.uniform(0.002, 0.01), r.uniform(0.0, 0.005)]])


def te_form_factors(seed: int = 1969, f: float = 1.33, theta=None):
    """-vg and SOC options of trigonal Te for the free parameters theta
    (te_params(seed) by default)."""
    keys = te_shells(f)
    th = te_params(seed) if theta is None else np.asarray(theta, float)
    vg = _fmt(keys) + "," + ",".join([_fmt(th[:8])] * 3)
    soc = ["-use_uniform_us_so", "-uniform_us_so_val", f"{th[8]:.6f}",
           "-ua_so", ",".join(f"{k:.6f}:{th[9]:.6f}" for k in keys[:4])]
    return vg, soc


def te_param_map(natom: int = 3, nshell: int = 8, nua: int = 4) -> np.ndarray:
    """J with full = J @ theta: theta (8 form factors, lambda_S, lambda_A) to
    the problem's parameter vector (vg[atom][shell], lambda_S, lambda_A per key)."""
    J = np.zeros((natom * nshell + 1 + nua, nshell + 2))
    for a in range(natom):
        for s in range(nshell):
            J[a * nshell + s, s] = 1.0
    J[natom * nshell, nshell] = 1.0
    J[natom * nshell + 1:, nshell + 1] = 1.0
    return J


def workload(name: str, workdir: str):
    """Returns (argv, nspectra, nsolves) of a named workload; k-files go to workdir.

    si_band / si_epsLL: config 1 (Si, 121-point path; 8^3 grid, NEPS 15, 1000 w)
    gaas_epsij[_N]:     config 2 (GaAs + SOC, N^3 grid (16), NEPS 27, 2000 w, Lorentzian)
    wz_epsLL[_N]:       config 3 (wurtzite, N_G 401, 24x24x16 grid (N x N x 3N/4), NEPS 59, 2000 w)
    te_band / te_epsLL: config 5 (trigonal Te + SOC, 2 N_G = 570; 121-point path; 10x10x8 grid)"""
    os.makedirs(workdir, exist_ok=True)
    if name == "si_band":
        argv = ["-switch", "band", "-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "110",
                "-nband", "16", "-nvalence", "8", "-qpath", "G,X,W,L,G", "-qnum", "30,30,30,30"]
        return argv, 0, 122
    if name == "si_epsLL":
        kf = os.path.join(workdir, "k_zb_8.txt")
        nk = make_kfile(kf, "zb", 8, 8, 8)
        argv = ["-switch", "epsLL", "-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "110",
                "-kpoint", "0", "-kpointfile", kf, "-qvec", "0.01,0,0", "-neps", "15", "-nband", "16",
                "-nvalence", "8", "-nfreq", "1000", "-dfreq", "0.02", "-delta", "0", "-epsilon", "0.1", "-kk", "1"]
        return argv, 1, 1 + 2 * nk
    if name.startswith("gaas_epsij"):
        n = int(name.split("_")[-1]) if name.count("_") == 2 else 16
        kf = os.path.join(workdir, f"k_zb_{n}.txt")
        nk = make_kfile(kf, "zb", n, n, n)
        vg, soc = gaas_form_factors()
        argv = ["-switch", "epsij", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", "120",
                "-kpoint", "0", "-kpointfile", kf, "-qvec", "0.01,0,0", "-neps", "27", "-nband", "16",
                "-nvalence", "8", "-nfreq", "2000", "-dfreq", "0.0125", "-delta", "1", "-epsilon", "0.05",
                "-kk", "1"] + soc
        return argv, 1, 1 + 2 * nk
    if name == "wz_epsLL" or name.startswith("wz_epsLL_"):
        # wz_epsLL_N: the same on an N x N x (3N/4) grid (profiling-size cases)
        n = int(name.split("_")[-1]) if name.count("_") == 2 else 24
        nz = max(1, 3 * n // 4) if n != 24 else 16
        kf = os.path.join(workdir, f"k_wz_{n}_{nz}.txt")
        nk = make_kfile(kf, "wz", n, n, nz, f=1.626)
        argv = ["-switch", "epsLL", "-crystal", "wz", "-a", "3.19", "-f", "1.626", "-u", "0.375",
                "-vg", wz_form_factors(), "-encut", "260", "-kpoint", "0", "-kpointfile", kf,
                "-qvec", "0.01,0,0", "-neps", "59", "-nband", "48", "-nvalence", "16", "-nfreq", "2000",
                "-dfreq", "0.015", "-delta", "0", "-epsilon", "0.1", "-kk", "1"]
        return argv, 1, 1 + 2 * nk
    if name == "te_band":
        vg, soc = te_form_factors()
        argv = ["-switch", "band", "-crystal", "te", "-a", "4.45", "-f", "1.33", "-u", "0.264", "-vg", vg,
                "-encut", "120", "-nband", "24", "-nvalence", "18", "-qpath", "G,A,H,K,G",
                "-qnum", "30,30,30,30"] + soc
        return argv, 0, 122
    if name == "te_epsLL":
        vg, soc = te_form_factors()
        kf = os.path.join(workdir, "k_te_10_8.txt")
        nk = make_kfile(kf, "te", 10, 10, 8, f=1.33)
        argv = ["-switch", "epsLL", "-crystal", "te", "-a", "4.45", "-f", "1.33", "-u", "0.264", "-vg", vg,
                "-encut", "120", "-kpoint", "0", "-kpointfile", kf, "-qvec", "0.01,0,0", "-neps", "15",
                "-nband", "24", "-nvalence", "18", "-nfreq", "1000", "-dfreq", "0.01", "-delta", "0",
                "-epsilon", "0.05", "-kk", "1"] + soc
        return argv, 1, 1 + 2 * nk
    raise KeyError(name)


def main(argv=None):
    """python -m picomax_b200.workloads NAME [extra picomax options]

    Runs the picomax CLI on a named workload (k-point files are written to a
    temporary directory, outputs too) and prints the CLI's progress output."""
    import subprocess
    import sys
    import tempfile

    from ._capi import CLI_PATH
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print(main.__doc__)
        return 2
    with tempfile.TemporaryDirectory() as tmp:
        args, _, _ = workload(argv[0], tmp)
        r = subprocess.run([CLI_PATH] + args + argv[1:] + ["-wdir", tmp, "-outputfile", argv[0]])
        return r.returncode


if __name__ == "__main__":
    raise SystemExit(main())
