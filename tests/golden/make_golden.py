"""Generates the golden fixtures in tests/golden/ by running the reference
PicoMax rebuilt from source (oracle/_ref, see oracle/Makefile).

Usage:  python tests/golden/make_golden.py        (needs oracle/_ref built)

Each fixture <name>.npz holds the argv (without -wdir/-outputfile/-kpointfile),
the k-point list written to the kpointfile, the reference's .dat (and .gpt for
the chi switches) and the wall time. The cases are small so that the
reference finishes in seconds; they cover band / epsij / epsLL, with and
without spin-orbit coupling, the four broadening models, KK on and off, and
zinc-blende, rock-salt, wurtzite and trigonal presets.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from picomax_b200.kgrid import gamma_grid, write_kfile  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
SI_VG = "3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08"
# GaAs-like: V_S +- V_A at |G|^2 = 3, 4, 8, 11 (Ry), drawn once from a seed.
_r = np.random.default_rng(20240606)
_vs = _r.uniform(-0.3, 0.3, 4)
_va = _r.uniform(-0.3, 0.3, 4)
GAAS_VG = ",".join(["3", "4", "8", "11"] + [f"{x:.6f}" for x in _vs + _va] + [f"{x:.6f}" for x in _vs - _va])
WZ_VG = ("0.378233,1.333333,1.512930,1.711566," + ",".join(["-0.119900,0.224132,-0.296841,0.192737"] * 4))
GAAS_SOC = ["-use_uniform_us_so", "-uniform_us_so_val", "0.004", "-ua_so", "3:0.002,4:0.0015,8:0.001,11:0.0005"]

# generic k-points for epsxyz: away from the time-reversal-invariant momenta,
# where every level is a Kramers pair and chi_xyz (which mixes the first N_G
# spinor components) depends on the eigensolver's basis inside the pair
K_GENERIC = [[0.11, 0.23, 0.05], [0.31, -0.17, 0.09], [-0.07, 0.19, -0.26], [0.41, 0.08, 0.21]]

CASES = {
    # name: (binary, argv, kgrid or None)
    "si_band": ("picomax_ref", ["-switch", "band", "-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "110",
                                "-nband", "16", "-nvalence", "8", "-qpath", "G,X,W,L,G", "-qnum", "30,30,30,30"], None),
    "gaas_soc_band": ("picomax_ref", ["-switch", "band", "-crystal", "zb", "-a", "5.65", "-vg", GAAS_VG, "-encut",
                                      "120", "-nband", "16", "-nvalence", "8", "-qpath", "L,G,X", "-qnum", "6,6"]
                      + GAAS_SOC, None),
    "si_epsij": ("picomax_ref_guard", ["-switch", "epsij", "-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut",
                                       "80", "-nband", "16", "-nvalence", "8", "-neps", "4", "-nfreq", "120",
                                       "-dfreq", "0.1", "-delta", "0", "-epsilon", "0.1", "-kk", "1",
                                       "-qvec", "0.01,0,0"], ("zb", 3, 3, 3)),
    "gaas_soc_epsij": ("picomax_ref_guard", ["-switch", "epsij", "-crystal", "zb", "-a", "5.65", "-vg", GAAS_VG,
                                             "-encut", "80", "-nband", "16", "-nvalence", "8", "-neps", "4",
                                             "-nfreq", "120", "-dfreq", "0.125", "-delta", "1", "-epsilon", "0.05",
                                             "-kk", "1", "-qvec", "0.01,0,0"] + GAAS_SOC, ("zb", 2, 2, 2)),
    "si_epsLL": ("picomax_ref_ll", ["-switch", "epsLL", "-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "80",
                                    "-nband", "16", "-nvalence", "8", "-neps", "4", "-nfreq", "120", "-dfreq",
                                    "0.1", "-delta", "0", "-epsilon", "0.1", "-kk", "1", "-qvec", "0.01,0,0"],
                 ("zb", 3, 3, 3)),
    "gaas_soc_epsLL_pv": ("picomax_ref_ll", ["-switch", "epsLL", "-crystal", "zb", "-a", "5.65", "-vg", GAAS_VG,
                                             "-encut", "80", "-nband", "16", "-nvalence", "8", "-neps", "4",
                                             "-nfreq", "120", "-dfreq", "0.125", "-delta", "2", "-epsilon", "0.3",
                                             "-kk", "0", "-qvec", "0.02,0.01,0"] + GAAS_SOC, ("zb", 2, 2, 2)),
    "gaas_soc_epsxyz": ("picomax_ref_ll", ["-switch", "epsxyz", "-crystal", "zb", "-a", "5.65", "-vg", GAAS_VG,
                                           "-encut", "80", "-nband", "16", "-nvalence", "8", "-neps", "4",
                                           "-nfreq", "120", "-dfreq", "0.125", "-delta", "0", "-epsilon", "0.1",
                                           "-kk", "1", "-qvec", "0.01,0,0"] + GAAS_SOC, ("list", K_GENERIC)),
    "gaas_soc_epsxyz_pv": ("picomax_ref_ll", ["-switch", "epsxyz", "-crystal", "zb", "-a", "5.65", "-vg", GAAS_VG,
                                              "-encut", "80", "-nband", "16", "-nvalence", "8", "-neps", "3",
                                              "-nfreq", "100", "-dfreq", "0.125", "-delta", "1", "-epsilon", "0.05",
                                              "-kk", "0", "-qvec", "0.02,0.01,0"] + GAAS_SOC, ("list", K_GENERIC)),
    "wz_epsij_rect": ("picomax_ref_guard", ["-switch", "epsij", "-crystal", "wz", "-a", "3.19", "-f", "1.626", "-u",
                                            "0.375", "-vg", WZ_VG, "-encut", "50", "-nband", "24", "-nvalence", "8",
                                            "-neps", "3", "-nfreq", "100", "-dfreq", "0.15", "-delta", "3",
                                            "-epsilon", "0.4", "-kk", "0", "-qvec", "0.03,0,0"],
                      ("wz", 2, 2, 2)),
}


def _strip_kfile(argv):
    """argv without -kpoint / -kpointfile (the fixture carries its k list)."""
    out, i = [], 0
    while i < len(argv):
        if argv[i] in ("-kpoint", "-kpointfile"):
            i += 2
            continue
        out.append(argv[i])
        i += 1
    return out


def _subset(K, count, skip=None):
    """`count` points of the grid K taken at an even stride (deterministic),
    leaving out the points `skip` rejects."""
    idx = [i for i in range(len(K)) if skip is None or not skip(K[i])]
    step = max(1, len(idx) // count)
    return K[np.array(idx[::step][:count])]


def _on_gamma_l(k):
    """k on the Gamma-L line (|kx| = |ky| = |kz| != 0): NBAND 16 of Si cuts the
    Lambda_3 pair there, and chi then depends on the eigensolver's basis."""
    a = np.abs(k)
    return a[0] > 1e-9 and abs(a[0] - a[1]) < 1e-9 and abs(a[0] - a[2]) < 1e-9


def _is_gamma(k):
    """Gamma: with the wurtzite seed the states nvalence-1 and nvalence are
    degenerate there, so E_ref sits on both and their occupation is decided by
    rounding (no implementation can reproduce another's)."""
    return bool(np.all(np.abs(k) < 1e-12))


def config_cases():
    """The benchmark configurations at their own shape (encut / N_G, NEPS,
    frequencies, broadening, SOC, preset, form-factor seeds) on a subset of
    each configuration's own Gamma-centred k grid, sized so that the
    reference finishes in seconds to a few minutes."""
    from picomax_b200.workloads import workload
    with tempfile.TemporaryDirectory() as tmp:
        si, _, _ = workload("si_epsLL", tmp)
        ga, _, _ = workload("gaas_epsij", tmp)
        wz, _, _ = workload("wz_epsLL", tmp)
        teb, _, _ = workload("te_band", tmp)
        tel, _, _ = workload("te_epsLL", tmp)
    Ksi, _ = gamma_grid("zb", 8, 8, 8)
    Kga, _ = gamma_grid("zb", 16, 16, 16)
    Kwz, _ = gamma_grid("wz", 24, 24, 16, 1.626)
    Kte, _ = gamma_grid("te", 10, 10, 8, 1.33)
    return {
        # config 1: Si epsLL, N_G 113, NEPS 15, 1000 w, Gaussian 0.1 eV, KK
        "cfg1_si_epsLL": ("picomax_ref_ll", _strip_kfile(si), ("list", _subset(Ksi, 32, _on_gamma_l))),
        # config 2: GaAs + SOC epsij, n 274, NEPS 27, 2000 w, Lorentzian 0.05 eV, KK;
        # 128 k-points give > 2048 transitions per 256-wide frequency tile, so
        # the mixed path's periodic FP64 flush of the TMEM accumulator runs
        "cfg2_gaas_epsij": ("picomax_ref_guard", _strip_kfile(ga), ("list", _subset(Kga, 128))),
        # config 3: wurtzite epsLL, N_G 401, NEPS 59, 2000 w, Gaussian 0.1 eV, KK
        "cfg3_wz_epsLL": ("picomax_ref_ll", _strip_kfile(wz), ("list", _subset(Kwz, 4, _is_gamma))),
        # config 5: trigonal Te + SOC (n 570): 121-point band path and epsLL
        "cfg5_te_band": ("picomax_ref", teb, None),
        "cfg5_te_epsLL": ("picomax_ref_ll", _strip_kfile(tel), ("list", _subset(Kte, 16))),
    }


def _reduce_chi(dat, argv, nk_rows=None):
    """Fixture form of a large chi .dat ([re|im][3][3][nq][pairs][nf]): every
    row (re/im, i, j, q, pair) at a stride of frequencies, the rows of the
    first three pairs ((0,0), (1,0), (1,1): the head and its neighbours) at
    every frequency, every row's sum over frequencies, and max |value|."""
    neps = int(argv[argv.index("-neps") + 1])
    nf = int(argv[argv.index("-nfreq") + 1])
    npairs = neps * (neps + 1) // 2
    rows = dat.reshape(-1, npairs, nf)
    fstride = max(1, (rows.shape[0] * npairs * nf) // 150000)
    fsel = np.arange(0, nf, fstride)
    return {"dat_absmax": np.abs(dat).max(), "dat_size": np.int64(dat.size), "fsel": fsel,
            "dat_fsel": rows[:, :, fsel], "dat_head": rows[:, :3, :], "dat_rowsum": rows.sum(axis=2)}


def run_case(name, binary, argv, grid, tmp, reduce=False):
    args = list(argv)
    K = None
    if grid is not None and grid[0] == "list":
        K = np.asarray(grid[1], float)
        W = np.ones(len(K))
        kf = os.path.join(tmp, f"{name}_k.txt")
        write_kfile(kf, K, W)
        args += ["-kpoint", "0", "-kpointfile", kf]
    elif grid is not None:
        crystal, n1, n2, n3 = grid
        K, W = gamma_grid(crystal, n1, n2, n3)
        kf = os.path.join(tmp, f"{name}_k.txt")
        write_kfile(kf, K, W)
        args += ["-kpoint", "0", "-kpointfile", kf]
    cmd = [os.path.join(REF, binary)] + args + ["-wdir", tmp, "-outputfile", name]
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    dt = time.time() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}")
    dat = np.fromfile(os.path.join(tmp, name + ".dat"), np.float64)
    out = {"argv": np.array(argv), "binary": binary, "seconds": dt}
    if reduce and "-neps" in argv:
        out.update(_reduce_chi(dat, argv))
    else:
        out["dat"] = dat
    gpt = os.path.join(tmp, name + ".gpt")
    if os.path.exists(gpt) and not reduce:
        out["gpt"] = np.fromfile(gpt, np.float64)
    if K is not None:
        out["kpts"] = K
        if grid[0] != "list":
            out["kgrid"] = np.array(grid[1:], np.int64)
            out["kcrystal"] = grid[0]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: {dat.size} values, {dt:.2f} s")


# -debug 3 dumps: the reference prints its G list, k list and q list
# (src/pmx_io.cpp:572-603) and exits; the text after "planewave energy
# cutoff" is compared line by line with pmx_problem_dump.
DUMPS = {
    "zb_path": ["-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "110", "-qpath", "G,X,W,L,G",
                "-qnum", "30,30,30,30"],
    "zb_fcc_bz": ["-crystal", "zb", "-a", "5.65", "-vg", SI_VG, "-encut", "150", "-kpoint", "1", "-kpointorder", "4",
                  "-qvec", "0.01,0,0,0.1,0.2,0.3"],
    "zb_box": ["-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "120", "-gsym", "0"],
    "zb_cohen_chadi": ["-crystal", "zb", "-a", "5.43", "-vg", SI_VG, "-encut", "90", "-kpoint", "3",
                       "-kpointorder", "4"],
    "rs_bz": ["-crystal", "rs", "-a", "5.0", "-vg", SI_VG, "-encut", "160", "-kpoint", "1", "-kpointorder", "3"],
    "wz_bz": ["-crystal", "wz", "-a", "3.19", "-f", "1.626", "-u", "0.375", "-vg", "1,2,3,4,5,6,7,8,9,10",
              "-encut", "200", "-qpath", "G,A,H,K,G", "-qnum", "5,5,5,5", "-kpoint", "1", "-kpointorder", "4"],
    "te_bz": ["-crystal", "te", "-a", "4.45", "-f", "1.33", "-u", "0.264", "-vg", "1,2,0.1,0.2,0.3,0.4,0.5,0.6",
              "-encut", "150", "-qpath", "G,A,H,K,G", "-qnum", "3,3,3,3", "-kpoint", "1", "-kpointorder", "3"],
    "hex2d_bz": ["-crystal", "hex", "-a", "2.46", "-vg", "1,0.1,0.2", "-encut", "100", "-kpoint", "1",
                 "-kpointorder", "6", "-qpath", "G,M,K,G", "-qnum", "4,4,4"],
}


def run_dump(name, argv):
    cmd = [os.path.join(REF, "picomax_ref")] + argv + ["-debug", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}")
    text = r.stdout[r.stdout.index("planewave energy cutoff"):]
    with open(os.path.join(HERE, "dumps", name + ".txt"), "w") as fh:
        fh.write(" ".join(argv) + "\n" + text)
    print(f"dump {name}: {text.count(chr(10))} lines")


def main(names=None):
    os.makedirs(os.path.join(HERE, "dumps"), exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name, (binary, argv, grid) in CASES.items():
            if names and name not in names:
                continue
            run_case(name, binary, argv, grid, tmp)
        # configuration-shape cases only when named (minutes of host time)
        for name, (binary, argv, grid) in config_cases().items():
            if names and name in names:
                run_case(name, binary, argv, grid, tmp, reduce=True)
    for name, argv in DUMPS.items():
        if names and name not in names:
            continue
        run_dump(name, argv)


if __name__ == "__main__":
    main(sys.argv[1:])
