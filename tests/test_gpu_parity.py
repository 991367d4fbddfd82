"""CUDA path (through the C-ABI) against the reference rebuilt from source
(golden fixtures) and against the numpy restatement.

Tolerances (FP64 path): band energies 1e-9 eV absolute; chi spectra 1e-8 of
the largest |value| of the spectrum set (the reference itself is not
bit-reproducible run to run, ~3e-16 relative); Kramers-Kronig 1e-10 relative.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden_args, load_golden

import picomax_b200 as pm
import pmx_oracle as O

pytestmark = pytest.mark.gpu

CHI_CASES = ["si_epsij", "gaas_soc_epsij", "si_epsLL", "gaas_soc_epsLL_pv", "wz_epsij_rect", "gaas_soc_epsxyz",
             "gaas_soc_epsxyz_pv"]


@pytest.mark.parametrize("name", ["si_band", "gaas_soc_band"])
def test_band_vs_reference(ctx, name, tmp_path):
    g = load_golden(name)
    p = pm.Problem(golden_args(g, tmp_path))
    eb = ctx.band(p)
    assert np.max(np.abs(eb.ravel() - g["dat"])) < 1e-9


def _switch(args):
    name = args[args.index("-switch") + 1]
    return {"epsij": pm.SWITCH_EPSIJ, "epsLL": pm.SWITCH_EPSLL, "epsxyz": pm.SWITCH_EPSXYZ}[name]


@pytest.mark.parametrize("name", CHI_CASES)
def test_chi_fp64_vs_reference(ctx, name, tmp_path):
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    sw = _switch(args)
    re, im = ctx.chi(p, sw, pm.PREC_FP64)
    n = re.size
    ref_re, ref_im = g["dat"][:n], g["dat"][n:]
    scale = max(np.abs(ref_re).max(), np.abs(ref_im).max())
    assert np.max(np.abs(re - ref_re)) <= 1e-8 * scale
    assert np.max(np.abs(im - ref_im)) <= 1e-8 * scale


def test_hamiltonian_vs_oracle(ctx):
    args = ("-crystal zb -a 5.65 -encut 40 -vg 3,4,8,11,0.1,-0.2,0.05,0.02,-0.1,0.1,0.03,-0.01 "
            "-use_uniform_us_so -uniform_us_so_val 0.01 -ua_so 3:0.004,8:0.002").split()
    p = pm.Problem(args)
    cr, mat, gcut, _ = O.from_args(args)
    G, _ = p.gvectors()
    ks = np.array([[0.1, 0.2, 0.3], [0.5, 0.5, 0.5]])
    H = ctx.hamiltonian(p, ks)
    for k, h in zip(ks, H):
        ref = O.hamiltonian(cr, mat, G, k)
        assert np.max(np.abs(h - ref)) < 1e-12 * np.max(np.abs(ref))


def _random_hermitian(rng, n, degenerate=False):
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = (A + A.conj().T) / 2
    if degenerate:  # exact pairs, as the doubled spinor spectrum without SOC
        h = n // 2
        B = A[:h, :h]
        U, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        A = U @ np.kron(B, np.eye(2)) @ U.conj().T
        A = (A + A.conj().T) / 2
    return A


@pytest.mark.parametrize("n,degenerate", [(40, False), (113, False), (120, True), (226, False), (300, True)])
def test_heev_vs_numpy(ctx, n, degenerate):
    rng = np.random.default_rng(n)
    A = np.stack([_random_hermitian(rng, n, degenerate) for _ in range(3)])
    nev = 16
    w, Z = ctx.heev(A, nev)
    for b in range(3):
        ref = np.linalg.eigvalsh(A[b])[:nev]
        scale = np.max(np.abs(np.linalg.eigvalsh(A[b])))
        assert np.max(np.abs(w[b] - ref)) < 1e-12 * scale * n
        R = A[b] @ Z[b] - Z[b] * w[b]
        assert np.max(np.linalg.norm(R, axis=0)) < 1e-10 * scale
        assert np.max(np.abs(Z[b].conj().T @ Z[b] - np.eye(nev))) < 1e-10


@pytest.mark.parametrize("n,nev", [(300, 300), (120, 120), (400, 260)])
def test_heev_all_eigenpairs(ctx, n, nev):
    """More eigenvalues than eigensolver threads (plain bisection) and full spectra."""
    rng = np.random.default_rng(n + nev)
    A = np.stack([_random_hermitian(rng, n) for _ in range(2)])
    w, Z = ctx.heev(A, nev)
    for b in range(2):
        ref = np.linalg.eigvalsh(A[b])[:nev]
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(w[b] - ref)) < 1e-12 * scale * n
        R = A[b] @ Z[b] - Z[b] * w[b]
        assert np.max(np.linalg.norm(R, axis=0)) < 1e-10 * scale
        assert np.max(np.abs(Z[b].conj().T @ Z[b] - np.eye(nev))) < 1e-10


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("n,nev,vectors", [(900, 16, True), (1200, 8, True), (1000, 24, False)])
def test_heev_large_n(n, nev, vectors, schedule):
    """n > 800: schedule 0 is the two-stage solver with stage 1's V and Y in
    global memory; schedule 1 the one-stage solver, whose per-warp partial
    sums live in global scratch above n = 832."""
    from conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(n)
    A = np.stack([_random_hermitian(rng, n) for _ in range(2)])
    c = pm.Context(0)
    c.set_schedule(schedule)
    w, Z = c.heev(A, nev, vectors=vectors)
    c.close()
    for b in range(2):
        full = np.linalg.eigvalsh(A[b])
        scale = np.max(np.abs(full))
        assert np.max(np.abs(w[b] - full[:nev])) < 1e-12 * scale * n
        if vectors:
            R = A[b] @ Z[b] - Z[b] * w[b]
            assert np.max(np.linalg.norm(R, axis=0)) < 1e-10 * scale
            assert np.max(np.abs(Z[b].conj().T @ Z[b] - np.eye(nev))) < 1e-10


def test_kk_vs_oracle(ctx):
    rng = np.random.default_rng(3)
    nf, rows, dw = 300, 7, 0.05
    re = rng.standard_normal((rows, nf))
    im = rng.standard_normal((rows, nf))
    r1, i1 = ctx.kk(re, im, dw)
    r0, i0 = O.kk_transform(re, im, dw * np.arange(nf), dw)
    assert np.max(np.abs(r1 - r0)) < 1e-10 * np.max(np.abs(r0))
    assert np.max(np.abs(i1 - i0)) < 1e-10 * np.max(np.abs(i0))


@pytest.mark.parametrize("name", ["si_band", "si_epsLL", "gaas_soc_epsij", "gaas_soc_epsxyz"])
def test_cli_files_vs_reference(name, tmp_path):
    """The picomax executable writes byte-compatible .dat/.gpt files."""
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    r = subprocess.run([pm.CLI_PATH] + args + ["-wdir", str(tmp_path), "-outputfile", "out"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    dat = np.fromfile(os.path.join(tmp_path, "out.dat"), np.float64)
    assert dat.size == g["dat"].size
    scale = np.abs(g["dat"]).max()
    tol = 1e-9 if name.endswith("band") else 1e-8 * scale
    assert np.max(np.abs(dat - g["dat"])) <= tol
    if "gpt" in g:
        assert np.array_equal(np.fromfile(os.path.join(tmp_path, "out.gpt"), np.float64), g["gpt"])


@pytest.mark.parametrize("name", CHI_CASES)
def test_chi_mixed_vs_reference(ctx, name, tmp_path):
    """Split-BF16 tensor-core contraction: within 1e-4 of the largest |value|."""
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    sw = _switch(args)
    re, im = ctx.chi(p, sw, pm.PREC_MIXED)
    n = re.size
    ref_re, ref_im = g["dat"][:n], g["dat"][n:]
    scale = max(np.abs(ref_re).max(), np.abs(ref_im).max())
    assert np.max(np.abs(re - ref_re)) <= 1e-4 * scale
    assert np.max(np.abs(im - ref_im)) <= 1e-4 * scale


def test_eps_macroscopic_vs_oracle(ctx, tmp_path):
    """eps_M = 1/[eps^-1]_00 of the LL block (restated macroscopic.m) on the
    reference's own chi_LL spectrum."""
    g = load_golden("si_epsLL")
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    neps, nf = p.info.neps, p.info.nfreq
    npairs = neps * (neps + 1) // 2
    n = g["dat"].size // 2
    re = g["dat"][:n].reshape(3, 3, 1, npairs, nf)[0, 0]
    im = g["dat"][n:].reshape(3, 3, 1, npairs, nf)[0, 0]
    eps = ctx.eps_macroscopic(neps, re, im)
    ref = O.eps_macroscopic(re[0], im[0], neps)
    assert np.max(np.abs(eps[0] - ref)) <= 1e-10 * np.max(np.abs(ref))
    # the fused path (chi + eps_M in one call) agrees with the two-step one
    cre, cim, eps2 = ctx.chi_epsm(p, pm.SWITCH_EPSLL, pm.PREC_FP64)
    e3 = ctx.eps_macroscopic(neps, cre.reshape(3, 3, 1, npairs, nf)[0, 0], cim.reshape(3, 3, 1, npairs, nf)[0, 0])
    assert np.max(np.abs(eps2 - e3)) <= 1e-12 * np.max(np.abs(e3))
    assert np.max(np.abs(eps2[0] - ref)) <= 1e-7 * np.max(np.abs(ref))


def test_degenerate_cut_reported(ctx, tmp_path):
    """NBAND cutting the Lambda_3 pair of Si (k on Gamma-L) is detected."""
    from picomax_b200.kgrid import write_kfile
    kf = os.path.join(str(tmp_path), "k.txt")
    write_kfile(kf, np.array([[0.25, 0.25, 0.25], [0.1, 0.2, 0.3]]), np.ones(2))
    args = ("-switch epsLL -crystal zb -a 5.43 -vg 3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08 -encut 60 "
            "-nband 16 -nvalence 8 -neps 2 -nfreq 20 -dfreq 0.5 -qvec 0.01,0,0 -kpoint 0").split() + [
        "-kpointfile", kf]
    p = pm.Problem(args)
    ctx.chi(p, pm.SWITCH_EPSLL)
    assert ctx.degenerate_cuts() >= 1


@pytest.mark.parametrize("n,nev,degenerate", [(420, 20, False), (570, 49, True), (600, 33, False), (800, 24, True)])
def test_heev_two_stage_beyond_shared_memory(ctx, n, nev, degenerate):
    """Padded sizes 432-800: the two-stage solver with stage 1's Y and stage 2's
    band in the reflector buffer's work area (global memory) instead of shared
    memory; Kramers-degenerate spectra included."""
    rng = np.random.default_rng(n + 7)
    A = np.stack([_random_hermitian(rng, n, degenerate) for _ in range(2)])
    w, Z = ctx.heev(A, nev)
    for b in range(2):
        full = np.linalg.eigvalsh(A[b])
        scale = np.max(np.abs(full))
        assert np.max(np.abs(w[b] - full[:nev])) < 1e-12 * scale * n
        R = A[b] @ Z[b] - Z[b] * w[b]
        assert np.max(np.linalg.norm(R, axis=0)) < 1e-10 * scale
        assert np.max(np.abs(Z[b].conj().T @ Z[b] - np.eye(nev))) < 1e-10


def _qvec(K):
    return ",".join(f"{x:.6f}" for x in np.asarray(K).ravel())


def test_heev_schedules_agree():
    """Every eigensolver schedule the autotuner can pick gives the same spectrum."""
    from conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    g = load_golden("gaas_soc_band")
    args = [str(a) for a in g["argv"]]
    # 200 band points so that the autotuner runs (>= 148 matrices in one batch)
    rng = np.random.default_rng(5)
    K = rng.uniform(-0.5, 0.5, (200, 3))
    base = args[args.index("-crystal"):]
    base = base[:base.index("-qpath")] + base[base.index("-qnum") + 2:]
    p = pm.Problem(["-switch", "band", "-qvec", _qvec(K)] + base)
    c1 = pm.Context(0)
    e1 = c1.band(p)  # autotuned (trial of every schedule on the first batch)
    assert c1.tuning()["heev"], "the autotuner did not run"
    c2 = pm.Context(0)
    c2.set_autotune(False)
    e2 = c2.band(p)  # default schedule
    assert e1.shape == (200, 16)
    assert np.max(np.abs(e1 - e2)) < 1e-10
    c1.close()
    c2.close()


@pytest.mark.parametrize("encut", [120, 160])
def test_heev_each_schedule(encut):
    """Each fixed eigensolver schedule (direct, prefetch rings, row partials in
    shared memory, grouped column-dot reductions) against the oracle's spectrum on the global-memory path
    (N_G 137 and 181 plane waves with spin-orbit: n = 274 and 362)."""
    from conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    from picomax_b200.workloads import gaas_form_factors
    vg, socargs = gaas_form_factors()
    rng = np.random.default_rng(17)
    K = rng.uniform(-0.5, 0.5, (6, 3))
    args = ["-switch", "band", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", str(encut), "-qvec", _qvec(K),
            "-nband", "24", "-nvalence", "8"] + socargs
    p = pm.Problem(args)
    cr, mat, gcut, o = O.from_args(args)
    G, _ = p.gvectors()
    ref = O.band(cr, mat, G, p.qpoints(), 24, 8)
    assert ref.shape == (6, 24)
    for sched in range(6):
        c = pm.Context(0)
        c.set_schedule(sched)
        e = c.band(p)
        assert np.max(np.abs(e - ref)) < 1e-9, sched
        c.close()
    p.close()
