"""Point-group operations of the Hamiltonian (pmx_problem_symmetry, host) and
the grid reduction they drive, on the CPU.

* group orders of the presets (zincblende with two species: T_d, 24, and 48
  with time reversal; one species: O_h through the non-symmorphic inversion;
  rocksalt O_h; wurtzite C_6v 12 / 24; Te D_3 6 / 12), the identity first,
  closure under products;
* the same sets as the oracle's independent search by atom mapping
  (oracle/pmx_oracle.py point_group_ops) for Hamiltonians without spin-orbit
  coupling;
* every operation keeps the spectrum: eigenvalues of the numpy Hamiltonian
  (oracle/pmx_oracle.py hamiltonian, pinned to the reference) at k and at R k
  agree to 1e-9 of the spectrum's scale, with and without spin-orbit
  coupling (the reference's spin-orbit model drops the screw operations of
  Te, and the search drops them with it);
* the oracle's grid reduction: orbits partition the grid, 29 points for the
  8^3 fcc grid under O_h.
"""
import numpy as np
import pytest

import pmx_oracle as O
import picomax_b200 as pm

GAAS = "-crystal zb -a 5.65 -vg 3,4,8,11,-0.21,0.01,0.04,0.08,-0.23,0,0.05,0.08 -encut 50"
SI = "-crystal zb -a 5.43 -vg 3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08 -encut 50"
RS = "-crystal rs -a 5.6 -vg 3,4,8,11,-0.21,0.01,0.04,0.08,-0.23,0,0.05,0.08 -encut 50"
SOC = " -use_uniform_us_so -uniform_us_so_val 0.002 -ua_so 3:0.001,4:0.001"


def _hex(name):
    """wz / te argv with form-factor keys on the first three real shells."""
    base = ("-crystal wz -a 3.19 -f 1.626 -u 0.375 -encut 30" if name == "wz"
            else "-crystal te -a 4.45 -f 1.33 -u 0.264 -encut 22")
    nat = 4 if name == "wz" else 3
    p0 = pm.Problem((base + " -vg 1," + ",".join(["0"] * nat)).split())
    G, _ = p0.gvectors()
    p0.close()
    g2 = np.unique(np.round((G ** 2).sum(1), 6))[1:4]
    vg = list(g2) + ([-0.2, 0.1, 0.05] * 2 + [-0.3, 0.12, 0.04] * 2 if nat == 4 else [-0.2, 0.1, 0.05] * 3)
    return base + " -vg " + ",".join(f"{x:.6f}" for x in vg), g2


def _problem(args):
    return pm.Problem(args.split())


@pytest.mark.parametrize("args,n0,n1", [(GAAS, 24, 48), (SI, 48, 48), (RS, 48, 48), (GAAS + SOC, 24, 48)])
def test_cubic_group_orders(args, n0, n1):
    p = _problem(args)
    o0, o1 = p.symmetry_ops(0), p.symmetry_ops(pm.KGRID_TIME_REVERSAL)
    assert len(o0) == n0 and len(o1) == n1
    assert np.array_equal(o0[0], np.eye(3, dtype=np.int32))
    p.close()


@pytest.mark.parametrize("name,n0,n1", [("wz", 12, 24), ("te", 6, 12)])
def test_hex_group_orders(name, n0, n1):
    args, _ = _hex(name)
    p = _problem(args)
    assert len(p.symmetry_ops(0)) == n0 and len(p.symmetry_ops(pm.KGRID_TIME_REVERSAL)) == n1
    p.close()


def _closed(ops):
    S = {tuple(m.ravel()) for m in ops}
    return all(tuple((a @ b).ravel()) in S for a in ops for b in ops)


@pytest.mark.parametrize("which", ["gaas", "si", "rs", "wz", "te", "gaas_soc", "te_soc"])
def test_ops_form_a_group_and_match_oracle(which):
    if which in ("wz", "te", "te_soc"):
        args, g2 = _hex(which[:2])
        if which == "te_soc":
            args += f" -use_uniform_us_so -uniform_us_so_val 0.002 -ua_so {g2[0]:.6f}:0.001"
    else:
        args = {"gaas": GAAS, "si": SI, "rs": RS, "gaas_soc": GAAS + SOC}[which]
    p = _problem(args)
    for flags in (0, pm.KGRID_TIME_REVERSAL):
        ops = p.symmetry_ops(flags).astype(np.int64)
        assert _closed(ops)
        if "soc" not in which:
            cr, mat, _, _ = O.from_args(args.split())
            species = [tuple(r) for r in mat.vg]
            ref = O.point_group_ops(cr, species, time_reversal=bool(flags))
            assert {tuple(m.ravel()) for m in ops} == {tuple(m.ravel()) for m in ref}
    p.close()


@pytest.mark.parametrize("which", ["gaas_soc", "wz", "te_soc"])
def test_ops_keep_the_spectrum(which):
    if which == "gaas_soc":
        args = GAAS.replace("-encut 50", "-encut 30") + SOC
    else:
        args, g2 = _hex(which[:2])
        if which == "te_soc":
            args += f" -use_uniform_us_so -uniform_us_so_val 0.002 -ua_so {g2[0]:.6f}:0.001"
    p = _problem(args)
    G, _ = p.gvectors()
    cr, mat, _, _ = O.from_args(args.split())
    ops = p.symmetry_ops(pm.KGRID_TIME_REVERSAL).astype(float)
    Bm = cr.recip.T
    Bi = np.linalg.inv(Bm)
    k = np.array([0.071, -0.043, 0.029])
    e0 = np.linalg.eigvalsh(O.hamiltonian(cr, mat, G, k))
    scale = np.abs(e0).max()
    rng = np.random.default_rng(1)
    for M in ops[rng.permutation(len(ops))[:8]]:
        R = Bm @ M @ Bi
        e = np.linalg.eigvalsh(O.hamiltonian(cr, mat, G, R @ k))
        assert np.abs(e - e0).max() <= 1e-9 * scale
    p.close()


def test_oracle_reduction_partitions_the_grid():
    cr = O.Crystal("zb", 5.65)
    oh = O.point_group_ops(cr, [0, 1], time_reversal=True)
    idx, w = O.ibz_reduce(oh, (8, 8, 8))
    assert len(idx) == 29 and w.sum() == 512
    idx, w = O.ibz_reduce(oh, (6, 6, 6))
    assert w.sum() == 216 and len(idx) == 16
    ident = np.eye(3, dtype=int)[None]
    idx, w = O.ibz_reduce(ident, (3, 4, 5))
    assert len(idx) == 60 and np.all(w == 1)
