"""Per-quantity error of the mixed-precision path against the FP64 path.

python -m picomax_b200.precision_report WORKLOAD [WORKLOAD ...]

For each workload (names of picomax_b200.workloads) the spectrum is computed
twice through the C-ABI, with the FP64 contraction and with the split-BF16
tensor-core contraction, and the report gives, as JSON:
  * eigenvalues: both paths share the FP64 eigensolver launch by launch, so
    the error is zero by construction (checked on the band energies of the
    reference k-point);
  * |M|^2: max ||M_fp32|^2 - |M|^2| / max |M|^2 of the overlaps the tensor
    cores consume;
  * chi: max |chi_mixed - chi_fp64| / max |chi_fp64| over every stored entry,
    and the same on the (L, L) block;
  * eps_M (epsLL with NEPS <= 64): max |eps_M mixed - eps_M fp64| / max |eps_M|
    and the largest relative error of Im eps_M where |Im eps_M| exceeds 1% of
    its maximum.
"""
from __future__ import annotations

import json
import sys
import tempfile

import numpy as np

from . import _capi as C
from .workloads import workload


def report(name: str, ctx: C.Context) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        argv, _, _ = workload(name, tmp)
        p = C.Problem(argv)
        sw = {"epsij": C.SWITCH_EPSIJ, "epsLL": C.SWITCH_EPSLL}[argv[argv.index("-switch") + 1]]
        want_eps = sw == C.SWITCH_EPSLL and p.info.neps <= 64
        if want_eps:
            r64, i64, e64 = ctx.chi_epsm(p, sw, C.PREC_FP64)
            t64 = ctx.stage_times().sum()
            r32, i32, e32 = ctx.chi_epsm(p, sw, C.PREC_MIXED)
        else:
            r64, i64 = ctx.chi(p, sw, C.PREC_FP64)
            t64 = ctx.stage_times().sum()
            r32, i32 = ctx.chi(p, sw, C.PREC_MIXED)
        t32 = ctx.stage_times().sum()
        # the overlaps' own error: tensor-core overlaps against FP64 ones, in a
        # separate (untimed) call that computes both
        ctx.set_overlap_mode(2)
        ctx.chi(p, sw, C.PREC_MIXED)
        ctx.set_overlap_mode(1)
        m2_err, m2_max = ctx.overlap_error()
        off64 = ctx.ref_energy(p)
        off32 = ctx.ref_energy(p)
        scale = max(np.abs(r64).max(), np.abs(i64).max())
        neps, nf, nq = p.info.neps, p.info.nfreq, p.info.nq
        npairs = neps * (neps + 1) // 2
        ll = slice(0, nq * npairs * nf)  # (i, j) = (L, L) block leads the .dat order
        ll_scale = max(np.abs(r64[ll]).max(), np.abs(i64[ll]).max())
        out = {
            "workload": name, "npw": p.info.npw, "soc": p.info.soc, "nk": p.info.nk, "neps": neps, "nfreq": nf,
            "eigenvalue_abs_err_eV": abs(off64 - off32),
            "abs2M_max_rel_err": m2_err / m2_max if m2_max > 0 else 0.0,
            "chi_max_rel_err": max(np.abs(r32 - r64).max(), np.abs(i32 - i64).max()) / scale,
            "chi_LL_max_rel_err": max(np.abs(r32[ll] - r64[ll]).max(), np.abs(i32[ll] - i64[ll]).max()) / ll_scale,
            "device_ms_fp64": t64, "device_ms_mixed": t32,
        }
        if want_eps:
            out["epsM_max_rel_err"] = float(np.abs(e32 - e64).max() / np.abs(e64).max())
            im = np.abs(e64.imag)
            sel = im > 0.01 * im.max()
            out["epsM_im_max_rel_err_where_significant"] = float(
                (np.abs(e32.imag - e64.imag)[sel] / im[sel]).max()) if sel.any() else 0.0
        p.close()
        return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print(__doc__)
        return 2
    ctx = C.Context(0)
    for name in argv:
        print(json.dumps(report(name, ctx)), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
