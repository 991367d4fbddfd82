"""Parameter recovery for trigonal Te through the adjoint (differentiation workload).

python -m picomax_b200.te_fit [--steps 200] [--lr 0.05] [--fd-h 1e-5,1e-6] [--no-fd]

Free parameters theta (Ry): 8 form factors shared by the 3 atoms, lambda_S
(uniform over |G|^2) and lambda_A (first 4 shells); te_params() draws the
starting point from a seed, and the targets come from the method itself at
seeded perturbed parameters theta* (form factors +- 0.02 Ry, lambda +- 20 %):

  L(theta) = sum over the 121-point G-A-H-K-G path of (E_n(k) - E*_n(k))^2
           + sum over 1000 w of (Im eps_M(w) - Im eps_M*(w))^2
             (eps_M on the 10x10x8 Gamma-centred grid, NEPS 15, Gaussian 0.05 eV)

The gradient comes from the hand-written adjoint (picomax_b200.autograd);
it is first checked against central finite differences of L (step --fd-h),
D(h) = (L(theta + h e_p) - L(theta - h e_p)) / 2h, and against their
Richardson extrapolation (4 D(h/2) - D(h)) / 3, which cancels the h^2 term of
the truncation error (for lambda_S, ~0.003 Ry, a step of 1e-5 Ry is 0.3 % of
the parameter, and D(h)'s truncation error dominates), then Adam runs --steps
steps. One JSON line per phase goes to stdout.
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
import time

import numpy as np
import torch

from . import _capi as C
from .autograd import band, eps_m
from .workloads import te_param_map, te_params, workload

FAMILIES = ("assemble", "heev", "overlap", "contract_f64", "scale", "kk", "adj_epsm", "adj_kk", "adj_contract",
            "adj_mbar", "adj_zbar", "adj_eig", "adj_resolvent", "adj_hgrad", "adj_hscatter")


def perturbed(theta0: np.ndarray, seed: int = 1970) -> np.ndarray:
    r = np.random.default_rng(seed)
    t = theta0.copy()
    t[:8] += r.uniform(-0.02, 0.02, 8)
    t[8:] *= 1.0 + r.uniform(-0.2, 0.2, 2)
    return t


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--lr", type=float, default=0.05, help="Adam step in units of --scale")
    ap.add_argument("--decay", type=float, default=0.985)
    ap.add_argument("--scale", default="0.02,0.002", help="parameter scale (Ry) of form factors, SOC")
    ap.add_argument("--fd-h", default="1e-5", help="comma-separated finite-difference steps (Ry)")
    ap.add_argument("--no-fd", action="store_true")
    ap.add_argument("--kgrid", default="10,10,8", help="k grid of the eps_M term")
    a = ap.parse_args(argv)

    tmp = tempfile.mkdtemp()
    bargs, _, _ = workload("te_band", tmp)
    eargs, _, _ = workload("te_epsLL", tmp)
    if a.kgrid != "10,10,8":
        from .kgrid import make_kfile
        n1, n2, n3 = (int(x) for x in a.kgrid.split(","))
        kf = f"{tmp}/k_te_custom.txt"
        make_kfile(kf, "te", n1, n2, n3, f=1.33)
        eargs[eargs.index("-kpointfile") + 1] = kf
    pb, pe = C.Problem(bargs), C.Problem(eargs)
    ctx = C.Context(0)
    J = te_param_map()
    theta0 = te_params()
    theta_star = perturbed(theta0)

    # targets
    with torch.no_grad():
        ts = torch.tensor(theta_star, dtype=torch.float64)
        E_star = band(ts, pb, ctx, J).clone()
        t_star = eps_m(ts, pe, ctx, J).imag.clone()

    def loss_fn(theta):
        E = band(theta, pb, ctx, J)
        eps = eps_m(theta, pe, ctx, J)
        return ((E - E_star) ** 2).sum() + ((eps.imag - t_star) ** 2).sum()

    def timed_grad(theta_np):
        th = torch.tensor(theta_np, dtype=torch.float64, requires_grad=True)
        t0 = time.perf_counter()
        L = loss_fn(th)
        t1 = time.perf_counter()
        L.backward()
        t2 = time.perf_counter()
        return float(L.detach()), th.grad.numpy().copy(), t1 - t0, t2 - t1

    before = {f: ctx.kernel_time(f) for f in FAMILIES}
    L0, g0, t_fwd, t_bwd = timed_grad(theta0)
    kt = {f: round(ctx.kernel_time(f)[0] - before[f][0], 3) for f in FAMILIES}
    info = {"phase": "gradient", "npw": pe.info.npw, "nh": 2 * pe.info.npw, "nk": pe.info.nk,
            "nq_band": pb.info.nq, "nfreq": pe.info.nfreq, "loss": L0, "forward_s": t_fwd, "backward_s": t_bwd,
            "kernel_ms": {f: v for f, v in kt.items() if v > 0}, "grad": g0.tolist()}
    print(json.dumps(info), flush=True)
    ident = np.abs(g0) > 1e-9 * np.abs(g0).max()

    def central(h):
        fd = np.zeros_like(g0)
        with torch.no_grad():
            for p in range(len(theta0)):
                tp, tm = theta0.copy(), theta0.copy()
                tp[p] += h
                tm[p] -= h
                fd[p] = (float(loss_fn(torch.tensor(tp))) - float(loss_fn(torch.tensor(tm)))) / (2 * h)
        return fd

    def rel_err(fd):
        big = np.abs(fd) > 1e-9 * np.abs(fd).max()  # parameters the loss depends on
        return np.where(big, np.abs(g0 - fd) / np.where(big, np.abs(fd), 1.0), 0.0)

    for h in ([] if a.no_fd else [float(x) for x in a.fd_h.split(",")]):
        t0 = time.perf_counter()
        fd = central(h)
        fd2 = central(h / 2)
        rich = (4.0 * fd2 - fd) / 3.0
        rel, relr = rel_err(fd), rel_err(rich)
        print(json.dumps({"phase": "finite_differences", "h_Ry": h, "fd": fd.tolist(),
                          "rel_err_per_param": rel.tolist(), "max_rel_err": float(rel.max()),
                          "max_abs_err_over_max_grad": float(np.abs(g0 - fd).max() / np.abs(fd).max()),
                          "fd_richardson": rich.tolist(), "rel_err_per_param_richardson": relr.tolist(),
                          "max_rel_err_richardson": float(relr.max()),
                          "seconds": time.perf_counter() - t0}), flush=True)

    # Adam on u = (theta - theta0) / scale: one step size for parameters whose
    # magnitudes differ by two orders (form factors ~0.1 Ry, SOC ~0.005 Ry)
    sf, ss = (float(x) for x in a.scale.split(","))
    scale = torch.tensor([sf] * 8 + [ss, ss], dtype=torch.float64)
    base = torch.tensor(theta0, dtype=torch.float64)
    u = torch.zeros(len(theta0), dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([u], lr=a.lr)
    sched = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=a.decay)
    t0 = time.perf_counter()
    for step in range(a.steps):
        opt.zero_grad()
        L = loss_fn(base + scale * u)
        L.backward()
        opt.step()
        sched.step()
        err = float(np.abs((base + scale * u).detach().numpy() - theta_star).max())
        if step % 20 == 0 or step == a.steps - 1:
            print(json.dumps({"phase": "adam", "step": step, "loss": float(L.detach()),
                              "max_abs_param_err_Ry": err}), flush=True)
    dt = time.perf_counter() - t0
    final = (base + scale * u).detach().numpy()
    with torch.no_grad():
        Lf = float(loss_fn(torch.tensor(final)))
    print(json.dumps({"phase": "result", "steps": a.steps, "seconds": dt, "s_per_step": dt / max(a.steps, 1),
                      "loss_start": L0, "loss_end": Lf, "theta_start": theta0.tolist(),
                      "theta_true": theta_star.tolist(), "theta_end": final.tolist(),
                      "max_abs_param_err_start_Ry": float(np.abs(theta0 - theta_star).max()),
                      "max_abs_param_err_end_Ry": float(np.abs(final - theta_star).max()),
                      # parameters the loss does not depend on (form factors of shells whose
                      # structure factor vanishes) cannot be recovered
                      "identifiable": ident.tolist(),
                      "max_abs_param_err_identifiable_end_Ry": float(np.abs(final - theta_star)[ident].max()),
                      "max_rel_param_err_identifiable_end": float(
                          (np.abs(final - theta_star) / np.abs(theta_star))[ident].max())}), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
