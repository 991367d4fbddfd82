"""Benchmark: eps_M(q, w) / chi(q, w) spectra per second of the picomax B200 path.

Workload (default): GaAs zinc-blende with spin-orbit coupling, epsij switch,
16x16x16 Gamma-centred k grid (4096 k + 4096 k+q eigensolves of 274x274
complex), 27 local-field G, NBAND 16 / nvalence 8, 2000 frequencies over
0-25 eV, Lorentzian 0.05 eV, Kramers-Kronig (picomax_b200/workloads.py,
"gaas_epsij"). One step = one spectrum: every eigensolve, the overlaps, the
contraction, scaling and KK of one (crystal, q).

Reported: `value` = spectra/s of the mixed-precision path with results left
in HBM (CUDA events on the library's stream), `fp64` = the same with the FP64
contraction, `e2e` = spectra/s through pmx_chi with host buffers (pinned),
every host<->device copy inside the timed region. With --gpus N each rank runs
its own spectra (independent (crystal, q) units, no collective on the data
path; weak scaling) and the slowest rank's time counts.

`--impl reference` times the reference PicoMax (rebuilt from source in
oracle/_ref, OpenMP on every host core) on a bounded sample of the same
workload: the first 64 of the 4096 k-points; its per-stage timings are scaled
to the full grid (k-dependent stages x 64, the Kramers-Kronig stage as is).
"""
import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "eps_M(q,w) spectra/s, mixed vs FP64 GPU at <=1e-4 rel err; eigensolve k-pts/s"
FP64_TFLOPS_NOMINAL = 37.0  # B200 FP64 (HGX spec sheet); no measured FP64 peak on this pool


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gaas_epsij")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="leave out the timed reference sample (minutes of host time on the larger workloads)")
    return ap.parse_args()


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device=0):
        self.samples = []
        self.dev = device
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in self.samples for n, v in zip(names, s[4:8]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def profiled_heev_bytes(n):
    """DRAM bytes per matrix of the eigensolver at size n from the committed
    ncu summary (dram__bytes_read.sum + dram__bytes_write.sum of one capture
    divided by its matrices), or None when no capture covers this n."""
    path = os.path.join(ROOT, "profiles", "heev_kernel_gaas_epsij_8.md")
    if not os.path.exists(path):
        return None
    m = re.search(rf"dram_bytes_per_matrix n={n}: ([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def _ref_run(binary, argv, lines, sample, tmp, env):
    """One run of the reference binary on the first `sample` k-points of the
    workload's k-point file: (k-dependent stage seconds, Kramers-Kronig seconds)."""
    kfs = os.path.join(tmp, "k_sample.txt")
    with open(kfs, "w") as fh:
        fh.write(lines[0] + "\n" + str(sample) + "\n" + "\n".join(lines[2:2 + sample]) + "\n")
    argv = list(argv)
    argv[argv.index("-kpointfile") + 1] = kfs
    r = subprocess.run([binary] + argv + ["-wdir", tmp, "-outputfile", "ref"], capture_output=True, text=True,
                       env=env)
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}")
    el = [float(x) for x in re.findall(r"Elapsed time: ([0-9.eE+-]+) s", r.stdout)]
    # stdout order: G list, k list, [k stage, (overlaps, accumulation, KK)], total
    kk = el[5] if len(el) > 6 else 0.0
    return el[2] + el[3] + el[4], kk


def _ref_plan(binary, argv, lines, tmp, env, cores, target_s=15.0):
    """Sample size for about target_s seconds of k-dependent reference work per
    run: a first run on one k-point per host core (the reference's k loops are
    OpenMP-parallel), scaled up in whole multiples of the core count. Returns
    (sample, the first run's times when that run is the sample, else None)."""
    nk_full = int(lines[1])
    s0 = min(cores, nk_full)
    t0 = _ref_run(binary, argv, lines, s0, tmp, env)
    if t0[0] >= 0.5 * target_s or s0 == nk_full:
        return s0, t0
    grow = max(1, int(target_s / max(t0[0], 1e-3)))
    return min(nk_full, s0 * grow), None


def reference_arm(args, rank, world):
    if rank != 0:
        return
    from picomax_b200.workloads import workload
    tmp = tempfile.mkdtemp(prefix="pmx_ref_")
    argv, nspec, _ = workload(args.workload, tmp)
    binary = os.path.join(ROOT, "oracle", "_ref", "picomax_ref_ll" if "epsLL" in argv else "picomax_ref_guard")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference tree)"}))
        return
    lines = open(argv[argv.index("-kpointfile") + 1]).read().splitlines()
    nk_full = int(lines[1])
    cores = os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    try:
        sample, _ = _ref_plan(binary, argv, lines, tmp, env, cores)  # an extra, untimed warm-up run
        times = []
        for step in range(args.warmup + args.steps):
            kdep, kk = _ref_run(binary, argv, lines, sample, tmp, env)
            if step >= args.warmup:
                times.append(kdep * (nk_full / sample) + kk)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    t = sum(times) / len(times)
    v = nspec / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "spectra/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded form factors)",
        "config": {"workload": args.workload, "kpoints": nk_full},
        "cpu_baseline": {"value": v, "unit": "spectra/s", "cores": cores, "kind": "reference",
                         "sample": f"first {sample} of {nk_full} k-points per step; k-dependent stage times "
                                   f"x{nk_full / sample:.2f}, Kramers-Kronig as measured"},
        "e2e": {"value": v, "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    shutil.rmtree(tmp, ignore_errors=True)


def cpu_baseline_sample(wl_argv, nspec):
    """The reference on the host cores, on a sample of the workload's k-points
    sized for about 15 s of k-dependent work (see _ref_plan)."""
    binary = os.path.join(ROOT, "oracle", "_ref", "picomax_ref_ll" if "epsLL" in wl_argv else "picomax_ref_guard")
    if not os.path.exists(binary):
        return None
    tmp = tempfile.mkdtemp(prefix="pmx_cpu_")
    lines = open(wl_argv[wl_argv.index("-kpointfile") + 1]).read().splitlines()
    nk_full = int(lines[1])
    cores = os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    try:
        sample, res = _ref_plan(binary, wl_argv, lines, tmp, env, cores)
        kdep, kk = res if res is not None else _ref_run(binary, wl_argv, lines, sample, tmp, env)
    except RuntimeError:
        return None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    full = kdep * (nk_full / sample) + kk
    return {"value": nspec / full, "unit": "spectra/s", "cores": cores, "kind": "reference",
            "sample": f"reference (oracle/_ref, OpenMP) on the first {sample} of {nk_full} k-points; "
                      f"k-dependent stages x{nk_full / sample:.2f}, Kramers-Kronig as measured"}


def ours(args, rank, world):
    import numpy as np
    import torch

    import picomax_b200 as pm
    from picomax_b200.workloads import workload

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    tmp = tempfile.mkdtemp(prefix=f"pmx_bench{rank}_")
    argv, nspec, nsolves = workload(args.workload, tmp)
    prob = pm.Problem(argv)
    sw = {"epsij": pm.SWITCH_EPSIJ, "epsLL": pm.SWITCH_EPSLL}[argv[argv.index("-switch") + 1]]
    ctx = pm.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    nvals = prob.info.chi_values
    re_d = torch.empty(nvals, dtype=torch.float64, device=f"cuda:{dev}")
    im_d = torch.empty_like(re_d)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=f"cuda:{dev}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps

    mixed = lambda: ctx.chi_device(prob, sw, pm.PREC_MIXED, re_d.data_ptr(), im_d.data_ptr())
    fp64 = lambda: ctx.chi_device(prob, sw, pm.PREC_FP64, re_d.data_ptr(), im_d.data_ptr())
    for _ in range(args.warmup):
        mixed()
    # accuracy of the mixed path against the FP64 path on this workload
    fp64()
    ref_re, ref_im = re_d.clone(), im_d.clone()
    mixed()
    scale = max(ref_re.abs().max().item(), ref_im.abs().max().item())
    err = max((re_d - ref_re).abs().max().item(), (im_d - ref_im).abs().max().item()) / scale
    del ref_re, ref_im
    # kernel-family device times over the mixed timed region
    fams = ["assemble", "heev", "overlap", "contract_mixed", "contract_f64", "scale", "kk"]
    k0 = {f: ctx.kernel_time(f) for f in fams}
    l0 = ctx.kernel_launches()
    mma0 = ctx.mixed_mmas()
    with ClockSampler(dev) as clk:
        ms_mixed = timed(mixed, args.steps)
    l1 = ctx.kernel_launches()
    mma1 = ctx.mixed_mmas()
    k1 = {f: ctx.kernel_time(f) for f in fams}
    stage = ctx.stage_times()
    ms_fp64 = timed(fp64, max(1, args.fp64_steps))
    # end to end through pmx_chi with pinned host buffers
    re_h = torch.empty(nvals, dtype=torch.float64).pin_memory()
    im_h = torch.empty(nvals, dtype=torch.float64).pin_memory()
    lib = pm.load()
    import ctypes
    dptr = ctypes.POINTER(ctypes.c_double)
    rp = ctypes.cast(re_h.data_ptr(), dptr)
    ip = ctypes.cast(im_h.data_ptr(), dptr)

    def e2e_step():
        st = lib.pmx_chi(ctx.handle, prob.handle, sw, pm.PREC_MIXED, rp, ip)
        if st != 0:
            raise RuntimeError(lib.pmx_ctx_last_error(ctx.handle).decode())

    e2e_step()
    b0 = ctx.transfer_bytes()
    barrier()
    t0 = time.perf_counter()
    ms_e2e = timed(e2e_step, args.steps)
    wall_e2e = (time.perf_counter() - t0) / args.steps
    b1 = ctx.transfer_bytes()
    h2d = (b1[0] - b0[0]) // args.steps
    d2h = (b1[1] - b0[1]) // args.steps

    # roofline of the dominant kernel family of the mixed step
    per = {f: ((k1[f][0] - k0[f][0]) / args.steps, (k1[f][1] - k0[f][1]) / args.steps) for f in fams}
    dom = max(per, key=lambda f: per[f][0])
    n = prob.info.nh if prob.info.soc else prob.info.npw
    nb = prob.info.nband if prob.info.soc else (prob.info.nband + 1) // 2
    nk = prob.info.nk
    roof = None
    if dom == "heev":
        flops = nsolves * ((16.0 / 3.0) * n ** 3 + 8.0 * n * n * nb)
        ms_launch = per["heev"][0] / max(per["heev"][1], 1)
        flops_launch = flops / max(per["heev"][1], 1)
        ach = flops_launch / (ms_launch * 1e-3) / 1e12
        bpm = profiled_heev_bytes(n)
        traffic = bpm * nsolves / max(per["heev"][1], 1) if bpm else None
        roof = {"kernel": "heev_kernel", "bound": "fp64", "achieved": ach, "peak": FP64_TFLOPS_NOMINAL,
                "unit": "TFLOP/s", "frac": ach / FP64_TFLOPS_NOMINAL, "traffic": traffic,
                "traffic_source": "DRAM bytes per matrix of the ncu capture in profiles/heev_kernel_gaas_epsij_8.md "
                                  "x matrices per launch" if bpm else None,
                "peak_source": "nominal B200 FP64 (no measured FP64 peak in MEASURED_PEAKS.json)",
                "per_launch_ms": ms_launch, "launches_per_step": per["heev"][1]}
    # the tensor-core contraction, whichever kernel dominates: tcgen05 MMA
    # instructions (2*128*256*16 flop each, the three split products counted)
    # over the contract_mixed stage time (the mixed kernel plus its small
    # helper kernels), against the measured cuBLAS bf16 burst peak
    roof_mixed = None
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        peaks = {}
    mma_step = (mma1 - mma0) / args.steps
    if mma_step > 0 and per["contract_mixed"][0] > 0:
        tf = mma_step * 2.0 * 128 * 256 * 16 / (per["contract_mixed"][0] * 1e-3) / 1e12
        pk = peaks.get("bf16_tflops") or 1590.0
        roof_mixed = {"kernel": "mixed_kernel", "bound": "tensor", "achieved": tf, "peak": pk, "unit": "TFLOP/s",
                      "frac": tf / pk, "mma_per_step": mma_step,
                      "peak_source": "measured bf16 burst (MEASURED_PEAKS.json)" if peaks.get("bf16_tflops")
                      else "fallback 1.59 PFLOP/s"}
    if dom == "contract_mixed":
        roof = dict(roof_mixed or {"kernel": "mixed_kernel", "bound": "tensor", "unit": "TFLOP/s"}, traffic=None)
    n_eig = 1 + 2 * nk
    out = {
        "metric": METRIC, "value": world * nspec / (ms_mixed * 1e-3), "unit": "spectra/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 eigensolve + split-bf16 tensor contraction",
        "data": "synthetic (seeded form factors, generated k grid)",
        "config": {"workload": args.workload, "material": "GaAs zb + SOC" if "gaas" in args.workload else
                   args.workload, "npw": prob.info.npw, "nh": n, "nk": nk, "neps": prob.info.neps,
                   "nfreq": prob.info.nfreq, "l2": "working set > L2 (eigenvectors + overlaps ~1.9 GB)"},
        "fp64": {"value": world * nspec / (ms_fp64 * 1e-3), "unit": "spectra/s", "ms_per_step": ms_fp64},
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "mixed_max_rel_err_vs_fp64": err,
        "eig_kpts_per_s": world * n_eig / (per["heev"][0] * 1e-3 + per["assemble"][0] * 1e-3),
        "stage_ms": {f: per[f][0] for f in fams},
        "e2e": {"value": world * nspec / (ms_e2e * 1e-3), "unit": "spectra/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "wall_ms_per_step": wall_e2e * 1e3},
        "gpu_launches": int((l1 - l0) / args.steps),
        "roofline": roof, "roofline_mixed_contraction": roof_mixed, "clocks": clk.summary(),
        "degenerate_cuts": ctx.degenerate_cuts(),
        "autotune": ctx.tuning(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_sample(argv, nspec)
        out["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    shutil.rmtree(tmp, ignore_errors=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    rank, world = dist_init(args.gpus)
    if args.impl == "reference":
        reference_arm(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    ours(args, rank, world)


if __name__ == "__main__":
    main()
