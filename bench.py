"""Benchmark: eps_M(q, w) / chi(q, w) spectra per second of the picomax B200 path.

Workload (default): GaAs zinc-blende with spin-orbit coupling, epsij switch,
16x16x16 Gamma-centred k grid (4096 k + 4096 k+q eigensolves of 274x274
complex), 27 local-field G, NBAND 16 / nvalence 8, 2000 frequencies over
0-25 eV, Lorentzian 0.05 eV, Kramers-Kronig (picomax_b200/workloads.py,
"gaas_epsij"). One step = one spectrum: every eigensolve, the overlaps, the
contraction, scaling and KK of one (crystal, q); for an epsLL workload the
step also forms eps_M(q, w) on the device.

Reported: `value` = spectra/s of the mixed-precision path with results left
in HBM (CUDA events on the library's stream), `fp64` = the same with the FP64
contraction, `e2e` = spectra/s through pmx_chi with host buffers (pinned),
every host<->device copy inside the timed region. With --gpus N each rank runs
its own spectra (independent (crystal, q) units, no collective on the data
path; weak scaling) and the slowest rank's time counts. `extra_workloads`
repeats the measurement (fewer steps) on the wurtzite epsLL workload
(N_G 401, NEPS 59, 24x24x16 k) and on the Te + SOC epsLL workload (n 570,
NEPS 15, 10x10x8 k) unless --no-extra.

`--impl reference` times the reference PicoMax (rebuilt from source in
oracle/_ref, OpenMP on every host core) on a bounded sample of the same
workload: k-points taken at an even stride through the workload's k file,
as many as about 15 s of k-dependent work per step needs (one per host core
first, then whole multiples of the core count). `ms_per_step` is the measured
time of one sampled step; `value` is the full spectrum rate estimated from it
(k-dependent stage times scaled by the full grid over the sample, the
Kramers-Kronig stage as measured), stated in `cpu_baseline.sample`.
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
FP64_TFLOPS_NOMINAL = 37.0  # B200 FP64 (HGX spec sheet)


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
    ap.add_argument("--no-extra", action="store_true", help="leave out the wurtzite and Te epsLL measurements")
    ap.add_argument("--schedule", type=int, default=-1,
                    help="fixed eigensolver schedule (default -1: the autotuner picks; 0 is the two-stage solver "
                         "where it applies) - for profiler runs, whose serialised launches skew the autotuner")
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
    path = os.path.join(ROOT, "profiles", "heev2_gaas_epsij.md")
    if not os.path.exists(path):
        return None
    m = re.search(rf"dram_bytes_per_matrix n={n}: ([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def workload_config(name, info):
    """The `config` object of both arms: the workload and its sizes."""
    n = info.nh if info.soc else info.npw
    return {"workload": name, "material": "GaAs zb + SOC" if name.startswith("gaas") else name,
            "npw": info.npw, "nh": n, "nk": info.nk, "neps": info.neps, "nfreq": info.nfreq,
            "l2": "working set > L2 (eigenvectors + overlaps ~1.9 GB)"}


def _ref_run(binary, argv, lines, sample, tmp, env):
    """One run of the reference binary on `sample` k-points taken at an even
    stride through the workload's k-point file: (k-dependent stage seconds,
    Kramers-Kronig seconds, wall seconds)."""
    kfs = os.path.join(tmp, "k_sample.txt")
    pts = lines[2:2 + int(lines[1])]
    stride = max(1, len(pts) // sample)
    with open(kfs, "w") as fh:  # an even stride through the zone, not its first points
        fh.write(lines[0] + "\n" + str(sample) + "\n" + "\n".join(pts[::stride][:sample]) + "\n")
    argv = list(argv)
    argv[argv.index("-kpointfile") + 1] = kfs
    t0 = time.perf_counter()
    r = subprocess.run([binary] + argv + ["-wdir", tmp, "-outputfile", "ref"], capture_output=True, text=True,
                       env=env)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}")
    el = [float(x) for x in re.findall(r"Elapsed time: ([0-9.eE+-]+) s", r.stdout)]
    # stdout order: G list, k list, [k stage, (overlaps, accumulation, KK)], total
    kk = el[5] if len(el) > 6 else 0.0
    return el[2] + el[3] + el[4], kk, wall


def _ref_plan(binary, argv, lines, tmp, env, cores, target_s=15.0):
    """Sample size for about target_s seconds of k-dependent reference work per
    run: a first run on one k-point per host core (the reference's k loops are
    OpenMP-parallel), scaled up in whole multiples of the core count. Returns
    (sample, the first run's times when that run is the sample, else None)."""
    nk_full = int(lines[1])
    s0 = min(cores, nk_full)
    t0 = _ref_run(binary, argv, lines, s0, tmp, env)[:2]
    if t0[0] >= 0.5 * target_s or s0 == nk_full:
        return s0, t0
    grow = max(1, int(target_s / max(t0[0], 1e-3)))
    return min(nk_full, s0 * grow), None


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import picomax_b200 as pm
    from picomax_b200.workloads import workload
    tmp = tempfile.mkdtemp(prefix="pmx_ref_")
    argv, nspec, _ = workload(args.workload, tmp)
    binary = os.path.join(ROOT, "oracle", "_ref", "picomax_ref_ll" if "epsLL" in argv else "picomax_ref_guard")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference tree)"}))
        return
    prob = pm.Problem(argv)  # host-side parsing only: the same config object as the GPU arm
    config = workload_config(args.workload, prob.info)
    prob.close()
    lines = open(argv[argv.index("-kpointfile") + 1]).read().splitlines()
    nk_full = int(lines[1])
    cores = os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    try:
        sample, _ = _ref_plan(binary, argv, lines, tmp, env, cores)  # an extra, untimed warm-up run
        est, walls = [], []
        for step in range(args.warmup + args.steps):
            kdep, kk, wall = _ref_run(binary, argv, lines, sample, tmp, env)
            if step >= args.warmup:
                est.append(kdep * (nk_full / sample) + kk)
                walls.append(wall)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    t = sum(est) / len(est)
    v = nspec / t
    desc = (f"{sample} of {nk_full} k-points at an even stride per step (reference oracle/_ref, OpenMP); "
            f"full-spectrum time estimated as k-dependent stages x{nk_full / sample:.2f} + Kramers-Kronig "
            f"as measured: {t:.1f} s per spectrum")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "spectra/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
        "ms_per_spectrum_estimated": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded form factors)",
        "config": config,
        "cpu_baseline": {"value": v, "unit": "spectra/s", "cores": cores, "kind": "reference", "sample": desc},
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
        kdep, kk = res if res is not None else _ref_run(binary, wl_argv, lines, sample, tmp, env)[:2]
    except RuntimeError:
        return None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    full = kdep * (nk_full / sample) + kk
    return {"value": nspec / full, "unit": "spectra/s", "cores": cores, "kind": "reference",
            "sample": f"reference (oracle/_ref, OpenMP) on {sample} of {nk_full} k-points at an even stride; "
                      f"k-dependent stages x{nk_full / sample:.2f}, Kramers-Kronig as measured"}


def measure(name, steps, warmup, fp64_steps, rank, world, dev, with_e2e=True, schedule=-1):
    """One workload: mixed and FP64 spectra/s (device-resident), accuracy of the
    mixed path against the FP64 one, per-stage device times, e2e through the
    C-ABI with host buffers, launches and tensor-core MMAs of the timed region."""
    import ctypes

    import torch

    import picomax_b200 as pm
    from picomax_b200.workloads import workload

    tmp = tempfile.mkdtemp(prefix=f"pmx_bench{rank}_")
    argv, nspec, nsolves = workload(name, tmp)
    prob = pm.Problem(argv)
    swname = argv[argv.index("-switch") + 1]
    sw = {"epsij": pm.SWITCH_EPSIJ, "epsLL": pm.SWITCH_EPSLL}[swname]
    ctx = pm.Context(dev)
    if schedule >= 0:
        ctx.set_schedule(schedule)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    nvals = prob.info.chi_values
    re_d = torch.empty(nvals, dtype=torch.float64, device=f"cuda:{dev}")
    im_d = torch.empty_like(re_d)
    # eps_M(q, w) is part of an epsLL step (the (L, L) block's macroscopic function)
    epsm_d = (torch.empty(prob.info.nq * prob.info.nfreq * 2, dtype=torch.float64, device=f"cuda:{dev}")
              if swname == "epsLL" else None)
    eptr = epsm_d.data_ptr() if epsm_d is not None else 0

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, nsteps):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps):
            fn()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=f"cuda:{dev}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms / nsteps

    mixed = lambda: ctx.chi_device(prob, sw, pm.PREC_MIXED, re_d.data_ptr(), im_d.data_ptr(), eptr)
    fp64 = lambda: ctx.chi_device(prob, sw, pm.PREC_FP64, re_d.data_ptr(), im_d.data_ptr(), eptr)
    for _ in range(warmup):
        mixed()
    # accuracy of the mixed path against the FP64 path on this workload
    fp64()
    ref_re, ref_im = re_d.clone(), im_d.clone()
    ref_eps = epsm_d.clone() if epsm_d is not None else None
    mixed()
    scale = max(ref_re.abs().max().item(), ref_im.abs().max().item())
    err = max((re_d - ref_re).abs().max().item(), (im_d - ref_im).abs().max().item()) / scale
    err_eps = ((epsm_d - ref_eps).abs().max() / ref_eps.abs().max()).item() if ref_eps is not None else None
    del ref_re, ref_im, ref_eps
    # kernel-family device times over the mixed timed region
    fams = ["assemble", "heev", "transitions", "overlap", "overlap_tc", "contract_mixed", "contract_f64", "scale",
            "kk", "epsm"]
    k0 = {f: ctx.kernel_time(f) for f in fams}
    l0 = ctx.kernel_launches()
    mma0 = ctx.mixed_mmas()
    with ClockSampler(dev) as clk:
        ms_mixed = timed(mixed, steps)
    l1 = ctx.kernel_launches()
    mma1 = ctx.mixed_mmas()
    k1 = {f: ctx.kernel_time(f) for f in fams}
    ms_fp64 = timed(fp64, max(1, fp64_steps))
    out_e2e = None
    if with_e2e:
        # end to end through pmx_chi (pmx_chi_epsm for epsLL) with pinned host buffers
        re_h = torch.empty(nvals, dtype=torch.float64).pin_memory()
        im_h = torch.empty(nvals, dtype=torch.float64).pin_memory()
        eps_h = torch.empty(prob.info.nq * prob.info.nfreq * 2, dtype=torch.float64).pin_memory()
        lib = pm.load()
        dptr = ctypes.POINTER(ctypes.c_double)
        rp = ctypes.cast(re_h.data_ptr(), dptr)
        ip = ctypes.cast(im_h.data_ptr(), dptr)
        ep = ctypes.cast(eps_h.data_ptr(), dptr)

        def e2e_step():
            if epsm_d is not None:
                st = lib.pmx_chi_epsm(ctx.handle, prob.handle, sw, pm.PREC_MIXED, rp, ip, ep)
            else:
                st = lib.pmx_chi(ctx.handle, prob.handle, sw, pm.PREC_MIXED, rp, ip)
            if st != 0:
                raise RuntimeError(lib.pmx_ctx_last_error(ctx.handle).decode())

        e2e_step()
        b0 = ctx.transfer_bytes()
        barrier()
        t0 = time.perf_counter()
        ms_e2e = timed(e2e_step, steps)
        wall_e2e = (time.perf_counter() - t0) / steps
        b1 = ctx.transfer_bytes()
        out_e2e = {"value": world * nspec / (ms_e2e * 1e-3), "unit": "spectra/s",
                   "h2d_bytes_per_step": int((b1[0] - b0[0]) // steps),
                   "d2h_bytes_per_step": int((b1[1] - b0[1]) // steps), "wall_ms_per_step": wall_e2e * 1e3}
    per = {f: ((k1[f][0] - k0[f][0]) / steps, (k1[f][1] - k0[f][1]) / steps) for f in fams}
    info = prob.info
    res = {
        "name": name, "argv": argv, "nspec": nspec, "nsolves": nsolves, "info": info,
        "value": world * nspec / (ms_mixed * 1e-3), "ms_per_step": ms_mixed,
        "fp64": {"value": world * nspec / (ms_fp64 * 1e-3), "unit": "spectra/s", "ms_per_step": ms_fp64},
        "mixed_over_fp64": ms_fp64 / ms_mixed, "mixed_max_rel_err_vs_fp64": err,
        "epsm_max_rel_err_vs_fp64": err_eps, "per": per, "launches": (l1 - l0) / steps,
        "mma_step": (mma1 - mma0) / steps, "clocks": clk.summary(), "e2e": out_e2e,
        "degenerate_cuts": ctx.degenerate_cuts(), "autotune": ctx.tuning(),
        "config": workload_config(name, info), "tmp": tmp,
    }
    ctx.close()
    return res


def fp64_peak_tflops(dev):
    """FP64 denominator measured in this run: cuBLAS DGEMM (torch.matmul) of
    8192 x 8192 float64 matrices, 2 warm-up and 5 timed products between CUDA
    events, best of the five (2 * 8192^3 flop each)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{dev}")
    b = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{dev}")
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def heev_roofline(m, fp64_peak=None):
    """Roofline of the eigensolver (the dominant kernel family): algorithmic
    FP64 work per launch over the event-timed launch duration, against the
    FP64 peak measured in this run (cuBLAS DGEMM; the nominal figure beside
    it); DRAM traffic from the committed ncu capture."""
    info = m["info"]
    n = info.nh if info.soc else info.npw
    nb = info.nband if info.soc else (info.nband + 1) // 2
    per = m["per"]
    nl = max(per["heev"][1], 1)
    flops = m["nsolves"] * ((16.0 / 3.0) * n ** 3 + 8.0 * n * n * nb)
    ms_launch = per["heev"][0] / nl
    ach = flops / nl / (ms_launch * 1e-3) / 1e12
    bpm = profiled_heev_bytes(n)
    pk = fp64_peak or FP64_TFLOPS_NOMINAL
    return {"kernel": "heev (two-stage: sb_kernel, sbtrd_kernel, tri_eig_kernel, eig2_back_kernel)",
            "bound": "fp64", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
            "frac": ach / pk, "frac_of_nominal": ach / FP64_TFLOPS_NOMINAL,
            "traffic": bpm * m["nsolves"] / nl if bpm else None,
            "traffic_source": "DRAM bytes per matrix of the ncu capture in profiles/heev2_gaas_epsij.md x matrices "
                              "per launch" if bpm else None,
            "peak_source": ("cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure); "
                            "frac_of_nominal against the 37 TFLOP/s spec") if fp64_peak else
                           "nominal B200 FP64 (no measured FP64 peak)",
            "per_launch_ms": ms_launch, "launches_per_step": per["heev"][1],
            "algorithmic_flop_per_matrix": (16.0 / 3.0) * n ** 3 + 8.0 * n * n * nb}


def mixed_roofline(m, peaks):
    """The split-BF16 tcgen05 contraction: MMA instructions of the step
    (2*128*256*16 flop each, the three split products counted) over the
    contract_mixed stage time, against the measured bf16 peaks."""
    per = m["per"]
    if not (m["mma_step"] > 0 and per["contract_mixed"][0] > 0):
        return None
    tf = m["mma_step"] * 2.0 * 128 * 256 * 16 / (per["contract_mixed"][0] * 1e-3) / 1e12
    pk = peaks.get("bf16_tflops") or 1590.0
    pks = peaks.get("bf16_tflops_sustained") or 1400.0
    return {"kernel": "mixed_kernel", "bound": "tensor", "achieved": tf, "peak": pk, "unit": "TFLOP/s",
            "frac": tf / pk, "frac_of_sustained": tf / pks, "useful_single_product_frac_of_sustained": tf / 3 / pks,
            "mma_per_step": m["mma_step"],
            "peak_source": "measured bf16 burst and sustained (MEASURED_PEAKS.json)" if peaks.get("bf16_tflops")
            else "fallback 1.59 PFLOP/s"}


def ours(args, rank, world):
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    m = measure(args.workload, args.steps, args.warmup, args.fp64_steps, rank, world, dev, schedule=args.schedule)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        peaks = {}
    per = m["per"]
    dom = max(per, key=lambda f: per[f][0])
    roof_mixed = mixed_roofline(m, peaks)
    fp64_pk = fp64_peak_tflops(dev)
    roof = heev_roofline(m, fp64_pk) if dom == "heev" else dict(roof_mixed or {"kernel": "mixed_kernel", "bound": "tensor",
                                                                       "unit": "TFLOP/s"}, traffic=None)
    n_eig = 1 + 2 * m["info"].nk
    out = {
        "metric": METRIC, "value": m["value"], "unit": "spectra/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 eigensolve + split-bf16 tensor contraction",
        "data": "synthetic (seeded form factors, generated k grid)",
        "config": m["config"],
        "fp64": m["fp64"], "mixed_over_fp64": m["mixed_over_fp64"],
        "mixed_max_rel_err_vs_fp64": m["mixed_max_rel_err_vs_fp64"],
        "eig_kpts_per_s": world * n_eig / (per["heev"][0] * 1e-3 + per["assemble"][0] * 1e-3),
        "stage_ms": {f: per[f][0] for f in per},
        "e2e": m["e2e"],
        "gpu_launches": int(m["launches"]),
        "roofline": roof, "roofline_heev": heev_roofline(m, fp64_pk), "roofline_mixed_contraction": roof_mixed,
        "clocks": m["clocks"], "degenerate_cuts": m["degenerate_cuts"], "autotune": m["autotune"],
    }
    if world == 1 and not args.no_extra:
        # the wurtzite epsLL workload (config 3: N_G 401, NEPS 59, 24x24x16 k), where the mixed path's
        # tensor-core contraction replaces most of the FP64 path's time, and the Te + SOC epsLL workload
        # (config 5's grid: n 570, NEPS 15, 10x10x8 k), where the FP64 eigensolver is nearly all of it
        out["extra_workloads"] = {}
        for name, steps in (("wz_epsLL", 2), ("te_epsLL", 3)):
            w = measure(name, steps, 3, 1, rank, world, dev, with_e2e=False, schedule=args.schedule)
            shutil.rmtree(w["tmp"], ignore_errors=True)
            out["extra_workloads"][name] = {
                "value": w["value"], "unit": "spectra/s", "ms_per_step": w["ms_per_step"], "steps": steps,
                "warmup": 3, "fp64": w["fp64"], "mixed_over_fp64": w["mixed_over_fp64"],
                "mixed_max_rel_err_vs_fp64": w["mixed_max_rel_err_vs_fp64"],
                "epsm_max_rel_err_vs_fp64": w["epsm_max_rel_err_vs_fp64"], "config": w["config"],
                "stage_ms": {f: w["per"][f][0] for f in w["per"]}, "roofline_heev": heev_roofline(w, fp64_pk),
                "roofline_mixed_contraction": mixed_roofline(w, peaks), "clocks": w["clocks"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_sample(m["argv"], m["nspec"])
    shutil.rmtree(m["tmp"], ignore_errors=True)
    if rank == 0:
        print(json.dumps(out))
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
