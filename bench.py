#!/usr/bin/env python
"""Headline benchmark: adaptive Laplace KIFMM throughput at N = 1M.

Workload (default --config c2): 1,000,000 points from a mixture of 16
isotropic Gaussians (sigma log-uniform in [1e-3, 1e-1], centres uniform in
[-1, 1]^2) plus 20 % of the points on the unit circle, charges N(0, 1),
Nequiv = 32, Ncutoff = 64, Laplace kernel, seeded synthetic data.

A step is the whole FMM on one point set, as the reference's FMM class runs it:
build_tree + precompute + build_expansions(tau) + evaluate_to_points(x, y, True).
`value` is Mpts/s with the inputs already in HBM (device pointers through the
C ABI); `e2e` is the same step through the public Python API with pinned host
buffers, host->device and device->host copies inside the timed region.
The relative error max|u - u_ref| / max|u_ref| is measured against an FP64
direct sum at 4,096 seeded sample targets.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun every rank runs an independent replica (the FMM does not shard);
value = all points processed / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Laplace FMM Mpts/s at N=1M, mixed vs plain at 1e-7 rel err; p50/p99 latency"
L2_FLUSH_BYTES = 256 << 20


# ------------------------------------------------------------ generators
def gen_uniform(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.standard_normal(n)


def gen_mixture(n, seed):
    rng = np.random.default_rng(seed)
    nc = int(0.2 * n)
    ng = n - nc
    th = rng.uniform(0, 2 * np.pi, nc)
    cx = rng.uniform(-1, 1, 16)
    cy = rng.uniform(-1, 1, 16)
    sig = 10 ** rng.uniform(-3, -1, 16)
    lab = rng.integers(0, 16, ng)
    x = np.concatenate([cx[lab] + sig[lab] * rng.standard_normal(ng), np.cos(th)])
    y = np.concatenate([cy[lab] + sig[lab] * rng.standard_normal(ng), np.sin(th)])
    return x, y, rng.standard_normal(n)


def gen_annulus(n, seed):
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0.25, 1, n))
    th = rng.uniform(0, 2 * np.pi, n)
    return r * np.cos(th), r * np.sin(th), rng.uniform(-1, 1, n)


CONFIGS = {
    "c1": dict(desc="uniform [-1,1]^2, N=20k, Nequiv 24, Ncutoff 64", gen=gen_uniform, n=20_000, neq=24, cut=64,
               kernel=0, k=0.0),
    "c2": dict(desc="Gaussian mixture + 20% unit circle, N=1M, Nequiv 32, Ncutoff 64", gen=gen_mixture,
               n=1_000_000, neq=32, cut=64, kernel=0, k=0.0),
    "c3": dict(desc="uniform [-1,1]^2, N=4M, Nequiv 32, Ncutoff 64", gen=gen_uniform, n=4_000_000, neq=32, cut=64,
               kernel=0, k=0.0),
    "c4": dict(desc="annulus 0.5<r<1, N=2M, K0 k=10, Nequiv 40, Ncutoff 48", gen=gen_annulus, n=2_000_000, neq=40,
               cut=48, kernel=1, k=10.0),
}


def kernel_obj(cfg):
    import pykifmm2d_b200 as P
    return P.LaplaceKernel() if cfg["kernel"] == 0 else P.ModifiedHelmholtzKernel(cfg["k"])


def make_fmm(cfg, x, y, precision, stream=None, m2l="auto", planned=False):
    import pykifmm2d_b200 as P
    kern = kernel_obj(cfg)
    return P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), cfg["neq"],
                 cfg["cut"], precision=precision, stream=stream, m2l=m2l, planned=planned)


def sample_targets(n):
    return np.random.default_rng(123).choice(n, min(n, 4096), replace=False)


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [v.strip() for v in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- our arm
def flush_l2(torch, buf):
    buf.zero_()


def time_full_steps(torch, cfg, xd, yd, td, precision, steps, warmup, flush, profile=False, m2l="auto"):
    """Full pipeline on device-resident inputs; returns per-step ms (CUDA events)."""
    from pykifmm2d_b200 import _lib as B
    stream = torch.cuda.Stream()  # the plan's own created stream (not the legacy default stream)
    f = make_fmm(cfg, xd, yd, precision, stream=stream.cuda_stream, m2l=m2l)
    f._bench_stream = stream
    out = torch.empty_like(xd)
    lib = B.load()
    times = []
    launches = 0
    phase = np.zeros(len(B.PHASES))
    for it in range(warmup + steps):
        timed = it >= warmup
        flush_l2(torch, flush)
        if timed and profile:
            lib.kifmm_set_profiling(f._plan, 1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = lib.kifmm_launch_count()
        a.record(stream)
        f.build_tree()
        f.precompute()
        f.build_expansions(td)
        f.evaluate_to_points(xd, yd, True, out=out)
        b.record(stream)
        torch.cuda.synchronize()
        if timed:
            times.append(a.elapsed_time(b))
            launches += lib.kifmm_launch_count() - l0
            if profile:
                ms = np.zeros(len(B.PHASES))
                lib.kifmm_get_phase_times(f._plan, ms.ctypes.data, None, 1)
                lib.kifmm_set_profiling(f._plan, 0)
                phase += ms
    return times, launches, phase / max(steps, 1), f, out


def leaf_alone_ms(torch, f, xd, yd, flush, reps=3):
    """Event-timed leaf phase (Taylor coefficients + the single-pass L2P + P2P
    kernel) of evaluations at the sources on the plan's current expansions."""
    from pykifmm2d_b200 import _lib as B
    lib = B.load()
    out = torch.empty_like(xd)
    vals = []
    for it in range(reps + 1):
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        lib.kifmm_set_profiling(f._plan, 1)
        f.evaluate_to_points(xd, yd, True, out=out)
        torch.cuda.synchronize()
        ms = np.zeros(len(B.PHASES))
        lib.kifmm_get_phase_times(f._plan, ms.ctypes.data, None, 1)
        lib.kifmm_set_profiling(f._plan, 0)
        if it:
            vals.append(float(ms[B.PHASES.index("leaf")]))
    return statistics.mean(vals)


def time_apply_steps(torch, f, xd, yd, td, steps, warmup, flush):
    stream = f._bench_stream
    out = torch.empty_like(xd)
    times = []
    for it in range(warmup + steps):
        flush_l2(torch, flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        f.build_expansions(td)
        f.evaluate_to_points(xd, yd, True, out=out)
        b.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            times.append(a.elapsed_time(b))
    return times


def time_e2e(torch, cfg, x, y, tau, precision, steps, warmup):
    """Through the public API with pinned host buffers (copies in the timed region)."""
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.from_numpy(y).pin_memory()
    tp = torch.from_numpy(tau).pin_memory()
    outp = torch.empty(x.size, dtype=torch.float64).pin_memory()
    times = []
    for it in range(warmup + steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = make_fmm(cfg, xp, yp, precision)
        f.build_tree()
        f.precompute()
        f.build_expansions(tp)
        f.evaluate_to_points(xp, yp, True, out=outp)
        t1 = time.perf_counter()
        del f
        if it >= warmup:
            times.append((t1 - t0) * 1e3)
    return times, outp.numpy().copy()


def rel_err(pot, ref, idx):
    return float(np.abs(pot[idx] - ref).max() / np.abs(ref).max())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return d, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def p2p_flops_per_pair(kernel):
    # Laplace: 2 sub, mul + fma for r^2, 1 lg2, 1 fma = 8 flops per pair;
    # modified Helmholtz: ~40 (sqrt + K0 series)
    return 8.0 if kernel == 0 else 40.0


def measured_traffic():
    """DRAM bytes per launch of the profiled kernels, from the committed ncu
    summary profiles/traffic_laplace_mixture_1m.txt (lines: kernel_name bytes)."""
    out = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", "traffic_laplace_mixture_1m.txt")):
            p = line.split()
            if len(p) == 2 and not line.startswith("#"):
                out[p[0]] = float(p[1])
    except OSError:
        pass
    return out


def build_rooflines(cfg, info, phase, precision, pk, pk_src, n):
    """Rooflines of the dominant kernel (the leaf L2P+P2P kernel), of the
    tensor-core M2L and of the Morton radix sort, from the phase timers
    (CUDA events on the plan's stream, averaged over the timed steps)."""
    from pykifmm2d_b200 import _lib as B
    ph = dict(zip(B.PHASES, phase))
    clk = pk.get("sm_max_mhz", 1965.0) * 1e6
    traffic = measured_traffic()
    out = {}
    fp32_peak = 148 * 128 * 2 * clk / 1e12          # TFLOP/s, FFMA = 2 flops
    fp64_peak = fp32_peak / 2
    pairs = float(info.n_p2p_pairs)
    fl = pairs * p2p_flops_per_pair(cfg["kernel"])
    t = ph["leaf"] * 1e-3
    if t > 0:
        peak = fp32_peak if precision == "mixed" else fp64_peak
        ach = fl / t / 1e12
        name = "k_leaf_eval_f" if precision == "mixed" else "k_leaf_eval_d"
        out["dominant"] = {
            "kernel": name + " (P2P + L2P, one launch per step)", "bound": "fp32" if precision == "mixed" else "fp64",
            "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "traffic": traffic.get(name),
            "work": f"{pairs:.4g} P2P pairs x {p2p_flops_per_pair(cfg['kernel']):.0f} flops per launch",
            "sfu_frac": (pairs / t) / (148 * 16 * clk),
            "peak_source": f"SIMT peak 148 SMs x 128 lanes x 2 flops at sm_max_mhz ({pk_src}); "
                           "sfu_frac = pairs/s over 16 lg2/clk/SM"}
    tm = ph["m2l"] * 1e-3
    if precision == "mixed" and tm > 0:
        Q = cfg["neq"]
        useful = 2.0 * Q * Q * float(info.n_m2l_pairs)
        int8_peak = 2 * pk["bf16_tflops"]
        ach = useful / tm / 1e12
        out["m2l"] = {"kernel": "k_m2l_tc<int8> (+ source slicing)", "bound": "tensor", "achieved": ach,
                      "peak": int8_peak, "unit": "TFLOP/s", "frac": ach / int8_peak,
                      "traffic": traffic.get("k_m2l_tc"),
                      "work": f"useful M2L flops 2 Q^2 x {info.n_m2l_pairs} V-list pairs; the int8 form "
                              "executes 15 slice products of the dense 4Qx4Q direction blocks",
                      "peak_source": f"dense int8 = 2 x measured bf16 {pk['bf16_tflops']} TFLOP/s ({pk_src})"}
    ts = ph["sort"] * 1e-3
    if ts > 0:
        byts = 52.0 * n  # algorithmic: read x, y, tau (24 B), write sorted x, y, tau and an i32 index (28 B)
        ach = byts / ts / 1e9
        out["sort"] = {"kernel": "Morton keys + onesweep radix sort (k_keys_dev, k_os_hist, k_os_pass)",
                       "bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                       "frac": ach / pk["hbm_gbs"], "traffic": traffic.get("k_os_pass"),
                       "work": "52 B per point: the algorithmic minimum of sorting the points (read x, y, tau; "
                               "write them sorted with an int32 index)",
                       "executed_bytes": 4 * 36.0 * n,
                       "peak_source": pk_src}
    out["composite"] = composite_roofline(cfg, info, ph, precision, pk, pk_src, n)
    return out


def composite_roofline(cfg, info, ph, precision, pk, pk_src, n):
    """t_ideal / t_measured over the phases of one step: each phase's
    algorithmic work at the peak of the unit that bounds it.
      P2P    pairs at the lg2 rate (16/clk/SM) for Laplace, 40 flops per pair
             at the FP32 peak for K0 (FP64 peak in the plain form);
      P2M    Q kernel evaluations per source point, L2P Q per point, 8 flops
             each at the FP32 peak (FP64 peak in the plain form);
      M2L    2 Q^2 per V-list pair at dense int8 (2 x measured bf16) in the
             mixed form, at the FP64 tensor rate (128 flops/clk/SM) in the plain one;
      M2M, L2L  2 Q (4Q) per split cell each way at the FP64 tensor rate;
      sort   52 B per point at the measured HBM bandwidth.
    t_measured is the sum of the same phases' event times."""
    clk = pk.get("sm_max_mhz", 1965.0) * 1e6
    fp32 = 148 * 128 * 2 * clk
    fp64 = fp32 / 2
    dmma = 148 * 128 * clk
    lg2 = 148 * 16 * clk
    Q = cfg["neq"]
    mixed = precision == "mixed"
    pairs = float(info.n_p2p_pairs)
    if cfg["kernel"] == 0 and mixed:
        t_p2p = pairs / lg2
    else:
        t_p2p = pairs * p2p_flops_per_pair(cfg["kernel"]) / (fp32 if mixed else fp64)
    evals = Q * float(info.n_p2m_points) + Q * float(n)
    t_p2m_l2p = evals * 8.0 / (fp32 if mixed else fp64)
    m2l_fl = 2.0 * Q * Q * float(info.n_m2l_pairs)
    t_m2l = m2l_fl / (2 * pk["bf16_tflops"] * 1e12) if mixed else m2l_fl / dmma
    n_split = max(0.0, (float(info.n_nodes) - 1) / 4)
    t_lvl = 2 * (2.0 * Q * 4 * Q * n_split) / dmma
    t_sort = 52.0 * n / (pk["hbm_gbs"] * 1e9)
    t_ideal = t_p2p + t_p2m_l2p + t_m2l + t_lvl + t_sort
    keys = ["tree", "p2m", "m2m", "m2l", "l2l", "leaf"]
    t_meas = sum(ph[k] for k in keys) * 1e-3
    return {"t_ideal_ms": t_ideal * 1e3, "t_measured_ms": t_meas * 1e3,
            "frac": t_ideal / t_meas if t_meas > 0 else None,
            "ideal_ms": {"p2p": t_p2p * 1e3, "p2m_l2p": t_p2m_l2p * 1e3, "m2l": t_m2l * 1e3,
                         "m2m_l2l": t_lvl * 1e3, "sort": t_sort * 1e3},
            "measured_phases": keys, "peak_source": pk_src}


def run_ours(args, cfg, rank, world, dist):
    import torch
    from pykifmm2d_b200 import _lib as B
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    x, y, tau = cfg["gen"](cfg["n"], 0)
    n = x.size
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    td = torch.from_numpy(tau).cuda()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    precision = args.precision
    lib = B.load()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    with ClockSampler(dev) as clk:
        times, launches, _, f, out = time_full_steps(torch, cfg, xd, yd, td, precision, args.steps, args.warmup,
                                                     flush, profile=False)
    barrier()
    clocks = clk.summary()
    # phase split from separate profiled steps (the timer events stay out of the timed steps)
    _, _, phase, _, _ = time_full_steps(torch, cfg, xd, yd, td, precision, 3, 1, flush, profile=True)
    # In a step the near field at the sources runs under the far-field chain,
    # sharing the SMs, so its phase time is not the kernel's own: the leaf
    # kernel alone (near + far field in one pass, a second evaluation on the
    # same expansions) is timed for the roofline.
    leaf_alone = leaf_alone_ms(torch, f, xd, yd, flush)
    tot = float(sum(times))
    if dist is not None:
        t = torch.tensor([tot], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = float(t.item())
    ms_step = tot / len(times)
    value = world * n / (ms_step * 1e-3) / 1e6
    info = f.tree_info()
    res = {}
    if rank == 0:
        # accuracy against the FP64 direct sum on the GPU (KAS)
        idx = sample_targets(n)
        import pykifmm2d_b200 as P
        KF, KA, KAS = P.Get_Kernel_Functions(kernel_obj(cfg))
        ref = np.zeros(idx.size)
        KAS(x, y, tau, ref, targets=idx)
        pot = out.cpu().numpy()
        res["err"] = rel_err(pot, ref, idx)
        # apply-only (tree and operators reused, repeated densities)
        at = time_apply_steps(torch, f, xd, yd, td, max(3, args.steps // 2), 2, flush)
        res["apply_ms"] = statistics.mean(at)
        # plain FP64 form for the mixed-vs-plain comparison
        if precision != "fp64":
            pt, _, _, fp, outp = time_full_steps(torch, cfg, xd, yd, td, "fp64", max(3, args.steps // 2), 2, flush)
            res["plain_ms"] = statistics.mean(pt)
            res["plain_err"] = rel_err(outp.cpu().numpy(), ref, idx)
            res["plain_apply_ms"] = statistics.mean(time_apply_steps(torch, fp, xd, yd, td, 3, 1, flush))
            del fp
            _, _, res["plain_phase"], _, _ = time_full_steps(torch, cfg, xd, yd, td, "fp64", 2, 1, flush,
                                                             profile=True)
            pe_t, pe_pot = time_e2e(torch, cfg, x, y, tau, "fp64", 5, 4)
            res["plain_e2e_ms"] = statistics.mean(pe_t)
            res["plain_e2e_err"] = rel_err(pe_pot, ref, idx)
        else:
            res["plain_ms"], res["plain_err"], res["plain_apply_ms"] = ms_step, res["err"], res["apply_ms"]
            res["plain_phase"] = phase
        # the first steps from freshly pinned buffers run ~20% slower: six untimed ones
        e2e_t, e2e_pot = time_e2e(torch, cfg, x, y, tau, precision, args.steps, max(args.warmup, 6))
        res["e2e_ms"] = statistics.mean(e2e_t)
        res["e2e_err"] = rel_err(e2e_pot, ref, idx)
        if precision == "fp64":
            res["plain_e2e_ms"], res["plain_e2e_err"] = res["e2e_ms"], res["e2e_err"]
        if args.extra_configs:
            res["c3_forms"] = run_c3_forms(torch, flush)
            res["c4"] = run_c4(torch, flush)
            res["planned"] = run_planned(torch, flush)
            res["next_rows"] = run_next_rows(torch, flush)
    if rank != 0:
        return None
    pk, pk_src = peaks()
    names = B.PHASES
    ph_roof = np.array(phase, dtype=float)
    ph_roof[names.index("leaf")] = leaf_alone
    rooflines = build_rooflines(cfg, info, ph_roof, precision, pk, pk_src, n)
    if "dominant" in rooflines:
        rooflines["dominant"]["timing"] = (
            "leaf kernel alone: event-timed single-pass evaluation at the sources on the step's expansions "
            f"({leaf_alone:.4f} ms, Taylor coefficients included); in the timed steps its near-field part runs "
            "on a low-priority stream under the far-field chain (phases_ms.leaf counts it there)")
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "Mpts/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded generator, seed 0)",
        "config": {"workload": cfg["desc"], "n_points": n, "kernel": "laplace" if cfg["kernel"] == 0 else "k0",
                   "nequiv": cfg["neq"], "ncutoff": cfg["cut"], "precision": precision,
                   "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) before every timed step",
                   "step": "build_tree + precompute + build_expansions + evaluate_to_points(check_self)"},
        "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99))},
        "rel_err": res["err"],
        "plain_fp64": {"ms_per_step": res["plain_ms"], "mpts_s": n / (res["plain_ms"] * 1e-3) / 1e6,
                       "rel_err": res["plain_err"], "apply_ms": res["plain_apply_ms"],
                       "phases_ms": {nm: float(v) for nm, v in zip(names, res["plain_phase"])},
                       "e2e": {"value": n / (res["plain_e2e_ms"] * 1e-3) / 1e6, "unit": "Mpts/s",
                               "ms_per_step": res["plain_e2e_ms"], "rel_err": res["plain_e2e_err"],
                               "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 8 * n},
                       "mixed_over_plain": {"step": res["plain_ms"] / ms_step,
                                            "e2e": res["plain_e2e_ms"] / res["e2e_ms"]}},
        "apply_only": {"ms": res["apply_ms"], "mpts_s": n / (res["apply_ms"] * 1e-3) / 1e6},
        "phases_ms": {nm: float(v) for nm, v in zip(names, phase)},
        "tree": {"levels": info.levels, "nodes": info.n_nodes, "leaves": info.n_leaves, "outside_root": info.n_outside,
                 "p2p_pairs": info.n_p2p_pairs},
        "roofline": rooflines["dominant"],
        "roofline_tensor_m2l": rooflines.get("m2l"),
        "roofline_hbm_sort": rooflines.get("sort"),
        "roofline_composite": rooflines.get("composite"),
        "e2e": {"value": n / (res["e2e_ms"] * 1e-3) / 1e6, "unit": "Mpts/s",
                "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 8 * n, "ms_per_step": res["e2e_ms"],
                "rel_err": res["e2e_err"]},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    for k in ("c3_forms", "c4", "planned", "next_rows"):
        if k in res:
            line[k] = res[k]
    if args.serve_requests > 0:
        line["serving"] = run_serving(args, dev)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, x, y, tau, repeats=3)
        line["cpu_baseline_numba_reference"] = numba_reference_baseline(cfg, x, y, tau)
    return line


# ------------------------------------------- extra configurations (same run)
def _direct_ref(cfg, x, y, tau, idx):
    import pykifmm2d_b200 as P
    KF, KA, KAS = P.Get_Kernel_Functions(kernel_obj(cfg))
    ref = np.zeros(idx.size)
    KAS(x, y, tau, ref, targets=idx)
    return ref


def _form_line(torch, cfg, xd, yd, td, flush, precision, m2l, ref, idx, steps=3, warmup=2):
    times, launches, _, f, out = time_full_steps(torch, cfg, xd, yd, td, precision, steps, warmup, flush, m2l=m2l)
    _, _, phase, _, _ = time_full_steps(torch, cfg, xd, yd, td, precision, 2, 1, flush, profile=True, m2l=m2l)
    from pykifmm2d_b200 import _lib as B
    ms = statistics.mean(times)
    err = rel_err(out.cpu().numpy(), ref, idx)
    return {"precision": precision, "m2l": m2l, "ms_per_step": ms, "mpts_s": xd.numel() / (ms * 1e-3) / 1e6,
            "rel_err": err, "meets_1e-7": err <= 1e-7, "meets_1e-5": err <= 1e-5,
            "phases_ms": {nm: float(v) for nm, v in zip(B.PHASES, phase)}}, f


def run_c3_forms(torch, flush):
    """Precision forms on the 4M uniform cloud (Nequiv 32): each M2L form of
    the mixed precision (FP32 near field) and the plain FP64 form, with the
    max relative error at 4,096 seeded targets against the FP64 direct sum."""
    cfg = CONFIGS["c3"]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    idx = sample_targets(x.size)
    ref = _direct_ref(cfg, x, y, tau, idx)
    xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
    forms = {}
    for name, precision, m2l in (("int8", "mixed", "int8"), ("bf16x3", "mixed", "bf16x3"),
                                 ("fp16x3", "mixed", "fp16x3"), ("fp32", "mixed", "fp32"),
                                 ("fp64_plain", "fp64", "auto")):
        forms[name], f = _form_line(torch, cfg, xd, yd, td, flush, precision, m2l, ref, idx)
        del f
    return {"workload": cfg["desc"], "n_points": x.size, "targets": int(idx.size),
            "error": "max |u - u_direct| / max |u_direct| at 4,096 seeded targets, FP64 direct sum on the GPU",
            "forms": forms,
            "meet_1e-7": sorted(k for k, v in forms.items() if v["meets_1e-7"]),
            "meet_1e-5": sorted(k for k, v in forms.items() if v["meets_1e-5"])}


def run_c4(torch, flush):
    """Modified Helmholtz K0 (k = 10) on the 2M annulus (Nequiv 40, Ncutoff
    48): mixed and plain forms, error at 4,096 targets against the FP64 direct
    sum, and the K0 near-field kernel against the FP32 peak at 40 flops per
    pair."""
    cfg = CONFIGS["c4"]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    idx = sample_targets(x.size)
    ref = _direct_ref(cfg, x, y, tau, idx)
    xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
    out = {"workload": cfg["desc"], "n_points": x.size}
    pk, pk_src = peaks()
    for name, precision in (("mixed", "mixed"), ("plain_fp64", "fp64")):
        line, f = _form_line(torch, cfg, xd, yd, td, flush, precision, "auto", ref, idx)
        info = f.tree_info()
        out[name] = line
        if precision == "mixed":
            clk = pk.get("sm_max_mhz", 1965.0) * 1e6
            peak = 148 * 128 * 2 * clk / 1e12
            t = line["phases_ms"]["leaf"] * 1e-3
            ach = float(info.n_p2p_pairs) * 40.0 / t / 1e12 if t > 0 else None
            out["roofline_k0_p2p"] = {
                "kernel": "k_leaf_eval_f<K0> (P2P + L2P)", "bound": "fp32", "achieved": ach, "peak": peak,
                "unit": "TFLOP/s", "frac": ach / peak if ach else None,
                "work": f"{info.n_p2p_pairs} P2P pairs x 40 flops (K0 series) per launch",
                "peak_source": f"SIMT peak at sm_max_mhz ({pk_src})"}
            out["tree"] = {"levels": info.levels, "nodes": info.n_nodes, "p2p_pairs": info.n_p2p_pairs,
                           "m2l_pairs": info.n_m2l_pairs}
        del f
    out["mixed_over_plain"] = out["plain_fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def run_planned(torch, flush, steps=5):
    """Planned applies (the reference's fmm_planner / planned_fmm): repeated
    densities on one tree with the P2M, L2P and near-field kernel values kept
    in HBM, against the same applies on the fly; per workload and precision:
    the apply (build_expansions + evaluate_to_points at the sources) in ms,
    the one-time matrix build, the matrices' bytes and the planned leaf
    kernel's bytes per second against the measured HBM bandwidth."""
    import pykifmm2d_b200 as P
    from pykifmm2d_b200 import _lib as B
    pk, pk_src = peaks()
    lib = B.load()
    out = {}
    for cname in ("c2", "c4"):
        cfg = CONFIGS[cname]
        x, y, tau = cfg["gen"](cfg["n"], 0)
        xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
        res = {"workload": cfg["desc"]}
        for precision in ("mixed", "fp64"):
            line = {}
            for planned in (False, True):
                stream = torch.cuda.Stream()
                f = make_fmm(cfg, xd, yd, precision, stream=stream.cuda_stream, planned=planned)
                f._bench_stream = stream
                f.build_tree()
                f.precompute()
                o = torch.empty_like(xd)
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                f.build_expansions(td)  # planned: builds the matrices
                f.evaluate_to_points(xd, yd, True, out=o)
                b.record(stream)
                torch.cuda.synchronize()
                first = a.elapsed_time(b)
                ms = statistics.mean(time_apply_steps(torch, f, xd, yd, td, steps, 2, flush))
                lib.kifmm_set_profiling(f._plan, 1)
                f.build_expansions(td)
                f.evaluate_to_points(xd, yd, True, out=o)
                ph = np.zeros(len(B.PHASES))
                lib.kifmm_get_phase_times(f._plan, ph.ctypes.data, None, 1)
                lib.kifmm_set_profiling(f._plan, 0)
                ph = dict(zip(B.PHASES, ph))
                info = f.tree_info()
                key = "planned" if planned else "on_the_fly"
                line[key] = {"apply_ms": ms, "mpts_s": x.size / (ms * 1e-3) / 1e6, "first_apply_ms": first,
                             "leaf_ms": ph["leaf"], "p2m_ms": ph["p2m"]}
                if planned:
                    nb = 4 if precision == "mixed" else 8
                    leaf_bytes = float(info.n_p2p_pairs) * nb + 8.0 * cfg["neq"] * x.size + 24.0 * x.size
                    ach = leaf_bytes / (ph["leaf"] * 1e-3) / 1e9 if ph["leaf"] > 0 else None
                    line[key].update({"matrix_bytes": int(info.planned_bytes),
                                      "roofline_leaf": {"kernel": "k_planned_leaf (L2P + near field as matrices)",
                                                        "bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"],
                                                        "unit": "GB/s", "frac": ach / pk["hbm_gbs"] if ach else None,
                                                        "work": f"{nb} B per near-field pair + 8 Q B per point "
                                                                "(L2P block) + charges and potentials",
                                                        "peak_source": pk_src}})
                del f
            line["speedup"] = line["on_the_fly"]["apply_ms"] / line["planned"]["apply_ms"]
            res[precision] = line
        out[cname] = res
    return out


def _timed(torch, stream, flush, fn, steps=5, warmup=2):
    """ms per call of fn() on `stream` (CUDA events, L2 flushed before each)."""
    ts = []
    for it in range(warmup + steps):
        flush_l2(torch, flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            ts.append(a.elapsed_time(b))
    return statistics.mean(ts)


def run_next_rows(torch, flush):
    """The rows beside the path, each with its error at 4,096 seeded targets
    against the FP64 direct sum on the GPU:
    * separate targets (evaluate_to_points(x, y, check_self=False), the
      reference's laplace2.py use): 10M uniform targets from the 1M mixture plan;
    * complex values (FMM(..., iscomplex=True), the reference's hankel.py):
      Helmholtz (i/4) H0(k r), k = 2, 1M uniform points, Nequiv 24, Ncutoff 50,
      complex N(0,1) densities, FP64;
    * circulant E2C (the FFT solve of svd_fmm.py) on the K0 annulus, whose
      operators differ per level: precompute and full step against the dense
      inverse."""
    import pykifmm2d_b200 as P
    from pykifmm2d_b200 import _lib as B
    lib = B.load()
    out = {}
    # separate targets
    cfg = CONFIGS["c2"]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        f = make_fmm(cfg, xd, yd, "mixed", stream=stream.cuda_stream)
        f.build_tree()
        f.precompute()
        f.build_expansions(td)
        nt = 10_000_000
        rng = np.random.default_rng(7)
        tx, ty = rng.uniform(-1, 1, nt), rng.uniform(-1, 1, nt)
        txd, tyd = torch.from_numpy(tx).cuda(), torch.from_numpy(ty).cuda()
        o = torch.empty(nt, dtype=torch.float64, device="cuda")
        ms = _timed(torch, stream, flush, lambda: f.evaluate_to_points(txd, tyd, False, out=o))
        idx = np.random.default_rng(123).choice(nt, 4096, replace=False)
        ref = np.zeros(idx.size)
        P.Get_Kernel_Functions(kernel_obj(cfg))[1](x, y, tx[idx], ty[idx], tau, ref)
        got = o.cpu().numpy()[idx]
        out["separate_targets"] = {
            "workload": f"{cfg['desc']}; {nt} targets uniform in [-1,1]^2, check_self=False",
            "precision": "mixed", "evaluate_ms": ms, "mtargets_s": nt / (ms * 1e-3) / 1e6,
            "rel_err": float(np.abs(got - ref).max() / np.abs(ref).max())}
        del f
    # complex Helmholtz
    n = 1_000_000
    rng = np.random.default_rng(0)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    tau = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    xd, yd, td = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), torch.from_numpy(tau).cuda()
    H0 = P.HelmholtzKernel(2.0)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        oc = torch.empty(n, dtype=torch.complex128, device="cuda")

        def step():
            g = P.FMM(xd, yd, P.Get_Kernel_Functions(H0), P.prepare_numba_functions_on_the_fly(H0), 24, 50, True,
                      stream=stream.cuda_stream)
            g.build_tree()
            g.precompute()
            g.build_expansions(td)
            g.evaluate_to_points(xd, yd, True, out=oc)
            step.g = g
        ms = _timed(torch, stream, flush, step, steps=3)
        g = step.g
        ams = _timed(torch, stream, flush, lambda: (g.build_expansions(td), g.evaluate_to_points(xd, yd, True, out=oc)),
                     steps=3)
        idx = sample_targets(n)
        ref = np.zeros(idx.size, dtype=np.complex128)
        P.Get_Kernel_Functions(H0)[2](x, y, tau, ref, targets=idx)
        got = oc.cpu().numpy()[idx]
        out["complex_helmholtz"] = {
            "workload": "Helmholtz (i/4) H0(k r), k = 2, N = 1M uniform in [-1,1]^2, Nequiv 24, Ncutoff 50, "
                        "complex N(0,1) densities", "precision": "fp64 (complex)", "ms_per_step": ms,
            "mpts_s": n / (ms * 1e-3) / 1e6, "apply_ms": ams,
            "rel_err": float(np.abs(got - ref).max() / np.abs(ref).max())}
        del g, step.g
    # circulant E2C
    cfg = CONFIGS["c4"]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
    idx = sample_targets(x.size)
    ref = _direct_ref(cfg, x, y, tau, idx)
    kern = kernel_obj(cfg)
    res = {"workload": cfg["desc"]}
    for e2c in ("dense", "circulant"):
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            oo = torch.empty_like(xd)

            def full():
                h = P.FMM(xd, yd, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern),
                          cfg["neq"], cfg["cut"], precision="mixed", stream=stream.cuda_stream, e2c=e2c)
                h.build_tree()
                h.precompute()
                h.build_expansions(td)
                h.evaluate_to_points(xd, yd, True, out=oo)
                full.h = h
            ms = _timed(torch, stream, flush, full, steps=3)
            h = full.h
            info = np.zeros(len(B.PHASES))
            lib.kifmm_set_profiling(h._plan, 1)
            h.precompute()  # the operators again, timed by the plan's phase events
            lib.kifmm_get_phase_times(h._plan, info.ctypes.data, None, 1)
            lib.kifmm_set_profiling(h._plan, 0)
            ph = dict(zip(B.PHASES, info))
            res[e2c] = {"ms_per_step": ms, "mpts_s": x.size / (ms * 1e-3) / 1e6,
                        "operators_ms": float(ph["operators"] + ph["precompute"]),
                        "rel_err": rel_err(oo.cpu().numpy(), ref, idx)}
            del h, full.h
    out["circulant_e2c"] = res
    return out


# ------------------------------------------------------- serving stream
def run_serving(args, device):
    """Mixed-size request stream through pykifmm2d_b200.serving: first all
    requests at once (closed system) to measure capacity, then the same
    requests with Poisson arrivals at 70% of that rate; latency per request =
    completion - arrival (tree build, operators, every density's host->device
    copy, graph replay and device->host copy)."""
    from pykifmm2d_b200 import serving as S
    srv = S.Server(device=device, slots=args.serve_slots, keep_pots=False)
    srv.run(S.make_stream(4, 0.0, seed=99, nmax=20_000, applies=(2, 2)), realtime=False)  # warm-up
    _, cap = srv.run(S.make_stream(args.serve_requests, 0.0, seed=0), realtime=False)
    rate = 0.7 * cap["requests_per_s"]
    _, st = srv.run(S.make_stream(args.serve_requests, rate, seed=0), realtime=True)
    srv.close()
    out = {
        "requests": st["requests"], "failed": st["failed"] + cap["failed"],
        "mix": "70% Laplace / 30% K0 (k in {1,10,50}), N log-uniform in [1e3, 3e5] (mixture + circle points), "
               "8-32 fresh N(0,1) densities per request (drawn on the device), Nequiv 32, Ncutoff 64",
        "batched_mixed": {"precision": "mixed", "slots": st["slots"], "graphs": True,
                          "capacity_requests_per_s": cap["requests_per_s"],
                          "capacity_mpts_s": cap["point_applies_per_s"] / 1e6, "offered_requests_per_s": rate,
                          "offered_load": 0.7, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                          "mean_ms": st["mean_ms"], "point_applies_per_s": st["point_applies_per_s"],
                          "mpts_s": st["point_applies_per_s"] / 1e6, "wall_s": st["wall_s"]},
        "hbm_budget_bytes": st["hbm_budget_bytes"],
    }
    if args.serve_packed_slots > 0:
        # the same requests and arrival times through the packed batches: every
        # step one graph launch over all admitted requests, their M2L in one
        # tensor-core launch and their near fields in one launch per kernel kind
        pk = S.Server(device=device, slots=args.serve_packed_slots, keep_pots=False, packed=True)
        pk.run(S.make_stream(4, 0.0, seed=99, nmax=20_000, applies=(2, 2)), realtime=False)  # warm-up
        _, pcap = pk.run(S.make_stream(args.serve_requests, 0.0, seed=0), realtime=False)
        _, ps = pk.run(S.make_stream(args.serve_requests, rate, seed=0), realtime=True)
        pk.close()
        out["failed"] += pcap["failed"] + ps["failed"]
        out["packed_mixed"] = {"precision": "mixed", "slots": ps["slots"], "graphs": True, "packed": True,
                               "capacity_requests_per_s": pcap["requests_per_s"],
                               "capacity_mpts_s": pcap["point_applies_per_s"] / 1e6,
                               "offered_requests_per_s": rate, "p50_ms": ps["p50_ms"], "p99_ms": ps["p99_ms"],
                               "mean_ms": ps["mean_ms"], "mpts_s": ps["point_applies_per_s"] / 1e6,
                               "wall_s": ps["wall_s"], "steps": ps["steps"], "captures": ps["captures"],
                               "mean_batch": ps["mean_batch"]}
    if args.serve_plain:
        # the same requests and arrival times, one at a time, plain FP64, no graphs
        plain = S.Server(device=device, slots=1, keep_pots=False, precision="fp64", graphs=False)
        _, sp = plain.run(S.make_stream(args.serve_requests, rate, seed=0), realtime=True)
        plain.close()
        out["failed"] += sp["failed"]
        out["one_at_a_time_plain"] = {"precision": "fp64", "slots": 1, "graphs": False,
                                      "offered_requests_per_s": rate, "p50_ms": sp["p50_ms"],
                                      "p99_ms": sp["p99_ms"], "mean_ms": sp["mean_ms"],
                                      "point_applies_per_s": sp["point_applies_per_s"],
                                      "mpts_s": sp["point_applies_per_s"] / 1e6, "wall_s": sp["wall_s"]}
    return out


# ------------------------------------------------------- CPU baseline
def cpu_baseline(cfg, x, y, tau, repeats=3, threads=None):
    """The oracle (C restatement of the reference, OpenMP) on the host cores."""
    from oracle import oracle as O
    nthr = threads or os.cpu_count()
    O.set_threads(nthr)
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        f = O.OracleFMM(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
        f.build_expansions(tau)
        f.evaluate_to_points(x, y, True)
        ts.append(time.perf_counter() - t0)
        del f
    med = statistics.median(ts)
    cpu = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": x.size / med / 1e6, "unit": "Mpts/s", "cores": nthr, "kind": "port",
            "sample": f"full workload ({x.size} points), median of {repeats} runs, {med:.2f} s each; CPU: {cpu}"}


def numba_reference_baseline(cfg, x, y, tau, repeats=2):
    """The reference's own numba path (class_fmm.FMM with its i8[4] import
    shim) from baseline/_ref, timed on all host cores in a subprocess; a second
    CPU number beside the oracle port (which stays the reference arm)."""
    ref = os.path.join(ROOT, "baseline", "_ref", "pykifmm2d", "class_fmm.py")
    if not os.path.exists(ref):
        return {"unavailable": "baseline/_ref (pip install of the reference) is not present"}
    if cfg["kernel"] != 0:
        return {"unavailable": "timed for the Laplace workload only"}
    try:
        import numba  # noqa: F401
    except Exception:
        return {"unavailable": "numba is not importable on this host"}
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    try:
        np.savez(path, x=x, y=y, tau=tau)
        env = dict(os.environ, NUMBA_NUM_THREADS=str(os.cpu_count()))
        out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "run_reference_numba.py"), path,
                              str(cfg["neq"]), str(cfg["cut"]), str(repeats)], capture_output=True, text=True,
                             env=env, timeout=900)
        line = [l for l in out.stdout.splitlines() if l.startswith("{")]
        if not line:
            return {"unavailable": "reference run failed: " + out.stderr.strip()[-300:]}
        d = json.loads(line[-1])
    finally:
        os.unlink(path)
    return {"value": x.size / d["seconds"] / 1e6, "unit": "Mpts/s", "cores": d["threads"], "kind": "reference",
            "sample": f"the reference's class_fmm.FMM (numba {d['numba']}, import shim i8[4] -> i8[:]) on the full "
                      f"workload ({x.size} points), build_tree + precompute + build_expansions + "
                      f"evaluate_to_points(check_self), JIT warmed on 5,000 points, median of {len(d['runs'])} runs "
                      f"({d['seconds']:.2f} s each)"}


def run_reference(args, cfg):
    x, y, tau = cfg["gen"](cfg["n"], 0)
    from oracle import oracle as O
    nthr = os.cpu_count()
    O.set_threads(nthr)
    ts = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        f = O.OracleFMM(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
        f.build_expansions(tau)
        f.evaluate_to_points(x, y, True)
        dt = time.perf_counter() - t0
        del f
        if it >= args.warmup:
            ts.append(dt)
    ms = 1e3 * statistics.mean(ts)
    v = x.size / (ms * 1e-3) / 1e6
    return {
        "metric": METRIC, "value": v, "unit": "Mpts/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator, seed 0)", "impl": "reference",
        "config": {"workload": cfg["desc"], "n_points": x.size, "kernel": "laplace" if cfg["kernel"] == 0 else "k0",
                   "nequiv": cfg["neq"], "ncutoff": cfg["cut"], "precision": "fp64",
                   "parallelism": "host threads (rank 0 only)", "l2": "n/a (CPU)",
                   "step": "build_tree + precompute + build_expansions + evaluate_to_points(check_self)"},
        "latency_ms": {"p50": float(np.percentile(ts, 50)) * 1e3, "p99": float(np.percentile(ts, 99)) * 1e3},
        "cpu_baseline": {"value": v, "unit": "Mpts/s", "cores": nthr, "kind": "port",
                         "sample": f"full workload ({x.size} points) per step; the reference is pure Python + "
                                   "numba, so its algorithm runs as the C/OpenMP restatement in oracle/"},
        "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="only the timed pipeline steps (for ncu launch lists); prints phase times")
    ap.add_argument("--n", type=int, default=0, help="override the number of points (profiling small cases)")
    ap.add_argument("--serve-requests", type=int, default=1024,
                    help="requests in the serving stream (0 skips it)")
    ap.add_argument("--serve-slots", type=int, default=32,
                    help="concurrent requests in the serving stream (one stream and graph each)")
    ap.add_argument("--serve-packed-slots", type=int, default=64,
                    help="requests per packed batch in the packed serving run (0 skips it)")
    ap.add_argument("--no-serve-plain", dest="serve_plain", action="store_false",
                    help="skip the one-at-a-time plain-FP64 run of the serving stream")
    ap.add_argument("--no-extra-configs", dest="extra_configs", action="store_false",
                    help="skip the 4M-point M2L-form comparison and the 2M-point K0 annulus")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.n:
        cfg["n"] = args.n
        cfg["desc"] += f" (N overridden to {args.n})"
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.profile_run:
        import torch
        from pykifmm2d_b200 import _lib as B
        x, y, tau = cfg["gen"](cfg["n"], 0)
        xd, yd, td = (torch.from_numpy(v).cuda() for v in (x, y, tau))
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        times, launches, phase, _, _ = time_full_steps(torch, cfg, xd, yd, td, args.precision, args.steps,
                                                       args.warmup, flush, profile=True)
        print(json.dumps({"ms_per_step": statistics.mean(times), "launches_per_step": launches / args.steps,
                          "phases_ms": {nm: float(v) for nm, v in zip(B.PHASES, phase)}}))
        return 0
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, cfg)), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        line = run_ours(args, cfg, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
