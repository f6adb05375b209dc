"""Benchmark of the Wilson hopping matrix on B200 (one JSON line on rank 0).

Workload: FP64 Wilson hopping matrix H on a 32^3x64 lattice (random SU(3)
links, Gaussian spinor), the reference's single-device benchmark size. One
step = one full-lattice application H = (H_eo, H_oe), which the reference's
driver times as an eo+oe pair of calls (tests/test_hopping.c:291-301).
GFLOP/s use 1320 flop per output site.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value     : device-resident full-lattice kernel, inputs in HBM, CUDA events.
e2e       : the reference-facing C-ABI (plqcd_hopping_matrix_eo/oe on host
            arrays from amalloc'd pinned memory), host<->device copies of each
            call's input and output parity inside the timed region.
roofline  : the dominant kernel's algorithmic bytes / launch time against the
            measured HBM copy bandwidth.
cpu_baseline / --impl reference: the reference's own plain-C OpenMP hopping
            pair compiled from its sources (oracle/_ref), on the host cores.

Multi-GPU (torchrun): independent replicas, one lattice per GPU, no
collective on the data path; barrier + max over ranks for the timing.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_BENCH = (32, 32, 32, 64)
FLOP_PER_SITE = 1320
# algorithmic (compulsory) bytes per output site
BYTES_PARITY = {0: 192 + 8 * 144 + 192, 1: 96 + 8 * 72 + 96}        # F64 / F32, 18-real, one parity
BYTES_FULL = {0: 192 + 4 * 144 + 192, 1: 96 + 4 * 72 + 96}          # full lattice: each link read once
BYTES_F32_12 = 96 + 8 * 48 + 96
BYTES_HALF_12 = 52 + 8 * 24 + 52
# DRAM bytes (read + write) per site of one full-lattice F64 launch at 32^3x64,
# from single-pass ncu captures of each configuration
# (profiles/dslash_full_f64_dram_32x32x32x64.txt): variant -> bytes/site.
# Variant 2 is the cp.async kernel, 1000*kind + 100*stages + rows a TMA kernel
# (kind 1: a stage per direction; 2-5: own-line rows staged once per tile).
# 2216 is captured with the full-lattice default tile order (blocks of half
# the z extent x all t-slices), the others with the earlier 8 x 8 (z, t)
# blocks.
DRAM_BYTES_PER_SITE_F64_FULL = {
    2: 2127234136 / 2097152, 1204: 2191090112 / 2097152, 2204: 2253279192 / 2097152,
    4304: 2204120856 / 2097152, 1304: 2527646688 / 2097152, 1408: 2198568976 / 2097152,
    2216: (1778083584 + 387864064) / 2097152,
}


def dram_bytes_per_site(cfg):
    """ncu DRAM bytes per site of the full-lattice F64 configuration `cfg`,
    or None when that configuration has no capture."""
    v = 2 if cfg is None else cfg[0]
    return DRAM_BYTES_PER_SITE_F64_FULL.get(v)


def traffic_bytes(cfg, V):
    b = dram_bytes_per_site(cfg)
    return None if b is None else round(b * V)


def traffic_note(cfg, L) -> str:
    """Where roofline.traffic comes from: not measured in this run."""
    if dram_bytes_per_site(cfg) is None:
        return "no ncu capture of this configuration (see profiles/ for the captured ones)"
    return ("ncu dram bytes (read + write) of one launch of this configuration at 32^3x64, taken from the "
            "single-pass capture in profiles/dslash_full_f64_dram_32x32x32x64.txt, not measured in this run"
            + ("" if tuple(L) == (32, 32, 32, 64) else "; scaled by sites"))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

class Dist:
    """Replica bookkeeping: one process per GPU, no collective on the data
    path; only the timing uses a barrier and a max over ranks."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cuda"

    def init(self, backend="nccl"):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist
            self.device = "cuda" if backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        if not sm:
            return None
        busy = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref): the reference's own plain-C OpenMP pair
# ---------------------------------------------------------------------------

def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_reference_time(L, qin, u, steps: int, warmup: int, budget_s: float | None):
    """Seconds per full H (eo+oe) of the compiled reference, from its own
    return values (lib/dirac.c:405-407): the best of the sampled pairs after
    the warm-up, as the reference's own timing loop reports its best
    (tests/test_hopping.c:291-330). Returns (best_sec, mean_sec, steps_run,
    threads, kind)."""
    from oracle import oracle as O
    nthr = host_threads()
    try:
        ref = O.CompiledReference("patched")
        kind = "reference"
    except FileNotFoundError:
        ref = None
        kind = "port"
    out = np.zeros_like(qin)
    R = None if ref is not None else O.Restatement()

    def one():
        if ref is not None:
            return ref.hop("full", L, qin, u, out, nthreads=nthr)[1]
        t0 = time.perf_counter()
        R.hop("full", L, qin, u, nthreads=nthr)
        return time.perf_counter() - t0

    for _ in range(warmup):
        one()
    ts = []
    t_start = time.time()
    while len(ts) < steps and (budget_s is None or time.time() - t_start < budget_s or not ts):
        ts.append(one())
    return min(ts), sum(ts) / len(ts), len(ts), nthr, kind


def host_fields(L, seed):
    """API-layout host fields (qin, u) generated on the host with numpy."""
    from oracle import oracle as O
    V = O.volume(L)
    rng = np.random.default_rng(seed)
    return O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)


def run_reference(args, d: Dist):
    """--impl reference: the reference's CPU implementation of the path."""
    if d.rank != 0:
        return 0
    L = L_BENCH
    V = int(np.prod(L))
    qin, u = host_fields(L, 1234)
    # bounded sample: at most args.steps pairs and about a minute of CPU time
    sec, mean, n, nthr, kind = cpu_reference_time(L, qin, u, args.steps, args.warmup, 60.0)
    gflops = V * FLOP_PER_SITE / sec / 1e9
    line = {
        "impl": "reference", "metric": "Dslash GFLOP/s", "value": round(gflops, 3), "unit": "GFLOP/s",
        "n_gpus": args.gpus, "steps": n, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (random SU(3) links, Gaussian spinor)",
        "config": {"workload": "FP64 Wilson hopping matrix, full lattice (eo+oe), 32^3x64",
                   "lattice": list(L), "flop_per_site": FLOP_PER_SITE},
        "cpu_baseline": {"value": round(gflops, 3), "unit": "GFLOP/s", "cores": nthr, "kind": kind,
                         "sample": f"best of {n} full-lattice applications (eo+oe) at 32^3x64 after "
                                   f"{args.warmup} warm-up, times from the reference's own return values "
                                   f"(mean {V * FLOP_PER_SITE / mean / 1e9:.2f} GFLOP/s)"},
        "e2e": {"value": round(gflops, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def tuned_config(P, pattern: str):
    """(variant, block) the autotuner chose for the first cache key that
    contains `pattern`, or None."""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "tune.json")
        if P.lib().plqcd_tune_save(path.encode()) != 0 or not os.path.exists(path):
            return None
        for line in open(path):
            try:
                e = json.loads(line)
            except ValueError:
                continue
            if pattern in e.get("key", ""):
                return e["variant"], e["block"]
    return None


def kernel_name(cfg) -> str:
    """Name of the hopping kernel a (variant, block) configuration runs."""
    if cfg is None:
        return "k_dslash_pipe<F64,18,full>"
    v, b = cfg
    if v >= 2000:
        kind = v // 1000
        own = kind - 1 if kind <= 3 else kind - 3
        form = ", one box per stage" if kind >= 4 else ""
        return (f"k_dslash_tma_xy<F64,18> ({own} own-line + {(v // 100) % 10} ring buffers{form}, "
                f"{v % 100} rows per tile, full lattice)")
    if v >= 1000:
        return f"k_dslash_tma<F64,18> ({(v // 100) % 10} stages, {v % 100} rows per tile, full lattice)"
    if v in (2, 3):
        return f"k_dslash_pipe<F64,18,full> (depth {v}, block {b})"
    return f"k_dslash<F64,18,full> (block {b})"


def time_kernel(torch, fn, steps: int, warmup: int, d: Dist | None = None):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if d:
        d.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    if d:
        d.barrier()
    return e0.elapsed_time(e1)


def run_ours(args, d: Dist):
    import torch

    import plqcd_b200 as P
    torch.cuda.set_device(d.local)
    hbm, peak_kind = measured_peaks()
    L = args.lattice
    lat = P.Lattice(L, d.local, torch.cuda.current_stream().cuda_stream)
    V, Vh = lat.V, lat.Vh

    def buf(prec):
        return torch.empty(lat.spinor_bytes(prec), dtype=torch.uint8, device="cuda")

    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(1234 + d.rank)
    fe, fo, oe_, oo_ = buf(P.F64), buf(P.F64), buf(P.F64), buf(P.F64)
    lat.spinor_gaussian(fe, P.F64, 0, 77 + d.rank)
    lat.spinor_gaussian(fo, P.F64, 1, 77 + d.rank)

    K, W = args.steps, args.warmup
    if args.only == "sharded":  # the t-slab decomposition held on one device
        res = run_sharded(torch, P, lat, g64, fe, fo, args)
        if d.rank == 0:
            print(json.dumps({"only": "sharded", "sharded": res}))
        return 0
    if args.only == "mrhs":  # the multi-RHS kernels alone (profiling runs)
        res = run_mrhs(torch, P, lat, g64, args, args.mrhs_nrhs)
        if d.rank == 0:
            print(json.dumps({"only": "mrhs", "lattice": list(L), "mrhs_dslash": res}))
        return 0
    if args.only == "batch":  # the batched multi-RHS solve alone, against one FP64 CG solve
        be, bo, xe, xo = buf(P.F64), buf(P.F64), buf(P.F64), buf(P.F64)
        lat.spinor_gaussian(be, P.F64, 0, 4242)
        lat.spinor_gaussian(bo, P.F64, 1, 4242)
        prm = P.cg_param(kappa=0.12, tol=1e-10)
        P.invert_cg(lat, g64, None, xe, xo, be, bo, P.cg_param(kappa=0.12, tol=1e-10, max_iter=4),
                    raise_on_error=False)
        f64s = sorted(P.invert_cg(lat, g64, None, xe, xo, be, bo, prm).seconds for _ in range(3))[1]
        del be, bo, xe, xo
        res = run_batch(torch, P, d, args, f64s)
        if d.rank == 0:
            print(json.dumps({"only": "batch", "delta": args.delta, "f64_cg_seconds": f64s, "batch": res}))
        return 0
    if args.only == "cg":  # profiling runs of the solver section alone
        cg = run_cg(torch, P, lat, g64, buf, args)
        if d.rank == 0:
            print(json.dumps({"only": "cg", "cg": cg}))
        return 0

    # ---- headline: full lattice H, FP64, device resident ------------------
    full = lambda: lat.dslash_full(g64, oe_, oo_, fe, fo, P.F64)
    clk = ClockSampler(d.local)
    clk.start()
    ms = time_kernel(torch, full, K, W, d)
    clocks = clk.stop()
    ms_max = d.max(ms)
    t_step = ms_max / 1e3 / K
    head_cfg = tuned_config(P, f"dslash|p{P.F64}|r18|full|{'x'.join(map(str, L))}|")
    if os.environ.get("PLQCD_DSLASH_FULL_STAGES"):  # forced (profiling runs)
        head_cfg = (int(os.environ["PLQCD_DSLASH_FULL_STAGES"]), 0)
    value = d.world * V * FLOP_PER_SITE / t_step / 1e9
    achieved = V * BYTES_FULL[0] / t_step / 1e9
    sustained = run_sustained(torch, full, t_step, V, hbm, d, args) if args.sustained_s > 0 else None

    # ---- per-parity kernels (the drop-in and solver building block) ---------
    Kp = K if args.only == "dslash" else max(10, K // 2)
    eo = lambda: lat.dslash(g64, oe_, fo, P.EVEN, P.F64)
    oe = lambda: lat.dslash(g64, oo_, fe, P.ODD, P.F64)
    ms_eo = time_kernel(torch, eo, Kp, W)
    ms_oe = time_kernel(torch, oe, Kp, W)
    t_eo, t_oe = ms_eo / 1e3 / Kp, ms_oe / 1e3 / Kp
    parity = {
        "eo_gflops": round(Vh * FLOP_PER_SITE / t_eo / 1e9, 1),
        "oe_gflops": round(Vh * FLOP_PER_SITE / t_oe / 1e9, 1),
        "eo_gbs": round(Vh * BYTES_PARITY[0] / t_eo / 1e9, 1),
        "oe_gbs": round(Vh * BYTES_PARITY[0] / t_oe / 1e9, 1),
        "pair_gflops": round(V * FLOP_PER_SITE / (t_eo + t_oe) / 1e9, 1),
    }

    # ---- FP32 (config: FP64 and FP32 at 32^3x64) ------------------------------
    g32 = P.Gauge(lat, P.F32, 18)
    g32.copy_from(g64)
    f32e, f32o, o32e, o32o = buf(P.F32), buf(P.F32), buf(P.F32), buf(P.F32)
    lat.spinor_convert(f32e, P.F32, fe, P.F64)
    lat.spinor_convert(f32o, P.F32, fo, P.F64)
    ms32 = time_kernel(torch, lambda: lat.dslash_full(g32, o32e, o32o, f32e, f32o, P.F32), Kp, W)
    ms32e = time_kernel(torch, lambda: lat.dslash(g32, o32e, f32o, P.EVEN, P.F32), Kp, W)
    t32, t32e = ms32 / 1e3 / Kp, ms32e / 1e3 / Kp
    fp32 = {"full_gflops": round(V * FLOP_PER_SITE / t32 / 1e9, 1),
            "full_gbs": round(V * BYTES_FULL[1] / t32 / 1e9, 1),
            "eo_gflops": round(Vh * FLOP_PER_SITE / t32e / 1e9, 1),
            "eo_gbs": round(Vh * BYTES_PARITY[1] / t32e / 1e9, 1)}
    del g32, f32e, f32o, o32e, o32o

    if args.only == "dslash":
        if d.rank == 0:
            print(json.dumps({"metric": "Dslash GFLOP/s", "value": round(value, 1), "unit": "GFLOP/s",
                              "lattice": list(L), "only": "dslash", "kernel": kernel_name(head_cfg),
                              "frac": round(achieved / hbm, 4), "clocks": clocks, "sustained": sustained,
                              "per_parity_f64": parity,
                              "f32": fp32}))
        return 0

    # ---- e2e through the reference-facing C-ABI (host arrays) ---------------
    e2e = run_e2e(torch, P, lat, g64, fe, fo, d, args)

    # ---- even/odd CG: FP64 vs mixed precision, time to 1e-10 ----------------
    cg = run_cg(torch, P, lat, g64, buf, args) if not args.skip_cg else None
    del fe, fo, oe_, oo_
    mrhs = run_mrhs(torch, P, lat, g64, args) if not args.skip_batch else None
    # ---- batched multi-RHS, multi-lattice solve in one graph launch ----------
    batch = None
    if not args.skip_batch:
        batch = run_batch(torch, P, d, args, cg["f64"]["seconds"] if cg else None)
    # ---- reduced precision at 48^3x96: error against FP64 --------------------
    reduced = run_reduced(torch, P, d, args) if not args.skip_reduced else None

    # ---- CPU baseline (rank 0, N = 1 only) ----------------------------------
    cpu = None
    if d.world == 1 and not args.no_cpu:
        qin = e2e.pop("_qin")
        u = e2e.pop("_u")
        sec, mean, n, nthr, kind = cpu_reference_time(L, qin, u, 1000, 1, args.cpu_budget)
        cpu = {"value": round(V * FLOP_PER_SITE / sec / 1e9, 3), "unit": "GFLOP/s", "cores": nthr, "kind": kind,
               "sample": f"best of {n} full-lattice applications (eo+oe) at 32^3x64 after 1 warm-up, "
                         f"times from the reference's own return values "
                         f"(mean {V * FLOP_PER_SITE / mean / 1e9:.2f} GFLOP/s)"}
    e2e.pop("_qin", None)
    e2e.pop("_u", None)

    line = {
        "metric": "Dslash GFLOP/s", "value": round(value, 1), "unit": "GFLOP/s", "n_gpus": d.world,
        "steps": K, "warmup": W, "ms_per_step": round(t_step * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (random SU(3) links from a counter-based generator, Gaussian spinor)",
        "config": {"workload": "FP64 Wilson hopping matrix, full lattice (eo+oe in one launch), 32^3x64",
                   "lattice": list(L), "flop_per_site": FLOP_PER_SITE, "links": "18-real",
                   "l2": "inputs larger than L2 (1.5 GB per step vs 126 MB)",
                   "parallelism": f"replicas x{d.world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "peak_kind": peak_kind,
                     "bytes_per_site": BYTES_FULL[0], "kernel": kernel_name(head_cfg),
                     "traffic": traffic_bytes(head_cfg, V),
                     "traffic_note": traffic_note(head_cfg, L)},
        "sustained": sustained,
        "per_parity_f64": parity,
        "f32": fp32,
        "e2e": e2e,
        "cg": cg,
        "mrhs_dslash": mrhs,
        "batch": batch,
        "reduced_precision": reduced,
        "gpu_launches": K,
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def write_input_file(L) -> str:
    """Key-value input file for init_plqcd (lib/start.c:84-107): one
    process, one host thread."""
    fd, path = tempfile.mkstemp(suffix=".input")
    with os.fdopen(fd, "w") as f:
        f.write("".join(f"L{k} {int(L[k])}\n" for k in range(4)))
        f.write("".join(f"NPROC{k} 1\n" for k in range(4)))
        f.write("NTHREAD 1\nALIGN 6\n")
    return path


def run_sustained(torch, full, t_step, V, hbm, d: Dist, args):
    """The headline launch back to back for about --sustained-s seconds, with
    its own clock samples: the rate once the power cap has settled the SM
    clock, beside the short --steps window of `value`."""
    n = max(10, int(args.sustained_s / max(t_step, 1e-6)))
    clk = ClockSampler(d.local)
    clk.start()
    ms = d.max(time_kernel(torch, full, n, 3, d))
    clocks = clk.stop()
    t = ms / 1e3 / n
    return {"launches": n, "seconds": round(ms / 1e3, 3), "ms_per_launch": round(t * 1e3, 4),
            "gflops": round(d.world * V * FLOP_PER_SITE / t / 1e9, 1),
            "achieved_gbs": round(V * BYTES_FULL[0] / t / 1e9, 1), "frac": round(V * BYTES_FULL[0] / t / 1e9 / hbm, 4),
            "clocks": clocks}


def run_e2e(torch, P, lat, g64, fe, fo, d: Dist, args):
    """eo+oe through plqcd_hopping_matrix_*_sse3_assymbly on pinned host
    arrays, copies included, wall clock (the calls are synchronous). The
    link array is registered once with plqcd_gauge_update, as a caller that
    keeps its links fixed over many hops does; every call moves its spinor
    parity up and its output parity down."""
    L = lat.dims
    V = lat.V
    os.environ["PLQCD_DEVICE"] = str(d.local)
    path = write_input_file(L)
    P.finalize_plqcd()
    if P.init_plqcd(path) != 0:
        raise RuntimeError(P.last_error())
    os.unlink(path)
    lib = P.lib()
    nq, nu = V * 192, 4 * V * 144
    pq, pout, pu = lib.amalloc(nq, 6), lib.amalloc(nq, 6), lib.amalloc(nu, 6)
    mk = lambda p, n: np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), (n // 8,)).view(
        np.complex128)
    qin, qout, u = mk(pq, nq).reshape(V, 12), mk(pout, nq).reshape(V, 12), mk(pu, nu).reshape(4 * V, 9)
    P.check(lib.plqcd_gauge_store_host(g64.handle, pu))
    P.check(lib.plqcd_gauge_update(pu))
    aos = torch.zeros((V, 12), dtype=torch.complex128, device="cuda")
    lat.spinor_export(fe, P.F64, 0, aos)
    lat.spinor_export(fo, P.F64, 1, aos)
    lat.synchronize()
    qin[:] = aos.cpu().numpy()
    del aos
    qout[:] = 0
    Ke = max(3, min(args.steps, args.e2e_steps))
    for _ in range(max(1, min(args.warmup, 3))):
        P.hopping_matrix("eo", qin, qout, u)
        P.hopping_matrix("oe", qin, qout, u)
    d.barrier()
    t0 = time.perf_counter()
    for _ in range(Ke):
        P.hopping_matrix("eo", qin, qout, u)
        P.hopping_matrix("oe", qin, qout, u)
    dt = time.perf_counter() - t0
    d.barrier()
    dt = d.max(dt)
    kms, h2d, d2h = P.dropin_last_stats()
    res = {"value": round(d.world * V * FLOP_PER_SITE * Ke / dt / 1e9, 2), "unit": "GFLOP/s",
           "h2d_bytes_per_step": int(2 * h2d), "d2h_bytes_per_step": int(2 * d2h), "steps": Ke,
           "ms_per_step": round(dt / Ke * 1e3, 3),
           "api": "plqcd_hopping_matrix_eo/oe_sse3_assymbly on amalloc'd (pinned) host arrays; "
                  "link array registered once with plqcd_gauge_update (uploaded by the first call, "
                  "kept on the device); each call moves its spinor parity up and its output down"}
    # keep copies for the CPU baseline before the pinned blocks go away
    res["_qin"] = np.array(qin)
    res["_u"] = np.array(u)
    P.finalize_plqcd()
    lib.afree(pq)
    lib.afree(pout)
    lib.afree(pu)
    return res


def run_sharded(torch, P, lat, g64, fe, fo, args):
    """The t-slab decomposition (plqcd_b200/shard.py) with all `--shards`
    slabs held by this process on one GPU, ghost slices copied in place: the
    eo+oe pair over the slabs against the unsharded pair on the same fields.
    The difference is the decomposition's own cost (ghost copies, separate
    interior and boundary launches on site ranges); between GPUs the copies
    become NCCL transfers overlapped with the interior slices."""
    from plqcd_b200 import shard as SH
    L, N = lat.dims, args.shards
    stream = torch.cuda.current_stream().cuda_stream
    u = g64.store_host()
    aos = torch.zeros((lat.V, 12), dtype=torch.complex128, device="cuda")
    lat.spinor_export(fe, P.F64, 0, aos)
    lat.spinor_export(fo, P.F64, 1, aos)
    lat.synchronize()
    q = aos.cpu().numpy()
    del aos
    # one stream per slab (slab 0 on the current one): the slabs' hop launches overlap
    side = [torch.cuda.Stream() for _ in range(N - 1)]
    shards = [SH.ShardedLattice(L, r, N, lat.device, stream if r == 0 else side[r - 1].cuda_stream)
              for r in range(N)]
    T = SH.LocalTransport(N)
    gauges = [s.gauge_from_global(u) for s in shards]
    del u
    SH.exchange_gauge(shards, gauges, T)
    ins = {p: [s.import_global(q, 1 - p) for s in shards] for p in (0, 1)}
    outs = {p: [s.field(P.F64) for s in shards] for p in (0, 1)}

    def sharded():
        for p in (0, 1):
            SH.dslash(shards, gauges, outs[p], ins[p], p, P.F64, T)
        SH.join_streams(shards)  # the timing events sit on slab 0's stream

    oe_, oo_ = (torch.empty(lat.spinor_bytes(P.F64), dtype=torch.uint8, device="cuda") for _ in range(2))

    def single():
        lat.dslash(g64, oe_, fo, P.EVEN, P.F64)
        lat.dslash(g64, oo_, fe, P.ODD, P.F64)

    # the two are timed in alternating blocks (the clock drifts under the
    # power cap over a run): the medians of 7 blocks of K pairs each
    K, W = max(10, args.steps // 10), max(3, args.warmup)
    for _ in range(W):
        sharded()
        single()
    t_sh, t_1 = [], []
    for _ in range(7):
        t_sh.append(time_kernel(torch, sharded, K, 1) / 1e3 / K)
        t_1.append(time_kernel(torch, single, K, 1) / 1e3 / K)
    ratio = statistics.median([a / b for a, b in zip(t_sh, t_1)])
    t_sh, t_1 = statistics.median(t_sh), statistics.median(t_1)
    # host time to enqueue one sharded pair (Python, ctypes, stream events)
    torch.cuda.synchronize()
    h0 = time.perf_counter()
    for _ in range(K):
        sharded()
    host_us = (time.perf_counter() - h0) / K * 1e6
    torch.cuda.synchronize()
    ghost = sum(2 * sum(n for _, n in s.geo.spinor_slices(P.F64, 1)) for s in shards)
    return {"lattice": list(L), "slabs": N, "slab_t": shards[0].geo.Lt,
            "sharded_gflops": round(lat.V * FLOP_PER_SITE / t_sh / 1e9, 1),
            "single_pair_gflops": round(lat.V * FLOP_PER_SITE / t_1 / 1e9, 1),
            "overhead": round(ratio - 1, 4),
            "device_us_per_pair": round(t_sh * 1e6, 1), "host_enqueue_us_per_pair": round(host_us, 1),
            "ghost_bytes_per_hop": ghost,
            "note": "all slabs on one GPU, one stream each; ghost slices copied on the device"}


def run_cg(torch, P, lat, g64, buf, args):
    """Even/odd CG on D^dag D at kappa = 0.12, Gaussian source, to a true
    relative residual of 1e-10: FP64 against mixed precision (F32 and F16
    inner operators with 12-real links, FP64 reliable updates). Device time
    of each whole solve; the error of every mixed solution against the FP64
    one is reported."""
    kappa, tol = 0.12, 1e-10
    bs = lat.spinor_bytes(P.F64)
    be, bo = buf(P.F64), buf(P.F64)
    lat.spinor_gaussian(be, P.F64, 0, 4242)
    lat.spinor_gaussian(bo, P.F64, 1, 4242)
    sloppy = {"f64": None, "f32": (P.F32, 12), "f16": (P.F16, 12)}
    out, xs = {}, {}
    for name, fmt in sloppy.items():
        gs = None
        if fmt:
            gs = P.Gauge(lat, *fmt)
            gs.copy_from(g64)
        prec = fmt[0] if fmt else P.F64
        xe, xo = buf(P.F64), buf(P.F64)
        # warm-up: a few iterations tune every kernel configuration the solve uses
        P.invert_cg(lat, g64, gs, xe, xo, be, bo, P.cg_param(kappa=kappa, tol=tol, max_iter=4, sloppy_prec=prec),
                    raise_on_error=False)
        # three solves from x = 0; the median device time is reported (one solve
        # is ~15-35 ms, and single solves vary by a few percent between runs)
        runs = [P.invert_cg(lat, g64, gs, xe, xo, be, bo,
                            P.cg_param(kappa=kappa, tol=tol, sloppy_prec=prec, delta=args.delta))
                for _ in range(3)]
        info = sorted(runs, key=lambda i: i.seconds)[1]
        out[name] = {"iterations": info.iterations, "reliable_updates": info.reliable_updates,
                     "seconds": round(info.seconds, 5), "seconds_runs": [round(i.seconds, 5) for i in runs],
                     "schur_residual": info.schur_residual, "true_residual": info.true_residual}
        xs[name] = (xe, xo)
        del gs
    lat.synchronize()
    # F64 fields are plain doubles: compare the solutions as float64 vectors
    x64 = torch.cat([xs["f64"][0], xs["f64"][1]]).view(torch.float64)
    for name in ("f32", "f16"):
        diff = torch.cat([xs[name][0], xs[name][1]]).view(torch.float64) - x64
        out[name]["error_vs_f64"] = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(x64))
    # the F16 solve again, as one CUDA-graph launch (no host round trips)
    gs16 = P.Gauge(lat, P.F16, 12)
    gs16.copy_from(g64)
    xe, xo = buf(P.F64), buf(P.F64)
    item = dict(lat=lat, g64=g64, g_sloppy=gs16, nrhs=1, x_even=xe, x_odd=xo, b_even=be, b_odd=bo)
    P.invert_cg_batch([item], P.cg_param(kappa=kappa, tol=tol, sloppy_prec=P.F16, max_iter=3), True,
                      raise_on_error=False)
    ig, res = P.invert_cg_batch([item], P.cg_param(kappa=kappa, tol=tol, sloppy_prec=P.F16, delta=args.delta), True)
    lat.synchronize()
    diff = torch.cat([xe, xo]).view(torch.float64) - x64
    out["f16_graph"] = {"iterations": ig.iterations, "reliable_updates": ig.reliable_updates,
                        "seconds": round(ig.seconds, 5), "schur_residual": ig.max_schur_residual,
                        "true_residual": res[0], "graph_launches": ig.graph_launches,
                        "error_vs_f64": float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(x64))}
    del gs16
    best = min(("f32", "f16", "f16_graph"), key=lambda n: out[n]["seconds"])
    out["speedup_mixed_vs_f64"] = round(out["f64"]["seconds"] / out[best]["seconds"], 3)
    out["best_mixed"] = best
    out["config"] = {"lattice": list(lat.dims), "kappa": kappa, "tol": tol, "source": "Gaussian",
                     "operator": "even/odd preconditioned Mhat^dag Mhat, CG", "delta": args.delta}
    return out


def run_mrhs(torch, P, lat, g64, args, nrhs=8):
    """Multi-RHS hopping throughput at the benchmark lattice: bytes per site
    and RHS = 2 * spinor + 8 * link / nrhs. For the FP32-computing formats
    the RHS-pair kernel (variant 2002) and the scalar kernels, and for the
    16-bit ones the tensor-core kernel (3001), are also timed forced (keys
    variant/block), beside the tuner's choice."""
    res = {"nrhs": nrhs}
    for name, prec, recon, sb, lb in (("f64_18", P.F64, 18, 192, 144), ("f64_12", P.F64, 12, 192, 96),
                                      ("f32_12", P.F32, 12, 96, 48),
                                      ("f16_12", P.F16, 12, 52, 24), ("bf16_12", P.BF16, 12, 52, 24)):
        if args.mrhs_formats and name not in args.mrhs_formats.split(","):
            continue
        g = g64 if (prec, recon) == (P.F64, 18) else P.Gauge(lat, prec, recon)
        if g is not g64:
            g.copy_from(g64)
        bs = lat.spinor_bytes(prec)
        a = torch.empty(nrhs * bs, dtype=torch.uint8, device="cuda")
        o = torch.empty(nrhs * bs, dtype=torch.uint8, device="cuda")
        for r in range(nrhs):
            lat.spinor_gaussian(a[r * bs:(r + 1) * bs], prec, 1, 900 + r)
        per = lat.Vh * nrhs

        def rate(t):
            return {"gflops": round(per * FLOP_PER_SITE / t / 1e9, 1),
                    "gbs": round(per * (2 * sb + 8 * lb / nrhs) / t / 1e9, 1),
                    "site_rhs_per_s": per / t, "us": round(t * 1e6, 2)}

        hop = lambda: lat.dslash_mrhs(g, o, a, nrhs, P.EVEN, prec)
        res[name] = rate(time_kernel(torch, hop, 20, 3) / 20 / 1e3)
        cfg = tuned_config(P, f"dslash_mrhs|p{prec}|r{recon}|plain|n{nrhs}|{lat.dims[0]}x")
        res[name]["tuned_variant"] = cfg[0] if cfg else None
        if args.mrhs_forced:  # profiling runs: only these forced configurations
            forced = {}
            for vb in args.mrhs_forced.split(","):
                v, blk = (int(x) for x in vb.split("/"))
                os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"] = str(v), str(blk)
                try:
                    forced[f"{v}/{blk}"] = rate(time_kernel(torch, hop, 20, 3) / 20 / 1e3)["us"]
                finally:
                    del os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"]
            res[name]["forced_us"] = forced
        elif prec == P.F64:
            forced = {}
            # 4xxx: links shared in shared memory; 1xxxxx-8xxxxx: TMA-staged
            # rows with RHS tiles (100000 * RHS per tile + TMA variant)
            for v, blk in ((4208, 256), (4204, 128), (4308, 256), (4304, 128), (100, 128), (102, 64), (2, 128),
                           (1022, 64), (402202, 0), (402102, 0), (404202, 0), (402201, 0), (202202, 0),
                           (802101, 0)):
                os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"] = str(v), str(blk)
                try:
                    forced[f"{v}/{blk}"] = rate(time_kernel(torch, hop, 20, 3) / 20 / 1e3)["us"]
                finally:
                    del os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"]
            res[name]["forced_us"] = forced
        else:
            forced = {}
            cand = [(2002, 64), (2002, 128), (2022, 64), (2022, 128), (2032, 64), (2102, 64), (2102, 128),
                    (2122, 64), (2122, 128), (102, 128), (2, 128)]
            if prec in (P.F16, P.BF16):
                cand += [(3001, 128), (1042, 128), (1022, 64)]
            for v, blk in cand:
                os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"] = str(v), str(blk)
                try:
                    forced[f"{v}/{blk}"] = rate(time_kernel(torch, hop, 20, 3) / 20 / 1e3)["us"]
                finally:
                    del os.environ["PLQCD_MRHS_VARIANT"], os.environ["PLQCD_MRHS_BLOCK"]
            res[name]["forced_us"] = forced
        del a, o
        if g is not g64:
            del g
    return res


def run_batch(torch, P, d: Dist, args, f64_single_seconds: float | None):
    """Batched multi-RHS solves in one graph launch: 16^3x32 (32 RHS),
    24^3x48 (16 RHS), 32^3x64 (8 RHS), each with its own random SU(3) field
    and Gaussian sources, kappa = 0.12, mixed precision (F16 inner operator)
    to 1e-10; against the same solves one at a time in FP64."""
    kappa, tol = 0.12, 1e-10
    spec = [((16, 16, 16, 32), 32), ((24, 24, 24, 48), 16), ((32, 32, 32, 64), 8)]
    stream = torch.cuda.current_stream().cuda_stream
    items = []
    for k, (L, n) in enumerate(spec):
        lat = P.Lattice(L, d.local, stream)
        g64 = P.Gauge(lat, P.F64, 18)
        g64.random(31 + k)
        gs = P.Gauge(lat, P.F16, 12)
        gs.copy_from(g64)
        bs = lat.spinor_bytes(P.F64)
        blk = [torch.empty(n * bs, dtype=torch.uint8, device="cuda") for _ in range(4)]
        for r in range(n):
            lat.spinor_gaussian(blk[0][r * bs:(r + 1) * bs], P.F64, 0, 1000 * k + r)
            lat.spinor_gaussian(blk[1][r * bs:(r + 1) * bs], P.F64, 1, 1000 * k + r)
        items.append(dict(lat=lat, g64=g64, g_sloppy=gs, nrhs=n, b_even=blk[0], b_odd=blk[1], x_even=blk[2],
                          x_odd=blk[3]))
    prm = P.cg_param(kappa=kappa, tol=tol, sloppy_prec=P.F16, delta=args.delta)
    graph = not args.eager
    P.invert_cg_batch(items, P.cg_param(kappa=kappa, tol=tol, sloppy_prec=P.F16, max_iter=3), graph,
                      raise_on_error=False)  # warm-up: tunes every launch configuration
    info, res = P.invert_cg_batch(items, prm, graph)
    site_rhs = sum(it["lat"].V * it["nrhs"] for it in items)
    out = {"lattices": [[list(L), n] for L, n in spec], "kappa": kappa, "tol": tol, "sloppy": "f16_12",
           "delta": args.delta,
           "graph_launches": info.graph_launches, "iterations": info.iterations,
           "reliable_updates": info.reliable_updates, "seconds": round(info.seconds, 4),
           "max_schur_residual": info.max_schur_residual, "max_true_residual": info.max_true_residual,
           "site_rhs_per_s": site_rhs / info.seconds}
    # the same solves one at a time, FP64 CG
    seq = 0.0
    for it in items:
        lat, bs = it["lat"], it["lat"].spinor_bytes(P.F64)
        xe, xo = torch.empty(bs, dtype=torch.uint8, device="cuda"), torch.empty(bs, dtype=torch.uint8, device="cuda")
        for r in range(it["nrhs"]):
            sl = slice(r * bs, (r + 1) * bs)
            if r == 0:  # tune this lattice's FP64 kernels outside the timing
                P.invert_cg(lat, it["g64"], None, xe, xo, it["b_even"][sl], it["b_odd"][sl],
                            P.cg_param(kappa=kappa, tol=tol, max_iter=3), raise_on_error=False)
            inf1 = P.invert_cg(lat, it["g64"], None, xe, xo, it["b_even"][sl], it["b_odd"][sl],
                               P.cg_param(kappa=kappa, tol=tol))
            seq += inf1.seconds
    out["sequential_f64_seconds"] = round(seq, 4)
    out["sequential_f64_site_rhs_per_s"] = site_rhs / seq
    out["speedup_vs_sequential_f64"] = round(seq / info.seconds, 3)
    # multi-RHS mixed CG at 32^3x64 (8 RHS) alone, per RHS, against one plain
    # FP64 CG: the median of three solves (single solves vary by a few percent)
    it = items[2]
    runs = [P.invert_cg_batch([it], prm, graph)[0] for _ in range(3)]
    info8 = sorted(runs, key=lambda r: r.seconds)[1]
    out["mrhs_32x32x32x64"] = {"nrhs": it["nrhs"], "seconds": round(info8.seconds, 4),
                               "seconds_runs": [round(r.seconds, 4) for r in runs],
                               "seconds_per_rhs": round(info8.seconds / it["nrhs"], 5),
                               "iterations": info8.iterations, "reliable_updates": info8.reliable_updates,
                               "max_true_residual": info8.max_true_residual}
    if f64_single_seconds:
        out["mrhs_32x32x32x64"]["speedup_per_rhs_vs_plain_f64_cg"] = round(
            f64_single_seconds / (info8.seconds / it["nrhs"]), 3)
    for it in items:
        it["lat"].synchronize()
    items.clear()
    return out


def run_reduced(torch, P, d: Dist, args):
    """Reduced-precision hopping at 48^3x96: relative L2 error of the eo
    output against the FP64 kernel, and each kernel's bandwidth."""
    L = (48, 48, 48, 96)
    lat = P.Lattice(L, d.local, torch.cuda.current_stream().cuda_stream)
    Vh = lat.Vh
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(77)

    def buf(prec):
        return torch.empty(lat.spinor_bytes(prec), dtype=torch.uint8, device="cuda")

    fin, ref = buf(P.F64), buf(P.F64)
    lat.spinor_gaussian(fin, P.F64, 1, 5)
    lat.dslash(g64, ref, fin, P.EVEN, P.F64)
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    lat.spinor_norm2(ref, P.F64, 1, nrm)
    ref2 = float(nrm)
    res = {"lattice": list(L)}
    t64 = time_kernel(torch, lambda: lat.dslash(g64, ref, fin, P.EVEN, P.F64), 20, 3) / 20 / 1e3
    res["f64_18"] = {"rel_l2_vs_f64": 0.0, "gbs": round(Vh * 1536 / t64 / 1e9, 1),
                     "gflops": round(Vh * FLOP_PER_SITE / t64 / 1e9, 1)}
    for name, prec, recon, bps in (("f32_18", P.F32, 18, 768), ("f32_12", P.F32, 12, 576),
                                   ("f16_12", P.F16, 12, 296), ("bf16_12", P.BF16, 12, 296)):
        g = P.Gauge(lat, prec, recon)
        g.copy_from(g64)
        a, o = buf(prec), buf(prec)
        lat.spinor_convert(a, prec, fin, P.F64)
        t = time_kernel(torch, lambda: lat.dslash(g, o, a, P.EVEN, prec), 20, 3) / 20 / 1e3
        back = buf(P.F64)
        lat.spinor_convert(back, P.F64, o, prec)
        diff = back.view(torch.float64) - ref.view(torch.float64)
        err = float(torch.linalg.vector_norm(diff)) / ref2 ** 0.5
        res[name] = {"rel_l2_vs_f64": err, "gbs": round(Vh * bps / t / 1e9, 1),
                     "gflops": round(Vh * FLOP_PER_SITE / t / 1e9, 1)}
        del g, a, o, back, diff
    del g64
    lat.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--sustained-s", type=float, default=3.0,
                    help="seconds of the back-to-back headline loop of the `sustained` record (0: skip)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=40)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU-baseline sampling")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--skip-cg", action="store_true")
    ap.add_argument("--skip-reduced", action="store_true")
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--delta", type=float, default=0.003,
                    help="reliable-update threshold of the mixed solvers (0.003: 4 FP64 reliable updates at "
                         "32^3x64, against 5 at 0.01; below 0.003 the 16-bit recursion stalls)")
    ap.add_argument("--lattice", default=",".join(map(str, L_BENCH)),
                    help="L0,L1,L2,L3 of the hopping-matrix workload (default 32,32,32,64)")
    ap.add_argument("--only", choices=["all", "dslash", "cg", "mrhs", "batch", "sharded"], default="all",
                    help="dslash / cg: only that section (profiling runs); sharded: the t-slab "
                         "decomposition with --shards slabs held on one GPU")
    ap.add_argument("--shards", type=int, default=4, help="slabs of --only sharded")
    ap.add_argument("--eager", action="store_true",
                    help="batched solves as eager loops instead of one graph launch (ncu does not profile "
                         "the kernels of graphs with conditional nodes)")
    ap.add_argument("--mrhs-formats", default="", help="comma list of the multi-RHS formats to time (default all)")
    ap.add_argument("--mrhs-nrhs", type=int, default=8, help="RHS of --only mrhs")
    ap.add_argument("--mrhs-forced", default="",
                    help="--only mrhs: comma list of variant/block configurations to time forced (default: a "
                         "built-in list)")
    args = ap.parse_args()
    args.lattice = tuple(int(x) for x in args.lattice.split(","))
    d = Dist()
    if args.impl == "reference":
        return run_reference(args, d)
    d.init("nccl")
    try:
        return run_ours(args, d)
    finally:
        d.close()


if __name__ == "__main__":
    sys.exit(main())
