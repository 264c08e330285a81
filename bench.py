#!/usr/bin/env python
"""Throughput of 1024^2 grid transport solves on B200 (residual <= 1e-7).

One step = one batch of `--batch` independent 1024x1024 solves of the single-large-
solve workload (6 random filled disks / convex polygons, value 1 on background
1e-3, Gaussian blur sigma = 5 px, normalised to mean 1; seeded synthetic data),
solved together by the library's batched engine; value = solves/s over all ranks.
Multi-GPU runs are weak-scaled: every rank solves its own batch, no collective on
the data path (instances are independent).

Fields beyond the base contract:
  e2e           the same metric through the public C ABI with host (pinned) inputs
                and outputs, host<->device copies inside the timed region
  plain         solves/s of the plain single-instance form: the same densities
                solved one call at a time
  roofline      dominant kernel: algorithmic bytes (or flops) / its CUDA-event time
  cpu_baseline  the reference library (compiled from its own sources) timed on this
                host: one full 1024^2 solve on one core, rank 0 at N=1 only

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1024^2 OT solves/s at residual<=1e-7"
UNIT = "solves/s"
N_GRID = 1024
THRESHOLD = 1e-7
SIGMA_PX = 5.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=8)
    p.add_argument("--n", type=int, default=N_GRID)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-mixed", action="store_true")
    p.add_argument("--precision", default="split", choices=["split", "fp64"],
                   help="headline arithmetic: split (FP32 integration and transforms with FP64 sums, "
                        "line search and potential; the single-solve workload's stated precision) or fp64")
    p.add_argument("--no-other-precision", action="store_true")
    p.add_argument("--no-locate", action="store_true")
    p.add_argument("--no-barycenter", action="store_true")
    p.add_argument("--no-tensor", action="store_true")
    p.add_argument("--no-config1", action="store_true")
    p.add_argument("--mixed-count", type=int, default=64)
    p.add_argument("--sample-iters", type=int, default=10, help="reference arm: iterations per warm-up step")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_first_seed(rank):
    """Each rank solves its own densities (seeds 1000*rank + k): the batch shards across
    ranks with no collective on the data path."""
    return 1000 * rank


def max_over_ranks(value, world, device="cuda"):
    """The slowest rank's time: every rank calls it with its own value (a collective with
    the same steps on every rank); the identity for one rank."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(instances_per_rank, world, ms_per_step):
    """Whole-job throughput: the instances of all ranks over the slowest rank's step time."""
    return instances_per_rank * world / (ms_per_step / 1e3)


def densities(n, count, first_seed):
    from otmap_b200 import workloads as W

    return [W.to_cells(W.blurred_shapes(n, first_seed + k, sigma_px=SIGMA_PX)) for k in range(count)]


def config(args, world, extra=None):
    c = {"workload": f"{args.n}x{args.n} blurred shapes (6 disks/convex polygons, sigma 5 px, floor 1e-3), "
                     f"threshold {THRESHOLD:g}, batch {args.batch} per GPU",
         "grid": args.n, "batch_per_gpu": args.batch, "global_batch": args.batch * world,
         "threshold": THRESHOLD, "parallelism": f"independent instances x{world}"}
    if extra:
        c.update(extra)
    return c


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"otmap_b200_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the timed region starts once the sampler is running (its first line is written)
        t0 = time.time()
        while time.time() - t0 < 3.0 and self.proc.poll() is None:
            self.f.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# Algorithmic bytes per cell moved by one launch of each iteration kernel (FP64 arrays
# read + written once each; halos, L2 hits and scalars not counted):
#   sweep_sums    reads psi, d_hat, d_prev, r_k, r_{k-1}                    5 x 8 B
#   sweep_update  reads psi, d_hat, d_prev, r_k; writes d, psi', r'          7 x 8 B
#   dct_* / fft_* one pass of the cosine transform: reads + writes a line    2 x 8 B
# Every active instance runs each kernel once per iteration, so the cells a kernel
# touched over the timed steps are sum over instances of iterations x n^2 (x steps).
# Split precision (FP32 r, d_hat, d and transform temporaries; FP64 psi):
#   sweep32_sums    psi 8 + d_hat, d_prev, r_k, r_{k-1} 4 each                    24 B
#   sweep32_update  reads psi 8, d_hat, d_prev, r_k 4 each; writes psi' 8, d 4, r' 4  36 B
#   dct32_*         one pass of the FP32 cosine transform                          8 B
ALG_BYTES_PER_CELL = {"sweep_sums": 40, "sweep_update": 56, "dct_rows_fwd": 16, "dct_cols": 16, "dct_rows_inv": 16,
                      "fft_rows_fwd": 16, "fft_cols": 16, "fft_rows_inv": 16,
                      "sweep32_sums": 24, "sweep32_update": 36, "dct32_rows_fwd": 8, "dct32_cols": 8,
                      "dct32_rows_inv": 8}


def load_traffic():
    """DRAM bytes per cell per launch measured by ncu (profiles/traffic_per_cell.json)."""
    p = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def kernel_rates(prof, cell_iters, peaks):
    """Achieved algorithmic bandwidth of every profiled iteration kernel."""
    out = {}
    for name, (ms, cnt) in (prof or {}).items():
        rec = {"ms": ms, "launches": cnt, "avg_launch_us": 1e3 * ms / max(cnt, 1)}
        if name in ALG_BYTES_PER_CELL and ms > 0:
            gbs = ALG_BYTES_PER_CELL[name] * cell_iters / (ms / 1e3) / 1e9
            rec.update({"achieved_gbs": gbs, "frac_of_hbm": gbs / peaks["hbm_gbs"]})
        out[name] = rec
    return out


def load_pipes():
    """FP64 pipe and occupancy figures of the iteration kernels from one ncu capture
    (profiles/pipe_utilisation.json)."""
    p = os.path.join(ROOT, "profiles", "pipe_utilisation.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def roofline(prof, cell_iters, steps, peaks):
    """Dominant kernel: algorithmic bytes per launch / its average CUDA-event launch time."""
    if not prof:
        return None
    name, (ms, cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    if name not in ALG_BYTES_PER_CELL:
        return {"kernel": name, "launches": cnt, "total_ms": ms, "bound": None}
    per_launch_bytes = ALG_BYTES_PER_CELL[name] * cell_iters / cnt
    avg_s = ms / 1e3 / cnt
    achieved = per_launch_bytes / avg_s / 1e9
    traffic = load_traffic().get(name)
    cells_per_launch = cell_iters / cnt
    return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"],
            "traffic": traffic * cells_per_launch if traffic is not None else None,
            "alg_bytes_per_launch": per_launch_bytes, "avg_launch_us": avg_s * 1e6, "launches": cnt,
            "peak_source": peaks["source"],
            "traffic_source": "profiles/traffic_per_cell.json (ncu dram__bytes_read+write per cell, scaled)",
            **pipe_note(name)}


def pipe_note(name):
    """What bounds a kernel that sits below the HBM roofline while moving only its
    algorithmic bytes: its FP64 pipe share and occupancy from the committed ncu capture."""
    rec = load_pipes().get(name)
    if not rec:
        return {}
    return {"fp64_pipe_busy": rec["fp64_pipe"], "warps_active": rec["warps_active"], "registers": rec["registers"],
            "limiter": "latency of dependent FP64 operations at the occupancy the registers allow "
                       "(ncu: traffic equals the algorithmic bytes; see profiles/pipe_utilisation.json)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        d["source"] = "of measured: MEASURED_PEAKS.json hbm_gbs"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0,
            "source": "of fallback: 6.65 TB/s, a measured B200 copy bandwidth (MEASURED_PEAKS.json absent)"}


def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    from otmap_b200 import native as N

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n, B = args.n, args.batch
    ns = [n] * B
    host = densities(n, B, rank_first_seed(rank))
    dev_in = [torch.from_numpy(d).cuda() for d in host]
    V = (n + 1) ** 2
    opt = N.default_options()
    opt.threshold = THRESHOLD
    ns_c = (C.c_int * B)(*ns)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    prec_of = {"split": N.PRECISION_SPLIT, "fp64": N.PRECISION_FP64}

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    def measure(precision, with_e2e, with_profile, with_clocks):
        """One precision: warm-up, the timed steps (device-resident), optionally a profiled
        pass (host loop, per-kernel events) and the end-to-end pass (pinned host buffers)."""
        ctx = N.Context(local)
        ctx.set_precision(prec_of[precision])
        ctx.set_autotune(True)  # the sweeps' strip height timed on the first call
        stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        dev_out = [torch.empty((V, 2), dtype=torch.float64, device="cuda") for _ in range(B)]
        stats = (N.SolveStatsC * B)()

        def solve_batch(inp, out):
            dp = (C.c_void_p * B)(*[x.data_ptr() for x in inp])
            fp = (C.c_void_p * B)(*[x.data_ptr() for x in out])
            N.check(N.lib().otm_solve_batch(ctx.handle, B, ns_c, dp, C.byref(opt), fp, None, stats))

        def timed(inp, out, steps, profile=False):
            ctx.profile(-1)
            ctx.profile(1 if profile else 0)
            total = 0.0
            launches0 = ctx.launch_count()
            barrier()
            torch.cuda.synchronize()
            for _ in range(steps):
                flush.fill_(1.0)  # L2 flush between steps (outside the events)
                torch.cuda.synchronize()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                solve_batch(inp, out)
                b.record(stream)
                b.synchronize()
                total += a.elapsed_time(b)
            torch.cuda.synchronize()
            barrier()
            launches = ctx.launch_count() - launches0
            prof = ctx.profile_totals() if profile else None
            ctx.profile(0)
            return total, launches, prof

        ctx.init(n)
        for _ in range(args.warmup):
            solve_batch(dev_in, dev_out)
        torch.cuda.synchronize()
        clocks = Clocks(local) if with_clocks else None
        if clocks:
            clocks.start()
        t_ms, launches, _ = timed(dev_in, dev_out, args.steps)
        clk = clocks.stop() if clocks else None
        st_list = [stats[k] for k in range(B)]
        prof = None
        if with_profile:
            # per-kernel CUDA-event timing needs the host-driven loop (events around each
            # launch): a second pass over the same steps, for the kernel breakdown only
            _, _, prof = timed(dev_in, dev_out, args.steps, profile=True)
        t_ms = max_over_ranks(t_ms, world)
        ms_step = t_ms / args.steps
        rec = {"precision": precision, "value": job_value(B, world, ms_step), "ms_per_step": ms_step,
               "strip_rows": ctx.strip_rows(),
               "iterations": [s.iterations for s in st_list],
               "final_residual_max": max(s.residual for s in st_list), "gpu_launches": launches}
        if with_e2e:
            h_in = [torch.from_numpy(d).pin_memory() for d in host]
            h_out = [torch.empty((V, 2), dtype=torch.float64).pin_memory() for _ in range(B)]
            e_ms, _, _ = timed(h_in, h_out, args.steps)
            e_ms = max_over_ranks(e_ms, world)
            rec["e2e"] = {"value": job_value(B, world, e_ms / args.steps), "unit": UNIT,
                          "h2d_bytes_per_step": B * n * n * 8, "d2h_bytes_per_step": B * V * 2 * 8}
        ctx.close()
        return rec, dev_out, st_list, prof, clk

    head, dev_out, st_list, prof, clk = measure(args.precision, not args.no_e2e, True, True)
    other = None
    other_out = None
    if not args.no_other_precision:
        oprec = "fp64" if args.precision == "split" else "split"
        other, other_out, other_st, _, _ = measure(oprec, not args.no_e2e, False, False)
    value, ms_step, launches = head["value"], head["ms_per_step"], head["gpu_launches"]
    e2e = head.get("e2e")
    ctx = N.Context(local)
    ctx.set_precision(prec_of[args.precision])
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    plain = None
    if not args.no_plain:
        plain = bench_plain(local, n, dev_in, [torch.empty((V, 2), dtype=torch.float64, device="cuda")
                                               for _ in range(B)], opt, prec_of[args.precision],
                            steps=min(args.steps, 5))

    adjoint = None if args.no_adjoint else bench_adjoint(ctx, stream)
    locate = None if args.no_locate else bench_locate(ctx, stream, n, dev_in[0])
    bary = None if args.no_barycenter else bench_barycenter(local, cpu=(rank == 0 and world == 1 and
                                                                    not args.no_cpu_baseline))
    tensor = None if args.no_tensor else bench_tensor(local, n, dev_in, opt, steps=min(args.steps, 5))
    cfg1 = None if args.no_config1 else bench_config1(local, cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
    mixed = None if args.no_mixed else bench_mixed(stream, args.mixed_count, precision=prec_of[args.precision])

    peaks = load_peaks()
    cell_iters = args.steps * sum(st.iterations * nn * nn for st, nn in zip(st_list, ns))
    roof = roofline(prof, cell_iters, args.steps, peaks)
    kernels = kernel_rates(prof, cell_iters, peaks)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_map = cpu_baseline(host[0], n, locate_points=None if args.no_locate else LOCATE_POINTS)
        if ref_map is not None:
            parity = parity_vs_reference(ctx, n, ref_map, dev_out[0], st_list[0],
                                         None if args.no_locate else LOCATE_POINTS)
            parity["precision"] = args.precision
            if other_out is not None:
                import numpy as np

                g = other_out[0].double().cpu().numpy()
                parity["other_precision"] = {
                    "precision": other["precision"],
                    "max_vertex_err": float(np.abs(g - ref_map.fwd()).max()),
                    "iterations_gpu": int(other_st[0].iterations), "residual_gpu": float(other_st[0].residual)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": "f32 cells / f64 sums" if args.precision == "split" else "f64",
                "data": "synthetic (seeded blurred-shape densities, generated on the host in FP64)",
                "config": config(args, world, {"l2": "256 MiB write between steps; working set > L2"}),
                "precision": args.precision, "strip_rows": head["strip_rows"], "iterations": head["iterations"],
                "final_residual_max": head["final_residual_max"], "gpu_launches": launches,
                "e2e": e2e, "other_precision": other, "plain": plain, "parity": parity, "adjoint": adjoint, "batched_mixed": mixed, "locate": locate, "barycenter": bary, "tensor_transform": tensor, "config1": cfg1, "roofline": roof, "kernels": kernels, "clocks": clk,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    ctx.close()


def bench_mixed(stream, count=64, repeats=2, threshold=1e-6, precision=0):
    """Many uneven instances: `count` Gaussian mixtures (4..16 components, floor 1e-3), n
    drawn log-uniformly from {128, 256, 512, 1024}, residual <= 1e-6. Batched = one
    otm_solve_batch call; plain = one otm_solve call per instance on its own context; both
    on the device-side graph loop, timed with CUDA events, best of `repeats`. Throughput in
    1024^2-equivalent solves/s (sum n^2 / 1024^2)."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    imgs = W.batched_mixtures(count, seed=11)
    ns = [im.shape[0] for im in imgs]
    eq = sum(n * n for n in ns) / 1024.0 ** 2
    dev = [torch.from_numpy(W.to_cells(im)).cuda() for im in imgs]
    outs = [torch.empty(((n + 1) ** 2, 2), dtype=torch.float64, device="cuda") for n in ns]
    opt = N.default_options()
    opt.threshold = threshold
    ctx = N.Context(torch.cuda.current_device())
    ctx.set_precision(precision)
    ctx.set_autotune(True)
    stream = torch.cuda.ExternalStream(ctx.stream())
    for n in sorted(set(ns)):
        ctx.init(n)
    stats = (N.SolveStatsC * count)()
    ns_c = (C.c_int * count)(*ns)
    dp = (C.c_void_p * count)(*[d.data_ptr() for d in dev])
    fp = (C.c_void_p * count)(*[f.data_ptr() for f in outs])

    def timed(fn, reps):
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        return best

    batch = lambda: N.check(N.lib().otm_solve_batch(ctx.handle, count, ns_c, dp, C.byref(opt), fp, None, stats))
    batch()  # warm-up: builds the graph (and tunes the strip height)
    rows_batched = ctx.strip_rows()
    l0 = ctx.launch_count()
    t_batch = timed(batch, repeats)
    launches = (ctx.launch_count() - l0) // repeats
    iters = [stats[k].iterations for k in range(count)]
    # plain: one otm_solve call per instance on a separate context (graph loop; its
    # workspace cache keeps one workspace and captured graph per size), warmed up first
    ctx_plain = N.Context(torch.cuda.current_device())
    ctx_plain.set_precision(precision)
    ctx_plain.set_autotune(True)
    for n in sorted(set(ns)):
        ctx_plain.init(n)
    stream_p = torch.cuda.ExternalStream(ctx_plain.stream())

    def plain():
        for k in range(count):
            N.check(N.lib().otm_solve(ctx_plain.handle, ns[k], C.c_void_p(dev[k].data_ptr()), C.byref(opt),
                                      C.c_void_p(outs[k].data_ptr()), None, None))

    plain()
    best = None
    for _ in range(repeats):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream_p)
        plain()
        b.record(stream_p)
        b.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    t_plain = best
    ctx.close()
    ctx_plain.close()
    return {"workload": f"{count} Gaussian mixtures, n log-uniform in {{128,256,512,1024}}, residual <= {threshold:g}",
            "sizes": {str(n): ns.count(n) for n in sorted(set(ns))}, "equivalent_1024_solves": eq,
            "batched_ms": t_batch, "batched_value": eq / (t_batch / 1e3), "batched_gpu_launches": launches,
            "plain_ms": t_plain, "plain_value": eq / (t_plain / 1e3),
            "unit": "1024^2-equivalent solves/s", "batched_over_plain": t_plain / t_batch,
            "plain_timing": f"CUDA events around {count} sequential otm_solve calls on a separate warmed-up context "
                            "(device-side graph loop, one cached workspace per size), best of %d" % repeats,
            "iterations_min_max": [min(iters), max(iters)], "strip_rows_batched": rows_batched,
            "autotune": "strip height of the sweeps timed on each context's first call of a configuration"}


def bench_adjoint(ctx, stream, n=512, repeats=3):
    """Cost of the implicit adjoint on the softmax-logits workload (512^2, density =
    blur(softmax(z)), sigma 8 px): gradient time over the time of one forward iteration."""
    import ctypes as C

    import numpy as np
    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    _, img = W.softmax_logits(n, 0, sigma_px=8.0)
    dens = torch.from_numpy(W.to_cells(img)).cuda()
    V = (n + 1) ** 2
    fwd = torch.empty((V, 2), dtype=torch.float64, device="cuda")
    q = torch.randn((V, 2), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    out = {}
    grads = {}

    def timed(fn):
        best = None
        for _ in range(repeats):
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r = fn()
            b.record(stream)
            b.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        return best, r

    opt = N.default_options()
    opt.threshold = THRESHOLD
    st = N.SolveStatsC()
    ctx.init(n)
    t_solve, _ = timed(lambda: N.check(N.lib().otm_solve(ctx.handle, n, C.c_void_p(dens.data_ptr()), C.byref(opt),
                                                         C.c_void_p(fwd.data_ptr()), None, C.byref(st))))
    per_iter = t_solve / max(st.iterations, 1)
    for name, mode in (("one_step", N.ADJOINT_ONE_STEP), ("krylov", N.ADJOINT_KRYLOV)):
        ao = N.AdjointOptionsC()
        N.lib().otm_default_adjoint_options(C.byref(ao))
        ao.mode = mode
        ast = N.AdjointStatsC()
        g = torch.empty(n * n, dtype=torch.float64, device="cuda")
        t, _ = timed(lambda: N.check(N.lib().otm_adjoint(ctx.handle, n, C.c_void_p(dens.data_ptr()),
                                                        C.c_void_p(fwd.data_ptr()), C.c_void_p(q.data_ptr()),
                                                        C.byref(ao), C.c_void_p(g.data_ptr()), C.byref(ast))))
        grads[name] = g.double().cpu().numpy()
        out[name] = {"ms": t, "per_forward_iteration": t / per_iter, "poisson_solves": ast.iterations,
                     "relative_residual": ast.relative_residual}
    ref = grads["krylov"]
    out["one_step"]["relative_error_vs_krylov"] = float(np.linalg.norm(grads["one_step"] - ref) / np.linalg.norm(ref))
    # truncated GMRES: k Arnoldi steps (k Poisson solves) and the final lambda = M^+ (V y)
    curve = []
    for k in range(1, 9):
        ao = N.AdjointOptionsC()
        N.lib().otm_default_adjoint_options(C.byref(ao))
        ao.mode = N.ADJOINT_KRYLOV
        ao.tol = 0.0
        ao.max_iter = k
        ao.restart = max(k, 8)
        ast = N.AdjointStatsC()
        g = torch.empty(n * n, dtype=torch.float64, device="cuda")
        t, _ = timed(lambda: N.check(N.lib().otm_adjoint(ctx.handle, n, C.c_void_p(dens.data_ptr()),
                                                        C.c_void_p(fwd.data_ptr()), C.c_void_p(q.data_ptr()),
                                                        C.byref(ao), C.c_void_p(g.data_ptr()), C.byref(ast))))
        gh = g.double().cpu().numpy()
        curve.append({"k": k, "poisson_solves": ast.iterations, "ms": t, "per_forward_iteration": t / per_iter,
                      "relative_error_vs_krylov": float(np.linalg.norm(gh - ref) / np.linalg.norm(ref)),
                      "relative_residual": ast.relative_residual})
    out["truncated_gmres"] = curve
    meets = [c["k"] for c in curve if c["relative_error_vs_krylov"] <= 1e-3]
    out["smallest_k_within_1e-3"] = meets[0] if meets else None
    out.update({"workload": f"{n}^2 blur(softmax(N(0,1) logits)), sigma 8 px; dL/dfwd random",
                "forward_solve_ms": t_solve, "forward_iterations": st.iterations, "forward_iteration_ms": per_iter})
    return out


def cpu_baseline(density_cells, n, locate_points=None):
    """The reference (oracle/_ref, compiled from the reference sources) on one host core;
    with locate_points, also its inversion (BVH build + queries, apply_inverse_map) of that
    many points and its rasterization of the forward mesh at n x n. Returns the record and
    the reference's map (for the parity check)."""
    from oracle import ref

    if not ref.available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}, None
    s = ref.RefSolver()
    t_init = s.init(n)
    m = s.solve(density_cells, threshold=THRESHOLD)
    out = {"value": 1.0 / m.seconds, "unit": UNIT, "cores": 1, "kind": "reference",
           "sample": f"one full {n}^2 solve of the rank-0 instance 0 density ({m.iterations} iterations, "
                     f"residual {m.residual:.3g}); solve {m.seconds:.2f} s, init (LDLT factorisation, "
                     f"cached per size by the reference) {t_init:.2f} s excluded",
           "init_seconds": t_init, "solve_seconds": m.seconds}
    if locate_points:
        from otmap_b200 import workloads as W

        pts = W.random_points(locate_points, LOCATE_SEED)
        _, t_inv = m.apply_inverse(pts)
        _, t_ras = ref.rasterize(m.fwd(), n, m.density(), n, n)
        out["locate"] = {"inverse_queries_per_s": locate_points / t_inv, "inverse_seconds": t_inv,
                         "raster_pixels_per_s": n * n / t_ras, "raster_seconds": t_ras,
                         "sample": f"{locate_points} FP32-drawn points through apply_inverse_map (BVH build "
                                   f"included); rasterize_image of the forward mesh at {n}x{n}; one core"}
    return out, m


def parity_vs_reference(ctx, n, ref_map, gpu_fwd, gpu_stats, locate_points=None):
    """Outside the timed region: the benchmarked GPU solve of instance 0 against the
    reference's own FP64 solve of the same density (max vertex error, iteration counts,
    final residuals); the GPU's inversion of `locate_points` FP32-drawn points and its
    raster, both on the reference's forward mesh, against the reference's."""
    import numpy as np

    from oracle import ref
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    fwd_ref = ref_map.fwd()
    dens_ref = ref_map.density()
    g = gpu_fwd.double().cpu().numpy() if hasattr(gpu_fwd, "cpu") else np.asarray(gpu_fwd)
    out = {"oracle": "the reference library (oracle/_ref, FP64, Eigen SimplicialLDLT) on the same density",
           "max_vertex_err": float(np.abs(g - fwd_ref).max()),
           "iterations_gpu": int(gpu_stats.iterations), "iterations_ref": int(ref_map.iterations),
           "residual_gpu": float(gpu_stats.residual), "residual_ref": float(ref_map.residual)}
    if locate_points:
        pts = W.random_points(locate_points, LOCATE_SEED)
        pos_ref, _ = ref_map.apply_inverse(pts)
        nh_ref, _, _ = ref.query_all(fwd_ref, n, pts)
        tm = ot.TransportMap(n, fwd_ref, dens_ref, context=ctx)
        p = np.ascontiguousarray(pts.copy())
        nh = np.zeros(p.shape[0], dtype=np.int32)
        tm.apply_inverse(p, None, nh)
        ties = nh_ref > 1
        diff = (p != pos_ref).any(axis=1)
        img_ref, _ = ref.rasterize(fwd_ref, n, dens_ref, n, n)
        img = np.empty((n, n))
        ot.rasterize_image(fwd_ref, dens_ref, img, n=n, context=ctx)
        out.update({"inverse_points": int(locate_points), "inverse_nhits_mismatch": int((nh != nh_ref).sum()),
                    "inverse_position_mismatch": int(diff.sum()), "inverse_ties": int(ties.sum()),
                    "inverse_tie_position_mismatch": int(diff[ties].sum()),
                    "raster_pixels": n * n, "raster_pixel_mismatch": int((img != img_ref).sum())})
    return out


def bench_plain(device, n, dev_in, dev_out, opt, precision, steps=5):
    """The plain single-instance form: one otm_solve call per density, on its own context
    (graph loop, workspace and graph warmed up by an untimed pass), CUDA events around
    each step of len(dev_in) calls; best step."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N

    ctx = N.Context(device)
    ctx.set_precision(precision)
    ctx.init(n)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", device))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        for x, y in zip(dev_in, dev_out):
            N.check(N.lib().otm_solve(ctx.handle, n, C.c_void_p(x.data_ptr()), C.byref(opt), C.c_void_p(y.data_ptr()),
                                      None, None))

    step()
    times = []
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    ctx.close()
    B = len(dev_in)
    return {"value": B / (min(times) / 1e3), "unit": UNIT, "ms_per_step_best": min(times),
            "ms_per_step_median": sorted(times)[len(times) // 2],
            "form": f"{B} sequential otm_solve calls per step (one density each) on a separate warmed-up context, "
                    "device-side graph loop, CUDA events; best of %d steps, L2 flushed between steps" % steps}


LOCATE_POINTS = 1 << 20
LOCATE_SEED = 7


def bench_barycenter(device, n=512, res=512, cpu=True):
    """The bilinear barycenter pipeline at 512^2: four blurred-shape densities (the
    single-solve generator at 512^2, blur sigma 2.5 px) solved in one batch, their inverse
    meshes at the origin grid by GPU point location, the 5 x 5 grid of bilinear
    barycenters rasterized at 512^2; then the gradient of the L2 loss between the centre
    barycenter and a seeded Gaussian-mixture image with respect to the four densities
    (otm_barycenter_loss, Krylov adjoint). Host buffers in and out, wall clock around each
    whole phase after a warm-up. With cpu, the reference's forward pipeline on one core
    (oracle/_ref: 4 solves, 4 inversions, 25 rasters)."""
    import ctypes as C

    import numpy as np
    import torch

    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    ctx = N.Context(device)
    dens = [W.to_cells(W.blurred_shapes(n, 100 + k, sigma_px=2.5)) for k in range(4)]
    means = [d.mean() for d in dens]
    target = W.gaussian_mixture(res, 17)
    grid = ot.grid_vertices(n)
    steps = [0.0, 0.25, 0.5, 0.75, 1.0]

    grid_dev = torch.from_numpy(grid).cuda()

    def forward():
        # host densities in, 25 host images out; the inverse meshes stay on the device
        maps = ot.solve_batch(dens, context=ctx)
        inv = []
        for m in maps:
            p = grid_dev.clone()
            m.apply_inverse(p)
            inv.append(p)
        imgs = [ot.barycenter_image(inv, a, b, means, res, context=ctx, want_mesh=False)[0]
                for a in steps for b in steps]
        return maps, imgs

    forward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    maps, imgs = forward()
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    w = ot.bilinear_weights(0.5, 0.5)
    ot.barycenter_loss(dens, w, target, context=ctx)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss, img, grads, st = ot.barycenter_loss(dens, w, target, context=ctx)
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    out = {"workload": f"4 blurred-shape densities {n}^2 (sigma 2.5 px), 5x5 bilinear barycenters rasterized at "
                       f"{res}^2; gradient of sum (centre image - Gaussian-mixture target)^2 w.r.t. the 4 densities",
           "forward_ms": 1e3 * t_fwd, "forward_iterations": [m.stats.iterations for m in maps],
           "gradient_ms": 1e3 * t_grad, "loss": loss, "adjoint_solves": list(st.adjoint_solves)[:4],
           "adjoint_residual": list(st.adjoint_residual)[:4],
           "timing": "wall clock, host densities in and host images out (inverse meshes kept on the device), "
                     "after one warm-up of each phase"}
    ctx.close()
    if cpu:
        from oracle import ref

        if ref.available():
            t0 = time.perf_counter()
            rs = ref.RefSolver()
            rs.init(n)
            t_init = time.perf_counter() - t0
            t0 = time.perf_counter()
            rmaps = [rs.solve(d) for d in dens]
            inv = []
            for m in rmaps:
                p, _ = m.apply_inverse(grid)
                inv.append(p)
            for a in steps:
                for b in steps:
                    ref.barycenter(n, inv, a, b, means, res, res)
            out["cpu_reference_forward_ms"] = 1e3 * (time.perf_counter() - t0)
            out["cpu_reference_init_ms"] = 1e3 * t_init
            out["cpu_reference_sample"] = "the same forward pipeline in the reference library on one core (init excluded)"
    return out


def bench_config1(device, cpu=True, n=256, seed=0, repeats=5):
    """The reference's own CPU-sized case: one 256^2 Gaussian-mixture solve (8 Gaussians +
    floor 1e-3, residual <= 1e-7, FP64 mode) and the inversion of its 257^2 grid vertices
    (locator build included), device-resident buffers, CUDA events around the whole unit,
    median of `repeats` after a warm-up. With cpu, the same unit in the reference library on
    one core (init, the per-size factorisation, excluded as the reference caches it)."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    ctx = N.Context(device)
    ctx.init(n)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", device))
    dens_h = W.to_cells(W.gaussian_mixture(n, seed))
    dens = torch.from_numpy(dens_h).cuda()
    V = (n + 1) ** 2
    fwd = torch.empty((V, 2), dtype=torch.float64, device="cuda")
    adj = torch.empty(n * n, dtype=torch.float64, device="cuda")
    grid = torch.from_numpy(ot.grid_vertices(n)).cuda()
    pts = torch.empty_like(grid)
    opt = N.default_options()
    opt.threshold = THRESHOLD
    st = N.SolveStatsC()
    missing = C.c_long(0)

    def unit():
        N.check(N.lib().otm_solve(ctx.handle, n, C.c_void_p(dens.data_ptr()), C.byref(opt), C.c_void_p(fwd.data_ptr()),
                                  C.c_void_p(adj.data_ptr()), C.byref(st)))
        h = C.c_void_p()
        N.check(N.lib().otm_map_create(ctx.handle, n, C.c_void_p(fwd.data_ptr()), C.c_void_p(adj.data_ptr()),
                                       C.byref(h)))
        pts.copy_(grid)
        N.check(N.lib().otm_map_inverse(h, C.c_void_p(pts.data_ptr()), V, None, None, C.byref(missing)))
        N.lib().otm_map_destroy(h)

    unit()
    times = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        unit()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    med = sorted(times)[len(times) // 2]
    rec = {"workload": f"{n}^2 Gaussian mixture (8 Gaussians, floor 1e-3, seed {seed}), residual <= {THRESHOLD}, FP64; "
                       f"inversion of the {n + 1}^2 grid vertices (locator build included)",
           "ms": med, "units_per_s": 1e3 / med, "iterations": int(st.iterations), "residual": float(st.residual),
           "inverse_missing": int(missing.value),
           "timing": "CUDA events around solve + map + inversion, device-resident buffers, median of %d" % repeats}
    ctx.close()
    if cpu:
        from oracle import ref

        if ref.available():
            rs = ref.RefSolver()
            rs.init(n)
            m = rs.solve(dens_h, threshold=THRESHOLD)
            _, t_inv = m.apply_inverse(ot.grid_vertices(n))
            rec["cpu_reference"] = {"seconds": m.seconds + t_inv, "solve_seconds": m.seconds,
                                    "inverse_seconds": t_inv, "iterations": int(m.iterations), "cores": 1,
                                    "units_per_s": 1.0 / (m.seconds + t_inv)}
            import numpy as np

            rec["max_vertex_err_vs_reference"] = float(np.abs(fwd.cpu().numpy() - m.fwd()).max())
    return rec


def bench_tensor(device, n, dev_in, opt, steps=5):
    """The batch of the headline step in split precision with the tensor-core cosine
    transform (OTM_POISSON_TENSOR): solves/s (device-resident, CUDA events, best step)
    and the per-launch time of the tensor-core kernel from a profiled pass."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N

    B = len(dev_in)
    ctx = N.Context(device)
    ctx.set_precision(N.PRECISION_SPLIT)
    ctx.set_poisson(N.POISSON_TENSOR)
    ctx.init(n)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", device))
    V = (n + 1) ** 2
    out = [torch.empty((V, 2), dtype=torch.float64, device="cuda") for _ in range(B)]
    stats = (N.SolveStatsC * B)()
    ns = (C.c_int * B)(*([n] * B))
    dp = (C.c_void_p * B)(*[x.data_ptr() for x in dev_in])
    fp = (C.c_void_p * B)(*[x.data_ptr() for x in out])
    run = lambda: N.check(N.lib().otm_solve_batch(ctx.handle, B, ns, dp, C.byref(opt), fp, None, stats))
    run()
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    ctx.profile(-1)
    ctx.profile(1)
    run()
    prof = ctx.profile_totals()
    ctx.profile(0)
    ctx.close()
    its = [stats[k].iterations for k in range(B)]
    rec = {"value": B / (min(times) / 1e3), "unit": UNIT, "ms_per_step_best": min(times), "iterations": its,
           "final_residual_max": max(stats[k].residual for k in range(B)),
           "form": "split precision, OTM_POISSON_TENSOR (tcgen05 3xTF32 products), same batch as the headline"}
    if prof and "dct_tc" in prof:
        ms, cnt = prof["dct_tc"]
        # four n x n x n products per instance-iteration: 8 n^3 algorithmic flops (the
        # 3xTF32 split issues three MMAs per product, 24 n^3 on the tensor pipe)
        flops = 8.0 * n ** 3 * sum(its)
        peaks = load_peaks()
        tf = flops / (ms / 1e3) / 1e12
        rec["dct_tc"] = {"ms": ms, "launches": cnt, "avg_launch_us": 1e3 * ms / max(cnt, 1),
                         "algorithmic_tflops": tf, "issued_tflops": 3 * tf,
                         "frac_issued_of_tf32_peak": 3 * tf / (peaks["bf16_tflops"] / 2),
                         "note": "one launch per product, four per iteration; tf32 peak taken as half the "
                                 "measured bf16 GEMM rate (" + peaks["source"].split(":")[0] + ")"}
    return rec


def bench_locate(ctx, stream, n, dens_dev, repeats=5):
    """Inversion and rasterization of one n^2 map on the GPU (device-resident buffers):
    the point locator build, 2^20 FP32-drawn query points through otm_map_inverse, and
    rasterize_image of the forward mesh at n x n, each timed with CUDA events."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    V = (n + 1) ** 2
    fwd = torch.empty((V, 2), dtype=torch.float64, device="cuda")
    adj = torch.empty(n * n, dtype=torch.float64, device="cuda")
    opt = N.default_options()
    opt.threshold = THRESHOLD
    N.check(N.lib().otm_solve(ctx.handle, n, C.c_void_p(dens_dev.data_ptr()), C.byref(opt),
                              C.c_void_p(fwd.data_ptr()), C.c_void_p(adj.data_ptr()), None))
    pts0 = torch.from_numpy(W.random_points(LOCATE_POINTS, LOCATE_SEED)).cuda()
    pts = pts0.clone()
    img = torch.empty((n, n), dtype=torch.float64, device="cuda")
    missing = C.c_long(0)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    build, inv, ras = [], [], []
    for _ in range(repeats):
        h = C.c_void_p()
        N.check(N.lib().otm_map_create(ctx.handle, n, C.c_void_p(fwd.data_ptr()), C.c_void_p(adj.data_ptr()),
                                       C.byref(h)))
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record(stream)
        N.check(N.lib().otm_map_init_inverse(h))
        b.record(stream)
        b.synchronize()
        build.append(a.elapsed_time(b))
        pts.copy_(pts0)
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record(stream)
        N.check(N.lib().otm_map_inverse(h, C.c_void_p(pts.data_ptr()), LOCATE_POINTS, None, None, C.byref(missing)))
        b.record(stream)
        b.synchronize()
        inv.append(a.elapsed_time(b))
        a, b = ev(), ev()
        a.record(stream)
        N.check(N.lib().otm_rasterize(ctx.handle, n, C.c_void_p(fwd.data_ptr()), C.c_void_p(adj.data_ptr()), n, n,
                                      C.c_void_p(img.data_ptr())))
        b.record(stream)
        b.synchronize()
        ras.append(a.elapsed_time(b))
        N.lib().otm_map_destroy(h)
    med = lambda v: sorted(v)[len(v) // 2]
    return {"workload": f"one {n}^2 forward map; {LOCATE_POINTS} query points drawn in FP32 (seed {LOCATE_SEED}); "
                        f"raster {n}x{n} with the map's density",
            "locator_build_ms": med(build), "inverse_ms": med(inv), "inverse_queries_per_s": LOCATE_POINTS / (med(inv) / 1e3),
            "inverse_missing": missing.value, "raster_ms": med(ras), "raster_pixels_per_s": n * n / (med(ras) / 1e3),
            "timing": "CUDA events around each call, device-resident buffers, median of %d" % repeats}



# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU code path on all host cores


def _ref_worker(args_tuple):
    n, seed, steps, warmup, sample_iters, barrier = args_tuple
    sys.path.insert(0, ROOT)
    from oracle import ref

    from otmap_b200 import workloads as W

    d = W.to_cells(W.blurred_shapes(n, seed, sigma_px=SIGMA_PX))
    s = ref.RefSolver()
    s.init(n)
    for _ in range(warmup):  # untimed warm-up: a bounded number of iterations each
        s.solve(d, threshold=THRESHOLD, max_iter=sample_iters)
    barrier.wait()
    t0 = time.time()
    per_step, its, res = [], [], []
    for _ in range(steps):  # one step = one whole solve of this process's density
        a = time.perf_counter()
        m = s.solve(d, threshold=THRESHOLD)
        per_step.append(time.perf_counter() - a)
        its.append(m.iterations)
        res.append(m.residual)
    t1 = time.time()
    return t0, t1, per_step, its, res


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp

    n, B = args.n, args.batch
    total = B * world
    seeds = [1000 * r + k for r in range(world) for k in range(B)]
    cores = len(os.sched_getaffinity(0))
    # One single-threaded reference process per host core (the reference has no threads),
    # each solving one density of the batch (densities repeat when there are more cores
    # than densities): the throughput of all cores on a steady stream of such solves.
    P = max(1, min(cores, 32))  # each process holds a factorisation of the n^2 Laplacian
    ctxm = mp.get_context("spawn")
    with ctxm.Manager() as mgr:
        barrier = mgr.Barrier(P)
        with ctxm.Pool(P) as pool:
            res = pool.map(_ref_worker, [(n, seeds[p % total], args.steps, args.warmup, args.sample_iters, barrier)
                                         for p in range(P)])
    t_start = min(r[0] for r in res)
    t_end = max(r[1] for r in res)
    wall = t_end - t_start
    solves = P * args.steps
    value = solves / wall
    ms_step = 1e3 * wall / args.steps
    its = [it for r in res for it in r[3]]
    per = [t for r in res for t in r[2]]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded blurred-shape densities, generated on the host in FP64)",
            "config": config(args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": P, "kind": "reference",
                             "sample": f"{P} processes of the reference library (oracle/_ref, Eigen "
                                       f"SimplicialLDLT, single-threaded), one per host core, each solving one "
                                       f"of the {total} densities; one step = one whole solve per process "
                                       f"({P} solves), timed from a common barrier to the last process's end; "
                                       f"value = {solves} solves / {wall:.1f} s wall; iterations {min(its)}-"
                                       f"{max(its)}, solve time {min(per):.2f}-{max(per):.2f} s; init "
                                       f"(factorisation) and {args.warmup} warm-up steps of "
                                       f"{args.sample_iters} iterations excluded"},
            "timed_wall_s": wall,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
