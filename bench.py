"""Benchmark of the H2 apply path (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): JIT-mode H2 matmul,
3-D Matern-3/2 kernel (1 + sqrt3 r/l) exp(-sqrt3 r/l) with l = 1, N = 1,000,000
points i.i.d. uniform in [0, N^(1/3)]^3 (seeded), reltol 1e-6, 16 right-hand sides
i.i.d. standard normal.  The H2 representation is built once by H2Pack's own
construction (numerical proxy points, default leaf size 400); a step is one
H2 matmul of the 16 right-hand sides.  value = right-hand-side matvecs per second
over all ranks (16 per step), FP32-mixed arithmetic (re-centred FP32 kernel
evaluation, FP64 accumulation across blocks); the plain FP64 path is timed beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n N]

--impl reference runs H2Pack's own CPU H2P_matmul (the reference library built from
its sources into oracle/_ref) on the same configuration with all host cores; a step
is one 16-RHS matmul.  Multi-GPU: independent replicas, one per rank (the path has no
exchange step); value sums the ranks, time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H2 matvecs/s (N=1M Matern-3/2 JIT, 16 RHS)"
UNIT = "matvecs/s"
PP_FILE = os.path.join("/tmp", "h2b200_pp_matern32_1e-6.dat")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=1_000_000)
    p.add_argument("--nvec", type=int, default=16)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--check-rows", type=int, default=10_000)
    return p.parse_args()


def points(n, seed=20240):
    rng = np.random.default_rng(seed)
    return rng.random((3, n)) * n ** (1.0 / 3.0)


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_reference(args):
    """H2Pack's own CPU path: H2P_matmul with the same 16 right-hand sides, on the
    reference library built from H2Pack's sources (oracle/_ref), all host cores.
    One step is one H2P_matmul; steps beyond a 150 s budget are not run (one call
    takes tens of seconds at N = 1M), and the line reports the steps actually timed."""
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    nv = args.nvec
    coord = points(args.n)
    t0 = time.time()
    R = O.RefH2("matern32", [1.0], coord, 1e-6, BD_JIT=1, proxy="id", pp_fname=PP_FILE, n_thread=cores)
    build_s = time.time() - t0
    X = np.random.default_rng(1).standard_normal((R.N, nv))
    budget, ts, warm = 150.0, [], 0
    t_start = time.time()
    for _ in range(args.warmup):
        if time.time() - t_start > budget / 3:
            break
        R.matmul(X)
        warm += 1
    for _ in range(args.steps):
        t = time.perf_counter()
        R.matmul(X)
        ts.append(time.perf_counter() - t)
        if time.time() - t_start > budget:
            break
    sec = sum(ts) / len(ts)
    v = nv / sec
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": len(ts), "warmup": warm,
        "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"H2 JIT matmul, Matern-3/2 l=1, N={args.n}, reltol 1e-6, {nv} RHS N(0,1) "
                               "(H2Pack CPU H2P_matmul)",
                   "n": args.n, "nvec": nv, "build_seconds": build_s, "openmp_threads": R.info["n_thread"],
                   "steps_requested": args.steps, "warmup_requested": args.warmup, "time_budget_s": budget},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": R.info["n_thread"], "kind": "reference",
                         "sample": f"{len(ts)} H2P_matmul calls ({nv} RHS) of H2Pack compiled from its sources, "
                                   f"full N={args.n}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    R.close()


def run_ours(args):
    import torch
    world, rank, local, pg = dist_init(args)
    torch.cuda.set_device(local)
    from h2pack_b200 import H2Matrix, direct_sum
    nv = args.nvec
    coord = points(args.n, seed=20240 + rank)
    t0 = time.time()
    H = H2Matrix("matern32", coord, [1.0], 1e-6, BD_JIT=1, proxy="id", pp_fname=PP_FILE, precision="mixed",
                 n_thread=os.cpu_count())
    build_s = time.time() - t0
    img = H.image()
    N = H.N
    g = torch.Generator(device="cuda").manual_seed(7 + rank)
    X = torch.randn(N, nv, dtype=torch.float64, device="cuda", generator=g)
    Y = torch.empty_like(X)

    def timed(steps, warm):
        for _ in range(warm):
            img.matmul_device(X, Y)
        torch.cuda.synchronize()
        barrier(pg)
        s0 = img.stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            img.matmul_device(X, Y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        s1 = img.stats()
        return ms, s0, s1

    # ---- mixed precision (headline)
    with ClockSampler(local) as clk:
        ms, s0, s1 = timed(args.steps, args.warmup)
    ms_max = max_over_ranks(pg, ms)
    value = world * nv * 1e3 / ms_max
    Ym = Y.clone()
    phase = [(b - a) / args.steps for a, b in zip(s0["ms_phase"], s1["ms_phase"])]
    launches = s1["n_launches"] - s0["n_launches"]

    # ---- plain FP64 path
    fp64 = None
    if not args.no_fp64:
        H.set_precision("fp64")
        ms64, _, _ = timed(max(3, args.steps // 2), 1)
        ms64 = max_over_ranks(pg, ms64)
        fp64 = {"value": world * nv * 1e3 / ms64, "ms_per_step": ms64}
        Y64 = Y.clone()
        H.set_precision("mixed")

    # ---- end to end through the drop-in H2P_matmul with pinned host buffers
    Xh = X.cpu().pin_memory()
    Yh = torch.empty_like(Xh).pin_memory()
    for _ in range(2):
        H.matmul_raw(101, nv, Xh.data_ptr(), nv, Yh.data_ptr(), nv)
    barrier(pg)
    t = time.perf_counter()
    ke = max(3, args.steps // 2)
    for _ in range(ke):
        H.matmul_raw(101, nv, Xh.data_ptr(), nv, Yh.data_ptr(), nv)
    e2e_s = max_over_ranks(pg, (time.perf_counter() - t) / ke)
    e2e = {"value": world * nv / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(Xh.numel() * 8),
           "d2h_bytes_per_step": int(Yh.numel() * 8), "ms_per_step": 1e3 * e2e_s}

    # ---- accuracy against the FP64 direct sum on sampled rows
    err = {}
    if rank == 0 and args.check_rows > 0:
        rng = np.random.default_rng(11)
        rows = np.sort(rng.choice(H.N, min(args.check_rows, H.N), replace=False))
        cols = [0, nv // 2]
        Xc = X.cpu().numpy()
        for name, Ycur in (("mixed", Ym), ("fp64", Y64 if fp64 else None)):
            if Ycur is None:
                continue
            Yc = Ycur.cpu().numpy()
            e = []
            for c in cols:
                yd = direct_sum("matern32", [1.0], coord, Xc[:, c], coord[:, rows])
                e.append(float(np.linalg.norm(Yc[rows, c] - yd) / np.linalg.norm(yd)))
            err[name] = max(e)

    # ---- roofline of the dominant kernel (far-field JIT: on-the-fly B blocks x 16 RHS)
    st = img.stats()
    flop_per_pair = 13 + 4 * nv      # Matern32_3D_krnl_bimv_flop = 17 per pair for one RHS, 4 of them the bi-matvec
    far_flops = st["jit_pairs_B"] * flop_per_pair
    far_ms = phase[1]
    peak_fp32 = 148 * 128 * 2 * 1.965e9 / 1e12
    roofline = {"bound": "fp32", "kernel": "k_jit (far field, on-the-fly B x 16 RHS)",
                "achieved": far_flops / (far_ms * 1e-3) / 1e12, "peak": peak_fp32, "unit": "TFLOP/s",
                "frac": far_flops / (far_ms * 1e-3) / 1e12 / peak_fp32, "traffic": None,
                "peak_source": "nominal FP32 FMA peak 148 SM x 128 lanes x 2 x 1.965 GHz (no measured FP32 figure)",
                "flop_model": f"unordered point pairs x ({flop_per_pair}) = H2Pack JIT_flops model with 16 RHS"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(H, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32-mixed (FP32 kernel eval, FP64 accumulation)", "data": "synthetic",
            "config": {"workload": f"H2 JIT matmul, Matern-3/2 l=1, N={args.n} uniform in [0,N^(1/3)]^3, "
                                   f"reltol 1e-6, {nv} RHS N(0,1), numerical proxy points, leaf 400",
                       "n": args.n, "nvec": nv, "parallelism": f"replicas x{world}",
                       "l2": "working set (U arena, coordinates, vectors) > 126 MB L2, no flush",
                       "build_seconds": build_s,
                       "n_node": H.info["n_node"], "max_level": H.info["max_level"],
                       "jit_pairs_B": st["jit_pairs_B"], "jit_pairs_D": st["jit_pairs_D"]},
            "phase_ms": {"gather+up": phase[0], "B_far": phase[1], "down": phase[2], "D_near": phase[3],
                         "assemble": phase[4]},
            "fp64": fp64, "rel_err_vs_direct": err, "e2e": e2e, "gpu_launches": int(launches),
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    H.close()
    if pg is not None:
        pg.destroy_process_group()


def cpu_baseline(H, args):
    """H2Pack's CPU H2P_matmul (reference library) on the same handle and 16 RHS: one call."""
    try:
        from oracle import oracle as O
        lib = O.libref()
    except Exception as e:  # pragma: no cover - reported, not fatal
        return {"value": None, "unavailable": str(e)}
    nv = args.nvec
    X = np.random.default_rng(3).standard_normal((H.N, nv))
    Y = np.zeros((H.N, nv))
    t = time.perf_counter()
    lib.H2P_matmul(H.h2pack, 101, nv, O.dptr(X), nv, O.dptr(Y), nv)
    sec = time.perf_counter() - t
    return {"value": nv / sec, "unit": UNIT, "cores": H.info["n_thread"], "kind": "reference",
            "sample": f"1 H2P_matmul ({nv} RHS) of H2Pack compiled from its sources on the same N={args.n} "
                      f"handle, {sec:.1f} s"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
