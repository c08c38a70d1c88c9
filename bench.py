"""Benchmark of the GMG-PCG Poisson solve (one step = one full solve to 1e-6 relative residual).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload: ring512 -- the adaptive 5-level octree with 512x512x1024 effective resolution
(domain 1x1x2, leaves at levels 2-6 refined around a synthetic vortex ring, box obstacle),
seeded synthetic velocity -> divergence right-hand side.  Prints one JSON line on rank 0.

  value     solves/s with inputs resident in HBM (device-timed, CUDA events, L2 flushed
            between steps by writing a 256 MiB buffer)
  e2e       solves/s through cirrus_gmg_solve_host with pinned host buffers: H2D of b,
            solve, D2H of x inside the timed region
  roofline  the dominant kernel (Gauss-Seidel colour sweep on the finest level), algorithmic
            bytes / CUDA-event duration against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (FP32 mirror of the reference arithmetic, OpenMP) on a bounded
            sample of PCG iterations of the same workload, extrapolated to solves/s

Multi-GPU (torchrun): replicas only -- every rank solves its own instance (seed = rank); no
collective on the data path; value = all ranks' solves / max-over-ranks time.
--impl reference runs the reference's own CUDA build (oracle/_ref) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GS_BYTES_PER_CELL = 9.0  # read x 4 + rhs 2 (one colour) + mask 1 + write x 2 (algorithmic)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ring512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"cirrus_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier_max(pg, value: float) -> float:
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def build_instance(name: str, seed: int):
    from cirrus_b200 import DeviceGrid, workloads as W

    b = W.build(W.make(name, seed))
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    return b, g


def cpu_baseline(b, rhs, budget_s: float = 10.0, max_solves: int = 5) -> dict:
    """The CPU oracle (FP32 mirror of the reference arithmetic, all host threads): full solves of
    the same workload to 1e-6, repeated until about `budget_s` seconds have elapsed."""
    from oracle import oracle as O

    f = O.CpuOracle(b.tiles)
    f.set_ctypes(b.ctypes)
    solves, its = 0, 0
    t0 = time.perf_counter()
    while solves < max_solves and (solves == 0 or time.perf_counter() - t0 < budget_s):
        f.set_channel_f32(1, rhs)
        it, rel, _ = f.solve(O.CpuOracle.FP32, 1000, 1e-6)
        solves += 1
        its = it
    dt = time.perf_counter() - t0
    return {"seconds": dt, "threads": O.num_threads(), "solves": solves, "iters": its}


def run_ours(args, world, rank, local, pg):
    import torch

    from cirrus_b200 import GMGSolver, B_CHANNEL, TMP_CHANNEL

    b, g = build_instance(args.workload, seed=rank)
    rhs = g.get_channel(B_CHANNEL)
    g.copy_channel(TMP_CHANNEL, B_CHANNEL)  # keep b resident for restoring between steps
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    solver = GMGSolver()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    iters_seen, launches = [], []

    def one(timed: bool):
        g.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, rel = solver.solve(g, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        iters_seen.append(it)
        launches.append(solver.last_result.kernel_launches)
        if rel >= 1e-6:
            raise RuntimeError(f"solve did not converge: rel {rel}")
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        one(False)
    iters_seen.clear()
    launches.clear()
    clocks = None
    clk = Clocks(local)
    if rank == 0:
        clk.start()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    times = [one(True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    if rank == 0:
        clocks = clk.stop()
    total_ms = barrier_max(pg, sum(times))

    # end to end: host buffers through the public C ABI (H2D b, solve, D2H x)
    b_host = torch.from_numpy(rhs.reshape(-1)).pin_memory()
    x_host = torch.empty_like(b_host).pin_memory()
    b_np, x_np = b_host.numpy(), x_host.numpy()
    for _ in range(2):
        solver.solve_host(g, b_np, x_np, stream=sh)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.solve_host(g, b_np, x_np, stream=sh)
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    e2e_total = barrier_max(pg, sum(e2e_times))

    # roofline of the dominant kernel: GS colour sweep on the finest level, same data, on `stream`
    maxl = int(b.tiles[:, 0].max())
    mg_cells = int(((b.tiles[:, 0] == maxl) & ((b.tiles[:, 4] & 3) != 0)).sum()) * 512
    g.copy_channel(3, B_CHANNEL, sh)
    reps = 200
    for _ in range(10):
        g.gauss_seidel_sweep(maxl, 4, 3, 0, stream=sh)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(reps):
        g.gauss_seidel_sweep(maxl, 4, 3, i & 1, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    gs_ms = e0.elapsed_time(e1) / reps
    peaks = measured_peaks()
    achieved = mg_cells * GS_BYTES_PER_CELL / (gs_ms * 1e-3) / 1e9

    n = args.steps * world
    value = n / (total_ms * 1e-3)
    dof = g.dof
    out = {
        "metric": "Poisson solves/s to 1e-6 relative residual (GMG-PCG, reference arithmetic)",
        "value": round(value, 3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (fp64 CG scalars)",
        "data": "synthetic (seeded face velocities, divergence right-hand side)",
        "config": {"workload": args.workload, "tiles": int(b.tiles.shape[0]), "dof": int(dof),
                   "effective_resolution": "512x512x1024" if args.workload == "ring512" else args.workload,
                   "levels": f"leaves {int(b.tiles[(b.tiles[:, 4] & 1) != 0, 0].min())}-{maxl}",
                   "tolerance": 1e-6, "stopping_rule": "recursive ||r||/||b|| < tol, checked every iteration",
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "mdof_per_s": round(dof * value / 1e6, 2),
        "iters_per_solve": int(statistics.median(iters_seen)),
        "latency_ms": {"p50": round(float(np.percentile(times, 50)), 4), "p99": round(float(np.percentile(times, 99)), 4)},
        "gpu_launches": int(sum(launches)),
        "e2e": {"value": round(n / (e2e_total * 1e-3), 3), "unit": "solves/s",
                "h2d_bytes_per_step": int(rhs.nbytes), "d2h_bytes_per_step": int(rhs.nbytes)},
        "roofline": {"kernel": "k_gs_sweep (finest level, one colour)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": int(mg_cells * GS_BYTES_PER_CELL),
                     "launch_us": round(gs_ms * 1e3, 3), "traffic": None},
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cb = cpu_baseline(b, rhs)
        out["cpu_baseline"] = {"value": round(cb["solves"] / cb["seconds"], 4), "unit": "solves/s", "cores": cb["threads"],
                               "kind": "port",
                               "sample": f"{cb['solves']} full solves of {args.workload} to 1e-6 ({cb['iters']} PCG "
                                         f"iterations each) by the CPU oracle (FP32 mirror of the reference "
                                         f"arithmetic, OpenMP), {cb['seconds']:.1f} s wall"}
    return out


def run_reference(args, world, rank, local, pg):
    from oracle import oracle as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libcirrus_ref.so was not built (needs the reference tree)"}
    import torch

    from cirrus_b200 import workloads as W

    w = W.make(args.workload, seed=rank)
    b = W.build(w)
    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    rhs = ref.rhs(b.velocity)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    times, iters = [], []

    def one():
        ref.set_channel(1, rhs)
        flush.zero_()
        torch.cuda.synchronize()
        it, rel, ms = ref.solve(1000, 1e-6, 1, 10, 1, w.pure_neumann)
        iters.append(it)
        return ms

    for _ in range(args.warmup):
        one()
    iters.clear()
    clk = Clocks(local)
    if rank == 0:
        clk.start()
    if pg is not None:
        pg.barrier()
    times = [one() for _ in range(args.steps)]
    clocks = clk.stop() if rank == 0 else None
    total = barrier_max(pg, sum(times))
    n = args.steps * world
    value = n / (total * 1e-3)
    leaf = (b.tiles[:, 4] & 1) != 0
    dof = int(((b.ctypes[leaf] & 2) != 0).sum())
    return {
        "impl": "reference",
        "metric": "Poisson solves/s to 1e-6 relative residual (GMG-PCG, reference arithmetic)",
        "value": round(value, 3), "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total / args.steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (fp64 CG scalars)", "data": "synthetic (seeded face velocities, divergence right-hand side)",
        "config": {"workload": args.workload, "tiles": int(b.tiles.shape[0]), "dof": dof, "tolerance": 1e-6,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "mdof_per_s": round(dof * value / 1e6, 2), "iters_per_solve": int(statistics.median(iters)),
        "latency_ms": {"p50": round(float(np.percentile(times, 50)), 4), "p99": round(float(np.percentile(times, 99)), 4)},
        "e2e": {"value": round(value, 3), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 3), "unit": "solves/s", "cores": 1, "kind": "reference",
                         "sample": f"the reference's own CUDA build of GMGSolver::solve (oracle/_ref) on this GPU, "
                                   f"one host thread, {args.steps} full solves timed like FluidEuler::project"},
        "clocks": clocks,
    }


def main():
    args = parse()
    if args.impl == "reference":
        # the reference arm runs on rank 0 only; other ranks exit without work or collectives
        if int(os.environ.get("RANK", "0")) != 0:
            return
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(run_reference(args, 1, 0, int(os.environ.get("LOCAL_RANK", "0")), None)), flush=True)
        return
    world, rank, local, pg = dist_setup(args)
    out = run_ours(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
