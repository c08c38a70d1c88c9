"""Benchmark of the GMG-PCG Poisson solve.  One step = one batched solve: K independent
instances of the workload (K = 32 by default), each to 1e-6 relative residual, in one graph launch.

    python bench.py [--gpus N] [--steps S] [--warmup W] [--batch K] [--impl ours|reference]
                    [--workload NAME]

Default workload: ring512 -- the adaptive 5-level octree with 512x512x1024 effective resolution
(domain 1x1x2, leaves at levels 2-6 refined around a synthetic vortex ring, box obstacle),
seeded synthetic velocity -> divergence right-hand side; instance i of rank r uses velocity seed
r*K + i.  Prints one JSON line on rank 0.

  value     solves/s of the batched solver with inputs resident in HBM (device-timed, CUDA events,
            L2 flushed between steps by writing a 256 MiB buffer)
  e2e       the same through the C ABI with pinned host buffers: every step's H2D of the batch's
            b, solve and D2H of x inside the timed region, pipelined over two grids
            (cirrus_gmg_solve_host_submit/wait: one batch's copies overlap the other's solve);
            e2e.serial is the synchronous cirrus_gmg_solve_host, one step after the other
  latency_ms  one instance solved alone (batch of one): p50/p99 over the steps
  roofline  the dominant kernel (the fused Laplacian, ~a quarter of an iteration): algorithmic
            bytes / CUDA-event duration against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (FP32 mirror of the reference arithmetic, OpenMP) on full solves
            of one instance, about 10 s of work

Multi-GPU (torchrun): replicas only -- every rank solves its own batch; no collective on the
data path; value = all ranks' solves / max-over-ranks time.
--impl reference runs the reference's own CUDA build (oracle/_ref), one solve at a time.
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

# algorithmic bytes of the Laplacian apply: 9 per cell of every launched LEAF|GHOST tile (read x 4
# + cell type 1, write A x 4); the fused kernel's ghost-to-parent accumulation is not credited
LAP_BYTES_PER_CELL = 9
# DRAM bytes (read + write) of one fused-Laplacian launch from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum), per (workload, batch): captured on the 16-instance
# batch; 32 instances of the same topology move twice the bytes (every instance's tiles are
# processed the same way), so that entry is the 16-instance capture doubled
LAP_TRAFFIC_K16 = 336610048 + 66957824
LAP_TRAFFIC_PER_LAUNCH = {("ring512", 16): LAP_TRAFFIC_K16, ("ring512", 32): 2 * LAP_TRAFFIC_K16}


def ghost_parent_tiles(tiles) -> int:
    """LEAF tiles with at least one GHOST child (their A p receives the children's sums after the
    Laplacian, so its p.Ap part is formed by a separate small kernel)."""
    index = {(int(l), int(x), int(y), int(z)) for l, x, y, z, _ in tiles}
    parents = set()
    for l, x, y, z, tp in tiles:
        if tp & 4 and (int(l) - 1, int(x) // 2, int(y) // 2, int(z) // 2) in index:
            parents.add((int(l) - 1, int(x) // 2, int(y) // 2, int(z) // 2))
    return len(parents)


def b_iter_bytes(tiles, pure_neumann: bool = False) -> float:
    """Bytes one PCG iteration moves on the reference's schedule (level_iters 1, coarsest_iters 10),
    from the per-kernel bytes per cell of the reference's kernels: 9 N_LG + 11.5 N_G + 62 N_leaf +
    12 N_all + sum over levels >= 1 of (55 N_l + 19 G_l) + 180 N_0 (+ 14 N_leaf pure Neumann),
    N_* cells of LEAF, GHOST, LEAF|GHOST, all tiles; N_l, G_l cells of LEAF|NONLEAF and GHOST tiles
    at level l."""
    lvl, typ = tiles[:, 0], tiles[:, 4]
    leaf, mg, ghost = (typ & 1) != 0, (typ & 3) != 0, (typ & 4) != 0
    c = 512
    n_leaf, n_g = int(leaf.sum()) * c, int(ghost.sum()) * c
    b = 9 * (n_leaf + n_g) + 11.5 * n_g + 62 * n_leaf + 12 * len(tiles) * c
    for l in range(1, int(lvl.max()) + 1):
        b += 55 * int((mg & (lvl == l)).sum()) * c + 19 * int((ghost & (lvl == l)).sum()) * c
    b += 180 * int((mg & (lvl == 0)).sum()) * c
    if pure_neumann:
        b += 14 * n_leaf
    return b


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--pools", type=int, default=4,
                    help="solve each step's batch as this many grids at once (cirrus_gmg_solve_grids; 1: one grid)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ring512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-batch64", action="store_true", help="skip the 64-instance random-spheres batch")
    ap.add_argument("--no-side-configs", action="store_true", help="skip the uniform128 / sphere256 single-solve lines")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="for a profiler: launch each staged stencil kernel once at the finest level (NVTX range "
                         "'kernels'), then one batched solve with direct kernel launches (NVTX range 'solve'); no timing")
    ap.add_argument("--lap-shape", type=int, default=-1, help="pin the Laplacian's launch shape (0-19) after autotuning")
    ap.add_argument("--shape-sweep", action="store_true",
                    help="time every launch shape of the fused Laplacian and of the four V-cycle stencil kernels at the "
                         "finest level (warm, CUDA events, 40 back-to-back launches, best of 3); one JSON line")
    return ap.parse_args()


class Clocks:
    """NVML sampling (read-only) of the SM clock and clock-event reasons every 10 ms during the
    timed region, in a background thread."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device: int):
        self.device = device
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.thread = None
        self.err = None

    def start(self):
        import threading

        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # NVML missing or device not found: report instead of failing the bench
            self.err = f"nvml unavailable: {type(e).__name__}"
            return
        self.stop_flag = False

        def run():
            while not self.stop_flag:
                try:
                    self.samples.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for n, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(n)
                except Exception:
                    pass
                time.sleep(0.01)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": [self.err or "not sampled"]}
        self.stop_flag = True
        self.thread.join()
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "samples": len(self.samples), "reasons": sorted(self.reasons)}


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
    """The max of a per-rank value over the ranks (the only collective of the replica path)."""
    if pg is None:
        return value
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def batch_seeds(rank: int, batch: int) -> list[int]:
    """Velocity seeds of rank `rank`'s instances: disjoint across ranks (replicas, weak scaling)."""
    return [rank * batch + i for i in range(batch)]


def build_batch(name: str, seeds: list[int]):
    """K instances of one workload topology with their own seeded velocities; projection
    right-hand side in channel 1 and a copy in channel 5."""
    from cirrus_b200 import DeviceGrid, workloads as W

    b = W.build(W.make(name, seeds[0]))
    g = DeviceGrid([b.topology] * len(seeds))
    for i, sd in enumerate(seeds):
        vel = b.velocity if sd == seeds[0] else W.face_velocity(b.tiles, sd)
        for a in range(3):
            g.set_channel_instance(i, 6 + a, vel[a])
    g.projection_rhs()
    return b, g


SERVE_SESSIONS = 16


def run_serving(rank: int, n_requests: int = 96, rates=(100.0, 400.0), slots: int = 8) -> dict:
    """Serving loop under Poisson arrivals over 16 sessions (independent problems) with effective
    sizes log-uniform over 32^3 - 512^3, 1-5 levels of leaves, each refined around a seeded
    sphere or vortex ring (workloads.random_session); each request is the next right-hand side of
    its session (a 1e-3 relative change, as from the next time step), warm-started from the
    session's previous pressure, mixed precision to 1e-6.  Sessions of similar size share batched
    pools and waiting requests are merged into one launch per pool (continuous batching).  Reported
    per arrival rate: throughput, p50/p99 latency (arrival to completion) and requests per launch,
    against the same arrival stream served one at a time by plain FP32 cold solves (service times
    measured, queueing computed from them)."""
    import torch

    from cirrus_b200 import B_CHANNEL, DeviceGrid, GMGSolver, Server, workloads as W

    base = []
    for w in W.serving_sessions(SERVE_SESSIONS, seed0=1000 * rank):
        b = W.build(w)
        g = DeviceGrid(b.topology)
        for a in range(3):
            g.set_channel(6 + a, b.velocity[a])
        g.projection_rhs()
        base.append((b, g.get_channel(B_CHANNEL)))
        g.close()
    out = {"sessions": {b.workload.name: {"tiles": int(b.tiles.shape[0]), "dof": b.dof()} for b, _ in base}, "slots": slots,
           "requests": n_requests, "precision": "mixed (FP32 V-cycle, FP64 defect correction), warm start", "tolerance": 1e-6,
           "rates": []}
    rng = np.random.default_rng(1000 + rank)
    for rate in rates:
        picks = rng.integers(0, len(base), n_requests)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
        bs = [(base[k][1] * (1 + np.float32(1e-3) * rng.standard_normal(base[k][1].shape).astype(np.float32))).astype(np.float32)
              for k in picks]
        srv = Server(40 << 30, slots)
        sids = [srv.add_session(b.topology) for b, _ in base]
        warm = [np.zeros_like(r) for _, r in base]
        for k, x in enumerate(warm):  # each session has solved once before the stream starts
            srv.submit(sids[k], base[k][1], x)
        got = 0
        while got < len(base):
            got += len(srv.poll(wait_ms=1000))
        xs = [np.zeros_like(x) for x in bs]
        t0 = time.perf_counter()
        sub, done = {}, {}
        for i in range(n_requests):
            while time.perf_counter() - t0 < arrivals[i]:
                for c in srv.poll(wait_ms=0):
                    done[c["ticket"]] = c
                time.sleep(0.0002)
            sub[srv.submit(sids[picks[i]], bs[i], xs[i])] = i
        while len(done) < n_requests:
            for c in srv.poll(wait_ms=1000):
                done[c["ticket"]] = c
        span = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        lat = np.array([done[t]["latency_ms"] for t in sub])
        ok = all(done[t]["status"] == 0 and done[t]["rel_residual"] < 1e-6 for t in sub)
        # the same stream one at a time: plain FP32 solves from x = 0 (service times on the GPU)
        grids = [DeviceGrid(b.topology) for b, _ in base]
        solver = GMGSolver()
        stream = torch.cuda.current_stream()
        svc = []
        for i in range(n_requests):
            g = grids[picks[i]]
            g.set_channel(B_CHANNEL, bs[i])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.solve(g, stream=stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            svc.append(e0.elapsed_time(e1))
        for g in grids:
            g.close()
        finish, lat1 = 0.0, []
        for i in range(n_requests):
            finish = max(finish, arrivals[i] * 1e3) + svc[i]
            lat1.append(finish - arrivals[i] * 1e3)
        out["rates"].append({
            "arrival_rate_rps": rate, "throughput_rps": round(n_requests / span, 2),
            "launches": st["launches"], "requests_per_launch": round(st["requests"] / max(st["launches"], 1), 2),
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "all_converged": ok, "peak_resident_gb": round(st["peak_bytes"] / 2**30, 3),
            "one_at_a_time_fp32": {"throughput_rps": round(n_requests / (finish / 1e3), 2),
                                   "p50_ms": round(float(np.percentile(lat1, 50)), 3),
                                   "p99_ms": round(float(np.percentile(lat1, 99)), 3)}})
    return out


def run_batch64(args) -> dict:
    """The batched configuration: 64 independent random-sphere instances (64^3-256^3 effective,
    1-4 levels) per step, held as `--pools` grids (instances dealt round-robin) solved at once in
    mixed precision, each instance to a 1e-6 FP64 true relative residual; autotuned launch shapes
    and smoother sweep counts."""
    import torch

    from cirrus_b200 import B_CHANNEL, KERNEL_LAPLACIAN, PRECISION_MIXED_FP64, TMP_CHANNEL, DeviceGrid, GMGSolver, workloads as W

    bs = [W.build(w) for w in W.batch_of_spheres(64)]
    P = args.pools if args.pools >= 1 and 64 % args.pools == 0 else 1
    pools = []
    for q in range(P):
        mine = bs[q::P]
        g = DeviceGrid([b.topology for b in mine])
        for i, b in enumerate(mine):
            for a in range(3):
                g.set_channel_instance(i, 6 + a, b.velocity[a])
        g.projection_rhs()
        g.autotune()
        g.copy_channel(TMP_CHANNEL, B_CHANNEL)
        pools.append(g)
    stream = torch.cuda.current_stream()
    s = GMGSolver(precision=PRECISION_MIXED_FP64)
    # smoother sweep counts from the sweep tuner (timed trial solves of the first grid)
    li, ci = s.autotune_sweeps(pools[0], stream=stream.cuda_stream)
    times = []
    for i in range(args.warmup + args.steps):
        for g in pools:
            g.copy_channel(B_CHANNEL, TMP_CHANNEL, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.solve_grids(pools, stream=stream.cuda_stream, level_iters=li, coarsest_iters=ci)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1))
    res = list(s.last_results)
    lap_shape = pools[0].get_launch_shape(KERNEL_LAPLACIAN, 0)  # 8-11: the TMA-staged pipeline
    dof = sum(g.instance_dof(i) for g in pools for i in range(g.num_instances))
    for g in pools:
        g.close()
    value = 64 * len(times) / (sum(times) * 1e-3)
    return {"value": round(value, 2), "unit": "solves/s", "instances": 64, "pools": P,
            "tiles": int(sum(b.tiles.shape[0] for b in bs)),
            "mdof_per_s": round(dof / 64 * value / 1e6, 1), "ms_per_batch": round(float(np.mean(times)), 3),
            "all_converged": all(r.status == 0 and r.true_rel_residual < 1e-6 for r in res),
            "max_pcg_iters": int(max(r.iters for r in res)), "precision": "mixed, 1e-6 FP64 true residual",
            "sweeps": {"level_iters": li, "coarsest_iters": ci, "source": "sweep tuner"},
            "laplacian_launch_shape": lap_shape}


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


# PoissonTile<float> as the reference's grid holds it in device memory: 33,104-byte records,
# channel c at float offset 736 c, the 512 cell-type bytes at byte 32,576 (the layout the
# tile-holder files use too)
TILE_RECORD_BYTES, TILE_CHANNEL_STRIDE, TILE_CELLTYPE_OFFSET = 33104, 736, 32576


def dropin_call_site(args, g1, ctypes_host, sh) -> dict:
    """The drop-in's work at FluidEuler::project's call site (src/FluidEuler.h:591-601), one
    instance: the reference keeps its tiles as separate device records, and a fresh solver object
    per projection compares their cell types with the bound pool's on the device, gathers b from
    the records, solves, and scatters x and the residual back (the C ABI calls
    include/cirrus_gmg_dropin.hpp makes after its first bind), timed with the host clock around the
    whole call as FluidEuler::project times the solve."""
    import ctypes as C
    import torch

    from cirrus_b200 import B_CHANNEL, GMGSolver, lib

    n = g1.num_tiles
    rec = torch.zeros(n * TILE_RECORD_BYTES, dtype=torch.uint8, device="cuda")
    f32 = rec.view(torch.float32).view(n, TILE_RECORD_BYTES // 4)
    b = torch.from_numpy(g1.get_channel(B_CHANNEL)).cuda()
    f32[:, TILE_CHANNEL_STRIDE:TILE_CHANNEL_STRIDE + 512] = b
    ct = torch.from_numpy(np.ascontiguousarray(ctypes_host, dtype=np.uint8).reshape(n, 512)).cuda()
    rec.view(n, TILE_RECORD_BYTES)[:, TILE_CELLTYPE_OFFSET:TILE_CELLTYPE_OFFSET + 512] = ct
    base = rec.data_ptr()
    ptrs = (C.c_void_p * n)(*[base + i * TILE_RECORD_BYTES for i in range(n)])
    L = lib()
    assert L.cirrus_grid_set_tile_pointers(g1.handle, ptrs) == 0
    solver = GMGSolver()
    changed = C.c_int()
    times, iters = [], []
    torch.cuda.synchronize()
    for i in range(args.warmup + args.steps):
        f32[:, TILE_CHANNEL_STRIDE:TILE_CHANNEL_STRIDE + 512] = b  # the reference's next right-hand side
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        assert L.cirrus_grid_compare_tile_cell_types(g1.handle, TILE_CELLTYPE_OFFSET, C.c_void_p(sh), C.byref(changed), None) == 0
        assert L.cirrus_grid_gather_tiles(g1.handle, 1, TILE_CHANNEL_STRIDE * 4, C.c_void_p(sh)) == 0
        solver.solve(g1, stream=sh)
        assert L.cirrus_grid_scatter_tiles(g1.handle, 0, 0, C.c_void_p(sh)) == 0
        assert L.cirrus_grid_scatter_tiles(g1.handle, 1, TILE_CHANNEL_STRIDE * 4, C.c_void_p(sh)) == 0
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append((time.perf_counter() - t0) * 1e3)
            iters.append(solver.last_result.iters)
        assert changed.value == 0
    return {"value": round(1e3 / float(np.mean(times)), 3), "unit": "solves/s", "p50_ms": round(float(np.percentile(times, 50)), 4),
            "iters": int(max(iters)),
            "api": "cirrus_grid_compare_tile_cell_types + cirrus_grid_gather_tiles + cirrus_gmg_solve + cirrus_grid_scatter_tiles x2 "
                   "on tiles held as separate PoissonTile<float> device records (one instance, host clock around the call)",
            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 4}


def run_ours(args, world, rank, local, pg):
    import torch

    from cirrus_b200 import (B_CHANNEL, KERNEL_GS_SWEEP, KERNEL_LAPLACIAN, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP,
                             KERNEL_RESIDUAL_RESTRICT, TMP_CHANNEL, U_CHANNEL, DeviceGrid, GMGSolver)

    K = args.batch
    P = args.pools if args.pools >= 1 and K % args.pools == 0 else 1
    seeds = batch_seeds(rank, K)
    b, g = build_batch(args.workload, seeds)
    g.autotune()  # launch shapes per kernel and level for this grid (results unchanged)
    rhs = g.get_channel(B_CHANNEL)
    g.copy_channel(TMP_CHANNEL, B_CHANNEL)  # keep b resident for restoring between steps
    # the step's batch as P grids of K/P instances solved at once, each grid's solve graph on its
    # own stream (cirrus_gmg_solve_grids): one grid's latency-bound coarse levels overlap another's
    # large launches
    pools = [g]
    if P > 1:
        pools = [build_batch(args.workload, seeds[q * K // P:(q + 1) * K // P])[1] for q in range(P)]
        for gp in pools:
            gp.autotune()
            gp.copy_channel(TMP_CHANNEL, B_CHANNEL)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    solver = GMGSolver()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    iters_seen, launches = [], []

    def check_converged(res):
        worst = max(r[1] for r in res)
        if worst >= 1e-6:
            raise RuntimeError(f"solve did not converge: rel {worst}")

    def one():
        for gp in pools:
            gp.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = [r for pr in solver.solve_grids(pools, stream=sh) for r in pr]
        e1.record(stream)
        torch.cuda.synchronize()
        iters_seen.extend(r[0] for r in res)
        # each result carries its grid's whole launch count: one per pool
        launches.append(sum(solver.last_results[q * (K // P)].kernel_launches for q in range(P)))
        worst = max(r[1] for r in res)
        if worst >= 1e-6:
            raise RuntimeError(f"solve did not converge: rel {worst}")
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        one()
    iters_seen.clear()
    launches.clear()
    clocks = None
    clk = Clocks(local)
    if rank == 0:
        clk.start()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed solves
    times = [one() for _ in range(args.steps)]
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if rank == 0:
        clocks = clk.stop()
    total_ms = barrier_max(pg, sum(times))

    # end to end: host buffers through the public C ABI.  Serial: cirrus_gmg_solve_host (H2D of the
    # batch's b, solve, D2H of x, return).  Pipelined (the reported e2e): two grids holding the
    # same batch, each with its own stream, cirrus_gmg_solve_host_submit/wait alternating between
    # them, so that one batch's copies overlap the other batch's solve; every step still copies its
    # b from pinned host memory and its x back to pinned host memory inside the timed region.
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
    e2e_serial_total = barrier_max(pg, sum(e2e_times))

    # two sets of the step's grids (the pools, and as many grids again with the same topologies and
    # launch shapes), each grid with its own stream and pinned host buffers
    tuned = (KERNEL_LAPLACIAN, KERNEL_GS_SWEEP, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT)
    twins = []
    for gp in pools:
        gq = DeviceGrid([b.topology] * gp.num_instances)
        for kern in tuned:
            for lv in range(b.topology.num_layers):
                gq.set_launch_shape(gp.get_launch_shape(kern, lv), kern, lv)
        twins.append(gq)
    sets = [pools, twins]
    side = [[torch.cuda.Stream() for _ in range(P)] for _ in range(2)]
    streams = [[sh] + [s.cuda_stream for s in side[0][1:]], [s.cuda_stream for s in side[1]]]
    hosts = []
    for _ in range(2):
        hs = []
        for gp in pools:
            bh = torch.from_numpy(gp.get_channel(TMP_CHANNEL).reshape(-1)).pin_memory()
            hs.append((bh.numpy(), torch.empty_like(bh).pin_memory().numpy()))
        hosts.append(hs)
    step_bytes = sum(h[0].nbytes for h in hosts[0])

    def e2e_pipeline(steps):
        pending = [False, False]
        for k in range(steps):
            j = k % 2
            if pending[j]:
                for gq in sets[j]:
                    check_converged(solver.solve_host_wait(gq))
            for q, gq in enumerate(sets[j]):
                solver.solve_host_submit(gq, *hosts[j][q], stream=streams[j][q])
            pending[j] = True
        for j in (0, 1):
            if pending[j]:
                for gq in sets[j]:
                    check_converged(solver.solve_host_wait(gq))

    e2e_pipeline(4)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    t0 = time.perf_counter()
    e2e_pipeline(args.steps)
    e2e_total = barrier_max(pg, (time.perf_counter() - t0) * 1e3)
    for gq in twins:
        gq.close()

    # roofline of the dominant kernel (fused Laplacian over the batch's LEAF|GHOST tiles), timed
    # with CUDA events on the stream it is launched on
    g.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
    g.copy_channel(2, B_CHANNEL, sh)
    reps = 50
    g.bench_launch(KERNEL_LAPLACIAN, 0, 5, stream=sh)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.bench_launch(KERNEL_LAPLACIAN, 0, reps, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    lap_ms = e0.elapsed_time(e1) / reps
    n_leaf = int(((b.tiles[:, 4] & 1) != 0).sum()) * K
    n_ghost = int(((b.tiles[:, 4] & 4) != 0).sum()) * K
    lap_bytes = (n_leaf + n_ghost) * 512 * LAP_BYTES_PER_CELL
    pap_bytes = (n_leaf - ghost_parent_tiles(b.tiles) * K) * 512 * 8
    peaks = measured_peaks()
    achieved = lap_bytes / (lap_ms * 1e-3) / 1e9
    biter = b_iter_bytes(b.tiles)

    # the V-cycle's stencil kernels at the finest level, each against the survey's bytes per cell
    # of the reference kernels it performs (fusion-credited: the pre-smoother is two colour
    # sweeps, the prolongation kernel a prolongation + update and one colour)
    typ, lvl = b.tiles[:, 4], b.tiles[:, 0]
    lmax = int(lvl.max())
    n_mg = int((((typ & 3) != 0) & (lvl == lmax)).sum()) * K * 512
    n_gh = int((((typ & 4) != 0) & (lvl == lmax)).sum()) * K * 512
    n_lf = int((((typ & 1) != 0) & (lvl == lmax)).sum()) * K * 512
    stencil = []
    for name, kern, nbytes in [("k_presmooth (2 colours from x = 0)", KERNEL_PRESMOOTH, 18 * n_mg),
                               ("k_residual_restrict", KERNEL_RESIDUAL_RESTRICT, 9.5 * (n_mg + n_gh)),
                               ("k_prolong_sweep (prolongation + 1 colour)", KERNEL_PROLONG_SWEEP, 9.5 * (n_mg + n_gh) + 9 * n_mg),
                               # the last colour sweep also forms the r.z tile parts of its LEAF tiles,
                               # the work of the reference's separate Dot pass over r and z (8 B per cell)
                               ("k_gs_sweep (1 colour + r.z tile parts)", KERNEL_GS_SWEEP, 9 * n_mg + 8 * n_lf)]:
        g.bench_launch(kern, lmax, 4, stream=sh)
        e0.record(stream)
        g.bench_launch(kern, lmax, reps, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        us = e0.elapsed_time(e1) / reps * 1e3
        gbs = nbytes / (us * 1e-6) / 1e9
        stencil.append({"kernel": name, "level": lmax, "cells": n_mg, "algorithmic_bytes_per_launch": int(nbytes),
                        "launch_us": round(us, 2), "achieved": round(gbs, 1), "unit": "GB/s", "frac": round(gbs / peaks["hbm_gbs"], 4)})
    g.copy_channel(TMP_CHANNEL, B_CHANNEL, sh)  # the kernel launches overwrote channels 2-5, TMP held b

    # the mixed-precision batched solver (FP32 V-cycle and matvec, FP64 residual and defect
    # correction) to the same 1e-6 on the same batch, FP64 true residual checked per instance
    from cirrus_b200 import PRECISION_MIXED_FP64

    msolver = GMGSolver(precision=PRECISION_MIXED_FP64)
    mtimes, mres = [], []
    for i in range(args.warmup + args.steps):
        for gp in pools:
            gp.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        msolver.solve_grids(pools, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            mtimes.append(e0.elapsed_time(e1))
            mres = list(msolver.last_results)
    mixed_total = barrier_max(pg, sum(mtimes))
    if max(r.true_rel_residual for r in mres) >= 1e-6:
        raise RuntimeError("mixed-precision solve did not reach 1e-6")
    # the same with the smoother sweep counts of the sweep tuner (timed trial solves of this batch;
    # the FP64 tolerance fixes the result, so the preconditioner is free)
    g.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
    tli, tci = msolver.autotune_sweeps(g, stream=sh)
    ttimes, tres = [], []
    for i in range(args.warmup + args.steps):
        for gp in pools:
            gp.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        msolver.solve_grids(pools, stream=sh, level_iters=tli, coarsest_iters=tci)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            ttimes.append(e0.elapsed_time(e1))
            tres = list(msolver.last_results)
    tuned_total = barrier_max(pg, sum(ttimes))
    if max(r.true_rel_residual for r in tres) >= 1e-6:
        raise RuntimeError("sweep-tuned mixed-precision solve did not reach 1e-6")

    # the AMG variant (AMGSolver: explicit coefficients, coarse levels from the children) on the
    # same batch, FP32 to the same 1e-6
    from cirrus_b200 import AMGSolver

    asolver = AMGSolver()
    # its V-cycle uses channel 5 (which holds b between steps here) as scratch: b waits in channel 6
    for gp in pools:
        gp.copy_channel(U_CHANNEL, TMP_CHANNEL, sh)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    asolver.prepare_types_and_coeffs(pools[0], stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    amg_prepare_ms = e0.elapsed_time(e1)
    for gp in pools[1:]:
        asolver.prepare_types_and_coeffs(gp, stream=sh)
    atimes, ares = [], []
    for i in range(args.warmup + args.steps):
        for gp in pools:
            gp.copy_channel(B_CHANNEL, U_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        asolver.solve_grids(pools, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            atimes.append(e0.elapsed_time(e1))
            ares = list(asolver.last_results)
    amg_total = barrier_max(pg, sum(atimes))
    for gp in pools:
        gp.copy_channel(TMP_CHANNEL, U_CHANNEL, sh)
    if not all(r.status == 0 for r in ares):
        raise RuntimeError("AMG solve did not converge")

    # one instance alone (batch of one): latency
    b1, g1 = build_batch(args.workload, [rank * K])
    g1.autotune()
    g1.copy_channel(TMP_CHANNEL, B_CHANNEL)
    lat = []
    for i in range(args.warmup + args.steps):
        g1.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.solve(g1, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            lat.append(e0.elapsed_time(e1))
    single_iters = solver.last_result.iters
    g1.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)  # the solves left the residual in channel 1: b again
    dropin = dropin_call_site(args, g1, b1.ctypes, sh)
    if dropin["iters"] != single_iters:
        raise RuntimeError(f"drop-in call site solved in {dropin['iters']} iterations, the grid's own solve in {single_iters}")

    n = args.steps * world * K
    value = n / (total_ms * 1e-3)
    dof = g.dof // K
    maxl = int(b.tiles[:, 0].max())
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
        "config": bench_config(args.workload, K, b.tiles, b.ctypes, world),
        "mdof_per_s": round(dof * value / 1e6, 2),
        "iters_per_solve": int(statistics.median(iters_seen)),
        "latency_ms": {"single_p50": round(float(np.percentile(lat, 50)), 4), "single_p99": round(float(np.percentile(lat, 99)), 4),
                       "batch_p50": round(float(np.percentile(times, 50)), 4), "batch_p99": round(float(np.percentile(times, 99)), 4)},
        "single_solves_per_s": round(1e3 / float(np.mean(lat)), 3),
        "dropin_e2e": dropin,
        "mixed_precision": {"value": round(args.steps * world * K / (mixed_total * 1e-3), 3), "unit": "solves/s",
                            "precision": "FP32 V-cycle + matvec, FP64 residual and defect correction",
                            "tolerance": "1e-6 FP64 true relative residual per instance",
                            "pcg_iters_per_solve": int(statistics.median(r.iters for r in mres)),
                            "outer_iters_per_solve": int(statistics.median(r.outer_iters for r in mres)),
                            "max_true_rel_residual": float(max(r.true_rel_residual for r in mres)),
                            "sweep_tuned": {"value": round(args.steps * world * K / (tuned_total * 1e-3), 3), "unit": "solves/s",
                                            "sweeps": {"level_iters": tli, "coarsest_iters": tci, "source": "sweep tuner"},
                                            "pcg_iters_per_solve": int(statistics.median(r.iters for r in tres)),
                                            "max_true_rel_residual": float(max(r.true_rel_residual for r in tres))}},
        "amg_variant": {"value": round(args.steps * world * K / (amg_total * 1e-3), 3), "unit": "solves/s",
                        "solver": "AMGSolver (explicit face coefficients, coarse levels from the children), FP32 to 1e-6, "
                                  "the pools solved at once (cirrus_amg_solve_grids)",
                        "pcg_iters_per_solve": int(statistics.median(r.iters for r in ares)),
                        "prepare_ms": round(amg_prepare_ms, 3)},
        "gpu_launches": int(sum(launches)),
        "schedule": {"pools": P, "instances_per_pool": K // P,
                     "api": "cirrus_gmg_solve_grids: the step's instances as grids solved at once, each on its own stream"},
        "e2e": {"value": round(n / (e2e_total * 1e-3), 3), "unit": "solves/s",
                "h2d_bytes_per_step": int(step_bytes), "d2h_bytes_per_step": int(step_bytes),
                "api": f"cirrus_gmg_solve_host_submit/wait, two sets of {P} grid(s) of {K // P} instances alternating (copies of "
                       "one step's batch overlap the other set's solves; a set's grids solve at once on their own streams)",
                "serial": {"value": round(n / (e2e_serial_total * 1e-3), 3), "api": "cirrus_gmg_solve_host (copy, solve, copy, return)"}},
        "roofline": {"kernel": f"k_laplacian_fused ({K} instances, {n_leaf} LEAF + {n_ghost} GHOST tiles)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": int(lap_bytes), "bytes_per_cell": LAP_BYTES_PER_CELL,
                     "launch_us": round(lap_ms * 1e3, 3), "traffic": LAP_TRAFFIC_PER_LAUNCH.get((args.workload, K)),
                     "fusion_credited": {"bytes_per_launch": int(lap_bytes + pap_bytes),
                                         "achieved": round((lap_bytes + pap_bytes) / (lap_ms * 1e-3) / 1e9, 1),
                                         "frac": round((lap_bytes + pap_bytes) / (lap_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4),
                                         "note": "adds the p.Ap dot the launch forms for LEAF tiles without GHOST children "
                                                 "(8 B per cell: the reference's separate Dot pass over p and Ap)"}},
        "stencil_kernels": stencil,
        "laplacian_launch_shape": g.get_launch_shape(KERNEL_LAPLACIAN, 0),
        "whole_solve_bandwidth": {"value": round(biter * sum(iters_seen) / (total_ms * 1e-3) / 1e9, 1), "unit": "GB/s per GPU",
                                  "fusion_credited": True, "bytes_per_iteration_per_instance": int(biter),
                                  "frac_of_peak": round(biter * sum(iters_seen) / (total_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4)},
        "reference_log_figure": {"value": round(value * int(b.tiles.shape[0]) * 512 / 2**20, 1),
                                 "unit": "Mcells/s (numTotalTiles*512/2^20 per solve time, as FluidEuler prints, times solves)"},
        "clocks": clocks,
    }
    g1.close()
    if not args.no_side_configs:
        # the other configurations, one instance per solve as the reference arm runs them (C1:
        # uniform 128^3; C2: 3-level sphere, 256^3 effective), plain FP32 to 1e-6, device-timed
        out["side_configs"] = {}
        for name in SIDE_CONFIGS:
            sb, sg = build_batch(name, [0])
            sg.autotune()
            sg.copy_channel(TMP_CHANNEL, B_CHANNEL)
            ts, its = [], []
            for i in range(args.warmup + args.steps):
                sg.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                it, rel = solver.solve(sg, stream=sh)
                e1.record(stream)
                torch.cuda.synchronize()
                if not rel < 1e-6:
                    raise RuntimeError(f"{name}: solve did not converge: rel {rel}")
                if i >= args.warmup:
                    ts.append(e0.elapsed_time(e1))
                    its.append(it)
            sv = 1e3 / float(np.mean(ts))
            out["side_configs"][name] = {"solves_per_s": round(sv, 3), "mdof_per_s": round(sg.dof * sv / 1e6, 2),
                                         "tiles": int(sb.tiles.shape[0]), "dof": int(sg.dof), "iters": int(statistics.median(its)),
                                         "p50_ms": round(float(np.percentile(ts, 50)), 4)}
            sg.close()
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        rhs1 = rhs[: b.tiles.shape[0]] if K == 1 else g.get_channel_instance(0, TMP_CHANNEL)
        cb = cpu_baseline(b, rhs1)
        out["cpu_baseline"] = {"value": round(cb["solves"] / cb["seconds"], 4), "unit": "solves/s", "cores": cb["threads"],
                               "kind": "port",
                               "sample": f"{cb['solves']} full solves of one {args.workload} instance to 1e-6 ({cb['iters']} "
                                         f"PCG iterations each) by the CPU oracle (FP32 mirror of the reference "
                                         f"arithmetic, OpenMP), {cb['seconds']:.1f} s wall"}
    g.close()
    if rank == 0 and not args.no_serve:
        out["serving"] = run_serving(rank)
    if rank == 0 and not args.no_batch64:
        out["batch64_spheres"] = run_batch64(args)
    return out


def bench_config(workload: str, K: int, tiles: np.ndarray, ctypes: np.ndarray, world: int) -> dict:
    """The `config` of both arms' lines: the same dict for the same workload, batch and ranks."""
    leaf = (tiles[:, 4] & 1) != 0
    dof = int(((ctypes[leaf] & 2) != 0).sum())
    maxl = int(tiles[:, 0].max())
    return {"workload": f"{workload} x{K} batch", "instances_per_step": K, "tiles_per_instance": int(tiles.shape[0]),
            "dof_per_instance": dof,
            "effective_resolution": "512x512x1024" if workload == "ring512" else workload,
            "levels": f"leaves {int(tiles[leaf, 0].min())}-{maxl}",
            "tolerance": 1e-6, "stopping_rule": "recursive ||r||/||b|| < tol per instance, checked every iteration",
            "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"}


# the other configurations measured beside the headline one: one instance per solve (C1, C2)
SIDE_CONFIGS = ["uniform128", "sphere256"]


def ref_instance(name: str, seed: int):
    """A reference grid of workload `name` built by the reference's own code (oracle/_ref):
    tiles and neighbours from its IterativeRefine and CalculateNeighborTiles, the leaf cell-type
    rule from the workload definition (numpy), CalcCellTypesFromLeafs by the reference."""
    from oracle import oracle as O

    from cirrus_b200 import workloads as W  # workload geometry and seeded velocities (numpy only)

    w = W.make(name, seed=seed)
    ref = O.RefHarness(w)
    tiles = ref.tiles()
    ref.calc_neighbors()
    nbr6 = ref.neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, tiles, nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    return w, ref, tiles, ref.ctypes()


def run_reference(args, world, rank, local, pg):
    """The reference's own CUDA build (oracle/_ref/libcirrus_ref.so, which links nothing of this
    project) on the same workload and batch as the product arm: each step solves the same K
    instances (velocity seeds rank*K + i) one after another through the reference's stock
    GMGSolver::solve, each timed as FluidEuler::project times it (src/FluidEuler.h:595-601: host
    clock around the call, device synchronised on both sides); the right-hand side of each
    instance is loaded and L2 flushed before its solve, outside the timed call."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libcirrus_ref.so was not built (needs the reference tree)"}
    import torch

    from cirrus_b200 import workloads as W

    K = args.batch
    w, ref, tiles, ct = ref_instance(args.workload, batch_seeds(rank, K)[0])
    rhs = [ref.rhs(W.face_velocity(tiles, sd)) for sd in batch_seeds(rank, K)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    solve_ms, iters = [], []

    def one_step():
        total = 0.0
        for b in rhs:
            ref.set_channel(1, b)
            flush.zero_()
            torch.cuda.synchronize()
            it, rel, ms = ref.solve(1000, 1e-6, 1, 10, 1, w.pure_neumann)
            if not rel < 1e-6:
                raise RuntimeError(f"reference solve did not converge: rel {rel}")
            iters.append(it)
            solve_ms.append(ms)
            total += ms
        return total

    for _ in range(args.warmup):
        one_step()
    iters.clear()
    solve_ms.clear()
    clk = Clocks(local)
    if rank == 0:
        clk.start()
    times = [one_step() for _ in range(args.steps)]
    clocks = clk.stop() if rank == 0 else None
    total = sum(times)
    n = args.steps * world * K
    value = n / (total * 1e-3)
    cfg = bench_config(args.workload, K, tiles, ct, world)
    out = {
        "impl": "reference",
        "metric": "Poisson solves/s to 1e-6 relative residual (GMG-PCG, reference arithmetic)",
        "value": round(value, 3), "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total / args.steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (fp64 CG scalars)", "data": "synthetic (seeded face velocities, divergence right-hand side)",
        "config": cfg,
        "mdof_per_s": round(cfg["dof_per_instance"] * value / 1e6, 2), "iters_per_solve": int(statistics.median(iters)),
        "latency_ms": {"single_p50": round(float(np.percentile(solve_ms, 50)), 4),
                       "single_p99": round(float(np.percentile(solve_ms, 99)), 4),
                       "batch_p50": round(float(np.percentile(times, 50)), 4), "batch_p99": round(float(np.percentile(times, 99)), 4)},
        "single_solves_per_s": round(1e3 / float(np.mean(solve_ms)), 3),
        "e2e": {"value": round(value, 3), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 3), "unit": "solves/s", "cores": 1, "kind": "reference",
                         "sample": f"the reference's own CUDA build of GMGSolver::solve (oracle/_ref) on this GPU, one host "
                                   f"thread, {args.steps} steps of {K} full solves, each timed like FluidEuler::project"},
        "clocks": clocks,
    }
    del ref
    if not args.no_side_configs:
        out["side_configs"] = {}
        for name in SIDE_CONFIGS:
            sw, sref, st, sct = ref_instance(name, 0)
            srhs = sref.rhs(W.face_velocity(st, 0))
            ms_list, its = [], []
            for i in range(args.warmup + args.steps):
                sref.set_channel(1, srhs)
                flush.zero_()
                torch.cuda.synchronize()
                it, rel, ms = sref.solve(1000, 1e-6, 1, 10, 1, sw.pure_neumann)
                if i >= args.warmup:
                    ms_list.append(ms)
                    its.append(it)
            leaf = (st[:, 4] & 1) != 0
            dof = int(((sct[leaf] & 2) != 0).sum())
            sv = 1e3 / float(np.mean(ms_list))
            out["side_configs"][name] = {"solves_per_s": round(sv, 3), "mdof_per_s": round(dof * sv / 1e6, 2), "tiles": int(st.shape[0]),
                                         "dof": dof, "iters": int(statistics.median(its)),
                                         "p50_ms": round(float(np.percentile(ms_list, 50)), 4)}
            del sref
    return out


def profile_kernels(args):
    """The launches a profiler captures: the workload's batch built and autotuned as the bench does,
    then inside NVTX range 'kernels' the fused Laplacian and the four V-cycle stencil kernels at the
    finest level once each, and inside NVTX range 'solve' one batched solve launched kernel by kernel
    (a CUDA graph with a conditional node is not followed by every profiler)."""
    import torch

    from cirrus_b200 import (B_CHANNEL, KERNEL_GS_SWEEP, KERNEL_LAPLACIAN, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP,
                             KERNEL_RESIDUAL_RESTRICT, TMP_CHANNEL, GMGSolver)

    b, g = build_batch(args.workload, batch_seeds(0, args.batch))
    g.autotune()
    if args.lap_shape >= 0:
        g.set_launch_shape(args.lap_shape, KERNEL_LAPLACIAN)
    g.copy_channel(TMP_CHANNEL, B_CHANNEL)
    sh = torch.cuda.current_stream().cuda_stream
    lmax = int(b.tiles[:, 0].max())
    g.copy_channel(2, B_CHANNEL, sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("kernels")
    g.bench_launch(KERNEL_LAPLACIAN, 0, 1, stream=sh)
    for kern in (KERNEL_PRESMOOTH, KERNEL_RESIDUAL_RESTRICT, KERNEL_PROLONG_SWEEP, KERNEL_GS_SWEEP):
        g.bench_launch(kern, lmax, 1, stream=sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    g.copy_channel(B_CHANNEL, TMP_CHANNEL, sh)
    g.set_launch_mode(True)
    torch.cuda.nvtx.range_push("solve")
    GMGSolver().solve_batch(g, stream=sh)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    g.close()


def shape_sweep(args) -> dict:
    """Per staged kernel and launch shape, the warm time of one launch over the workload's batch:
    the data the autotuner chooses from (shapes never change results)."""
    import torch

    from cirrus_b200 import (KERNEL_GS_SWEEP, KERNEL_LAPLACIAN, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT,
                             lib)

    b, g = build_batch(args.workload, batch_seeds(0, args.batch))
    rng = np.random.default_rng(0)
    for c in (2, 3, 4):  # the channels the kernels read in cirrus_bench_launch
        g.set_channel(c, rng.standard_normal((g.num_tiles, 512)).astype(np.float32))
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    lmax = int(b.tiles[:, 0].max())
    out = {"workload": args.workload, "instances": args.batch, "level": lmax, "unit": "us per launch", "kernels": {}}
    for name, kern, level in (("k_laplacian_fused", KERNEL_LAPLACIAN, 0), ("k_gs_sweep", KERNEL_GS_SWEEP, lmax),
                              ("k_presmooth", KERNEL_PRESMOOTH, lmax), ("k_prolong_sweep", KERNEL_PROLONG_SWEEP, lmax),
                              ("k_residual_restrict", KERNEL_RESIDUAL_RESTRICT, lmax)):
        res = {}
        shape = 0
        while lib().cirrus_grid_set_launch_shape(g.handle, kern, level, shape) == 0:
            g.bench_launch(kern, level, 4, stream=sh)
            ts = []
            for _ in range(3):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.bench_launch(kern, level, 40, stream=sh)
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1) / 40 * 1e3)
            res[str(shape)] = round(min(ts), 2)
            shape += 1
        out["kernels"][name] = res
    g.close()
    return out


def main():
    args = parse()
    if args.shape_sweep:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(shape_sweep(args)), flush=True)
        return
    if args.profile_kernels:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        profile_kernels(args)
        return
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
