"""Serving loop: sessions submitted as they arrive, run concurrently on slots, admitted against an
HBM budget, warm-started from their previous pressure.  Every session's solves are deterministic
and independent of the other sessions, so each result is bit-identical alone (one slot, one
request at a time) and in the mix (several slots, all requests queued at once); eviction under a
tight budget keeps the pressure on the host, so warm starts and results are unchanged too."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, Server, workloads as W

pytestmark = pytest.mark.gpu

NAMES = ["sphere64_small", "ring64_small", "uniform32_small"]
BUDGET_OK = 1 << 34


def rhs_of(b):
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    g.close()
    return rhs


def estimate(b):
    return b.tiles.shape[0] * (512 * (10 * 4 + 3 * 8 + 4 + 3) + 512) + (4 << 20)


def requests(built_cache, sessions=None):
    """Two solves per session: b, then a perturbed b (the second starts warm).  sessions: built
    workloads (default: NAMES)."""
    out = []
    for b in sessions or [built_cache(n) for n in NAMES]:
        r0 = rhs_of(b)
        rng = np.random.default_rng(len(out))
        # the next right-hand side of the same problem, as from the next time step: 1e-3 relative change
        r1 = (r0 * (1 + np.float32(1e-3) * rng.standard_normal(r0.shape).astype(np.float32))).astype(np.float32)
        out.append((b, [r0, r1]))
    return out


def run(reqs, slots, budget, together, deadline_s=120.0, pool_size=8):
    import time

    t_end = time.monotonic() + deadline_s
    srv = Server(budget, slots, pool_size)
    sids = [srv.add_session(b.topology) for b, _ in reqs]
    xs, done = {}, {}
    order = [(s, k) for k in range(2) for s in range(len(reqs))]  # interleaved sessions
    for s, k in order:
        b, rhs = reqs[s]
        x = np.zeros_like(rhs[k])
        t = srv.submit(sids[s], rhs[k], x)
        xs[t] = (s, k, x)
        if not together:
            while t not in done:
                assert time.monotonic() < t_end, "serving loop made no progress"
                for c in srv.poll(wait_ms=1000):
                    done[c["ticket"]] = c
    while len(done) < len(order):
        assert time.monotonic() < t_end, "serving loop made no progress"
        for c in srv.poll(wait_ms=1000):
            done[c["ticket"]] = c
    stats = srv.stats()
    srv.close()
    res = {}
    for t, (s, k, x) in xs.items():
        res[(s, k)] = (done[t], x)
    return res, stats


@pytest.mark.parametrize("mix", ["fixed", "random_sessions"])
def test_serve_same_alone_and_in_mix_with_warm_starts(built_cache, mix):
    """fixed: three small named workloads; random_sessions: four problems of the serving
    configuration's generator (sizes log-uniform 32^3-512^3, 1-5 levels, sphere or vortex-ring
    refinement; the small draws, seeds 1, 2, 3 and 9)."""
    sessions = None if mix == "fixed" else [W.build(W.random_session(s)) for s in (1, 2, 3, 9)]
    reqs = requests(built_cache, sessions)
    alone, _ = run(reqs, 1, BUDGET_OK, together=False)
    mix, st = run(reqs, 4, BUDGET_OK, together=True)
    for key, (c, x) in alone.items():
        c2, x2 = mix[key]
        assert c["status"] == 0 and c2["status"] == 0
        assert c["rel_residual"] < 1e-6
        assert c["warm"] == (1 if key[1] == 1 else 0) == c2["warm"]
        assert (c["iters"], c["outer_iters"]) == (c2["iters"], c2["outer_iters"])
        assert np.array_equal(x.view(np.uint32), x2.view(np.uint32))
    # a warm start from the previous pressure needs fewer PCG iterations than the cold solve
    for s in range(len(reqs)):
        assert alone[(s, 1)][0]["iters"] < alone[(s, 0)][0]["iters"]
    assert st["resident_sessions"] == len(reqs) and st["evictions"] == 0


def test_serve_budget_admission_evicts_and_keeps_results(built_cache):
    reqs = requests(built_cache)
    ref, _ = run(reqs, 2, BUDGET_OK, together=True)
    budget = max(estimate(b) for b, _ in reqs) + (1 << 20)  # room for one session at a time
    # one session per pool, so that the budget admits one pool at a time; the results are those
    # of the shared pools above
    tight, st = run(reqs, 2, budget, together=True, pool_size=1)
    assert st["peak_bytes"] <= budget and st["evictions"] > 0
    for key, (c, x) in ref.items():
        c2, x2 = tight[key]
        assert c2["status"] == 0
        assert np.array_equal(x.view(np.uint32), x2.view(np.uint32))


def test_serve_refuses_a_session_larger_than_the_budget(built_cache):
    b = built_cache("sphere64_small")
    rhs = rhs_of(b)
    srv = Server(estimate(b) // 2, 1)
    s = srv.add_session(b.topology)
    x = np.zeros_like(rhs)
    t = srv.submit(s, rhs, x)
    c = srv.poll(wait_ms=5000)
    srv.close()
    assert len(c) == 1 and c[0]["ticket"] == t and c[0]["status"] == 7


def test_serve_merges_waiting_requests_into_one_launch(built_cache):
    """Requests of several sessions queued while their shared pool is busy are solved in one
    batched launch (fewer launches than requests, each completion reporting its batch), with the
    bits of each request solved alone."""
    sessions = [W.build(W.random_session(s)) for s in (1, 2, 3, 9)]
    reqs = requests(built_cache, sessions)
    alone, _ = run(reqs, 1, BUDGET_OK, together=False)
    srv = Server(BUDGET_OK, 1, 8)
    sids = [srv.add_session(b.topology) for b, _ in reqs]
    xs, done = {}, {}
    for s, (b, rhs) in enumerate(reqs):  # every session's first solve queued at once
        x = np.zeros_like(rhs[0])
        xs[srv.submit(sids[s], rhs[0], x)] = (s, x)
    while len(done) < len(reqs):
        for c in srv.poll(wait_ms=1000):
            done[c["ticket"]] = c
    st = srv.stats()
    srv.close()
    assert st["requests"] == len(reqs) and st["launches"] < len(reqs)
    assert max(c["batch"] for c in done.values()) > 1
    for t, (s, x) in xs.items():
        assert done[t]["status"] == 0
        assert np.array_equal(x.view(np.uint32), alone[(s, 0)][1].view(np.uint32))
