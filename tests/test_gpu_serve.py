"""Served builds (svo_server): every request's result is the same alone and
in the mix -- bit for bit, whatever batch and stream it landed in."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WAIT_US = 60_000_000  # a request not built within a minute fails the test instead of hanging it


def _same(a, b):
    assert a.depth == b.depth
    assert a.nodes().tobytes() == b.nodes().tobytes()
    assert a.vertices().tobytes() == b.vertices().tobytes()
    assert a.edges().tobytes() == b.edges().tobytes()
    assert a.keys().tobytes() == b.keys().tobytes()


def _requests(n, seed, res_choices=(64, 128, 256, 512)):
    from svo_b200 import meshgen

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        v, f = meshgen.batch_mesh(rng)
        out.append((v, f, int(rng.choice(res_choices))))
    return out


@pytest.mark.parametrize("workers,max_batch,budget", [(2, 8, 8 << 30), (3, 64, 40 << 30), (1, 1, 1)])
def test_mix_equals_alone(gpu_ctx, svo_mod, workers, max_batch, budget):
    reqs = _requests(16, seed=7)
    srv = svo_mod.Server(gpu_ctx, budget, workers=workers, max_batch=max_batch)
    tickets = [srv.submit(*r) for r in reqs]
    for t, (p, f, res) in zip(tickets, reqs):
        r, st, lat = srv.wait(t, timeout_us=WAIT_US)
        assert st == 0 and lat > 0
        _same(r, gpu_ctx.build(p, f, res))
        srv.release(t)
    s = srv.stats()
    assert s["built"] == len(reqs) and s["queued"] == 0 and s["reserved_bytes"] == 0
    srv.close()


def test_arrivals_while_busy(gpu_ctx, svo_mod):
    """Requests submitted from another thread while batches are on the GPU."""
    import torch

    reqs = _requests(24, seed=8, res_choices=(128, 256, 512))
    dev = [(torch.from_numpy(p).cuda(), torch.from_numpy(f).cuda(), r) for p, f, r in reqs]
    srv = svo_mod.Server(gpu_ctx, 16 << 30, workers=3, max_batch=4)
    tickets = [None] * len(dev)

    def client():
        for i, m in enumerate(dev):
            tickets[i] = srv.submit(*m)
            time.sleep(0.0005)

    th = threading.Thread(target=client)
    th.start()
    th.join()
    for t, m in zip(tickets, dev):
        r, st, _ = srv.wait(t, timeout_us=WAIT_US)
        assert st == 0
        _same(r, gpu_ctx.build(*m))
        srv.release(t)
    assert srv.stats()["batches"] >= 2
    srv.close()


def test_failures_in_the_mix(gpu_ctx, svo_mod):
    reqs = _requests(4, seed=9)
    pts = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.2, 0.1]], dtype=np.float32)
    bad = (pts, np.zeros((0, 3), np.int32), 8)
    mix = [reqs[0], bad, reqs[1], reqs[2], bad, reqs[3]]
    srv = svo_mod.Server(gpu_ctx, 40 << 30, workers=2, max_batch=8)
    tickets = [srv.submit(*m) for m in mix]
    for t, m in zip(tickets, mix):
        r, st, _ = srv.wait(t, timeout_us=WAIT_US)
        if m is bad:
            assert st == svo_mod.ERR_EMPTY and r is None
        else:
            assert st == 0
            _same(r, gpu_ctx.build(*m))
        srv.release(t)
    srv.close()


def test_wait_timeout_and_close_with_pending(gpu_ctx, svo_mod):
    reqs = _requests(6, seed=10, res_choices=(512,))
    srv = svo_mod.Server(gpu_ctx, 40 << 30, workers=1, max_batch=1)
    tickets = [srv.submit(*m) for m in reqs]
    first = srv.wait(tickets[-1], timeout_us=0)
    assert first is None or first[1] == 0  # not finished yet, or already done
    srv.close()  # finishes the queue and frees the unreleased results


def test_completion_order(gpu_ctx, svo_mod):
    reqs = _requests(10, seed=11)
    srv = svo_mod.Server(gpu_ctx, 40 << 30, workers=2, max_batch=4)
    tickets = {srv.submit(*m): m for m in reqs}
    seen = set()
    for _ in range(len(reqs)):
        t, r, st, lat = srv.next(timeout_us=WAIT_US)
        assert st == 0 and t in tickets and t not in seen
        seen.add(t)
        _same(r, gpu_ctx.build(*tickets[t]))
        srv.release(t)
    assert srv.next(timeout_us=1000) is None
    srv.close()


def test_cancel_queued(gpu_ctx, svo_mod):
    """A request still in the queue can be withdrawn: it finishes at once with
    ERR_CANCELLED and no result; the others are built as if it never came; a
    request already finished cannot be cancelled."""
    from svo_b200 import meshgen

    soup, _, _ = meshgen.torus_slivers(200_000)
    small = _requests(2, seed=12, res_choices=(64,))
    srv = svo_mod.Server(gpu_ctx, 40 << 30, workers=1, max_batch=1)
    big = srv.submit(soup, None, 512)  # keeps the one worker busy while the rest queue up
    t1 = srv.submit(*small[0])
    t2 = srv.submit(*small[1])
    srv.cancel(t2)
    r, st, _ = srv.wait(t2, timeout_us=WAIT_US)
    assert st == svo_mod.ERR_CANCELLED and r is None
    for t, m in ((big, (soup, None, 512)), (t1, small[0])):
        got = srv.wait(t, timeout_us=WAIT_US)
        assert got is not None, "request not built in time"
        r, st, _ = got
        assert st == 0
        _same(r, gpu_ctx.build(*m))
    with pytest.raises(svo_mod.SvoError) as e:
        srv.cancel(t1)
    assert e.value.code == svo_mod.ERR_INVALID_ARGUMENT
    for t in (big, t1, t2):
        srv.release(t)
    s = srv.stats()
    assert s["built"] == 2 and s["reserved_bytes"] == 0 and s["queued"] == 0
    srv.close()


def test_budget_holds_when_results_outgrow_estimates(gpu_ctx, svo_mod):
    """A soup of 100k scattered slivers, whose octree is several times the
    admission estimate, with a budget that holds one such result: the
    estimates admit three requests into one batch, but once their exact sizes
    are known only one is built at a time and the rest wait for memory; every
    result is still correct and the reservations never exceed the budget."""
    from svo_b200 import meshgen

    soup = meshgen.slivers(100_000, np.random.default_rng(5)).reshape(-1, 3)
    flags = svo_mod.FLAG_NO_VERT_EDGE
    alone = gpu_ctx.build(soup, None, 256, flags)
    exact = alone.num_nodes * 168 + alone.num_keys * 8
    est = svo_mod.estimate_bytes(soup.shape[0], 0, 256, flags)
    assert exact > 3 * est  # the estimate really is far too small
    budget = int(1.5 * (exact + est))
    srv = svo_mod.Server(gpu_ctx, budget, workers=2, max_batch=8, flags=flags)
    tickets = [srv.submit(soup, None, 256) for _ in range(3)]
    for t in tickets:  # each result is released before the next request is awaited
        got = srv.wait(t, timeout_us=WAIT_US)
        assert got is not None, f"request {t} not built in time; server {srv.stats()}, budget {budget}, " \
                                f"exact {exact}, estimate {est}"
        r, st, _ = got
        assert st == 0
        assert r.nodes().tobytes() == alone.nodes().tobytes() and r.keys().tobytes() == alone.keys().tobytes()
        srv.release(t)
    s = srv.stats()
    assert s["built"] == 3 and s["batches"] == 3 and s["reserved_bytes"] == 0
    assert 0 < s["peak_reserved_bytes"] <= budget
    srv.close()


def test_served_results_match_oracle(gpu_ctx, svo_mod, oracle_mod):
    """Served results against the oracle directly (not only against builds of
    the same library): nodes, vertex/edge arrays and keys, bit for bit."""
    from parity import assert_same

    reqs = _requests(6, seed=13, res_choices=(32, 64, 128))
    srv = svo_mod.Server(gpu_ctx, 8 << 30, workers=2, max_batch=4)
    tickets = [srv.submit(*m) for m in reqs]
    for t, (p, f, res) in zip(tickets, reqs):
        r, st, _ = srv.wait(t, timeout_us=WAIT_US)
        assert st == 0
        assert_same(r, oracle_mod.build_svo(p, f, res))
        srv.release(t)
    srv.close()


def test_fleet_spreads_requests_and_matches_alone(gpu_ctx, svo_mod):
    """svo_fleet over two contexts (two GPUs in production; here two contexts
    of one GPU, which share nothing and never wait on each other): requests
    spread over both members, every result is bit for bit the plain build's,
    svo_fleet_next reports each ticket once, and released tickets leave the
    fleet."""
    reqs = _requests(20, seed=14)
    ctx2 = svo_mod.Context(0)
    fleet = svo_mod.Fleet([gpu_ctx, ctx2], 16 << 30, workers=2, max_batch=8)
    tickets = [fleet.submit(*r) for r in reqs]
    assert len(set(tickets)) == len(tickets)
    members = [fleet.member(t) for t in tickets]
    assert set(members) == {0, 1}
    by_ticket = dict(zip(tickets, reqs))
    seen = set()
    for _ in reqs:
        got = fleet.next(timeout_us=WAIT_US)
        assert got is not None, f"request not built in time; {fleet.stats()}"
        t, r, st, lat = got
        assert t in by_ticket and t not in seen and st == 0 and lat > 0
        seen.add(t)
        _same(r, gpu_ctx.build(*by_ticket[t]))
        fleet.release(t)
        assert fleet.member(t) == -1
    assert fleet.next(timeout_us=1000) is None
    stats = fleet.stats()
    assert [s["built"] for s in stats] == [members.count(0), members.count(1)]
    assert all(s["reserved_bytes"] == 0 and s["queued"] == 0 for s in stats)
    with pytest.raises(svo_mod.SvoError) as e:
        fleet.wait(tickets[0], timeout_us=0)
    assert e.value.code == svo_mod.ERR_INVALID_ARGUMENT
    fleet.close()
    ctx2.close()


def test_fleet_cancel_and_wait(gpu_ctx, svo_mod):
    """A request queued behind a large one on its member is cancelled through
    the fleet: svo_fleet_wait and svo_fleet_next report it with ERR_CANCELLED;
    the large builds on both members are unaffected."""
    from svo_b200 import meshgen

    soup, _, _ = meshgen.torus_slivers(200_000)
    small = _requests(1, seed=15, res_choices=(64,))[0]
    ctx2 = svo_mod.Context(0)
    fleet = svo_mod.Fleet([gpu_ctx, ctx2], 8 << 30, workers=1, max_batch=1)
    a = fleet.submit(soup, None, 512)
    b = fleet.submit(soup, None, 512)
    c = fleet.submit(*small)  # both members hold one large request: the tie goes to member 0
    assert (fleet.member(a), fleet.member(b), fleet.member(c)) == (0, 1, 0)
    fleet.cancel(c)
    r, st, _ = fleet.wait(c, timeout_us=WAIT_US)
    assert st == svo_mod.ERR_CANCELLED and r is None
    alone = gpu_ctx.build(soup, None, 512)
    order = []
    for _ in range(3):
        got = fleet.next(timeout_us=WAIT_US)
        assert got is not None, "request not built in time"
        t, r, st, _ = got
        order.append(t)
        if t == c:
            assert st == svo_mod.ERR_CANCELLED and r is None
        else:
            assert st == 0
            _same(r, alone)
    assert sorted(order) == sorted([a, b, c]) and order[0] == c
    for t in (a, b, c):
        fleet.release(t)
    assert all(s["reserved_bytes"] == 0 for s in fleet.stats())
    fleet.close()
    ctx2.close()
