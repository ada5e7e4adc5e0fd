"""The serving loop (le2d_server_*): continuous batching under an HBM budget.

Each result must be the same alone and in the mix: requests submitted while others
are on the GPU join the running persistent launches, and every one of them must
equal (bit for bit -- the same per-node operations) the same problem solved alone
through le_step; the single-solve path is checked against the reference elsewhere.
"""
import threading
import time

import numpy as np
import pytest

from le2d_b200 import capi, workloads
from oracle.oracle import ST_AOS, ST_SOA

from test_batch_gpu import small_set, solve_alone

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return capi.Lib("f")


def test_mix_equals_alone(lib):
    probs = small_set(31, 12, 20, 260, 20, 150)
    with capi.Server(lib, 1 << 30, window_steps=16) as srv:
        tickets = []
        for k, p in enumerate(probs):  # staggered arrivals: later requests join running windows
            st = ST_SOA if k % 4 == 3 else ST_AOS
            tickets.append((srv.submit(srv_problem(lib, p, st), disks=p.disks), p, st))
            time.sleep(0.002 * (k % 3))
        spans = []
        for t, p, st in tickets:
            assert t > 0
            assert srv.wait(t, 60.0) == 0
            got = srv.result(t)
            want, _ = solve_alone(lib, p, st)
            assert got.tobytes() == want.tobytes(), (p.nx, p.ny, p.steps, st)
            spans.append(srv.times(t))
        s = srv.stats()
        assert s["completed"] == len(probs) and s["failed"] == 0
        assert s["windows"] >= 2
        # continuous batching: some request was admitted while another was on the device
        joined = [b for b in spans for a in spans if a is not b and a[1] < b[1] < a[2]]
        assert joined, spans


def srv_problem(lib, p, stype=ST_AOS, receiver_row=-1, every=10):
    return lib.le2d_problem(p.nx, p.ny, p.hx, p.hy, p.dt, p.c1, p.c2, p.rho, p.steps, stype, receiver_row, every)


def test_receivers(lib):
    p = small_set(32, 1, 60, 90, 40, 40)[0]
    with capi.Server(lib, 1 << 28, window_steps=7) as srv:
        t = srv.submit(srv_problem(lib, p, ST_AOS, p.ny // 4, 10), disks=p.disks, want=capi.LE2D_WANT_RECEIVERS)
        assert srv.wait(t, 60.0) == 0
        rec = srv.result(t)
        _, samples = solve_alone(lib, p, ST_AOS, sample_row=p.ny // 4, every=10)
        assert rec.tobytes() == samples.astype(np.float32).tobytes()


def test_budget_admission(lib):
    """Three requests that each need more than half the budget run one after another;
    a request larger than the budget is refused at submission."""
    n = 512
    p = workloads.Problem(n, n, 1, 1, 2, 1, 1, 0.25, 30, [(256.0, 256.0, 40.0, 1.0)])
    need = 2 * 5 * n * n * 4
    with capi.Server(lib, int(need * 1.6), window_steps=8) as srv:
        ts = [srv.submit(srv_problem(lib, p), disks=p.disks) for _ in range(3)]
        assert all(t > 0 for t in ts)
        big = workloads.Problem(2048, 2048, 1, 1, 2, 1, 1, 0.25, 5, [])
        assert srv.submit(srv_problem(lib, big)) == -capi.LE2D_EBUDGET
        want, _ = solve_alone(lib, p, ST_AOS)
        spans = []
        for t in ts:
            assert srv.wait(t, 60.0) == 0
            assert srv.result(t).tobytes() == want.tobytes()
            spans.append(srv.times(t))
        spans.sort(key=lambda s: s[1])
        for a, b in zip(spans, spans[1:]):
            assert b[1] >= a[2] - 1e-6  # admitted only after the previous one finished


def test_invalid_requests(lib):
    with capi.Server(lib, 1 << 26, window_steps=8) as srv:
        bad = workloads.Problem(2, 10, 1, 1, 2, 1, 1, 0.25, 5, [])
        assert srv.submit(srv_problem(lib, bad)) == -capi.LE2D_EINVAL
        ok = workloads.Problem(10, 10, 1, 1, 2, 1, 1, 0.25, 5, [])
        assert srv.submit(srv_problem(lib, ok), want=capi.LE2D_WANT_RECEIVERS) == -capi.LE2D_EINVAL
        cfl = workloads.Problem(10, 10, 1, 1, 2, 1, 1, 0.9, 5, [])  # k1 = 1.8: rejected at admission
        t = srv.submit(srv_problem(lib, cfl))
        assert t > 0 and srv.wait(t, 30.0) == capi.LE2D_EINVAL


def test_concurrent_submitters(lib):
    """Several client threads submit at once; every result matches the solve alone."""
    probs = small_set(33, 9, 16, 120, 10, 60)
    results = {}
    with capi.Server(lib, 1 << 28, window_steps=10) as srv:
        def client(chunk):
            for p in chunk:
                t = srv.submit(srv_problem(lib, p), disks=p.disks)
                assert srv.wait(t, 60.0) == 0
                results[id(p)] = srv.result(t)
        th = [threading.Thread(target=client, args=(probs[i::3],)) for i in range(3)]
        for x in th:
            x.start()
        for x in th:
            x.join()
    for p in probs:
        want, _ = solve_alone(lib, p, ST_AOS)
        assert results[id(p)].tobytes() == want.tobytes()


def test_failed_solve_fails_alone(lib, monkeypatch):
    """A solve whose device work stalls (test hook: the first tile of the server's first
    window never publishes) fails with LE2D_ETIMEOUT after the bounded wait; the requests
    beside it complete and equal their solves alone."""
    monkeypatch.setenv("LE2D_TEST_STALL_TILE", "0")
    victim = workloads.Problem(300, 200, 1, 1, 2, 1, 1, 0.25, 40, [(150.0, 100.0, 30.0, 1.0)])
    others = small_set(34, 5, 16, 120, 4, 7)  # fewer steps than the window: ordered after the victim
    with capi.Server(lib, 1 << 28, window_steps=8) as srv:
        tv = srv.submit(srv_problem(lib, victim), disks=victim.disks)
        ts = [srv.submit(srv_problem(lib, p), disks=p.disks) for p in others]
        assert srv.wait(tv, 60.0) == capi.LE2D_ETIMEOUT
        for t, p in zip(ts, others):
            assert srv.wait(t, 60.0) == 0
            want, _ = solve_alone(lib, p, ST_AOS)
            assert srv.result(t).tobytes() == want.tobytes()
        s = srv.stats()
        assert s["failed"] == 1 and s["completed"] == len(others)


def test_abandoned_requests_and_shutdown_mid_flight(lib):
    """A client that dies after submitting (its thread exits without waiting or releasing):
    its requests still complete without holding up anyone else's, and their tickets stay
    pollable.  A server destroyed while requests are queued and running returns promptly
    and gives its device memory back: a server with the same budget runs afterwards."""
    probs = small_set(35, 4, 40, 200, 20, 60)
    budget = 1 << 29
    with capi.Server(lib, budget, window_steps=8) as srv:
        abandoned = []
        dead = threading.Thread(target=lambda: abandoned.extend(
            srv.submit(srv_problem(lib, p), disks=p.disks) for p in probs[:3]))
        dead.start()
        dead.join()  # the client is gone
        t = srv.submit(srv_problem(lib, probs[3]), disks=probs[3].disks)
        assert srv.wait(t, 60.0) == 0
        want, _ = solve_alone(lib, probs[3], ST_AOS)
        assert srv.result(t).tobytes() == want.tobytes()
        deadline = time.time() + 60
        while any(srv.poll(a) == 0 for a in abandoned) and time.time() < deadline:
            time.sleep(0.01)
        assert [srv.poll(a) for a in abandoned] == [1, 1, 1]
        assert srv.stats()["completed"] == 4
    big = workloads.Problem(2048, 2048, 1, 1, 2, 1, 1, 0.25, 4000, [(1024.0, 1024.0, 100.0, 1.0)])
    srv = capi.Server(lib, budget, window_steps=64)
    ts = [srv.submit(srv_problem(lib, big), disks=big.disks) for _ in range(5)]
    assert all(x > 0 for x in ts)
    time.sleep(0.2)  # some admitted and running, others queued
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 30.0
    with capi.Server(lib, budget, window_steps=8) as srv2:
        t = srv2.submit(srv_problem(lib, probs[0]), disks=probs[0].disks)
        assert srv2.wait(t, 60.0) == 0
        assert srv2.stats()["arena_capacity"] >= budget * 0.99
