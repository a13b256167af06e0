"""The serving loop's scheduling (eimp_b200/serving.py) on the CPU with fake
slots: continuous batching across request sizes, results independent of the
batch a request lands in, admission within the device-memory budget, overlap
of launches, and refusal of requests that can never fit."""
import threading
import time

import numpy as np
import pytest

from eimp_b200.serving import Server


class FakeSlot:
    """Per-target outputs that depend only on the target's genotypes; records
    the memory reserved by the launches in flight."""
    Mref = 7

    def __init__(self, log, lock, bytes_per_target, delay=0.02):
        self.log, self.lock, self.bpt, self.delay = log, lock, bytes_per_target, delay

    def run(self, gt):
        n = gt.shape[0]
        with self.lock:
            self.log["inflight"] += n * self.bpt
            self.log["peak"] = max(self.log["peak"], self.log["inflight"])
            self.log["running"] += 1
            self.log["max_running"] = max(self.log["max_running"], self.log["running"])
        time.sleep(self.delay)
        s = gt.astype(np.uint64).sum(axis=1)
        mats = np.stack([s, s * 3], axis=1)
        pats = np.stack([s + 1, s * 5], axis=1)
        dos = np.repeat((gt[:, :1].astype(np.float32) + np.arange(self.Mref, dtype=np.float32)), 2, axis=0)
        bits = np.repeat(s[:, None] & 1, 2, axis=0)
        with self.lock:
            self.log["inflight"] -= n * self.bpt
            self.log["running"] -= 1
        return mats, pats, bits, dos

    def close(self):
        pass


def make_server(slots=2, max_batch=16, budget=float("inf"), bpt=1.0, delay=0.02):
    log = {"inflight": 0.0, "peak": 0.0, "running": 0, "max_running": 0}
    lock = threading.Lock()
    srv = Server([FakeSlot(log, lock, bpt, delay) for _ in range(slots)], max_batch_targets=max_batch,
                 mem_budget=budget, bytes_per_target=bpt)
    return srv, log


def requests(rng, k, M=11):
    return [rng.integers(0, 4, size=(int(rng.integers(1, 9)), M), dtype=np.uint8) for _ in range(k)]


def test_results_match_alone_and_in_the_mix():
    rng = np.random.default_rng(5)
    reqs = requests(rng, 30)
    alone, _ = make_server(slots=1, max_batch=1, delay=0.0)
    ref = [alone.submit(g).result() for g in reqs]
    alone.close()
    srv, log = make_server(slots=2, max_batch=16)
    futs = [srv.submit(g) for g in reqs]
    out = [f.result(timeout=30) for f in futs]
    batches = srv.batch_sizes()
    srv.close()
    for a, b, g in zip(ref, out, reqs):
        for k in ("mats", "pats", "bits", "dosages"):
            np.testing.assert_array_equal(getattr(a, k), getattr(b, k))
        assert b.mats.shape[0] == g.shape[0] and b.dosages.shape[0] == 2 * g.shape[0]
    assert max(batches) > 8, "queued requests of different sizes should share launches"
    assert all(n <= 16 or n == 0 for n in batches)
    assert log["max_running"] == 2, "the two slots should run launches at the same time"
    assert len(srv.latencies()) == len(reqs)


def test_memory_budget_bounds_the_launches_in_flight():
    rng = np.random.default_rng(6)
    srv, log = make_server(slots=4, max_batch=8, budget=10.0, bpt=1.0)
    futs = [srv.submit(g) for g in requests(rng, 40)]
    for f in futs:
        f.result(timeout=60)
    srv.close()
    assert 0 < log["peak"] <= 10.0


def test_requests_arriving_while_busy_are_admitted():
    rng = np.random.default_rng(7)
    srv, log = make_server(slots=1, max_batch=64, delay=0.05)
    first = srv.submit(requests(rng, 1)[0])
    time.sleep(0.01)   # the first launch is running
    late = [srv.submit(g) for g in requests(rng, 5)]
    first.result(timeout=10)
    res = [f.result(timeout=10) for f in late]
    srv.close()
    # the late requests were queued together and served by one launch
    assert len({r.batch_targets for r in res}) == 1 and res[0].batch_targets == sum(r.mats.shape[0] for r in res)


def test_oversize_request_is_refused():
    srv, _ = make_server(slots=1, budget=5.0, bpt=1.0)
    f = srv.submit(np.zeros((6, 11), np.uint8))
    with pytest.raises(MemoryError):
        f.result(timeout=5)
    ok = srv.submit(np.zeros((5, 11), np.uint8)).result(timeout=5)
    srv.close()
    assert ok.mats.shape[0] == 5
