"""Request server scheduling on the CPU with a fake executor: every request
completes, concurrency stays within the slots and working memory within the
budget, later arrivals overlap running requests (continuous batching), a
small request passes a large one that does not fit until the bypass limit,
idle datasets are evicted to the dataset budget, and the latency statistics."""
import threading
import time

import numpy as np
import pytest

from midapack_b200.serve import DatasetSpec, Request, Result, Server, latency_stats, draw_specs, poisson_arrivals


class FakeExecutor:
    def __init__(self, seconds_per_sample=1e-7):
        self.k = seconds_per_sample
        self.lock = threading.Lock()
        self.running = 0
        self.max_running = 0
        self.starts = {}
        self.prepared = []
        self.released = []

    @staticmethod
    def work_bytes(spec):
        return spec.n_samples

    @staticmethod
    def data_bytes(data):
        return data["bytes"]

    def start_slot(self, slot):
        pass

    def stop_slot(self, slot):
        pass

    def prepare(self, spec):
        self.prepared.append(spec.key)
        return {"bytes": spec.n_samples // 2, "key": spec.key}

    def release(self, data):
        self.released.append(data["key"])

    def run(self, slot, data, req):
        with self.lock:
            self.running += 1
            self.max_running = max(self.max_running, self.running)
            self.starts[req.rid] = time.perf_counter()
        time.sleep(self.k * req.spec.n_samples)
        with self.lock:
            self.running -= 1
        x = np.full(3, float(req.noise_seed))
        return Result(req.rid, req.spec.key, req.precision, x, None, 10, True, req.spec.n_samples)


def _spec(key, n):
    return DatasetSpec(key, 1, n, 8, 6, 4, 1.0)


def test_all_complete_within_slots_and_budget():
    ex = FakeExecutor()
    srv = Server(ex, slots=3, work_budget=3_000_000, dataset_budget=10_000_000)
    specs = [_spec(f"d{i}", 200_000 + 100_000 * i) for i in range(4)]
    tickets = [srv.submit(Request(r, specs[r % 4], noise_seed=r)) for r in range(20)]
    res = [t.wait(30) for t in tickets]
    srv.close()
    assert [r.rid for r in res] == list(range(20))
    assert all(r.error is None and r.x[0] == r.rid for r in res)
    assert ex.max_running <= 3 and srv.max_running <= 3
    assert srv.peak_work <= 3_000_000
    assert srv.max_running == 3
    assert sorted(set(ex.prepared)) == ["d0", "d1", "d2", "d3"]


def test_later_arrival_overlaps_running_request():
    ex = FakeExecutor(seconds_per_sample=1e-6)
    srv = Server(ex, slots=2, work_budget=10_000_000)
    long = srv.submit(Request(0, _spec("a", 400_000), 0))  # 0.4 s
    time.sleep(0.05)
    short = srv.submit(Request(1, _spec("b", 20_000), 1))  # arrives while the first runs
    r_short, r_long = short.wait(10), long.wait(10)
    srv.close()
    assert r_short.t_end < r_long.t_end
    assert r_short.t_start < r_long.t_end


def test_first_fit_and_bypass_limit():
    ex = FakeExecutor(seconds_per_sample=1e-6)
    srv = Server(ex, slots=4, work_budget=1_000_000, max_bypass_s=0.25)
    big0 = srv.submit(Request(0, _spec("a", 700_000), 0))   # runs 0.7 s
    time.sleep(0.02)
    big1 = srv.submit(Request(1, _spec("b", 700_000), 1))   # does not fit until big0 ends
    small = srv.submit(Request(2, _spec("c", 100_000), 2))  # fits now: passes big1
    r_small = small.wait(10)
    assert r_small.t_start < big0.wait(10).t_end
    time.sleep(0.3)  # big1 has now waited longer than the bypass limit
    late = srv.submit(Request(3, _spec("d", 100_000), 3))
    r_big1, r_late = big1.wait(10), late.wait(10)
    srv.close()
    assert r_late.t_start >= r_big1.t_start


def test_idle_datasets_evicted_to_budget():
    ex = FakeExecutor(seconds_per_sample=1e-8)
    srv = Server(ex, slots=1, work_budget=10_000_000, dataset_budget=150_000)
    for r, n in enumerate([200_000, 200_000, 200_000]):
        srv.submit(Request(r, _spec(f"k{r}", n), r)).wait(10)
    keys = srv.resident_keys()
    srv.close()
    assert keys == ["k2"]
    assert ex.released[:2] == ["k0", "k1"]


def test_oversized_request_rejected():
    srv = Server(FakeExecutor(), slots=1, work_budget=1000)
    with pytest.raises(ValueError):
        srv.submit(Request(0, _spec("a", 10_000), 0))
    srv.close()


def test_latency_stats_and_workload_draws():
    rs = [Result(i, "a", "mixed", None, None, 5, True, 10, t_arrival=0.0 + i, t_start=0.0, t_end=1.0 + i)
          for i in range(10)]
    st = latency_stats(rs)
    assert st["n"] == 10 and abs(st["p50_ms"] - 1000.0) < 1e-6 and abs(st["solves_per_s"] - 10 / 10.0) < 1e-9
    specs = draw_specs(200, seed=3)
    assert all(1 <= s.n_det <= 32 and (1 << 18) - 1 <= s.n_samp <= (1 << 23) + 1 for s in specs)
    assert all(64 <= s.width <= 1025 and -1 <= s.height - (3 * s.width) // 4 <= 6 for s in specs)
    assert all(s.n_samples >= 15 * s.width * (3 * s.width) // 4 or s.width <= 65 for s in specs)
    assert all(min((s.width * s.height) % 25, 25 - (s.width * s.height) % 25) >= 3 for s in specs)
    assert all(256 <= s.lam <= 16384 and 0.1 <= s.fknee <= 5.0 for s in specs)
    off = poisson_arrivals(2000, 50.0, seed=1)
    assert np.all(np.diff(off) > 0) and abs(2000 / off[-1] - 50.0) < 5.0
