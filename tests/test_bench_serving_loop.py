"""bench.py's serving loop (Serving.run / Serving.measure) on CPU against a fake server: a
request that fails with a status, a result call that raises, and a result that never comes are
counted as failed and reported, and the loop always returns instead of waiting forever."""

import importlib.util
import os
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_serving_loop", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class FakeServer:
    """Completes request i 0.5 ms after submission with status codes[i] (0 when absent); a
    status of None makes the result call raise, "hang" makes it time out (the CKG_TIMEOUT
    status, after the timeout it is given)."""

    TIMEOUT = 9

    def __init__(self, codes=None):
        self.t0, self.times, self.codes, self.waits = time.perf_counter(), [], dict(codes or {}), []

    def _submit(self, owner):
        t = (time.perf_counter() - self.t0) * 1e6
        self.times.append((t, t, t + 500.0))
        return len(self.times) - 1

    def submit_mul(self, o, a, b):
        return self._submit(o)

    def submit_rotate(self, o, a, steps):
        return self._submit(o)

    def submit_matvec(self, o, d, stride, diag, x):
        return self._submit(o)

    def result_times(self, i, timeout_ms):
        self.waits.append(timeout_ms)
        code = self.codes.get(i, 0)
        if code is None:
            raise RuntimeError("result call failed")
        if code == "hang":
            time.sleep(timeout_ms * 1e-3)
            return self.TIMEOUT, None, (0.0, 0.0, 0.0)
        return code, None, self.times[i]

    def stats(self):
        keys = ("batches", "multi_owner_batches", "key_hits", "key_misses", "key_evictions", "key_upload_bytes",
                "budget_waits", "hbm_budget", "peak_device_bytes")
        return dict.fromkeys(keys, 0)


def serving(bench, srv, owners=4):
    sv = bench.Serving.__new__(bench.Serving)
    sv.rng, sv.owners, sv.srv = np.random.default_rng(3), owners, srv
    sv.steps = list(range(1, 8)) + [8 * k for k in range(1, 8)]
    sv.slot = {g: g for g in range(owners)}
    sv.inputs = {g: [("ct", g, lv) for lv in (23, 17, 11, 5)] for g in range(owners)}
    sv.diag = {23: "diag23", 11: "diag11"}
    sv.key_bytes, sv.register_s = owners * bench.Serving.key_bytes_per_owner(), 0.0
    return sv


def test_all_served(bench):
    sv = serving(bench, FakeServer())
    res = sv.measure(requests=40, load=0.7)
    assert res["served"] == 40 and res["failed"] == 0 and res["p50_ms"] == pytest.approx(0.5)


def test_failed_status_is_counted_not_fatal(bench, capsys):
    # ids 96 + 40 + 3: the timed run's fourth request fails with the out-of-memory status
    sv = serving(bench, FakeServer({96 + 40 + 3: 7}))
    res = sv.measure(requests=40, load=0.7)
    assert res["served"] == 39 and res["failed"] == 1
    assert "status 7" in capsys.readouterr().err


def test_raising_result_call_ends_the_run(bench, capsys):
    sv = serving(bench, FakeServer({5: None}))
    t, _ = sv.run(20)
    assert len(t) == 5 and sv.failed == 15
    assert "result call failed" in capsys.readouterr().err


def test_result_deadline_bounds_the_wait(bench, monkeypatch):
    monkeypatch.setattr(bench, "SERVE_RESULT_DEADLINE_S", 0.2)
    srv = FakeServer({2: "hang"})
    sv = serving(bench, srv)
    t0 = time.perf_counter()
    t, _ = sv.run(10)
    assert time.perf_counter() - t0 < 5.0
    assert len(t) == 2 and sv.failed == 8
    assert all(0 < w <= 200 for w in srv.waits)
