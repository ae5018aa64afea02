"""bench.py's CPU baseline sampler (the `cpu_baseline` leg and the `--impl reference` arm) on a
few key switches: it walks the seeded op mix in order with none skipped, generates the Galois key
of every rotation it draws before timing, and reports a positive rate with the sample described."""

import importlib.util
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_cpu_baseline", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def path(bench):
    return bench.CpuPath(2)


def test_take_walks_the_mix_in_order(bench, path):
    start = path.pos
    ops = path.take(5)
    assert sum(kind != "pmul" for kind, _, _ in ops) == 5
    assert ops == [path.ops[(start + i) % len(path.ops)] for i in range(len(ops))]
    assert path.pos == (start + len(ops)) % len(path.ops)
    rot_elts = {path.O.galois_elt(path.P.n, s) for kind, _, s in ops if kind == "rot"}
    assert rot_elts <= set(path.gk)  # every drawn rotation has its key before it is timed


def test_sample_rate_and_description(bench, path):
    v, sample = bench.cpu_sample(path, key_switches=3)
    assert v > 0
    m = re.match(r"(\d+) key switches of the seeded op mix in order, none skipped \((\d+) HMult.*?, (\d+) rotations", sample)
    assert m and int(m.group(1)) == 3 and int(m.group(2)) + int(m.group(3)) == 3
    assert "on 2 threads" in sample


def test_host_description(bench):
    host = bench.cpu_host()
    assert host["logical_cpus"] == os.cpu_count() and host["cpu_model"]
