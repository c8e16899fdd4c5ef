"""bench.py's record helpers (no GPU): the byte models behind `roofline`, the per-stage
roofline fractions, the metric name and workload selection of the plain form."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_records_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def args(bench, *argv):
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_byte_models_at_512(bench):
    w = bench.workload(args(bench), 4)
    p0 = 512 * 424
    n = 512 ** 3
    assert bench.algorithmic_bytes(w.config, "integrate") == 2 * 4 * n + 4 * p0   # 1.0746 GB
    assert bench.algorithmic_bytes(w.config, "raycast") == 2 * n + 32 * p0        # value plane + maps
    # ICP {10, 5, 4} iterations at levels 0, 1, 2: 64 bytes per pixel and iteration
    assert bench.algorithmic_bytes(w.config, "track") == 64 * (10 * p0 + 5 * p0 // 4 + 4 * p0 // 16)


def test_stage_rooflines(bench):
    w = bench.workload(args(bench), 4)
    per = {"integrate": 0.2, "raycast": 0.1, "track": 0.0}
    r = bench.stage_rooflines(w, per, 6000.0)
    assert set(r) == {"integrate", "raycast"}  # a stage without a time is left out
    assert r["integrate"]["achieved"] == pytest.approx(bench.algorithmic_bytes(w.config, "integrate") / 0.2e-3 / 1e9)
    assert r["integrate"]["frac"] == pytest.approx(r["integrate"]["achieved"] / 6000.0)
    assert r["integrate"]["traffic"] == bench.measured_traffic(w.name, "integrate")


def test_plain_workloads_and_metric(bench):
    w2 = bench.workload(args(bench), 4)
    assert w2.name == "c2_precision_512" and bench.plain_metric(w2) == bench.PLAIN_METRIC
    w1 = bench.workload(args(bench, "--workload", "c1"), 4)
    assert w1.name == "c1_plain_128" and "128^3" in bench.plain_metric(w1)
    c = bench.plain_config(w1, args(bench, "--workload", "c1"), 1)
    assert c["storage"] == "f32f32" and c["jtj"] == "fp32" and c["dim_m"] == 1.5
    # the frame generator renders the workload's own scene
    _, f = bench._gen((w1.name, 128, w1.config.storage, w1.config.jtj, 4, 2))
    assert (f == w1.frame(2)).all()


def test_launch_shape_flag(bench):
    a = args(bench, "--launch-shape", "32,4")
    assert tuple(int(x) for x in a.launch_shape.split(",")) == (32, 4)
