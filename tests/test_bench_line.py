"""bench.py's output contract on CPU, from the two lines one B200 run printed
(tests/golden/bench_lines_b200.json): the last line carries every key the
benchmark contract asks for, its summary is what `summary()` makes of the
detail line, it stays short enough to survive a 3000-byte tail of stdout even
with every float at full precision, and both arms describe the same workload."""
import json
import random
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

LINES = json.loads((ROOT / "tests" / "golden" / "bench_lines_b200.json").read_text())


def _extras(detail):
    skip = ("kernels", "profiled_bytes", "first_gates_n30", "host_cpus")
    return {k: v for k, v in detail.items() if k not in skip}


def test_last_line_has_the_contract_keys():
    last = LINES["last_line"]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks", "cpu_baseline"):
        assert k in last, k
    r = last["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    assert set(last["e2e"]) >= {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert last["cpu_baseline"]["kind"] in ("port", "reference")
    assert last["config"] == bench.bench_config(last["config"]["qubits"], last["n_gpus"])


def test_summary_is_recomputed_from_the_detail_line():
    d = LINES["detail_line"]["detail"]
    last = LINES["last_line"]
    s = bench.summary(_extras(d), last["summary"]["layered30"]["plain_s"], d["first_gates_n30"])
    want = last["summary"]
    assert s["vqe24"] == want["vqe24"]
    assert s["layered30"]["autotuned"] == want["layered30"]["autotuned"]
    assert set(s["layered30"]["fused"]) <= set(want["layered30"]["fused"])
    assert s["dm14"]["n12_layer_vs_oracle"] == want["dm14"]["n12_layer_vs_oracle"]


def _perturb(x, rng):
    """Every float replaced by a full-precision float of the same magnitude."""
    if isinstance(x, float):
        return x * (1.0 + 1e-9 * rng.random()) if x else x
    if isinstance(x, dict):
        return {k: _perturb(v, rng) for k, v in x.items()}
    if isinstance(x, list):
        return [_perturb(v, rng) for v in x]
    return x


def test_last_line_fits_a_3000_byte_tail():
    rng = random.Random(7)
    d = _perturb(LINES["detail_line"]["detail"], rng)
    last = dict(LINES["last_line"])
    last["summary"] = bench.summary(_extras(d), 21.5432109876, d["first_gates_n30"])
    text = json.dumps(last, separators=(",", ":"))
    # the driver keeps about 3000 bytes of stdout, including its own header
    # and the stderr marker
    assert len(text) < 2900, len(text)
