"""Circuit JSON (src/json.rs), the yao-state-v1 file format
(yao-cli/src/state_io.rs) and the CLI commands simulate / probs / expect /
measure,
checked against the outputs yao-rs generated for its documentation examples
(docs/src/examples/generated/results/*.json)."""
import io
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import yao_rs as Y
from yao_rs.cli import parse_operator
from yao_rs.json_io import JsonError, circuit_from_json, circuit_to_json, read_state, write_state

ROOT = Path(__file__).resolve().parent.parent


def examples(golden):
    return golden("cli_examples")["cases"]


def test_examples_through_the_oracle(golden):
    """Parse each example circuit and reproduce yao-rs's CLI output with the oracle."""
    for case in examples(golden):
        c = circuit_from_json(json.dumps(case["circuit"]))
        z = np.zeros(1 << c.nbits, complex)
        z[0] = 1
        out = O.apply_circuit(c, z)
        res = case["result"]
        if "probabilities" in res:
            p = O.probs(out, c.nbits, res["locs"])
            assert np.max(np.abs(p - np.array(res["probabilities"]))) < 1e-10, case["name"]
        else:
            op = parse_operator(res["operator"])
            v = O.expect_arrayreg(out, c.nbits, op)
            ev = res["expectation_value"]
            assert abs(v - complex(ev["re"], ev["im"])) < 1e-10, case["name"]


def test_json_round_trip(golden):
    for case in examples(golden):
        c = circuit_from_json(json.dumps(case["circuit"]))
        c2 = circuit_from_json(circuit_to_json(c))
        assert len(c.elements) == len(c2.elements)
        for a, b in zip(c.elements, c2.elements):
            assert type(a) is type(b)
            if isinstance(a, Y.PositionedGate):
                assert a.gate == b.gate and a.target_locs == b.target_locs
                assert a.control_locs == b.control_locs and list(a.control_configs) == list(b.control_configs)
    custom = Y.Circuit.qubits(2, [Y.put([0, 1], Y.Gate.Custom(np.eye(4) * 1j, False, "iI")), Y.label(1, "note"),
                                  Y.channel([0], Y.NoiseChannel.BitFlip(0.1))])
    back = circuit_from_json(circuit_to_json(custom))
    assert len(back.elements) == 2  # the channel is dropped (src/json.rs:115-131)
    assert np.array_equal(back.elements[0].gate.matrix(), np.eye(4) * 1j)


def test_json_errors():
    with pytest.raises(JsonError, match="requires params"):
        circuit_from_json('{"num_qubits": 1, "elements": [{"type": "gate", "gate": "Rx", "targets": [0]}]}')
    with pytest.raises(JsonError, match="Unknown gate type"):
        circuit_from_json('{"num_qubits": 1, "elements": [{"type": "gate", "gate": "Q", "targets": [0]}]}')
    with pytest.raises(JsonError, match="validation"):
        circuit_from_json('{"num_qubits": 1, "elements": [{"type": "gate", "gate": "X", "targets": [3]}]}')
    with pytest.raises(JsonError, match="parse error"):
        circuit_from_json("{not json")


def test_state_file_round_trip():
    rng = np.random.default_rng(0)
    v = rng.normal(size=8) + 1j * rng.normal(size=8)
    b = io.BytesIO()
    write_state(v, b)
    raw = b.getvalue()
    header = json.loads(raw.split(b"\n", 1)[0])
    assert header == {"format": "yao-state-v1", "num_qubits": 3, "dims": [2, 2, 2], "num_elements": 8,
                      "dtype": "complex128"}
    assert len(raw.split(b"\n", 1)[1]) == 8 * 16
    assert np.array_equal(read_state(io.BytesIO(raw)), v)
    bad = raw.replace(b"yao-state-v1", b"yao-state-v9")
    with pytest.raises(JsonError, match="Unknown state format"):
        read_state(io.BytesIO(bad))


def test_operator_parser():
    p = parse_operator("Z(0)Z(1) - 0.5*X(2) + Y(1)")
    assert p.coeffs() == [1.0, -0.5, 1.0]
    assert [s.ops() for s in p.opstrings()] == [[(0, Y.Op.Z), (1, Y.Op.Z)], [(2, Y.Op.X)], [(1, Y.Op.Y)]]
    assert parse_operator("-P0(3)").coeffs() == [-1.0]
    with pytest.raises(ValueError):
        parse_operator("Q(1)")


def _cli(*args, stdin=None):
    env = dict(os.environ, PYTHONPATH=str(ROOT / "yao-rs_b200"))
    return subprocess.run([sys.executable, "-m", "yao_rs.cli", *args], input=stdin, capture_output=True,
                          env=env, check=True)


@pytest.mark.gpu
def test_cli_examples_on_gpu(golden, tmp_path):
    for case in examples(golden):
        cpath = tmp_path / f"{case['name']}.json"
        cpath.write_text(json.dumps(case["circuit"]))
        res = case["result"]
        if "probabilities" in res:
            out = json.loads(_cli("run", str(cpath), "--probs", "--json").stdout)
            assert np.max(np.abs(np.array(out["probabilities"]) - res["probabilities"])) < 1e-10, case["name"]
        else:
            out = json.loads(_cli("run", str(cpath), "--op", res["operator"], "--json").stdout)
            assert abs(out["expectation_value"]["re"] - res["expectation_value"]["re"]) < 1e-10
    # simulate -> state file -> probs with locs, and expect from the file
    case = [c for c in examples(golden) if c["name"] == "qft4"][0]
    cpath = tmp_path / "qft4.json"
    cpath.write_text(json.dumps(case["circuit"]))
    spath = tmp_path / "qft4.state"
    _cli("simulate", str(cpath), "--output", str(spath))
    st = read_state(open(spath, "rb"))
    c = circuit_from_json(cpath.read_text())
    z = np.zeros(16, complex)
    z[0] = 1
    assert np.max(np.abs(st - O.apply_circuit(c, z))) == 0.0
    marg = json.loads(_cli("probs", str(spath), "--locs", "2,0", "--json").stdout)
    assert np.max(np.abs(np.array(marg["probabilities"]) - O.probs(st, 4, [2, 0]))) < 1e-15
    e = json.loads(_cli("expect", str(spath), "X(0) + 0.5*Z(1)Z(3)", "--json").stdout)
    ref = O.expect_arrayreg(st, 4, parse_operator("X(0) + 0.5*Z(1)Z(3)"))
    assert abs(e["expectation_value"]["re"] - ref.real) < 1e-12


def test_measure_sampling_rule_and_format():
    """sample_outcomes follows sample_from_probs / decode_outcome_bits
    (src/measure.rs:140-156) draw by draw, and format_measurement lays out
    counts as yao-cli does (yao-cli/src/commands/mod.rs:54-100)."""
    from yao_rs.cli import format_measurement, sample_outcomes

    def one(p, r):
        acc = 0.0
        for i, x in enumerate(p):
            acc += x
            if r < acc:
                return i
        return len(p) - 1

    rng = np.random.default_rng(11)
    for m in (1, 2, 3, 5):
        p = rng.random(1 << m)
        p[rng.random(1 << m) < 0.3] = 0.0
        p /= p.sum()
        draws = np.concatenate([rng.random(500), [0.0, np.nextafter(1.0, 0.0)], np.cumsum(p)[:-1]])
        got = sample_outcomes(p, m, draws)
        for r, o in zip(draws, got):
            i = one(p, float(r))
            assert o == [(i >> (m - 1 - b)) & 1 for b in range(m)]
    human, obj = format_measurement([[1, 0], [0, 1], [1, 0]], 3, [2, 0], 4)
    assert human.splitlines() == ["Measurement results (3 shots):", "  |01> : 1 (33.3%)", "  |10> : 2 (66.7%)"]
    assert obj == {"num_qubits": 4, "shots": 3, "locs": [2, 0], "counts": {"01": 1, "10": 2},
                   "outcomes": [[1, 0], [0, 1], [1, 0]]}


@pytest.mark.gpu
def test_cli_measure_on_gpu(tmp_path):
    """measure over a state file: the outcomes are those the oracle's
    marginal probabilities give for the same seeded draws."""
    from yao_rs.cli import sample_outcomes

    rng = np.random.default_rng(5)
    n = 6
    st = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    st /= np.linalg.norm(st)
    spath = tmp_path / "s.state"
    with open(spath, "wb") as f:
        write_state(st, f)
    for locs, arg in (([3, 0, 5], ["--locs", "3,0,5"]), (list(range(n)), [])):
        out = json.loads(_cli("measure", str(spath), "--shots", "300", "--seed", "17", *arg, "--json").stdout)
        draws = np.random.default_rng(17).random(300)
        want = sample_outcomes(O.probs(st, n, locs), len(locs), draws)
        assert out["outcomes"] == want
        assert out["shots"] == 300 and sum(out["counts"].values()) == 300
        assert out["locs"] == (locs if arg else None)
