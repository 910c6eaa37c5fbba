"""CPU tests of the library's host side: the C ABI loads and exports every
symbol of include/yao_gpu.h, and the host-only code (gate matrices, Kraus
operators, circuit validation, noise parameter checks) matches yao-rs.
No device code runs here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import yao_rs as Y
from helpers import gate_kind, matrix_reim, noise_from_key
from yao_rs import Gate, NoiseChannel
from yao_rs import _abi as A

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "yao_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yao_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    names = header_functions()
    assert len(names) >= 50
    L = C.CDLL(str(A.LIB_PATH))
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(A.SIGNATURES), set(names) ^ set(A.SIGNATURES)


def test_abi_version_and_error_string():
    assert A.lib().yao_abi_version() == 1
    assert isinstance(A.lib().yao_last_error(), bytes)


def test_gate_matrices_match_golden(golden):
    for g in golden("gates")["gates"]:
        exp = np.asarray(g["matrix_re"]) + 1j * np.asarray(g["matrix_im"])
        p = g["params"]
        gate = Gate(gate_kind(g["name"]), p)
        got = gate.matrix()
        assert np.max(np.abs(got - exp)) < 1e-10, g["name"]
        # and bit-identical to the oracle's restatement
        assert np.array_equal(got, O.gate_matrix(gate_kind(g["name"]), p)), g["name"]


def test_kraus_superop_match_golden(golden):
    for key, fx in golden("noise")["kraus"].items():
        ch = noise_from_key(key)
        ks = ch.kraus_operators()
        assert len(ks) == fx["num_kraus"]
        for k, e in zip(ks, fx["kraus"]):
            assert np.max(np.abs(k - matrix_reim(e))) < 1e-10, key
        assert np.max(np.abs(ch.superop() - matrix_reim(fx["superop"]))) < 1e-10, key
        e, keep = ch._element()
        for k, ko in zip(ks, O.noise_kraus(e)):
            assert np.array_equal(k, ko), key


def test_depolarizing_two_qubit_kraus():
    ch = NoiseChannel.Depolarizing(2, 0.2)
    ks = ch.kraus_operators()
    assert len(ks) == 16 and ks[0].shape == (4, 4)
    s = sum(k.conj().T @ k for k in ks)
    assert np.max(np.abs(s - np.eye(4))) < 1e-12
    e, keep = ch._element()
    for k, ko in zip(ks, O.noise_kraus(e)):
        assert np.array_equal(k, ko)


@pytest.mark.parametrize("ch,msg", [
    (NoiseChannel.BitFlip(1.5), "must be in \\[0, 1\\]"),
    (NoiseChannel.PauliChannel(0.5, 0.4, 0.3), "sum <= 1"),
    (NoiseChannel.AmplitudeDamping(0.1, 2.0), "excited_population"),
    (NoiseChannel.ThermalRelaxation(1.0, 3.0, 0.1), "t2"),
    (NoiseChannel.Reset(0.7, 0.6), "Reset probabilities"),
])
def test_noise_parameter_validation(ch, msg):
    """src/noise.rs:90-176: invalid parameters are rejected with its messages."""
    with pytest.raises(Y.YaoError, match=msg):
        ch.kraus_operators()


def test_circuit_validation_errors():
    """src/circuit.rs:150-272 and src/unit_tests/circuit.rs."""
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.PositionedGate(Gate.X, [0], [1], [True, False])])
    assert e.value.kind == "ControlConfigLengthMismatch"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.put([2], Gate.X)])
    assert e.value.kind == "LocOutOfRange"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.control([0], [0], Gate.X)])
    assert e.value.kind == "OverlappingLocs"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit([3, 2], [Y.control([0], [1], Gate.X)])
    assert e.value.kind == "ControlSiteNotQubit"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit([3, 2], [Y.put([0], Gate.X)])
    assert e.value.kind == "NamedGateTargetNotQubit"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.put([0, 1], Gate.H)])
    assert e.value.kind == "MatrixSizeMismatch"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.channel([0, 1], NoiseChannel.BitFlip(0.1))])
    assert e.value.kind == "MatrixSizeMismatch"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.channel([1, 1], NoiseChannel.Depolarizing(2, 0.1))])
    assert e.value.kind == "OverlappingLocs"
    with pytest.raises(Y.CircuitError) as e:
        Y.Circuit.qubits(2, [Y.label(5, "x")])
    assert e.value.kind == "LocOutOfRange"
    # valid qudit circuit with a custom gate (validation only; ArrayReg is qubit-only)
    Y.Circuit([3], [Y.put([0], Gate.Custom(np.eye(3)))])


def test_parameters_dispatch_dagger():
    """src/circuit.rs:308-378 and src/gate.rs:198-281."""
    c = Y.Circuit.qubits(2, [Y.put([0], Gate.Rx(0.1)), Y.put([0, 1], Gate.FSim(0.2, 0.3)), Y.put([1], Gate.H),
                             Y.control([0], [1], Gate.Phase(0.4))])
    assert c.num_params() == 4
    assert c.parameters() == [0.1, 0.2, 0.3, 0.4]
    c.dispatch([1.0, 2.0, 3.0, 4.0])
    assert c.parameters() == [1.0, 2.0, 3.0, 4.0]
    with pytest.raises(AssertionError):
        c.dispatch([1.0])
    d = c.dagger()
    assert [el.gate for el in d.elements] == [Gate.Phase(-4.0), Gate.H, Gate.FSim(-2.0, -3.0), Gate.Rx(-1.0)]
    assert Gate.S.dagger() == Gate.Phase(-np.pi / 2)
    assert Gate.T.dagger() == Gate.Phase(-np.pi / 4)
    sx = Gate.SqrtX.dagger()
    assert np.allclose(sx.matrix() @ Gate.SqrtX.matrix(), np.eye(2))
    iw = Gate.ISWAP.dagger()
    assert np.allclose(iw.matrix() @ Gate.ISWAP.matrix(), np.eye(4))


def test_operator_string_normalisation():
    """src/operator.rs:27-33: stable sort by site, Op::I dropped."""
    s = Y.OperatorString([(2, Y.Op.Z), (0, Y.Op.X), (1, Y.Op.I), (0, Y.Op.Y)])
    assert s.ops() == [(0, Y.Op.X), (0, Y.Op.Y), (2, Y.Op.Z)]
    p = Y.OperatorPolynomial.single(0, Y.Op.Z, 2.0) + Y.OperatorPolynomial.identity()
    assert len(p) == 2 and p.coeffs() == [2.0, 1.0]
    assert (-p).coeffs() == [-2.0, -1.0]


def test_plan_info_host_only():
    """The TILED / FUSED planner runs on the host: every gate lands in a pass,
    fused blocks never outnumber the gates, tensor-core ops appear only for
    complex64 FUSED plans with 2^12 tiles."""
    from helpers import layered_circuit, random_circuit
    rng = np.random.default_rng(3)
    for n in (8, 14, 20):
        c = random_circuit(rng, n, 200, max_ctrl=2)
        tiled = Y.plan_info(c, Y.C128, Y.MODE_TILED, 0, 10, 2)
        assert tiled["single_gate_passes"] == 0 and tiled["tensor_core_ops"] == 0
        assert tiled["ops"] <= len(c.elements) and tiled["passes"] >= 1
        for k in (2, 4, 5):
            f = Y.plan_info(c, Y.C64, Y.MODE_FUSED, k, 12, 3)
            assert f["blocks"] <= len(c.elements) and f["ops"] == f["blocks"]
            f128 = Y.plan_info(c, Y.C128, Y.MODE_FUSED, k, 12, 3)
            assert f128["tensor_core_ops"] == 0 and f128["blocks"] == f["blocks"]
    c = layered_circuit(16, 10, seed=1)
    f = Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 12, 3)
    assert f["tensor_core_ops"] > 0
    assert Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 11, 3)["tensor_core_ops"] == 0
    with pytest.raises(Y.YaoError):
        Y.plan_info(c, Y.C64, Y.MODE_PLAIN, 5, 12, 3)


def test_planner_low_bits_and_one_qubit_runs():
    """Planner rules on the 30-qubit, 40-layer benchmark circuit: bits 0..3
    are always tile bits and do not count against a pass's moving bits, and
    consecutive 1-qubit gates on one qubit are multiplied together before
    fusion.  Each layer's Rx.Ry.Rz on a qubit is one gate, so TILED keeps
    every gate as its own op while FUSED k = 1 needs one block per qubit and
    layer plus the CNOTs at most."""
    import sys
    sys.path.insert(0, str(ROOT))
    import bench
    n, layers = 30, 40
    c = Y.Circuit.qubits(n, [el for l in range(layers) for el in bench.layer_elements(Y, n, l)])
    ngates = len(c.elements)
    assert ngates == 4180
    tiled = Y.plan_info(c, Y.C128, Y.MODE_TILED, 0, 12, 3)
    assert tiled["ops"] == ngates and tiled["passes"] <= 200
    f1 = Y.plan_info(c, Y.C128, Y.MODE_FUSED, 1, 12, 3)
    # at most one block per merged 1-qubit run or CNOT (blocks also absorb
    # later gates on their qubits)
    assert f1["blocks"] <= ngates - 2 * n * layers
    f5 = Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 12, 3)
    assert f5["blocks"] == 130 and f5["passes"] <= 70 and f5["tensor_core_ops"] == 109


def test_grad_plan_reorders_commuting_steps(monkeypatch):
    """expect_grad's tiled reverse sweep for the VQE ansatz at n = 24 (8
    layers of Ry.Rz on every qubit and a CNOT ring, 384 parameters): list
    scheduling over the steps' qubits lets a pass take steps on disjoint
    qubits out of sweep order, halving the passes of the in-order plan; every
    parameter keeps one generator dot, and every Ry.Rz pair folds into one
    op next to its CNOT.  Within register segments, a CNOT merges into the
    folded run on its target (191 of the 192 CNOTs in the list-scheduled
    plan, 7 in sweep order)."""
    from helpers import vqe_ansatz
    rng = np.random.default_rng(2024)
    c = vqe_ansatz(24, 8, rng.uniform(-3, 3, size=2 * 24 * 8))
    got = Y.grad_plan_info(c)
    assert got == {"passes": 23, "ops": 193, "dots": 384}
    monkeypatch.setenv("YAO_ADJ_XFOLD", "0")
    assert Y.grad_plan_info(c) == {"passes": 23, "ops": 384, "dots": 384}
    monkeypatch.delenv("YAO_ADJ_XFOLD")
    monkeypatch.setenv("YAO_ADJ_REORDER", "0")
    assert Y.grad_plan_info(c) == {"passes": 45, "ops": 377, "dots": 384}
    # a 3-qubit gate sends expect_grad to the per-gate form
    wide = Y.Circuit.qubits(4, [Y.put([0, 1, 2], Gate.Custom(np.eye(8), False, "I3"))])
    with pytest.raises(Y.YaoError):
        Y.grad_plan_info(wide)


def test_gate_generator_matrices():
    """Gate::generator_matrix (src/gate.rs:153-193): the oracle's entries
    bit for bit, the definition G = (dU/dtheta_i) U^-1 by central differences,
    and the assert on i as an error with yao-rs's message."""
    cases = [(Gate.Rx(0.7), 0), (Gate.Ry(-1.3), 0), (Gate.Rz(2.1), 0), (Gate.Phase(0.4), 0),
             (Gate.FSim(0.3, 1.1), 0), (Gate.FSim(0.3, 1.1), 1)]
    h = 1e-6
    for g, i in cases:
        G = g.generator_matrix(i)
        assert np.array_equal(G, O.gate_generator(g.kind, i)), (g, i)
        hi, lo = list(g.params), list(g.params)
        hi[i] += h
        lo[i] -= h
        dU = (Gate(g.kind, hi).matrix() - Gate(g.kind, lo).matrix()) / (2 * h)
        assert np.max(np.abs(dU @ np.linalg.inv(g.matrix()) - G)) < 1e-8, (g, i)
    for g, i, np_ in ((Gate.Rx(0.1), 1, 1), (Gate.FSim(0.1, 0.2), 2, 2), (Gate.H, 0, 0),
                      (Gate.Custom(np.eye(2)), 0, 0)):
        with pytest.raises(Y.YaoError) as e:
            g.generator_matrix(i)
        assert f"generator_matrix index {i} out of range (num_params={np_})" in str(e.value)
    with pytest.raises(ValueError):
        Gate.Rx(0.1).generator_matrix(-1)
