"""Pins the CPU oracle to yao-rs's golden vectors and known answers.

Mirrors yao-rs's own tests: src/unit_tests/instruct_qubit.rs:49-410,
tests/suites/apply.rs:699-733, tests/suites/measure.rs:680-705,
src/unit_tests/gate.rs (gates.json), src/unit_tests/noise.rs:307-501,
bitbasis/src/iterate_control.rs:165-219, bitbasis/src/bit_ops.rs:119-195,
src/unit_tests/ad.rs:18-225.  These run on the CPU only.
"""
import math

import numpy as np
import pytest

import oracle as O
import yao_rs as Y
from helpers import (circuit_from_case, gate_kind, matrix_pairs, matrix_reim, named_gate, noise_from_key, pairs, state,
                     tfim)
from yao_rs import Gate

TOL_GOLDEN = 1e-10  # the tolerance yao-rs's own tests use for these fixtures (1e-8 for instruct "all cases")


def close(a, b, tol):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) <= tol


# --------------------------------------------------------------- bitbasis
def test_itercontrol_known_answers():
    # bitbasis/src/iterate_control.rs:165-219
    assert O.itercontrol(7, [0, 2, 3, 6], [1, 0, 1, 0]) == [9, 11, 25, 27, 41, 43, 57, 59]
    assert O.itercontrol(3, [], []) == list(range(8))
    assert O.itercontrol(2, [0, 1], [1, 0]) == [1]
    pos = [0, 2, 4, 6, 8, 10, 12, 14, 16, 18]
    cfg = [1, 0, 1, 0, 1, 0, 1, 0, 1, 0]
    vals = O.itercontrol(19, pos, cfg)
    assert len(vals) == 1 << 9
    for b in vals:
        for p, c in zip(pos, cfg):
            assert (b >> p) & 1 == c
    assert O.controller([0, 2], [1, 0], 0b001)
    assert not O.controller([0, 2], [1, 0], 0b101)
    assert not O.controller([0, 2], [1, 0], 0b000)


def test_bit_ops_known_answers():
    # bitbasis/src/bit_ops.rs:119-195
    L = O.lib()
    import ctypes as C
    arr = (C.c_uint64 * 2)(0, 2)
    assert L.orc_bmask(arr, 2) == 0b101
    assert L.orc_bmask(arr, 0) == 0
    assert L.orc_bmask_range(1, 4) == 0b1110
    assert L.orc_swapbits(0b1011, 1, 2) == 0b1101
    assert L.orc_swapbits(0b1010, 1, 3) == 0b1010
    assert L.orc_breflect(0b1011, 4) == 0b1101
    assert L.orc_neg(0b1111, 4) == 0
    assert L.orc_neg(0b0111, 4) == 0b1000
    assert L.orc_btruncate(0b101101, 3) == 0b101
    assert L.orc_btruncate(0b101101, 0) == 0


# ------------------------------------------------------------ instruct.json
def _case_matrix(case):
    if "gate_matrix" in case:
        return matrix_pairs(case["gate_matrix"])
    name = case.get("gate_name", "")
    if name in ("PSWAP", "CPHASE", ""):
        return None  # not in the Gate enum (yao-rs skips these, instruct_qubit.rs:247)
    return named_gate(name, case.get("theta", 0.0)).matrix()


def instruct_cases(golden):
    return [c for c in golden("instruct")["cases"]]


def test_instruct_all_cases(golden):
    """src/unit_tests/instruct_qubit.rs:265-370 plus the multi-site cases."""
    tested = 0
    for case in instruct_cases(golden):
        label = case["label"]
        if "regression" in label or "measure" in label or "locs" not in case:
            continue
        m = _case_matrix(case)
        if m is None:
            continue
        n = case["nbits"]
        locs = case["locs"]
        ctrl = case.get("ctrl_locs", [])
        bits = case.get("ctrl_bits", [])
        inp = pairs(case["input_state"])
        exp = pairs(case["output_state"])
        d2 = m.size
        if d2 == 4 and len(locs) == 1:
            out = (O.instruct("1q_controlled", inp, n, locs[0], m.reshape(-1), ctrl, bits, len(ctrl)) if ctrl
                   else O.instruct("1q", inp, n, locs[0], m.reshape(-1)))
        elif d2 == 16 and len(locs) == 2:
            out = (O.instruct("2q_controlled", inp, n, locs, m.reshape(-1), ctrl, bits, len(ctrl)) if ctrl
                   else O.instruct("2q", inp, n, locs, m.reshape(-1)))
        elif d2 == 4 and len(locs) > 1 and not ctrl:
            # "X/Y/Z on all sites": the 1-qubit gate on every listed site
            out = inp
            for loc in locs:
                out = O.instruct("1q", out, n, loc, m.reshape(-1))
        else:
            continue
        assert close(out, exp, 1e-10), label
        tested += 1
    assert tested >= 40


def test_instruct_regression_2q(golden):
    """src/unit_tests/instruct_qubit.rs:376-410: 20 random 2q gates on 10 qubits."""
    case = [c for c in instruct_cases(golden) if "regression" in c["label"]][0]
    g = matrix_pairs(case["gate_matrix"]).reshape(-1)
    st = pairs(case["input_state"])
    for p in case["gate_pairs"]:
        st = O.instruct("2q", st, case["nbits"], list(p), g)
    assert close(st, pairs(case["output_state"]), 1e-10)


def test_instruct_diag_paths_match_dense(golden):
    """The diagonal and X/SWAP instruct paths against the dense ones."""
    rng = np.random.default_rng(5)
    n = 6
    psi = rng.normal(size=64) + 1j * rng.normal(size=64)
    d = np.exp(1j * rng.uniform(-3, 3, 2))
    for loc in range(n):
        a = O.instruct("1q_diag", psi, n, loc, d)
        b = O.instruct("1q", psi, n, loc, np.array([d[0], 0, 0, d[1]]))
        assert close(a, b, 1e-14)
        x = O.instruct("x", psi, n, loc)
        y = O.instruct("1q", psi, n, loc, np.array([0, 1, 1, 0], dtype=complex))
        assert close(x, y, 0)
    d4 = np.exp(1j * rng.uniform(-3, 3, 4))
    for locs in ([1, 4], [4, 1], [0, 5]):
        a = O.instruct("2q_diag", psi, n, locs, d4)
        b = O.instruct("2q", psi, n, locs, np.diag(d4).reshape(-1))
        assert close(a, b, 1e-14)
        s = O.instruct("swap", psi, n, locs)
        t = O.instruct("2q", psi, n, locs, Gate.SWAP.matrix().reshape(-1))
        assert close(s, t, 0)


# --------------------------------------------------------------- apply.json
def test_apply_ground_truth(golden):
    """tests/suites/apply.rs:699-733 (qudit cases are out of scope: ArrayReg is qubit-only)."""
    tested = 0
    for case in golden("apply")["cases"]:
        if not all(d == 2 for d in case["dims"]):
            continue
        c = circuit_from_case(case)
        inp = state(case["input_state_re"], case["input_state_im"])
        out = O.apply_circuit(c, inp)
        assert close(out, state(case["output_state_re"], case["output_state_im"]), TOL_GOLDEN), case["label"]
        tested += 1
    assert tested >= 60


def test_measure_ground_truth(golden):
    """tests/suites/measure.rs:680-705."""
    cases = golden("measure")["cases"]
    for case in cases:
        case2 = dict(case, dims=[2] * case["num_qubits"])
        c = circuit_from_case(case2)
        n = case["num_qubits"]
        z = np.zeros(1 << n, complex)
        z[0] = 1
        out = O.apply_circuit(c, z)
        assert close(O.probs(out, n), case["probabilities"], TOL_GOLDEN), case["label"]
    assert len(cases) == 11


def test_pysim_ground_truth(golden):
    """States from yao-rs's numpy simulator (scripts/reference_simulate.py)."""
    for case in golden("pysim")["cases"]:
        circ = case["circuit"]
        n = circ["num_qubits"]
        els = []
        for el in circ["elements"]:
            g = named_gate(el["gate"], (el.get("params") or [0.0])[0])
            cs = el.get("controls", [])
            els.append(Y.PositionedGate(g, el["targets"], cs, el.get("control_configs", [True] * len(cs))))
        c = Y.Circuit.qubits(n, els)
        z = np.zeros(1 << n, complex)
        z[0] = 1
        out = O.apply_circuit(c, z)
        assert close(out, state(case["state_re"], case["state_im"]), 1e-12), case["label"]


def test_ordering_known_answer():
    """tests/suites/measure.rs:588-607: index 4 of 3 qubits is qubit 0 = 1."""
    psi = np.zeros(8, complex)
    psi[4] = 1
    assert list(O.probs(psi, 3, [0])) == [0.0, 1.0]


# ---------------------------------------------------------------- gates.json
def test_gate_matrices(golden):
    for g in golden("gates")["gates"]:
        exp = np.asarray(g["matrix_re"]) + 1j * np.asarray(g["matrix_im"])
        kind = gate_kind(g["name"])
        params = g["params"]
        got = O.gate_matrix(kind, params)
        assert close(got, exp, 1e-10), (g["name"], params)


# ---------------------------------------------------------------- noise.json
def test_kraus_and_superop(golden):
    data = golden("noise")
    for key, fx in data["kraus"].items():
        ch = noise_from_key(key)
        e, keep = ch._element()
        ks = O.noise_kraus(e)
        assert len(ks) == fx["num_kraus"], key
        for k, exp in zip(ks, fx["kraus"]):
            assert close(k, matrix_reim(exp), 1e-10), key
        assert close(O.noise_superop(e), matrix_reim(fx["superop"]), 1e-10), key


def _dm_case_circuit(key):
    H = Gate.H
    if key == "h_amplitude_damping_0.3":
        return Y.Circuit.qubits(1, [Y.put([0], H), Y.channel([0], Y.NoiseChannel.AmplitudeDamping(0.3, 0.0))]), None
    if key == "bitflip_0.1_on_zero":
        return Y.Circuit.qubits(1, [Y.channel([0], Y.NoiseChannel.BitFlip(0.1))]), None
    if key == "h_phaseflip_0.1":
        return Y.Circuit.qubits(1, [Y.put([0], H), Y.channel([0], Y.NoiseChannel.PhaseFlip(0.1))]), None
    if key == "h_depolarizing_0.1":
        return Y.Circuit.qubits(1, [Y.put([0], H), Y.channel([0], Y.NoiseChannel.Depolarizing(1, 0.1))]), None
    if key == "bell_depolarizing_q0_0.1":
        bell = np.zeros(4, complex)
        bell[0] = bell[3] = 1 / math.sqrt(2)
        return Y.Circuit.qubits(2, [Y.channel([0], Y.NoiseChannel.Depolarizing(1, 0.1))]), bell
    raise KeyError(key)


def dm_cases(golden):
    out = []
    for key, fx in golden("noise")["dm_cases"].items():
        c, psi = _dm_case_circuit(key)
        n = len(fx["dims"])
        if psi is None:
            psi = np.zeros(1 << n, complex)
            psi[0] = 1
        out.append((key, c, psi, n, matrix_reim(fx["rho"])))
    return out


def test_dm_cases(golden):
    """noise.json dm_cases (tests/fixtures/generate_noise.jl:119-155; loc 0 = MSB)."""
    for key, c, psi, n, exp in dm_cases(golden):
        rho = O.dm_apply_circuit(c, O.dm_from_reg(psi, n))
        assert close(rho.reshape(1 << n, 1 << n), exp, 1e-10), key


def test_dm_expectations(golden):
    """noise.json expectations: <Z>, <X> after H (+ channel)."""
    ex = golden("noise")["expectations"]
    cases = {
        "z_h_phaseflip_0.1": ([Y.put([0], Gate.H), Y.channel([0], Y.NoiseChannel.PhaseFlip(0.1))], Y.Op.Z),
        "z_h_pure": ([Y.put([0], Gate.H)], Y.Op.Z),
        "x_h_depolarizing_0.1": ([Y.put([0], Gate.H), Y.channel([0], Y.NoiseChannel.Depolarizing(1, 0.1))], Y.Op.X),
    }
    for key, (els, op) in cases.items():
        c = Y.Circuit.qubits(1, els)
        rho = O.dm_apply_circuit(c, O.dm_from_reg(np.array([1, 0], complex), 1))
        v = O.expect_dm(rho, 1, Y.OperatorPolynomial.single(0, op, 1.0))
        assert abs(v - complex(ex[key]["value_re"], ex[key]["value_im"])) < 1e-10, key


def test_dm_known_answers():
    """src/density_matrix.rs:270-360 tests."""
    z = np.array([1, 0, 0, 0], complex)
    rho = O.dm_from_reg(z, 2)
    assert abs(O.dm_trace(rho, 2) - 1) < 1e-12
    assert abs(O.dm_purity(rho, 2) - 1) < 1e-12
    ghz = np.array([1, 0, 0, 1], complex) / math.sqrt(2)
    red = O.dm_partial_tr(O.dm_from_reg(ghz, 2), 2, [1])
    assert abs(O.dm_purity(red, 1) - 0.5) < 1e-12
    assert abs(O.dm_trace(red, 1) - 1) < 1e-12
    c = Y.Circuit.qubits(1, [Y.channel([0], Y.NoiseChannel.BitFlip(0.5))])
    r2 = O.dm_apply_circuit(c, O.dm_from_reg(np.array([1, 0], complex), 1))
    assert abs(O.dm_purity(r2, 1) - 0.5) < 1e-10


def test_dm_entropy_known_answers():
    """von_neumann_entropy (src/density_matrix.rs:114-123) restated in the
    oracle: 0 for a pure state, ln 2 for half of a Bell pair, n ln 2 for the
    maximally mixed state; density_matrix_from_reg keeps locs ascending."""
    z = np.zeros(8, complex)
    z[5] = 1
    assert abs(O.dm_von_neumann_entropy(O.dm_from_reg(z, 3), 3)) < 1e-14
    bell = np.array([1, 0, 0, 1], complex) / math.sqrt(2)
    for keep in ([0], [1]):
        red = O.density_matrix_from_reg(bell, 2, keep)
        assert abs(O.dm_von_neumann_entropy(red, 1) - math.log(2.0)) < 1e-14
    mixed = (np.eye(4) / 4).astype(complex).ravel()
    assert abs(O.dm_von_neumann_entropy(mixed, 2) - 2 * math.log(2.0)) < 1e-14
    # |psi> = |0>|+> (loc 0 = |0>, the most significant bit).  partial_tr
    # reads a loc as bit `loc` of the index counted from the least
    # significant end (src/density_matrix.rs:90-101), so keeping loc 1 keeps
    # the most significant qubit, |0><0|, and keeping loc 0 keeps |+><+|.
    plus0 = np.array([1, 1, 0, 0], complex) / math.sqrt(2)
    assert np.allclose(O.density_matrix_from_reg(plus0, 2, [1]), [1, 0, 0, 0])
    assert np.allclose(O.density_matrix_from_reg(plus0, 2, [0]), np.full(4, 0.5))


# ---------------------------------------------------------------------- AD
def h_z(site):
    return Y.OperatorPolynomial.single(site, Y.Op.Z, 1.0)


def h_x(site):
    return Y.OperatorPolynomial.single(site, Y.Op.X, 1.0)


def test_ad_analytic():
    """src/unit_tests/ad.rs:18-60."""
    z1 = np.array([1, 0], complex)
    for t in [0.0, 0.3, 0.7, 1.57, 2.0, -0.5]:
        v, g = O.expect_grad(h_z(0), Y.Circuit.qubits(1, [Y.put([0], Gate.Rx(t))]), z1)
        assert abs(v - math.cos(t)) < 1e-10 and abs(g[0] + math.sin(t)) < 1e-10
    for t in [0.0, 0.3, 0.7, 1.57, -0.2]:
        v, g = O.expect_grad(h_x(0), Y.Circuit.qubits(1, [Y.put([0], Gate.Ry(t))]), z1)
        assert abs(v - math.sin(t)) < 1e-10 and abs(g[0] - math.cos(t)) < 1e-10
    for t in [0.1, 0.9, 1.3, -0.4]:
        c = Y.Circuit.qubits(1, [Y.put([0], Gate.H), Y.put([0], Gate.Rz(t))])
        v, g = O.expect_grad(h_x(0), c, z1)
        assert abs(v - math.cos(t)) < 1e-10 and abs(g[0] + math.sin(t)) < 1e-10


def test_ad_rejects_channels():
    """src/unit_tests/ad.rs:169-185 (should_panic "noise channel")."""
    c = Y.Circuit.qubits(1, [Y.put([0], Gate.Rx(0.3)), Y.channel([0], Y.NoiseChannel.BitFlip(0.1))])
    with pytest.raises(ValueError, match="noise channel"):
        O.expect_grad(h_z(0), c, np.array([1, 0], complex))


def test_ad_finite_difference():
    """src/unit_tests/ad.rs:187-225: central differences, h = 1e-5, tol 1e-6."""
    rng = np.random.default_rng(3)
    n = 3
    els = []
    for _ in range(3):
        for q in range(n):
            els.append(Y.put([q], Gate.Rx(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
        els.append(Y.control([0], [1], Gate.Ry(float(rng.uniform(-3, 3)))))
        els.append(Y.put([1, 2], Gate.FSim(float(rng.uniform(-3, 3)), float(rng.uniform(-3, 3)))))
        els.append(Y.control([2], [0], Gate.Phase(float(rng.uniform(-3, 3)))))
    c = Y.Circuit.qubits(n, els)
    op = tfim(n, 0.7)
    psi0 = np.zeros(8, complex)
    psi0[0] = 1
    v, g = O.expect_grad(op, c, psi0)
    p0 = c.parameters()
    h = 1e-5
    for i in range(len(p0)):
        pp, pm = list(p0), list(p0)
        pp[i] += h
        pm[i] -= h
        c.dispatch(pp)
        fp = O.expect_arrayreg(O.apply_circuit(c, psi0), n, op).real
        c.dispatch(pm)
        fm = O.expect_arrayreg(O.apply_circuit(c, psi0), n, op).real
        assert abs((fp - fm) / (2 * h) - g[i]) < 1e-6, i
    c.dispatch(p0)


def test_sample_and_measure_bookkeeping():
    """src/measure.rs:140-240: sequential cumsum sampling and post-processing."""
    p = np.array([0.1, 0.2, 0.3, 0.4])
    assert O.sample_from_probs(p, 0.0) == 0
    assert O.sample_from_probs(p, 0.1) == 1
    assert O.sample_from_probs(p, 0.2999) == 1
    assert O.sample_from_probs(p, 0.3) == 1  # 0.1 + 0.2 rounds above 0.3
    assert O.sample_from_probs(p, 0.31) == 2
    assert O.sample_from_probs(p, 0.99999) == 3
    # GHZ(3): measuring loc 0 fixes every qubit
    psi = np.zeros(8, complex)
    psi[0] = psi[7] = 1 / math.sqrt(2)
    out, rem, st = O.measure_with_postprocess(psi, 3, [0], 2, 0, 0.75)
    assert out == [1]
    assert abs(rem[3] - 1) < 1e-12
    out, _, st = O.measure_with_postprocess(psi, 3, [0, 2], 1, 0, 0.75)
    assert out == [1, 1]
    assert abs(st[2] - 1) < 1e-12  # |111> reset on locs 0 and 2 -> |010>
