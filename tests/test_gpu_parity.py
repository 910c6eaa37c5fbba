"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle
and yao-rs's golden vectors.

Bars: PLAIN and TILED application, density-matrix evolution, partial
trace, full probabilities, the lambda vector and measurement bookkeeping
are bit-exact (max |diff| == 0); reductions (expectation values, norms,
purity, marginal probabilities, gradients) agree to 1e-12 relative;
FUSED (FP64) to 1e-10 with 1 - F <= 1e-12; FUSED on complex64 to
1 - F <= 1e-6.
"""
import math

import numpy as np
import pytest

import oracle as O
import yao_rs as Y
from helpers import (circuit_from_case, layered_circuit, matrix_pairs, matrix_reim, named_gate, noise_from_key, pairs,
                     qft_circuit, random_circuit, random_state, state, tfim, vqe_ansatz)
from yao_rs import Gate, NoiseChannel

pytestmark = pytest.mark.gpu

MODES = [Y.MODE_PLAIN, Y.MODE_TILED]


def maxdiff(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0


def gpu_apply(c, psi, mode=Y.MODE_PLAIN, k=0):
    r = Y.ArrayReg.from_vec(c.nbits, psi)
    Y.apply_inplace(c, r, mode, k)
    return r.state_vec()


# ------------------------------------------------------------------ golden
def test_instruct_cases_bit_exact(golden):
    """instruct.json cases as one-gate circuits (Custom matrices follow the
    same dispatch as the named gates)."""
    tested = 0
    for case in golden("instruct")["cases"]:
        if "locs" not in case or "regression" in case["label"]:
            continue
        if "gate_matrix" in case:
            g = Gate.Custom(matrix_pairs(case["gate_matrix"]))
        elif case.get("gate_name") in (None, "PSWAP", "CPHASE"):
            continue
        else:
            g = named_gate(case["gate_name"], case.get("theta", 0.0))
        n, locs = case["nbits"], case["locs"]
        ctrl, bits = case.get("ctrl_locs", []), case.get("ctrl_bits", [])
        if g.num_sites() == 1 and len(locs) > 1:
            els = [Y.put([l], g) for l in locs]
        else:
            els = [Y.PositionedGate(g, locs, ctrl, [bool(b) for b in bits])]
        c = Y.Circuit.qubits(n, els)
        inp = pairs(case["input_state"])
        for mode in MODES:
            out = gpu_apply(c, inp, mode)
            assert maxdiff(out, O.apply_circuit(c, inp)) == 0.0, case["label"]
            assert maxdiff(out, pairs(case["output_state"])) < 1e-10, case["label"]
        tested += 1
    assert tested >= 40


def test_instruct_regression_2q(golden):
    case = [c for c in golden("instruct")["cases"] if "regression" in c["label"]][0]
    g = Gate.Custom(matrix_pairs(case["gate_matrix"]))
    c = Y.Circuit.qubits(case["nbits"], [Y.put(list(p), g) for p in case["gate_pairs"]])
    out = gpu_apply(c, pairs(case["input_state"]))
    assert maxdiff(out, pairs(case["output_state"])) < 1e-10


def test_apply_ground_truth(golden):
    tested = 0
    for case in golden("apply")["cases"]:
        if not all(d == 2 for d in case["dims"]):
            continue
        c = circuit_from_case(case)
        inp = state(case["input_state_re"], case["input_state_im"])
        ref = O.apply_circuit(c, inp)
        for mode in MODES:
            out = gpu_apply(c, inp, mode)
            assert maxdiff(out, ref) == 0.0, case["label"]
        assert maxdiff(out, state(case["output_state_re"], case["output_state_im"])) < 1e-10, case["label"]
        tested += 1
    assert tested >= 60


def test_apply_rejects_qudits(golden):
    case = [c for c in golden("apply")["cases"] if not all(d == 2 for d in c["dims"])][0]
    c = circuit_from_case(case)
    r = Y.ArrayReg.zero_state(len(case["dims"]))
    with pytest.raises(Y.YaoError, match="qubit-only"):
        Y.apply_inplace(c, r)
    with pytest.raises(Y.YaoError, match="mismatch"):
        Y.apply_inplace(Y.Circuit.qubits(3, [Y.put([0], Gate.H)]), Y.ArrayReg.zero_state(2))


def test_measure_ground_truth(golden):
    for case in golden("measure")["cases"]:
        c = circuit_from_case(dict(case, dims=[2] * case["num_qubits"]))
        r = Y.apply(c, Y.ArrayReg.zero_state(case["num_qubits"]))
        assert maxdiff(Y.probs(r), case["probabilities"]) < 1e-10, case["label"]


def test_pysim_ground_truth(golden):
    for case in golden("pysim")["cases"]:
        circ = case["circuit"]
        n = circ["num_qubits"]
        els = []
        for el in circ["elements"]:
            g = named_gate(el["gate"], (el.get("params") or [0.0])[0])
            cs = el.get("controls", [])
            els.append(Y.PositionedGate(g, el["targets"], cs, el.get("control_configs", [True] * len(cs))))
        c = Y.Circuit.qubits(n, els)
        out = Y.apply(c, Y.ArrayReg.zero_state(n)).state_vec()
        assert maxdiff(out, state(case["state_re"], case["state_im"])) < 1e-12, case["label"]


# ------------------------------------------------------- random circuits
@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 11, 13, 15])
def test_random_circuits_bit_exact(n):
    rng = np.random.default_rng(100 + n)
    for rep in range(3):
        c = random_circuit(rng, n, 60, max_ctrl=min(3, n - 1) if n > 1 else 0)
        psi = random_state(rng, n)
        ref = O.apply_circuit(c, psi)
        for mode in MODES:
            out = gpu_apply(c, psi, mode)
            assert maxdiff(out, ref) == 0.0, (n, rep, mode)


@pytest.mark.parametrize("n", [4, 12, 16])
def test_fused_fp64_and_c64(n):
    rng = np.random.default_rng(7 + n)
    c = random_circuit(rng, n, 120, max_ctrl=2)
    psi = random_state(rng, n)
    ref = O.apply_circuit(c, psi)
    for k in (2, 4, 5, 6):
        out = gpu_apply(c, psi, Y.MODE_FUSED, k)
        assert maxdiff(out, ref) < 1e-10, k
        assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-12, k
    r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
    Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
    out = r.state_vec().astype(np.complex128)
    assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6


def test_autotune_and_tile_shapes(monkeypatch):
    """The autotuner's choice is a valid shape, leaves the register alone, and
    every tile shape it can pick keeps TILED bit-exact and FUSED in bounds."""
    rng = np.random.default_rng(99)
    n = 15
    c = random_circuit(rng, n, 150, max_ctrl=2)
    psi = random_state(rng, n)
    ref = O.apply_circuit(c, psi)
    r = Y.ArrayReg.from_vec(n, psi)
    ch = Y.autotune(c, r, Y.MODE_TILED)
    assert 10 <= ch["tile_bits"] <= 12 and 2 <= ch["reg_bits"] <= 3
    assert maxdiff(r.state_vec(), psi) == 0.0
    Y.apply_inplace(c, r, Y.MODE_TILED)
    assert maxdiff(r.state_vec(), ref) == 0.0
    r = Y.ArrayReg.from_vec(n, psi)
    ch = Y.autotune(c, r, Y.MODE_FUSED, 0)
    assert 2 <= ch["k"] <= 6
    Y.apply_inplace(c, r, Y.MODE_FUSED, 0)
    assert maxdiff(r.state_vec(), ref) < 1e-10
    # complex64: the width and whether dense blocks take the tensor cores
    r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
    ch = Y.autotune(c, r, Y.MODE_FUSED, 0)
    assert 2 <= ch["k"] <= 6 and ch["tensor_cores"] in (0, 1)
    assert ch["tensor_cores"] == 0 or (ch["tile_bits"] == 12 and 3 <= ch["k"] <= 5)
    Y.apply_inplace(c, r, Y.MODE_FUSED, 0)
    out = r.state_vec().astype(np.complex128)
    assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6
    for tb, rb in ((10, 2), (11, 2), (11, 3), (12, 3), (12, 2), (9, 1)):
        monkeypatch.setenv("YAO_TILE_BITS", str(tb))
        monkeypatch.setenv("YAO_REG_BITS", str(rb))
        assert maxdiff(gpu_apply(c, psi, Y.MODE_TILED), ref) == 0.0, (tb, rb)
        assert maxdiff(gpu_apply(c, psi, Y.MODE_FUSED, 4), ref) < 1e-10, (tb, rb)
    for tb, rb in ((13, 4), (12, 4), (11, 2), (12, 3)):
        monkeypatch.setenv("YAO_TILE_BITS", str(tb))
        monkeypatch.setenv("YAO_REG_BITS", str(rb))
        r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
        Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
        out = r.state_vec().astype(np.complex128)
        assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6, (tb, rb)


def test_batched_launch():
    """Uneven circuits (3..14 qubits, 1..6 layers) in one persistent launch:
    TILED is bit-exact against the oracle, FUSED (c128 and c64) within its
    bars; registers of other circuits are not touched."""
    rng = np.random.default_rng(404)
    circuits, states = [], []
    for i in range(24):
        n = int(rng.integers(3, 15))
        c = random_circuit(rng, n, int(rng.integers(5, 80)), max_ctrl=2) if i % 3 == 0 else \
            layered_circuit(n, int(rng.integers(1, 7)), seed=int(rng.integers(1 << 30)))
        circuits.append(c)
        states.append(random_state(rng, n))
    refs = [O.apply_circuit(c, s) for c, s in zip(circuits, states)]
    regs = [Y.ArrayReg.from_vec(c.nbits, s) for c, s in zip(circuits, states)]
    Y.batch_apply(circuits, regs, Y.MODE_TILED)
    for r, ref in zip(regs, refs):
        assert maxdiff(r.state_vec(), ref) == 0.0
    for k in (2, 5):
        regs = [Y.ArrayReg.from_vec(c.nbits, s) for c, s in zip(circuits, states)]
        Y.batch_apply(circuits, regs, Y.MODE_FUSED, k)
        for r, ref in zip(regs, refs):
            assert maxdiff(r.state_vec(), ref) < 1e-10
    regs = [Y.ArrayReg.from_vec(c.nbits, s).to_precision(Y.C64) for c, s in zip(circuits, states)]
    Y.batch_apply(circuits, regs, Y.MODE_FUSED, 2)
    for r, ref in zip(regs, refs):
        out = r.state_vec().astype(np.complex128)
        assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6


def test_layered_circuit_exact_and_roundtrip():
    """The layered workload (Rx, Ry, Rz per qubit + CNOT brickwork) at n=16
    against the oracle, and apply -> dagger round trip at n=24."""
    c = layered_circuit(16, 4, seed=11)
    z = np.zeros(1 << 16, complex)
    z[0] = 1
    ref = O.apply_circuit(c, z)
    for mode in MODES:
        assert maxdiff(gpu_apply(c, z, mode), ref) == 0.0
    big = layered_circuit(24, 3, seed=12)
    r = Y.ArrayReg.zero_state(24)
    Y.apply_inplace(big, r, Y.MODE_TILED)
    n1 = r.norm()
    Y.apply_inplace(big.dagger(), r, Y.MODE_TILED)
    v = r.state_vec()
    assert abs(n1 - 1) < 1e-12
    assert abs(v[0] - 1) < 1e-11 and np.max(np.abs(v[1:])) < 1e-11


def test_qft20_bit_exact():
    """QFT on 20 qubits (H + 190 controlled phases + 10 SWAPs) on a seeded
    Gaussian state, against the oracle (max-abs 0; the bar is 1e-12)."""
    rng = np.random.default_rng(2026)
    psi = random_state(rng, 20)
    c = qft_circuit(20)
    assert len(c.elements) == 220
    ref = O.apply_circuit(c, psi)
    for mode in MODES:
        assert maxdiff(gpu_apply(c, psi, mode), ref) == 0.0


def test_channels_ignored_in_pure_apply():
    """src/apply.rs:139-143: channels are skipped on an ArrayReg."""
    c = Y.Circuit.qubits(2, [Y.put([0], Gate.H), Y.channel([1], NoiseChannel.BitFlip(0.3)), Y.label(0, "x")])
    z = np.array([1, 0, 0, 0], complex)
    assert maxdiff(gpu_apply(c, z), O.apply_circuit(c, z)) == 0.0


# ---------------------------------------------------------- registers
def test_register_constructors_and_reductions():
    n = 10
    r = Y.ArrayReg.deterministic_state(n)
    ref = O.deterministic_state(n)
    assert maxdiff(r.state_vec(), ref) < 1e-15
    assert abs(r.norm() - 1) < 1e-13
    assert abs(Y.ArrayReg.zero_state(3).state_vec()[0] - 1) == 0
    g = Y.ArrayReg.ghz_state(3).state_vec()
    assert abs(g[0] - 1 / math.sqrt(2)) < 1e-15 and abs(g[7] - 1 / math.sqrt(2)) < 1e-15
    u = Y.ArrayReg.uniform_state(2).state_vec()
    assert np.allclose(u, 0.5)
    p = Y.ArrayReg.product_state([1, 0, 1]).state_vec()
    assert p[5] == 1 and np.sum(np.abs(p)) == 1
    rng = np.random.default_rng(1)
    a, b = random_state(rng, n), random_state(rng, n)
    ra, rb = Y.ArrayReg.from_vec(n, a), Y.ArrayReg.from_vec(n, b)
    f = ra.fidelity(rb)
    assert abs(f - O.fidelity(a, b, n)) < 1e-14
    ra2 = Y.ArrayReg.from_vec(n, a * 3.0)
    ra2.normalize()
    assert maxdiff(ra2.state_vec(), a) < 1e-15
    # complex64 round trip
    c64 = ra.to_precision(Y.C64)
    assert maxdiff(c64.state_vec(), a) < 1e-7
    assert abs(ra.fidelity(c64) - 1) < 1e-7


# ------------------------------------------------------------ expectation
OPS = [Y.Op.I, Y.Op.X, Y.Op.Y, Y.Op.Z, Y.Op.P0, Y.Op.P1, Y.Op.Pu, Y.Op.Pd]


def random_polynomial(rng, n, nterms):
    coeffs, strs = [], []
    for _ in range(nterms):
        k = int(rng.integers(0, min(4, n) + 1))
        sites = [int(s) for s in rng.integers(0, n, size=k)]  # duplicates allowed
        ops = [OPS[int(rng.integers(len(OPS)))] for _ in sites]
        strs.append(Y.OperatorString(list(zip(sites, ops))))
        coeffs.append(complex(rng.normal(), rng.normal()))
    return Y.OperatorPolynomial(coeffs, strs)


@pytest.mark.parametrize("n", [1, 3, 7, 12])
def test_expect_arrayreg(n):
    rng = np.random.default_rng(40 + n)
    psi = random_state(rng, n)
    r = Y.ArrayReg.from_vec(n, psi)
    for _ in range(5):
        op = random_polynomial(rng, n, 12)
        got, ref = Y.expect_arrayreg(r, op), O.expect_arrayreg(psi, n, op)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (got, ref)
    op = tfim(n)
    assert abs(Y.expect_arrayreg(r, op) - O.expect_arrayreg(psi, n, op)) < 1e-12


# ----------------------------------------------------------------------- AD
def test_expect_grad_matches_oracle_and_fd():
    rng = np.random.default_rng(9)
    n = 6
    els = []
    for _ in range(3):
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rx(float(rng.uniform(-3, 3)))))
        els.append(Y.control([0], [3], Gate.Ry(float(rng.uniform(-3, 3)))))
        els.append(Y.PositionedGate(Gate.Phase(float(rng.uniform(-3, 3))), [2], [4, 5], [True, False]))
        els.append(Y.put([1, 4], Gate.FSim(float(rng.uniform(-3, 3)), float(rng.uniform(-3, 3)))))
        els.append(Y.put([2], Gate.SqrtW))
        els.append(Y.control([1], [2], Gate.X))
        els.append(Y.put([0, 5], Gate.ISWAP))
    c = Y.Circuit.qubits(n, els)
    op = tfim(n, 0.8) + Y.OperatorPolynomial.single(2, Y.Op.Y, 0.3)
    psi0 = random_state(rng, n)
    r0 = Y.ArrayReg.from_vec(n, psi0)
    v, g = Y.expect_grad(op, c, r0)
    vo, go = O.expect_grad(op, c, psi0)
    assert abs(v - vo) < 1e-12
    assert np.max(np.abs(np.array(g) - np.array(go))) < 1e-11
    p0 = c.parameters()
    h = 1e-5
    for i in range(0, len(p0), 3):
        pp, pm = list(p0), list(p0)
        pp[i] += h
        pm[i] -= h
        c.dispatch(pp)
        fp = Y.expect_arrayreg(Y.apply(c, r0), op).real
        c.dispatch(pm)
        fm = Y.expect_arrayreg(Y.apply(c, r0), op).real
        assert abs((fp - fm) / (2 * h) - g[i]) < 1e-6
    c.dispatch(p0)


def test_expect_grad_batch_matches_single_sets():
    """Many parameter sets of one circuit in one sweep: every set's energy
    and gradient equal expect_grad on that set (and the oracle)."""
    rng = np.random.default_rng(31)
    n = 6
    els = []
    for _ in range(2):
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(0.1)))
            els.append(Y.put([q], Gate.Rz(0.2)))
            els.append(Y.put([q], Gate.Rx(0.0)))
        els.append(Y.control([0], [3], Gate.Ry(0.3)))
        els.append(Y.PositionedGate(Gate.Phase(0.4), [2], [4, 5], [True, False]))
        els.append(Y.put([4, 1], Gate.FSim(0.5, 0.6)))
        els.append(Y.put([2], Gate.SqrtW))
        els.append(Y.control([1], [2], Gate.X))
        els.append(Y.put([0, 5], Gate.ISWAP))
        els.append(Y.put([3, 1], Gate.SWAP))
    c = Y.Circuit.qubits(n, els)
    op = tfim(n, 0.8) + Y.OperatorPolynomial.single(2, Y.Op.Y, 0.3) + \
        Y.OperatorPolynomial([0.25 - 0.1j], [Y.OperatorString([(0, Y.Op.X), (3, Y.Op.Y)])])
    psi0 = random_state(rng, n)
    r0 = Y.ArrayReg.from_vec(n, psi0)
    p_own = c.parameters()
    sets = rng.uniform(-math.pi, math.pi, size=(5, c.num_params()))
    vals, grads = Y.expect_grad_batch(op, c, sets, r0)
    assert c.parameters() == p_own
    assert grads.shape == (5, c.num_params())
    for s in range(5):
        c.dispatch(list(sets[s]))
        v, g = Y.expect_grad(op, c, r0)
        assert abs(vals[s] - v) < 1e-12
        assert np.max(np.abs(grads[s] - np.array(g))) < 1e-11
        if s < 2:
            vo, go = O.expect_grad(op, c, psi0)
            assert abs(vals[s] - vo) < 1e-12
            assert np.max(np.abs(grads[s] - np.array(go))) < 1e-11
    c.dispatch(p_own)
    # the register is untouched and an empty batch is a no-op
    assert maxdiff(r0.state_vec(), psi0) == 0.0
    v0, g0 = Y.expect_grad_batch(op, c, np.zeros((0, c.num_params())), r0)
    assert v0.shape == (0,) and g0.shape == (0, c.num_params())


def test_expect_grad_batch_vqe_many_sets():
    """64 sets of the VQE ansatz at n=10 against per-set oracle runs."""
    n, layers, nsets = 10, 2, 64
    rng = np.random.default_rng(5)
    sets = rng.uniform(-math.pi, math.pi, size=(nsets, 2 * n * layers))
    c = vqe_ansatz(n, layers, sets[0])
    op = tfim(n)
    vals, grads = Y.expect_grad_batch(op, c, sets, Y.ArrayReg.zero_state(n))
    z = np.zeros(1 << n, complex)
    z[0] = 1
    for s in (0, 17, 63):
        c.dispatch(list(sets[s]))
        vo, go = O.expect_grad(op, c, z)
        assert abs(vals[s] - vo) < 1e-12
        assert np.max(np.abs(grads[s] - go)) < 1e-11


def test_expect_grad_rejects_channels():
    c = Y.Circuit.qubits(1, [Y.put([0], Gate.Rx(0.3)), Y.channel([0], NoiseChannel.BitFlip(0.1))])
    with pytest.raises(Y.YaoError, match="noise channel"):
        Y.expect_grad(Y.OperatorPolynomial.single(0, Y.Op.Z, 1.0), c, Y.ArrayReg.zero_state(1))


def test_vqe_gradient_small():
    """The VQE ansatz (Ry.Rz layers + CNOT ring) with the TFIM Hamiltonian at
    n=10, against the oracle."""
    n, layers = 10, 3
    rng = np.random.default_rng(77)
    params = rng.uniform(-math.pi, math.pi, size=2 * n * layers)
    c = vqe_ansatz(n, layers, params)
    op = tfim(n)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    v, g = Y.expect_grad(op, c, Y.ArrayReg.zero_state(n))
    vo, go = O.expect_grad(op, c, z)
    assert abs(v - vo) < 1e-12
    assert np.max(np.abs(np.array(g) - go)) < 1e-11


# -------------------------------------------------------------- measurement
def test_probs_and_marginals():
    rng = np.random.default_rng(5)
    n = 9
    psi = random_state(rng, n)
    r = Y.ArrayReg.from_vec(n, psi)
    assert maxdiff(Y.probs(r), O.probs(psi, n)) == 0.0
    for locs in ([0], [8], [3, 1], [0, 4, 8], [7, 2, 5, 1], list(range(n)), []):
        assert maxdiff(Y.probs(r, locs), O.probs(psi, n, locs)) < 1e-15, locs
    with pytest.raises(Y.YaoError, match="out of range"):
        Y.probs(r, [9])
    with pytest.raises(Y.YaoError, match="duplicate"):
        Y.probs(r, [1, 1])


class FixedRng:
    def __init__(self, r):
        self.r = r

    def random(self):
        return self.r


@pytest.mark.parametrize("post", ["none", "reset", "remove"])
def test_measure_with_postprocess(post):
    rng = np.random.default_rng(11)
    n = 7
    for trial in range(6):
        psi = random_state(rng, n)
        locs = [int(x) for x in rng.permutation(n)[: int(rng.integers(1, 4))]]
        rr = float(rng.uniform(0.01, 0.99))
        reset_val = int(rng.integers(0, 1 << len(locs)))
        code = {"none": 0, "reset": 1, "remove": 2}[post]
        pp = {"none": Y.PostProcess.NoPostProcess, "reset": Y.PostProcess.ResetTo(reset_val),
              "remove": Y.PostProcess.RemoveMeasured}[post]
        r = Y.ArrayReg.from_vec(n, psi)
        res = Y.measure_with_postprocess(r, locs, pp, FixedRng(rr))
        oo, orem, ost = O.measure_with_postprocess(psi, n, locs, code, reset_val, rr)
        assert res.outcome == oo
        assert maxdiff(r.state_vec(), ost) < 1e-14
        if post == "remove":
            assert maxdiff(res.removed.state_vec(), orem) < 1e-14
            assert abs(res.removed.norm() - 1) < 1e-13


# ----------------------------------------------------------- density matrix
CHANNELS = [
    lambda: NoiseChannel.BitFlip(0.13), lambda: NoiseChannel.PhaseFlip(0.21),
    lambda: NoiseChannel.Depolarizing(1, 0.17), lambda: NoiseChannel.PauliChannel(0.1, 0.05, 0.2),
    lambda: NoiseChannel.Reset(0.1, 0.2), lambda: NoiseChannel.AmplitudeDamping(0.3, 0.1),
    lambda: NoiseChannel.PhaseDamping(0.25), lambda: NoiseChannel.PhaseAmplitudeDamping(0.2, 0.1, 0.3),
    lambda: NoiseChannel.ThermalRelaxation(1.0, 1.5, 0.2, 0.05),
]


def random_noisy_circuit(rng, n, depth):
    base = random_circuit(rng, n, depth, max_ctrl=min(2, n - 1) if n > 1 else 0)
    els = []
    for el in base.elements:
        els.append(el)
        if rng.random() < 0.5:
            q = int(rng.integers(n))
            if n >= 2 and rng.random() < 0.3:
                a, b = [int(x) for x in rng.permutation(n)[:2]]
                els.append(Y.channel([a, b], NoiseChannel.Depolarizing(2, 0.07)))
            else:
                els.append(Y.channel([q], CHANNELS[int(rng.integers(len(CHANNELS)))]()))
    return Y.Circuit.qubits(n, els)


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_density_matrix_bit_exact(n):
    rng = np.random.default_rng(300 + n)
    c = random_noisy_circuit(rng, n, 25)
    psi = random_state(rng, n)
    rho0 = O.dm_from_reg(psi, n)
    ref = O.dm_apply_circuit(c, rho0)
    d = Y.DensityMatrix.from_reg(Y.ArrayReg.from_vec(n, psi))
    assert maxdiff(d.state_data(), rho0) == 0.0
    d.apply(c)
    out = d.state_data()
    assert maxdiff(out, ref) == 0.0
    t = d.trace()
    assert abs(t - O.dm_trace(ref, n)) < 1e-13
    assert abs(d.purity() - O.dm_purity(ref, n)) < 1e-12
    for traced in ([0], [n - 1], list(range(0, n, 2))):
        if len(set(traced)) >= n:
            continue
        assert maxdiff(d.partial_tr(traced).state_data(), O.dm_partial_tr(ref, n, traced)) == 0.0
    op = random_polynomial(rng, n, 6)
    assert abs(Y.expect_dm(d, op) - O.expect_dm(ref, n, op)) < 1e-12
    assert maxdiff(Y.probs(d), O.dm_probs(ref, n)) == 0.0
    assert maxdiff(Y.probs(d, [n - 1, 0] if n > 1 else [0]), O.dm_probs(ref, n, [n - 1, 0] if n > 1 else [0])) == 0.0


@pytest.mark.parametrize("paths", [{}, {"YAO_DM_XOR2H": "0"}, {"YAO_DM_MONO": "0"},
                                   {"YAO_DM_MONO": "0", "YAO_DM_XOR": "0"}])
def test_density_matrix_channel_kernels_agree(monkeypatch, paths):
    """Every channel kernel is bit-exact against the oracle: the register
    forms (1-qubit row-monomial channels, Pauli-type XOR channels, 2-qubit
    ones with one or two threads per group) and, with them switched off, the
    shared-memory Kraus-sum kernel."""
    for k, v in paths.items():
        monkeypatch.setenv(k, v)
    n = 6
    rng = np.random.default_rng(377)
    c = random_noisy_circuit(rng, n, 30)
    psi = random_state(rng, n)
    ref = O.dm_apply_circuit(c, O.dm_from_reg(psi, n))
    d = Y.DensityMatrix.from_reg(Y.ArrayReg.from_vec(n, psi))
    d.apply(c)
    assert maxdiff(d.state_data(), ref) == 0.0


@pytest.mark.parametrize("n", [1, 2, 5, 8])
def test_density_matrix_superop_form(n):
    """FUSED density-matrix form (rho as a 2n-qubit vector through the fused
    tile passes, channels as superoperators) against the oracle's Kraus sums:
    1e-12, trace preserved."""
    rng = np.random.default_rng(700 + n)
    c = random_noisy_circuit(rng, n, 25)
    psi = random_state(rng, n)
    ref = O.dm_apply_circuit(c, O.dm_from_reg(psi, n))
    d = Y.DensityMatrix.from_reg(Y.ArrayReg.from_vec(n, psi))
    d.apply(c, Y.MODE_FUSED)
    assert maxdiff(d.state_data(), ref) < 1e-12
    assert abs(d.trace() - O.dm_trace(ref, n)) < 1e-12
    with pytest.raises(Y.YaoError):
        d.apply(c, Y.MODE_TILED)


def test_density_matrix_golden(golden):
    from test_oracle_golden import dm_cases
    for key, c, psi, n, exp in dm_cases(golden):
        d = Y.DensityMatrix.from_reg(Y.ArrayReg.from_vec(n, psi))
        d.apply(c)
        assert maxdiff(d.matrix(), exp) < 1e-10, key


def test_density_matrix_purity_large():
    """Purity through the tiled transpose kernel (dim >= 64) against numpy."""
    n = 8
    rng = np.random.default_rng(8)
    c = random_noisy_circuit(rng, n, 20)
    d = Y.DensityMatrix.from_reg(Y.ArrayReg.from_vec(n, random_state(rng, n)))
    d.apply(c)
    m = d.matrix()
    assert abs(d.purity() - np.real(np.trace(m @ m))) < 1e-12
    assert abs(d.purity() - O.dm_purity(d.state_data(), n)) < 1e-12
    mixed = Y.DensityMatrix.mixed([0.5, 0.5], [Y.ArrayReg.zero_state(1), Y.ArrayReg.product_state([1])])
    assert abs(mixed.purity() - 0.5) < 1e-12


@pytest.mark.parametrize("n", [4, 6, 8])
def test_von_neumann_entropy_of_reduced_noisy_state(n):
    """The reduced state of a noisy circuit (partial trace of the last qubit,
    as tests/suites/benchmark_validation.rs:256-276 of yao-rs does) and its
    entropy, against the oracle's restatement of von_neumann_entropy (the
    1e-15 eigenvalue filter included), to 1e-12."""
    rng = np.random.default_rng(900 + n)
    c = random_noisy_circuit(rng, n, 30)
    d = Y.DensityMatrix.from_reg(Y.ArrayReg.zero_state(n))
    d.apply(c)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    ref = O.dm_apply_circuit(c, O.dm_from_reg(z, n))
    red = d.partial_tr([n - 1])
    red_ref = O.dm_partial_tr(ref, n, [n - 1])
    assert maxdiff(red.state_data(), red_ref) == 0.0
    s, s_ref = red.von_neumann_entropy(), O.dm_von_neumann_entropy(red_ref, n - 1)
    assert s > 0.0
    assert abs(s - s_ref) < 1e-12, (s, s_ref)
    # the full noisy state has entropy too; a pure state has none
    assert abs(d.von_neumann_entropy() - O.dm_von_neumann_entropy(ref, n)) < 1e-12
    assert abs(Y.DensityMatrix.zero_state(n).von_neumann_entropy()) < 1e-12


def test_density_matrix_from_reg_and_bell_entropy():
    """density_matrix_from_reg (src/density_matrix.rs:265-271) against the
    oracle (bit-exact), and the entanglement entropy of a Bell pair (ln 2)
    and of random states against the oracle."""
    bell = Y.ArrayReg.zero_state(2)
    Y.apply_inplace(Y.Circuit.qubits(2, [Y.put([0], Gate.H), Y.control([0], [1], Gate.X)]), bell)
    for keep in ([0], [1]):
        r = Y.density_matrix_from_reg(bell, keep)
        assert r.nbits() == 1
        assert abs(r.von_neumann_entropy() - math.log(2.0)) < 1e-12
    rng = np.random.default_rng(77)
    for n, keep in ((3, [1]), (5, [0, 3]), (7, [6, 2, 4]), (9, [0, 1, 2, 3])):
        psi = random_state(rng, n)
        r = Y.density_matrix_from_reg(Y.ArrayReg.from_vec(n, psi), keep)
        ref = O.density_matrix_from_reg(psi, n, keep)
        assert maxdiff(r.state_data(), ref) == 0.0, (n, keep)
        s, s_ref = r.von_neumann_entropy(), O.dm_von_neumann_entropy(ref, len(keep))
        assert abs(s - s_ref) < 1e-12, (n, keep, s, s_ref)


def test_batch_bounded_wait_reports_timeout(monkeypatch):
    """The batched launch's dependency wait is bounded: with circuit 0's
    second pass made to wait for a count that never comes (test hook), the
    wait gives up after 0.2 s, the call fails with YAO_ERR_TIMEOUT, and the
    context keeps working."""
    from yao_rs import _abi as A
    rng = np.random.default_rng(5)
    circuits = [layered_circuit(8, 3, seed=11), layered_circuit(8, 2, seed=12)]
    states = [random_state(rng, 8) for _ in circuits]
    monkeypatch.setenv("YAO_TILE_BITS", "6")
    monkeypatch.setenv("YAO_AUTOTUNE", "0")
    monkeypatch.setenv("YAO_TEST_BATCH_STALL", "1")
    regs = [Y.ArrayReg.from_vec(8, s) for s in states]
    with pytest.raises(Y.YaoError) as ei:
        Y.batch_apply(circuits, regs, Y.MODE_TILED)
    assert ei.value.status == A.YAO_ERR_TIMEOUT
    monkeypatch.delenv("YAO_TEST_BATCH_STALL")
    regs = [Y.ArrayReg.from_vec(8, s) for s in states]
    Y.batch_apply(circuits, regs, Y.MODE_TILED)
    for c, s, r in zip(circuits, states, regs):
        assert maxdiff(r.state_vec(), O.apply_circuit(c, s)) == 0.0


def test_tensor_core_bounded_waits_report_timeout(monkeypatch):
    """The tensor-core block's two mbarrier waits (operand copy, MMA
    completion) are bounded: with the test hook set, the block issues
    neither the copy nor the MMAs, so nothing is in flight and both waits
    give up after 0.1 s; the call fails with YAO_ERR_TIMEOUT, the tensor
    memory is freed, and the context keeps working."""
    from yao_rs import _abi as A
    n = 12
    rng = np.random.default_rng(31)
    # one dense 5-qubit block (no controls) in one 2^12 tile
    els = []
    for _ in range(12):
        a, b = (int(x) for x in rng.choice(5, size=2, replace=False))
        els.append(Y.put([a, b], Gate.FSim(float(rng.uniform(0, 3)), float(rng.uniform(0, 3)))))
        els.append(Y.put([a], Gate.Rx(float(rng.uniform(0, 3)))))
    c = Y.Circuit.qubits(n, els)
    psi = random_state(rng, n)
    ref = O.apply_circuit(c, psi)
    monkeypatch.setenv("YAO_TILE_BITS", "12")
    monkeypatch.setenv("YAO_REG_BITS", "3")
    monkeypatch.setenv("YAO_AUTOTUNE", "0")
    plan = Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 12, 3)
    assert plan["tensor_core_ops"] >= 1
    monkeypatch.setenv("YAO_TEST_TC_STALL", "1")
    r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
    with pytest.raises(Y.YaoError) as ei:
        Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
    assert ei.value.status == A.YAO_ERR_TIMEOUT
    monkeypatch.delenv("YAO_TEST_TC_STALL")
    r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
    Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
    out = r.state_vec().astype(np.complex128)
    assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6


@pytest.mark.parametrize("n", [12, 16])
def test_integer_tensor_core_blocks_keep_the_norm(monkeypatch, n):
    """The integer form of the complex64 tensor-core blocks (exact int8
    products summed in int32, every rounding to nearest) on the layered
    circuit, without the FP64 norm restore: normalised 1 - F <= 1e-9 against
    the oracle, and a norm drift that is unbiased rounding noise.  X is rounded to
    h = 2^(e - 20) with 2^(e-1) <= the tile's largest |component|, so one
    block moves the squared norm by 2 Re<x|d>, of standard deviation
    h / sqrt(3) per unit norm: about 4.4e-6 / sqrt(2N) for a spread state of
    N amplitudes (largest component near 4 rms).  The drift must stay within
    6 of those deviations over the run's blocks (a random walk), and below a
    tenth of the TF32 form's drift, whose truncating FP32 accumulation
    shrinks the norm by about 8e-7 per block."""
    c = layered_circuit(n, 12, seed=n)
    psi = random_state(np.random.default_rng(900 + n), n)
    ref = O.apply_circuit(c, psi)
    monkeypatch.setenv("YAO_TILE_BITS", "12")
    monkeypatch.setenv("YAO_REG_BITS", "3")
    monkeypatch.setenv("YAO_AUTOTUNE", "0")
    monkeypatch.setenv("YAO_NORM_RESTORE", "0")
    blocks = Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 12, 3)["tensor_core_ops"]
    assert blocks >= 4
    drift = {}
    for variant in ("8", "0"):
        monkeypatch.setenv("YAO_TC_VARIANT", variant)
        r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
        Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
        out = r.state_vec().astype(np.complex128)
        drift[variant] = np.vdot(out, out).real - 1.0
        if variant == "8":
            # the state's error apart from its norm: normalised infidelity
            assert 1 - abs(np.vdot(ref, out)) ** 2 / np.vdot(out, out).real <= 1e-9
    sd = 4.4e-6 / math.sqrt(2 * (1 << n))
    assert abs(drift["8"]) <= 6 * sd * math.sqrt(blocks), (drift, blocks)
    assert drift["0"] < 0 and abs(drift["8"]) < 0.1 * abs(drift["0"]), drift


@pytest.mark.parametrize("n,k", [(13, 5), (16, 5), (14, 4), (15, 3)])
def test_tensor_core_blocks(monkeypatch, n, k):
    """Dense 3..5-qubit blocks of complex64 FUSED runs on the tensor cores
    (widened to 5 qubits; 3 x TF32 products, FP32 accumulation in tensor
    memory) agree with the oracle to 1 - F <= 1e-6 and with the CUDA-core
    form to 1e-5 of the largest amplitude."""
    rng = np.random.default_rng(500 + n)
    c = layered_circuit(n, 6, seed=n)
    psi = random_state(rng, n)
    ref = O.apply_circuit(c, psi)
    monkeypatch.setenv("YAO_TILE_BITS", "12")
    monkeypatch.setenv("YAO_REG_BITS", "3")
    outs = {}
    from yao_rs import _abi as A
    for tc in ("1", "0"):
        monkeypatch.setenv("YAO_TC", tc)
        r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
        A.profile(True)
        Y.apply_inplace(c, r, Y.MODE_FUSED, k)
        kernels = {p["kernel"] for p in A.profile_report()}
        A.profile(False)
        assert ("tile_pass_tc" in kernels) == (tc == "1"), kernels
        outs[tc] = r.state_vec().astype(np.complex128)
        assert 1 - abs(np.vdot(ref, outs[tc])) ** 2 < 1e-6, tc
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(outs["1"] - outs["0"])) < 1e-5 * scale
    assert np.max(np.abs(outs["1"] - ref)) < 1e-5 * scale


def test_edge_cases_empty_and_tiny():
    """Empty circuits, annotation-only circuits, 1- and 2-qubit registers in
    every form, empty batches and empty operators behave like yao-rs."""
    rng = np.random.default_rng(11)
    for n in (1, 2, 3):
        psi = random_state(rng, n)
        empty = Y.Circuit.qubits(n, [])
        for mode in (Y.MODE_PLAIN, Y.MODE_TILED, Y.MODE_FUSED):
            assert maxdiff(gpu_apply(empty, psi, mode), psi) == 0.0
        c = random_circuit(rng, n, 30, max_ctrl=min(2, n - 1))
        ref = O.apply_circuit(c, psi)
        assert maxdiff(gpu_apply(c, psi, Y.MODE_TILED), ref) == 0.0
        assert maxdiff(gpu_apply(c, psi, Y.MODE_FUSED, 0), ref) < 1e-12
        r = Y.ArrayReg.from_vec(n, psi).to_precision(Y.C64)
        Y.apply_inplace(c, r, Y.MODE_FUSED, 0)
        assert 1 - abs(np.vdot(ref, r.state_vec().astype(np.complex128))) ** 2 < 1e-6
    c = Y.Circuit.qubits(2, [Y.label(0, "a"), Y.label(1, "b")])
    r = Y.ArrayReg.zero_state(2)
    Y.apply_inplace(c, r, Y.MODE_FUSED)
    assert maxdiff(r.state_vec(), [1, 0, 0, 0]) == 0.0
    Y.batch_apply([], [], Y.MODE_TILED)
    assert Y.expect_arrayreg(Y.ArrayReg.zero_state(3), Y.OperatorPolynomial.zero()) == 0
    v, g = Y.expect_grad(Y.OperatorPolynomial.single(0, Y.Op.Z, 1.0), Y.Circuit.qubits(1, [Y.put([0], Gate.H)]),
                         Y.ArrayReg.zero_state(1))
    assert abs(v) < 1e-15 and g == []


def test_batched_fused_c64_norm_restored():
    """Complex64 FUSED batches of circuits with 256 gates or more get their
    FP64 input norm restored, like a single register: every circuit within
    1 - F <= 1e-6 of the oracle, norm 1 to 1e-6, and close to the same
    circuit applied alone."""
    rng = np.random.default_rng(77)
    circuits = [layered_circuit(n, 8, seed=n) for n in (12, 13, 14, 15, 12, 14)]
    assert all(len(c.elements) >= 256 for c in circuits)
    states = [random_state(rng, c.nbits) for c in circuits]
    refs = [O.apply_circuit(c, s) for c, s in zip(circuits, states)]
    regs = [Y.ArrayReg.from_vec(c.nbits, s).to_precision(Y.C64) for c, s in zip(circuits, states)]
    Y.batch_apply(circuits, regs, Y.MODE_FUSED, 5)
    for c, s, r, ref in zip(circuits, states, regs, refs):
        out = r.state_vec().astype(np.complex128)
        assert 1 - abs(np.vdot(ref, out)) ** 2 < 1e-6
        assert abs(np.vdot(out, out).real - 1) < 1e-6
        one = Y.ArrayReg.from_vec(c.nbits, s).to_precision(Y.C64)
        Y.apply_inplace(c, one, Y.MODE_FUSED, 5)
        assert np.max(np.abs(one.state_vec() - out)) < 1e-5 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,tbits,rb", [(12, 3, 11, 3), (13, 4, 12, 3), (14, 5, 12, 3), (13, 5, 11, 3),
                                          (12, 4, 10, 2), (11, 3, 10, 2)])
def test_fp64_tensor_core_blocks(monkeypatch, n, k, tbits, rb):
    """Dense 3..5-qubit blocks of complex128 FUSED runs on the FP64 tensor
    cores (mma.sync m8n8k4 f64) agree with the oracle and with the CUDA-core
    form to 1e-12 of the largest amplitude, also with controlled dense gates
    in the circuit."""
    rng = np.random.default_rng(900 + n)
    els = list(layered_circuit(n, 5, seed=n).elements)
    d = 1 << 3
    u, _ = np.linalg.qr(rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d)))
    els.append(Y.control([0], [2, 5, n - 1], Y.Gate.Custom(u)))
    els.append(Y.put([1, n - 2, 3], Y.Gate.Custom(u.T)))
    c = Y.Circuit.qubits(n, els)
    psi = random_state(rng, n)
    ref = O.apply_circuit(c, psi)
    monkeypatch.setenv("YAO_TILE_BITS", str(tbits))
    monkeypatch.setenv("YAO_REG_BITS", str(rb))
    outs = {}
    for dm in ("1", "0"):
        monkeypatch.setenv("YAO_DMMA", dm)
        outs[dm] = gpu_apply(c, psi, Y.MODE_FUSED, k)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(outs["1"] - ref)) < 1e-12 * scale
    assert np.max(np.abs(outs["1"] - outs["0"])) < 1e-12 * scale


SWEEP_FORMS = {"segments": {}, "one_op": {"YAO_ADJ_SEGMENTS": "0"}, "in_order": {"YAO_ADJ_REORDER": "0"},
               "in_order_one_op": {"YAO_ADJ_REORDER": "0", "YAO_ADJ_SEGMENTS": "0"},
               "segments_per_lane_controls": {"YAO_ADJ_UPAIR": "0"}, "segments_no_x_fold": {"YAO_ADJ_XFOLD": "0"}}


@pytest.mark.parametrize("form", list(SWEEP_FORMS))
@pytest.mark.parametrize("n", [7, 13, 16])
def test_expect_grad_tiled_sweep_matches_per_gate(monkeypatch, n, form):
    """The reverse sweep over shared-memory tiles of psi and lambda gives the
    per-gate sweep's energy and gradient (and the oracle's) to 1e-11, with
    controls inside and outside the tiles, 2-qubit parametric gates, SWAP,
    ISWAP, X, diagonal and controlled dense 1-qubit steps; in every form of
    the tiled sweep: register segments (steps re-sequenced within a pass) or
    one op at a time, steps moved across commuting ones or kept in order.
    Every third qubit carries a run of three parametric steps (three
    generator dots of one folded run)."""
    rng = np.random.default_rng(40 + n)
    els = []
    for _ in range(2):
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
            if q % 3 == 0:
                els.append(Y.put([q], Gate.Rx(float(rng.uniform(-3, 3)))))
        els.append(Y.put([n - 4], Gate.T))
        els.append(Y.control([n - 3], [2], Gate.H))
        els.append(Y.PositionedGate(Gate.Rz(float(rng.uniform(-3, 3))), [n - 1], [1], [False]))
        els.append(Y.put([0], Gate.SqrtX))
        els.append(Y.control([0], [n - 1], Gate.Ry(float(rng.uniform(-3, 3)))))
        els.append(Y.control([n - 1], [1], Gate.Rx(float(rng.uniform(-3, 3)))))
        els.append(Y.PositionedGate(Gate.Phase(float(rng.uniform(-3, 3))), [2], [n - 2, 0], [True, False]))
        els.append(Y.put([1, n - 3], Gate.FSim(float(rng.uniform(-3, 3)), float(rng.uniform(-3, 3)))))
        els.append(Y.put([n // 2, 0], Gate.ISWAP))
        els.append(Y.put([3, n - 1], Gate.SWAP))
        els.append(Y.control([n - 2], [n // 2], Gate.X))
        for q in range(n):
            els.append(Y.control([q], [(q + 1) % n], Gate.X))
    c = Y.Circuit.qubits(n, els)
    op = tfim(n, 0.7) + Y.OperatorPolynomial.single(1, Y.Op.Y, 0.3)
    psi0 = random_state(rng, n)
    r0 = Y.ArrayReg.from_vec(n, psi0)
    for k, v in SWEEP_FORMS[form].items():
        monkeypatch.setenv(k, v)
    v1, g1 = Y.expect_grad(op, c, r0)
    monkeypatch.setenv("YAO_ADJ_TILES", "0")
    v0, g0 = Y.expect_grad(op, c, r0)
    vo, go = O.expect_grad(op, c, psi0)
    assert abs(v1 - v0) < 1e-12 and abs(v1 - vo) < 1e-12
    assert np.max(np.abs(np.array(g1) - np.array(g0))) < 1e-11
    assert np.max(np.abs(np.array(g1) - np.array(go))) < 1e-11
    assert maxdiff(r0.state_vec(), psi0) == 0.0


def test_expect_grad_cnot_folds_into_segment_runs(monkeypatch):
    """CNOTs merge into the folded Ry.Rz run on their target inside a
    register segment, before it (the CNOT follows the run in the circuit) and
    after it (the CNOT precedes the run), controlled by the segment's other
    qubit (one coefficient set per pair) or by another qubit, in the tile or
    out of it (one set per group): the plan has fewer ops and energy and
    gradient still
    match the per-gate sweep, the unmerged sweep and the oracle to 1e-11."""
    rng = np.random.default_rng(123)
    n = 14
    els = []
    for layer in range(3):
        for q in range(0, n - 1, 2):
            els.append(Y.control([q + 1], [q], Gate.X))  # before the run on q
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
        for q in range(layer % 2, n - 1, 2):
            els.append(Y.control([q], [q + 1], Gate.X))  # after the run on q + 1
    for layer in range(4):  # brickwork: rotations, then CNOTs on alternating pairs
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(float(rng.uniform(-3, 3)))))
            els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
        for q in range(layer % 2, n - 1, 2):
            els.append(Y.control([q], [q + 1], Gate.X))
    c = Y.Circuit.qubits(n, els)
    merged = Y.grad_plan_info(c)
    monkeypatch.setenv("YAO_ADJ_XFOLD", "0")
    plain = Y.grad_plan_info(c)
    monkeypatch.delenv("YAO_ADJ_XFOLD")
    assert merged["ops"] <= plain["ops"] - 5 and merged["dots"] == plain["dots"]
    op = tfim(n, 0.9) + Y.OperatorPolynomial.single(3, Y.Op.Y, 0.25)
    psi0 = random_state(rng, n)
    r0 = Y.ArrayReg.from_vec(n, psi0)
    v1, g1 = Y.expect_grad(op, c, r0)
    monkeypatch.setenv("YAO_ADJ_XFOLD", "0")
    v2, g2 = Y.expect_grad(op, c, r0)
    monkeypatch.setenv("YAO_ADJ_TILES", "0")
    v0, g0 = Y.expect_grad(op, c, r0)
    vo, go = O.expect_grad(op, c, psi0)
    for v, g in ((v1, g1), (v2, g2), (v0, g0)):
        assert abs(v - vo) < 1e-12
        assert np.max(np.abs(np.array(g) - np.array(go))) < 1e-11


def test_expect_grad_wide_gate_takes_per_gate_sweep():
    """A circuit with a 3-qubit gate: the tiled reverse sweep declines it and
    the per-gate sweep runs; energy and gradient still match the oracle."""
    rng = np.random.default_rng(71)
    n = 8
    d = 8
    u, _ = np.linalg.qr(rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d)))
    els = []
    for q in range(n):
        els.append(Y.put([q], Gate.Ry(float(rng.uniform(-3, 3)))))
    els.append(Y.put([1, 4, 6], Gate.Custom(u)))
    for q in range(n):
        els.append(Y.put([q], Gate.Rz(float(rng.uniform(-3, 3)))))
        els.append(Y.control([q], [(q + 1) % n], Gate.X))
    c = Y.Circuit.qubits(n, els)
    op = tfim(n, 0.6)
    psi0 = random_state(rng, n)
    v, g = Y.expect_grad(op, c, Y.ArrayReg.from_vec(n, psi0))
    vo, go = O.expect_grad(op, c, psi0)
    assert abs(v - vo) < 1e-12
    assert np.max(np.abs(np.array(g) - np.array(go))) < 1e-11
