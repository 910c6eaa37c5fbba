"""Shared helpers of the test-suite: golden-case parsing and circuit builders."""
from __future__ import annotations

import math

import numpy as np

import yao_rs as Y
from yao_rs import Gate


def state(re, im):
    return np.asarray(re, dtype=np.float64) + 1j * np.asarray(im, dtype=np.float64)


def pairs(v):
    return np.array([complex(a, b) for a, b in v], dtype=np.complex128)


def matrix_pairs(m):
    return np.array([[complex(a, b) for a, b in row] for row in m], dtype=np.complex128)


def matrix_reim(m):
    return np.asarray(m["re"], dtype=np.float64) + 1j * np.asarray(m["im"], dtype=np.float64)


def gate_from_spec(spec) -> Gate:
    """tests/common/mod.rs:166-212 (gate_from_spec) of yao-rs."""
    n = spec["name"]
    p = spec.get("params", [])
    if n == "Custom":
        m = np.asarray(spec["matrix_re"]) + 1j * np.asarray(spec["matrix_im"])
        return Gate.Custom(m, False, spec.get("label", "Custom"))
    if n in ("Phase", "Rx", "Ry", "Rz"):
        return getattr(Gate, n)(p[0])
    if n == "FSim":
        return Gate.FSim(p[0], p[1])
    return getattr(Gate, n)


def circuit_from_case(case) -> Y.Circuit:
    """tests/common/mod.rs:216-241 (circuit_from_case)."""
    els = []
    for spec in case["gates"]:
        g = gate_from_spec(spec)
        if not spec["controls"]:
            els.append(Y.put(spec["targets"], g))
        else:
            cfg = spec["control_configs"] or [True] * len(spec["controls"])
            els.append(Y.PositionedGate(g, spec["targets"], spec["controls"], cfg))
    return Y.Circuit(case["dims"], els)


def named_gate(name, theta=0.0, phi=0.0):
    if name in ("Rx", "Ry", "Rz", "Phase"):
        return getattr(Gate, name)(theta)
    if name == "FSim":
        return Gate.FSim(theta, phi)
    return getattr(Gate, name)


_KINDS = {"X": 0, "Y": 1, "Z": 2, "H": 3, "S": 4, "T": 5, "SWAP": 6, "Phase": 7, "Rx": 8, "Ry": 9, "Rz": 10,
          "SqrtX": 11, "SqrtY": 12, "SqrtW": 13, "ISWAP": 14, "FSim": 15}


def gate_kind(name):
    """enum yao_gate_kind of a gate name."""
    return _KINDS[name]


def noise_from_key(key):
    """Channel of a noise.json 'kraus' entry key."""
    parts = key.split("_")
    vals = []
    for t in parts:
        try:
            vals.append(float(t))
        except ValueError:
            pass
    if key.startswith("phase_amp_damping"):
        return Y.NoiseChannel.PhaseAmplitudeDamping(*vals)
    if key.startswith("depolarizing"):
        return Y.NoiseChannel.Depolarizing(int(vals[0]), vals[1])
    if key.startswith("amplitude_damping"):
        return Y.NoiseChannel.AmplitudeDamping(vals[0], vals[1])
    if key.startswith("thermal_relaxation"):
        return Y.NoiseChannel.ThermalRelaxation(*vals)
    if key.startswith("pauli"):
        return Y.NoiseChannel.PauliChannel(*vals)
    if key.startswith("bit_flip"):
        return Y.NoiseChannel.BitFlip(vals[0])
    if key.startswith("phase_flip"):
        return Y.NoiseChannel.PhaseFlip(vals[0])
    if key.startswith("phase_damping"):
        return Y.NoiseChannel.PhaseDamping(vals[0])
    raise KeyError(key)


# ---------------------------------------------------------- random circuits
ONE_Q = ["X", "Y", "Z", "H", "S", "T", "SqrtX", "SqrtY", "SqrtW", "Rx", "Ry", "Rz", "Phase"]
TWO_Q = ["SWAP", "ISWAP", "FSim"]


def random_gate(rng, name):
    if name in ("Rx", "Ry", "Rz", "Phase"):
        return getattr(Gate, name)(float(rng.uniform(-math.pi, math.pi)))
    if name == "FSim":
        return Gate.FSim(float(rng.uniform(-math.pi, math.pi)), float(rng.uniform(-math.pi, math.pi)))
    return getattr(Gate, name)


def random_unitary(rng, d):
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_circuit(rng, n, depth, max_ctrl=2, custom=True, diag_custom=True):
    """Every gate kind, controls with random configurations, Custom 1..3-qubit
    dense and diagonal gates."""
    els = []
    for _ in range(depth):
        r = rng.random()
        if r < 0.6 or n < 2:
            g = random_gate(rng, ONE_Q[rng.integers(len(ONE_Q))])
            nt = 1
        elif r < 0.8:
            g = random_gate(rng, TWO_Q[rng.integers(len(TWO_Q))])
            nt = 2
        elif custom:
            nt = int(rng.integers(1, min(3, n) + 1))
            d = 1 << nt
            if diag_custom and rng.random() < 0.3:
                g = Gate.Custom(np.diag(np.exp(1j * rng.uniform(-3, 3, d))), True, "D")
            else:
                g = Gate.Custom(random_unitary(rng, d), False, "U")
        else:
            continue
        if nt > n:
            continue
        qs = [int(x) for x in rng.permutation(n)]
        t = qs[:nt]
        nc = int(rng.integers(0, min(max_ctrl, n - nt) + 1))
        c = qs[nt:nt + nc]
        cfg = [bool(rng.random() < 0.7) for _ in c]
        els.append(Y.PositionedGate(g, t, c, cfg))
    return Y.Circuit.qubits(n, els)


def reverse_index_bits(m, k):
    """The k-qubit matrix m with the bit order of its row and column index
    reversed."""
    p = [int(format(i, f"0{k}b")[::-1], 2) for i in range(1 << k)]
    return np.asarray(m)[np.ix_(p, p)]


def as_tensor_export_reads(circuit):
    """The circuit whose state-vector apply equals the contraction of yao-rs's
    tensor-network export of `circuit`.  The state-vector path reads a k-qubit
    matrix with target_locs[0] as the least significant index bit
    (sort_unitary_2q / instruct_nq, src/instruct_qubit.rs:214-231), the
    export reshapes it row-major with target_locs[0] as the most significant
    axis (gate_to_tensor, src/tensors.rs:26-80); the two agree for matrices
    symmetric under that reversal (SWAP, ISWAP, FSim, CZ-like diagonals), so
    only Custom multi-target matrices are rewritten."""
    els = []
    for e in circuit.elements:
        if isinstance(e, Y.PositionedGate) and e.gate._matrix is not None and len(e.target_locs) > 1:
            m = reverse_index_bits(e.gate._matrix, len(e.target_locs))
            g = Gate.Custom(m, e.gate._is_diagonal, "R")
            els.append(Y.PositionedGate(g, list(e.target_locs), list(e.control_locs), list(e.control_configs)))
        else:
            els.append(e)
    return Y.Circuit.qubits(circuit.nbits, els)


def random_state(rng, n):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def qft_circuit(n, swaps=True):
    """QFT: H(i), control(i+j -> i, Phase(2 pi / 2^(j+1))) (easybuild.rs:55-70),
    then SWAP(i, n-1-i) for i < n/2."""
    els = []
    for i in range(n):
        els.append(Y.put([i], Gate.H))
        for j in range(1, n - i):
            els.append(Y.control([i + j], [i], Gate.Phase(2.0 * math.pi / float(1 << (j + 1)))))
    if swaps:
        for i in range(n // 2):
            els.append(Y.put([i, n - 1 - i], Gate.SWAP))
    return Y.Circuit.qubits(n, els)


def layered_circuit(n, layers, seed, layer0=0):
    """Layered random circuit: per layer Rx, Ry, Rz on every qubit (angles
    U[0, 2 pi)), then CNOT on (2i, 2i+1) on even layers, (2i+1, 2i+2) on odd."""
    rng = np.random.default_rng(seed)
    els = []
    for layer in range(layer0, layer0 + layers):
        ang = rng.uniform(0.0, 2.0 * math.pi, size=(n, 3))
        for q in range(n):
            els.append(Y.put([q], Gate.Rx(float(ang[q, 0]))))
            els.append(Y.put([q], Gate.Ry(float(ang[q, 1]))))
            els.append(Y.put([q], Gate.Rz(float(ang[q, 2]))))
        start = 0 if layer % 2 == 0 else 1
        for a in range(start, n - 1, 2):
            els.append(Y.control([a], [a + 1], Gate.X))
    return Y.Circuit.qubits(n, els)


def vqe_ansatz(n, layers, params):
    """Hardware-efficient ansatz: per layer Ry, Rz on every qubit, then a
    CNOT ring i -> i+1 mod n."""
    els = []
    k = 0
    for _ in range(layers):
        for q in range(n):
            els.append(Y.put([q], Gate.Ry(float(params[k]))))
            els.append(Y.put([q], Gate.Rz(float(params[k + 1]))))
            k += 2
        for q in range(n):
            els.append(Y.control([q], [(q + 1) % n], Gate.X))
    return Y.Circuit.qubits(n, els)


def tfim(n, h=1.0):
    """H = -sum Z_i Z_{i+1 mod n} - h sum X_i."""
    coeffs, strs = [], []
    for i in range(n):
        coeffs.append(-1.0)
        strs.append(Y.OperatorString([(i, Y.Op.Z), ((i + 1) % n, Y.Op.Z)]))
    for i in range(n):
        coeffs.append(-h)
        strs.append(Y.OperatorString([(i, Y.Op.X)]))
    return Y.OperatorPolynomial(coeffs, strs)
