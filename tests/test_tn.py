"""Tensor networks of circuits (yao-rs src/einsum.rs, src/tensors.rs) and
their contraction on the GPU (the role of src/contractor.rs and
src/torch_contractor.rs).

CPU: the oracle's restatement (oracle/tn.py) reproduces every golden case of
yao-rs's tests/data/einsum.json (qudits included) through its own numpy
contraction; the library's networks equal the oracle's exactly (labels,
leg order, sizes and tensor data, bit for bit) for every builder.
GPU: the library's contraction agrees with the oracle's to 1e-12, with the
state-vector oracle on qubit circuits, and with the golden outputs; edge
cases (empty circuit, scalar networks, outer products, labels on more than
two tensors) and the rejected inputs.

yao-rs's export and its state-vector apply read a Custom k-qubit matrix with
opposite index bit orders (see helpers.as_tensor_export_reads); the golden
cases hold only 2-qubit gates symmetric under that reversal.  The
state-vector comparisons therefore run the oracle on the circuit with those
matrices' index bits reversed, and one test pins the difference itself.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
import tn as OT
import yao_rs as Y
from helpers import as_tensor_export_reads, circuit_from_case, random_circuit, random_state, state
from yao_rs import Gate, NoiseChannel


def same_network(lib, ref):
    assert lib.ixs == [list(x) for x in ref["ixs"]]
    assert lib.iy == list(ref["iy"])
    assert lib.size_dict == {int(k): int(v) for k, v in ref["size"].items()}
    assert len(lib.tensors) == len(ref["tensors"])
    for a, b in zip(lib.tensors, ref["tensors"]):
        b = np.asarray(b)
        assert a.shape == b.shape
        assert np.array_equal(a, b), np.max(np.abs(a - b))


def noisy_circuit(rng, n, depth):
    base = random_circuit(rng, n, depth, max_ctrl=min(2, n - 1) if n > 1 else 0)
    els = []
    chans = [lambda: NoiseChannel.Depolarizing(1, 0.1), lambda: NoiseChannel.AmplitudeDamping(0.2, 0.1),
             lambda: NoiseChannel.PhaseDamping(0.3), lambda: NoiseChannel.PauliChannel(0.1, 0.05, 0.2)]
    for el in base.elements:
        els.append(el)
        if rng.random() < 0.4:
            if n >= 2 and rng.random() < 0.3:
                a, b = [int(x) for x in rng.permutation(n)[:2]]
                els.append(Y.channel([a, b], NoiseChannel.Depolarizing(2, 0.07)))
            else:
                els.append(Y.channel([int(rng.integers(n))], chans[int(rng.integers(len(chans)))]()))
    return Y.Circuit.qubits(n, els)


def one_term(rng, n):
    ops = [(int(s), Y.Op(int(rng.integers(0, 8)))) for s in rng.permutation(n)[: int(rng.integers(1, n + 1))]]
    return Y.OperatorPolynomial([complex(rng.normal(), rng.normal())], [Y.OperatorString(ops)])


# ------------------------------------------------------------------ CPU
def test_oracle_reproduces_golden_einsum_cases(golden):
    """Every case of yao-rs's einsum.json (boundary network, no pins)."""
    cases = golden("einsum")["cases"]
    assert len(cases) == 72
    for case in cases:
        c = circuit_from_case(case)
        out = OT.contract(OT.circuit_to_einsum(c, boundary=True)).reshape(-1)
        exp = state(case["output_state_re"], case["output_state_im"])
        assert np.max(np.abs(out - exp)) < 1e-10, case["label"]


def test_networks_match_oracle_golden(golden):
    for case in golden("einsum")["cases"]:
        c = circuit_from_case(case)
        same_network(Y.circuit_to_einsum(c), OT.circuit_to_einsum(c))
        same_network(Y.circuit_to_einsum_with_boundary(c), OT.circuit_to_einsum(c, boundary=True))
        n = len(case["dims"])
        same_network(Y.circuit_to_overlap(c), OT.circuit_to_einsum(c, boundary=True, final_state=range(n)))


@pytest.mark.parametrize("n", [1, 2, 4, 6])
def test_networks_match_oracle_random(n):
    rng = np.random.default_rng(60 + n)
    for rep in range(3):
        c = random_circuit(rng, n, 25, max_ctrl=min(2, n - 1) if n > 1 else 0)
        same_network(Y.circuit_to_einsum(c), OT.circuit_to_einsum(c))
        pins = [int(x) for x in rng.permutation(n)[: int(rng.integers(0, n + 1))]]
        same_network(Y.circuit_to_einsum_with_boundary(c, pins), OT.circuit_to_einsum(c, True, pins))
        op = one_term(rng, n)
        same_network(Y.circuit_to_expectation(c, op), OT.circuit_to_expectation(c, op))
        nc = noisy_circuit(rng, n, 15)
        same_network(Y.circuit_to_einsum_dm(nc), OT.circuit_to_einsum_dm(nc))
        same_network(Y.circuit_to_expectation_dm(nc, op), OT.circuit_to_expectation_dm(nc, op))


def test_export_reads_multi_qubit_matrices_msb_first():
    """A Custom 2-qubit matrix: the export's contraction equals the state
    vector of the bit-reversed matrix, not of the matrix itself (yao-rs's
    own behaviour, restated by the oracle and the library alike)."""
    rng = np.random.default_rng(3)
    u = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
    c = Y.Circuit.qubits(2, [Y.put([0], Gate.H), Y.put([0, 1], Gate.Custom(u, False, "U"))])
    z = np.zeros(4, complex)
    z[0] = 1
    out = OT.contract(OT.circuit_to_einsum(c, boundary=True)).reshape(-1)
    assert np.max(np.abs(out - O.apply_circuit(as_tensor_export_reads(c), z))) < 1e-14
    assert np.max(np.abs(out - O.apply_circuit(c, z))) > 1e-3
    same_network(Y.circuit_to_einsum_with_boundary(c), OT.circuit_to_einsum(c, boundary=True))


def test_network_builders_reject_what_yao_rs_rejects():
    c = Y.Circuit.qubits(2, [Y.put([0], Gate.H)])
    two = Y.OperatorPolynomial([1.0, 1.0], [Y.OperatorString([(0, Y.Op.Z)]), Y.OperatorString([(1, Y.Op.Z)])])
    with pytest.raises(Y.YaoError, match="single-term"):
        Y.circuit_to_expectation(c, two)
    with pytest.raises(Y.YaoError, match="single-term"):
        Y.circuit_to_expectation_dm(c, two)
    # the zero operator: a zero scalar tensor, no operator legs
    zero = Y.OperatorPolynomial([], [])
    net = Y.circuit_to_expectation(c, zero)
    same_network(net, OT.circuit_to_expectation(c, zero))
    # a network with a label twice on one tensor is not contracted
    bad = Y.TensorNetwork([[0, 0]], [], [np.eye(2)], {0: 2})
    with pytest.raises(Y.YaoError):
        bad._handle()
    mism = Y.TensorNetwork([[0, 1]], [0], [np.ones(3)], {0: 2, 1: 2})
    with pytest.raises(Y.YaoError, match="data length"):
        mism._handle()


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_contract_golden_einsum_cases(golden):
    for case in golden("einsum")["cases"]:
        c = circuit_from_case(case)
        out = Y.einsum.contract(Y.circuit_to_einsum_with_boundary(c)).reshape(-1)
        exp = state(case["output_state_re"], case["output_state_im"])
        assert np.max(np.abs(out - exp)) < 1e-10, case["label"]
        # circuit_to_einsum's open input legs contracted with |0>
        net = Y.circuit_to_einsum(c)
        d = case["dims"]
        ins = [Y.TensorNetwork([[i]], [i], [np.eye(d[i])[0]], {i: d[i]}) for i in range(len(d))]
        full = Y.TensorNetwork(net.ixs + [x.ixs[0] for x in ins], net.iy, net.tensors + [x.tensors[0] for x in ins],
                               net.size_dict)
        out2 = Y.einsum.contract(full).reshape(-1)
        assert np.max(np.abs(out2 - exp)) < 1e-10, case["label"]


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 3, 5, 8, 10])
def test_contract_matches_oracle_and_state_vector(n):
    rng = np.random.default_rng(70 + n)
    c = random_circuit(rng, n, 40, max_ctrl=min(2, n - 1) if n > 1 else 0)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    psi = O.apply_circuit(as_tensor_export_reads(c), z)
    out = Y.einsum.contract(Y.circuit_to_einsum_with_boundary(c)).reshape(-1)
    assert np.max(np.abs(out - psi)) < 1e-12
    assert np.max(np.abs(out - OT.contract(OT.circuit_to_einsum(c, boundary=True)).reshape(-1))) < 1e-12
    amp = Y.einsum.contract(Y.circuit_to_overlap(c))
    assert amp.shape == () and abs(amp - psi[0]) < 1e-12
    pins = [int(x) for x in rng.permutation(n)[: n // 2]]
    part = Y.einsum.contract(Y.circuit_to_einsum_with_boundary(c, pins))
    ref = OT.contract(OT.circuit_to_einsum(c, True, pins))
    assert np.max(np.abs(part - ref)) < 1e-12
    op = one_term(rng, n)
    e = Y.einsum.contract(Y.circuit_to_expectation(c, op))
    assert abs(e - OT.contract(OT.circuit_to_expectation(c, op))) < 1e-12
    # against the state-vector expectation (the coefficient sits on the
    # first op's matrix, so <O> times the coefficient)
    assert abs(e - O.expect_arrayreg(psi, n, op)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 4])
def test_contract_density_matrix_networks(n):
    rng = np.random.default_rng(80 + n)
    c = noisy_circuit(rng, n, 20)
    rho = Y.einsum.contract(Y.circuit_to_einsum_dm(c)).reshape(1 << n, 1 << n)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    ref = O.dm_apply_circuit(as_tensor_export_reads(c), O.dm_from_reg(z, n)).reshape(1 << n, 1 << n)
    assert np.max(np.abs(rho - ref)) < 1e-12
    assert np.max(np.abs(rho - OT.contract(OT.circuit_to_einsum_dm(c)).reshape(1 << n, 1 << n))) < 1e-12
    op = one_term(rng, n)
    e = Y.einsum.contract(Y.circuit_to_expectation_dm(c, op))
    assert abs(e - OT.contract(OT.circuit_to_expectation_dm(c, op))) < 1e-12


@pytest.mark.gpu
def test_contract_edge_cases():
    # empty circuit: |0...0>
    c = Y.Circuit.qubits(3, [])
    out = Y.einsum.contract(Y.circuit_to_einsum_with_boundary(c)).reshape(-1)
    assert out[0] == 1 and np.all(out[1:] == 0)
    # a label on three tensors (diagonal gates share labels), a disconnected
    # factor (outer product) and a summed label present on one tensor only
    rng = np.random.default_rng(5)
    a, b, d = rng.normal(size=(2, 3)) + 1j, rng.normal(size=(3,)) + 0j, rng.normal(size=(3, 2)) - 1j
    e, f = rng.normal(size=(4,)) + 2j, rng.normal(size=(2, 5)) + 0j
    net = Y.TensorNetwork([[0, 1], [1], [1, 2], [3], [4, 5]], [0, 2, 3],
                          [a, b, d, e, f], {0: 2, 1: 3, 2: 2, 3: 4, 4: 2, 5: 5})
    got = Y.einsum.contract(net)
    want = np.einsum("ij,j,jk,l,mn->ikl", a, b, d, e, f)
    assert np.max(np.abs(got - want)) < 1e-12
    # scalar network with long summed legs (the warp-per-output kernel)
    x, y = rng.normal(size=(64, 8)) + 1j, rng.normal(size=(64, 8)) - 1j
    s = Y.einsum.contract(Y.TensorNetwork([[0, 1], [0, 1]], [], [x, y], {0: 64, 1: 8}))
    assert abs(s - np.sum(x * y)) < 1e-11
    # output leg order is the requested one
    t = rng.normal(size=(2, 3, 4)) + 0j
    out = Y.einsum.contract(Y.TensorNetwork([[7, 8, 9]], [9, 7, 8], [t], {7: 2, 8: 3, 9: 4}))
    assert np.array_equal(out, np.transpose(t, (2, 0, 1)))


# ------------------------------------------ explicit contraction order
def test_tree_to_path_post_order_pairs():
    from yao_rs.einsum import tree_to_path
    assert tree_to_path(((0, 1), (2, 3)), 4) == [(0, 1), (2, 3), (4, 5)]
    # a node of more than two subtrees contracts left to right
    assert tree_to_path([0, 1, 2, 3], 4) == [(0, 1), (4, 2), (5, 3)]
    assert tree_to_path([[3, 1], 0, 2], 4) == [(3, 1), (4, 0), (5, 2)]
    assert tree_to_path(0, 1) == [] and tree_to_path((), 0) == []
    for bad, t in (([0, 0], 2), ([0, 1], 3), ([0, [1]], 2), ((0, 5), 3), ([0, True], 2)):
        with pytest.raises(ValueError):
            tree_to_path(bad, t)


def _range_tree(rng, lo, hi):
    """A binary tree over tensors lo..hi-1 whose every subtree is a contiguous
    range, split at a random point (rng) or in the middle (rng None).  Over a
    circuit's network in gate order such a subtree is an operator on at most
    every wire, so its result keeps few legs."""
    if hi - lo == 1:
        return lo
    m = (lo + hi) // 2 if rng is None else int(rng.integers(lo + 1, hi))
    return (_range_tree(rng, lo, m), _range_tree(rng, m, hi))


def _largest_intermediate(net, tree):
    """Elements of the largest tensor a contraction in the order of `tree`
    makes: a label stays while the output or another remaining tensor has it."""
    from yao_rs.einsum import tree_to_path
    legs = [set(x) for x in net.ixs]
    alive = set(range(len(legs)))
    big = 1
    for a, b in tree_to_path(tree, len(legs)):
        alive -= {a, b}
        rest = set(net.iy).union(*(legs[t] for t in alive)) if alive else set(net.iy)
        legs.append((legs[a] | legs[b]) & rest)
        alive.add(len(legs) - 1)
        big = max(big, math.prod(net.size_dict[l] for l in legs[-1]))
    return big


def _trees(rng, net):
    T = len(net.tensors)
    out = [list(range(T)), list(range(T))[::-1], _range_tree(None, 0, T), _range_tree(rng, 0, T)]
    for t in out:
        assert _largest_intermediate(net, t) <= 1 << 20
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 5, 8])
def test_contract_with_tree_matches_greedy_oracle_and_state_vector(n):
    rng = np.random.default_rng(90 + n)
    c = random_circuit(rng, n, 30, max_ctrl=min(2, n - 1))
    net = Y.circuit_to_einsum_with_boundary(c)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    psi = O.apply_circuit(as_tensor_export_reads(c), z)
    greedy = Y.contract_tn(net).reshape(-1)
    # in gate order (one growing state), backwards (one growing operator),
    # balanced and random trees of contiguous ranges
    for tree in _trees(rng, net):
        out = Y.contract_with_tree(net, tree).reshape(-1)
        assert np.max(np.abs(out - psi)) < 1e-12
        assert np.max(np.abs(out - greedy)) < 1e-12
    op = one_term(rng, n)
    enet = Y.circuit_to_expectation(c, op)
    want = OT.contract(OT.circuit_to_expectation(c, op))
    for tree in _trees(rng, enet):
        e = Y.contract_with_tree(enet, tree)
        assert e.shape == () and abs(e - want) < 1e-12


@pytest.mark.gpu
def test_contract_dm_with_tree_matches_the_density_matrix():
    rng = np.random.default_rng(95)
    n = 3
    c = noisy_circuit(rng, n, 15)
    net = Y.circuit_to_einsum_dm(c)
    z = np.zeros(1 << n, complex)
    z[0] = 1
    ref = O.dm_apply_circuit(as_tensor_export_reads(c), O.dm_from_reg(z, n)).reshape(1 << n, 1 << n)
    for tree in _trees(rng, net):
        rho = Y.contract_dm_with_tree(net, tree).reshape(1 << n, 1 << n)
        assert np.max(np.abs(rho - ref)) < 1e-12
    assert np.max(np.abs(rho - Y.contract_dm(net).reshape(1 << n, 1 << n))) < 1e-12


@pytest.mark.gpu
def test_contract_path_outer_products_and_rejected_paths():
    rng = np.random.default_rng(6)
    a, b, d = rng.normal(size=(2, 3)) + 1j, rng.normal(size=(3,)) + 0j, rng.normal(size=(3, 2)) - 1j
    e, f = rng.normal(size=(4,)) + 2j, rng.normal(size=(2, 5)) + 0j
    net = Y.TensorNetwork([[0, 1], [1], [1, 2], [3], [4, 5]], [0, 2, 3],
                          [a, b, d, e, f], {0: 2, 1: 3, 2: 2, 3: 4, 4: 2, 5: 5})
    want = np.einsum("ij,j,jk,l,mn->ikl", a, b, d, e, f)
    # pairs without a shared label first (outer products), then the rest
    for tree in (((3, 4), ((0, 1), 2)), ((0, 3), (4, (2, 1))), [4, 3, 2, 1, 0]):
        assert np.max(np.abs(Y.contract_with_tree(net, tree) - want)) < 1e-12
    # paths that break the rules fail before reaching the GPU, with a message
    h = net._handle()
    try:
        n = C.c_size_t()
        A = Y._abi
        A.check(A.lib().yao_tn_output_len(h, C.byref(n)))
        out = np.zeros(2 * n.value)
        for path, msg in (([0, 1, 5, 2, 6, 3], "T - 1 pairs"),
                          ([0, 1, 5, 2, 6, 3, 7, 7], "distinct"),
                          ([0, 1, 5, 2, 6, 3, 7, 9], "distinct earlier"),
                          ([0, 1, 1, 2, 6, 3, 7, 4], "already contracted")):
            p = np.asarray(path, dtype=np.uint32)
            st = A.lib().yao_tn_contract_path(A.context(None), h, p.ctypes.data_as(A.u32p), len(path) // 2,
                                              out.ctypes.data_as(A.dptr), n.value)
            assert st == A.YAO_ERR_INVALID_ARGUMENT, path
            assert msg in A.lib().yao_last_error().decode(), (path, A.lib().yao_last_error())
    finally:
        Y._abi.lib().yao_tn_free(h)
    # the library still contracts after the refusals
    assert np.max(np.abs(Y.contract_with_tree(net, [0, 1, 2, 3, 4]) - want)) < 1e-12
