"""Tensor networks of circuits (yao-rs src/einsum.rs) and their contraction
on the GPU (the role of src/contractor.rs / src/torch_contractor.rs).

A TensorNetwork holds the einsum code (ixs: the labels of each tensor's
legs, iy: the output labels), the tensors (numpy complex128 arrays, one axis
per leg, row-major) and the size of every label, as yao-rs's TensorNetwork
(src/einsum.rs:16-21) does.  The builders run in the library (C ABI
yao_tn_from_circuit); contract() sends any network to the GPU
(yao_tn_contract).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A


class TensorNetwork:
    """TensorNetwork { code: EinCode { ixs, iy }, tensors, size_dict }."""

    def __init__(self, ixs, iy, tensors, size_dict):
        self.ixs = [list(map(int, x)) for x in ixs]
        self.iy = list(map(int, iy))
        self.tensors = [np.asarray(t, dtype=np.complex128) for t in tensors]
        self.size_dict = {int(k): int(v) for k, v in size_dict.items()}

    def __repr__(self):
        return f"TensorNetwork({len(self.tensors)} tensors, output {self.iy})"

    # -- C ABI round trip
    @staticmethod
    def _from_handle(h):
        nt, nl, ne, nlab = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
        no = C.c_uint32()
        A.check(A.lib().yao_tn_counts(h, C.byref(nt), C.byref(nl), C.byref(ne), C.byref(no), C.byref(nlab)))
        ranks = (C.c_uint32 * max(1, nt.value))()
        labels = (C.c_int64 * max(1, nl.value))()
        data = np.zeros(2 * max(1, ne.value))
        iy = (C.c_int64 * max(1, no.value))()
        lids = (C.c_int64 * max(1, nlab.value))()
        ldims = (C.c_uint32 * max(1, nlab.value))()
        A.check(A.lib().yao_tn_export(h, ranks, labels, data.ctypes.data_as(A.dptr), iy, lids, ldims))
        size = {lids[i]: ldims[i] for i in range(nlab.value)}
        ixs, tensors, lo, do = [], [], 0, 0
        cdata = data[:2 * ne.value].view(np.complex128)
        for t in range(nt.value):
            legs = [labels[lo + i] for i in range(ranks[t])]
            lo += ranks[t]
            shape = [size[l] for l in legs]
            cnt = int(np.prod(shape)) if shape else 1
            tensors.append(cdata[do:do + cnt].reshape(shape).copy())
            do += cnt
            ixs.append(legs)
        return TensorNetwork(ixs, [iy[i] for i in range(no.value)], tensors, size)

    def _handle(self):
        ranks = (C.c_uint32 * max(1, len(self.ixs)))(*[len(x) for x in self.ixs])
        flat = [l for x in self.ixs for l in x]
        labels = (C.c_int64 * max(1, len(flat)))(*flat)
        data = np.concatenate([np.ascontiguousarray(t, dtype=np.complex128).ravel() for t in self.tensors]) \
            if self.tensors else np.zeros(1, np.complex128)
        data = np.ascontiguousarray(data)
        keys = list(self.size_dict)
        lids = (C.c_int64 * max(1, len(keys)))(*keys)
        ldims = (C.c_uint32 * max(1, len(keys)))(*[self.size_dict[k] for k in keys])
        iy = (C.c_int64 * max(1, len(self.iy)))(*self.iy)
        h = C.c_void_p()
        nel = sum(int(t.size) for t in self.tensors)
        A.check(A.lib().yao_tn_create(len(self.ixs), ranks, labels, data.view(np.float64).ctypes.data_as(A.dptr),
                                      nel, len(keys), lids, ldims, len(self.iy), iy, C.byref(h)))
        return h


def _build(circuit, kind, pinned=(), op=None):
    h = C.c_void_p()
    pins = (C.c_uint32 * max(1, len(pinned)))(*pinned)
    if op is not None:
        arr, keep = op.terms_array()
        nterms = len(op)
    else:
        arr, keep, nterms = None, None, 0
    A.check(A.lib().yao_tn_from_circuit(circuit.handle, kind, pins, len(pinned), arr, nterms, C.byref(h)))
    try:
        return TensorNetwork._from_handle(h)
    finally:
        A.lib().yao_tn_free(h)


def circuit_to_einsum(circuit):
    """circuit_to_einsum (src/einsum.rs:34-119): input legs 0..n-1 stay open."""
    return _build(circuit, A.TN_EINSUM)


def circuit_to_einsum_with_boundary(circuit, final_state=()):
    """circuit_to_einsum_with_boundary (src/einsum.rs:151-252): |0> on every
    input, <0| on the outputs of the sites in final_state."""
    return _build(circuit, A.TN_BOUNDARY, list(final_state))


def circuit_to_overlap(circuit):
    """circuit_to_overlap (src/einsum.rs:127-131): <0|U|0> as a scalar network."""
    return _build(circuit, A.TN_OVERLAP)


def circuit_to_expectation(circuit, operator):
    """circuit_to_expectation (src/einsum.rs:274-500): <0|U^dagger O U|0>
    for a single-term (or empty) OperatorPolynomial."""
    return _build(circuit, A.TN_EXPECTATION, op=operator)


def circuit_to_einsum_dm(circuit):
    """circuit_to_einsum_dm (src/einsum.rs:519-665): ket labels 1..n, bra
    labels negative, channels as superoperators."""
    return _build(circuit, A.TN_DM)


def circuit_to_expectation_dm(circuit, operator):
    """circuit_to_expectation_dm (src/einsum.rs:673-761): tr(O rho)."""
    return _build(circuit, A.TN_EXPECTATION_DM, op=operator)


def contract(tn: TensorNetwork, device: int | None = None) -> np.ndarray:
    """Contract the network on the GPU (pairwise, greedy order, complex128);
    the result has one axis per output label, in the order of tn.iy."""
    return _contract(tn, device, None)


def tree_to_path(tree, ntensors: int) -> list[tuple[int, int]]:
    """The pair list of a contraction tree, in post order: a leaf is a tensor
    index, a node a list or tuple of two or more subtrees (contracted left to
    right, like a NestedEinsum node's args).  Pair s names two of the
    network's tensors 0..ntensors-1 or the results ntensors + r of pairs
    r < s.  Raises ValueError unless every tensor is a leaf exactly once."""
    pairs: list[tuple[int, int]] = []
    seen: set[int] = set()

    def walk(t):
        if isinstance(t, (int, np.integer)) and not isinstance(t, bool):
            t = int(t)
            if not 0 <= t < ntensors or t in seen:
                raise ValueError(f"contraction tree: leaf {t} is not a tensor of the network or appears twice")
            seen.add(t)
            return t
        if not isinstance(t, (list, tuple)) or len(t) < 2:
            raise ValueError("contraction tree: a node has two or more subtrees")
        acc = walk(t[0])
        for sub in t[1:]:
            pairs.append((acc, walk(sub)))
            acc = ntensors + len(pairs) - 1
        return acc

    if ntensors == 0:
        return []
    walk(tree)
    if len(seen) != ntensors:
        raise ValueError(f"contraction tree covers {len(seen)} of the network's {ntensors} tensors")
    return pairs


def contract_with_tree(tn: TensorNetwork, tree, device: int | None = None) -> np.ndarray:
    """contract_with_tree / contract_dm_with_tree (src/contractor.rs:20-32):
    contract on the GPU in the order of `tree` (see tree_to_path), complex128;
    the result as from contract()."""
    return _contract(tn, device, tree_to_path(tree, len(tn.tensors)))


# yao-rs's density-matrix forms take the same networks here
contract_dm = contract
contract_dm_with_tree = contract_with_tree


def _contract(tn, device, path):
    h = tn._handle()
    try:
        n = C.c_size_t()
        A.check(A.lib().yao_tn_output_len(h, C.byref(n)))
        out = np.zeros(2 * max(1, n.value))
        if path is None:
            A.check(A.lib().yao_tn_contract(A.context(device), h, out.ctypes.data_as(A.dptr), n.value))
        else:
            flat = np.ascontiguousarray(np.asarray(path, dtype=np.uint32).reshape(-1))
            A.check(A.lib().yao_tn_contract_path(A.context(device), h, flat.ctypes.data_as(A.u32p), len(path),
                                                 out.ctypes.data_as(A.dptr), n.value))
    finally:
        A.lib().yao_tn_free(h)
    res = out[:2 * n.value].view(np.complex128)
    return res.reshape([tn.size_dict[l] for l in tn.iy]) if tn.iy else res.reshape(())
