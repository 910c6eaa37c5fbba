"""CPU restatement of yao-rs's tensor-network export and a numpy contraction.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker of the library's
tensor-network builders and GPU contraction; the library never imports it.
Gate matrices come from the C oracle (oracle.c, gate.rs restated), Custom
matrices from the circuit, superoperators from the C oracle (noise.rs).
Networks are dicts {"ixs", "iy", "tensors", "size"} with tensors as numpy
arrays, one axis per leg (row-major), like yao-rs's TensorNetwork.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle as O

# op_matrix (src/operator.rs:53-65): I, X, Y, Z, P0, P1, Pu, Pd
_OPS = {
    0: [[1, 0], [0, 1]], 1: [[0, 1], [1, 0]], 2: [[0, -1j], [1j, 0]], 3: [[1, 0], [0, -1]],
    4: [[1, 0], [0, 0]], 5: [[0, 0], [0, 1]], 6: [[0, 1], [0, 0]], 7: [[0, 0], [1, 0]],
}


def op_matrix(op):
    return np.array(_OPS[int(op)], dtype=np.complex128)


def _matrix(gate):
    """Gate::matrix (src/gate.rs:63-68) and is_diagonal (:98-104)."""
    if gate._matrix is not None:
        return gate._matrix, gate._is_diagonal
    m = O.gate_matrix(gate.kind, gate.params)
    return m, bool(O.lib().orc_gate_is_diagonal(C.c_int32(gate.kind)))


def gate_to_tensor(pg, dims):
    """gate_to_tensor (src/tensors.rs:26-80) with build_controlled_matrix
    (:82-138): returns (tensor, diagonal-without-controls)."""
    all_locs = list(pg.control_locs) + list(pg.target_locs)
    all_dims = [dims[l] for l in all_locs]
    m, diag = _matrix(pg.gate)
    has_ctrl = len(pg.control_locs) > 0
    if diag and not has_ctrl:
        tdims = [dims[l] for l in pg.target_locs]
        return np.array([m[i, i] for i in range(int(np.prod(tdims)))]).reshape(tdims), True
    total = int(np.prod(all_dims))
    if not has_ctrl:
        full = m
    else:
        cdims = [dims[l] for l in pg.control_locs]
        cfg = list(pg.control_configs) or [True] * len(cdims)
        trig, stride = 0, 1
        for i in reversed(range(len(cdims))):  # compute_trigger_index (:140-150)
            trig += int(bool(cfg[i])) * stride
            stride *= cdims[i]
        tdim = total // int(np.prod(cdims))
        full = np.zeros((total, total), np.complex128)
        for ci in range(int(np.prod(cdims))):
            for tr in range(tdim):
                row = ci * tdim + tr
                if ci == trig:
                    full[row, ci * tdim:(ci + 1) * tdim] = m[tr, :]
                else:
                    full[row, ci * tdim + tr] = 1.0
    assert full.shape == (total, total)
    return np.asarray(full).reshape(all_dims + all_dims), False


def _gates(circuit):
    import yao_rs as Y
    return [e for e in circuit.elements if isinstance(e, Y.PositionedGate)]


def _add_gates(circuit, net, cur, nxt):
    for pg in _gates(circuit):
        t, diag = gate_to_tensor(pg, circuit.dims)
        if diag:
            net["ixs"].append([cur[l] for l in pg.target_locs])
        else:
            locs = list(pg.control_locs) + list(pg.target_locs)
            fresh = list(range(nxt, nxt + len(locs)))
            for l, f in zip(locs, fresh):
                net["size"][f] = circuit.dims[l]
            nxt += len(locs)
            net["ixs"].append(fresh + [cur[l] for l in locs])
            for l, f in zip(locs, fresh):
                cur[l] = f
        net["tensors"].append(t)
    return nxt


def _e0(d):
    v = np.zeros(d, np.complex128)
    v[0] = 1
    return v


def circuit_to_einsum(circuit, boundary=False, final_state=()):
    """circuit_to_einsum (src/einsum.rs:34-119) and, with boundary=True,
    circuit_to_einsum_with_boundary (:151-252)."""
    n = len(circuit.dims)
    net = {"ixs": [], "iy": [], "tensors": [], "size": {i: circuit.dims[i] for i in range(n)}}
    cur = list(range(n))
    if boundary:
        for i in range(n):
            net["ixs"].append([i])
            net["tensors"].append(_e0(circuit.dims[i]))
    _add_gates(circuit, net, cur, n)
    if boundary:
        for q in final_state:
            net["ixs"].append([cur[q]])
            net["tensors"].append(_e0(circuit.dims[q]))
    pinned = set(final_state) if boundary else set()
    net["iy"] = [cur[i] for i in range(n) if i not in pinned]
    return net


def circuit_to_expectation(circuit, op):
    """circuit_to_expectation (src/einsum.rs:274-500)."""
    n = len(circuit.dims)
    net = {"ixs": [], "iy": [], "tensors": [], "size": {i: circuit.dims[i] for i in range(n)}}
    cur = list(range(n))
    for i in range(n):
        net["ixs"].append([i])
        net["tensors"].append(_e0(circuit.dims[i]))
    nxt = _add_gates(circuit, net, cur, n)
    terms = list(op)
    if not terms:
        net["ixs"].append([])
        net["tensors"].append(np.zeros((), np.complex128))
    else:
        assert len(terms) == 1
        coeff, s = terms[0]
        ops = s.ops()
        site_op = {}
        for site, o in ops:
            site_op[site] = o
        first = ops[0][0] if ops else None
        for i in range(n):
            if i in site_op:
                m = op_matrix(site_op[i])
                if first is None or i == first:
                    m = m * coeff
            else:
                m = op_matrix(0)
            net["size"][nxt] = circuit.dims[i]
            net["ixs"].append([nxt, cur[i]])
            net["tensors"].append(m)
            cur[i] = nxt
            nxt += 1
    for pg in reversed(_gates(circuit)):
        t, diag = gate_to_tensor(pg, circuit.dims)
        t = np.conj(t)
        if diag:
            net["ixs"].append([cur[l] for l in pg.target_locs])
            net["tensors"].append(t)
            continue
        locs = list(pg.control_locs) + list(pg.target_locs)
        k = len(locs)
        t = np.transpose(t, list(range(k, 2 * k)) + list(range(k)))
        fresh = list(range(nxt, nxt + k))
        for l, f in zip(locs, fresh):
            net["size"][f] = circuit.dims[l]
        nxt += k
        net["ixs"].append(fresh + [cur[l] for l in locs])
        net["tensors"].append(np.ascontiguousarray(t))
        for l, f in zip(locs, fresh):
            cur[l] = f
    for i in range(n):
        net["ixs"].append([cur[i]])
        net["tensors"].append(_e0(circuit.dims[i]))
    return net


def circuit_to_einsum_dm(circuit):
    """circuit_to_einsum_dm (src/einsum.rs:519-665)."""
    import yao_rs as Y
    n = len(circuit.dims)
    net = {"ixs": [], "iy": [], "tensors": [], "size": {}}
    slot = [i + 1 for i in range(n)]
    for i in range(n):
        net["size"][slot[i]] = net["size"][-slot[i]] = circuit.dims[i]
    nxt = n + 1
    for i in range(n):
        net["ixs"] += [[slot[i]], [-slot[i]]]
        net["tensors"] += [_e0(circuit.dims[i]), _e0(circuit.dims[i])]
    for el in circuit.elements:
        if isinstance(el, Y.PositionedGate):
            t, diag = gate_to_tensor(el, circuit.dims)
            if diag:
                ket = [slot[l] for l in el.target_locs]
                net["ixs"] += [ket, [-x for x in ket]]
                net["tensors"] += [t, np.conj(t)]
            else:
                locs = list(el.control_locs) + list(el.target_locs)
                fresh = list(range(nxt, nxt + len(locs)))
                nxt += len(locs)
                for l, f in zip(locs, fresh):
                    net["size"][f] = net["size"][-f] = circuit.dims[l]
                net["ixs"] += [fresh + [slot[l] for l in locs], [-f for f in fresh] + [-slot[l] for l in locs]]
                net["tensors"] += [t, np.conj(t)]
                for l, f in zip(locs, fresh):
                    slot[l] = f
        elif isinstance(el, Y.PositionedChannel):
            arr, keep = Y.elements_array([el])
            S = O.noise_superop(arr[0])
            locs = list(el.locs)
            d = circuit.dims[locs[0]]
            fresh = list(range(nxt, nxt + len(locs)))
            nxt += len(locs)
            for l, f in zip(locs, fresh):
                net["size"][f] = net["size"][-f] = circuit.dims[l]
            net["ixs"].append([-f for f in fresh] + fresh + [-slot[l] for l in locs] + [slot[l] for l in locs])
            net["tensors"].append(S.reshape([d] * (4 * len(locs))))
            for l, f in zip(locs, fresh):
                slot[l] = f
    net["iy"] = slot + [-s for s in slot]
    return net


def circuit_to_expectation_dm(circuit, op):
    """circuit_to_expectation_dm (src/einsum.rs:673-761)."""
    net = circuit_to_einsum_dm(circuit)
    n = len(circuit.dims)
    ket, bra = net["iy"][:n], net["iy"][n:]
    net["iy"] = []
    terms = list(op)
    if not terms:
        net["ixs"].append([])
        net["tensors"].append(np.zeros((), np.complex128))
        return net
    assert len(terms) == 1
    coeff, s = terms[0]
    site_op = {site: o for site, o in s.ops()}
    for i in range(n):
        m = op_matrix(site_op.get(i, 0))
        if i == 0:
            m = m * coeff
        net["ixs"].append([bra[i], ket[i]])
        net["tensors"].append(m)
    return net


def contract(net):
    """The network contracted with numpy: tensors folded into the result
    one at a time (tensor order), each pair by np.einsum; a label is summed
    once no later tensor and no output carries it."""
    ixs, ts, iy = net["ixs"], net["tensors"], net["iy"]
    if not ts:
        return np.ones((), np.complex128)
    res, rl = np.asarray(ts[0]), list(ixs[0])
    for t in range(1, len(ts)):
        later = set(iy)
        for u in range(t + 1, len(ts)):
            later.update(ixs[u])
        keep = [l for l in dict.fromkeys(rl + list(ixs[t])) if l in later]
        letters = {l: i for i, l in enumerate(dict.fromkeys(rl + list(ixs[t])))}
        res = np.einsum(res, [letters[l] for l in rl], np.asarray(ts[t]), [letters[l] for l in ixs[t]],
                        [letters[l] for l in keep])
        rl = keep
    # remaining summed labels, then the output order
    letters = {l: i for i, l in enumerate(rl)}
    return np.einsum(res, [letters[l] for l in rl], [letters[l] for l in iy])
