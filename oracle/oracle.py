"""ctypes wrapper of the CPU oracle (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU-baseline
leg of the benchmark use it as the checker.  The library under test never
imports it.  Elements and operator terms use the C wire format of
include/yao_gpu.h, marshalled by the yao_rs binding.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None


def build():
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        L = _lib
        d, u32, u64, i32, sz = C.c_double, C.c_uint32, C.c_uint64, C.c_int32, C.c_size_t
        vp = C.c_void_p
        L.orc_itercontrol.argtypes = [u32, vp, vp, u32, vp]
        L.orc_itercontrol_get.restype = u64
        L.orc_itercontrol_get.argtypes = [vp, u64]
        L.orc_controller.argtypes = [vp, vp, u32, u64]
        L.orc_bmask.restype = u64
        L.orc_bmask.argtypes = [vp, u32]
        L.orc_bmask_range.restype = u64
        L.orc_bmask_range.argtypes = [u64, u64]
        for f in ("orc_swapbits",):
            getattr(L, f).restype = u64
            getattr(L, f).argtypes = [u64, u64, u64]
        for f in ("orc_breflect", "orc_neg", "orc_btruncate"):
            getattr(L, f).restype = u64
            getattr(L, f).argtypes = [u64, u64]
        L.orc_norm.restype = d
        L.orc_fidelity.restype = d
        L.orc_dm_purity.restype = d
        L.orc_sample_from_probs.restype = u64
        L.orc_sample_from_probs.argtypes = [vp, u64, d]
        L.orc_measure_with_postprocess.argtypes = [u32, vp, vp, u32, i32, u64, d, vp, vp]
        L.orc_expect_grad.argtypes = [u32, vp, sz, vp, sz, vp, vp, vp, sz]
        L.orc_apply_inplace.argtypes = [u32, vp, sz, vp]
        L.orc_dm_apply.argtypes = [u32, vp, sz, vp]
        L.orc_expect_arrayreg.argtypes = [u32, vp, vp, sz, vp]
        L.orc_expect_dm.argtypes = [u32, vp, vp, sz, vp]
        L.orc_probs.argtypes = [u32, vp, vp, i32, vp]
        L.orc_dm_probs.argtypes = [u32, vp, vp, i32, vp]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _u64(xs):
    return np.ascontiguousarray(np.array(list(xs), dtype=np.uint64).reshape(-1)) if len(xs) else np.zeros(1, np.uint64)


def _c(state):
    return np.ascontiguousarray(state, dtype=np.complex128).copy()


# ----------------------------------------------------------------- bitbasis
class IterCtl(C.Structure):
    _fields_ = [("n", C.c_uint64), ("base", C.c_uint64), ("nchunks", C.c_int32), ("pad", C.c_int32),
                ("masks", C.c_uint64 * 64), ("factors", C.c_uint64 * 64)]


def itercontrol(nbits, positions, configs):
    ic = IterCtl()
    pos, cfg = _u64(positions), _u64(configs)
    st = lib().orc_itercontrol(nbits, _p(pos), _p(cfg), len(positions), C.byref(ic))
    if st != 0:
        raise ValueError("invalid itercontrol arguments")
    return [lib().orc_itercontrol_get(C.byref(ic), k) for k in range(ic.n)]


def controller(cbits, cvals, basis):
    return bool(lib().orc_controller(_p(_u64(cbits)), _p(_u64(cvals)), len(cbits), basis))


# ----------------------------------------------------------------- instruct
def instruct(name, state, nbits, *args):
    """Call orc_instruct_<name> on a copy of `state`; returns the new state."""
    # arguments: complex arrays -> double*, lists -> uint64_t*, ints -> uint32_t
    st = _c(state)
    f = getattr(lib(), "orc_instruct_" + name)
    keep, cargs = [], []
    for a in args:
        if isinstance(a, np.ndarray):
            k = np.ascontiguousarray(a, dtype=np.complex128)
            keep.append(k)
            cargs.append(_p(k))
        elif isinstance(a, (list, tuple)):
            k = _u64(a)
            keep.append(k)
            cargs.append(_p(k))
        else:
            cargs.append(C.c_uint32(a))
    f(_p(st), C.c_uint32(nbits), *cargs)
    return st


# --------------------------------------------------------------------- gates
def gate_matrix(kind, params=()):
    out = np.zeros(16, np.complex128)
    p = np.zeros(4)
    p[: len(params)] = params
    dim = C.c_uint32()
    if lib().orc_gate_matrix(kind, _p(p), _p(out), C.byref(dim)) != 0:
        raise ValueError("not a named gate")
    d = dim.value
    return out[: d * d].reshape(d, d)


def gate_generator(kind, i):
    """gate.rs:153-193 (generator_matrix) through orc_gate_generator."""
    out = np.zeros(16, np.complex128)
    dim = C.c_uint32()
    if lib().orc_gate_generator(kind, i, _p(out), C.byref(dim)) != 0:
        raise ValueError("not a parametric gate")
    d = dim.value
    return out[: d * d].reshape(d, d)


def noise_kraus(element):
    out = np.zeros(256 * 256, np.complex128)
    nk, dim = C.c_uint32(), C.c_uint32()
    st = lib().orc_noise_kraus(C.byref(element), _p(out), 256, C.byref(nk), C.byref(dim))
    if st != 0:
        raise ValueError("invalid channel")
    d = dim.value
    return [out[i * d * d:(i + 1) * d * d].reshape(d, d).copy() for i in range(nk.value)]


def noise_superop(element):
    out = np.zeros(256 * 256, np.complex128)
    d2 = C.c_uint32()
    if lib().orc_noise_superop(C.byref(element), _p(out), C.byref(d2)) != 0:
        raise ValueError("invalid channel")
    d = d2.value
    return out[: d * d].reshape(d, d).copy()


# ------------------------------------------------------------------- circuits
def apply(elements_arr, nelems, nbits, state):
    st = _c(state)
    if lib().orc_apply_inplace(nbits, C.cast(elements_arr, C.c_void_p), nelems, _p(st)) != 0:
        raise ValueError("oracle apply failed")
    return st


def apply_circuit(circuit, state):
    """Apply a yao_rs.Circuit with the oracle."""
    from yao_rs import elements_array
    arr, keep = elements_array(circuit.elements)
    return apply(arr, len(circuit.elements), circuit.nbits, state)


def deterministic_state(nbits):
    st = np.zeros(1 << nbits, np.complex128)
    lib().orc_deterministic_state(C.c_uint32(nbits), _p(st))
    return st


def norm(state, nbits):
    return lib().orc_norm(C.c_uint32(nbits), _p(np.ascontiguousarray(state, np.complex128)))


def fidelity(a, b, nbits):
    return lib().orc_fidelity(C.c_uint32(nbits), _p(np.ascontiguousarray(a, np.complex128)),
                              _p(np.ascontiguousarray(b, np.complex128)))


# ------------------------------------------------------------- density matrix
def dm_from_reg(psi, nbits):
    rho = np.zeros(1 << (2 * nbits), np.complex128)
    lib().orc_dm_from_reg(C.c_uint32(nbits), _p(np.ascontiguousarray(psi, np.complex128)), _p(rho))
    return rho


def dm_apply_circuit(circuit, rho):
    from yao_rs import elements_array
    arr, keep = elements_array(circuit.elements)
    r = _c(rho)
    if lib().orc_dm_apply(circuit.nbits, C.cast(arr, C.c_void_p), len(circuit.elements), _p(r)) != 0:
        raise ValueError("oracle dm apply failed")
    return r


def dm_trace(rho, nbits):
    out = np.zeros(2)
    lib().orc_dm_trace(C.c_uint32(nbits), _p(np.ascontiguousarray(rho, np.complex128)), _p(out))
    return complex(out[0], out[1])


def dm_purity(rho, nbits):
    return lib().orc_dm_purity(C.c_uint32(nbits), _p(np.ascontiguousarray(rho, np.complex128)))


def dm_partial_tr(rho, nbits, traced):
    tr = np.array(list(traced) or [0], dtype=np.uint32)
    nk = nbits - len(set(traced))
    out = np.zeros(1 << (2 * nk), np.complex128)
    lib().orc_dm_partial_tr(C.c_uint32(nbits), _p(np.ascontiguousarray(rho, np.complex128)), _p(tr),
                            C.c_uint32(len(traced)), _p(out))
    return out


def dm_von_neumann_entropy(rho, nbits):
    """DensityMatrix::von_neumann_entropy (src/density_matrix.rs:114-123) with
    hermitian_eigenvalues (:227-242): eigenvalues of the self-adjoint matrix
    read from its lower triangle, clamped at 0, those above 1e-15 summed as
    -sum lambda ln lambda in ascending order.  yao-rs solves the eigenproblem
    with faer (self_adjoint_eigenvalues, Side::Lower); numpy's eigvalsh with
    UPLO='L' reads the same triangle."""
    d = 1 << nbits
    ev = np.linalg.eigvalsh(np.asarray(rho, np.complex128).reshape(d, d), UPLO="L")
    acc = 0.0
    for v in np.maximum(ev, 0.0):
        if v > 1e-15:
            acc += float(v) * math.log(float(v))
    return -acc


def density_matrix_from_reg(psi, nbits, locs):
    """density_matrix_from_reg (src/density_matrix.rs:265-271): from_reg,
    then partial_tr over every loc not in `locs` (ascending)."""
    traced = [l for l in range(nbits) if l not in locs]
    return dm_partial_tr(dm_from_reg(psi, nbits), nbits, traced)


# ---------------------------------------------------------------- observables
def expect_arrayreg(psi, nbits, op):
    arr, keep = op.terms_array()
    out = np.zeros(2)
    lib().orc_expect_arrayreg(nbits, _p(np.ascontiguousarray(psi, np.complex128)), C.cast(arr, C.c_void_p),
                              len(op), _p(out))
    return complex(out[0], out[1])


def expect_dm(rho, nbits, op):
    arr, keep = op.terms_array()
    out = np.zeros(2)
    lib().orc_expect_dm(nbits, _p(np.ascontiguousarray(rho, np.complex128)), C.cast(arr, C.c_void_p), len(op),
                        _p(out))
    return complex(out[0], out[1])


def expect_grad(op, circuit, psi0):
    from yao_rs import elements_array
    tarr, tkeep = op.terms_array()
    earr, ekeep = elements_array(circuit.elements)
    n = circuit.num_params()
    grad = np.zeros(max(1, n))
    val = C.c_double()
    st = lib().orc_expect_grad(circuit.nbits, C.cast(tarr, C.c_void_p), len(op), C.cast(earr, C.c_void_p),
                               len(circuit.elements), _p(np.ascontiguousarray(psi0, np.complex128)),
                               C.byref(val), _p(grad), n)
    if st == -1:
        raise ValueError("expect_grad: circuit contains a noise channel")
    if st != 0:
        raise ValueError("expect_grad failed")
    return val.value, list(grad[:n])


# ---------------------------------------------------------------- measurement
def probs(psi, nbits, locs=None):
    if locs is None:
        out = np.zeros(1 << nbits)
        lib().orc_probs(nbits, _p(np.ascontiguousarray(psi, np.complex128)), None, -1, _p(out))
        return out
    L = np.array(list(locs) or [0], dtype=np.uint32)
    out = np.zeros(1 << len(locs))
    lib().orc_probs(nbits, _p(np.ascontiguousarray(psi, np.complex128)), _p(L), len(locs), _p(out))
    return out


def dm_probs(rho, nbits, locs=None):
    if locs is None:
        out = np.zeros(1 << nbits)
        lib().orc_dm_probs(nbits, _p(np.ascontiguousarray(rho, np.complex128)), None, -1, _p(out))
        return out
    L = np.array(list(locs) or [0], dtype=np.uint32)
    out = np.zeros(1 << len(locs))
    lib().orc_dm_probs(nbits, _p(np.ascontiguousarray(rho, np.complex128)), _p(L), len(locs), _p(out))
    return out


def sample_from_probs(p, r):
    return int(lib().orc_sample_from_probs(_p(np.ascontiguousarray(p, np.float64)), len(p), r))


def measure_with_postprocess(psi, nbits, locs, post, reset_val, r):
    """Returns (outcome, new_state_or_None, post-measurement state)."""
    st = _c(psi)
    L = np.array(list(locs) or [0], dtype=np.uint32)
    out = np.zeros(max(1, len(locs)), np.uint8)
    removed = np.zeros(1 << (nbits - len(locs)), np.complex128)
    rc = lib().orc_measure_with_postprocess(nbits, _p(st), _p(L), len(locs), post, reset_val, r, _p(out),
                                            _p(removed))
    if rc != 0:
        raise ValueError("invalid measurement")
    return [int(x) for x in out[: len(locs)]], (removed if post == 2 else None), st
