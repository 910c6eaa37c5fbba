"""apply / expect / expect_grad / probs / measurement (yao-rs src/apply.rs,
src/expect.rs, src/ad.rs, src/measure.rs) on the GPU registers."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from .register import ArrayReg, DensityMatrix


def apply_inplace(circuit, reg: ArrayReg, mode: int = A.MODE_PLAIN, k: int = 0):
    """apply_inplace (src/apply.rs:123-147).

    mode: MODE_PLAIN (one kernel per gate, bit-exact), MODE_TILED (gates run
    in shared-memory tiles, bit-exact) or MODE_FUSED (k-qubit fused blocks)."""
    A.check(A.lib().yao_apply_inplace_mode(circuit.handle, reg.handle, mode, k))
    return reg


def apply(circuit, reg: ArrayReg, mode: int = A.MODE_PLAIN, k: int = 0) -> ArrayReg:
    """apply (src/apply.rs:150-154): returns a new register."""
    out = reg.clone()
    apply_inplace(circuit, out, mode, k)
    return out


def autotune(circuit, reg: ArrayReg, mode: int = A.MODE_FUSED, k: int = 0) -> dict:
    """Time the TILED / FUSED execution choices for this circuit on a scratch
    copy of `reg` and keep the fastest for later calls; returns the choice."""
    out = (C.c_int32 * 4)()
    A.check(A.lib().yao_autotune(circuit.handle, reg.handle, mode, k, out))
    return {"k": out[0], "tile_bits": out[1], "reg_bits": out[2], "tensor_cores": out[3]}


def plan_info(circuit, precision=A.C128, mode=A.MODE_FUSED, k=5, tile_bits=12, reg_bits=3) -> dict:
    """The host plan of a TILED / FUSED run (no device needed)."""
    out = (C.c_int64 * 7)()
    A.check(A.lib().yao_plan_info(circuit.handle, precision, mode, k, tile_bits, reg_bits, out))
    keys = ("passes", "single_gate_passes", "ops", "tensor_core_ops", "wide_ops", "register_segments", "blocks")
    return dict(zip(keys, [int(x) for x in out]))


def grad_plan_info(circuit) -> dict:
    """The host plan of expect_grad's tiled reverse sweep (no device needed)."""
    out = (C.c_int64 * 3)()
    A.check(A.lib().yao_grad_plan_info(circuit.handle, out))
    return dict(zip(("passes", "ops", "dots"), [int(x) for x in out]))


def batch_apply(circuits, regs, mode: int = A.MODE_PLAIN, k: int = 0):
    cs = (C.c_void_p * max(1, len(circuits)))(*[c.handle for c in circuits])
    rs = (C.c_void_p * max(1, len(regs)))(*[r.handle for r in regs])
    A.check(A.lib().yao_batch_apply(cs, rs, len(regs), mode, k))


def expect_arrayreg(reg: ArrayReg, op) -> complex:
    """expect_arrayreg (src/expect.rs:7-11)."""
    arr, keep = op.terms_array()
    out = (C.c_double * 2)()
    A.check(A.lib().yao_expect_arrayreg(reg.handle, arr, len(op), out))
    return complex(out[0], out[1])


def expect_dm(dm: DensityMatrix, op) -> complex:
    """expect_dm (src/expect.rs:38-42); site s is bit s of the index."""
    arr, keep = op.terms_array()
    out = (C.c_double * 2)()
    A.check(A.lib().yao_expect_dm(dm.handle, arr, len(op), out))
    return complex(out[0], out[1])


def expect_grad(observable, circuit, psi0: ArrayReg):
    """expect_grad (src/ad.rs:75-156): (Re <psi|H|psi>, gradient in
    Circuit::parameters() order)."""
    arr, keep = observable.terms_array()
    n = circuit.num_params()
    grad = (C.c_double * max(1, n))()
    val = C.c_double()
    A.check(A.lib().yao_expect_grad(arr, len(observable), circuit.handle, psi0.handle, C.byref(val), grad, n))
    return val.value, [grad[i] for i in range(n)]


def expect_grad_batch(observable, circuit, params, psi0: ArrayReg):
    """expect_grad for many parameter vectors (rows of `params`) of one
    circuit in one batched sweep; returns (energies[nsets], grads[nsets, np])."""
    P = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1, circuit.num_params()))
    nsets = P.shape[0]
    arr, keep = observable.terms_array()
    vals = np.zeros(nsets)
    grads = np.zeros((nsets, circuit.num_params()))
    A.check(A.lib().yao_expect_grad_batch(arr, len(observable), circuit.handle, P.ctypes.data_as(A.dptr), nsets,
                                          psi0.handle, vals.ctypes.data_as(A.dptr), grads.ctypes.data_as(A.dptr)))
    return vals, grads


def probs(state, locs=None) -> np.ndarray:
    """probs (src/measure.rs:82-87) for an ArrayReg or a DensityMatrix."""
    n = state.nbits()
    if locs is None:
        out = np.empty(1 << n, dtype=np.float64)
        L = (C.c_uint32 * 1)()
        nl = -1
    else:
        locs = list(locs)
        out = np.empty(1 << len(locs), dtype=np.float64)
        L = (C.c_uint32 * max(1, len(locs)))(*locs)
        nl = len(locs)
    f = A.lib().yao_dm_probs if isinstance(state, DensityMatrix) else A.lib().yao_probs
    A.check(f(state.handle, L, nl, out.ctypes.data_as(A.dptr)))
    return out


class PostProcess:
    """PostProcess (src/measure.rs:18-23)."""

    def __init__(self, kind, value=0):
        self.kind = kind
        self.value = value

    NoPostProcess = None  # set below
    RemoveMeasured = None

    @staticmethod
    def ResetTo(v):  # noqa: N802
        return PostProcess(A.POST_RESET_TO, int(v))

    def __eq__(self, other):
        return isinstance(other, PostProcess) and (self.kind, self.value) == (other.kind, other.value)


PostProcess.NoPostProcess = PostProcess(A.POST_NONE)
PostProcess.RemoveMeasured = PostProcess(A.POST_REMOVE_MEASURED)


@dataclass
class MeasureResult:
    """MeasureResult (src/measure.rs:26-30): `removed` is set for RemoveMeasured."""
    outcome: list
    removed: ArrayReg | None = None


def measure_with_postprocess(reg: ArrayReg, locs, post: PostProcess, rng) -> MeasureResult:
    """measure_with_postprocess (src/measure.rs:243-274).

    The uniform draw r = rng.random() is made here and handed to the library,
    which samples the outcome from the marginal probabilities on the host
    with yao-rs's sequential rule."""
    locs = list(locs)
    L = (C.c_uint32 * max(1, len(locs)))(*locs)
    out = (C.c_uint8 * max(1, len(locs)))()
    r = float(rng.random())
    rem = C.c_void_p()
    A.check(A.lib().yao_measure_with_postprocess(reg.handle, L, len(locs), post.kind, post.value, r, out,
                                                 C.byref(rem)))
    outcome = [out[i] for i in range(len(locs))]
    if post.kind == A.POST_REMOVE_MEASURED:
        return MeasureResult(outcome, ArrayReg(rem, reg._device))
    return MeasureResult(outcome)
