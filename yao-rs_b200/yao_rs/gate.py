"""Gate enum (yao-rs src/gate.rs:7-35).

Named gates are plain values (``Gate.X``, ``Gate.Rx(0.5)``); their matrices
come from the library's host code (yao_gate_matrix), which builds them with
gate.rs's formulas.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi as A

_NAMES = {A.GATE_X: "X", A.GATE_Y: "Y", A.GATE_Z: "Z", A.GATE_H: "H", A.GATE_S: "S", A.GATE_T: "T",
          A.GATE_SWAP: "SWAP", A.GATE_PHASE: "Phase", A.GATE_RX: "Rx", A.GATE_RY: "Ry",
          A.GATE_RZ: "Rz", A.GATE_SQRTX: "SqrtX", A.GATE_SQRTY: "SqrtY", A.GATE_SQRTW: "SqrtW",
          A.GATE_ISWAP: "ISWAP", A.GATE_FSIM: "FSim", A.GATE_CUSTOM: "Custom"}
_NPARAMS = {A.GATE_PHASE: 1, A.GATE_RX: 1, A.GATE_RY: 1, A.GATE_RZ: 1, A.GATE_FSIM: 2}
_DIAG = {A.GATE_Z, A.GATE_S, A.GATE_T, A.GATE_PHASE, A.GATE_RZ}


class Gate:
    """One yao-rs Gate variant."""

    __slots__ = ("kind", "params", "_matrix", "_is_diagonal", "label")

    def __init__(self, kind: int, params=(), matrix=None, is_diagonal=False, label=""):
        self.kind = int(kind)
        self.params = tuple(float(p) for p in params)
        self._matrix = None if matrix is None else np.ascontiguousarray(matrix, dtype=np.complex128)
        self._is_diagonal = bool(is_diagonal)
        self.label = label

    # -- constructors of the parametric variants
    @staticmethod
    def Phase(theta):  # noqa: N802 - yao-rs variant name
        return Gate(A.GATE_PHASE, (theta,))

    @staticmethod
    def Rx(theta):  # noqa: N802
        return Gate(A.GATE_RX, (theta,))

    @staticmethod
    def Ry(theta):  # noqa: N802
        return Gate(A.GATE_RY, (theta,))

    @staticmethod
    def Rz(theta):  # noqa: N802
        return Gate(A.GATE_RZ, (theta,))

    @staticmethod
    def FSim(theta, phi):  # noqa: N802
        return Gate(A.GATE_FSIM, (theta, phi))

    @staticmethod
    def Custom(matrix, is_diagonal=False, label="Custom"):  # noqa: N802
        m = np.asarray(matrix, dtype=np.complex128)
        if m.ndim != 2 or m.shape[0] != m.shape[1]:
            raise ValueError("Custom gate matrix must be square")
        return Gate(A.GATE_CUSTOM, (), m, is_diagonal, label)

    # -- gate.rs:63-145
    def matrix(self) -> np.ndarray:
        if self.kind == A.GATE_CUSTOM:
            return self._matrix.copy()
        out = np.zeros(16, dtype=np.complex128)
        dim = C.c_uint32()
        p = (C.c_double * 4)(*(list(self.params) + [0.0] * (4 - len(self.params))))
        A.check(A.lib().yao_gate_matrix(self.kind, p, out.ctypes.data_as(A.dptr), C.byref(dim)))
        d = dim.value
        return out[: d * d].reshape(d, d)

    # -- gate.rs:153-193
    def generator_matrix(self, i: int) -> np.ndarray:
        """G = (dU/dtheta_i) U^-1 of parameter i (constant for every
        parametric gate); raises YaoError for i >= num_params()."""
        if i < 0:
            raise ValueError(f"generator_matrix index {i} is negative")
        out = np.zeros(16, dtype=np.complex128)
        dim = C.c_uint32()
        A.check(A.lib().yao_gate_generator_matrix(self.kind, i, out.ctypes.data_as(A.dptr), C.byref(dim)))
        d = dim.value
        return out[: d * d].reshape(d, d)

    def num_sites(self) -> int:
        if self.kind in (A.GATE_SWAP, A.GATE_ISWAP, A.GATE_FSIM):
            return 2
        if self.kind == A.GATE_CUSTOM:
            d = self._matrix.shape[0]
            n = int(round(math.log2(d)))
            assert 1 << n == d, f"Matrix dimension {d} is not a power of 2"
            return n
        return 1

    def matrix_dim(self) -> int:
        if self.kind == A.GATE_CUSTOM:
            return self._matrix.shape[0]
        return 4 if self.kind in (A.GATE_SWAP, A.GATE_ISWAP, A.GATE_FSIM) else 2

    def is_diagonal(self) -> bool:
        if self.kind == A.GATE_CUSTOM:
            return self._is_diagonal
        return self.kind in _DIAG

    def num_params(self) -> int:
        return _NPARAMS.get(self.kind, 0)

    def get_params(self) -> list:
        return list(self.params[: self.num_params()])

    def set_params(self, vals):
        assert len(vals) == self.num_params(), (
            f"set_params length {len(vals)} does not match num_params {self.num_params()}")
        self.params = tuple(float(v) for v in vals)

    # gate.rs:198-281
    def dagger(self) -> "Gate":
        k = self.kind
        if k in (A.GATE_H, A.GATE_X, A.GATE_Y, A.GATE_Z, A.GATE_SWAP):
            return Gate(k)
        if k == A.GATE_S:
            return Gate.Phase(-math.pi / 2)
        if k == A.GATE_T:
            return Gate.Phase(-math.pi / 4)
        if k in (A.GATE_RX, A.GATE_RY, A.GATE_RZ, A.GATE_PHASE):
            return Gate(k, (-self.params[0],))
        if k == A.GATE_FSIM:
            return Gate.FSim(-self.params[0], -self.params[1])
        m = self.matrix().conj().T.copy()
        diag = self._is_diagonal if k == A.GATE_CUSTOM else False
        label = (self.label if k == A.GATE_CUSTOM else _NAMES[k]) + "†"
        return Gate(A.GATE_CUSTOM, (), m, diag, label)

    def __eq__(self, other):
        if not isinstance(other, Gate) or other.kind != self.kind or other.params != self.params:
            return False
        if self.kind == A.GATE_CUSTOM:
            return (np.array_equal(self._matrix, other._matrix)
                    and self._is_diagonal == other._is_diagonal and self.label == other.label)
        return True

    def __hash__(self):
        return hash((self.kind, self.params))

    def __repr__(self):
        if self.kind == A.GATE_CUSTOM:
            return self.label
        n = _NAMES[self.kind]
        if self.params:
            return f"{n}({', '.join(f'{p:.4f}' for p in self.params)})"
        return n


for _k in (A.GATE_X, A.GATE_Y, A.GATE_Z, A.GATE_H, A.GATE_S, A.GATE_T, A.GATE_SWAP, A.GATE_SQRTX,
           A.GATE_SQRTY, A.GATE_SQRTW, A.GATE_ISWAP):
    setattr(Gate, _NAMES[_k], Gate(_k))
