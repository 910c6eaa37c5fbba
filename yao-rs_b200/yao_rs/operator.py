"""Operators (yao-rs src/operator.rs): Op, OperatorString, OperatorPolynomial, op_matrix."""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _abi as A


class Op(enum.IntEnum):
    I = A.OP_I  # noqa: E741
    X = A.OP_X
    Y = A.OP_Y
    Z = A.OP_Z
    P0 = A.OP_P0
    P1 = A.OP_P1
    Pu = A.OP_PU
    Pd = A.OP_PD


_MATS = {
    Op.I: [[1, 0], [0, 1]], Op.X: [[0, 1], [1, 0]], Op.Y: [[0, -1j], [1j, 0]], Op.Z: [[1, 0], [0, -1]],
    Op.P0: [[1, 0], [0, 0]], Op.P1: [[0, 0], [0, 1]], Op.Pu: [[0, 1], [0, 0]], Op.Pd: [[0, 0], [1, 0]],
}


def op_matrix(op) -> np.ndarray:
    """op_matrix (src/operator.rs:53-65)."""
    return np.array(_MATS[Op(op)], dtype=np.complex128)


class OperatorString:
    """OperatorString (src/operator.rs:21-51): stable-sorted by site, Op::I dropped."""

    __slots__ = ("_ops",)

    def __init__(self, ops):
        ops = sorted(((int(s), Op(o)) for s, o in ops), key=lambda t: t[0])
        self._ops = [(s, o) for s, o in ops if o != Op.I]

    @staticmethod
    def identity():
        return OperatorString([])

    def ops(self):
        return list(self._ops)

    def __len__(self):
        return len(self._ops)

    def is_empty(self):
        return not self._ops

    def __eq__(self, other):
        return isinstance(other, OperatorString) and self._ops == other._ops

    def __hash__(self):
        return hash(tuple(self._ops))

    def __repr__(self):
        return "".join(f"{o.name}({s})" for s, o in self._ops) or "I"


class OperatorPolynomial:
    """OperatorPolynomial (src/operator.rs:67-153): sum_i c_i O_i."""

    def __init__(self, coeffs, opstrings):
        coeffs = [complex(c) for c in coeffs]
        opstrings = list(opstrings)
        assert len(coeffs) == len(opstrings)
        self._coeffs = coeffs
        self._opstrings = opstrings

    @staticmethod
    def single(site, op, coeff=1.0):
        return OperatorPolynomial([coeff], [OperatorString([(site, op)])])

    @staticmethod
    def identity():
        return OperatorPolynomial([1.0], [OperatorString.identity()])

    @staticmethod
    def zero():
        return OperatorPolynomial([], [])

    def __len__(self):
        return len(self._coeffs)

    def is_empty(self):
        return not self._coeffs

    def coeffs(self):
        return list(self._coeffs)

    def opstrings(self):
        return list(self._opstrings)

    def __iter__(self):
        return iter(zip(self._coeffs, self._opstrings))

    def __add__(self, other):
        return OperatorPolynomial(self._coeffs + other._coeffs, self._opstrings + other._opstrings)

    def __neg__(self):
        return OperatorPolynomial([-c for c in self._coeffs], self._opstrings)

    def __mul__(self, scalar):
        return OperatorPolynomial([c * scalar for c in self._coeffs], self._opstrings)

    __rmul__ = __mul__

    def terms_array(self):
        """The C wire form (yao_term[]) and the buffers it points to."""
        keep = []
        arr = (A.yao_term * max(1, len(self._coeffs)))()
        for i, (c, s) in enumerate(self):
            ops = s.ops()
            sites = (C.c_uint32 * max(1, len(ops)))(*[o[0] for o in ops])
            codes = (C.c_int32 * max(1, len(ops)))(*[int(o[1]) for o in ops])
            keep += [sites, codes]
            arr[i].coeff_re = c.real
            arr[i].coeff_im = c.imag
            arr[i].nops = len(ops)
            arr[i].sites = C.cast(sites, C.POINTER(C.c_uint32))
            arr[i].ops = C.cast(codes, C.POINTER(C.c_int32))
        return arr, keep

    def __repr__(self):
        return " + ".join(f"{c}*{s!r}" for c, s in self) or "0"
