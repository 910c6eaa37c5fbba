"""NoiseChannel enum (yao-rs src/noise.rs:16-60).

Kraus operators and superoperators are built by the library's host code
(yao_noise_kraus / yao_noise_superop) with noise.rs's formulas; invalid
parameters raise YaoError with noise.rs's panic message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A


class NoiseChannel:
    __slots__ = ("kind", "params", "n", "mats")

    def __init__(self, kind, params=(), n=1, mats=None):
        self.kind = int(kind)
        self.params = tuple(float(p) for p in params)
        self.n = int(n)
        self.mats = None if mats is None else [np.ascontiguousarray(m, dtype=np.complex128) for m in mats]

    # -- variants
    @staticmethod
    def BitFlip(p):  # noqa: N802
        return NoiseChannel(A.NOISE_BIT_FLIP, (p,))

    @staticmethod
    def PhaseFlip(p):  # noqa: N802
        return NoiseChannel(A.NOISE_PHASE_FLIP, (p,))

    @staticmethod
    def Depolarizing(n, p):  # noqa: N802
        return NoiseChannel(A.NOISE_DEPOLARIZING, (p,), n=n)

    @staticmethod
    def PauliChannel(px, py, pz):  # noqa: N802
        return NoiseChannel(A.NOISE_PAULI_CHANNEL, (px, py, pz))

    @staticmethod
    def Reset(p0, p1):  # noqa: N802
        return NoiseChannel(A.NOISE_RESET, (p0, p1))

    @staticmethod
    def AmplitudeDamping(gamma, excited_population=0.0):  # noqa: N802
        return NoiseChannel(A.NOISE_AMPLITUDE_DAMPING, (gamma, excited_population))

    @staticmethod
    def PhaseDamping(gamma):  # noqa: N802
        return NoiseChannel(A.NOISE_PHASE_DAMPING, (gamma,))

    @staticmethod
    def PhaseAmplitudeDamping(amplitude, phase, excited_population=0.0):  # noqa: N802
        return NoiseChannel(A.NOISE_PHASE_AMPLITUDE_DAMPING, (amplitude, phase, excited_population))

    @staticmethod
    def ThermalRelaxation(t1, t2, time, excited_population=0.0):  # noqa: N802
        return NoiseChannel(A.NOISE_THERMAL_RELAXATION, (t1, t2, time, excited_population))

    @staticmethod
    def Coherent(matrix):  # noqa: N802
        return NoiseChannel(A.NOISE_COHERENT, (), mats=[matrix])

    @staticmethod
    def Custom(kraus_ops):  # noqa: N802
        return NoiseChannel(A.NOISE_CUSTOM, (), mats=list(kraus_ops))

    # -- noise.rs:64-85
    def num_qubits(self) -> int:
        if self.kind == A.NOISE_DEPOLARIZING:
            return self.n
        if self.kind in (A.NOISE_COHERENT, A.NOISE_CUSTOM):
            d = self.mats[0].shape[0]
            assert d & (d - 1) == 0, f"channel dimension {d} is not a power of 2"
            return d.bit_length() - 1
        return 1

    def fill_element(self, e: A.yao_element, keep: list, locs):
        e.kind = A.ELEM_CHANNEL
        e.type = self.kind
        arr = (C.c_uint32 * max(1, len(locs)))(*locs)
        keep.append(arr)
        e.targets = C.cast(arr, C.POINTER(C.c_uint32))
        e.ntargets = len(locs)
        e.depol_n = self.n
        for i, p in enumerate(self.params):
            e.params[i] = p
        if self.mats is not None:
            flat = np.ascontiguousarray(np.concatenate([m.reshape(-1) for m in self.mats]))
            keep.append(flat)
            e.matrix = flat.ctypes.data_as(A.dptr)
            e.matrix_dim = self.mats[0].shape[0]
            e.nkraus = len(self.mats)

    def _element(self):
        keep = []
        e = A.yao_element()
        n = self.num_qubits() if self.kind != A.NOISE_DEPOLARIZING else self.n
        self.fill_element(e, keep, list(range(n)))
        return e, keep

    # noise.rs:183-352
    def kraus_operators(self):
        e, keep = self._element()
        cap = 256
        out = np.zeros(cap * 16 * 16, dtype=np.complex128)
        nk, dim = C.c_uint32(), C.c_uint32()
        A.check(A.lib().yao_noise_kraus(C.byref(e), out.ctypes.data_as(A.dptr), cap, C.byref(nk),
                                        C.byref(dim)))
        d = dim.value
        return [out[i * d * d:(i + 1) * d * d].reshape(d, d).copy() for i in range(nk.value)]

    # noise.rs:359-379
    def superop(self):
        e, keep = self._element()
        out = np.zeros(256 * 256, dtype=np.complex128)
        d2 = C.c_uint32()
        A.check(A.lib().yao_noise_superop(C.byref(e), out.ctypes.data_as(A.dptr), C.byref(d2)))
        d = d2.value
        return out[: d * d].reshape(d, d).copy()

    def __repr__(self):
        return f"NoiseChannel(kind={self.kind}, params={self.params}, n={self.n})"
