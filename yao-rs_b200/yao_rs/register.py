"""Device-resident registers: ArrayReg (yao-rs src/register.rs) and
DensityMatrix (src/density_matrix.rs).

The amplitudes live in GPU memory for the lifetime of the object; ``state``
/ ``state_vec()`` copy them to a numpy array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A


class Register:
    """Register trait (src/register.rs:7-11)."""

    def nbits(self) -> int:
        raise NotImplementedError

    def apply(self, circuit):
        raise NotImplementedError

    def state_data(self):
        raise NotImplementedError


class ArrayReg(Register):
    """Dense state vector on the GPU (src/register.rs:15-18)."""

    def __init__(self, handle, device=None):
        self._h = handle
        self._device = device
        n = C.c_uint32()
        A.check(A.lib().yao_reg_nbits(handle, C.byref(n)))
        self._nbits = n.value
        p = C.c_int32()
        A.check(A.lib().yao_reg_precision(handle, C.byref(p)))
        self.precision = p.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and A._lib is not None:
            A.lib().yao_reg_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- constructors (src/register.rs:21-96)
    @staticmethod
    def zero_state(nbits, precision=A.C128, device=None):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_zero_state(A.context(device), nbits, precision, C.byref(h)))
        return ArrayReg(h, device)

    @staticmethod
    def from_vec(nbits, state, device=None):
        v = np.ascontiguousarray(state, dtype=np.complex128)
        assert v.size == 1 << nbits
        h = C.c_void_p()
        A.check(A.lib().yao_reg_from_host(A.context(device), nbits, v.ctypes.data_as(A.dptr), C.byref(h)))
        return ArrayReg(h, device)

    @staticmethod
    def rand_state(nbits, rng, device=None):
        """Uniform re/im in [-0.5, 0.5), normalised (src/register.rs:35-45).

        ``rng`` is a numpy Generator; yao-rs draws from the rand crate, so
        the stream itself differs."""
        dim = 1 << nbits
        v = (rng.random(dim) - 0.5) + 1j * (rng.random(dim) - 0.5)
        v /= np.sqrt(np.sum(np.abs(v) ** 2))
        return ArrayReg.from_vec(nbits, v, device)

    @staticmethod
    def uniform_state(nbits, device=None):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_uniform_state(A.context(device), nbits, C.byref(h)))
        return ArrayReg(h, device)

    @staticmethod
    def ghz_state(nbits, device=None):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_ghz_state(A.context(device), nbits, C.byref(h)))
        return ArrayReg(h, device)

    @staticmethod
    def deterministic_state(nbits, device=None):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_deterministic_state(A.context(device), nbits, C.byref(h)))
        return ArrayReg(h, device)

    @staticmethod
    def product_state(bits, device=None):
        """|bits> with bits[0] the most significant qubit (loc 0)."""
        bits = list(bits)
        basis = 0
        for b in bits:
            basis = (basis << 1) | (1 if b else 0)
        h = C.c_void_p()
        A.check(A.lib().yao_reg_product_state(A.context(device), len(bits), basis, C.byref(h)))
        return ArrayReg(h, device)

    # -- accessors
    def nbits(self):
        return self._nbits

    def nqubits(self):
        return self._nbits

    def state_vec(self) -> np.ndarray:
        dt = np.complex128 if self.precision == A.C128 else np.complex64
        out = np.empty(1 << self._nbits, dtype=dt)
        A.check(A.lib().yao_reg_to_host(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    state = property(state_vec)
    state_data = state_vec

    def set_state(self, state):
        dt = np.complex128 if self.precision == A.C128 else np.complex64
        v = np.ascontiguousarray(state, dtype=dt)
        assert v.size == 1 << self._nbits
        A.check(A.lib().yao_reg_upload(self._h, v.ctypes.data_as(C.c_void_p)))

    def clone(self):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_clone(self._h, C.byref(h)))
        return ArrayReg(h, self._device)

    def to_precision(self, precision):
        h = C.c_void_p()
        A.check(A.lib().yao_reg_convert(self._h, precision, C.byref(h)))
        return ArrayReg(h, self._device)

    # src/register.rs:98-124
    def norm(self) -> float:
        v = C.c_double()
        A.check(A.lib().yao_reg_norm(self._h, C.byref(v)))
        return v.value

    def normalize(self):
        A.check(A.lib().yao_reg_normalize(self._h))

    def fidelity(self, other) -> float:
        v = C.c_double()
        A.check(A.lib().yao_reg_fidelity(self._h, other._h, C.byref(v)))
        return v.value

    def max_abs_diff(self, other) -> float:
        v = C.c_double()
        A.check(A.lib().yao_reg_max_abs_diff(self._h, other._h, C.byref(v)))
        return v.value

    def apply(self, circuit):
        """Register::apply (src/register.rs:132-134)."""
        from .ops import apply_inplace
        apply_inplace(circuit, self)
        return self

    def __repr__(self):
        return f"ArrayReg(nbits={self._nbits}, precision={'c128' if self.precision == A.C128 else 'c64'})"


class DensityMatrix(Register):
    """Row-major density matrix on the GPU (src/density_matrix.rs:9-12)."""

    def __init__(self, handle, device=None):
        self._h = handle
        self._device = device
        n = C.c_uint32()
        A.check(A.lib().yao_dm_nbits(handle, C.byref(n)))
        self._nbits = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and A._lib is not None:
            A.lib().yao_dm_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @staticmethod
    def from_reg(reg: ArrayReg):
        h = C.c_void_p()
        A.check(A.lib().yao_dm_from_reg(reg.handle, C.byref(h)))
        return DensityMatrix(h, reg._device)

    @staticmethod
    def zero_state(nbits, device=None):
        h = C.c_void_p()
        A.check(A.lib().yao_dm_zero_state(A.context(device), nbits, C.byref(h)))
        return DensityMatrix(h, device)

    @staticmethod
    def from_matrix(nbits, rho, device=None):
        m = np.ascontiguousarray(rho, dtype=np.complex128)
        assert m.size == 1 << (2 * nbits)
        h = C.c_void_p()
        A.check(A.lib().yao_dm_from_host(A.context(device), nbits, m.ctypes.data_as(A.dptr), C.byref(h)))
        return DensityMatrix(h, device)

    @staticmethod
    def mixed(weights, regs, device=None):
        assert len(regs) > 0 and len(weights) == len(regs)
        w = (C.c_double * len(weights))(*weights)
        hs = (C.c_void_p * len(regs))(*[r.handle for r in regs])
        h = C.c_void_p()
        A.check(A.lib().yao_dm_mixed(A.context(device), w, hs, len(regs), C.byref(h)))
        return DensityMatrix(h, device)

    def nbits(self):
        return self._nbits

    def clone(self):
        h = C.c_void_p()
        A.check(A.lib().yao_dm_clone(self._h, C.byref(h)))
        return DensityMatrix(h, self._device)

    def state_data(self) -> np.ndarray:
        """Row-major flat copy, rho[row * dim + col]."""
        out = np.empty(1 << (2 * self._nbits), dtype=np.complex128)
        A.check(A.lib().yao_dm_to_host(self._h, out.ctypes.data_as(A.dptr)))
        return out

    state = property(state_data)

    def matrix(self) -> np.ndarray:
        d = 1 << self._nbits
        return self.state_data().reshape(d, d)

    # src/density_matrix.rs:63-112
    def trace(self) -> complex:
        out = (C.c_double * 2)()
        A.check(A.lib().yao_dm_trace(self._h, out))
        return complex(out[0], out[1])

    def purity(self) -> float:
        v = C.c_double()
        A.check(A.lib().yao_dm_purity(self._h, C.byref(v)))
        return v.value

    def partial_tr(self, traced_locs):
        """Trace out `traced_locs` (bit positions, least significant first,
        as in src/density_matrix.rs:80-112)."""
        t = (C.c_uint32 * max(1, len(traced_locs)))(*traced_locs)
        h = C.c_void_p()
        A.check(A.lib().yao_dm_partial_tr(self._h, t, len(traced_locs), C.byref(h)))
        return DensityMatrix(h, self._device)

    def von_neumann_entropy(self) -> float:
        """-sum lambda ln lambda over eigenvalues > 1e-15 (src/density_matrix.rs:114-121).

        The eigen-solve of the (small, reduced) matrix runs on the host."""
        ev = np.linalg.eigvalsh(self.matrix())
        ev = np.maximum(ev, 0.0)
        ev = ev[ev > 1e-15]
        return float(-np.sum(ev * np.log(ev)))

    def apply(self, circuit, mode=A.MODE_PLAIN):
        """Register::apply for DensityMatrix (src/density_matrix.rs:249-259).

        mode=MODE_FUSED runs rho as a 2n-qubit vector through the fused
        tile passes, channels as superoperators (not bit-identical to the
        Kraus sums; ~1e-14)."""
        A.check(A.lib().yao_dm_apply_mode(self._h, circuit.handle, mode))
        return self

    def __repr__(self):
        return f"DensityMatrix(nbits={self._nbits})"


def density_matrix_from_reg(reg: ArrayReg, locs):
    """density_matrix_from_reg (src/density_matrix.rs:262-268)."""
    full = DensityMatrix.from_reg(reg)
    traced = [l for l in range(reg.nqubits()) if l not in locs]
    return full.partial_tr(traced)
