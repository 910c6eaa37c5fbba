"""yao_expect_arrayreg_noalloc: the expectation value without any allocation.

Some callers cannot allocate device memory when they ask for an expectation
value: their memory pool already holds nearly all of the GPU's memory for
state vectors, or they must not stall the GPU (cudaFree synchronises the
device).  For them the library offers this entry point, whose reduction
scratch is a fixed file-scope device array.  This test calls it through the
C ABI and checks it against yao_expect_arrayreg, twice in a row (the second
call reuses the array the first one left behind), checks that inputs beyond
its stated limits are refused, and checks that a call on a fresh context
changes the device's free memory by nothing.  It lives in its own file so
that it runs after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import yao_rs as Y
from helpers import random_state, tfim
from yao_rs import _abi as A

pytestmark = pytest.mark.gpu

OPS = [Y.Op.I, Y.Op.X, Y.Op.Y, Y.Op.Z, Y.Op.P0, Y.Op.P1, Y.Op.Pu, Y.Op.Pd]


def noalloc(reg, op):
    arr, keep = op.terms_array()
    out = (C.c_double * 2)()
    st = A.lib().yao_expect_arrayreg_noalloc(reg.handle, arr, len(op), out)
    return st, complex(out[0], out[1])


def test_noalloc_expectation_matches_regular_entry_point():
    rng = np.random.default_rng(2718)
    for n in (5, 18):
        reg = Y.ArrayReg.from_vec(n, random_state(rng, n))
        coeffs, strs = [], []
        for _ in range(40):
            k = int(rng.integers(0, 5))
            sites = [int(s) for s in rng.integers(0, n, size=k)]
            strs.append(Y.OperatorString([(s, OPS[int(rng.integers(len(OPS)))]) for s in sites]))
            coeffs.append(complex(rng.normal(), rng.normal()))
        op = tfim(n) + Y.OperatorPolynomial(coeffs, strs)
        if len(op) > 64:
            op = Y.OperatorPolynomial(op.coeffs()[:64], op.opstrings()[:64])
        ref = Y.expect_arrayreg(reg, op)
        for call in range(2):
            st, got = noalloc(reg, op)
            assert st == A.YAO_OK, A.lib().yao_last_error().decode()
            assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (n, call, got, ref)


def test_noalloc_rejects_inputs_beyond_its_limits():
    reg = Y.ArrayReg.zero_state(4)
    too_many = Y.OperatorPolynomial([1.0] * 65, [Y.OperatorString([(0, Y.Op.Z)])] * 65)
    st, _ = noalloc(reg, too_many)
    assert st == A.YAO_ERR_INVALID_ARGUMENT
    assert "64 terms" in A.lib().yao_last_error().decode()
    long_term = Y.OperatorPolynomial([1.0], [Y.OperatorString([(i % 4, Y.Op.Z) for i in range(65)])])
    st, _ = noalloc(reg, long_term)
    assert st == A.YAO_ERR_INVALID_ARGUMENT
    assert "64 ops" in A.lib().yao_last_error().decode()
    # a successful call after a refused one leaves no stale message behind
    st, got = noalloc(reg, Y.OperatorPolynomial.single(0, Y.Op.Z, 1.0))
    assert st == A.YAO_OK and got == 1.0
    assert A.lib().yao_last_error().decode() == ""


def test_noalloc_call_allocates_no_device_memory():
    """On a context whose reduction scratch was never sized, the call leaves
    the device's free memory exactly as it was (a cudaMalloc, even of a few
    bytes, takes at least a page)."""
    torch = pytest.importorskip("torch")
    torch.cuda.mem_get_info(0)  # the primary context exists before measuring
    n = 16
    rng = np.random.default_rng(99)
    psi = random_state(rng, n)
    amps = np.ascontiguousarray(np.stack([psi.real, psi.imag], axis=-1).ravel())
    ctx, reg = C.c_void_p(), C.c_void_p()
    A.check(A.lib().yao_ctx_create(0, C.byref(ctx)))
    try:
        A.check(A.lib().yao_reg_from_host(ctx, n, amps.ctypes.data_as(A.dptr), C.byref(reg)))
        A.check(A.lib().yao_ctx_synchronize(ctx))
        op = tfim(n)
        arr, keep = op.terms_array()
        out = (C.c_double * 2)()
        free0, _ = torch.cuda.mem_get_info(0)
        for _ in range(2):
            A.check(A.lib().yao_expect_arrayreg_noalloc(reg, arr, len(op), out))
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, (free0, free1)
        ref = (C.c_double * 2)()
        A.check(A.lib().yao_expect_arrayreg(reg, arr, len(op), ref))
        assert abs(complex(out[0], out[1]) - complex(ref[0], ref[1])) <= 1e-12 * max(1.0, abs(ref[0]))
    finally:
        if reg.value:
            A.lib().yao_reg_free(reg)
        A.lib().yao_ctx_destroy(ctx)
