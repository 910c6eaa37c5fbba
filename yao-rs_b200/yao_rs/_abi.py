"""ctypes binding of include/yao_gpu.h (the C ABI of libyao_gpu.so).

The library is loaded from this directory.  If it is missing, the binding
raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libyao_gpu.so"

# ----------------------------------------------------------------- enums
YAO_OK = 0
YAO_ERR_INVALID_ARGUMENT = -1
YAO_ERR_CIRCUIT = -2
YAO_ERR_QUBIT_ONLY = -3
YAO_ERR_NBITS_MISMATCH = -4
YAO_ERR_CHANNEL_IN_AD = -5
YAO_ERR_NOISE_PARAM = -6
YAO_ERR_MEASURE_LOCS = -7
YAO_ERR_OUT_OF_MEMORY = -8
YAO_ERR_CUDA = -9
YAO_ERR_NO_DEVICE = -10
YAO_ERR_UNSUPPORTED = -11
YAO_ERR_TIMEOUT = -12

ELEM_GATE, ELEM_CHANNEL, ELEM_ANNOTATION = 0, 1, 2

(GATE_X, GATE_Y, GATE_Z, GATE_H, GATE_S, GATE_T, GATE_SWAP, GATE_PHASE, GATE_RX, GATE_RY, GATE_RZ,
 GATE_SQRTX, GATE_SQRTY, GATE_SQRTW, GATE_ISWAP, GATE_FSIM, GATE_CUSTOM) = range(17)

(NOISE_BIT_FLIP, NOISE_PHASE_FLIP, NOISE_DEPOLARIZING, NOISE_PAULI_CHANNEL, NOISE_RESET,
 NOISE_AMPLITUDE_DAMPING, NOISE_PHASE_DAMPING, NOISE_PHASE_AMPLITUDE_DAMPING,
 NOISE_THERMAL_RELAXATION, NOISE_COHERENT, NOISE_CUSTOM) = range(11)

OP_I, OP_X, OP_Y, OP_Z, OP_P0, OP_P1, OP_PU, OP_PD = range(8)

POST_NONE, POST_RESET_TO, POST_REMOVE_MEASURED = 0, 1, 2
C128, C64 = 0, 1
MODE_PLAIN, MODE_TILED, MODE_FUSED = 0, 1, 2


class yao_element(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("type", C.c_int32),
        ("ntargets", C.c_uint32),
        ("nctrl", C.c_uint32),
        ("targets", C.POINTER(C.c_uint32)),
        ("ctrl_locs", C.POINTER(C.c_uint32)),
        ("ctrl_configs", C.POINTER(C.c_uint8)),
        ("matrix", C.POINTER(C.c_double)),
        ("matrix_dim", C.c_uint32),
        ("nkraus", C.c_uint32),
        ("is_diagonal", C.c_int32),
        ("depol_n", C.c_int32),
        ("nconfigs", C.c_uint32),
        ("reserved", C.c_uint32),
        ("params", C.c_double * 4),
    ]


class yao_term(C.Structure):
    _fields_ = [
        ("coeff_re", C.c_double),
        ("coeff_im", C.c_double),
        ("nops", C.c_uint32),
        ("reserved", C.c_uint32),
        ("sites", C.POINTER(C.c_uint32)),
        ("ops", C.POINTER(C.c_int32)),
    ]


vp = C.c_void_p
pp = C.POINTER(C.c_void_p)
dptr = C.POINTER(C.c_double)
u32p = C.POINTER(C.c_uint32)
i32 = C.c_int32
u32 = C.c_uint32
u64 = C.c_uint64
sz = C.c_size_t

# name: (restype, argtypes)
SIGNATURES = {
    "yao_last_error": (C.c_char_p, []),
    "yao_abi_version": (C.c_int, []),
    "yao_ctx_create": (C.c_int, [C.c_int, pp]),
    "yao_ctx_destroy": (C.c_int, [vp]),
    "yao_ctx_synchronize": (C.c_int, [vp]),
    "yao_ctx_launch_count": (C.c_int, [vp, C.POINTER(u64)]),
    "yao_ctx_stream": (C.c_int, [vp, pp]),
    "yao_ctx_profile": (C.c_int, [vp, C.c_int]),
    "yao_ctx_profile_report": (C.c_int, [vp, C.c_char_p, sz]),
    "yao_circuit_create": (C.c_int, [u32p, u32, C.POINTER(yao_element), sz, pp, C.POINTER(i32)]),
    "yao_circuit_free": (None, [vp]),
    "yao_circuit_num_params": (C.c_int, [vp, C.POINTER(sz)]),
    "yao_circuit_parameters": (C.c_int, [vp, dptr, sz]),
    "yao_circuit_dispatch": (C.c_int, [vp, dptr, sz]),
    "yao_circuit_dagger": (C.c_int, [vp, pp]),
    "yao_gate_matrix": (C.c_int, [i32, dptr, dptr, u32p]),
    "yao_gate_generator_matrix": (C.c_int, [i32, u32, dptr, u32p]),
    "yao_noise_kraus": (C.c_int, [C.POINTER(yao_element), dptr, u32, u32p, u32p]),
    "yao_noise_superop": (C.c_int, [C.POINTER(yao_element), dptr, u32p]),
    "yao_reg_zero_state": (C.c_int, [vp, u32, i32, pp]),
    "yao_reg_from_host": (C.c_int, [vp, u32, dptr, pp]),
    "yao_reg_uniform_state": (C.c_int, [vp, u32, pp]),
    "yao_reg_ghz_state": (C.c_int, [vp, u32, pp]),
    "yao_reg_deterministic_state": (C.c_int, [vp, u32, pp]),
    "yao_reg_product_state": (C.c_int, [vp, u32, u64, pp]),
    "yao_reg_free": (None, [vp]),
    "yao_reg_clone": (C.c_int, [vp, pp]),
    "yao_reg_convert": (C.c_int, [vp, i32, pp]),
    "yao_reg_nbits": (C.c_int, [vp, u32p]),
    "yao_reg_precision": (C.c_int, [vp, C.POINTER(i32)]),
    "yao_reg_to_host": (C.c_int, [vp, vp]),
    "yao_reg_upload": (C.c_int, [vp, vp]),
    "yao_reg_device_ptr": (C.c_int, [vp, pp]),
    "yao_reg_norm": (C.c_int, [vp, dptr]),
    "yao_reg_normalize": (C.c_int, [vp]),
    "yao_reg_fidelity": (C.c_int, [vp, vp, dptr]),
    "yao_reg_max_abs_diff": (C.c_int, [vp, vp, dptr]),
    "yao_apply_inplace": (C.c_int, [vp, vp]),
    "yao_apply": (C.c_int, [vp, vp, pp]),
    "yao_apply_inplace_mode": (C.c_int, [vp, vp, i32, i32]),
    "yao_autotune": (C.c_int, [vp, vp, i32, i32, C.POINTER(i32)]),
    "yao_plan_info": (C.c_int, [vp, i32, i32, i32, i32, i32, C.POINTER(C.c_int64)]),
    "yao_grad_plan_info": (C.c_int, [vp, C.POINTER(C.c_int64)]),
    "yao_dm_from_reg": (C.c_int, [vp, pp]),
    "yao_dm_zero_state": (C.c_int, [vp, u32, pp]),
    "yao_dm_from_host": (C.c_int, [vp, u32, dptr, pp]),
    "yao_dm_mixed": (C.c_int, [vp, dptr, pp, sz, pp]),
    "yao_dm_free": (None, [vp]),
    "yao_dm_clone": (C.c_int, [vp, pp]),
    "yao_dm_nbits": (C.c_int, [vp, u32p]),
    "yao_dm_to_host": (C.c_int, [vp, dptr]),
    "yao_dm_apply": (C.c_int, [vp, vp]),
    "yao_dm_apply_mode": (C.c_int, [vp, vp, i32]),
    "yao_dm_trace": (C.c_int, [vp, dptr]),
    "yao_dm_purity": (C.c_int, [vp, dptr]),
    "yao_dm_partial_tr": (C.c_int, [vp, u32p, u32, pp]),
    "yao_expect_arrayreg": (C.c_int, [vp, C.POINTER(yao_term), sz, dptr]),
    "yao_expect_arrayreg_noalloc": (C.c_int, [vp, C.POINTER(yao_term), sz, dptr]),
    "yao_expect_dm": (C.c_int, [vp, C.POINTER(yao_term), sz, dptr]),
    "yao_expect_grad": (C.c_int, [C.POINTER(yao_term), sz, vp, vp, dptr, dptr, sz]),
    "yao_probs": (C.c_int, [vp, u32p, i32, dptr]),
    "yao_dm_probs": (C.c_int, [vp, u32p, i32, dptr]),
    "yao_measure_with_postprocess": (C.c_int, [vp, u32p, u32, i32, u64, C.c_double,
                                               C.POINTER(C.c_uint8), pp]),
    "yao_batch_apply": (C.c_int, [pp, pp, sz, i32, i32]),
    "yao_expect_grad_batch": (C.c_int, [C.POINTER(yao_term), sz, vp, dptr, sz, vp, dptr, dptr]),
    "yao_tn_from_circuit": (C.c_int, [vp, i32, u32p, u32, C.POINTER(yao_term), sz, pp]),
    "yao_tn_create": (C.c_int, [sz, u32p, C.POINTER(C.c_int64), dptr, sz, sz, C.POINTER(C.c_int64), u32p, u32,
                                C.POINTER(C.c_int64), pp]),
    "yao_tn_free": (None, [vp]),
    "yao_tn_counts": (C.c_int, [vp, C.POINTER(sz), C.POINTER(sz), C.POINTER(sz), u32p, C.POINTER(sz)]),
    "yao_tn_export": (C.c_int, [vp, u32p, C.POINTER(C.c_int64), dptr, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                u32p]),
    "yao_tn_output_len": (C.c_int, [vp, C.POINTER(sz)]),
    "yao_tn_contract": (C.c_int, [vp, vp, dptr, sz]),
    "yao_tn_contract_path": (C.c_int, [vp, vp, u32p, sz, dptr, sz]),
}

# enum yao_tn_kind
TN_EINSUM, TN_BOUNDARY, TN_OVERLAP, TN_EXPECTATION, TN_DM, TN_EXPECTATION_DM = range(6)

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise ImportError(
                        f"{LIB_PATH} is missing: build it with `python yao-rs_b200/build.py`")
                L = C.CDLL(str(LIB_PATH))
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


class YaoError(RuntimeError):
    """A failed library call; `status` is the negative yao_status code.

    yao-rs panics on these conditions; the message keeps its wording."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class CircuitError(YaoError):
    """Circuit::new returned Err(CircuitError); `kind` is the variant."""

    KINDS = {1: "ControlConfigLengthMismatch", 2: "LocOutOfRange", 3: "OverlappingLocs",
             4: "ControlSiteNotQubit", 5: "NamedGateTargetNotQubit", 6: "MatrixSizeMismatch"}

    def __init__(self, status, message, kind):
        super().__init__(status, message)
        self.kind = self.KINDS.get(kind, "Unknown")


def check(status: int):
    if status != YAO_OK:
        msg = lib().yao_last_error().decode()
        raise YaoError(status, msg)


# ---------------------------------------------------------------- context
_ctx = {}


def context(device: int | None = None):
    """Per-device library context (created on first use)."""
    if device is None:
        device = int(os.environ.get("YAO_DEVICE", "0"))
    c = _ctx.get(device)
    if c is None:
        h = C.c_void_p()
        check(lib().yao_ctx_create(device, C.byref(h)))
        c = _ctx[device] = h
    return c


def launch_count(device: int | None = None) -> int:
    n = C.c_uint64()
    check(lib().yao_ctx_launch_count(context(device), C.byref(n)))
    return n.value


def stream_ptr(device: int | None = None) -> int:
    """The cudaStream_t (as an integer) the context launches on."""
    s = C.c_void_p()
    check(lib().yao_ctx_stream(context(device), C.byref(s)))
    return s.value or 0


def synchronize(device: int | None = None):
    check(lib().yao_ctx_synchronize(context(device)))


def profile(enable: bool, device: int | None = None):
    """Turn per-launch CUDA-event timing on or off (clears the records)."""
    check(lib().yao_ctx_profile(context(device), 1 if enable else 0))


def profile_report(device: int | None = None) -> list:
    import json
    buf = C.create_string_buffer(1 << 16)
    check(lib().yao_ctx_profile_report(context(device), buf, len(buf)))
    return json.loads(buf.value.decode())
