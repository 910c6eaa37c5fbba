"""yao_rs — Python mirror of the yao-rs crate API (src/lib.rs:25-48) over the
B200 library libyao_gpu.so.

Circuits, gates, noise channels and operators are host values; registers
and density matrices live in GPU memory.  Every compute call goes through
the C ABI of include/yao_gpu.h; there is no CPU fallback.
"""
from . import _abi, einsum
from ._abi import (C64, C128, MODE_FUSED, MODE_PLAIN, MODE_TILED, CircuitError, YaoError, context,
                   launch_count)
from .circuit import (Circuit, PositionedAnnotation, PositionedChannel, PositionedGate, channel, control,
                      elements_array, label, put)
from .gate import Gate
from .noise import NoiseChannel
from .operator import Op, OperatorPolynomial, OperatorString, op_matrix
from .ops import (MeasureResult, PostProcess, apply, apply_inplace, autotune, batch_apply, expect_arrayreg, expect_dm, expect_grad_batch,
                  expect_grad, grad_plan_info, measure_with_postprocess, plan_info, probs)
from .einsum import (TensorNetwork, circuit_to_einsum, circuit_to_einsum_dm, circuit_to_einsum_with_boundary,
                     circuit_to_expectation, circuit_to_expectation_dm, circuit_to_overlap, contract, contract_dm,
                     contract_dm_with_tree, contract_with_tree)
from .einsum import contract as contract_tn
from .register import ArrayReg, DensityMatrix, Register, density_matrix_from_reg

__all__ = [
    "ArrayReg", "C64", "C128", "Circuit", "CircuitError", "DensityMatrix", "Gate", "MODE_FUSED", "MODE_PLAIN",
    "MODE_TILED", "MeasureResult", "NoiseChannel", "Op", "OperatorPolynomial", "OperatorString",
    "PositionedAnnotation", "PositionedChannel", "PositionedGate", "PostProcess", "Register", "YaoError",
    "apply", "apply_inplace", "autotune", "batch_apply", "channel", "context", "control", "density_matrix_from_reg",
    "elements_array", "expect_arrayreg", "expect_dm", "expect_grad", "expect_grad_batch", "grad_plan_info", "label", "launch_count",
    "measure_with_postprocess", "op_matrix", "plan_info", "probs", "put", "TensorNetwork", "circuit_to_einsum",
    "circuit_to_einsum_dm", "circuit_to_einsum_with_boundary", "circuit_to_expectation", "circuit_to_expectation_dm",
    "circuit_to_overlap", "contract", "contract_dm", "contract_dm_with_tree", "contract_tn", "contract_with_tree",
    "einsum",
]
