"""Circuit IR (yao-rs src/circuit.rs): PositionedGate, CircuitElement, Circuit,
put / control / channel / label.

A Circuit is validated by the library (yao_circuit_create restates
Circuit::new, src/circuit.rs:150-272) and keeps its library handle; the
element list stays available on the Python side.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .gate import Gate
from .noise import NoiseChannel


@dataclass
class PositionedGate:
    gate: Gate
    target_locs: list
    control_locs: list = field(default_factory=list)
    control_configs: list = field(default_factory=list)

    def all_locs(self):
        return list(self.control_locs) + list(self.target_locs)


@dataclass
class PositionedChannel:
    channel: NoiseChannel
    locs: list


@dataclass
class PositionedAnnotation:
    text: str
    loc: int


def put(target_locs, gate: Gate):
    """put (src/circuit.rs:435-437): a gate without controls."""
    return PositionedGate(gate, list(target_locs), [], [])


def control(ctrl_locs, target_locs, gate: Gate):
    """control (src/circuit.rs:454-457): active-high controls."""
    return PositionedGate(gate, list(target_locs), list(ctrl_locs), [True] * len(ctrl_locs))


def channel(locs, noise: NoiseChannel):
    """channel (src/circuit.rs:460-465)."""
    return PositionedChannel(noise, list(locs))


def label(loc, text):
    """label (src/circuit.rs:486-491): a no-op annotation."""
    return PositionedAnnotation(str(text), int(loc))


def _fill_gate(e: A.yao_element, pg: PositionedGate, keep: list):
    e.kind = A.ELEM_GATE
    e.type = pg.gate.kind
    t = (C.c_uint32 * max(1, len(pg.target_locs)))(*pg.target_locs)
    c = (C.c_uint32 * max(1, len(pg.control_locs)))(*pg.control_locs)
    cfg = (C.c_uint8 * max(1, len(pg.control_configs)))(*[1 if v else 0 for v in pg.control_configs])
    keep += [t, c, cfg]
    e.targets = C.cast(t, C.POINTER(C.c_uint32))
    e.ntargets = len(pg.target_locs)
    e.ctrl_locs = C.cast(c, C.POINTER(C.c_uint32))
    e.nctrl = len(pg.control_locs)
    e.ctrl_configs = C.cast(cfg, C.POINTER(C.c_uint8))
    e.nconfigs = len(pg.control_configs)
    for i, p in enumerate(pg.gate.params):
        e.params[i] = p
    if pg.gate.kind == A.GATE_CUSTOM:
        m = np.ascontiguousarray(pg.gate._matrix, dtype=np.complex128)
        keep.append(m)
        e.matrix = m.ctypes.data_as(A.dptr)
        e.matrix_dim = m.shape[0]
        e.is_diagonal = 1 if pg.gate._is_diagonal else 0


def elements_array(elements):
    """The C wire form of a list of circuit elements (and the buffers it points to)."""
    keep = []
    arr = (A.yao_element * max(1, len(elements)))()
    for i, el in enumerate(elements):
        e = arr[i]
        if isinstance(el, PositionedGate):
            _fill_gate(e, el, keep)
        elif isinstance(el, PositionedChannel):
            el.channel.fill_element(e, keep, el.locs)
        elif isinstance(el, PositionedAnnotation):
            e.kind = A.ELEM_ANNOTATION
            t = (C.c_uint32 * 1)(el.loc)
            keep.append(t)
            e.targets = C.cast(t, C.POINTER(C.c_uint32))
            e.ntargets = 1
        else:
            raise TypeError(f"not a circuit element: {el!r}")
    return arr, keep


class Circuit:
    """Circuit (src/circuit.rs:136-144)."""

    def __init__(self, dims, elements):
        self.dims = [int(d) for d in dims]
        self.elements = list(elements)
        self.nbits = len(self.dims)
        self._handle = None
        self._build()

    @staticmethod
    def qubits(nbits, elements):
        return Circuit([2] * nbits, elements)

    def _build(self):
        arr, keep = elements_array(self.elements)
        dims = (C.c_uint32 * max(1, len(self.dims)))(*self.dims)
        h = C.c_void_p()
        ce = C.c_int32(0)
        st = A.lib().yao_circuit_create(dims, len(self.dims), arr, len(self.elements), C.byref(h),
                                        C.byref(ce))
        if st != A.YAO_OK:
            msg = A.lib().yao_last_error().decode()
            if st == A.YAO_ERR_CIRCUIT:
                raise A.CircuitError(st, msg, ce.value)
            raise A.YaoError(st, msg)
        self._handle = h

    @property
    def handle(self):
        return self._handle

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and A._lib is not None:
            A.lib().yao_circuit_free(h)
            self._handle = None

    def num_sites(self):
        return self.nbits

    def total_dim(self):
        return int(np.prod(self.dims))

    # src/circuit.rs:308-352
    def num_params(self) -> int:
        return sum(el.gate.num_params() for el in self.elements if isinstance(el, PositionedGate))

    def parameters(self) -> list:
        out = []
        for el in self.elements:
            if isinstance(el, PositionedGate):
                out += el.gate.get_params()
        return out

    def dispatch(self, params):
        params = list(params)
        assert len(params) == self.num_params(), (
            f"dispatch length {len(params)} does not match num_params {self.num_params()}")
        off = 0
        for el in self.elements:
            if isinstance(el, PositionedGate):
                n = el.gate.num_params()
                if n:
                    el.gate = Gate(el.gate.kind, params[off:off + n])
                    off += n
        buf = (C.c_double * max(1, len(params)))(*params)
        A.check(A.lib().yao_circuit_dispatch(self._handle, buf, len(params)))

    # src/circuit.rs:360-378
    def dagger(self) -> "Circuit":
        els = []
        for el in reversed(self.elements):
            if isinstance(el, PositionedGate):
                els.append(PositionedGate(el.gate.dagger(), list(el.target_locs), list(el.control_locs),
                                          list(el.control_configs)))
            else:
                els.append(el)
        return Circuit(self.dims, els)

    def __repr__(self):
        lines = [f"nqubits: {self.nbits}"]
        for el in self.elements:
            if isinstance(el, PositionedGate):
                if el.control_locs:
                    lines.append(f"  C(q[{', '.join(map(str, el.control_locs))}]) {el.gate!r} @ "
                                 f"q[{', '.join(map(str, el.target_locs))}]")
                else:
                    lines.append(f"  {el.gate!r} @ q[{', '.join(map(str, el.target_locs))}]")
            elif isinstance(el, PositionedChannel):
                lines.append(f"  {el.channel!r} @ q[{', '.join(map(str, el.locs))}]")
            else:
                lines.append(f'  "{el.text}" @ q[{el.loc}]')
        return "\n".join(lines)
