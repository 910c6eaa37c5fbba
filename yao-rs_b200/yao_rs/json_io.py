"""Circuit JSON (yao-rs src/json.rs) and the binary state file format
yao-state-v1 (yao-cli/src/state_io.rs).

JSON: {"num_qubits": n, "elements": [{"type": "gate", "gate": name,
"targets": [...], "params": [...], "controls": [...], "control_configs":
[...], "matrix": [[[re, im], ...], ...], "is_diagonal": bool, "label": str},
{"type": "label", "text": str, "loc": int}]}.  Channels are not part of the
format (circuit_to_json drops them, src/json.rs:115-131).

State file: one JSON header line {"format": "yao-state-v1", "num_qubits",
"dims", "num_elements", "dtype": "complex128"} followed by num_elements
little-endian (re, im) f64 pairs.
"""
from __future__ import annotations

import io
import json
import sys

import numpy as np

from .circuit import Circuit, PositionedAnnotation, PositionedChannel, PositionedGate, label
from .gate import Gate

_SIMPLE = {"X": "X", "CNOT": "X", "CX": "X", "Y": "Y", "Z": "Z", "H": "H", "S": "S", "T": "T", "SWAP": "SWAP",
           "SqrtX": "SqrtX", "SqrtY": "SqrtY", "SqrtW": "SqrtW", "ISWAP": "ISWAP"}


class JsonError(ValueError):
    pass


def _gate_from_json(gj) -> Gate:
    """gate_json_to_element (src/json.rs:142-222)."""
    name = gj.get("gate")
    if name in _SIMPLE:
        return getattr(Gate, _SIMPLE[name])
    if name in ("Phase", "Rx", "Ry", "Rz"):
        p = gj.get("params")
        if p is None:
            raise JsonError(f"{name} gate requires params")
        if len(p) == 0:
            raise JsonError(f"{name} gate requires at least 1 parameter")
        return getattr(Gate, name)(float(p[0]))
    if name == "FSim":
        p = gj.get("params")
        if p is None:
            raise JsonError("FSim gate requires params")
        if len(p) < 2:
            raise JsonError("FSim gate requires 2 parameters")
        return Gate.FSim(float(p[0]), float(p[1]))
    if name == "Custom":
        m = gj.get("matrix")
        if m is None:
            raise JsonError("Custom gate requires matrix")
        if len(m) == 0:
            raise JsonError("Custom gate matrix cannot be empty")
        ncols = len(m[0])
        if any(len(r) != ncols for r in m):
            raise JsonError("Custom gate matrix rows must have equal length")
        arr = np.array([[complex(a, b) for a, b in r] for r in m], dtype=np.complex128)
        return Gate.Custom(arr, bool(gj.get("is_diagonal", False)), gj.get("label", ""))
    raise JsonError(f"Unknown gate type: {name}")


def circuit_from_json(text: str) -> Circuit:
    """circuit_from_json (src/json.rs:230-250)."""
    try:
        cj = json.loads(text)
    except json.JSONDecodeError as e:
        raise JsonError(f"JSON parse error: {e}") from None
    n = int(cj["num_qubits"])
    els = []
    for ej in cj["elements"]:
        t = ej.get("type")
        if t == "gate":
            g = _gate_from_json(ej)
            ctrls = list(ej.get("controls") or [])
            cfg = ej.get("control_configs")
            cfg = [bool(c) for c in cfg] if cfg is not None else [True] * len(ctrls)
            els.append(PositionedGate(g, list(ej["targets"]), ctrls, cfg))
        elif t == "label":
            els.append(label(int(ej["loc"]), ej["text"]))
        else:
            raise JsonError(f"JSON parse error: unknown element type {t!r}")
    try:
        return Circuit.qubits(n, els)
    except Exception as e:  # CircuitError
        raise JsonError(f"Circuit validation error: {e}") from None


def circuit_to_json(c: Circuit) -> str:
    """circuit_to_json (src/json.rs:112-140); channels are dropped."""
    names = {0: "X", 1: "Y", 2: "Z", 3: "H", 4: "S", 5: "T", 6: "SWAP", 7: "Phase", 8: "Rx", 9: "Ry", 10: "Rz",
             11: "SqrtX", 12: "SqrtY", 13: "SqrtW", 14: "ISWAP", 15: "FSim", 16: "Custom"}
    out = []
    for el in c.elements:
        if isinstance(el, PositionedGate):
            g = el.gate
            d = {"type": "gate", "gate": names[g.kind], "targets": list(el.target_locs)}
            if g.params:
                d["params"] = list(g.params)
            if el.control_locs:
                d["controls"] = list(el.control_locs)
                d["control_configs"] = [bool(v) for v in el.control_configs]
            if g.kind == 16:
                d["label"] = g.label
                d["matrix"] = [[[float(z.real), float(z.imag)] for z in row] for row in g.matrix()]
                d["is_diagonal"] = g.is_diagonal()
            out.append(d)
        elif isinstance(el, PositionedAnnotation):
            out.append({"type": "label", "text": el.text, "loc": el.loc})
        elif isinstance(el, PositionedChannel):
            continue
    return json.dumps({"num_qubits": c.nbits, "elements": out}, indent=2)


FORMAT_VERSION = "yao-state-v1"


def write_state(state: np.ndarray, f) -> None:
    """write_state_to_writer (yao-cli/src/state_io.rs:23-45)."""
    v = np.ascontiguousarray(state, dtype="<c16")
    n = int(v.size).bit_length() - 1
    header = {"format": FORMAT_VERSION, "num_qubits": n, "dims": [2] * n, "num_elements": int(v.size),
              "dtype": "complex128"}
    f.write(json.dumps(header, separators=(",", ":")).encode() + b"\n")
    f.write(v.tobytes())


def read_state(f) -> np.ndarray:
    """read_state_from_reader (yao-cli/src/state_io.rs:54-100)."""
    line = f.readline()
    try:
        h = json.loads(line)
    except json.JSONDecodeError as e:
        raise JsonError(f"Failed to parse state header: {e}") from None
    if h.get("format") != FORMAT_VERSION:
        raise JsonError(f"Unknown state format: {h.get('format')} (expected {FORMAT_VERSION})")
    if h.get("dtype") != "complex128":
        raise JsonError(f"Unsupported dtype: {h.get('dtype')} (expected complex128)")
    dims = h["dims"]
    if h["num_elements"] != int(np.prod(dims)):
        raise JsonError(f"Header mismatch: num_elements={h['num_elements']} but dims {dims} imply "
                        f"{int(np.prod(dims))} elements")
    if not all(d == 2 for d in dims):
        raise JsonError(f"Only qubit (d=2) states are supported, got dims {dims}")
    data = f.read(16 * h["num_elements"])
    if len(data) != 16 * h["num_elements"]:
        raise JsonError("Failed to read state data")
    return np.frombuffer(data, dtype="<c16").astype(np.complex128)


def load_state(path: str) -> np.ndarray:
    if path == "-":
        return read_state(sys.stdin.buffer)
    with open(path, "rb") as f:
        return read_state(f)


def save_state(state: np.ndarray, path: str | None) -> None:
    if path is None or path == "-":
        write_state(state, sys.stdout.buffer)
        sys.stdout.buffer.flush()
    else:
        with open(path, "wb") as f:
            write_state(state, f)


def state_bytes(state: np.ndarray) -> bytes:
    b = io.BytesIO()
    write_state(state, b)
    return b.getvalue()
