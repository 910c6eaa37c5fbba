"""Command line front end over the GPU path (the simulate / probs / expect /
measure commands of yao-cli, yao-cli/src/commands/{simulate,probs,expect,
measure}.rs).

    python -m yao_rs.cli simulate circuit.json [--input state] [--output out.state]
    python -m yao_rs.cli probs state|- [--locs 0,1] [--json]
    python -m yao_rs.cli expect state|- "Z(0)Z(1) + 0.5*X(2)" [--json]
    python -m yao_rs.cli measure state|- [--shots 1024] [--locs 0,1] [--seed S] [--json]
    python -m yao_rs.cli run circuit.json [--probs] [--op "Z(0)"] [--json]

States use the yao-state-v1 file format; `-` reads standard input.  The
expectation value is the library's (src/expect.rs), computed on the GPU.
"""
from __future__ import annotations

import argparse
import json
import re
import sys

import numpy as np

from .json_io import circuit_from_json, load_state, save_state
from .operator import Op, OperatorPolynomial, OperatorString
from .ops import apply, expect_arrayreg, probs
from .register import ArrayReg

_OPS = [("P0", Op.P0), ("P1", Op.P1), ("Pu", Op.Pu), ("Pd", Op.Pd), ("I", Op.I), ("X", Op.X), ("Y", Op.Y),
        ("Z", Op.Z)]


def parse_operator(text: str) -> OperatorPolynomial:
    """yao-cli/src/operator_parser.rs: terms split on top-level +/-, an
    optional `coeff*` prefix, then NAME(site) factors."""
    text = text.strip()
    if not text:
        raise ValueError("Empty operator expression")
    terms, cur, depth = [], "", 0
    for ch in text:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth = max(0, depth - 1)
        if ch in "+-" and depth == 0 and cur.strip():
            terms.append(cur)
            cur = "-" if ch == "-" else ""
            continue
        cur += ch
    if cur.strip():
        terms.append(cur)
    coeffs, strs = [], []
    for term in terms:
        term = term.strip()
        if "*" in term:
            c, rest = term.split("*", 1)
            coeff = float(c.replace(" ", ""))
        else:
            coeff = 1.0
            rest = term
            if rest.startswith("-"):
                coeff, rest = -1.0, rest[1:]
            elif rest.startswith("+"):
                rest = rest[1:]
        rest = rest.strip()
        ops = []
        while rest:
            for name, op in _OPS:
                if rest.startswith(name):
                    rest = rest[len(name):].strip()
                    break
            else:
                raise ValueError(f"Unknown operator in '{term}'")
            m = re.match(r"\(\s*(\d+)\s*\)", rest)
            if not m:
                raise ValueError(f"Expected '(site)' after operator name in '{term}'")
            ops.append((int(m.group(1)), op))
            rest = rest[m.end():].strip()
        if not ops:
            raise ValueError(f"No operators found in term: '{term}'")
        coeffs.append(coeff)
        strs.append(OperatorString(ops))
    return OperatorPolynomial(coeffs, strs)


def _emit(human: str, obj, as_json: bool):
    print(json.dumps(obj) if as_json else human)


def _probs_report(p, n, locs, as_json):
    m = len(locs) if locs is not None else n
    lines = ["Probabilities:"]
    for i, v in enumerate(p):
        if v > 1e-10:
            lines.append(f"  |{format(i, f'0{m}b') if m else ''}> : {v:.6f}")
    _emit("\n".join(lines), {"num_qubits": n, "locs": locs, "probabilities": [float(x) for x in p]}, as_json)


def _expect_report(op_str, v, as_json):
    human = (f"<{op_str}> = {v.real:.10f}" if abs(v.imag) < 1e-10
             else f"<{op_str}> = {v.real:.10f} + {v.imag:.10f}i")
    _emit(human, {"operator": op_str, "expectation_value": {"re": v.real, "im": v.imag}}, as_json)


def sample_outcomes(p, nlocs, draws):
    """One outcome per uniform draw r, by sample_from_probs and
    decode_outcome_bits (src/measure.rs:140-156): the first index whose
    running sum of p exceeds r (the last index if none does), as nlocs bits,
    most significant first."""
    cum = np.add.accumulate(np.asarray(p, dtype=np.float64))
    idx = np.minimum(np.searchsorted(cum, np.asarray(draws, dtype=np.float64), side="right"), len(cum) - 1)
    return [[(int(i) >> (nlocs - 1 - b)) & 1 for b in range(nlocs)] for i in idx]


def format_measurement(outcomes, shots, locs, n):
    """yao-cli/src/commands/mod.rs:54-100 (format_measurement): counts per
    outcome in outcome order, the human table and the JSON object."""
    counts = {}
    for o in outcomes:
        counts[tuple(o)] = counts.get(tuple(o), 0) + 1
    ordered = sorted(counts.items())
    human = [f"Measurement results ({shots} shots):"]
    for o, cnt in ordered:
        human.append(f"  |{''.join(map(str, o))}> : {cnt} ({cnt / shots * 100:.1f}%)")
    obj = {"num_qubits": n, "shots": shots, "locs": locs,
           "counts": {"".join(map(str, o)): cnt for o, cnt in ordered}, "outcomes": outcomes}
    return "\n".join(human), obj


def main(argv=None):
    ap = argparse.ArgumentParser(prog="yao_rs.cli")
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("simulate")
    s.add_argument("circuit")
    s.add_argument("--input")
    s.add_argument("--output")
    p = sub.add_parser("probs")
    p.add_argument("input")
    p.add_argument("--locs")
    p.add_argument("--json", action="store_true")
    e = sub.add_parser("expect")
    e.add_argument("input")
    e.add_argument("op")
    e.add_argument("--json", action="store_true")
    ms = sub.add_parser("measure")
    ms.add_argument("input")
    ms.add_argument("--shots", type=int, default=1024)
    ms.add_argument("--locs")
    ms.add_argument("--seed", type=int)
    ms.add_argument("--json", action="store_true")
    r = sub.add_parser("run")
    r.add_argument("circuit")
    r.add_argument("--input")
    r.add_argument("--probs", action="store_true")
    r.add_argument("--op")
    r.add_argument("--json", action="store_true")
    a = ap.parse_args(argv)

    def load_circuit(path):
        with (sys.stdin if path == "-" else open(path)) as f:
            return circuit_from_json(f.read())

    if a.cmd == "simulate":
        c = load_circuit(a.circuit)
        reg = ArrayReg.from_vec(c.nbits, load_state(a.input)) if a.input else ArrayReg.zero_state(c.nbits)
        out = apply(c, reg).state_vec()
        if a.output is None and sys.stdout.isatty():
            sys.exit("refusing to write binary state to terminal; use --output or a pipe")
        save_state(out, a.output)
    elif a.cmd == "probs":
        st = load_state(a.input)
        n = int(st.size).bit_length() - 1
        locs = [int(x) for x in a.locs.split(",")] if a.locs else None
        _probs_report(probs(ArrayReg.from_vec(n, st), locs), n, locs, a.json)
    elif a.cmd == "expect":
        st = load_state(a.input)
        n = int(st.size).bit_length() - 1
        _expect_report(a.op, expect_arrayreg(ArrayReg.from_vec(n, st), parse_operator(a.op)), a.json)
    elif a.cmd == "measure":
        # yao-cli/src/commands/measure.rs: `shots` draws without post-processing
        # (the state is never collapsed), so the marginal probabilities are
        # computed once on the GPU and every shot samples them
        st = load_state(a.input)
        n = int(st.size).bit_length() - 1
        locs = [int(x) for x in a.locs.split(",")] if a.locs else None
        mlocs = locs if locs is not None else list(range(n))
        p = probs(ArrayReg.from_vec(n, st), mlocs)
        rng = np.random.default_rng(a.seed)
        outcomes = sample_outcomes(p, len(mlocs), rng.random(a.shots))
        human, obj = format_measurement(outcomes, a.shots, locs, n)
        _emit(human, obj, a.json)
    else:
        c = load_circuit(a.circuit)
        reg = ArrayReg.from_vec(c.nbits, load_state(a.input)) if a.input else ArrayReg.zero_state(c.nbits)
        out = apply(c, reg)
        if a.probs or not a.op:
            _probs_report(probs(out), c.nbits, None, a.json)
        if a.op:
            _expect_report(a.op, expect_arrayreg(out, parse_operator(a.op)), a.json)
    return 0


if __name__ == "__main__":
    sys.exit(main())
