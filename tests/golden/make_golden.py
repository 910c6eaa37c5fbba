"""Regenerates the golden fixtures in tests/golden/.

    python tests/golden/make_golden.py --ref PATH_TO_YAO_RS

1. Copies yao-rs's committed golden vectors (tests/data/{instruct,apply,
   measure,gates,noise,einsum}.json, generated by yao-rs from Yao.jl) as
   compact JSON.
2. Runs yao-rs's own numpy simulator (scripts/reference_simulate.py, which
   supports H, X, Y, Z, Rx, Ry, Rz, Phase and SWAP with controls) on seeded
   random circuits and stores the final states as pysim.json.

Needs the yao-rs source tree; the fixtures it writes are committed so the
tests never read that tree.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import random
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def copy_reference_data(ref: Path):
    for name in ["instruct", "apply", "measure", "gates", "noise", "einsum"]:
        data = json.loads((ref / "tests" / "data" / f"{name}.json").read_text())
        (HERE / f"{name}.json").write_text(json.dumps(data, separators=(",", ":")))


def random_circuit(rng: random.Random, n: int, depth: int):
    names = ["H", "X", "Y", "Z", "Rx", "Ry", "Rz", "Phase", "SWAP"]
    els = []
    for _ in range(depth):
        name = rng.choice(names)
        nt = 2 if name == "SWAP" else 1
        if n < nt:
            continue
        qs = rng.sample(range(n), n)
        targets = qs[:nt]
        nc = rng.randint(0, min(2, n - nt))
        controls = qs[nt:nt + nc]
        params = [rng.uniform(-np.pi, np.pi)] if name in ("Rx", "Ry", "Rz", "Phase") else []
        el = {"type": "gate", "gate": name, "targets": targets, "params": params}
        if controls:
            el["controls"] = controls
            el["control_configs"] = [rng.random() < 0.7 for _ in controls]
        els.append(el)
    return {"num_qubits": n, "elements": els}


def make_pysim(ref: Path, count: int = 40, seed: int = 20261203):
    spec = importlib.util.spec_from_file_location("reference_simulate", ref / "scripts" / "reference_simulate.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rng = random.Random(seed)
    cases = []
    for i in range(count):
        n = rng.randint(1, 7)
        circ = random_circuit(rng, n, rng.randint(5, 40))
        state = mod.simulate(circ)
        cases.append({"label": f"pysim-{i}", "circuit": circ,
                      "state_re": [float(x) for x in state.real], "state_im": [float(x) for x in state.imag]})
    (HERE / "pysim.json").write_text(json.dumps({"seed": seed, "cases": cases}, separators=(",", ":")))


def copy_cli_examples(ref: Path):
    """The documentation examples of yao-cli: circuit JSON files and the
    `yao probs` / `yao expect` outputs yao-rs generated for them."""
    base = ref / "docs" / "src" / "examples" / "generated"
    cases = []
    for res in sorted((base / "results").glob("*.json")):
        stem = res.name.rsplit("-", 1)[0]
        circ = base / "circuits" / f"{stem}.json"
        if not circ.exists():
            continue
        cases.append({"name": stem, "circuit": json.loads(circ.read_text()), "result": json.loads(res.read_text())})
    (HERE / "cli_examples.json").write_text(json.dumps({"cases": cases}, separators=(",", ":")))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the yao-rs checkout to read the fixtures from")
    a = ap.parse_args()
    ref = Path(a.ref)
    copy_reference_data(ref)
    make_pysim(ref)
    copy_cli_examples(ref)
    print("wrote", sorted(p.name for p in HERE.glob("*.json")))
