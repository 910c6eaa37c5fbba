"""The C ABI as a C program sees it.

CPU: tests/c/abi_layout.c, compiled with gcc against include/yao_gpu.h,
prints the size and field offsets of the wire structs (yao_element,
yao_term); the ctypes mirror of the Python binding must agree with every
one.  GPU: tests/c/bell.c, a C caller linked against libyao_gpu.so, builds
a Bell pair through yao_circuit_create / yao_apply_inplace and reads back
the amplitudes, <Z0 Z1> and the probabilities."""
import ctypes as C
import math
import shutil
import subprocess
from pathlib import Path

import pytest

from yao_rs import _abi as A

ROOT = Path(__file__).resolve().parent.parent
SRC = Path(__file__).resolve().parent / "c"
INCLUDE = ROOT / "include"


def _gcc(tmp_path, name, extra=()):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not installed")
    exe = tmp_path / name
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(INCLUDE), str(SRC / f"{name}.c"), "-o", str(exe), *extra]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_wire_struct_layout_matches_ctypes(tmp_path):
    exe = _gcc(tmp_path, "abi_layout")
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    seen = dict(line.split() for line in out.splitlines())
    assert int(seen["abi_version"]) == A.lib().yao_abi_version()
    for struct in (A.yao_element, A.yao_term):
        name = struct.__name__
        assert int(seen[f"{name}.sizeof"]) == C.sizeof(struct), name
        for field, _ in struct._fields_:
            assert int(seen[f"{name}.{field}"]) == getattr(struct, field).offset, (name, field)
    assert sum(k.startswith("yao_element.") for k in seen) == len(A.yao_element._fields_) + 1
    assert sum(k.startswith("yao_term.") for k in seen) == len(A.yao_term._fields_) + 1


@pytest.mark.gpu
def test_c_caller_bell_pair(tmp_path):
    libdir = A.LIB_PATH.parent
    exe = _gcc(tmp_path, "bell", ["-L", str(libdir), "-lyao_gpu", f"-Wl,-rpath,{libdir}"])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    amps, probs, zz = {}, {}, None
    for line in r.stdout.splitlines():
        f = line.split()
        if f[0] == "amp":
            amps[int(f[1])] = (float(f[2]), float(f[3]))
        elif f[0] == "prob":
            probs[int(f[1])] = float(f[2])
        elif f[0] == "zz":
            zz = (float(f[1]), float(f[2]))
    h = 1.0 / math.sqrt(2.0)
    # (|00> + |11>) / sqrt 2: indices 0 and 3 (loc 0 is the most significant bit)
    expect = {0: h, 1: 0.0, 2: 0.0, 3: h}
    for i, a in expect.items():
        re, im = amps[i]
        assert abs(re - a) < 1e-15 and im == 0.0, (i, re, im)
        assert abs(probs[i] - a * a) < 1e-15, (i, probs[i])
    assert abs(zz[0] - 1.0) < 1e-15 and abs(zz[1]) < 1e-15
