"""Benchmark: 30-qubit layered circuit, FP64 gate-by-gate apply throughput.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the layered random circuit on n=30 qubits, complex128, 16 GiB
state): each layer applies Rx, Ry, Rz to every qubit (angles uniform in
[0, 2 pi), seeded per layer) and then a CNOT brickwork on (2i, 2i+1) for
even layers, (2i+1, 2i+2) for odd layers; 40 layers make the circuit
(4180 gates), input |0...0>.  One step = one layer through the PLAIN
(gate-by-gate, bit-exact) path; K = 40 steps is exactly one circuit.

metric/value: algorithmic HBM GB/s of the plain path (every gate reads and
writes the amplitudes it updates once: 2*16*2^30 bytes for an uncontrolled
dense or diagonal gate, half that for a CNOT), whole job over N GPUs.
Extra keys: seconds per circuit of the TILED (bit-exact) and FUSED k=5 forms
(FP64 and complex64 with split coefficients) with 1 - fidelity against the
FP64 result, and the VQE adjoint gradient rate (n=24, 384 parameters,
transverse-field Ising model).

Multi-GPU: replicas only (the simulation of one circuit does not shard
here); every rank runs the same per-GPU workload, value = all ranks' bytes /
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "yao-rs_b200"))

METRIC = "30q gate-apply HBM GB/s & s/circuit; VQE grads/s fused vs plain at 1-F<=1e-6"
NQ = 30
LAYERS = 40


# --------------------------------------------------------------- workload
def layer_elements(Y, n, layer, seed=2026):
    rng = np.random.default_rng([seed, layer])
    ang = rng.uniform(0.0, 2.0 * math.pi, size=(n, 3))
    els = []
    for q in range(n):
        els.append(Y.put([q], Y.Gate.Rx(float(ang[q, 0]))))
        els.append(Y.put([q], Y.Gate.Ry(float(ang[q, 1]))))
        els.append(Y.put([q], Y.Gate.Rz(float(ang[q, 2]))))
    start = 0 if layer % 2 == 0 else 1
    for a in range(start, n - 1, 2):
        els.append(Y.control([a], [a + 1], Y.Gate.X))
    return els


def layer_bytes(n, layer, amp_bytes=16):
    """Algorithmic bytes of one layer: 3n full-state gates + CNOTs on half."""
    full = 2 * amp_bytes * (1 << n)
    ncnot = len(range(0 if layer % 2 == 0 else 1, n - 1, 2))
    return 3 * n * full + ncnot * full // 2


def vqe_circuit(Y, n, layers, params):
    els, k = [], 0
    for _ in range(layers):
        for q in range(n):
            els.append(Y.put([q], Y.Gate.Ry(float(params[k]))))
            els.append(Y.put([q], Y.Gate.Rz(float(params[k + 1]))))
            k += 2
        for q in range(n):
            els.append(Y.control([q], [(q + 1) % n], Y.Gate.X))
    return Y.Circuit.qubits(n, els)


def tfim(Y, n):
    cs, ss = [], []
    for i in range(n):
        cs.append(-1.0)
        ss.append(Y.OperatorString([(i, Y.Op.Z), ((i + 1) % n, Y.Op.Z)]))
    for i in range(n):
        cs.append(-1.0)
        ss.append(Y.OperatorString([(i, Y.Op.X)]))
    return Y.OperatorPolynomial(cs, ss)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = str(gpu_index)
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and f[0] == self.idx:
                self.rows.append(f)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------ CPU baseline
def cpu_baseline_sample(n, budget_s, layer=0):
    """The oracle (C restatement of yao-rs's single-threaded CPU loops) on
    the first gates of layer 0 at n qubits, until `budget_s` seconds pass."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    import yao_rs as Y

    O.lib()
    els = layer_elements(Y, n, layer)
    st = np.empty(1 << n, dtype=np.complex128)
    st.fill(0)  # touch every page before timing
    st[0] = 1
    arr, keep = Y.elements_array(els)
    import ctypes as C
    t_total, b_total, gates = 0.0, 0.0, 0
    full = 2 * 16 * (1 << n)
    for i, el in enumerate(els):
        t0 = time.perf_counter()
        O.lib().orc_apply_inplace(n, C.cast(C.addressof(arr[i]), C.c_void_p), 1,
                                  st.ctypes.data_as(C.c_void_p))
        t_total += time.perf_counter() - t0
        b_total += full if not el.control_locs else full // 2
        gates += 1
        if t_total > budget_s:
            break
    return b_total / t_total / 1e9, gates, t_total, st, els[:gates]


def max_over_ranks(torch, ms, world, device):
    """The slowest rank's time (every rank calls this; one MAX all-reduce)."""
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gbps(bytes_per_rank, world, ms):
    """Whole-job GB/s: every rank moved bytes_per_rank in at most ms."""
    return world * bytes_per_rank / (ms / 1e3) / 1e9


def host_cpus():
    """CPUs this process may use: the machine's count, the affinity mask and
    the cgroup quota (cpu.max), which bounds how much host work can overlap."""
    out = {"cpu_count": os.cpu_count(), "affinity": len(os.sched_getaffinity(0))}
    try:
        out["cgroup_cpu_max"] = open("/sys/fs/cgroup/cpu.max").read().strip()
    except OSError:
        pass
    return out


def host_ram_gb():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


class Background:
    """fn(*args) in a thread.  The oracle's calls are ctypes calls into C,
    which release the GIL, so the CPU checks of large configurations run
    while the GPU measurements go on."""

    def __init__(self, fn, *args):
        self.out, self.err, self.s = None, None, None
        self.t = threading.Thread(target=self._run, args=(fn, args), daemon=True)
        self.t.start()

    def _run(self, fn, args):
        t0 = time.perf_counter()
        try:
            self.out = fn(*args)
        except Exception as e:  # reported with the result
            self.err = repr(e)
        self.s = time.perf_counter() - t0

    def result(self):
        self.t.join()
        if self.err:
            raise RuntimeError(self.err)
        return self.out


def sig(x, d=4):
    """Round floats to d significant digits (compact JSON)."""
    if isinstance(x, float):
        return float(f"{x:.{d}g}")
    if isinstance(x, dict):
        return {k: sig(v, d) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [sig(v, d) for v in x]
    return x


def bench_config(n, world):
    """The workload both arms measure: per-gate algorithmic GB/s of the PLAIN
    FP64 path on the layered circuit (one layer a step on the GPU; the CPU arm
    samples it one gate a step)."""
    return {"workload": f"layered random circuit n={n}, 40 layers (Rx,Ry,Rz + CNOT brickwork), PLAIN FP64 "
                        "gate by gate",
            "qubits": n, "state_bytes": 16 * (1 << n), "l2": "state larger than L2, no flush",
            "parallelism": f"replicas x{world}"}


# -------------------------------------------------------------- reference
def run_reference(args, rank, world):
    """yao-rs cannot run here (Rust; no toolchain): its CPU path is timed
    through the oracle, the C restatement of its loops, single-threaded like
    yao-rs.  One step = one gate of the layered circuit at n qubits."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import ctypes as C

    import oracle as O
    import yao_rs as Y

    n = args.qubits if host_ram_gb() > 3 * 16 * (1 << args.qubits) / 1e9 else min(args.qubits, 28)
    O.lib()
    gates = []
    for layer in range(LAYERS):
        gates += layer_elements(Y, n, layer)
    arr, keep = Y.elements_array(gates)
    st = np.empty(1 << n, dtype=np.complex128)
    st.fill(0)  # touch every page before timing
    st[0] = 1
    full = 2 * 16 * (1 << n)
    times, nbytes = [], []
    for s in range(args.warmup + args.steps):
        i = s % len(gates)
        t0 = time.perf_counter()
        O.lib().orc_apply_inplace(n, C.cast(C.addressof(arr[i]), C.c_void_p), 1, st.ctypes.data_as(C.c_void_p))
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
            nbytes.append(full if not gates[i].control_locs else full // 2)
    T = sum(times)
    v = sum(nbytes) / T / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * T / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": bench_config(n, world),
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": 1, "kind": "port",
                         "sample": f"one gate of the layered circuit per step (layer order), {args.steps} gates at "
                                   f"n={n}, oracle (C restatement of yao-rs instruct loops, -O3, 1 thread: yao-rs "
                                   "is single-threaded)"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=LAYERS)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=NQ)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--profile-case", default=None,
                    choices=["plain", "tiled", "fused64", "fused32", "fused32_tc", "pass1q", "fused64_dmma",
                             "fused64_cuda", "vqe", "grad24", "dm", "dm_fused", "dm_channel", "batch", "vqe_batch",
                             "tc_drift"],
                    help="run one small case of a kernel family (for ncu captures) and exit")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    import yao_rs as Y
    from yao_rs import _abi as A

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    n = args.qubits
    dev = local
    circuits = [Y.Circuit.qubits(n, layer_elements(Y, n, l)) for l in range(LAYERS)]
    stream = torch.cuda.ExternalStream(A.stream_ptr(dev), device=torch.device("cuda", dev))

    def barrier():
        A.synchronize(dev)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    reg = Y.ArrayReg.zero_state(n, device=dev)
    for i in range(args.warmup):
        Y.apply_inplace(circuits[i % LAYERS], reg)
    # timed region starts from |0...0>: K = 40 steps is one full circuit
    A.check(A.lib().yao_ctx_synchronize(A.context(dev)))
    del reg
    reg = Y.ArrayReg.zero_state(n, device=dev)
    barrier()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[dev] if vis else dev)
    clocks.start()
    time.sleep(0.3)
    A.profile(True, dev)
    launches0 = Y.launch_count(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        Y.apply_inplace(circuits[i % LAYERS], reg)
    e1.record(stream)
    e1.synchronize()
    launches = Y.launch_count(dev) - launches0
    prof = A.profile_report(dev)
    A.profile(False, dev)
    clk = clocks.stop()
    ms = max_over_ranks(torch, e0.elapsed_time(e1), world, f"cuda:{dev}")
    nbytes = sum(layer_bytes(n, i % LAYERS) for i in range(args.steps))
    value = job_gbps(nbytes, world, ms)
    prof_bytes = sum(p["bytes"] for p in prof)

    # roofline of the dominant kernel (largest share of device time)
    peak, peak_kind = measured_peaks()
    top = max(prof, key=lambda p: p["ms"])
    achieved = top["bytes"] / (top["ms"] / 1e3) / 1e9
    # DRAM traffic per launch of the dense 1-qubit kernel: ncu capture of
    # `bench.py --profile-case plain --qubits 27` (dram__bytes_read.sum +
    # dram__bytes_write.sum = 2.1475 + 2.0884 GB for 2^27 amplitudes), scaled
    # by the amplitudes one launch processes here.
    traffic = None
    if top["kernel"] == "gate_dense1":
        traffic = (2.1475e9 + 2.0884e9) * (1 << n) / (1 << 27)
    roofline = {"bound": "hbm", "kernel": top["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "bytes_per_launch": top["bytes"] / top["launches"], "launches": top["launches"],
                "avg_launch_ms": top["ms"] / top["launches"], "traffic": traffic,
                "traffic_source": "ncu at n=27 x 2^(n-27)" if traffic else None,
                "share": top["ms"] / sum(p["ms"] for p in prof)}
    kernels = [{"kernel": p["kernel"], "launches": p["launches"], "ms": round(p["ms"], 3),
                "GBps": round(p["bytes"] / (p["ms"] / 1e3) / 1e9, 1)} for p in prof]

    # e2e: host state in pinned memory -> upload, K layers, download, through the public API
    host = torch.zeros(1 << n, dtype=torch.complex128, pin_memory=True)
    host[0] = 1
    hp = host.data_ptr()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    A.check(A.lib().yao_reg_upload(reg.handle, A.C.c_void_p(hp)))
    for i in range(args.steps):
        Y.apply_inplace(circuits[i % LAYERS], reg)
    A.check(A.lib().yao_reg_to_host(reg.handle, A.C.c_void_p(hp)))
    f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(torch, f0.elapsed_time(f1), world, f"cuda:{dev}")
    state_bytes = 16 * (1 << n)
    e2e = {"value": job_gbps(nbytes, world, e2e_ms), "unit": "GB/s",
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps,
           "note": "one state upload + one download per K steps"}
    del host

    extras = {}
    cpu = None
    first_gates = None
    del reg
    if rank == 0 and world == 1 and not args.no_extras:
        extras = run_extras(Y, A, torch, stream, circuits, n, dev)
    if rank == 0 and world == 1:
        nb = n if host_ram_gb() > 2.5 * 16 * (1 << n) / 1e9 else min(n, 28)
        v, g, tt, cpu_state, gates = cpu_baseline_sample(nb, args.cpu_budget)
        cpu = {"value": v, "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"first {g} gates of layer 0 at n={nb} ({tt:.1f} s), oracle (C restatement of yao-rs's "
                         "loops)"}
        # parity at the benchmark's own size: the same gates from |0...0> on
        # the GPU (PLAIN), compared on the device with the oracle's state
        gr = Y.ArrayReg.zero_state(nb, device=dev)
        Y.apply_inplace(Y.Circuit.qubits(nb, gates), gr)
        cr = Y.ArrayReg.from_vec(nb, cpu_state, device=dev)
        first_gates = {"qubits": nb, "gates": g, "max_abs_diff_vs_oracle": gr.max_abs_diff(cr)}
        del gr, cr, cpu_state
    if rank == 0:
        line = {
            "metric": METRIC, "value": sig(value, 6), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sig(ms / args.steps, 6), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": bench_config(n, world),
            "roofline": sig(roofline), "e2e": sig(e2e), "gpu_launches": int(launches), "clocks": clk,
            "cpu_baseline": sig(cpu),
        }
        plain_s = ms / args.steps * LAYERS / 1e3
        # the full record (kernel tables, per-run lists, the DM <Z_i>) on a
        # line of its own; the last line stays short
        detail = {"detail": {"kernels": kernels, "profiled_bytes": prof_bytes, "first_gates_n30": first_gates,
                             "host_cpus": host_cpus(),
                             **extras}}
        print(json.dumps(detail), flush=True)
        line["summary"] = summary(extras, plain_s, first_gates)
        print(json.dumps(line, separators=(",", ":")), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def profile_case(args):
    """One layer of the layered circuit at --qubits (default 30; use 27 for a
    2 GiB state, still larger than L2) in one execution form, or one VQE
    gradient (n=20), or one noisy density-matrix layer (n=12); for ncu."""
    import yao_rs as Y
    from yao_rs import _abi as A

    n = args.qubits
    if args.profile_case == "tc_drift":
        return tc_drift(Y, A, min(n, 24))
    if args.profile_case == "vqe":
        nv = 20
        rng = np.random.default_rng(1)
        c = vqe_circuit(Y, nv, 2, rng.uniform(-3, 3, size=4 * nv))
        Y.expect_grad(tfim(Y, nv), c, Y.ArrayReg.zero_state(nv))
    elif args.profile_case == "grad24":
        # one expect_grad of the VQE ansatz (n = 24, 8 layers, 384
        # parameters) with the TFIM Hamiltonian: FUSED forward, tiled reverse
        # sweep
        rng = np.random.default_rng(2024)
        c = vqe_circuit(Y, 24, 8, rng.uniform(-math.pi, math.pi, size=2 * 24 * 8))
        Y.expect_grad(tfim(Y, 24), c, Y.ArrayReg.zero_state(24))
    elif args.profile_case == "batch":
        draws, cs = uneven_batch(Y, count=256)
        regs = [Y.ArrayReg.zero_state(nq, Y.C64) for nq, _ in draws]
        Y.batch_apply(cs, regs, Y.MODE_FUSED, 4)
    elif args.profile_case == "vqe_batch":
        rng = np.random.default_rng(16)
        sets = rng.uniform(-math.pi, math.pi, size=(512, 2 * 16 * 2))
        c = vqe_circuit(Y, 16, 2, sets[0])
        Y.expect_grad_batch(tfim(Y, 16), c, sets, Y.ArrayReg.zero_state(16))
    elif args.profile_case == "pass1q":
        # one complex64 tile pass holding a single 1-qubit block (the bare
        # load / store pipeline of a pass), run 4 times; 2^12 tiles unless
        # YAO_TILE_BITS / YAO_REG_BITS say otherwise
        os.environ.setdefault("YAO_TILE_BITS", "12")
        os.environ.setdefault("YAO_REG_BITS", "3")
        os.environ["YAO_AUTOTUNE"] = "0"
        c = Y.Circuit.qubits(n, [Y.put([0], Y.Gate.Ry(0.3))])
        r = Y.ArrayReg.zero_state(n, Y.C64)
        for _ in range(4):
            Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
    elif args.profile_case == "fused32_tc":
        # 8 layers as one circuit, dense 3..5-qubit blocks on the tensor cores
        os.environ.update(YAO_TILE_BITS="12", YAO_REG_BITS="3", YAO_AUTOTUNE="0")
        c = Y.Circuit.qubits(n, [el for l in range(8) for el in layer_elements(Y, n, l)])
        r = Y.ArrayReg.zero_state(n, Y.C64)
        Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
    elif args.profile_case in ("fused64_dmma", "fused64_cuda"):
        # 8 layers as one circuit, complex128 FUSED k = 4 on 2^11 tiles:
        # dense 3..4-qubit blocks on the FP64 tensor cores, or (cuda) on the
        # CUDA cores
        os.environ.update(YAO_TILE_BITS="11", YAO_REG_BITS="3", YAO_AUTOTUNE="0",
                          YAO_DMMA="1" if args.profile_case == "fused64_dmma" else "0")
        c = Y.Circuit.qubits(n, [el for l in range(8) for el in layer_elements(Y, n, l)])
        r = Y.ArrayReg.zero_state(n, Y.C128)
        Y.apply_inplace(c, r, Y.MODE_FUSED, 4)
    elif args.profile_case == "dm_channel":
        # one noisy layer at n = 12 (PLAIN): gate and channel passes, the
        # 2-qubit depolarizing channels through the register kernel
        d = Y.DensityMatrix.zero_state(12)
        d.apply(noisy_dm_circuit(Y, 12, 1))
    elif args.profile_case == "dm_fused":
        # three noisy layers of the benchmark's density-matrix circuit at
        # --qubits (12: a 24-bit vector of 268 MB, larger than L2) in the FUSED
        # superoperator form, with the shape the autotuner picks at n = 14
        # (k = 4 blocks on 2^11 tiles)
        os.environ.update(YAO_TILE_BITS="11", YAO_REG_BITS="3", YAO_AUTOTUNE="0")
        d = Y.DensityMatrix.zero_state(n)
        d.apply(noisy_dm_circuit(Y, n, 3), Y.MODE_FUSED)
    elif args.profile_case == "dm":
        nd = 12
        els = []
        for q in range(nd):
            els.append(Y.put([q], Y.Gate.Ry(0.3 + q)))
            els.append(Y.channel([q], Y.NoiseChannel.Depolarizing(1, 1e-3)))
        for q in range(0, nd - 1, 2):
            els.append(Y.control([q], [q + 1], Y.Gate.Z))
            els.append(Y.channel([q, q + 1], Y.NoiseChannel.Depolarizing(2, 1e-3)))
        for q in range(nd):
            els.append(Y.channel([q], Y.NoiseChannel.AmplitudeDamping(1e-3, 0.0)))
        d = Y.DensityMatrix.zero_state(nd)
        d.apply(Y.Circuit.qubits(nd, els))
        d.purity()
    else:
        mode, prec, k = {"plain": (Y.MODE_PLAIN, Y.C128, 0), "tiled": (Y.MODE_TILED, Y.C128, 0),
                         "fused64": (Y.MODE_FUSED, Y.C128, 5), "fused32": (Y.MODE_FUSED, Y.C64, 5)}[args.profile_case]
        c = Y.Circuit.qubits(n, layer_elements(Y, n, 0))
        r = Y.ArrayReg.zero_state(n, prec)
        Y.apply_inplace(c, r, mode, k)
    A.synchronize()
    print(f"profile case {args.profile_case} done: {Y.launch_count()} launches")


def tc_drift(Y, A, n):
    """Complex64 FUSED k = 5 on the layered circuit (40 layers) without the
    FP64 norm restore: the norm drift per tensor-core block, 1 - F and max
    |error| against the FP64 PLAIN result, for every tensor-core variant
    (YAO_TC_VARIANT bits: 2 separate correction accumulator, 8 the integer
    form with exact int32 accumulation) and for the CUDA-core split form,
    from |0...0> and from a random state; one JSON line per form and start."""
    import torch
    os.environ.update(YAO_TILE_BITS="12", YAO_REG_BITS="3", YAO_AUTOTUNE="0", YAO_NORM_RESTORE="0")
    c = Y.Circuit.qubits(n, [el for l in range(LAYERS) for el in layer_elements(Y, n, l)])
    info = Y.plan_info(c, Y.C64, Y.MODE_FUSED, 5, 12, 3)
    stream = torch.cuda.ExternalStream(A.stream_ptr(0), device=torch.device("cuda", 0))
    rng = np.random.default_rng(77)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    starts = {"zero": None, "random": v}
    forms = [("tc_v%d" % v_, "1", str(v_)) for v_ in (0, 2, 8)] + [("cuda_core", "0", "0")]
    for sname, sv in starts.items():
        def fresh(prec):
            if sv is None:
                return Y.ArrayReg.zero_state(n, prec)
            r0 = Y.ArrayReg.from_vec(n, sv)
            return r0 if prec == Y.C128 else r0.to_precision(prec)
        ref = fresh(Y.C128)
        Y.apply_inplace(c, ref)
        n0 = fresh(Y.C64).norm() ** 2
        for name, tc, var in forms:
            os.environ.update(YAO_TC=tc, YAO_TC_VARIANT=var)
            r = fresh(Y.C64)
            Y.apply_inplace(c, r, Y.MODE_FUSED, 5)  # warm-up
            r = fresh(Y.C64)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            A.synchronize()
            e0.record(stream)
            Y.apply_inplace(c, r, Y.MODE_FUSED, 5)
            e1.record(stream)
            e1.synchronize()
            nrm2 = r.norm() ** 2
            blocks = info["tensor_core_ops"] if tc == "1" else info["blocks"]
            f = ref.fidelity(r)
            print(json.dumps({"form": name, "start": sname, "qubits": n, "tc_blocks": info["tensor_core_ops"],
                              "blocks": info["blocks"], "norm2_minus_start": nrm2 - n0,
                              "norm2_drift_per_tc_block": (nrm2 - n0) / max(1, blocks),
                              "one_minus_fidelity": 1.0 - f,
                              "one_minus_fidelity_normalised": 1.0 - f / (nrm2 * ref.norm() ** 2),
                              "max_abs_err": ref.max_abs_diff(r), "ms": e0.elapsed_time(e1)}), flush=True)


def run_extras(Y, A, torch, stream, circuits, n, dev):
    """Full 40-layer circuit through the TILED and FUSED forms, 1 - F against
    the FP64 result, and the VQE gradient rate."""
    out = {}
    # the oracle at the configurations' own sizes: the VQE energy and all 384
    # gradient entries at n = 24, and one full noisy layer of the
    # density-matrix workload at n = 12, in threads while the FUSED forms run
    # (seconds-long kernels timed by CUDA events); joined before any
    # wall-clock or launch-bound measurement, which CPU contention would skew
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.lib()
    nv, lv = 24, 8
    rng = np.random.default_rng(2024)
    params = rng.uniform(-math.pi, math.pi, size=2 * nv * lv)
    vc = vqe_circuit(Y, nv, lv, params)
    op = tfim(Y, nv)
    z24 = np.zeros(1 << nv, complex)
    z24[0] = 1
    dm12 = noisy_dm_circuit(Y, 12, 1)
    rho12 = np.zeros(1 << 24, complex)
    rho12[0] = 1

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        A.synchronize(dev)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / 1e3

    # the 40 layers as one Circuit: tiles and fused blocks span layers
    whole = Y.Circuit.qubits(n, [el for l in range(LAYERS) for el in layer_elements(Y, n, l)])
    ref = Y.ArrayReg.zero_state(n, device=dev)
    # warm-up: the autotuner picks the tile shape on a prefix of the circuit
    # (scratch copy of the register), then one throwaway layer
    chosen = {"tiled": Y.autotune(whole, ref, Y.MODE_TILED)}
    Y.apply_inplace(circuits[0], ref, Y.MODE_TILED)
    del ref
    ref = Y.ArrayReg.zero_state(n, device=dev)
    t_tiled = timed(lambda: Y.apply_inplace(whole, ref, Y.MODE_TILED))
    out["s_per_circuit_tiled"] = t_tiled
    bg_vqe = Background(O.expect_grad, op, vc, z24)
    bg_dm = Background(O.dm_apply_circuit, dm12, rho12)
    forms = {}
    for name, prec, k in (("fused_f64_k5", Y.C128, 5), ("fused_f64_k4", Y.C128, 4), ("fused_c64_k5", Y.C64, 5),
                          ("fused_c64_k4", Y.C64, 4), ("fused_c64_k3", Y.C64, 3), ("fused_c64_auto", Y.C64, 0),
                          ("fused_f64_auto", Y.C128, 0), ("fused_c64_k5_int8_norestore", Y.C64, 5)):
        # the integer tensor-core form (exact int32 accumulation) without the
        # FP64 norm restore: its accuracy is its own
        extra = {"YAO_TC_VARIANT": "8", "YAO_NORM_RESTORE": "0"} if name.endswith("int8_norestore") else {}
        saved = {key: os.environ.get(key) for key in extra}
        os.environ.update(extra)
        r = Y.ArrayReg.zero_state(n, prec, device=dev)
        chosen[name] = Y.autotune(whole, r, Y.MODE_FUSED, k)
        Y.apply_inplace(circuits[0], r, Y.MODE_FUSED, k)
        # median of three runs (single runs of a few seconds vary with the
        # power cap); accuracy from the last
        ts = []
        for _ in range(3):
            del r
            r = Y.ArrayReg.zero_state(n, prec, device=dev)
            ts.append(timed(lambda: Y.apply_inplace(whole, r, Y.MODE_FUSED, k)))
        f = ref.fidelity(r)
        nrm2 = r.norm() ** 2
        forms[name] = {"s_per_circuit": sorted(ts)[1], "s_runs": ts, "one_minus_fidelity": max(0.0, 1.0 - f),
                       "one_minus_fidelity_normalised": 1.0 - f / nrm2, "norm2_minus_1": nrm2 - 1.0,
                       "max_abs_err": ref.max_abs_diff(r)}
        del r
        for key, v in saved.items():
            if v is None:
                os.environ.pop(key, None)
            else:
                os.environ[key] = v
    out["fused"] = forms
    out["autotuned"] = chosen
    del ref
    vo, go = bg_vqe.result()
    ref12 = bg_dm.result()
    # VQE: n=24, 8 layers of Ry.Rz on every qubit + CNOT ring, TFIM
    z = Y.ArrayReg.zero_state(nv, device=dev)
    Y.expect_grad(op, vc, z)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        val, g = Y.expect_grad(op, vc, z)
    dt = (time.perf_counter() - t0) / reps
    # central finite differences (eps = 1e-5) on a few parameters
    eps, fd_err = 1e-5, 0.0
    for i in (0, len(params) // 2, len(params) - 1):
        pp, pm = list(params), list(params)
        pp[i] += eps
        pm[i] -= eps
        fp = Y.expect_arrayreg(Y.apply(vqe_circuit(Y, nv, lv, pp), z), op).real
        fm = Y.expect_arrayreg(Y.apply(vqe_circuit(Y, nv, lv, pm), z), op).real
        fd = (fp - fm) / (2 * eps)
        fd_err = max(fd_err, abs(fd - g[i]) / max(1e-12, abs(g[i])))
    # the oracle's expect_grad at n = 24 on the same angles (one thread,
    # run in the background since the start of the extras)
    out["vqe"] = {"qubits": nv, "params": len(g), "gates": len(vc.elements), "grads_per_s": 1.0 / dt,
                  "s_per_grad": dt, "energy": val, "fd_max_rel_err": fd_err,
                  "oracle_energy_diff": abs(val - vo),
                  "oracle_max_abs_grad_diff": float(np.max(np.abs(np.asarray(go) - np.asarray(g)))),
                  "cpu_oracle_s_per_grad": bg_vqe.s}
    del z
    out["batched_vqe"] = vqe_batch_extra(Y, A, torch, stream, dev, timed)
    out["qft20"] = qft_extra(Y, A, torch, stream, dev, timed)
    out["noisy_dm14"] = dm_extra(Y, A, torch, stream, dev, timed)
    # one noisy layer at n = 12 against the oracle: PLAIN bit for bit, FUSED
    # (superoperators through the tile passes) to rounding
    d12 = {}
    for name, mode in (("plain", Y.MODE_PLAIN), ("fused", Y.MODE_FUSED)):
        d = Y.DensityMatrix.zero_state(12, device=dev)
        d.apply(dm12, mode)
        d12[name] = float(np.max(np.abs(d.state_data() - ref12)))
        del d
    out["noisy_dm14"]["n12_layer_vs_oracle"] = {"max_abs_diff": d12, "cpu_oracle_s": bg_dm.s}
    out["batched_circuits"] = batch_extra(Y, A, torch, stream, dev, timed)
    out["tn20"] = tn_extra(Y, A, dev)
    return out


def tn_extra(Y, A, dev):
    """The tensor network of the layered circuit at n = 20 (4 layers, |0>
    inputs, open outputs: circuit_to_einsum_with_boundary) contracted on the
    GPU (pairwise, greedy order), against the PLAIN state vector; the
    oracle's numpy contraction of the same network timed beside it."""
    n, layers = 20, 4
    c = Y.Circuit.qubits(n, [el for l in range(layers) for el in layer_elements(Y, n, l)])
    net = Y.circuit_to_einsum_with_boundary(c)
    Y.einsum.contract(net)  # warm-up
    t0 = time.perf_counter()
    out = Y.einsum.contract(net).reshape(-1)
    t_gpu = time.perf_counter() - t0
    r = Y.ArrayReg.zero_state(n, device=dev)
    Y.apply_inplace(c, r)
    diff = float(np.max(np.abs(out - r.state_vec())))
    sys.path.insert(0, str(ROOT / "oracle"))
    import tn as OT
    ref = {"ixs": net.ixs, "iy": net.iy, "tensors": net.tensors, "size": net.size_dict}
    t0 = time.perf_counter()
    OT.contract(ref)
    t_cpu = time.perf_counter() - t0
    return {"qubits": n, "tensors": len(net.tensors), "s_gpu": t_gpu, "s_cpu_numpy": t_cpu,
            "max_abs_diff_vs_state_vector": diff}


def summary(x, plain_s, first_gates):
    """The figures the benchmark's claims rest on, rounded, for the last
    line: n = 30 forms (s/circuit, 1 - F, max |err|, autotuned choice), the
    VQE gradient with its oracle and finite-difference checks, the batches,
    the noisy density matrix and the parity checks at the configs' sizes."""
    s = {"layered30": {"plain_s": plain_s, "first_gates_vs_oracle": first_gates}}
    if not x:
        return sig(s)
    L = s["layered30"]
    L["tiled_s"] = x["s_per_circuit_tiled"]
    # [s/circuit, 1 - F (normalised), |norm^2 - 1|]
    L["fused"] = {k.replace("fused_", ""): [sig(v["s_per_circuit"], 3), sig(v["one_minus_fidelity_normalised"], 2),
                                            sig(abs(v["norm2_minus_1"]), 2)]
                  for k, v in x["fused"].items() if k not in ("fused_c64_k3", "fused_c64_k4")}
    # the tuned choices of the auto forms (and of c64 k = 5): [k, tile bits,
    # register bits(, tensor cores for complex64)]
    L["autotuned"] = {k.replace("fused_", ""): [c["k"], c["tile_bits"], c["reg_bits"]] +
                      ([c["tensor_cores"]] if "c64" in k else [])
                      for k, c in x["autotuned"].items()
                      if k in ("tiled", "fused_c64_auto", "fused_f64_auto", "fused_c64_k5")}
    fs = {k: v["s_per_circuit"] for k, v in x["fused"].items()}
    L["c64_auto_speedup_vs_plain"] = plain_s / fs["fused_c64_auto"]
    L["c128_auto_speedup_vs_plain"] = plain_s / fs["fused_f64_auto"]
    L["c64_auto_over_c128_auto"] = fs["fused_c64_auto"] / fs["fused_f64_auto"]
    # the autotuner's choice against the best fixed width (1.0 = as good)
    L["auto_over_best_fixed"] = {
        "c64": fs["fused_c64_auto"] / min(v for k, v in fs.items() if k.startswith("fused_c64_k") and
                                         not k.endswith("norestore")),
        "c128": fs["fused_f64_auto"] / min(v for k, v in fs.items() if k.startswith("fused_f64_k"))}
    v = x["vqe"]
    s["vqe24"] = {k: v[k] for k in ("grads_per_s", "fd_max_rel_err", "oracle_energy_diff", "oracle_max_abs_grad_diff",
                                    "cpu_oracle_s_per_grad")}
    b = x["batched_vqe"]
    s["vqe16_batch"] = {k: b[k] for k in ("sets", "batched_grads_per_s", "single_grads_per_s",
                                          "max_grad_diff_vs_oracle")}
    c = x["batched_circuits"]
    s["batch2048"] = {"plain_s": c["s_plain"],
                      "forms": {k: [f["s"], f["speedup_vs_plain"], f["max_one_minus_fidelity"]]
                                for k, f in c["forms"].items() if k != "fused_c64_k2"}}
    d = x["noisy_dm14"]
    kern = {k["kernel"]: k["GBps"] for k in d["kernels"]}
    s["dm14"] = {"plain_s": d["s_per_circuit"], "fused_s": d["fused_superop"]["s_per_circuit"],
                 "purity": d["purity"], "fused_max_z_diff": d["fused_superop"]["max_z_diff"],
                 "kernel_GBps": kern, "channel_passes_GBps": d["channel_passes_GBps"],
                 "fused_kernel_GBps": {k["kernel"]: k["GBps"] for k in d["fused_superop"]["kernels"]},
                 "n12_layer_vs_oracle": d["n12_layer_vs_oracle"]["max_abs_diff"]}
    q = x["qft20"]
    s["qft20"] = {k: q[k] for k in ("s_per_circuit_plain", "s_per_circuit_tiled", "cpu_s_per_circuit",
                                    "max_abs_diff_vs_oracle")}
    t = x.get("tn20")
    if t:
        s["tn20"] = {k: t[k] for k in ("s_gpu", "s_cpu_numpy", "max_abs_diff_vs_state_vector")}
    return sig(s, 4)


def uneven_batch(Y, count=2048, seed=4096):
    """`count` circuits, n ~ U{10..20}, depth ~ U{10..50} layers of the
    layered-circuit layer type (circuit (n, d) is the first d layers of the
    n-qubit layered circuit, so equal draws share one Circuit)."""
    rng = np.random.default_rng(seed)
    draws = [(int(rng.integers(10, 21)), int(rng.integers(10, 51))) for _ in range(count)]
    layers, built = {}, {}
    for n, d in sorted(set(draws)):
        els = []
        for l in range(d):
            if (n, l) not in layers:
                layers[(n, l)] = layer_elements(Y, n, l)
            els += layers[(n, l)]
        built[(n, d)] = Y.Circuit.qubits(n, els)
    return draws, [built[x] for x in draws]


def batch_extra(Y, A, torch, stream, dev, timed):
    """2048 uneven circuits from |0...0>: the PLAIN per-circuit loop (FP64,
    the reference result) against one persistent launch per form: TILED
    complex128 (bit-exact), FUSED complex128 and FUSED complex64 with split
    coefficients (1 - F and max |error| against the PLAIN states)."""
    t0 = time.perf_counter()
    draws, circuits = uneven_batch(Y)
    build_s = time.perf_counter() - t0
    gates = sum(len(c.elements) for c in circuits)
    amps = sum(1 << n for n, _ in draws)
    res = {"circuits": len(circuits), "gates": gates, "amplitudes": amps, "host_build_s": build_s}
    ref = [Y.ArrayReg.zero_state(n, device=dev) for n, _ in draws]
    res["s_plain"] = timed(lambda: Y.batch_apply(circuits, ref, Y.MODE_PLAIN))
    forms = {}
    for name, mode, prec, k in (("tiled_c128", Y.MODE_TILED, Y.C128, 0), ("fused_c128_auto", Y.MODE_FUSED, Y.C128, 0),
                                ("fused_c64_auto", Y.MODE_FUSED, Y.C64, 0), ("fused_c64_k2", Y.MODE_FUSED, Y.C64, 2)):
        # warm-up: the whole batch once (the batch autotuner runs here, and
        # the kept table buffers reach their size)
        warm = [Y.ArrayReg.zero_state(n, prec, device=dev) for n, _ in draws]
        Y.batch_apply(circuits, warm, mode, k)
        del warm
        regs = [Y.ArrayReg.zero_state(n, prec, device=dev) for n, _ in draws]
        t0 = time.perf_counter()
        t = timed(lambda: Y.batch_apply(circuits, regs, mode, k))
        wall = time.perf_counter() - t0
        worst_f = max(max(0.0, 1.0 - a.fidelity(b)) for a, b in zip(ref, regs))
        worst_e = max(a.max_abs_diff(b) for a, b in zip(ref, regs))
        forms[name] = {"s": t, "wall_s": wall, "speedup_vs_plain": res["s_plain"] / t,
                       "max_one_minus_fidelity": worst_f, "max_abs_err": worst_e}
        del regs
    res["forms"] = forms
    del ref
    # CPU: the oracle (single thread) on 16 of the circuits with n <= 16,
    # extrapolated to the batch by amplitude-gate updates
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    rng = np.random.default_rng(7)
    small = [i for i, (nq, _) in enumerate(draws) if nq <= 16]
    pick = sorted(rng.choice(small, size=min(16, len(small)), replace=False).tolist())
    t0 = time.perf_counter()
    for i in pick:
        z = np.zeros(1 << draws[i][0], complex)
        z[0] = 1
        O.apply_circuit(circuits[i], z)
    t_s = time.perf_counter() - t0
    work = lambda idx: sum(len(circuits[i].elements) * (1 << draws[i][0]) for i in idx)
    res["cpu_oracle_sample"] = {"circuits": len(pick), "s": t_s, "threads": 1,
                                "s_batch_extrapolated": t_s * work(range(len(circuits))) / work(pick)}
    return res


def vqe_batch_extra(Y, A, torch, stream, dev, timed):
    """4096 parameter sets of the 8-layer Ry.Rz + CNOT-ring ansatz at n=16
    with the TFIM energy and adjoint gradient in one batched sweep, against
    expect_grad called set by set (rate from the first 32 sets, which are
    also compared)."""
    n, layers, nsets = 16, 8, 4096
    rng = np.random.default_rng(16)
    sets = rng.uniform(-math.pi, math.pi, size=(nsets, 2 * n * layers))
    c = vqe_circuit(Y, n, layers, sets[0])
    op = tfim(Y, n)
    z = Y.ArrayReg.zero_state(n, device=dev)
    # set by set first (before the batched sweep's large stream-ordered
    # allocation), then the batch
    ns = 32
    Y.expect_grad(op, c, z)
    single = []
    t0 = time.perf_counter()
    for s in range(ns):
        c.dispatch(list(sets[s]))
        single.append(Y.expect_grad(op, c, z))
    ts = (time.perf_counter() - t0) / ns
    Y.expect_grad_batch(op, c, sets[:8], z)
    t0 = time.perf_counter()
    vals, grads = Y.expect_grad_batch(op, c, sets, z)
    tb = time.perf_counter() - t0
    err_v = max(abs(v - vals[s]) for s, (v, g) in enumerate(single))
    err_g = max(float(np.max(np.abs(np.array(g) - grads[s]))) for s, (v, g) in enumerate(single))
    # CPU: the oracle's expect_grad (single thread) on set 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    c.dispatch(list(sets[0]))
    z0 = np.zeros(1 << n, complex)
    z0[0] = 1
    t0 = time.perf_counter()
    vo, go = O.expect_grad(op, c, z0)
    t_cpu = time.perf_counter() - t0
    return {"qubits": n, "params": int(sets.shape[1]), "sets": nsets, "batched_grads_per_s": nsets / tb,
            "batched_s": tb, "single_grads_per_s": 1.0 / ts, "speedup": ts * nsets / tb,
            "max_energy_diff": err_v, "max_grad_diff": err_g, "cpu_oracle_s_per_grad": t_cpu,
            "max_grad_diff_vs_oracle": float(np.max(np.abs(np.asarray(go) - grads[0])))}


def qft_circuit(Y, n):
    els = []
    for i in range(n):
        els.append(Y.put([i], Y.Gate.H))
        for j in range(1, n - i):
            els.append(Y.control([i + j], [i], Y.Gate.Phase(2.0 * math.pi / float(1 << (j + 1)))))
    for i in range(n // 2):
        els.append(Y.put([i, n - 1 - i], Y.Gate.SWAP))
    return Y.Circuit.qubits(n, els)


def qft_extra(Y, A, torch, stream, dev, timed):
    """QFT on 20 qubits (220 gates) on a seeded Gaussian state: s/circuit of
    the PLAIN and TILED forms, and the oracle's CPU time for the same run."""
    n = 20
    rng = np.random.default_rng(20)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    c = qft_circuit(Y, n)
    res = {"qubits": n, "gates": len(c.elements)}
    for name, mode in (("plain", Y.MODE_PLAIN), ("tiled", Y.MODE_TILED)):
        r = Y.ArrayReg.from_vec(n, psi, device=dev)
        Y.apply_inplace(c, r, mode)
        r.set_state(psi)
        # one circuit per timing, median of 11: a call of about a millisecond
        # is exposed to the shared host's scheduling, which a mean would carry
        ts = sorted(timed(lambda: Y.apply_inplace(c, r, mode)) for _ in range(11))
        res[f"s_per_circuit_{name}"] = ts[5]
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    ref = O.apply_circuit(c, psi)
    res["cpu_s_per_circuit"] = time.perf_counter() - t0
    r = Y.ArrayReg.from_vec(n, psi, device=dev)
    Y.apply_inplace(c, r, Y.MODE_TILED)
    res["max_abs_diff_vs_oracle"] = float(np.max(np.abs(r.state_vec() - ref)))
    return res


def noisy_dm_circuit(Y, n, layers, seed=14):
    """Per layer: Ry, Rz on every qubit (U[0, 2 pi)), each followed by
    Depolarizing(1, 1e-3); CZ brickwork (2i, 2i+1) / (2i+1, 2i+2), each CZ
    followed by Depolarizing(2, 1e-3); AmplitudeDamping(1e-3) on every qubit."""
    rng = np.random.default_rng(seed)
    els = []
    for layer in range(layers):
        for q in range(n):
            for G in (Y.Gate.Ry, Y.Gate.Rz):
                els.append(Y.put([q], G(float(rng.uniform(0, 2 * math.pi)))))
                els.append(Y.channel([q], Y.NoiseChannel.Depolarizing(1, 1e-3)))
        for a in range(0 if layer % 2 == 0 else 1, n - 1, 2):
            els.append(Y.control([a], [a + 1], Y.Gate.Z))
            els.append(Y.channel([a, a + 1], Y.NoiseChannel.Depolarizing(2, 1e-3)))
        for q in range(n):
            els.append(Y.channel([q], Y.NoiseChannel.AmplitudeDamping(1e-3, 0.0)))
    return Y.Circuit.qubits(n, els)


def dm_extra(Y, A, torch, stream, dev, timed):
    """Noisy density matrix, n = 14 (4^14 complex128 = 4.3 GB), 20 layers:
    s/circuit, <Z_i> for every qubit and the purity; the oracle's CPU time
    for the same circuit at n = 8 (full run) stands beside it."""
    n, layers = 14, 20
    c = noisy_dm_circuit(Y, n, layers)
    d = Y.DensityMatrix.zero_state(n, device=dev)
    d.apply(noisy_dm_circuit(Y, n, 1, seed=99))  # warm-up
    del d
    d = Y.DensityMatrix.zero_state(n, device=dev)
    A.profile(True, dev)
    t = timed(lambda: d.apply(c))
    prof = A.profile_report(dev)
    A.profile(False, dev)
    zs = [Y.expect_dm(d, Y.OperatorPolynomial.single(i, Y.Op.Z, 1.0)).real for i in range(n)]
    chans = [p for p in prof if p["kernel"].startswith("dm_channel")]
    res = {"qubits": n, "layers": layers, "elements": len(c.elements), "s_per_circuit": t,
           "purity": d.purity(), "trace_re": d.trace().real, "z": zs,
           "kernels": [{"kernel": p["kernel"], "launches": p["launches"], "ms": round(p["ms"], 2),
                        "GBps": round(p["bytes"] / (p["ms"] / 1e3) / 1e9, 1)} for p in prof],
           # every channel pass together (Pauli-type, row-monomial and general kernels)
           "channel_passes_GBps": round(sum(p["bytes"] for p in chans) / (sum(p["ms"] for p in chans) / 1e3) / 1e9, 1)
           if chans else None}
    # FUSED form: rho as a 28-qubit vector through the fused tile passes,
    # channels as superoperators
    f = Y.DensityMatrix.zero_state(n, device=dev)
    f.apply(c, Y.MODE_FUSED)  # warm-up: the autotuner's choice is kept per circuit structure
    del f
    f = Y.DensityMatrix.zero_state(n, device=dev)
    A.profile(True, dev)
    tf = timed(lambda: f.apply(c, Y.MODE_FUSED))
    prof = A.profile_report(dev)
    A.profile(False, dev)
    zf = [Y.expect_dm(f, Y.OperatorPolynomial.single(i, Y.Op.Z, 1.0)).real for i in range(n)]
    res["fused_superop"] = {
        "s_per_circuit": tf, "speedup_vs_plain": t / tf,
        "max_z_diff": max(abs(a - b) for a, b in zip(zs, zf)), "purity_diff": abs(f.purity() - res["purity"]),
        "kernels": [{"kernel": p["kernel"], "launches": p["launches"], "ms": round(p["ms"], 2),
                     "GBps": round(p["bytes"] / (p["ms"] / 1e3) / 1e9, 1)} for p in prof]}
    del f
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    ns = 8
    cs = noisy_dm_circuit(Y, ns, layers)
    rho0 = np.zeros(1 << (2 * ns), complex)
    rho0[0] = 1
    t0 = time.perf_counter()
    ref = O.dm_apply_circuit(cs, rho0)
    res["cpu_s_per_circuit_n8"] = time.perf_counter() - t0
    g = Y.DensityMatrix.zero_state(ns, device=dev)
    g.apply(cs)
    res["n8_max_abs_diff_vs_oracle"] = float(np.max(np.abs(g.state_data() - ref)))
    # one layer at n = 10 on the CPU, scaled to n = 14 (4^4) and 20 layers
    ns = 10
    c1 = noisy_dm_circuit(Y, ns, 1)
    rho0 = np.zeros(1 << (2 * ns), complex)
    rho0[0] = 1
    t0 = time.perf_counter()
    O.dm_apply_circuit(c1, rho0)
    t1 = time.perf_counter() - t0
    res["cpu_s_one_layer_n10"] = t1
    res["cpu_s_per_circuit_n14_extrapolated"] = t1 * layers * 4 ** (n - ns)
    del d
    return res


if __name__ == "__main__":
    main()
