#!/usr/bin/env python
"""Benchmark of the jaqsi circuit-execution hot path on B200.

Headline workload (N=1): the 24-qubit forward gate sweep in complex64 — 20
layers of RX/RY/RZ on every wire plus a CX ring (i -> i+1 mod n), seeded
uniform angles in [0, 2pi), |0..0>, expectation values of Z_i Z_{i+1} for the
open chain i = 0..22.  One step = one forward sweep + measurement.

  value   gate-pass HBM GB/s achieved by the step, inputs resident in HBM:
          the algorithmic bytes of the kernels this implementation runs per
          step (each tile pass reads and writes the state once; the
          measurement reads it) over the measured step time.  The same
          definition is applied to the reference's plan in the reference arm
          (500 passes + one read per observable), so the two are the bytes each
          implementation moves per second.  `reference_plan_equiv_gbs` is the
          reference plan's bytes over our step time (a speed-up in GB/s form).
  roofline  the dominant kernel (the tile pass): its algorithmic bytes per
          launch over its average launch duration, against the measured HBM
          copy bandwidth.
  e2e     the same metric through the public API (Script.execute) with the
          angles in host memory and the expectation values copied back.
  cpu_baseline / --impl reference: the reference's full compiled plan (500
          passes) executed by the oracle's OpenMP C restatement on all host
          cores (jaqsi itself runs on JAX, which is not installed here).

The other configurations run as extra legs, each with its error against a
float64 reference (the C oracle's plan, NumPy oracle, or central differences),
its own roofline figures and a CPU number:
  sweep_24q_c128   the headline sweep in complex128
  small_10q        10 qubits c128, 5 layers, <Z_i>, forward + gradient
  adjoint_20q      20 qubits, 50 layers Rot + range-CX, 3000 angles, gradient
  batched_adjoint  4096 uneven instances, expval + gradient in one CUDA graph
  noisy_dm_12q     12-qubit noisy density matrix, gradient per parameter set

Multi-GPU: single circuits do not shard, so N GPUs run N replicas of the
sweep (weak scaling), timed as the max over ranks; the batched instances split
over ranks by cost.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "adjoint grads/sec (batched) vs plain GPU sim at ≤1e-5 err; gate-pass HBM GB/s"
N_QUBITS, LAYERS, SEED = 24, 20, 2
# DRAM bytes per launch of the specialised tile pass, from one ncu capture
# (--set full, 2 launches of the 24-qubit complex64 sweep): reads 134.25 MB
# (the whole state once) + writes 74.5 / 75.6 MB (the rest of the write-back
# is still in the 126 MB L2 when the launch ends).
TILE_PASS_TRAFFIC = {(24, "c64"): 209.3e6}
# Shared-memory bandwidth of one B200, nominal: 148 SMs x 128 B/clock x 1.965 GHz.
SMEM_NOMINAL_GBS = 148 * 128 * 1.965


def _z_reads(n_obs):
    """Reads of the state by the Z-string measurement: one per 32 words (n >= 9)."""
    return math.ceil(n_obs / 32)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _angles():
    return np.random.default_rng(SEED).uniform(0, 2 * np.pi, (LAYERS, N_QUBITS, 3))


def _records(ang):
    from jaqsi_b200 import workloads as W

    return W.sweep_ansatz_records(N_QUBITS, LAYERS, ang)


def _host():
    """Host cores available to this process and the CPU model / L3 (lscpu)."""
    info = {"cores": len(os.sched_getaffinity(0))}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            k, _, v = line.partition(":")
            if k.strip() in ("Model name", "L3 cache"):
                info[k.strip().lower().replace(" ", "_")] = v.strip()
    except Exception:
        pass
    return info


class Clocks:
    """SM clock and throttle-reason samples while timing: NVML read-only
    queries every 10 ms (pynvml), else nvidia-smi every 200 ms."""

    _NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []  # (sm_mhz, sm_max_mhz, {reason: active})
        self.source = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _nvml_sampler(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
        except Exception:
            return None

        def sample():
            sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
            r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
            return float(sm), float(mx), {n: bool(r & b) for n, b in zip(self._NAMES, bits)}

        try:
            sample()
        except Exception:
            pynvml.nvmlShutdown()
            return None
        self._nvml = pynvml
        return sample

    def _smi_sampler(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

        def sample():
            out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                 timeout=5).stdout.strip()
            v = [x.strip() for x in out.split(",")]
            num = lambda x: float(x) if x.replace(".", "").isdigit() else None
            return num(v[0]), num(v[1]), {n: v[2 + i] == "Active" for i, n in enumerate(self._NAMES) if len(v) > 2 + i}

        return sample

    def __enter__(self):
        sample = self._nvml_sampler()
        self.source, period = ("nvml", 0.01) if sample else ("nvidia-smi", 0.2)
        if sample is None:
            sample = self._smi_sampler()

        def run():
            while not self._stop.is_set():
                try:
                    self.rows.append(sample())
                except Exception:
                    pass
                self._stop.wait(period)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass
            self._nvml = None

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows if r[0] is not None]
        mx = [r[1] for r in self.rows if r[1] is not None]
        reasons = sorted({n for r in self.rows for n, on in r[2].items() if on})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "sm_min_mhz": min(sm) if sm else None, "reasons": reasons, "samples": len(self.rows),
                "source": self.source}


class RefSweep:
    """The reference's compiled plan of the 24-qubit sweep (500 entries:
    jaqsi/simulation.py:214-335) run by the oracle's OpenMP C restatement on
    all host cores, one full pass over the state per entry (_run, :400-409),
    then one read of the state per Z_i Z_(i+1) (measure_state's diagonal
    path, :777-801)."""

    def __init__(self):
        from jaqsi_b200 import workloads as W
        from oracle import cplan

        t0 = time.perf_counter()
        self.plan = cplan.ReferencePlan(_records(_angles()), N_QUBITS)
        self.build_s = time.perf_counter() - t0
        self.masks = W.zz_masks(N_QUBITS)
        self.threads = cplan.threads()
        self.bufs = {}

    def step(self, dtype: str):
        """(seconds, expectation values) of one full step in c64 or c128."""
        single = dtype == "c64"
        rt = np.float32 if single else np.float64
        if dtype not in self.bufs:
            self.bufs[dtype] = tuple(np.zeros(2 << N_QUBITS, dtype=rt) for _ in range(2))
        t0 = time.perf_counter()
        st = self.plan.run(np.complex64 if single else np.complex128, bufs=self.bufs[dtype])
        ev = self.plan.expval_z(st, self.masks)
        return time.perf_counter() - t0, ev

    def bytes_per_step(self, dtype: str) -> float:
        elem = 8 if dtype == "c64" else 16
        return (2 * self.plan.passes + len(self.masks)) * (1 << N_QUBITS) * elem


def reference_arm(args):
    """The reference's CPU implementation of the path, timed on this host:
    the full 500-entry plan every step (no sampling)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ref = RefSweep()
    for _ in range(args.warmup):
        ref.step(args.dtype)
    times = [ref.step(args.dtype)[0] for _ in range(args.steps)]
    step = statistics.median(times)
    value = ref.bytes_per_step(args.dtype) / step / 1e9
    sample = (f"the full reference plan every step: {ref.plan.passes} passes of the {N_QUBITS}-qubit {LAYERS}-layer "
              f"sweep + {len(ref.masks)} Z_iZ_(i+1) reads, {ref.threads} OpenMP threads, median of {args.steps}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic (seeded angles)",
        "config": _config(args, ref.plan.passes, None),
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": ref.threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "host": _host(),
    }
    print(json.dumps(line))
    return 0


def _config(args, p_ref, p_ours):
    return {
        "workload": f"forward gate sweep, {N_QUBITS}-qubit statevector, {LAYERS} layers of RX/RY/RZ on every "
                    f"wire + CX ring, expval of Z_iZ_(i+1) (open chain)",
        "n_qubits": N_QUBITS, "layers": LAYERS, "seed": SEED, "dtype": args.dtype,
        "reference_plan_passes": p_ref, "our_passes": p_ours,
        "unfused_passes": LAYERS * 4 * N_QUBITS,  # one pass per recorded gate
        "value_def": "algorithmic bytes of the step's kernels (2 x state bytes per pass + 1 x per measurement "
                     "read) / step time; the reference arm counts its own plan the same way",
        "l2": "flushed between timed steps (256 MiB write); state 128 MiB (c64) / 256 MiB (c128)",
        "parallelism": f"replicas x{args.gpus}",
    }


class Direct:
    """One plan run straight through the C ABI with preallocated buffers
    (device-only timing of forward / adjoint / checkpointed reverse)."""

    def __init__(self, plan, batch, dev, grad):
        import torch

        from jaqsi_b200 import _lib as L

        self.L, self.plan, self.batch = L, plan, batch
        self.grad = grad  # None, "adjoint" or "backward"
        self.state = torch.empty((batch, plan.state_elems), dtype=plan.cdtype, device=dev)
        self.out = torch.empty((batch, max(plan.n_obs, 1)), dtype=torch.float64, device=dev)
        self.ct = torch.ones((batch, max(plan.n_obs, 1)), dtype=torch.float64, device=dev)
        self.ga = torch.empty((batch, max(plan.n_angles, 1)), dtype=torch.float64, device=dev)
        mode = {None: 0, "adjoint": 1, "backward": 2}[grad]
        self.wsb = max(plan.workspace_bytes(batch, 0), plan.workspace_bytes(batch, mode))
        self.ws = torch.empty(max(self.wsb, 1), dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.current_stream()

    def forward(self, angles):
        vp = ctypes.c_void_p
        self.L.check(self.plan._lib.jq_forward(
            self.plan.handle, self.batch, vp(angles.data_ptr()), None, None, 0, self.L.JQ_OUT_EXPVAL,
            vp(self.state.data_ptr()), vp(self.out.data_ptr()), vp(self.ws.data_ptr()), self.wsb,
            vp(self.stream.cuda_stream)))

    def gradient(self, angles):
        vp = ctypes.c_void_p
        lib = self.plan._lib
        if self.grad == "adjoint":
            self.L.check(lib.jq_adjoint(
                self.plan.handle, self.batch, vp(angles.data_ptr()), None, vp(self.state.data_ptr()),
                self.L.JQ_OUT_EXPVAL, vp(self.ct.data_ptr()), None, vp(self.ga.data_ptr()), None, None,
                vp(self.ws.data_ptr()), self.wsb, vp(self.stream.cuda_stream)))
        else:
            self.L.check(lib.jq_backward(
                self.plan.handle, self.batch, vp(angles.data_ptr()), None, None, 0, self.L.JQ_OUT_EXPVAL,
                vp(self.ct.data_ptr()), None, vp(self.ga.data_ptr()), None, None,
                vp(self.ws.data_ptr()), self.wsb, vp(self.stream.cuda_stream)))

    def time_ms(self, fn, steps, warmup=2, flush=None):
        import torch

        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            if flush is not None:
                flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(self.stream)
            fn()
            b.record(self.stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)


def _event_ms(fn, steps, warmup=1, flush=None):
    """Median CUDA-event time of fn() on the current stream (host work
    between the events counts: used for the public-API timings)."""
    import torch

    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def l2_copy_gbs(dev):
    """Measured L2 copy bandwidth: a 16 MiB buffer copied back and forth (both
    copies stay in the 126 MB L2); bytes read + written per second."""
    import torch

    a = torch.empty(16 << 20, dtype=torch.uint8, device=dev)
    b = torch.empty_like(a)

    def run():
        for _ in range(50):
            b.copy_(a)
            a.copy_(b)

    ms = _event_ms(run, 5, warmup=2)
    return 100 * 2 * a.numel() / (ms * 1e-3) / 1e9


def _plan_for(script, args_, obs, dt, n):
    from jaqsi_b200 import _lib as L
    from jaqsi_b200 import simulation as sim

    tape = script.record(*args_)
    lw = sim.lower_tape(tape, n)
    specs, okey = sim._lower_obs(obs, n)
    mode = L.JQ_DENSITY if sim.has_noise(tape) else L.JQ_STATEVECTOR
    plan = sim.get_plan(lw, specs, okey, n, mode, dt)
    return plan, lw


def _central_differences(script, obs, ang, idx, h=1e-4):
    """Central differences of sum_o <O_o> w.r.t. the flat angle indices idx,
    complex128 forwards on the GPU in one batched call."""
    import torch

    sets = np.repeat(ang[None], 2 * len(idx), axis=0)
    flat = sets.reshape(len(sets), -1)
    for k, i in enumerate(idx):
        flat[2 * k, i] += h
        flat[2 * k + 1, i] -= h
    out = script.execute("expval", obs, args=(torch.tensor(sets),), in_axes=(0,), dtype=torch.complex128)
    f = out.detach().cpu().numpy().sum(axis=1)
    return (f[0::2] - f[1::2]) / (2 * h)

def _batched_oracle(shapes, angles, parts):
    """Float64 NumPy oracle (forward + adjoint) on one seeded instance per
    qubit count: the GPU gradients' error against it, and the oracle's time
    scaled to the whole workload (per qubit count, by depth)."""
    from jaqsi_b200 import workloads as W
    from oracle import sim_np as O

    rng = np.random.default_rng(41)
    by_n = {}
    for i, (n, d) in enumerate(shapes):
        by_n.setdefault(n, []).append(i)
    err = 0.0
    per_layer_s = {}
    for n in sorted(by_n):
        i = int(rng.choice(by_n[n]))
        d = shapes[i][1]
        t0 = time.perf_counter()
        ev, g = O.adjoint_grad(W.rot_ring_records(n, d, angles[i]), n, [("PauliZ", [0])])
        per_layer_s[n] = (time.perf_counter() - t0) / d
        err = max(err, float(np.abs(parts[i][1] - g).max()), float(np.abs(parts[i][0] - ev).max()))
    total_s = sum(per_layer_s[n] * d for n, d in shapes)
    return {
        "max_abs_err_vs_fp64_oracle": err,
        "cpu_baseline": {"grads_per_s": len(shapes) / total_s, "s_per_step": total_s, "cores": 1, "kind": "port",
                         "sample": f"NumPy float64 oracle forward + adjoint of one seeded instance per qubit count "
                                   f"({len(per_layer_s)} instances), time per layer scaled to every instance"},
    }


def batched_adjoint_leg(args, dev, steps, warmup, world=1, rank=0, max_over_ranks=None, barrier=None, cpu=False):
    """4096 uneven instances (qubits uniform 6..16, 10..40 layers of Rot on
    every wire + CX ring, independent seeded angles, <Z_0>): expectation value
    plus the full adjoint gradient of every instance in one CUDA-graph launch,
    against the plain per-circuit forward kernel driven by parameter shift
    (2 forwards per angle + 1, every shifted set of an instance in one batched
    forward call) on a seeded sample of the instances, scaled to the workload.
    With N ranks the instances split by estimated cost (no exchange); the
    time is the max over ranks and the rate counts every rank's instances."""
    import torch

    import jaqsi_b200 as jq
    from jaqsi_b200 import _lib as L
    from jaqsi_b200 import simulation as sim

    rng = np.random.default_rng(4)
    count = args.batch_instances
    qlo, qhi = args.batch_qubits
    shapes = [(int(rng.integers(qlo, qhi + 1)), int(rng.integers(10, 41))) for _ in range(count)]
    angles = [rng.uniform(0, 2 * np.pi, (d, n, 3)) for n, d in shapes]

    def record(n, d, ang):
        a = ang.tolist()
        with jq.recording() as tape:
            for l in range(d):
                for w in range(n):
                    jq.Rot(a[l][w][0], a[l][w][1], a[l][w][2], wires=w)
                for w in range(n):
                    jq.CX(wires=[w, (w + 1) % n])
        return tape

    from jaqsi_b200.shard import instance_cost, partition

    mine = partition([instance_cost(n, 2 * n * d) for n, d in shapes], world)[rank]
    t0 = time.perf_counter()
    tapes = {i: record(*shapes[i], angles[i]) for i in (mine if world > 1 else range(count))}
    obs = [jq.PauliZ(0)]
    t1 = time.perf_counter()
    bg = jq.BatchedGradients([(tapes[i], shapes[i][0], obs) for i in mine], dtype=torch.complex64)
    print(f"[bench] batched leg: record {t1 - t0:.1f} s, build {time.perf_counter() - t1:.1f} s", file=sys.stderr,
          flush=True)
    stream = torch.cuda.current_stream()
    for _ in range(max(1, warmup)):
        bg.run()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        if barrier:
            barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        bg.run()
        b.record(stream)
        b.synchronize()
        t = a.elapsed_time(b)
        ts.append(max_over_ranks(t) if max_over_ranks else t)
    ms = statistics.median(ts)
    summary = {
        "workload": f"{count} instances, qubits uniform {qlo}..{qhi}, 10..40 layers of Rot on every wire + CX ring, "
                    f"<Z_0>, complex64, seeded (numpy default_rng(4))",
        "grads_per_s": count / (ms * 1e-3), "ms_per_step": ms, "steps": steps,
        "classes": bg.classes, "config": bg.config, "gpu_launches_per_step": "1 CUDA graph",
        "sharding": f"cost-balanced split over {world} ranks, time = max over ranks" if world > 1 else "1 GPU",
    }
    # shared-memory traffic: every op sweeps the instance's state once forward
    # and three times in the adjoint (psi, lambda, the gradient read), each
    # sweep one read + one write of 2^n complex64 amplitudes
    smem_bytes = sum(4 * 2 * (1 << n) * 8 * (2 * n * d) for n, d in (shapes[i] for i in mine))
    smem_gbs = smem_bytes / (ms * 1e-3) / 1e9
    summary["roofline"] = {"achieved_smem_gbs": smem_gbs, "frac_smem_nominal": smem_gbs / SMEM_NOMINAL_GBS,
                           "bytes_def": "4 state sweeps (read + write) per op, shared memory; nominal 148 SMs x "
                                        "128 B/clock x 1.965 GHz"}
    if world > 1:
        return summary
    ev, grad = bg.run()
    grad64 = grad.detach().cpu().numpy().copy()
    parts = bg.split(ev.detach().cpu().numpy(), grad64)

    # parameter-shift baseline and gradient error on a seeded sample
    srng = np.random.default_rng(40)
    sample = sorted(srng.choice(count, size=min(args.shift_sample, count), replace=False).tolist())
    shift_ms = 0.0
    work_sample = 0
    work_total = sum(6 * n * d + 1 for n, d in shapes)
    max_err = 0.0
    ps_err = 0.0
    ref = jq.BatchedGradients([(tapes[i], shapes[i][0], obs) for i in sample], dtype=torch.complex128)
    _, g128 = ref.run()
    g128 = g128.detach().cpu().numpy()
    off = 0
    for k, i in enumerate(sample):
        n, d = shapes[i]
        na = 3 * n * d
        max_err = max(max_err, float(np.abs(parts[i][1] - g128[off: off + na]).max()))
        off += na
        lw = sim.lower_tape(tapes[i], n)
        specs, okey = sim._lower_obs(obs, n)
        plan = sim.get_plan(lw, specs, okey, n, L.JQ_STATEVECTOR, torch.complex64, {"jit": -1})
        base = torch.tensor([float(v) for v in lw.angles], dtype=torch.float64, device=dev)
        sets = base.repeat(2 * na + 1, 1)
        idx = torch.arange(na, device=dev)
        sets[1 + idx, idx] += np.pi / 2
        sets[1 + na + idx, idx] -= np.pi / 2
        nb = sets.shape[0]
        state = torch.empty((nb, plan.state_elems), dtype=torch.complex64, device=dev)
        out = torch.empty((nb, plan.n_obs), dtype=torch.float64, device=dev)
        wsb = plan.workspace_bytes(nb, 0)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
        vp = ctypes.c_void_p
        sp = vp(stream.cuda_stream)

        def fwd():
            L.check(plan._lib.jq_forward(plan.handle, nb, vp(sets.data_ptr()), None, None, 0, L.JQ_OUT_EXPVAL,
                                         vp(state.data_ptr()), vp(out.data_ptr()), vp(ws.data_ptr()), wsb, sp))
            # gradient = (f(+) - f(-)) / 2 per angle
            return (out[1: 1 + na, 0] - out[1 + na:, 0]) * 0.5

        fwd()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        gps = fwd()
        b.record(stream)
        b.synchronize()
        shift_ms += a.elapsed_time(b)
        work_sample += 2 * na + 1
        ps_err = max(ps_err, float(np.abs(gps.cpu().numpy() - g128[off - na: off]).max()))
        del state, ws
    shift_total_ms = shift_ms * work_total / max(work_sample, 1)
    oracle = _batched_oracle(shapes, angles, parts) if cpu else {}
    return {
        **oracle,
        **summary,
        "param_shift_grads_per_s": count / (shift_total_ms * 1e-3),
        "param_shift_ms_scaled": shift_total_ms,
        "param_shift_sample": f"{len(sample)} seeded instances timed (one batched jq_forward of the 2P+1 shifted "
                              f"sets each), scaled by forwards {work_total}/{work_sample}",
        "speedup_vs_param_shift": shift_total_ms / ms,
        "max_abs_grad_err_vs_c128": max_err,
        "param_shift_max_abs_grad_err_vs_c128": ps_err,
    }


def sweep_leg(args, dt_name, dev, steps, warmup, flush, max_over_ranks=lambda x: x, clocks=None, e2e=True):
    """The 24-qubit sweep in one dtype: device-timed step (jq_forward with the
    measurement) and sweep (jq_sweep, the tile passes alone), and the same
    step through Script.execute with host angles (e2e)."""
    import torch

    import jaqsi_b200 as jq
    from jaqsi_b200 import _lib as L
    from jaqsi_b200 import simulation as sim
    from jaqsi_b200 import workloads as W

    dt = torch.complex64 if dt_name == "c64" else torch.complex128
    elem = 8 if dt_name == "c64" else 16
    n = N_QUBITS
    ang_t = torch.tensor(_angles())
    script = jq.Script(lambda a: W.sweep_ansatz(n, LAYERS, a), n_qubits=n)
    obs = W.zz_chain(n)
    tune = {"tile_bits": args.tile_bits} if args.tile_bits else None
    lw = sim.lower_tape(script.record(ang_t), n)
    specs, okey = sim._lower_obs(obs, n)
    plan = sim.get_plan(lw, specs, okey, n, L.JQ_STATEVECTOR, dt, tune)
    P = plan.info["n_passes_fwd"]
    angles = sim.gather_angles(lw.angles, dev)
    d = Direct(plan, 1, dev, None)
    vp = ctypes.c_void_p

    def fwd():
        d.forward(angles)

    def sweep():
        L.check(plan._lib.jq_sweep(plan.handle, 1, vp(angles.data_ptr()), None, vp(d.state.data_ptr()),
                                   vp(d.ws.data_ptr()), d.wsb, vp(d.stream.cuda_stream)))

    t0 = time.perf_counter()
    for _ in range(warmup):
        fwd()
        sweep()
    torch.cuda.synchronize()
    warm_s = time.perf_counter() - t0
    if clocks is not None:
        clocks.__enter__()
    step_ms = max_over_ranks(d.time_ms(fwd, steps, 0, flush))
    sweep_ms = max_over_ranks(d.time_ms(sweep, steps, 0, flush))
    if clocks is not None:
        clocks.__exit__(None, None, None)
    fwd()
    ev = d.out[0, : plan.n_obs].detach().cpu().numpy().copy()
    e2e_ms = None
    if e2e:
        def e2e_step():
            if tune is None:
                res = script.execute("expval", obs, args=(ang_t,), dtype=dt)
            else:  # a non-default tile width is reachable only below Script
                with sim.gc_paused():
                    res = sim.simulate_and_measure(script.record(ang_t), n, "expval", obs, False, dtype=dt,
                                                   tune=tune)
            return res.cpu()

        e2e_ms = max_over_ranks(_event_ms(e2e_step, steps, warmup=max(1, warmup), flush=flush))
    S = 1 << n
    meas_reads = _z_reads(plan.n_obs)
    res = {
        "plan": plan, "P": P, "step_ms": step_ms, "sweep_ms": sweep_ms, "e2e_ms": e2e_ms, "expvals": ev,
        "bytes_step": (2 * P + meas_reads) * S * elem, "pass_bytes": 2 * S * elem, "meas_reads": meas_reads,
        "warm_s": warm_s, "n_obs": plan.n_obs, "n_angles": plan.n_angles, "elem": elem,
    }
    del d
    return res


def small_10q_leg(dev, steps, cpu):
    """10 qubits, complex128, 5 layers of RX/RY/RZ on every wire + CX ring,
    seeded angles, <Z_i> on every wire: forward + adjoint gradient per step
    through Script.execute and backward (a latency-bound case: 16 KiB state)."""
    import torch

    import jaqsi_b200 as jq
    from jaqsi_b200 import workloads as W

    n, layers = 10, 5
    ang = np.random.default_rng(1).uniform(0, 2 * np.pi, (layers, n, 3))
    a = torch.tensor(ang, requires_grad=True)
    script = jq.Script(lambda x: W.sweep_ansatz(n, layers, x), n_qubits=n)
    obs = W.z_each(n)

    def step():
        a.grad = None
        ev = script.execute("expval", obs, args=(a,), dtype=torch.complex128)
        ev.sum().backward()
        return ev

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
    ev = step().detach().cpu().numpy()
    grad = a.grad.detach().cpu().numpy().reshape(-1)
    out = {"workload": "10 qubits c128, 5 layers RX/RY/RZ + CX ring, <Z_i> on every wire, forward + gradient",
           "ms_per_step": statistics.median(ts),
           "timed": "host wall clock around Script.execute + backward + synchronize (launch/host bound)"}
    if cpu:
        from oracle import sim_np as O

        recs = W.sweep_ansatz_records(n, layers, ang)
        t0 = time.perf_counter()
        ev_ref, g_ref = O.adjoint_grad(recs, n, [("PauliZ", [i]) for i in range(n)])
        cpu_s = time.perf_counter() - t0
        out["max_abs_err_vs_fp64"] = {"expval": float(np.abs(ev - ev_ref).max()),
                                      "grad": float(np.abs(grad - g_ref).max())}
        out["cpu_baseline"] = {"ms_per_step": cpu_s * 1e3, "cores": 1, "kind": "port",
                               "sample": "NumPy float64 oracle, op-by-op forward + adjoint, the whole step"}
    return out


def adjoint_20q_leg(dev, steps, cpu, hbm_peak, l2_gbs):
    """20 qubits, 50 layers of Rot on every wire + CX(i, i + r mod n) with
    r = (layer mod 19) + 1, 3000 seeded angles, sum_i Z_i Z_(i+1): forward +
    adjoint gradient, through the public API and device-only."""
    import torch

    import jaqsi_b200 as jq
    from jaqsi_b200 import simulation as sim
    from jaqsi_b200 import workloads as W

    n, layers = 20, 50
    ang = np.random.default_rng(3).uniform(0, 2 * np.pi, (layers, n, 3))
    script = jq.Script(lambda x: W.strongly_entangling(n, layers, x), n_qubits=n)
    obs = W.zz_chain(n)
    idx = W.sample_indices(np.random.default_rng(30), ang.shape, 64)
    fd = _central_differences(script, obs, ang, idx)
    out = {"workload": "20 qubits, 50 layers Rot + CX range (layer mod 19)+1, 3000 angles, sum Z_iZ_(i+1)",
           "timed": "forward + adjoint: public API (Script.execute + backward) and device-only (jq_forward + "
                    "jq_adjoint)"}
    grads = {}
    for dt, name in ((torch.complex64, "c64"), (torch.complex128, "c128")):
        a = torch.tensor(ang, requires_grad=True)

        def step():
            a.grad = None
            ev = script.execute("expval", obs, args=(a,), dtype=dt)
            ev.sum().backward()

        ms = _event_ms(step, steps)
        grads[name] = a.grad.detach().cpu().numpy().reshape(-1).copy()
        plan, lw = _plan_for(script, (torch.tensor(ang),), obs, dt, n)
        angles = sim.gather_angles(lw.angles, dev)
        d = Direct(plan, 1, dev, "adjoint")
        dev_ms = d.time_ms(lambda: (d.forward(angles), d.gradient(angles)), steps)
        elem = 8 if name == "c64" else 16
        S = 1 << n
        pf, pa = plan.info["n_passes_fwd"], plan.info["n_passes_adj"]
        bytes_ = (2 * pf + _z_reads(plan.n_obs) + 2 + 4 * pa) * S * elem
        achieved = bytes_ / (dev_ms * 1e-3) / 1e9
        out[name] = {
            "ms_per_grad": ms, "grads_per_s": 1e3 / ms, "device_ms_per_grad": dev_ms,
            "passes_fwd": pf, "passes_adj": pa, "algorithmic_bytes": bytes_,
            "roofline": {"achieved": achieved, "unit": "GB/s", "frac_hbm": achieved / hbm_peak,
                         "frac_l2_copy": achieved / l2_gbs if l2_gbs else None,
                         "note": "state 8 MiB (c64) / 16 MiB (c128): L2-resident, so the HBM fraction can "
                                 "exceed 1"},
            "max_abs_grad_err_vs_central_fd": float(np.abs(grads[name][idx] - fd).max()),
        }
        del d
    out["fd_check"] = "central differences h=1e-4 of complex128 GPU forwards on 64 seeded angles"
    out["max_abs_grad_err_c64_vs_c128"] = float(np.abs(grads["c64"] - grads["c128"]).max())
    if cpu:
        from oracle import sim_np as O

        sample_layers = 2
        recs = W.strongly_entangling_records(n, sample_layers, ang)
        t0 = time.perf_counter()
        O.adjoint_grad(recs, n, [("Pauli", [i, i + 1], "ZZ") for i in range(n - 1)])
        cpu_s = (time.perf_counter() - t0) * layers / sample_layers
        out["cpu_baseline"] = {"ms_per_grad": cpu_s * 1e3, "grads_per_s": 1 / cpu_s, "cores": 1, "kind": "port",
                               "sample": f"NumPy float64 oracle forward + adjoint of the first {sample_layers} of "
                                         f"{layers} layers, scaled x{layers // sample_layers}"}
    return out


def noisy_dm_leg(dev, sets, steps, cpu, hbm_peak, world=1, max_over_ranks=None, dtypes=("c128", "c64")):
    """12-qubit density matrix, 20 layers of RX/RY/RZ on every wire + CX
    ring, DepolarizingChannel(0.01) then AmplitudeDamping(0.005) on every
    wire each gate touches, sum_i <Z_i>: forward + checkpointed reverse
    gradient of `sets` seeded parameter sets per step through
    Script.execute(in_axes=(0,)) and backward, complex128 and complex64.
    With N ranks the parameter sets split over the ranks (jaqsi_b200.shard:
    rows per rank, all-gather of the results, all-reduce of the gradients);
    the time is the max over ranks."""
    import contextlib

    import torch

    import jaqsi_b200 as jq
    from jaqsi_b200 import shard
    from jaqsi_b200 import simulation as sim
    from jaqsi_b200 import workloads as W

    n, layers = 12, 20
    ang = np.random.default_rng(5).uniform(0, 2 * np.pi, (sets, layers, n, 3))
    script = jq.Script(lambda x: W.noisy_ansatz(n, layers, x), n_qubits=n)
    obs = W.z_each(n)
    idx = W.sample_indices(np.random.default_rng(50), ang.shape[1:], 16)
    fd = _central_differences(script, obs, ang[0], idx)
    out = {"workload": f"12-qubit density matrix (4096 x 4096), 20 layers RX/RY/RZ + CX ring, depolarizing 0.01 + "
                       f"amplitude damping 0.005 after every gate, sum <Z_i>, {sets} parameter sets per step",
           "sharding": f"parameter sets split over {world} ranks, time = max over ranks" if world > 1 else "1 GPU",
           "timed": "forward + checkpointed reverse: public API (Script.execute(in_axes) + backward) and "
                    "device-only (jq_forward + jq_backward, one parameter set)"}
    evs = {}
    for dt, name in ((torch.complex128, "c128"), (torch.complex64, "c64")):
        if name not in dtypes:
            continue
        p = torch.tensor(ang, requires_grad=True)
        holder = {}

        def step():
            p.grad = None
            with shard.batch_sharding() if world > 1 else contextlib.nullcontext():
                ev = script.execute("expval", obs, args=(p,), in_axes=(0,), dtype=dt)
                ev.sum().backward()
            holder["ev"] = ev

        ms = _event_ms(step, steps, warmup=1)
        if max_over_ranks is not None:
            ms = max_over_ranks(ms)
        evs[name] = holder["ev"][0].detach().cpu().numpy().copy()
        g0 = p.grad[0].detach().cpu().numpy().reshape(-1)
        plan, lw = _plan_for(script, (torch.tensor(ang[0]),), obs, dt, n)
        angles = sim.gather_angles(lw.angles, dev)
        d = Direct(plan, 1, dev, "backward")
        dev_ms = d.time_ms(lambda: (d.forward(angles), d.gradient(angles)), max(2, steps), warmup=1)
        elem = 8 if name == "c64" else 16
        S = 4 ** n
        P = plan.info["n_passes_fwd"]
        s = math.ceil(math.sqrt(P))
        # forward, checkpoint writes, one recompute of the forward, and a reverse
        # pass reading rho and lambda and writing lambda per forward pass
        bytes_ = (2 * P + 1 + math.ceil(P / s) + 2 * P + 3 * P) * S * elem
        achieved = bytes_ / (dev_ms * 1e-3) / 1e9
        out[name] = {
            "ms_per_grad": ms / sets, "s_per_step": ms * 1e-3, "device_ms_per_grad": dev_ms, "passes_fwd": P,
            "algorithmic_bytes_per_grad": bytes_,
            "roofline": {"achieved": achieved, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "bytes_def": "2P (forward) + P/ceil(sqrt P) checkpoints + 2P (recompute) + 3P (reverse) "
                                      "state transfers"},
            "max_abs_grad_err_vs_central_fd": float(np.abs(g0[idx] - fd).max()),
        }
        del d
    out["fd_check"] = "central differences h=1e-4 of complex128 GPU forwards on 16 seeded angles of set 0"
    if cpu:
        from oracle import cplan

        t0 = time.perf_counter()
        rp = cplan.ReferencePlan(W.noisy_ansatz_records(n, layers, ang[0]), n, mixed=True)
        rho = rp.run(np.complex128)
        ev_ref = rp.expval_z(rho, W.z_masks(n))
        cpu_s = time.perf_counter() - t0
        out["max_abs_err_vs_fp64"] = {k: float(np.abs(v - ev_ref).max()) for k, v in evs.items()}
        out["cpu_baseline"] = {"s_per_step": cpu_s * sets, "s_per_set_forward": cpu_s, "cores": cplan.threads(),
                               "kind": "port", "passes": rp.passes,
                               "sample": f"the reference's superoperator plan ({rp.passes} passes, float64) forward "
                                         f"for parameter set 0, OpenMP C, scaled x{sets}; forward only (the "
                                         f"reference has no reverse pass for noisy circuits)"}
    return out


def ours_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from oracle import sim_np as O

    p_ref = O.jaqsi_pass_count(_records(_angles()))
    barrier()
    clk = Clocks(local)
    sw = sweep_leg(args, args.dtype, dev, args.steps, args.warmup, flush, max_over_ranks, clocks=clk)
    barrier()
    print(f"[bench] 24-qubit plan warm-up (incl. specialisation) {sw['warm_s']:.1f} s", file=sys.stderr, flush=True)
    P, elem = sw["P"], sw["elem"]
    S = 1 << N_QUBITS
    value = world * sw["bytes_step"] / (sw["step_ms"] * 1e-3) / 1e9
    e2e_value = world * sw["bytes_step"] / (sw["e2e_ms"] * 1e-3) / 1e9
    ref_bytes = (2 * p_ref + N_QUBITS - 1) * S * elem
    peak, peak_kind = _peaks()
    achieved = P * sw["pass_bytes"] / (sw["sweep_ms"] * 1e-3) / 1e9
    launches = (2 + P + sw["meas_reads"]) * args.steps
    result = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sw["step_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.dtype, "data": "synthetic (seeded angles, |0..0>)",
        "config": _config(args, p_ref, P),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TILE_PASS_TRAFFIC.get((N_QUBITS, args.dtype)),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch of the "
                                       "specialised tile pass (2 launches captured, averaged)",
                     "peak_kind": peak_kind,
                     "kernel": "jqk* (tile pass specialised per plan by NVRTC)",
                     "launches_per_step": P,
                     "avg_launch_us": sw["sweep_ms"] * 1e3 / P, "bytes_per_launch": sw["pass_bytes"]},
        "e2e": {"value": e2e_value, "unit": "GB/s", "ms_per_step": sw["e2e_ms"],
                "h2d_bytes_per_step": int(sw["n_angles"] * 8), "d2h_bytes_per_step": int(sw["n_obs"] * elem // 2)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "reference_plan_equiv_gbs": world * ref_bytes / (sw["step_ms"] * 1e-3) / 1e9,
        "reference_plan_equiv_def": f"the reference plan's bytes ({p_ref} passes + {N_QUBITS - 1} reads) / our step "
                                    f"time",
    }
    expvals = sw["expvals"]
    del sw
    legs_t0 = time.perf_counter()
    cpu = rank == 0 and world == 1 and not args.no_cpu
    if args.dtype == "c64" and not args.no_legs:
        s2 = sweep_leg(args, "c128", dev, args.steps, 1, flush, max_over_ranks)
        a2 = s2["P"] * s2["pass_bytes"] / (s2["sweep_ms"] * 1e-3) / 1e9
        result["sweep_24q_c128"] = {
            "ms_per_step": s2["step_ms"], "gbs": world * s2["bytes_step"] / (s2["step_ms"] * 1e-3) / 1e9,
            "e2e_ms_per_step": s2["e2e_ms"], "passes": s2["P"],
            "roofline": {"achieved": a2, "frac": a2 / peak, "avg_launch_us": s2["sweep_ms"] * 1e3 / s2["P"],
                         "bytes_per_launch": s2["pass_bytes"]},
        }
        expvals128 = s2["expvals"]
        del s2
    if not args.no_legs:
        l2 = l2_copy_gbs(dev)
        result["l2_copy_gbs_measured"] = l2
        if not args.no_batch:
            t0 = time.perf_counter()
            result["batched_adjoint"] = batched_adjoint_leg(args, dev, max(3, args.steps // 2), args.warmup, world,
                                                            rank, max_over_ranks, barrier, cpu=cpu)
            print(f"[bench] batched leg {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
        t0 = time.perf_counter()
        result["adjoint_20q"] = adjoint_20q_leg(dev, max(3, args.steps // 2), cpu, peak, l2)
        t1 = time.perf_counter()
        result["noisy_dm_12q"] = noisy_dm_leg(dev, args.dm_sets, 1, cpu, peak, world, max_over_ranks)
        t2 = time.perf_counter()
        result["small_10q"] = small_10q_leg(dev, max(5, args.steps), cpu)
        print(f"[bench] 20-qubit adjoint leg {t1 - t0:.1f} s, noisy density leg {t2 - t1:.1f} s",
              file=sys.stderr, flush=True)
    if cpu:
        t0 = time.perf_counter()
        ref = RefSweep()
        ref.step(args.dtype)
        ts = []
        for _ in range(3):
            t, _ = ref.step(args.dtype)
            ts.append(t)
        s = statistics.median(ts)
        _, ev64 = ref.step("c128")
        errs = {args.dtype: float(np.abs(expvals - ev64).max())}
        if args.dtype == "c64" and not args.no_legs:
            errs["c128"] = float(np.abs(expvals128 - ev64).max())
            result["sweep_24q_c128"]["max_abs_err_vs_fp64"] = errs["c128"]
        result["max_abs_err_vs_fp64"] = errs[args.dtype]
        result["fp64_reference"] = ("the reference's 500-entry plan executed in float64 by the oracle's C "
                                    "restatement; 23 <Z_iZ_(i+1)> values")
        result["cpu_baseline"] = {
            "value": ref.bytes_per_step(args.dtype) / s / 1e9, "unit": "GB/s", "cores": ref.threads, "kind": "port",
            "sample": f"the full reference plan ({ref.plan.passes} passes + {len(ref.masks)} reads), 1 warm-up + "
                      f"3 timed runs, median",
            "ms_per_step": s * 1e3, "host": _host(),
        }
        print(f"[bench] CPU reference runs {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
    print(f"[bench] extra legs {time.perf_counter() - legs_t0:.1f} s", file=sys.stderr, flush=True)
    if rank == 0:
        print(json.dumps(result, default=float))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dtype", default="c64", choices=["c64", "c128"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baselines and float64 checks")
    ap.add_argument("--tile-bits", type=int, default=0, help="override the forward tile size (qubits per CTA)")
    ap.add_argument("--no-legs", action="store_true", help="run only the headline 24-qubit sweep")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-adjoint leg")
    ap.add_argument("--batch-instances", type=int, default=4096)
    ap.add_argument("--batch-qubits", type=int, nargs=2, default=[6, 16], metavar=("LO", "HI"),
                    help="qubit range of the batched instances")
    ap.add_argument("--only-batch", action="store_true",
                    help="run only the batched-adjoint leg on one GPU and print its JSON (profiling runs)")
    ap.add_argument("--shift-sample", type=int, default=24,
                    help="instances whose parameter-shift baseline is timed and scaled")
    ap.add_argument("--dm-sets", type=int, default=64, help="parameter sets of the noisy density-matrix leg")
    ap.add_argument("--dm-dtypes", nargs="+", default=["c128", "c64"], choices=["c128", "c64"],
                    help="dtypes of the noisy density-matrix leg with --only-dm")
    ap.add_argument("--only-dm", action="store_true",
                    help="run only the noisy density-matrix leg on one GPU and print its JSON (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.only_batch:
        import torch

        torch.cuda.set_device(0)
        args.shift_sample = min(args.shift_sample, args.batch_instances)
        print(json.dumps(batched_adjoint_leg(args, torch.device("cuda", 0), args.steps, args.warmup)))
        return 0
    if args.only_dm:
        import torch

        torch.cuda.set_device(0)
        print(json.dumps(noisy_dm_leg(torch.device("cuda", 0), args.dm_sets, 1, not args.no_cpu, _peaks()[0],
                                      dtypes=args.dm_dtypes), default=float))
        return 0
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
