"""The C ABI on CPU: exported symbols, struct layouts, the host planner's
schedules and its error behaviour.  No kernel is launched here."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import _lib as L
from jaqsi_b200 import simulation as sim
from oracle import sim_np as O
from tests.helpers import ansatz_layers, random_circuit, to_records

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "jqsim.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"JQ_API\s+[\w\s\*]+?\b(jq_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    declared = _declared()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(L.EXPORTED)
    out = subprocess.run(["nm", "-D", L.LIB_PATH], capture_output=True, text=True, check=True).stdout
    for name in declared:
        assert re.search(rf"\bT {name}\b", out), name


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "jqsim.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(jq_op), sizeof(jq_obs), sizeof(jq_tune),"
        " sizeof(jq_plan_info), offsetof(jq_op, const_mat), offsetof(jq_obs, mat), sizeof(jq_batch_config));"
        "return 0;}\n"
    )
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(L.JqOp), ctypes.sizeof(L.JqObs), ctypes.sizeof(L.JqTune), ctypes.sizeof(L.JqPlanInfo),
            L.JqOp.const_mat.offset, L.JqObs.mat.offset, ctypes.sizeof(L.JqBatchConfig)]
    assert got == want


def _plan(tape, n, obs=(), mode=L.JQ_STATEVECTOR, dtype=torch.complex128, tune=None):
    lw = sim.lower_tape(tape, n)
    specs, _ = sim._lower_obs(list(obs), n)
    return sim.Plan(lw.statics, specs, n, mode, dtype, tune)


def _schedule(plan, which):
    nb = plan.info["n_blocks"]
    bp = (ctypes.c_int32 * max(nb, 1))()
    bw = (ctypes.c_int32 * max(6 * nb, 1))()
    L.check(plan._lib.jq_plan_block_passes(plan.handle, which, bp, bw, nb))
    wires = [[w for w in bw[6 * b: 6 * b + 6] if w >= 0] for b in range(nb)]
    return list(bp[:nb]), wires


@pytest.mark.parametrize("which", [0, 1, 2])
@pytest.mark.parametrize("n,seed", [(5, 0), (9, 1), (16, 2)])
def test_schedule_respects_dependencies(n, seed, which):
    """Every block is in exactly one pass, and blocks sharing a wire run in
    program order (same pass: order kept inside the pass)."""
    rng = np.random.default_rng(seed)
    params = torch.linspace(0.1, 3.0, 2000, dtype=torch.float64)
    with jq.recording() as tape:
        random_circuit(n, 150, rng, params)
    plan = _plan(tape, n)
    bp, wires = _schedule(plan, which)
    assert all(p >= 0 for p in bp)
    last = {}
    for b, ws in enumerate(wires):
        for w in ws:
            if w in last:
                assert bp[last[w]] <= bp[b], (b, w)
            last[w] = b
    if which == 2:
        assert len(set(bp)) == len(bp)


def test_config2_pass_counts():
    """24-qubit, 20-layer RX/RY/RZ + CX-ring sweep: jaqsi runs 500 passes
    (restated _fuse/_fuse_runs), the tile schedule far fewer."""
    n, layers = 24, 20
    ang = np.random.default_rng(2).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        ansatz_layers(n, layers, ang)
    assert O.jaqsi_pass_count(to_records(tape)) == 500
    for dt in (torch.complex64, torch.complex128):
        info = _plan(tape, n, dtype=dt).info
        assert info["n_blocks"] == 960
        assert info["n_passes_fwd"] <= 80
        assert info["n_tile_ops_fwd"] == 960


def test_mixed_lowering_block_count():
    """Density plans fuse gates with the channels on their wire, like
    _compile_mixed (jaqsi/simulation.py:348-381)."""
    n = 3
    with jq.recording() as tape:
        jq.RX(0.3, wires=0)
        jq.DepolarizingChannel(0.1, wires=0)
        jq.AmplitudeDamping(0.2, wires=0)
        jq.RY(0.4, wires=0)
        jq.CX(wires=[0, 1])
    info = _plan(tape, n, mode=L.JQ_DENSITY).info
    assert info["n_bits"] == 6
    # one fused superoperator on (0, 3) and the CX on ket and bra wires
    assert info["n_blocks"] == 3


def test_invalid_inputs_raise():
    with jq.recording() as tape:
        jq.RX(0.1, wires=3)
    with pytest.raises(ValueError):
        sim.lower_tape(tape, 2)
    with jq.recording() as tape:
        jq.BitFlip(0.1, wires=0)
    lw = sim.lower_tape(tape, 1)
    with pytest.raises(ValueError, match="noise channel"):
        sim.Plan(lw.statics, [], 1, L.JQ_STATEVECTOR, torch.complex128)
    with pytest.raises(ValueError):
        jq.CX(wires=[0, 0])
    with pytest.raises(ValueError):
        jq.RX(0.1, wires=[0, 1])
    with pytest.raises(ValueError, match="Unknown measurement type"):
        sim._check_type("nope", False)
    with pytest.raises(ValueError, match="not defined for mixed"):
        sim._check_type("state", True)


def test_no_gpu_fails_loudly(monkeypatch):
    """The product has no CPU fallback."""
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="CUDA"):
        jq.Script(lambda: jq.H(0), 1).execute("probs")


def test_pauli_detection():
    m = np.kron(O.Z, O.Y) * 2.0
    assert sim._detect_pauli(m) == (0b01, 0b11, 1, 2.0)
    assert sim._detect_pauli(O.HAD) is None
    specs, _ = sim._lower_obs([jq.build_parity_observable([0, 2]), jq.PauliX(1)], 3)
    assert specs[0][:5] == ("P", 0, 0b101, 0, 1.0)
    assert specs[1][:5] == ("P", 0b010, 0, 0, 1.0)


def test_view_gather_matches_stack_and_gradient():
    """Angles that are element views of one tensor are gathered with one index
    op; values and gradients equal the per-angle stack."""
    base = torch.tensor(np.random.default_rng(0).uniform(0, 6, (4, 3, 3)), requires_grad=True)

    def circuit(a):
        for l in range(4):
            for w in range(3):
                jq.Rot(a[l, w, 0], a[l, w, 1], a[l, w, 2], wires=w)
            jq.RX(0.25, wires=0)
            jq.CX(wires=[0, 2])

    tape = jq.Script(circuit, 3).record(base)
    lw = sim.lower_tape(tape, 3)
    fast = sim._view_gather(lw.angles, torch.device("cpu"))
    assert fast is not None
    ref = torch.stack([v.double().reshape(()) if isinstance(v, torch.Tensor) else torch.tensor(float(v),
                       dtype=torch.float64) for v in lw.angles])
    assert torch.equal(fast, ref)
    w = torch.randn(ref.shape, dtype=torch.float64)
    g1, = torch.autograd.grad((fast * w).sum(), base)
    g2, = torch.autograd.grad((ref * w).sum(), base)
    assert torch.allclose(g1, g2)
    # views of different tensors fall back to the stack
    other = torch.zeros(2, requires_grad=True)
    assert sim._view_gather([base[0, 0, 0], other[1]], torch.device("cpu")) is None


def test_class_lowering_matches_generic(monkeypatch):
    """The per-class lowering shortcut produces exactly what each op's own
    _jq_lower / _jq_static_key give (plan key, statics, angle order)."""
    rng = np.random.default_rng(11)
    params = torch.linspace(0.1, 3.0, 3000, dtype=torch.float64, requires_grad=True)
    with jq.recording() as tape:
        random_circuit(7, 400, rng, params, channels=True)
        jq.Barrier(wires=[0, 1])
        jq.RX(0.25, wires=2)  # float angle: no gradient
        jq.H(wires=0, matrix=np.eye(2))  # instance matrix: generic path
    fast = sim.lower_tape(tape, 7)
    monkeypatch.setattr(sim, "_CLASS_LOWERING", {})
    monkeypatch.setattr(sim, "_class_lowering", lambda cls: "skip" if issubclass(cls, jq.Barrier) else False)
    slow = sim.lower_tape(tape, 7)
    assert fast.key == slow.key
    assert len(fast.statics) == len(slow.statics) == len(tape) - 1
    for a, b in zip(fast.statics, slow.statics):
        for x, y in zip(a, b):
            if isinstance(x, np.ndarray) or isinstance(y, np.ndarray):
                np.testing.assert_array_equal(x, y)
            elif isinstance(x, list):
                assert len(x) == len(y) and all(np.array_equal(u, v) for u, v in zip(x, y))
            else:
                assert x == y
    assert len(fast.angles) == len(slow.angles)
    assert all(u is v for u, v in zip(fast.angles, slow.angles))
    assert fast.unitary == slow.unitary


def test_gc_paused_restores_collector_state(monkeypatch):
    """Script.execute pauses the cyclic collector only for the call, also when
    the call raises, and leaves a collector that was off switched off."""
    import gc

    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    assert gc.isenabled()
    seen = []

    def circuit():
        seen.append(gc.isenabled())
        jq.H(0)

    with pytest.raises(RuntimeError, match="CUDA"):
        jq.Script(circuit, 1).execute("probs")
    assert seen == [False] and gc.isenabled()
    gc.disable()
    try:
        with sim.gc_paused():
            assert not gc.isenabled()
        assert not gc.isenabled()
    finally:
        gc.enable()


def _jit_source(plan):
    n = plan._lib.jq_plan_jit_source(plan.handle, None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    plan._lib.jq_plan_jit_source(plan.handle, buf, n + 1)
    return buf.value.decode()


def test_direct_store_addresses_match_tile_layout():
    """Specialised passes whose last register stage stores straight to global
    memory (forward: gt, adjoint: gpos) must write every register slot where
    the shared-memory tile copy-out would have put it: global offset =
    deposit(unswizzle(shared-memory offset)).  Checked on the emitted source
    of a 20-qubit complex64 plan (no GPU needed)."""
    n, layers = 20, 4
    ang = np.random.default_rng(12).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        ansatz_layers(n, layers, ang)
    plan = _plan(tape, n, obs=[jq.PauliZ(0)], dtype=torch.complex64, tune={"jit": 1})
    src = _jit_source(plan)
    kernels = re.split(r'extern "C" __global__', src)[1:]
    assert kernels
    unswz = lambda a: a ^ (((a >> 4) ^ (a >> 8) ^ (a >> 12)) & 15)
    checked = {"fwd": 0, "adj": 0}
    for k in kernels:
        hb = [int(x) for x in re.search(r"const u32 hb\[\] = \{([^}]*)\}", k).group(1).split(",")]
        m = re.search(r"prefetch8t<\d+, \d+, (\d+)>", k) or re.search(r"tile copy: \d+ tile bits, the lowest (\d+)", k)
        cb = int(m.group(1))

        def gdep(logical):
            g = 0
            for i in range(cb + len(hb)):
                if (logical >> i) & 1:
                    g |= (1 << i) if i < cb else hb[i - cb]
            return g

        adj = "lam" in k.split("{", 1)[0]
        base = "gpos" if adj else "gt"
        gline = re.search(r"u32 %s = 0;(.*)" % base, k)
        if gline is None:
            assert "__stcs(g + " not in k and "__stcs(psi + " not in k
            continue
        tbs = re.findall(r"u32 tb(\d+) = 0;(.*)", k)
        # forward: the last stage stores; adjoint: stage 0 (run last)
        tb_line = tbs[0][1] if adj else tbs[-1][1]
        tbits = [int(x) for x in re.findall(r"\^= (\d+)u;", tb_line)]
        gbits = [int(x) for x in re.findall(r"\^= (\d+)u;", gline.group(1))]
        assert gbits == [gdep(unswz(t)) for t in tbits]
        loads = re.findall(r"float2 %s(\d+) = %s\[\w+ \^ (\d+)u\];" % (("p", "sp") if adj else ("v", "s")), k)
        nr = 1 << (max(int(j) for j, _ in loads).bit_length())
        off = [int(o) for _, o in loads[-nr:]]
        stores = [int(y) for y in re.findall(r"__stcs\(%s \+ \(%s \^ (\d+)u\)" % ("psi \\+ goff" if adj else "g", base), k)]
        assert stores == [gdep(unswz(o)) for o in off]
        checked["adj" if adj else "fwd"] += 1
    assert checked["fwd"] > 0 and checked["adj"] > 0
