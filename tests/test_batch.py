"""Batched uneven instances (jq_batch): expectation values and full adjoint
gradients of many independent circuits in one CUDA-graph launch, against the
oracle's per-instance adjoint gradient.  Instances span all four classes
(one per warp, one per CTA, one per thread-block cluster of 2-8 CTAs, batched
tile passes) by choosing the class thresholds explicitly.
"""
import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from oracle import sim_np as O
from tests.helpers import obs_records, random_circuit, to_records

pytestmark = pytest.mark.gpu

TOL = {torch.complex64: 1e-5, torch.complex128: 1e-10}


def _instances(seed, count, nmin, nmax, with_dense=True):
    rng = np.random.default_rng(seed)
    inst, refs = [], []
    for i in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        depth = int(rng.integers(3, 14))
        params = torch.tensor(rng.uniform(0, 2 * np.pi, 20 * depth + 10))
        with jq.recording() as tape:
            random_circuit(n, depth, np.random.default_rng(1000 + i), params, wide=False)
        obs = [jq.PauliZ(wires=int(rng.integers(n))), jq.PauliX(wires=int(rng.integers(n)))]
        if n >= 2:
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            obs.append(jq.build_parity_observable([a, b]))
            obs.append(jq.PauliY(wires=b))
        if with_dense and i % 7 == 3:
            h = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
            obs.append(jq.Hermitian((h + h.conj().T) / 2, wires=int(rng.integers(n)), record=False))
        inst.append((tape, n, obs))
        refs.append((to_records(tape), n, obs_records(obs)))
    return inst, refs


def _check(bg, refs, ct, tol):
    ev, g = bg.run()
    torch.cuda.synchronize()
    parts = bg.split(ev.cpu().numpy(), g.cpu().numpy())
    o = 0
    for (recs, n, obs), (e_i, g_i) in zip(refs, parts):
        c = ct[o: o + len(obs)]
        o += len(obs)
        ev_ref, g_ref = O.adjoint_grad(recs, n, obs, ct=c)
        np.testing.assert_allclose(e_i, ev_ref, atol=tol)
        np.testing.assert_allclose(g_i, g_ref, atol=tol * max(1.0, np.abs(c).sum()))


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_batch_all_classes_match_oracle(dtype):
    inst, refs = _instances(11, 36, 1, 14)
    bg = jq.BatchedGradients(inst, dtype=dtype,
                             config=dict(warp_max_qubits=5, cta_max_qubits=9, warp_threads=128, cta_threads=256,
                                         cluster_bits=3))
    cls = bg.classes
    assert cls["warp"] > 0 and cls["cta"] > 0 and cls["tile"] > 0 and cls["cluster"] > 0, cls
    ct = np.random.default_rng(5).normal(size=bg.n_obs_total)
    bg.set_cotangents(torch.tensor(ct))
    _check(bg, refs, ct, TOL[dtype])
    # replay of the captured graph, then new angles through the same graph
    _check(bg, refs, ct, TOL[dtype])
    rng = np.random.default_rng(9)
    new = rng.uniform(0, 2 * np.pi, bg.n_angles_total)
    bg.set_angles(torch.tensor(new))
    o = 0
    refs2 = []
    for tape, n, obs in inst:
        recs = to_records(tape)
        out = []
        for name, wires, params in recs:
            # every float parameter is an angle, in recording order
            k = sum(1 for p in params if isinstance(p, float))
            assert k == len(params), (name, params)
            newp = [float(v) for v in new[o: o + k]]
            o += k
            out.append((name, wires, newp))
        refs2.append((out, n, obs_records(obs)))
    _check(bg, refs2, ct, TOL[dtype])


def test_batch_default_config_and_autotune():
    inst, refs = _instances(12, 40, 2, 15, with_dense=False)
    bg = jq.BatchedGradients(inst, dtype=torch.complex64)
    ones = np.ones(bg.n_obs_total)
    _check(bg, refs, ones, 1e-5)
    chosen = bg.autotune()
    assert chosen == bg.config
    _check(bg, refs, ones, 1e-5)


def test_batch_warp_only_small_circuits():
    inst, refs = _instances(13, 64, 1, 6, with_dense=False)
    bg = jq.BatchedGradients(inst, dtype=torch.complex128,
                             config=dict(warp_max_qubits=6, cta_max_qubits=6, warp_threads=64, cta_threads=128))
    assert bg.classes == {"warp": 64, "cta": 0, "tile": 0, "cluster": 0}
    _check(bg, refs, np.ones(bg.n_obs_total), 1e-10)


def test_batch_cluster_class_all_cluster_sizes():
    """Rot + CX-ring instances at 11, 12 and 13 qubits with a 10-qubit CTA
    slice: clusters of 2, 4 and 8 CTAs, against the oracle.  64 threads per
    CTA takes the vectorised exchange for one-target blocks on rank bits
    (16 amplitudes a thread, complex64); 128 threads the general one."""
    rng = np.random.default_rng(21)
    inst, refs = [], []
    for i in range(18):
        n = 11 + i % 3
        d = int(rng.integers(2, 5))
        ang = rng.uniform(0, 2 * np.pi, (d, n, 3))
        with jq.recording() as tape:
            for l in range(d):
                for w in range(n):
                    jq.Rot(float(ang[l, w, 0]), float(ang[l, w, 1]), float(ang[l, w, 2]), wires=w)
                for w in range(n):
                    jq.CX(wires=[w, (w + 1) % n])
            jq.CRY(0.3 + 0.1 * i, wires=[0, n - 1])
            jq.RZZ(0.7, wires=[1, n - 2])
            jq.SWAP(wires=[0, 5])
        obs = [jq.PauliZ(0), jq.PauliX(1), jq.build_parity_observable([0, n - 1]), jq.PauliY(n - 1)]
        inst.append((tape, n, obs))
        refs.append((to_records(tape), n, obs_records(obs)))
    for dtype in (torch.complex64, torch.complex128):
        for threads in (64, 128):
            bg = jq.BatchedGradients(inst, dtype=dtype,
                                     config=dict(warp_max_qubits=0, cta_max_qubits=10, warp_threads=64,
                                                 cta_threads=threads, cluster_bits=3))
            assert bg.classes["cluster"] == 18, bg.classes
            _check(bg, refs, np.ones(bg.n_obs_total), TOL[dtype])


def test_batch_register_stage_cluster_random_gates():
    """Random circuits over the gate library (one- and two-target dense,
    diagonal and permutation blocks, controls on register and thread bits)
    at 11-13 qubits with a 10-qubit CTA slice and 64 threads a CTA: the
    complex64 cluster class then runs as register stages (16 amplitudes a
    thread), stages with rank bits exchanging through distributed shared
    memory.  Against the oracle, with cotangent weights."""
    rng = np.random.default_rng(31)
    inst, refs = [], []
    for i in range(15):
        n = 11 + i % 3
        params = torch.tensor(rng.uniform(0, 2 * np.pi, 400))
        with jq.recording() as tape:
            for w in range(n):
                jq.H(wires=w)
            random_circuit(n, 90, np.random.default_rng(3000 + i), params, wide=False)
            jq.CCX(wires=[n - 1, 0, 5])
            jq.CSWAP(wires=[1, n - 2, 3])
        obs = [jq.PauliZ(0), jq.PauliX(n - 1), jq.build_parity_observable([2, n - 3]), jq.PauliY(n // 2)]
        inst.append((tape, n, obs))
        refs.append((to_records(tape), n, obs_records(obs)))
    bg = jq.BatchedGradients(inst, dtype=torch.complex64,
                             config=dict(warp_max_qubits=0, cta_max_qubits=10, warp_threads=64, cta_threads=64,
                                         cluster_bits=3))
    assert bg.classes["cluster"] == 15, bg.classes
    ct = np.random.default_rng(6).normal(size=bg.n_obs_total)
    bg.set_cotangents(torch.tensor(ct))
    _check(bg, refs, ct, 1e-5)
    _check(bg, refs, ct, 1e-5)
