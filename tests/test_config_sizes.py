"""Parity at the benchmark configurations' full sizes.

- 24-qubit, 20-layer RX/RY/RZ + CX-ring sweep: the 23 <Z_i Z_(i+1)> values of
  the GPU (complex64 and complex128) against the reference's own plan
  (jaqsi/simulation.py:214-335, 500 entries) executed in float64 by the
  oracle's C restatement; 1e-5 (complex64) / 1e-10 (complex128).
- 20-qubit, 50-layer Rot + range-CX circuit, 3000 angles, sum Z_i Z_(i+1):
  the adjoint gradient (jaqsi/simulation.py:546-655) against central
  differences (h = 1e-4) of complex128 GPU forwards on 64 seeded angles;
  complex64 within 1e-5, complex128 within 1e-7 (the circuit is a degree-1
  trigonometric polynomial in each angle, so the central difference is
  f' sin(h)/h: 1.7e-9 |f'| truncation, ~1e-9 rounding).
- 12-qubit noisy density matrix, 20 layers, depolarizing + amplitude damping
  after every gate, sum <Z_i>: the expectation values against the reference's
  superoperator plan (_compile_mixed, :348-381) in float64 (C oracle), and the
  checkpointed reverse-pass gradient against central differences of
  complex128 GPU forwards on 16 seeded angles (same tolerances).
"""
import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import workloads as W
from oracle import cplan

pytestmark = pytest.mark.gpu

TOL = {torch.complex64: 1e-5, torch.complex128: 1e-10}
GRAD_TOL = {torch.complex64: 1e-5, torch.complex128: 1e-7}
H = 1e-4
_CACHE = {}


def _np(t):
    return t.detach().cpu().numpy()


def _sweep24():
    if "sweep24" not in _CACHE:
        n, layers = 24, 20
        ang = np.random.default_rng(2).uniform(0, 2 * np.pi, (layers, n, 3))
        plan = cplan.ReferencePlan(W.sweep_ansatz_records(n, layers, ang), n)
        assert plan.passes == 500
        st = plan.run(np.complex128)
        _CACHE["sweep24"] = (ang, plan.expval_z(st, W.zz_masks(n)))
    return _CACHE["sweep24"]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_sweep_24q_vs_fp64_reference_plan(dtype):
    n, layers = 24, 20
    ang, want = _sweep24()
    script = jq.Script(lambda a: W.sweep_ansatz(n, layers, a), n_qubits=n)
    got = _np(script.execute("expval", W.zz_chain(n), args=(torch.tensor(ang),), dtype=dtype))
    err = np.abs(got - want).max()
    print(f"24q sweep {dtype}: max |GPU - fp64 reference plan| = {err:.3e}")
    assert err <= TOL[dtype]


def _central_differences(script, obs, ang, idx, dtype=torch.complex128):
    """(f(x + h e_i) - f(x - h e_i)) / 2h of f = sum of the expectation values,
    for every flat index i in idx, as one batched GPU forward."""
    sets = np.repeat(ang[None], 2 * len(idx), axis=0)
    flat = sets.reshape(len(sets), -1)
    for k, i in enumerate(idx):
        flat[2 * k, i] += H
        flat[2 * k + 1, i] -= H
    out = script.execute("expval", obs, args=(torch.tensor(sets),), in_axes=(0,), dtype=dtype)
    f = _np(out).sum(axis=1)
    return (f[0::2] - f[1::2]) / (2 * H)


def test_adjoint_20q_3000_angles_vs_central_differences():
    n, layers = 20, 50
    ang = np.random.default_rng(3).uniform(0, 2 * np.pi, (layers, n, 3))
    script = jq.Script(lambda a: W.strongly_entangling(n, layers, a), n_qubits=n)
    obs = W.zz_chain(n)
    idx = W.sample_indices(np.random.default_rng(30), ang.shape, 64)
    fd = _central_differences(script, obs, ang, idx)
    for dtype in (torch.complex64, torch.complex128):
        a = torch.tensor(ang, requires_grad=True)
        script.execute("expval", obs, args=(a,), dtype=dtype).sum().backward()
        g = _np(a.grad).reshape(-1)[idx]
        err = np.abs(g - fd).max()
        print(f"20q adjoint {dtype}: max |adjoint - central difference| over {len(idx)} angles = {err:.3e}")
        assert err <= GRAD_TOL[dtype]


def _noisy12():
    if "noisy12" not in _CACHE:
        n, layers = 12, 20
        ang = np.random.default_rng(5).uniform(0, 2 * np.pi, (layers, n, 3))
        plan = cplan.ReferencePlan(W.noisy_ansatz_records(n, layers, ang), n, mixed=True)
        rho = plan.run(np.complex128)
        _CACHE["noisy12"] = (ang, plan.expval_z(rho, W.z_masks(n)))
    return _CACHE["noisy12"]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_noisy_dm_12q_vs_fp64_reference_plan(dtype):
    n, layers = 12, 20
    ang, want = _noisy12()
    script = jq.Script(lambda a: W.noisy_ansatz(n, layers, a), n_qubits=n)
    got = _np(script.execute("expval", W.z_each(n), args=(torch.tensor(ang),), dtype=dtype))
    err = np.abs(got - want).max()
    print(f"12q noisy density {dtype}: max |GPU - fp64 reference plan| = {err:.3e}")
    assert err <= TOL[dtype]


def test_noisy_dm_12q_gradient_vs_central_differences():
    n, layers = 12, 20
    ang, _ = _noisy12()
    script = jq.Script(lambda a: W.noisy_ansatz(n, layers, a), n_qubits=n)
    obs = W.z_each(n)
    idx = W.sample_indices(np.random.default_rng(50), ang.shape, 16)
    fd = _central_differences(script, obs, ang, idx)
    for dtype in (torch.complex64, torch.complex128):
        a = torch.tensor(ang, requires_grad=True)
        script.execute("expval", obs, args=(a,), dtype=dtype).sum().backward()
        g = _np(a.grad).reshape(-1)[idx]
        err = np.abs(g - fd).max()
        print(f"12q noisy density gradient {dtype}: max |reverse pass - central difference| = {err:.3e}")
        assert err <= GRAD_TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_30_qubits_largest_statevector(dtype):
    """The largest statevector (30 qubits: 8 GiB complex64, 16 GiB
    complex128; offsets past 2^32 bytes): a product state of RY then RZ on
    every wire, where <Z_i> = cos(a_i) and <Z_i Z_j> = cos(a_i) cos(a_j)
    exactly, and the gradient of sum_i <Z_i> is -sin(a_i); plus the state's
    norm through the probabilities of a CX chain appended (a permutation)."""
    n = 30
    free, total = torch.cuda.mem_get_info()
    need = (2 ** n) * (8 if dtype == torch.complex64 else 16) * 3
    if free < need:
        pytest.skip(f"needs {need / 2**30:.0f} GiB free on the device")
    rng = np.random.default_rng(30)
    a = rng.uniform(0, np.pi, n)
    b = rng.uniform(0, 2 * np.pi, n)

    def circuit(x, z):
        for w in range(n):
            jq.RY(x[w], wires=w)
            jq.RZ(z[w], wires=w)

    script = jq.Script(circuit, n_qubits=n)
    x = torch.tensor(a, requires_grad=True)
    pairs = [(0, 29), (3, 17), (28, 29), (0, 1)]
    obs = [jq.PauliZ(w) for w in range(n)] + [jq.build_parity_observable(list(p)) for p in pairs]
    ev = script.execute("expval", obs, args=(x, torch.tensor(b)), dtype=dtype)
    tol = 1e-5 if dtype == torch.complex64 else 1e-10
    want = np.concatenate([np.cos(a), [np.cos(a[i]) * np.cos(a[j]) for i, j in pairs]])
    np.testing.assert_allclose(ev.detach().cpu().numpy(), want, atol=tol)
    ev[:n].sum().backward()
    np.testing.assert_allclose(x.grad.numpy(), -np.sin(a), atol=tol * 10)
    del ev
    torch.cuda.empty_cache()

    def chained(x, z):
        circuit(x, z)
        for w in range(n - 1):
            jq.CX(wires=[w, w + 1])

    p = jq.Script(chained, n_qubits=n).execute("probs", args=(torch.tensor(a), torch.tensor(b)), dtype=dtype)
    s = float(p.double().sum())
    assert abs(s - 1.0) < (1e-4 if dtype == torch.complex64 else 1e-10), s
    del p
    torch.cuda.empty_cache()
