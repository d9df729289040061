"""Pulse-level gates (jaqsi/evolution.py, jaqsi/operations.py:683-860).

CPU: the Hamiltonian algebra and its errors, and the oracle's Magnus schemes
against an independent adaptive ODE solve.
GPU: the batched Magnus kernel against the oracle's restatement of the same
scheme (1e-12), the closed form and the adaptive-solver requests against the
ODE solve, gradients w.r.t. pulse parameters against central differences,
and one launch per group of pending gates.
"""
import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from oracle import sim_np as O

X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]])
Z = np.diag([1.0, -1.0]).astype(complex)


def _np(t):
    return t.detach().cpu().numpy()


# coefficient functions written once for torch (the product) and numpy (the oracle)
def _drive(p, t):
    return p * (torch.sin(3 * t) if isinstance(t, torch.Tensor) else np.sin(3 * t))


def _ramp(p, t):
    return p[0] + p[1] * t


def _gauss(p, t):
    e = torch.exp if isinstance(t, torch.Tensor) else np.exp
    return p[0] * e(-((t - p[1]) ** 2) / 0.08)


def _herm(H, wires):
    return jq.Hermitian(H, wires=wires, record=False)


def test_hamiltonian_algebra_and_errors():
    h1 = _drive * _herm(X, 0)
    h2 = _ramp * _herm(Z, 0)
    s = h1 + h2
    assert s.n_terms == 2 and s.wires == [0]
    assert (h1 - h2).coeff_fns[1](np.array([1.0, 2.0]), 0.5) == pytest.approx(-2.0)
    with pytest.raises(ValueError):
        jq.ParametrizedHamiltonian([])
    with pytest.raises(ValueError):
        h1 + _ramp * _herm(Z, 1)
    with pytest.raises(ValueError):
        h1 + _ramp * _herm(np.kron(Z, Z), [0, 1])
    with pytest.raises(TypeError):
        _ = 3.0 * _herm(X, 0)
    with pytest.raises(ValueError):
        s.evolve(solver="rk4")
    with pytest.raises(ValueError):
        s.evolve()([0.1], 1.0)


def test_oracle_magnus_converges_to_the_ode_solution():
    fns, params = [lambda p, t: _drive(p, t), lambda p, t: _ramp(p, t)], [0.7, [0.2, 0.5]]
    ref = O.evolution_reference([X, Z], fns, params, 0.0, 1.5)
    assert np.abs(O.magnus_unitary([X, Z], fns, params, 0.0, 1.5, 256, 4) - ref).max() < 1e-10
    assert np.abs(O.magnus_unitary([X, Z], fns, params, 0.0, 1.5, 4000, 2) - ref).max() < 1e-7


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
CASES = {
    "1q": ([X, Z], [_drive, _ramp], [0.7, [0.2, 0.5]], [0]),
    "2q": ([np.kron(Z, Z), np.kron(X, np.eye(2)), np.kron(np.eye(2), Y)], [_ramp, _drive, _gauss],
           [[0.3, -0.4], 1.1, [0.9, 0.6]], [0, 1]),
    "3q": ([np.kron(np.kron(X, X), X), np.kron(np.kron(Z, np.eye(2)), Z)], [_drive, _ramp],
           [0.5, [0.1, 0.3]], [0, 1, 2]),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("solver,order", [("magnus2", 2), ("magnus4", 4)])
def test_magnus_kernel_matches_oracle(case, solver, order):
    H_mats, fns, params, wires = CASES[case]
    steps = 96
    ph = sum((f * _herm(H, wires) for f, H in zip(fns[1:], H_mats[1:])), fns[0] * _herm(H_mats[0], wires))
    T = [0.2, 1.4]
    with jq.recording() as tape:
        op = ph.evolve(solver=solver, magnus_steps=steps)(params, T)
    assert jq.resolve_pending(tape) == [1]
    want = O.magnus_unitary(H_mats, fns, params, T[0], T[1], steps, order)
    got = _np(op.matrix)
    np.testing.assert_allclose(got, want, atol=1e-12)
    np.testing.assert_allclose(got @ got.conj().T, np.eye(len(got)), atol=1e-12)


@pytest.mark.gpu
def test_adaptive_requests_match_the_ode_solution():
    # single term: closed form; several terms: fine-grid 4th-order Magnus
    single = _gauss * _herm(Y, 0)
    both = single + _drive * _herm(Z, 0)
    g1 = single.evolve()([[1.3, 0.4]], 0.9)
    g2 = both.evolve(solver="dopri5")([[1.3, 0.4], 0.8], 0.9)
    ref1 = O.evolution_reference([Y], [_gauss], [[1.3, 0.4]], 0.0, 0.9)
    ref2 = O.evolution_reference([Y, Z], [_gauss, _drive], [[1.3, 0.4], 0.8], 0.0, 0.9)
    np.testing.assert_allclose(_np(g1.matrix), ref1, atol=1e-10)
    np.testing.assert_allclose(_np(g2.matrix), ref2, atol=1e-9)


@pytest.mark.gpu
def test_pending_gates_solve_in_one_launch_per_group():
    ph = _drive * _herm(X, 0) + _ramp * _herm(Z, 0)
    gate = ph.evolve(solver="magnus4", magnus_steps=40)
    with jq.recording() as tape:
        for k in range(5):
            gate([0.1 * k, [0.3, -0.2 * k]], 1.0)
        (_gauss * _herm(Y, 0)).evolve(solver="magnus2", magnus_steps=30)([[0.5, 0.3]], 0.7)
    assert sorted(jq.resolve_pending(tape)) == [1, 5]
    for k, op in enumerate(tape[:5]):
        want = O.magnus_unitary([X, Z], [_drive, _ramp], [0.1 * k, [0.3, -0.2 * k]], 0.0, 1.0, 40, 4)
        np.testing.assert_allclose(_np(op.matrix), want, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["magnus4", "dopri8"])
def test_pulse_circuit_gradient_matches_central_differences(solver):
    """<Z0 Z1> of a circuit with a two-qubit pulse gate and a one-qubit drive,
    differentiated w.r.t. the pulse parameters through the kernel's reverse
    pass (or the closed form) and the circuit's adjoint."""
    zz = _ramp * _herm(np.kron(Z, Z), [0, 1]) + _drive * _herm(np.kron(X, np.eye(2)), [0, 1])
    g2 = zz.evolve(solver="magnus4", magnus_steps=64)
    g1 = (_gauss * _herm(X, 1)).evolve(solver=solver, magnus_steps=64)

    def circuit(p):
        jq.RY(0.3, wires=0)
        g2([p[0:2], p[2]], 1.2)
        g1([p[3:5]], 0.8)
        jq.RX(p[5], wires=0)

    script = jq.Script(circuit, n_qubits=2)
    obs = [jq.build_parity_observable([0, 1]), jq.PauliX(1)]
    x = torch.tensor([0.4, -0.7, 0.9, 1.1, 0.35, 0.2], dtype=torch.float64, requires_grad=True)
    script.execute("expval", obs, args=(x,)).sum().backward()
    h = 1e-5
    fd = []
    for i in range(len(x)):
        e = torch.zeros_like(x)
        e[i] = h
        fp = script.execute("expval", obs, args=(x.detach() + e,)).sum().item()
        fm = script.execute("expval", obs, args=(x.detach() - e,)).sum().item()
        fd.append((fp - fm) / (2 * h))
    np.testing.assert_allclose(_np(x.grad), fd, atol=1e-8)
