"""GPU parity: libjqsim (through Script / the C ABI) against the CPU oracle.

Tolerances: 1e-10 in complex128 and 1e-5 in complex64 against
the float64 oracle, for states, probabilities, densities, expectation values
and gradients.
"""
import json
import os

import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import simulation as sim
from oracle import sim_np as O
from tests.helpers import ansatz_layers, count_params, obs_records, random_circuit, to_records

pytestmark = pytest.mark.gpu
KNOWN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "reference_known_answers.json")))

TOL = {torch.complex64: 1e-5, torch.complex128: 1e-10}
DTYPES = [torch.complex64, torch.complex128]


def _np(t):
    return t.detach().cpu().resolve_conj().numpy()


def _obs_list(n, rng):
    obs = [jq.PauliZ(wires=int(rng.integers(n))), jq.PauliX(wires=int(rng.integers(n))),
           jq.PauliY(wires=int(rng.integers(n)))]
    if n >= 2:
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        obs.append(jq.build_parity_observable([a, b]))
        h = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
        obs.append(jq.Hermitian((h + h.conj().T) / 2, wires=[b, a], record=False))
    obs.append(jq.Hermitian(np.array([[0.25, 0.1 - 0.3j], [0.1 + 0.3j, -1.75]]), wires=int(rng.integers(n)),
                            record=False))
    return obs


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (5, 3), (8, 4), (11, 5)])
def test_forward_statevector(n, seed, dtype):
    rng = np.random.default_rng(seed)
    npar = count_params(n, 40, seed)
    params = torch.tensor(np.random.default_rng(100 + seed).uniform(0, 2 * np.pi, npar + 1))

    def circuit(p):
        random_circuit(n, 40, np.random.default_rng(seed), p)

    obs = _obs_list(n, rng)
    script = jq.Script(circuit, n_qubits=n)
    recs = to_records(script.record(params))
    psi = O.simulate_pure(recs, n)
    tol = TOL[dtype]
    np.testing.assert_allclose(_np(script.execute("state", args=(params,), dtype=dtype)), psi, atol=tol)
    np.testing.assert_allclose(_np(script.execute("probs", args=(params,), dtype=dtype)), np.abs(psi) ** 2, atol=tol)
    np.testing.assert_allclose(
        _np(script.execute("expval", obs, args=(params,), dtype=dtype)),
        O.expval_state(psi, n, obs_records(obs)), atol=tol)
    if n <= 8:
        np.testing.assert_allclose(_np(script.execute("density", args=(params,), dtype=dtype)),
                                   np.outer(psi, psi.conj()), atol=tol)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (5, 3)])
def test_forward_density(n, seed, dtype):
    rng = np.random.default_rng(seed)
    npar = count_params(n, 30, seed, channels=True)
    params = torch.tensor(np.random.default_rng(200 + seed).uniform(0, 2 * np.pi, npar + 1))

    def circuit(p):
        random_circuit(n, 30, np.random.default_rng(seed), p, channels=True)

    obs = _obs_list(n, rng)
    script = jq.Script(circuit, n_qubits=n)
    recs = to_records(script.record(params))
    rho = O.simulate_mixed(recs, n)
    tol = TOL[dtype]
    np.testing.assert_allclose(_np(script.execute("density", args=(params,), dtype=dtype)), rho, atol=tol)
    np.testing.assert_allclose(_np(script.execute("probs", args=(params,), dtype=dtype)), np.real(np.diag(rho)),
                               atol=tol)
    np.testing.assert_allclose(_np(script.execute("expval", obs, args=(params,), dtype=dtype)),
                               O.expval_density(rho, n, obs_records(obs)), atol=tol)
    with pytest.raises(ValueError, match="not defined for mixed"):
        script.execute("state", args=(params,), dtype=dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (6, 3), (9, 4)])
def test_adjoint_gradient(n, seed, dtype):
    rng = np.random.default_rng(seed)
    npar = count_params(n, 40, seed)
    base = np.random.default_rng(300 + seed).uniform(0, 2 * np.pi, npar + 1)
    params = torch.tensor(base, requires_grad=True)

    def circuit(p):
        random_circuit(n, 40, np.random.default_rng(seed), p)

    obs = _obs_list(n, rng)
    ct = rng.normal(size=len(obs))
    script = jq.Script(circuit, n_qubits=n)
    ev = script.execute("expval", obs, args=(params,), dtype=dtype)
    (ev.to(torch.float64) @ torch.tensor(ct, device=ev.device)).backward()
    recs = to_records(script.record(params.detach()))
    ev_ref, g_ref = O.adjoint_grad(recs, n, obs_records(obs), ct=ct)
    tol = TOL[dtype]
    np.testing.assert_allclose(_np(ev), ev_ref, atol=tol)
    g = _np(params.grad)[: len(g_ref)]
    np.testing.assert_allclose(g, g_ref, atol=tol * max(1.0, np.abs(ct).sum()))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("type", ["state", "probs", "density"])
def test_gradient_through_other_outputs(type, dtype):
    n, seed = 3, 7
    npar = count_params(n, 25, seed)
    base = np.random.default_rng(seed).uniform(0, 2 * np.pi, npar + 1)
    w = np.random.default_rng(8).normal(size=(2**n, 2**n)) + 1j * np.random.default_rng(9).normal(size=(2**n, 2**n))

    def circuit(p):
        random_circuit(n, 25, np.random.default_rng(seed), p)

    script = jq.Script(circuit, n_qubits=n)

    def f_ref(x):
        out = O.measure_state(O.simulate_pure(to_records(script.record(torch.tensor(x))), n), n, type)
        return float(np.real(np.sum(np.conj(w.reshape(out.shape) if type == "density" else w[0, : out.size]) * out)))

    params = torch.tensor(base, requires_grad=True)
    out = script.execute(type, args=(params,), dtype=dtype)
    wt = torch.tensor(w if type == "density" else w[0, : out.numel()], dtype=torch.complex128, device=out.device)
    torch.real(torch.sum(wt.conj() * out.to(torch.complex128))).backward()
    fd = O.finite_difference(f_ref, base, h=1e-6)
    np.testing.assert_allclose(_np(params.grad), fd, atol=max(TOL[dtype], 1e-7) * 100)


@pytest.mark.parametrize("dtype", DTYPES)
def test_density_gradient_checkpointed(dtype):
    """Noisy circuit: gradient by the checkpointed reverse pass vs central
    differences of the oracle (jaqsi falls back to plain autodiff here,
    jaqsi/simulation.py:715-720)."""
    n, seed = 3, 11
    npar = count_params(n, 30, seed, channels=True)
    base = np.random.default_rng(seed).uniform(0, 2 * np.pi, npar + 1)

    def circuit(p):
        random_circuit(n, 30, np.random.default_rng(seed), p, channels=True)

    obs = [jq.PauliZ(0), jq.PauliX(1), jq.build_parity_observable([0, 2])]
    script = jq.Script(circuit, n_qubits=n)
    params = torch.tensor(base, requires_grad=True)
    script.execute("expval", obs, args=(params,), dtype=dtype).sum().backward()

    def f(x):
        rho = O.simulate_mixed(to_records(script.record(torch.tensor(x))), n)
        return float(np.sum(O.expval_density(rho, n, obs_records(obs))))

    fd = O.finite_difference(f, base, h=1e-6)
    np.testing.assert_allclose(_np(params.grad), fd, atol=max(TOL[dtype] * 10, 1e-7))


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_reverse_pass_equals_generic(dtype):
    """The NVRTC-specialised checkpointed reverse pass (stage inputs kept in
    shared memory, in-register recompute inside a stage) against the generic
    reverse kernel, on an 8-qubit noisy circuit over the gate library with
    a Hermitian observable; angle and initial-state gradients."""
    n, seed = 8, 31
    npar = count_params(n, 70, seed, wide=True, channels=True)
    base = np.random.default_rng(seed).uniform(0, 2 * np.pi, npar + 1)
    init = np.random.default_rng(seed + 1).normal(size=2**n) + 1j * np.random.default_rng(seed + 2).normal(size=2**n)
    init /= np.linalg.norm(init)
    rng = np.random.default_rng(seed + 3)
    obs = _obs_list(n, rng)
    ct = rng.normal(size=len(obs))
    grads = []
    for jit in (1, -1):
        params = torch.tensor(base, requires_grad=True)
        psi0 = torch.tensor(init, dtype=dtype, device="cuda", requires_grad=True)
        with jq.recording() as tape:
            random_circuit(n, 70, np.random.default_rng(seed), params, wide=True, channels=True)
        ev = sim.simulate_and_measure(tape, n, "expval", obs, True, initial_state=psi0, dtype=dtype,
                                      tune={"jit": jit})
        (ev.to(torch.float64) @ torch.tensor(ct, device=ev.device)).backward()
        grads.append((_np(ev), _np(params.grad), _np(psi0.grad)))
    tol = TOL[dtype] * 10
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_allclose(a, b, atol=tol)


def test_bitflip_gradient_analytic():
    """-0.8 sin(theta) through BitFlip(0.1) (jaqsi/tests/test_adjoint.py:179-192)."""
    theta = torch.tensor(0.4, dtype=torch.float64, requires_grad=True)

    def circuit(t):
        jq.RX(t, wires=0)
        jq.BitFlip(0.1, wires=0)

    jq.Script(circuit, n_qubits=1).execute("expval", [jq.PauliZ(0)], args=(theta,))[0].backward()
    np.testing.assert_allclose(theta.grad.item(), -0.8 * np.sin(0.4), atol=1e-10)


def test_training_minimal_golden():
    """jaqsi/tests/test_training.py:33-66 through the GPU path (complex128)."""
    script = jq.Script(lambda p: (jq.RY(p[0], wires=0), jq.RY(p[1], wires=1), jq.CX(wires=[0, 1])), n_qubits=2)
    obs = [jq.PauliZ(wires=0)]

    def vg(p):
        t = torch.tensor(p, requires_grad=True)
        loss = script.execute("expval", obs, args=(t,))[0]
        loss.backward()
        return loss.item(), t.grad.numpy()

    ka = KNOWN["minimal_training_loop"]
    losses, params = O.adam_trajectory(vg, np.array([0.1, 0.2]), 0.05, 100)
    np.testing.assert_allclose(losses[24:100:25], ka["losses_24_100_25"], rtol=1e-12)
    np.testing.assert_allclose(params[0], ka["param0_final"], rtol=1e-12)
    np.testing.assert_allclose(params[1], ka["param1_final"], atol=1e-8)


def test_training_fit_golden():
    """jaqsi/tests/test_training.py:69-106: batched in_axes=(0, None) fit."""

    def model(x, w):
        jq.RX(x, wires=0)
        jq.RY(w[0], wires=0)
        jq.CX(wires=[0, 1])
        jq.RY(w[1], wires=1)

    script = jq.Script(model, n_qubits=2)
    obs = [jq.PauliZ(wires=0)]
    xs = torch.linspace(0.0, np.pi, 16, dtype=torch.float64)
    ys = torch.cos(xs)

    def vg(w):
        t = torch.tensor(w, requires_grad=True)
        pred = script.execute("expval", obs, args=(xs, t), in_axes=(0, None))[:, 0]
        loss = torch.mean((pred.cpu() - ys) ** 2)
        loss.backward()
        return loss.item(), t.grad.numpy()

    ka = KNOWN["fitting_data"]
    losses, weights = O.adam_trajectory(vg, np.array([0.1, 0.2]), 0.05, 100)
    np.testing.assert_allclose(losses[24:100:25], ka["losses_24_100_25"], rtol=1e-12, atol=1e-15)
    # bounded absolutely: see tests/test_oracle.py::test_training_fit_trajectory
    np.testing.assert_allclose(weights[0], ka["param0_final"], rtol=0, atol=2e-14)
    np.testing.assert_allclose(weights[1], ka["param1_final"], atol=1e-8)


@pytest.mark.parametrize("dtype", DTYPES)
def test_batched_matches_sequential(dtype):
    """in_axes batching equals per-sample execution (test_jaqsi.py:791-983),
    with batched and broadcast initial states (test_jaqsi.py:3053-3250)."""
    n = 3

    def circuit(x, w):
        jq.RX(x[0], wires=0)
        jq.RY(x[1], wires=1)
        jq.CRX(w[0], wires=[0, 2])
        jq.Rot(w[1], x[0], w[2], wires=2)
        jq.CX(wires=[2, 0])

    xs = torch.tensor(np.random.default_rng(0).uniform(0, 3, (5, 2)))
    w = torch.tensor([0.3, 0.8, -0.4])
    obs = [jq.PauliZ(0), jq.PauliY(2)]
    script = jq.Script(circuit, n_qubits=n)
    out = script.execute("expval", obs, args=(xs, w), in_axes=(0, None), dtype=dtype)
    seq = torch.stack([script.execute("expval", obs, args=(x, w), dtype=dtype) for x in xs])
    np.testing.assert_allclose(_np(out), _np(seq), atol=TOL[dtype])
    states = torch.tensor(np.random.default_rng(1).normal(size=(5, 8)) + 1j * np.random.default_rng(2).normal(size=(5, 8)))
    states = states / states.norm(dim=1, keepdim=True)
    outb = script.execute("probs", args=(xs, w), in_axes=(0, None), initial_state=states, dtype=dtype)
    for i in range(5):
        ref = O.measure_state(O.simulate_pure(to_records(script.record(xs[i], w)), n, _np(states[i])), n, "probs")
        np.testing.assert_allclose(_np(outb[i]), ref, atol=TOL[dtype])
    outc = script.execute("probs", args=(xs, w), in_axes=(0, None), initial_state=states[0], dtype=dtype)
    np.testing.assert_allclose(_np(outc[3]),
                               O.measure_state(O.simulate_pure(to_records(script.record(xs[3], w)), n, _np(states[0])),
                                               n, "probs"), atol=TOL[dtype])


def test_initial_state_gradient():
    """Cotangent of the initial state (jaqsi/tests/test_adjoint.py:121-135)."""
    n = 3
    psi0 = torch.arange(1, 2**n + 1, dtype=torch.float64).to(torch.complex128)
    psi0 = (psi0 / psi0.norm()).requires_grad_(True)
    p = torch.linspace(0.1, 1.9, 10, dtype=torch.float64)

    def circuit(p):
        jq.H(0)
        jq.RX(p[0], 0)
        jq.RY(p[1], 1)
        jq.CX([0, 1])
        jq.CRX(p[3], [1, 2])
        jq.Rot(p[4], p[5], p[6], 2)

    obs = [jq.PauliZ(0), jq.PauliX(1)]
    out = jq.Script(circuit, n).execute("expval", obs, args=(p,), initial_state=psi0)
    out.sum().backward()
    recs = to_records(jq.Script(circuit, n).record(p))
    base = _np(psi0.detach())

    def f(v):
        z = v[: 2**n] + 1j * v[2**n:]
        return float(np.sum(O.expval_state(O.simulate_pure(recs, n, z), n, obs_records(obs))))

    fd = O.finite_difference(f, np.concatenate([base.real, base.imag]))
    np.testing.assert_allclose(_np(psi0.grad), fd[: 2**n] + 1j * fd[2**n:], atol=1e-8)


def test_reference_state_cases():
    """Bell / GHZ / Toffoli / non-adjacent CX (jaqsi/tests/test_jaqsi.py:364-434)."""
    bell = jq.Script(lambda: (jq.H(0), jq.CX([0, 1])))
    np.testing.assert_allclose(_np(bell.execute("probs")), [0.5, 0, 0, 0.5], atol=1e-12)
    np.testing.assert_allclose(_np(bell.execute("expval", [jq.PauliX(0), jq.PauliX(1)])), [0, 0], atol=1e-12)
    ghz = jq.Script(lambda: (jq.H(0), jq.CX([0, 1]), jq.CCX([0, 1, 2])))
    p = np.zeros(8)
    p[[0, 7]] = 0.5
    np.testing.assert_allclose(_np(ghz.execute("probs")), p, atol=1e-12)
    na = jq.Script(lambda: (jq.H(0), jq.CX([0, 2])))
    p = np.zeros(8)
    p[[0, 5]] = 0.5
    np.testing.assert_allclose(_np(na.execute("probs")), p, atol=1e-12)
    t = torch.tensor(0.5, requires_grad=True, dtype=torch.float64)
    v = jq.Script(lambda th: jq.RX(th, 0)).execute("expval", [jq.PauliZ(0)], args=(t,))[0]
    v.backward()
    np.testing.assert_allclose([v.item(), t.grad.item()], [np.cos(0.5), -np.sin(0.5)], atol=1e-12)


@pytest.mark.parametrize(
    "factory",
    [
        lambda: jq.Id([3, 0]), lambda: jq.PauliX(3), lambda: jq.PauliZ(2), lambda: jq.S(0), lambda: jq.SWAP([3, 0]),
        lambda: jq.CX([3, 0]), lambda: jq.CY([0, 3]), lambda: jq.CZ([2, 0]), lambda: jq.CCX([3, 0, 2]),
        lambda: jq.CSWAP([2, 3, 0]), lambda: jq.RZ(0.4, 3), lambda: jq.RZZ(0.3, [3, 0]),
        lambda: jq.PauliRot(0.4, "ZIZ", [3, 1, 0]), lambda: jq.PauliRot(0.4, "XYZ", [3, 1, 0]),
        lambda: jq.ControlledPauliRot(0.4, "XY", [3, 0, 2]),
        lambda: jq.ControlledPauliRot(0.4, "Y", [3, 0, 2], n_controls=2),
        lambda: jq.ControlledPauliRot(0.4, "Z", [3, 0, 2], n_controls=2),
    ],
)
def test_isolated_gate_and_dagger(factory):
    """jaqsi/tests/test_gate_structure.py:154-184."""
    state = np.arange(1, 17) + 1j * np.arange(16, 0, -1)
    state = state / np.linalg.norm(state)
    with jq.recording():
        op = factory()
    for gate in (op, op.dagger()):
        out = jq.simulation.simulate_and_measure([gate], 4, "state", [], False, initial_state=torch.tensor(state))
        ref = O.apply_matrix(state, _np(gate.matrix), gate.wires, 4)
        np.testing.assert_allclose(_np(out), ref, atol=1e-12)


def test_unfused_schedule_matches_fused_at_24_qubits():
    """Full-size property check: the fused tile schedule and the one-pass-per-
    block schedule give the same 24-qubit state (complex64, 20 layers)."""
    n, layers = 24, 20
    ang = np.random.default_rng(2).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        ansatz_layers(n, layers, ang)
    obs = [jq.build_parity_observable([i, i + 1]) for i in range(n - 1)]
    a = sim.simulate_and_measure(tape, n, "expval", obs, False, dtype=torch.complex64)
    b = sim.simulate_and_measure(tape, n, "expval", obs, False, dtype=torch.complex64,
                                 tune={"no_fuse": 1, "jit": -1})
    c = sim.simulate_and_measure(tape, n, "expval", obs, False, dtype=torch.complex128)
    np.testing.assert_allclose(_np(a), _np(c), atol=1e-5)
    np.testing.assert_allclose(_np(b), _np(c), atol=1e-5)
    st = sim.simulate_and_measure(tape, n, "state", [], False, dtype=torch.complex64)
    assert abs(torch.linalg.vector_norm(st.to(torch.complex128)).item() - 1.0) < 1e-5


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_passes_match_oracle(dtype):
    """Per-plan NVRTC-specialised forward passes (auto for >= 2^16
    amplitudes) against the oracle on a random circuit over the gate library."""
    n, seed = 16, 21
    npar = count_params(n, 120, seed, wide=False)
    params = torch.tensor(np.random.default_rng(seed).uniform(0, 2 * np.pi, npar + 1))

    def circuit(p):
        random_circuit(n, 120, np.random.default_rng(seed), p, wide=False)

    script = jq.Script(circuit, n_qubits=n)
    psi = O.simulate_pure(to_records(script.record(params)), n)
    out = script.execute("state", args=(params,), dtype=dtype)
    np.testing.assert_allclose(_np(out), psi, atol=TOL[dtype])


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_equals_interpreter(dtype):
    """Same plan with and without NVRTC specialisation at 20 qubits."""
    n, layers = 20, 6
    ang = np.random.default_rng(5).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        ansatz_layers(n, layers, ang)
        jq.CRX(0.4, wires=[3, 17])
        jq.RZZ(0.7, wires=[19, 2])
        jq.ControlledPhaseShift(1.1, wires=[0, 18])
    a = sim.simulate_and_measure(tape, n, "state", [], False, dtype=dtype, tune={"jit": 1})
    b = sim.simulate_and_measure(tape, n, "state", [], False, dtype=dtype, tune={"jit": -1})
    np.testing.assert_allclose(_np(a), _np(b), atol=TOL[dtype])


def test_split_complex_stages_equal_interpreter(monkeypatch):
    """The optional split-complex register stages (JQ_JIT_SPLIT=1: pairs of
    amplitudes held as (re, re) / (im, im) lanes) against the interpreter,
    complex64, 20 qubits.  The distinct ckpt_stride keeps this plan out of
    the cache entries of the default specialisation."""
    n, layers = 20, 4
    ang = np.random.default_rng(9).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        ansatz_layers(n, layers, ang)
        jq.CRX(0.3, wires=[5, 14])
    monkeypatch.setenv("JQ_JIT_SPLIT", "1")
    a = sim.simulate_and_measure(tape, n, "state", [], False, dtype=torch.complex64,
                                 tune={"jit": 1, "ckpt_stride": 7})
    monkeypatch.delenv("JQ_JIT_SPLIT")
    b = sim.simulate_and_measure(tape, n, "state", [], False, dtype=torch.complex64, tune={"jit": -1})
    np.testing.assert_allclose(_np(a), _np(b), atol=TOL[torch.complex64])


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_adjoint_matches_oracle(dtype):
    """The NVRTC-specialised adjoint passes (the forward schedule run backwards,
    psi and lambda tiles in shared memory) against the oracle's adjoint
    gradient, for a random circuit over the gate library at 16 qubits."""
    n, seed = 16, 23
    rng = np.random.default_rng(seed)
    npar = count_params(n, 60, seed, wide=False)
    params = torch.tensor(np.random.default_rng(seed + 1).uniform(0, 2 * np.pi, npar + 1), requires_grad=True)

    def circuit(p):
        random_circuit(n, 60, np.random.default_rng(seed), p, wide=False)

    obs = _obs_list(n, rng)
    ct = rng.normal(size=len(obs))
    script = jq.Script(circuit, n_qubits=n)
    ev = script.execute("expval", obs, args=(params,), dtype=dtype)
    (ev.to(torch.float64) @ torch.tensor(ct, device=ev.device)).backward()
    ev_ref, g_ref = O.adjoint_grad(to_records(script.record(params.detach())), n, obs_records(obs), ct=ct)
    tol = TOL[dtype]
    np.testing.assert_allclose(_np(ev), ev_ref, atol=tol)
    np.testing.assert_allclose(_np(params.grad)[: len(g_ref)], g_ref, atol=tol * max(1.0, np.abs(ct).sum()))


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_adjoint_equals_interpreter(dtype):
    """Angle and initial-state gradients with and without NVRTC specialisation
    at 20 qubits (ansatz layers plus controlled and two-qubit rotations)."""
    n, layers = 20, 4
    ang0 = np.random.default_rng(6).uniform(0, 2 * np.pi, (layers, n, 3))
    init = np.random.default_rng(7).normal(size=2**n) + 1j * np.random.default_rng(8).normal(size=2**n)
    init /= np.linalg.norm(init)
    obs = [jq.build_parity_observable([i, i + 1]) for i in range(n - 1)] + [jq.PauliX(4), jq.PauliY(11)]
    grads = []
    for jit in (1, -1):
        ang = torch.tensor(ang0, requires_grad=True)
        x = torch.tensor(0.4, dtype=torch.float64, requires_grad=True)
        psi0 = torch.tensor(init, dtype=dtype, device="cuda", requires_grad=True)
        with jq.recording() as tape:
            ansatz_layers(n, layers, ang)
            jq.CRX(x, wires=[3, 17])
            jq.RZZ(0.7 * x, wires=[19, 2])
            jq.ControlledPhaseShift(1.1 * x, wires=[0, 18])
        ev = sim.simulate_and_measure(tape, n, "expval", obs, False, initial_state=psi0, dtype=dtype,
                                      tune={"jit": jit})
        ev.to(torch.float64).sum().backward()
        grads.append((_np(ev), _np(ang.grad), _np(x.grad), _np(psi0.grad)))
    tol = TOL[dtype]
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_allclose(a, b, atol=tol * 30)


def test_batch_beyond_grid_y_limit():
    """70,000 parameter sets in one call: the measurement and sampling kernels
    run instances along grid.y, at most 65,535 per launch."""
    import ctypes

    from jaqsi_b200 import _lib as L

    th = torch.linspace(0, 2 * np.pi, 70000, dtype=torch.float64)

    def pure(t):
        jq.RY(t, wires=0)
        jq.CX(wires=[0, 1])

    herm = jq.Hermitian(np.array([[0.5, 0.2], [0.2, -1.0]]), wires=1, record=False)
    ev = jq.Script(pure, n_qubits=2).execute("expval", [jq.PauliZ(1), herm], args=(th,), in_axes=(0,))
    c, s = np.cos(th.numpy() / 2) ** 2, np.sin(th.numpy() / 2) ** 2
    np.testing.assert_allclose(_np(ev[:, 0]), c - s, atol=1e-12)
    np.testing.assert_allclose(_np(ev[:, 1]), 0.5 * c - 1.0 * s, atol=1e-12)

    def noisy(t):
        jq.RX(t, wires=0)
        jq.AmplitudeDamping(0.25, wires=0)

    ev = jq.Script(noisy, n_qubits=1).execute("expval", [jq.PauliZ(0)], args=(th,), in_axes=(0,))
    p1 = 0.75 * np.sin(th.numpy() / 2) ** 2
    np.testing.assert_allclose(_np(ev[:, 0]), 1 - 2 * p1, atol=1e-12)

    # shot sampling straight through the C ABI: row r puts all mass on r mod 4
    batch, dim, shots = 70000, 4, 16
    probs = torch.zeros((batch, dim), dtype=torch.float64, device="cuda")
    probs[torch.arange(batch), torch.arange(batch) % dim] = 1.0
    counts = torch.empty((batch, dim), dtype=torch.int32, device="cuda")
    lib = L.lib()
    wsb = lib.jq_sample_workspace_bytes(batch, dim)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    vp = ctypes.c_void_p
    L.check(lib.jq_sample_shots(vp(probs.data_ptr()), batch, dim, shots, 7, vp(counts.data_ptr()), vp(ws.data_ptr()),
                                wsb, vp(torch.cuda.current_stream().cuda_stream)))
    want = torch.zeros_like(counts)
    want[torch.arange(batch), torch.arange(batch) % dim] = shots
    assert torch.equal(counts, want)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [9, 12])
def test_many_z_strings_one_read(n, dtype):
    """Z-string observables on n >= 9 qubits read the state once per 32 words
    (Walsh sums over 16 amplitudes a thread): 40 random words of weight 1..n,
    three batched parameter sets, against the oracle."""
    rng = np.random.default_rng(70 + n)
    words = []
    for _ in range(40):
        k = int(rng.integers(1, n + 1))
        words.append(sorted(int(w) for w in rng.choice(n, k, replace=False)))
    obs = [jq.PauliZ(wires=w[0]) if len(w) == 1 else jq.build_parity_observable(w) for w in words]
    npar = count_params(n, 60, n)
    params = torch.tensor(np.random.default_rng(7).uniform(0, 2 * np.pi, (3, npar + 1)))

    def circuit(p):
        for w in range(n):
            jq.H(wires=w)
        random_circuit(n, 60, np.random.default_rng(n), p)

    script = jq.Script(circuit, n_qubits=n)
    got = _np(script.execute("expval", obs, args=(params,), in_axes=(0,), dtype=dtype))
    for b in range(3):
        recs = to_records(script.record(params[b]))
        want = O.expval_state(O.simulate_pure(recs, n), n, obs_records(obs))
        np.testing.assert_allclose(got[b], want, atol=TOL[dtype])


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,tail", [(5, "affine"), (10, "affine"), (6, "toffoli")])
def test_trailing_permutations_absorbed_into_z_strings(n, tail, dtype):
    """Expectation-value plans absorb trailing X / CX / SWAP / constant
    diagonal blocks into their Z strings (jq_tune.expval_only): values and
    angle gradients against the oracle, which runs every gate.  A Toffoli
    (not affine) stops the absorption."""
    rng = np.random.default_rng(90 + n)
    npar = 3 * n
    base = rng.uniform(0, 2 * np.pi, npar)

    def circuit(p):
        for w in range(n):
            jq.Rot(p[3 * w], p[3 * w + 1], p[3 * w + 2], wires=w)
        for w in range(n):
            jq.CX(wires=[w, (w + 1) % n])
        if tail == "toffoli":
            jq.CCX(wires=[0, 1, 2])
        jq.PauliX(wires=1)
        jq.SWAP(wires=[0, n - 1])
        jq.CZ(wires=[1, 2])
        jq.S(wires=3)
        jq.CX(wires=[2, 4])

    obs = [jq.PauliZ(0), jq.build_parity_observable([1, 3]), jq.build_parity_observable(list(range(n))),
           jq.PauliZ(n - 1)]
    ct = rng.normal(size=len(obs))
    script = jq.Script(circuit, n_qubits=n)
    params = torch.tensor(base, requires_grad=True)
    ev = script.execute("expval", obs, args=(params,), dtype=dtype)
    (ev.to(torch.float64) @ torch.tensor(ct, device=ev.device)).backward()
    recs = to_records(script.record(torch.tensor(base)))
    ev_ref, g_ref = O.adjoint_grad(recs, n, obs_records(obs), ct=ct)
    np.testing.assert_allclose(_np(ev), ev_ref, atol=TOL[dtype])
    np.testing.assert_allclose(_np(params.grad), g_ref[:npar], atol=TOL[dtype] * max(1.0, np.abs(ct).sum()))
    # the same tape's state output runs every gate
    np.testing.assert_allclose(_np(script.execute("state", args=(params.detach(),), dtype=dtype)),
                               O.simulate_pure(recs, n), atol=TOL[dtype])


def test_absorbed_plan_measures_expectation_values_only():
    from jaqsi_b200 import _lib as L

    n = 4

    def circuit(p):
        jq.RY(p[0], wires=0)
        jq.CX(wires=[0, 1])
        jq.SWAP(wires=[1, 3])

    script = jq.Script(circuit, n_qubits=n)
    x = torch.tensor([0.4])
    lw = sim.lower_tape(script.record(x), n)
    specs, okey = sim._lower_obs([jq.PauliZ(3)], n)
    plan = sim.get_plan(lw, specs, okey, n, L.JQ_STATEVECTOR, torch.complex128)
    assert plan.info["n_blocks"] == 1  # CX and SWAP absorbed into the word
    ev = sim.run_plan(plan, L.JQ_OUT_EXPVAL, 1, sim.gather_angles(lw.angles, torch.device("cuda")), None, None, 0)
    np.testing.assert_allclose(_np(ev).ravel(), [np.cos(0.4)], atol=1e-12)
    with pytest.raises(ValueError, match="expectation values only"):
        sim.run_plan(plan, L.JQ_OUT_STATE, 1, sim.gather_angles(lw.angles, torch.device("cuda")), None, None, 0)
