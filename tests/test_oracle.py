"""The CPU oracle against the reference's own known answers (no GPU needed).

The training trajectories come from tests/golden/reference_known_answers.json
(extracted from the reference's test source by tests/golden/make_golden.py);
every other expected value is copied from the reference's test suite (the
file:line is given per test) or is the analytic answer that test asserts.
"""
import json
import os

import numpy as np
import pytest

from oracle import sim_np as O

KNOWN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "reference_known_answers.json")))


def _value_and_grad_minimal(p):
    # RY(p0) w0, RY(p1) w1, CX(0,1); cost <Z0>  (jaqsi/tests/test_training.py:43-52)
    recs = [("RY", [0], [p[0]]), ("RY", [1], [p[1]]), ("CX", [0, 1], [])]
    ev, g = O.adjoint_grad(recs, 2, [("PauliZ", [0])])
    return ev[0], g


def test_training_minimal_trajectory():
    """jaqsi/tests/test_training.py:33-66 (rtol 1e-12)."""
    ka = KNOWN["minimal_training_loop"]
    losses, params = O.adam_trajectory(_value_and_grad_minimal, np.array([0.1, 0.2]), 0.05, 100)
    np.testing.assert_allclose(losses[24:100:25], ka["losses_24_100_25"], rtol=1e-12)
    np.testing.assert_allclose(params[0], ka["param0_final"], rtol=1e-12)
    np.testing.assert_allclose(params[1], ka["param1_final"], atol=1e-8)


def _value_and_grad_fit(w):
    # RX(x) w0, RY(w0) w0, CX(0,1), RY(w1) w1; mse of <Z0> to cos(x)
    # (jaqsi/tests/test_training.py:69-106)
    xs = np.linspace(0.0, np.pi, 16)
    ys = np.cos(xs)
    preds = np.zeros(16)
    grad = np.zeros(2)
    for i, x in enumerate(xs):
        recs = [("RX", [0], [x]), ("RY", [0], [w[0]]), ("CX", [0, 1], []), ("RY", [1], [w[1]])]
        ev, _ = O.adjoint_grad(recs, 2, [("PauliZ", [0])])
        preds[i] = ev[0]
        ct = [2.0 * (ev[0] - ys[i]) / 16]
        _, g = O.adjoint_grad(recs, 2, [("PauliZ", [0])], ct=ct)
        grad += g[1:3]
    return np.mean((preds - ys) ** 2), grad


def test_training_fit_trajectory():
    """jaqsi/tests/test_training.py:69-106 (rtol 1e-12, atol 1e-15)."""
    ka = KNOWN["fitting_data"]
    losses, weights = O.adam_trajectory(_value_and_grad_fit, np.array([0.1, 0.2]), 0.05, 100)
    np.testing.assert_allclose(losses[24:100:25], ka["losses_24_100_25"], rtol=1e-12, atol=1e-15)
    # weights[0] ~ -8.6e-4 accumulates 100 Adam steps of size ~lr whose late
    # gradients are O(1e-7) differences of O(1) numbers: merely reordering the
    # 16-sample gradient sum moves it by ~3e-15, so it is bounded absolutely
    # (2e-14, ~1e-16 of the O(1) quantities it is computed from) where the
    # reference's rtol=1e-12 would mean 9e-16.
    np.testing.assert_allclose(weights[0], ka["param0_final"], rtol=0, atol=2e-14)
    np.testing.assert_allclose(weights[1], ka["param1_final"], atol=1e-8)


BELL = [("H", [0], []), ("CX", [0, 1], [])]


def test_bell_and_ghz():
    """jaqsi/tests/test_jaqsi.py:364-434."""
    for ob in ("PauliX", "PauliZ"):
        np.testing.assert_allclose(O.execute(BELL, 2, "expval", [(ob, [0]), (ob, [1])]), [0, 0], atol=1e-10)
    np.testing.assert_allclose(O.execute(BELL, 2, "probs"), [0.5, 0, 0, 0.5], atol=1e-10)
    ghz3 = BELL + [("CX", [1, 2], [])]
    p = np.zeros(8)
    p[[0, 7]] = 0.5
    np.testing.assert_allclose(O.execute(ghz3, 3, "probs"), p, atol=1e-10)
    np.testing.assert_allclose(O.execute(ghz3, 3, "expval", [("PauliZ", [i]) for i in range(3)]), 0, atol=1e-10)
    ghz4 = ghz3 + [("CX", [2, 3], [])]
    p = np.zeros(16)
    p[[0, 15]] = 0.5
    np.testing.assert_allclose(O.execute(ghz4, 4, "probs"), p, atol=1e-10)
    toff = BELL + [("CCX", [0, 1, 2], [])]
    np.testing.assert_allclose(O.execute(toff, 3, "probs"), O.execute(ghz3, 3, "probs"), atol=1e-10)
    nonadj = [("H", [0], []), ("CX", [0, 2], [])]
    p = np.zeros(8)
    p[[0, 5]] = 0.5
    np.testing.assert_allclose(O.execute(nonadj, 3, "probs"), p, atol=1e-10)


def test_analytic_gradients():
    """-sin(theta) (test_jaqsi.py:136-146) and -0.8 sin(theta) through a
    BitFlip(0.1) (test_adjoint.py:179-192)."""
    ev, g = O.adjoint_grad([("RX", [0], [0.5])], 1, [("PauliZ", [0])])
    np.testing.assert_allclose(ev[0], np.cos(0.5), atol=1e-12)
    np.testing.assert_allclose(g[0], -np.sin(0.5), atol=1e-12)

    def f(t):
        return O.execute([("RX", [0], [t[0]]), ("BitFlip", [0], [0.1])], 1, "expval", [("PauliZ", [0])])[0]

    np.testing.assert_allclose(O.finite_difference(f, np.array([0.4]))[0], -0.8 * np.sin(0.4), atol=1e-8)


def _rx_density(theta):
    psi = np.array([np.cos(theta / 2), -1j * np.sin(theta / 2)])
    return np.outer(psi, psi.conj())


def _apply_kraus(rho, ks):
    return sum(k @ rho @ k.conj().T for k in ks)


@pytest.mark.parametrize(
    "name,kr,param",
    [
        ("BitFlip", lambda p: [np.sqrt(1 - p) * O.I2, np.sqrt(p) * O.X], 0.1),
        ("PhaseFlip", lambda p: [np.sqrt(1 - p) * O.I2, np.sqrt(p) * O.Z], 0.2),
        ("DepolarizingChannel",
         lambda p: [np.sqrt(1 - p) * O.I2, np.sqrt(p / 3) * O.X, np.sqrt(p / 3) * O.Y, np.sqrt(p / 3) * O.Z], 0.3),
        ("AmplitudeDamping", lambda g: [np.diag([1, np.sqrt(1 - g)]), np.array([[0, np.sqrt(g)], [0, 0]])], 0.25),
        ("PhaseDamping", lambda g: [np.diag([1, np.sqrt(1 - g)]), np.diag([0, np.sqrt(g)])], 0.35),
    ],
)
def test_kraus_textbook(name, kr, param):
    """Textbook Kraus densities (jaqsi/tests/test_jaqsi.py:118-132, 612-686)."""
    theta = 0.7
    rho = O.execute([("RX", [0], [theta]), (name, [0], [param])], 1, "density")
    np.testing.assert_allclose(rho, _apply_kraus(_rx_density(theta), kr(param)), atol=1e-12)


def test_thermal_relaxation_t2_le_t1():
    """Analytic T1/T2 decay (jaqsi/tests/test_jaqsi.py:689-711)."""
    pe, t1, t2, tg, theta = 0.0, 1e-4, 5e-5, 1e-6, 1.0
    rho = O.execute([("RX", [0], [theta]), ("ThermalRelaxationError", [0], [pe, t1, t2, tg])], 1, "density")
    r = _rx_density(theta)
    e1, e2 = np.exp(-tg / t1), np.exp(-tg / t2)
    ref = np.array([[1 - e1 * r[1, 1], e2 * r[0, 1]], [e2 * r[1, 0], e1 * r[1, 1]]])
    np.testing.assert_allclose(rho, ref, atol=1e-7)


def test_density_validity():
    """Trace, Hermiticity, purity of a noisy Bell state (test_jaqsi.py:727-760)."""
    recs = BELL + [("DepolarizingChannel", [0], [0.05]), ("DepolarizingChannel", [1], [0.05])]
    rho = O.execute(recs, 2, "density")
    assert abs(np.trace(rho) - 1) < 1e-10
    np.testing.assert_allclose(rho, rho.conj().T, atol=1e-10)
    purity = np.real(np.trace(rho @ rho))
    assert purity <= 1 + 1e-10 and purity < 1 - 1e-6


def test_adjoint_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 3
    th = rng.uniform(0, 2 * np.pi, 7)

    def recs(t):
        return [("H", [0], []), ("RX", [0], [t[0]]), ("RY", [1], [t[1]]), ("CX", [0, 1], []),
                ("CRX", [1, 2], [t[2]]), ("Rot", [2], [t[3], t[4], t[5]]), ("PauliRot", [0, 2], [t[6], "XY"])]

    obs = [("PauliZ", [0]), ("PauliX", [1]), ("Pauli", [0, 2], "ZZ")]
    ct = np.array([0.3, -1.1, 0.7])
    _, g = O.adjoint_grad(recs(th), n, obs, ct=ct)
    fd = O.finite_difference(lambda t: ct @ O.expval_state(O.simulate_pure(recs(t), n), n, obs), th)
    np.testing.assert_allclose(g, fd, atol=1e-8)


def test_reference_fusion_counts():
    """_fuse block wires (jaqsi/tests/test_adjoint.py:233-248) and the mixed
    block layout (jaqsi/tests/test_jaqsi.py:772-786)."""
    recs = [("Matrix", [0], [np.eye(2)]), ("Matrix", [1], [np.eye(2)]), ("Matrix", [0], [np.eye(2)]),
            ("Matrix", [0, 1], [np.eye(4)]), ("Matrix", [0], [np.eye(2)])]
    assert [w for w, _ in O.fuse(recs)] == [(0,), (1,), (0, 1), (0,)]
    recs = [("Matrix", [0, 1], [np.eye(4)]), ("Matrix", [1], [np.eye(2)]), ("Matrix", [0, 1], [np.eye(4)])]
    assert [w for w, _ in O.fuse(recs)] == [(0, 1), (1,), (0, 1)]
    noisy = [("H", [q], []) for q in range(3)] + [
        ("RZ", [0], [0.7]), ("DepolarizingChannel", [0], [0.05]), ("RX", [0], [0.35]), ("BitFlip", [0], [0.1]),
        ("CX", [1, 2], []), ("CX", [1, 2], []), ("CCX", [0, 1, 2], []), ("RY", [2], [0.7]),
        ("AmplitudeDamping", [2], [0.2])]
    assert O.jaqsi_mixed_pass_count(noisy, 3) == 7
    # the reference's layered plan: 4 gates, 1 permutation run, 1 diagonal run, 1 gate
    # (jaqsi/tests/test_gate_structure.py:119-124)
    layered = ([("H", [i], []) for i in range(4)] + [("RY", [i], [0.3]) for i in range(4)]
               + [("CX", [i, (i + 1) % 4], []) for i in range(4)] + [("RZ", [i], [0.2]) for i in range(4)]
               + [("SWAP", [1, 2], [])])
    assert O.jaqsi_pass_count(layered) == 7


def test_mixed_matches_pure_for_unitaries():
    rng = np.random.default_rng(3)
    recs = [("RX", [0], [0.3]), ("CRY", [0, 2], [1.1]), ("Rot", [1], [0.2, 0.5, 0.9]), ("CCX", [2, 0, 1], []),
            ("RZZ", [1, 2], [0.4])]
    psi = O.simulate_pure(recs, 3)
    rho = O.simulate_mixed(recs + [("Matrix", [0], [np.eye(2)])], 3)
    np.testing.assert_allclose(rho, np.outer(psi, psi.conj()), atol=1e-12)
    del rng


def _layered_records(n, layers, rng, noisy=False):
    from jaqsi_b200 import workloads as W

    ang = rng.uniform(0, 2 * np.pi, (layers, n, 3))
    recs = W.noisy_ansatz_records(n, layers, ang) if noisy else W.sweep_ansatz_records(n, layers, ang)
    if not noisy:
        recs += W.strongly_entangling_records(n, 2, ang)
        recs += [("CZ", [w, (w + 3) % n], []) for w in range(n)]
        recs += [("CRX", [0, n - 2], [0.3]), ("SWAP", [1, n - 1], []), ("RZ", [2], [0.7]), ("RZ", [2], [0.2])]
    else:
        recs += [("CCX", [0, 2, 1], []), ("CRY", [1, 3], [0.4]), ("PhaseDamping", [2], [0.2])]
    return recs


@pytest.mark.parametrize("noisy", [False, True])
def test_c_plan_runner_matches_numpy_oracle(noisy):
    """oracle/jqoracle.c runs the reference's compiled plan (statevector:
    dense / gather / diagonal entries; density: fused superoperators) and
    must give the op-by-op NumPy oracle's state, in float64 and float32."""
    from oracle import cplan

    n = 4 if noisy else 9
    recs = _layered_records(n, 3, np.random.default_rng(11), noisy)
    want = O.simulate_mixed(recs, n).reshape(-1) if noisy else O.simulate_pure(recs, n)
    plan = cplan.ReferencePlan(recs, n, mixed=noisy)
    if noisy:
        assert plan.passes == O.jaqsi_mixed_pass_count(recs, n)
    else:
        assert plan.passes == O.jaqsi_pass_count(recs)
        assert {e[0] for e in plan.entries} == {"dense", "gather", "diag"}
        numpy_maps = [e[1] for e in O.jaqsi_plan(recs, n) if e[0] == "gather"]
        c_maps = [e[1] for e in plan.entries if e[0] == "gather"]
        assert all((a == b).all() for a, b in zip(numpy_maps, c_maps))
    np.testing.assert_allclose(plan.run(np.complex128), want, atol=1e-12)
    np.testing.assert_allclose(plan.run(np.complex64), want, atol=2e-6)
    obs = [("PauliZ", [i]) for i in range(n)]
    zs = plan.expval_z(plan.run(np.complex128), cplan.z_masks(n))
    ref = O.expval_density(want.reshape(2**n, 2**n), n, obs) if noisy else O.expval_state(want, n, obs)
    np.testing.assert_allclose(zs, ref, atol=1e-12)
