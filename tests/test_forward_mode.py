"""Forward-mode derivatives (torch.func.jvp / jacfwd) and torch.func.jacrev
through the simulation Function.

The reference routes jax.jvp / jax.jacfwd around its adjoint VJP and checks
them against jax.jacrev (jaqsi/tests/test_adjoint.py:136-150).  Here the jvp
rule forms J v from one batched reverse call, and jacrev batches the reverse
call over the stacked cotangents; both are checked against the plain
reverse-mode gradient.
"""
import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _rows_by_backward(f, x):
    """The Jacobian of f at x, one ordinary backward per output component."""
    y = f(x)
    rows = []
    for k in range(y.numel()):
        xx = x.detach().clone().requires_grad_(True)
        (g,) = torch.autograd.grad(f(xx).reshape(-1)[k], xx)
        rows.append(g.reshape(-1))
    return torch.stack(rows).reshape(tuple(y.shape) + tuple(x.shape))


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_jvp_and_jacfwd_match_reverse_mode(dtype):
    n, layers = 5, 2
    script = jq.Script(lambda a: W.strongly_entangling(n, layers, a), n_qubits=n)
    obs = W.zz_chain(n) + [jq.PauliX(1)]
    x = torch.tensor(np.random.default_rng(0).uniform(0, 2 * np.pi, (layers, n, 3)))

    def f(a):
        return script.execute("expval", obs, args=(a,), dtype=dtype).to(torch.float64)

    want = _rows_by_backward(f, x)
    tol = 1e-5 if dtype == torch.complex64 else 1e-10
    jf = torch.func.jacfwd(f)(x)
    np.testing.assert_allclose(_np(jf), _np(want), atol=tol)
    jr = torch.func.jacrev(f)(x)
    np.testing.assert_allclose(_np(jr), _np(want), atol=tol)
    v = torch.ones_like(x)
    _, tan = torch.func.jvp(f, (x,), (v,))
    np.testing.assert_allclose(_np(tan), _np(want.reshape(len(obs), -1).sum(1)), atol=tol * x.numel())


def test_jacfwd_of_probabilities_and_noisy_expectations():
    n = 3

    def pure(a):
        for w in range(n):
            jq.RY(a[w], wires=w)
        jq.CX(wires=[0, 2])
        jq.CRX(a[3], wires=[1, 0])

    def noisy(a):
        pure(a)
        jq.AmplitudeDamping(0.2, wires=1)
        jq.DepolarizingChannel(0.1, wires=2)

    x = torch.tensor([0.3, 1.2, -0.7, 0.9], dtype=torch.float64)
    fp = lambda a: jq.Script(pure, n_qubits=n).execute("probs", args=(a,))
    fn = lambda a: jq.Script(noisy, n_qubits=n).execute("expval", [jq.PauliZ(0), jq.PauliX(2)], args=(a,))
    for f in (fp, fn):
        np.testing.assert_allclose(_np(torch.func.jacfwd(f)(x)), _np(_rows_by_backward(f, x)), atol=1e-10)


def test_jvp_of_the_state_and_initial_state_tangent():
    n = 3
    psi0 = np.random.default_rng(1).normal(size=8) + 1j * np.random.default_rng(2).normal(size=8)
    psi0 = torch.tensor(psi0 / np.linalg.norm(psi0), dtype=torch.complex128, device="cuda")
    x = torch.tensor([0.4, -1.1], dtype=torch.float64)

    def circuit(a):
        jq.RX(a[0], wires=0)
        jq.CRY(a[1], wires=[0, 2])

    script = jq.Script(circuit, n_qubits=n)
    f = lambda a, s: script.execute("state", args=(a,), initial_state=s)
    va, vs = torch.tensor([0.5, -2.0], dtype=torch.float64), torch.randn(8, dtype=torch.complex128, device="cuda")
    out, tan = torch.func.jvp(f, (x, psi0), (va, vs))
    h = 1e-6
    fd = (f(x + h * va, psi0 + h * vs) - f(x - h * va, psi0 - h * vs)) / (2 * h)
    np.testing.assert_allclose(_np(tan), _np(fd), atol=1e-8)


# ---------------------------------------------------------------------------
# measure_density on the GPU (jaqsi/simulation.py:814-857)
# ---------------------------------------------------------------------------
def _random_rho(n, rng, batch=None):
    d = 2**n
    shape = (batch, d, d) if batch else (d, d)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    rho = a @ np.conj(np.swapaxes(a, -1, -2))
    return rho / np.trace(rho, axis1=-2, axis2=-1)[..., None, None]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_measure_density_matches_dense_reference(dtype):
    from jaqsi_b200 import simulation as sim
    from oracle import sim_np as O
    from tests.helpers import obs_records

    n = 4
    rng = np.random.default_rng(5)
    h = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    obs = [jq.PauliZ(0), jq.PauliX(2), jq.PauliY(3), jq.build_parity_observable([1, 3]),
           jq.Hermitian((h + h.conj().T) / 2, wires=[3, 0], record=False)]
    rho = _random_rho(n, rng, batch=3)
    tol = 1e-5 if dtype == torch.complex64 else 1e-12
    ev = sim.measure_density(torch.tensor(rho), n, "expval", obs, dtype=dtype)
    want = np.stack([O.expval_density(r, n, obs_records(obs)) for r in rho])
    np.testing.assert_allclose(_np(ev), want, atol=tol)
    pr = sim.measure_density(torch.tensor(rho[0]), n, "probs", [], dtype=dtype)
    np.testing.assert_allclose(_np(pr), np.real(np.diag(rho[0])), atol=tol)
    # gradient w.r.t. rho: d/dRe + i d/dIm of sum_o ct_o Re Tr(O_o rho) = sum_o ct_o O_o (Hermitian)
    ct = rng.normal(size=len(obs))
    r = torch.tensor(rho[1], dtype=torch.complex128, requires_grad=True)
    ev = sim.measure_density(r, n, "expval", obs, dtype=torch.complex128)
    (ev * torch.tensor(ct, device=ev.device)).sum().backward()
    lifted = sum(c * O.lifted(*O.obs_matrix(ob), n) for c, ob in zip(ct, obs_records(obs)))
    np.testing.assert_allclose(_np(r.grad), lifted, atol=1e-12)
