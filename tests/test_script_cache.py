"""Script's call-signature cache (the reference caches batched plans per
signature, jaqsi/script.py:695-705).

CPU: which circuits get a replay recipe (angles that are elements of the
argument tensors, or constants) and which fall back to recording every call
(value reads into Python, arithmetic on arguments, per-call matrices).
GPU: cached calls give the same results and gradients as uncached ones, for
eager and batched calls, and new argument values flow through the cache.
"""
import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import workloads as W
from jaqsi_b200.script import _NO_TRACE, _Trace


def _trace(script, args, kwargs=None, in_axes=None):
    kwargs = kwargs or {}
    key = script._trace_key("expval", args, kwargs, in_axes, None, None, None, None)
    assert key is not None
    return script._new_trace(key, args, kwargs)[1]


def test_recipe_of_indexed_arguments():
    n, layers = 6, 3
    ang = torch.tensor(np.random.default_rng(0).uniform(0, 2 * np.pi, (layers, n, 3)))
    tr = _trace(jq.Script(lambda a: W.sweep_ansatz(n, layers, a), n_qubits=n), (ang,))
    assert isinstance(tr, _Trace)
    assert tr.n_angles == ang.numel() and not tr.cpos
    assert torch.equal(tr.angles((ang,), torch.device("cpu")), ang.reshape(-1))
    new = ang + 1.0
    assert torch.equal(tr.angles((new,), torch.device("cpu")), new.reshape(-1))


def test_recipe_with_constants_and_several_arguments():
    def circuit(a, b, c):
        jq.RX(a[1], wires=0)
        jq.RY(0.7, wires=1)
        jq.Rot(b, a[0], c, wires=0)
        jq.CRX(b, wires=[0, 1])

    x, b = torch.tensor([0.3, 0.4]), torch.tensor(1.25)
    tr = _trace(jq.Script(circuit, n_qubits=2), (x, b, 0.5))
    assert isinstance(tr, _Trace)
    want = torch.tensor([0.4, 0.7, 1.25, 0.3, 0.5, 1.25], dtype=torch.float64)
    assert torch.allclose(tr.angles((x, b, 0.5), torch.device("cpu")), want)
    x2, b2 = torch.tensor([-1.0, 2.0]), torch.tensor(0.1)
    want2 = torch.tensor([2.0, 0.7, 0.1, -1.0, 0.5, 0.1], dtype=torch.float64)
    assert torch.allclose(tr.angles((x2, b2, 0.5), torch.device("cpu")), want2)


def test_recipe_batched_arguments():
    def circuit(a, b):
        jq.RX(a[1], wires=0)
        jq.RZ(b[0], wires=0)

    a = torch.tensor([[0.1, 0.2], [0.3, 0.4], [0.5, 0.6]])
    b = torch.tensor([0.9])
    sample = (a[0].contiguous(), b)
    tr = _trace(jq.Script(circuit, n_qubits=1), sample, in_axes=(0, None))
    assert isinstance(tr, _Trace)
    got = tr.angles((a, b), torch.device("cpu"), batch=3, in_axes=(0, None))
    want = torch.tensor([[0.2, 0.9], [0.4, 0.9], [0.6, 0.9]], dtype=torch.float64)
    assert torch.allclose(got, want.to(torch.float32).to(torch.float64))
    # batch axis 1
    at = a.t().contiguous()
    got = tr.angles((at, b), torch.device("cpu"), batch=3, in_axes=(1, None))
    assert torch.allclose(got, want.to(torch.float32).to(torch.float64))


@pytest.mark.parametrize("kind", ["branch", "float", "arithmetic", "item", "numpy"])
def test_value_dependent_circuits_are_not_cached(kind):
    def circuit(a):
        if kind == "branch":
            if a[0] > 0:
                jq.RX(a[1], wires=0)
        elif kind == "float":
            jq.RX(float(a[1]), wires=0)
        elif kind == "arithmetic":
            jq.RX(2 * a[1], wires=0)
        elif kind == "item":
            for _ in range(int(a[0].item() * 10)):
                jq.RY(a[1], wires=0)
        else:
            jq.RZ(np.sin(a[1]), wires=0)
        jq.RY(a[0], wires=0)

    assert _trace(jq.Script(circuit, n_qubits=1), (torch.tensor([0.3, 0.4]),)) is _NO_TRACE


def test_unhashable_or_tensor_kwargs_are_not_cached():
    s = jq.Script(lambda a, w=None: jq.RX(a[0], wires=0), n_qubits=1)
    assert s._trace_key("expval", (torch.zeros(1),), {"w": torch.zeros(1)}, None, None, None, None, None) is None
    assert s._trace_key("expval", (torch.zeros(1),), {"w": [1, 2]}, None, None, None, None, None) is not None
    assert s._trace_key("expval", (object(),), {}, None, None, None, None, None) is None
    s.cache_traces = False
    assert s._trace_key("expval", (torch.zeros(1),), {}, None, None, None, None, None) is None


# ---------------------------------------------------------------------------
# GPU: cached == uncached
# ---------------------------------------------------------------------------
def _np(t):
    return t.detach().cpu().numpy()


def _both(make_script, call):
    """call(script) on a cached and an uncached Script of the same circuit,
    three times each (first call builds the cache)."""
    out = []
    for cache in (True, False):
        s = make_script()
        s.cache_traces = cache
        out.append([call(s, k) for k in range(3)])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_cached_eager_calls_match_uncached(dtype):
    n, layers = 10, 4
    base = np.random.default_rng(1).uniform(0, 2 * np.pi, (layers, n, 3))
    obs = W.zz_chain(n) + [jq.PauliX(3)]

    def call(s, k):
        a = torch.tensor(base + 0.1 * k, requires_grad=True)
        ev = s.execute("expval", obs, args=(a,), dtype=dtype)
        ev.sum().backward()
        return _np(ev), _np(a.grad), _np(s.execute("probs", args=(a,), dtype=dtype))

    cached, plain = _both(lambda: jq.Script(lambda a: W.strongly_entangling(n, layers, a), n_qubits=n), call)
    for c, p in zip(cached, plain):
        for x, y in zip(c, p):
            np.testing.assert_allclose(x, y, atol=1e-12, rtol=0)


@pytest.mark.gpu
def test_cached_batched_calls_match_uncached():
    n, layers = 6, 3
    rng = np.random.default_rng(2)
    base = rng.uniform(0, 2 * np.pi, (5, layers, n, 3))
    shared = torch.tensor(0.3, dtype=torch.float64)

    def circuit(a, c):
        W.rot_ring(n, layers, a)
        jq.CRX(c, wires=[0, n - 1])
        jq.RZ(0.25, wires=2)

    def call(s, k):
        a = torch.tensor(base + 0.05 * k, requires_grad=True)
        c = shared.clone().requires_grad_(True)
        ev = s.execute("expval", [jq.PauliZ(0), jq.PauliY(2)], args=(a, c), in_axes=(0, None),
                       dtype=torch.complex128)
        ev.sum().backward()
        return _np(ev), _np(a.grad), _np(c.grad)

    cached, plain = _both(lambda: jq.Script(circuit, n_qubits=n), call)
    for c, p in zip(cached, plain):
        for x, y in zip(c, p):
            np.testing.assert_allclose(x, y, atol=1e-12, rtol=0)


@pytest.mark.gpu
def test_uncacheable_circuit_follows_new_values():
    """A branch on an argument value: every call re-records, so a different
    branch is taken when the value changes sign."""
    def circuit(a):
        if a[0] > 0:
            jq.PauliX(wires=0)
        jq.RY(a[1], wires=1)

    s = jq.Script(circuit, n_qubits=2)
    z0 = [s.execute("expval", [jq.PauliZ(0)], args=(torch.tensor([v, 0.2]),))[0].item() for v in (1.0, -1.0, 1.0)]
    np.testing.assert_allclose(z0, [-1.0, 1.0, -1.0], atol=1e-12)


@pytest.mark.gpu
def test_fingerprint_separates_structures():
    state = {"wires": 1}

    def circuit(a):
        for w in range(state["wires"]):
            jq.RX(a[0], wires=w)

    s = jq.Script(circuit, n_qubits=3)
    x = torch.tensor([0.5], dtype=torch.float64)
    one = s.execute("expval", [jq.PauliZ(1)], args=(x,), fingerprint=1)
    state["wires"] = 2
    two = s.execute("expval", [jq.PauliZ(1)], args=(x,), fingerprint=2)
    np.testing.assert_allclose([one.item(), two.item()], [1.0, np.cos(0.5)], atol=1e-12)
