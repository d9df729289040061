"""Committed golden fixtures (tests/golden, written by make_golden.py).

CPU: the fixtures still agree with the generator and the float64 oracle.
GPU: the CUDA path through ``Script`` reproduces the stored oracle vectors
(states / densities, probabilities, expectation values, adjoint gradients)
to 1e-10 in complex128 and 1e-5 in complex64.
"""
import json
import os

import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from tests.golden.make_golden import CASES, CT, golden_obs, oracle_outputs
from tests.helpers import random_circuit

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {torch.complex64: 1e-5, torch.complex128: 1e-10}


def _vectors():
    with np.load(os.path.join(HERE, "oracle_vectors.npz")) as z:
        return {k: z[k] for k in z.files}


def _case(name):
    v = _vectors()
    return {k.split("/", 1)[1]: a for k, a in v.items() if k.startswith(name + "/")}


def test_known_answers_fixture_matches_oracle_tests():
    """The known answers the oracle tests use are the fixture's numbers."""
    ka = json.load(open(os.path.join(HERE, "reference_known_answers.json")))
    assert ka["source"] == "jaqsi/tests/test_training.py"
    for key in ("minimal_training_loop", "fitting_data"):
        assert len(ka[key]["losses_24_100_25"]) == 4


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_vectors_pinned(name):
    """Regenerating a case gives the stored records and oracle outputs."""
    c = _case(name)
    recs, out = oracle_outputs(name, c["params"])
    assert json.dumps(recs) == str(c["records"])
    for k, v in out.items():
        np.testing.assert_allclose(np.asarray(v), c[k], rtol=0, atol=1e-12)


def _np(t):
    return t.detach().cpu().resolve_conj().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_golden(name, dtype):
    n, depth, seed, wide, channels = CASES[name]
    c = _case(name)
    tol = TOL[dtype]

    def circuit(p):
        random_circuit(n, depth, np.random.default_rng(seed), p, wide, channels)

    script = jq.Script(circuit, n_qubits=n)
    obs = golden_obs(n)
    params = torch.tensor(c["params"], requires_grad=True)
    ev = script.execute("expval", obs, args=(params,), dtype=dtype)
    np.testing.assert_allclose(_np(ev), c["expval"], rtol=0, atol=tol)
    pr = script.execute("probs", args=(params.detach(),), dtype=dtype)
    np.testing.assert_allclose(_np(pr), c["probs"], rtol=0, atol=tol)
    if channels:
        rho = script.execute("density", args=(params.detach(),), dtype=dtype)
        np.testing.assert_allclose(_np(rho), c["density"], rtol=0, atol=tol)
        return
    st = script.execute("state", args=(params.detach(),), dtype=dtype)
    np.testing.assert_allclose(_np(st), c["state"], rtol=0, atol=tol)
    ct = torch.tensor(CT[: len(obs)], dtype=torch.float64, device=ev.device)
    (ev.to(torch.float64) @ ct).backward()
    g = c["grad"]
    np.testing.assert_allclose(_np(params.grad)[: len(g)], g, rtol=0, atol=tol * sum(abs(x) for x in CT))
