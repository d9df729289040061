"""GPU shot sampling (jq_sample_shots): inverse-CDF draws over a float64
prefix sum with a counter-based generator.  The reference samples with JAX's
PRNG (jaqsi/simulation.py:860-917), whose stream cannot be reproduced, so the
checks are distributional (chi-square against the probabilities) plus exact
properties: zero-probability states never drawn, counts sum to the shots,
a seed reproduces the counts, multi-tile prefix sums."""
import ctypes

import numpy as np
import pytest
import torch
from scipy import stats

import jaqsi_b200 as jq
from jaqsi_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _sample(probs: np.ndarray, shots: int, seed: int) -> np.ndarray:
    p = torch.tensor(np.atleast_2d(probs), dtype=torch.float64, device="cuda")
    rows, dim = p.shape
    lib = L.lib()
    wsb = int(lib.jq_sample_workspace_bytes(rows, dim))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    counts = torch.empty((rows, dim), dtype=torch.int32, device="cuda")
    vp = ctypes.c_void_p
    L.check(lib.jq_sample_shots(vp(p.data_ptr()), rows, dim, shots, seed, vp(counts.data_ptr()), vp(ws.data_ptr()),
                                wsb, vp(torch.cuda.current_stream().cuda_stream)))
    return counts.cpu().numpy()


def test_chi_square_and_exact_properties():
    rng = np.random.default_rng(3)
    dim, shots = 1024, 2_000_000
    p = rng.random(dim) ** 3
    p[rng.choice(dim, 100, replace=False)] = 0.0
    p /= p.sum()
    c = _sample(p, shots, seed=11)[0]
    assert c.sum() == shots
    assert np.all(c[p == 0.0] == 0)
    m = p > 0
    chi2 = ((c[m] - shots * p[m]) ** 2 / (shots * p[m])).sum()
    assert stats.chi2.sf(chi2, m.sum() - 1) > 1e-6, chi2
    np.testing.assert_array_equal(c, _sample(p, shots, seed=11)[0])  # a seed reproduces the counts
    assert np.any(c != _sample(p, shots, seed=12)[0])


def test_rows_are_independent_distributions_and_unnormalised_ok():
    rng = np.random.default_rng(4)
    dim, shots = 256, 500_000
    P = rng.random((3, dim))
    P[1] = 0.0
    P[1, 17] = 2.5  # unnormalised point mass
    c = _sample(P, shots, seed=5)
    assert np.all(c.sum(axis=1) == shots)
    assert c[1, 17] == shots
    for r in (0, 2):
        p = P[r] / P[r].sum()
        chi2 = ((c[r] - shots * p) ** 2 / (shots * p)).sum()
        assert stats.chi2.sf(chi2, dim - 1) > 1e-6


def test_multi_tile_prefix_sum():
    """2^20 entries = 1024 scan tiles; mass on a few indices spread across
    tiles, including the first and the last."""
    dim, shots = 1 << 20, 400_000
    p = np.zeros(dim)
    idx = [0, 5, 300_001, 777_777, dim - 1]
    w = np.array([1, 2, 3, 4, 5], dtype=float)
    p[idx] = w / w.sum()
    p[123_456] = 1e-300  # below the resolution of the draws, never chosen in practice
    c = _sample(p, shots, seed=21)[0]
    assert c.sum() == shots
    nz = np.nonzero(c)[0].tolist()
    assert set(nz) <= set(idx + [123_456])
    exp = shots * w / w.sum()
    assert np.all(np.abs(c[idx] - exp) < 6 * np.sqrt(exp))


def test_script_shots_bell():
    def circuit():
        jq.H(wires=0)
        jq.CX(wires=[0, 1])

    s = jq.Script(circuit, n_qubits=2)
    shots = 200_000
    pr = s.execute("probs", shots=shots, key=7, dtype=torch.complex128).cpu().numpy()
    assert pr[1] == 0 and pr[2] == 0
    assert abs(pr[0] - 0.5) < 5 * np.sqrt(0.25 / shots)
    ev = s.execute("expval", [jq.PauliZ(0), jq.PauliZ(1)], shots=shots, key=8).cpu().numpy()
    assert np.all(np.abs(ev) < 5 / np.sqrt(shots))
    np.testing.assert_array_equal(pr, s.execute("probs", shots=shots, key=7, dtype=torch.complex128).cpu().numpy())
    # as in the reference, 'state' ignores shots (exact result); sample_shots
    # itself rejects other types (jaqsi/simulation.py:915-917)
    st = s.execute("state", shots=shots, dtype=torch.complex128).cpu().numpy()
    np.testing.assert_allclose(np.abs(st) ** 2, [0.5, 0, 0, 0.5], atol=1e-12)
    with pytest.raises(ValueError):
        jq.simulation.sample_shots(torch.tensor([0.5, 0, 0, 0.5], device="cuda"), 2, "state", [], shots, 1)
