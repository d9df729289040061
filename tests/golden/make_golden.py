"""Writes the committed golden fixtures of this directory.

* ``reference_known_answers.json``: the expected values that the reference's
  own training tests assert (jaqsi/tests/test_training.py:33-106), read from
  that file's source text with ``ast`` (the reference is not imported or run:
  it needs JAX, which is not installed).  Needs the reference checkout: its
  root is the first command-line argument, else $JAQSI_REFERENCE, else
  /root/reference; without one the file is kept as it is.
* ``oracle_vectors.npz``: seeded random circuits over the gate library (a
  noisy one included) with the float64 oracle's state / density,
  probabilities, expectation values and adjoint gradients.  The oracle is
  pinned by the known answers above (tests/test_oracle.py), and these vectors
  fix its outputs so the GPU parity tests compare against committed numbers.

Run from the repository root:  python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import ast
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import jaqsi_b200 as jq  # noqa: E402
from oracle import sim_np as O  # noqa: E402
from tests.helpers import count_params, obs_records, random_circuit, to_records  # noqa: E402

def reference_training_tests(root=None) -> str:
    """The reference's training tests under `root`, else $JAQSI_REFERENCE,
    else /root/reference."""
    root = root or os.environ.get("JAQSI_REFERENCE", "/root/reference")
    return os.path.join(root, "tests", "test_training.py")

# name: (qubits, depth, seed, 3-qubit gates, channels)
CASES = {
    "pure_n3": (3, 30, 101, True, False),
    "pure_n5": (5, 60, 102, True, False),
    "pure_n8": (8, 80, 103, True, False),
    "mixed_n3": (3, 25, 104, True, True),
}
CT = [1.0, -0.5, 0.25, 2.0]


def golden_obs(n):
    """Observables of every case: Z, X, Y words and a ZZ parity (dense)."""
    obs = [jq.PauliZ(wires=0), jq.PauliX(wires=n - 1), jq.PauliY(wires=n // 2)]
    if n >= 2:
        obs.append(jq.build_parity_observable([0, n - 1]))
    return obs


def case_params(name):
    n, depth, seed, wide, channels = CASES[name]
    npar = count_params(n, depth, seed, wide, channels)
    return np.random.default_rng(seed + 1000).uniform(0, 2 * np.pi, npar + 1)


def case_records(name, params):
    n, depth, seed, wide, channels = CASES[name]
    with jq.recording() as tape:
        random_circuit(n, depth, np.random.default_rng(seed), torch.tensor(params), wide, channels)
    return to_records(tape)


def oracle_outputs(name, params):
    """Everything the oracle says about one case (dict of arrays)."""
    n, _, _, _, channels = CASES[name]
    recs = case_records(name, params)
    obs = obs_records(golden_obs(n))
    ct = CT[: len(obs)]
    out = {"expval": O.execute(recs, n, "expval", obs), "probs": O.execute(recs, n, "probs")}
    if channels:
        out["density"] = O.execute(recs, n, "density")
    else:
        out["state"] = O.execute(recs, n, "state")
        _, out["grad"] = O.adjoint_grad(recs, n, obs, ct=ct)
    return recs, out


def _literal_values(fn: ast.FunctionDef):
    """(list literal, scalar literal) of the assert_allclose calls in *fn*:
    the loss samples and the first parameter's final value."""
    lists, scalars = [], []
    for node in ast.walk(fn):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "assert_allclose":
            want = node.args[1]
            if isinstance(want, ast.List):
                lists.append([ast.literal_eval(e) for e in want.elts])
            elif isinstance(want, (ast.Constant, ast.UnaryOp)):
                scalars.append(ast.literal_eval(want))
    return lists, scalars


def known_answers(path):
    tree = ast.parse(open(path).read())
    fns = {n.name: n for n in tree.body if isinstance(n, ast.FunctionDef)}
    out = {"source": "jaqsi/tests/test_training.py"}
    for key, fname, lines in (("minimal_training_loop", "test_minimal_training_loop", "33-66"),
                              ("fitting_data", "test_fitting_data", "69-106")):
        lists, scalars = _literal_values(fns[fname])
        out[key] = {"lines": lines, "losses_24_100_25": lists[0], "param0_final": scalars[0],
                    "param1_final": scalars[1]}
    return out


def main(root=None):
    path = reference_training_tests(root)
    if os.path.exists(path):
        with open(os.path.join(HERE, "reference_known_answers.json"), "w") as f:
            json.dump(known_answers(path), f, indent=1)
            f.write("\n")
    arrays = {}
    for name, (n, depth, seed, wide, channels) in CASES.items():
        params = case_params(name)
        recs, out = oracle_outputs(name, params)
        arrays[f"{name}/params"] = params
        arrays[f"{name}/records"] = np.array(json.dumps(recs))
        for k, v in out.items():
            arrays[f"{name}/{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "oracle_vectors.npz"), **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
