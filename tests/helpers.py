"""Shared test helpers: convert recorded jaqsi_b200 tapes to oracle records and
build seeded random circuits over the whole gate library."""
from __future__ import annotations

import numpy as np
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import gateset as g
from jaqsi_b200 import noise as nz

_CONST = {"Id", "PauliX", "PauliY", "PauliZ", "H", "S", "SWAP", "CX", "CY", "CZ", "CCX", "CSWAP", "Barrier"}
_ONE_ANGLE = {"RX", "RY", "RZ", "CRX", "CRY", "CRZ", "RXX", "RYY", "RZZ", "RZX", "ControlledPhaseShift"}


def _f(v):
    return float(v.detach().cpu()) if isinstance(v, torch.Tensor) else float(v)


def to_records(tape):
    """Oracle records (name, wires, params) of a recorded tape."""
    recs = []
    for op in tape:
        name = type(op).__name__
        w = list(op.wires)
        if name in _CONST and (op._matrix is type(op)._matrix or name in ("Id", "Barrier")):
            recs.append((name, w, []))
        elif name in _ONE_ANGLE:
            recs.append((name, w, [_f(op.parameters[0])]))
        elif name == "Rot":
            recs.append(("Rot", w, [_f(op.phi), _f(op.theta), _f(op.omega)]))
        elif name == "PauliRot":
            recs.append(("PauliRot", w, [_f(op.theta), op.pauli_word]))
        elif name == "ControlledPauliRot":
            recs.append(("ControlledPauliRot", w, [_f(op.theta), op.pauli_word, op.n_controls]))
        elif name == "DiagonalQubitUnitary":
            d = op.diag.detach().cpu().numpy() if isinstance(op.diag, torch.Tensor) else np.asarray(op.diag)
            recs.append(("DiagonalQubitUnitary", w, [d]))
        elif isinstance(op, nz.QubitChannel):
            recs.append(("QubitChannel", w, [op.kraus_matrices()]))
        elif isinstance(op, nz.KrausChannel):
            recs.append((name, w, [_f(v) for v in op.parameters]))
        else:
            m = op._matrix
            m = m.detach().cpu().numpy() if isinstance(m, torch.Tensor) else np.asarray(m)
            recs.append(("Matrix", w, [m]))
    return recs


def obs_records(obs):
    out = []
    for ob in obs:
        name = type(ob).__name__
        if name in ("PauliX", "PauliY", "PauliZ"):
            out.append((name, list(ob.wires)))
        else:
            m = ob._matrix
            m = m.detach().cpu().numpy() if isinstance(m, torch.Tensor) else np.asarray(m)
            out.append(("Matrix", list(ob.wires), m))
    return out


GATES_1Q = ["RX", "RY", "RZ", "Rot", "H", "S", "PauliX", "PauliY", "PauliZ"]
GATES_2Q = ["CX", "CY", "CZ", "SWAP", "CRX", "CRY", "CRZ", "ControlledPhaseShift", "RXX", "RYY", "RZZ", "RZX"]
GATES_3Q = ["CCX", "CSWAP", "PauliRot3", "CPauliRot"]


def random_circuit(n, depth, rng, params, wide=True, channels=False):
    """Record a random circuit; parametrised gates take successive entries of
    *params* (a 1-D tensor), so gradients w.r.t. *params* follow recording order."""
    slot = [0]

    def nxt():
        v = params[slot[0]]
        slot[0] += 1
        return v

    kinds = list(GATES_1Q)
    if n >= 2:
        kinds += GATES_2Q
    if n >= 3 and wide:
        kinds += GATES_3Q
    for _ in range(depth):
        kind = kinds[rng.integers(len(kinds))]
        if kind in GATES_1Q:
            w = int(rng.integers(n))
            if kind == "Rot":
                g.Rot(nxt(), nxt(), nxt(), wires=w)
            elif kind in ("RX", "RY", "RZ"):
                getattr(g, kind)(nxt(), wires=w)
            else:
                getattr(g, kind)(wires=w)
        elif kind in GATES_2Q:
            w = [int(x) for x in rng.choice(n, 2, replace=False)]
            if kind in ("CX", "CY", "CZ", "SWAP"):
                getattr(g, kind)(wires=w)
            else:
                getattr(g, kind)(nxt(), wires=w)
        else:
            w = [int(x) for x in rng.choice(n, 3, replace=False)]
            if kind == "PauliRot3":
                g.PauliRot(nxt(), "".join("XYZ"[int(c)] for c in rng.integers(0, 3, 3)), wires=w)
            elif kind == "CPauliRot":
                g.ControlledPauliRot(nxt(), "XY", wires=w, n_controls=1)
            else:
                getattr(g, kind)(wires=w)
        if channels and rng.random() < 0.5:
            w = int(rng.integers(n))
            c = rng.integers(5)
            if c == 0:
                nz.DepolarizingChannel(0.05, wires=w)
            elif c == 1:
                nz.AmplitudeDamping(0.1, wires=w)
            elif c == 2:
                nz.BitFlip(0.07, wires=w)
            elif c == 3:
                nz.PhaseDamping(0.2, wires=w)
            else:
                nz.PhaseFlip(0.03, wires=w)
    return slot[0]


def count_params(n, depth, seed, wide=True, channels=False):
    rng = np.random.default_rng(seed)
    dummy = torch.zeros(10 * depth + 10, dtype=torch.float64)
    with jq.recording():
        return random_circuit(n, depth, rng, dummy, wide, channels)


def ansatz_layers(n, layers, angles, cx_range=None):
    """RX/RY/RZ on every wire then a CX ring (the configs' ansatz)."""
    for l in range(layers):
        for w in range(n):
            g.RX(angles[l, w, 0], wires=w)
            g.RY(angles[l, w, 1], wires=w)
            g.RZ(angles[l, w, 2], wires=w)
        for w in range(n):
            g.CX(wires=[w, (w + 1) % n])
