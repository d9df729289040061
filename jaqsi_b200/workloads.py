"""Synthetic circuits of the benchmark configurations.

Each builder records its circuit on the active tape (call it inside a circuit
function given to ``Script``, or inside ``recording()``), and each has a
``*_records`` twin that returns the same circuit as plain
``(gate name, wires, params)`` tuples for CPU restatements.  Angles are
arrays indexed ``[layer, wire, k]``.

- ``sweep_ansatz``: RX, RY, RZ on every wire, then CX(i, i+1 mod n)
  (10 qubits / 5 layers with <Z_i>; 24 qubits / 20 layers with sum Z_i Z_(i+1)).
- ``strongly_entangling``: Rot(phi, theta, omega) on every wire, then
  CX(i, i+r mod n) with r = (layer mod (n-1)) + 1 (20 qubits, 50 layers).
- ``rot_ring``: Rot on every wire, then CX(i, i+1 mod n) (the batched uneven
  instances).
- ``noisy_ansatz``: ``sweep_ansatz`` with DepolarizingChannel(p) then
  AmplitudeDamping(gamma) on every wire a gate touches, after every gate
  (12-qubit density matrix, 20 layers).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

from jaqsi_b200 import gateset as g
from jaqsi_b200 import noise as nz

Record = Tuple[str, List[int], list]


def _cx_range(layer: int, n: int) -> int:
    return (layer % (n - 1)) + 1 if n > 1 else 0


def sweep_ansatz(n: int, layers: int, a) -> None:
    for l in range(layers):
        for w in range(n):
            g.RX(a[l, w, 0], wires=w)
            g.RY(a[l, w, 1], wires=w)
            g.RZ(a[l, w, 2], wires=w)
        for w in range(n):
            g.CX(wires=[w, (w + 1) % n])


def sweep_ansatz_records(n: int, layers: int, a) -> List[Record]:
    recs: List[Record] = []
    for l in range(layers):
        for w in range(n):
            recs += [("RX", [w], [float(a[l, w, 0])]), ("RY", [w], [float(a[l, w, 1])]),
                     ("RZ", [w], [float(a[l, w, 2])])]
        recs += [("CX", [w, (w + 1) % n], []) for w in range(n)]
    return recs


def strongly_entangling(n: int, layers: int, a) -> None:
    for l in range(layers):
        for w in range(n):
            g.Rot(a[l, w, 0], a[l, w, 1], a[l, w, 2], wires=w)
        r = _cx_range(l, n)
        for w in range(n):
            g.CX(wires=[w, (w + r) % n])


def strongly_entangling_records(n: int, layers: int, a) -> List[Record]:
    recs: List[Record] = []
    for l in range(layers):
        recs += [("Rot", [w], [float(a[l, w, 0]), float(a[l, w, 1]), float(a[l, w, 2])]) for w in range(n)]
        r = _cx_range(l, n)
        recs += [("CX", [w, (w + r) % n], []) for w in range(n)]
    return recs


def rot_ring(n: int, layers: int, a) -> None:
    for l in range(layers):
        for w in range(n):
            g.Rot(a[l, w, 0], a[l, w, 1], a[l, w, 2], wires=w)
        for w in range(n):
            g.CX(wires=[w, (w + 1) % n])


def rot_ring_records(n: int, layers: int, a) -> List[Record]:
    recs: List[Record] = []
    for l in range(layers):
        recs += [("Rot", [w], [float(a[l, w, 0]), float(a[l, w, 1]), float(a[l, w, 2])]) for w in range(n)]
        recs += [("CX", [w, (w + 1) % n], []) for w in range(n)]
    return recs


def noisy_ansatz(n: int, layers: int, a, p: float = 0.01, gamma: float = 0.005) -> None:
    gates = (g.RX, g.RY, g.RZ)
    for l in range(layers):
        for w in range(n):
            for k in range(3):
                gates[k](a[l, w, k], wires=w)
                nz.DepolarizingChannel(p, wires=w)
                nz.AmplitudeDamping(gamma, wires=w)
        for w in range(n):
            g.CX(wires=[w, (w + 1) % n])
            for q in (w, (w + 1) % n):
                nz.DepolarizingChannel(p, wires=q)
                nz.AmplitudeDamping(gamma, wires=q)


def noisy_ansatz_records(n: int, layers: int, a, p: float = 0.01, gamma: float = 0.005) -> List[Record]:
    recs: List[Record] = []
    for l in range(layers):
        for w in range(n):
            for k, name in enumerate(("RX", "RY", "RZ")):
                recs += [(name, [w], [float(a[l, w, k])]), ("DepolarizingChannel", [w], [p]),
                         ("AmplitudeDamping", [w], [gamma])]
        for w in range(n):
            recs.append(("CX", [w, (w + 1) % n], []))
            for q in (w, (w + 1) % n):
                recs += [("DepolarizingChannel", [q], [p]), ("AmplitudeDamping", [q], [gamma])]
    return recs


def zz_chain(n: int) -> list:
    """Observables Z_i Z_(i+1), i = 0..n-2 (the open chain)."""
    return [g.build_parity_observable([i, i + 1]) for i in range(n - 1)]


def z_each(n: int) -> list:
    """Observables Z_i, i = 0..n-1."""
    return [g.PauliZ(i) for i in range(n)]


def zz_masks(n: int) -> List[int]:
    """Flat-index bit masks of Z_i Z_(i+1) (wire 0 = most significant bit)."""
    return [(1 << (n - 1 - i)) | (1 << (n - 2 - i)) for i in range(n - 1)]


def z_masks(n: int) -> List[int]:
    return [1 << (n - 1 - i) for i in range(n)]


def sample_indices(rng, shape: Sequence[int], count: int) -> List[int]:
    """`count` distinct flat indices of an angles array of `shape`, seeded."""
    total = 1
    for s in shape:
        total *= int(s)
    return sorted(int(i) for i in rng.choice(total, size=min(count, total), replace=False))
