"""CPU oracle: a float64 NumPy restatement of jaqsi's simulation path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (jaqsi_b200/) imports or
calls this module; only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it, as the checker.

It follows the reference file by file:
  gate matrices      jaqsi/gateset.py:32-910 (RX/RY/RZ 399-451, CX/CY/CZ 459-512,
                     CCX 515-548, CSWAP 551-584, ControlledPhaseShift 587-619,
                     Rot 622-667, PauliRot 670-758, ControlledPauliRot 764-890)
  Kraus channels     jaqsi/noise.py:123-465
  op-by-op dense     jaqsi/operations.py:553-574 (apply_to_state),
  application        :617-644 (apply_to_density), noise.py:93-120
  fusion / plan      jaqsi/simulation.py:214-240 (_fuse), :290-335 (_fuse_runs),
                     :348-381 (_compile_mixed)  -- used for pass counts only
  measurement        jaqsi/simulation.py:735-857
  adjoint            jaqsi/simulation.py:546-655 (reverse walk: psi <- U^+ psi,
                     lam <- U^+ lam), with angle derivatives of each gate
  Adam               optax 0.2.8 ``optax.adam`` defaults (b1=0.9, b2=0.999,
                     eps=1e-8, eps_root=0), used by jaqsi/tests/test_training.py

Parity is pinned by the reference's own known answers (tests/test_oracle.py):
the training trajectories of jaqsi/tests/test_training.py:33-106 (rtol 1e-12),
Bell/GHZ values (tests/test_jaqsi.py:364-434), analytic gradients
(test_jaqsi.py:136-146, test_adjoint.py:179-192) and the textbook Kraus
densities (test_jaqsi.py:118-132, 612-711).  jaqsi itself (JAX) cannot be
imported in this build environment.

A circuit is a list of records ``(name, wires, params)``; ``name`` is a jaqsi
gate or channel class name, or "Matrix" with ``params = [matrix]``.
"""
from __future__ import annotations

import itertools
import string
from functools import reduce
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

I2 = np.eye(2, dtype=np.complex128)
X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
HAD = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
S_GATE = np.array([[1, 0], [0, 1j]], dtype=np.complex128)
PAULI = {"I": I2, "X": X, "Y": Y, "Z": Z}
P0 = np.array([[1, 0], [0, 0]], dtype=np.complex128)
P1 = np.array([[0, 0], [0, 1]], dtype=np.complex128)

Record = Tuple[str, Sequence[int], Sequence]

CHANNELS = ("BitFlip", "PhaseFlip", "DepolarizingChannel", "AmplitudeDamping", "PhaseDamping",
            "ThermalRelaxationError", "QubitChannel")


def pauli_tensor(word: str) -> np.ndarray:
    return reduce(np.kron, [PAULI[c] for c in word])


def rot(theta: float, P: np.ndarray) -> np.ndarray:
    """cos(t/2) I - i sin(t/2) P (gateset.py:399-405)."""
    return np.cos(theta / 2) * np.eye(P.shape[0]) - 1j * np.sin(theta / 2) * P


def drot(theta: float, P: np.ndarray) -> np.ndarray:
    return -0.5 * np.sin(theta / 2) * np.eye(P.shape[0]) - 0.5j * np.cos(theta / 2) * P


def controlled(inner: np.ndarray, n_controls: int) -> np.ndarray:
    d_t = inner.shape[0]
    dim = (2**n_controls) * d_t
    m = np.eye(dim, dtype=np.complex128)
    m[dim - d_t:, dim - d_t:] = inner
    return m


def gate_matrix(name: str, params: Sequence, k: int) -> np.ndarray:
    """Matrix of a recorded gate (first wire = most significant bit)."""
    p = list(params)
    if name == "Id":
        return np.eye(2**k, dtype=np.complex128)
    if name == "PauliX":
        return X.copy()
    if name == "PauliY":
        return Y.copy()
    if name == "PauliZ":
        return Z.copy()
    if name == "H":
        return HAD.copy()
    if name == "S":
        return S_GATE.copy()
    if name == "SWAP":
        return np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    if name in ("RX", "RY", "RZ"):
        return rot(float(p[0]), PAULI[name[1]])
    if name in ("CX", "CY", "CZ"):
        return np.kron(P0, I2) + np.kron(P1, PAULI[name[1]])
    if name == "CCX":
        return np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 5, 7, 6]]
    if name == "CSWAP":
        return np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 6, 5, 7]]
    if name == "ControlledPhaseShift":
        return np.diag([1, 1, 1, np.exp(1j * float(p[0]))]).astype(np.complex128)
    if name == "Rot":
        phi, theta, omega = (float(v) for v in p)
        return rot(omega, Z) @ rot(theta, Y) @ rot(phi, Z)
    if name == "PauliRot":
        return rot(float(p[0]), pauli_tensor(p[1]))
    if name in ("RXX", "RYY", "RZZ", "RZX"):
        return rot(float(p[0]), pauli_tensor(name[1:]))
    if name == "ControlledPauliRot":
        theta, word, nc = float(p[0]), p[1], int(p[2])
        return controlled(rot(theta, pauli_tensor(word)), nc)
    if name in ("CRX", "CRY", "CRZ"):
        return controlled(rot(float(p[0]), PAULI[name[2]]), 1)
    if name == "DiagonalQubitUnitary":
        return np.diag(np.asarray(p[0], dtype=np.complex128))
    if name == "Matrix":
        return np.asarray(p[0], dtype=np.complex128)
    raise KeyError(f"oracle: unknown gate {name!r}")


def gate_derivatives(name: str, params: Sequence, k: int) -> List[np.ndarray]:
    """d(matrix)/d(angle) for each real angle of a parametrised gate."""
    p = list(params)
    if name in ("RX", "RY", "RZ"):
        return [drot(float(p[0]), PAULI[name[1]])]
    if name == "Rot":
        phi, theta, omega = (float(v) for v in p)
        a, b, c = rot(phi, Z), rot(theta, Y), rot(omega, Z)
        return [c @ b @ drot(phi, Z), c @ drot(theta, Y) @ a, drot(omega, Z) @ b @ a]
    if name == "ControlledPhaseShift":
        return [np.diag([0, 0, 0, 1j * np.exp(1j * float(p[0]))]).astype(np.complex128)]
    if name == "PauliRot":
        return [drot(float(p[0]), pauli_tensor(p[1]))]
    if name in ("RXX", "RYY", "RZZ", "RZX"):
        return [drot(float(p[0]), pauli_tensor(name[1:]))]
    if name == "ControlledPauliRot":
        theta, word, nc = float(p[0]), p[1], int(p[2])
        d = controlled(drot(theta, pauli_tensor(word)), nc)
        n = d.shape[0]
        d[: n - 2 ** len(word), : n - 2 ** len(word)] = 0
        return [d]
    if name in ("CRX", "CRY", "CRZ"):
        d = controlled(drot(float(p[0]), PAULI[name[2]]), 1)
        d[:2, :2] = 0
        return [d]
    return []


def kraus(name: str, params: Sequence) -> List[np.ndarray]:
    """Kraus operators (noise.py:123-465)."""
    p = list(params)
    if name == "BitFlip":
        return [np.sqrt(1 - p[0]) * I2, np.sqrt(p[0]) * X]
    if name == "PhaseFlip":
        return [np.sqrt(1 - p[0]) * I2, np.sqrt(p[0]) * Z]
    if name == "DepolarizingChannel":
        q = p[0]
        return [np.sqrt(1 - q) * I2, np.sqrt(q / 3) * X, np.sqrt(q / 3) * Y, np.sqrt(q / 3) * Z]
    if name == "AmplitudeDamping":
        g = p[0]
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=np.complex128),
                np.array([[0, np.sqrt(g)], [0, 0]], dtype=np.complex128)]
    if name == "PhaseDamping":
        g = p[0]
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=np.complex128),
                np.array([[0, 0], [0, np.sqrt(g)]], dtype=np.complex128)]
    if name == "ThermalRelaxationError":
        pe, t1, t2, tg = (float(v) for v in p)
        eT1 = np.exp(-tg / t1)
        pr = 1.0 - eT1
        eT2 = np.exp(-tg / t2)
        if t2 <= t1:
            pz = (1.0 - pr) * (1.0 - eT2 / eT1) / 2.0
            pr0, pr1 = (1.0 - pe) * pr, pe * pr
            pid = 1.0 - pz - pr0 - pr1
            return [np.sqrt(pid) * I2, np.sqrt(pz) * Z, np.sqrt(pr0) * P0,
                    np.sqrt(pr0) * np.array([[0, 1], [0, 0]], dtype=np.complex128),
                    np.sqrt(pr1) * np.array([[0, 0], [1, 0]], dtype=np.complex128), np.sqrt(pr1) * P1]
        choi = np.array([[1 - pe * pr, 0, 0, eT2], [0, pe * pr, 0, 0], [0, 0, (1 - pe) * pr, 0],
                         [eT2, 0, 0, 1 - (1 - pe) * pr]], dtype=np.complex128)
        vals, vecs = np.linalg.eigh(choi)
        return [np.sqrt(abs(vals[i])) * vecs[:, i].reshape(2, 2, order="F") for i in range(4)]
    if name == "QubitChannel":
        return [np.asarray(K, dtype=np.complex128) for K in p[0]]
    raise KeyError(f"oracle: unknown channel {name!r}")


# ---------------------------------------------------------------------------
# dense application (operations.py:46-77, 553-574, 617-644)
# ---------------------------------------------------------------------------
def _subscript(n: int, k: int, axes: Sequence[int]) -> str:
    letters = string.ascii_letters
    state = list(letters[:n])
    contracted = [state[a] for a in axes]
    new = [letters[n + i] for i in range(k)]
    res = list(state)
    for i, a in enumerate(axes):
        res[a] = new[i]
    return "".join(new + contracted) + "," + "".join(state) + "->" + "".join(res)


def apply_matrix(psi: np.ndarray, U: np.ndarray, axes: Sequence[int], nax: int) -> np.ndarray:
    """Contract a 2^k x 2^k matrix into axes *axes* of a rank-nax tensor."""
    k = len(axes)
    t = psi.reshape((2,) * nax)
    out = np.einsum(_subscript(nax, k, tuple(axes)), U.reshape((2,) * 2 * k), t, optimize=True)
    return out.reshape(-1)


def initial_state(n: int, init: Optional[np.ndarray] = None) -> np.ndarray:
    if init is None:
        s = np.zeros(2**n, dtype=np.complex128)
        s[0] = 1.0
        return s
    return np.asarray(init, dtype=np.complex128).reshape(2**n).copy()


def simulate_pure(records: Sequence[Record], n: int, init=None) -> np.ndarray:
    """Op-by-op statevector evolution (the reference's own test oracle)."""
    psi = initial_state(n, init)
    for name, wires, params in records:
        if name == "Barrier":
            continue
        if name in CHANNELS:
            raise TypeError(f"{name} is a noise channel and cannot be applied to a pure statevector.")
        psi = apply_matrix(psi, gate_matrix(name, params, len(wires)), list(wires), n)
    return psi


def simulate_mixed(records: Sequence[Record], n: int, init=None) -> np.ndarray:
    """Op-by-op density evolution: U rho U^+ and sum_k K rho K^+."""
    psi = initial_state(n, init)
    rho = np.outer(psi, psi.conj()).reshape(-1)
    for name, wires, params in records:
        if name == "Barrier":
            continue
        bra = [w + n for w in wires]
        if name in CHANNELS:
            acc = np.zeros_like(rho)
            for K in kraus(name, params):
                r = apply_matrix(rho, K, list(wires), 2 * n)
                acc = acc + apply_matrix(r, K.conj(), bra, 2 * n)
            rho = acc
        else:
            U = gate_matrix(name, params, len(wires))
            rho = apply_matrix(apply_matrix(rho, U, list(wires), 2 * n), U.conj(), bra, 2 * n)
    d = 2**n
    return rho.reshape(d, d)


# ---------------------------------------------------------------------------
# observables and measurement (simulation.py:735-857)
# ---------------------------------------------------------------------------
def obs_matrix(ob) -> Tuple[np.ndarray, List[int]]:
    """(matrix, wires) of an observable given as (name, wires[, matrix])."""
    name, wires = ob[0], list(ob[1])
    if name in ("PauliX", "PauliY", "PauliZ"):
        return PAULI[name[-1]], wires
    if name == "Id":
        return np.eye(2 ** len(wires), dtype=np.complex128), wires
    if name == "Pauli":
        return pauli_tensor(ob[2]), wires
    if name == "Matrix":
        return np.asarray(ob[2], dtype=np.complex128), wires
    raise KeyError(f"oracle: unknown observable {name!r}")


def lifted(M: np.ndarray, wires: Sequence[int], n: int) -> np.ndarray:
    dim = 2**n
    eye = np.eye(dim, dtype=np.complex128)
    return np.stack([apply_matrix(eye[:, j], M, list(wires), n) for j in range(dim)], axis=1)


def apply_obs(psi: np.ndarray, ob, n: int) -> np.ndarray:
    M, wires = obs_matrix(ob)
    return apply_matrix(psi, M, wires, n)


def expval_state(psi: np.ndarray, n: int, obs) -> np.ndarray:
    return np.array([np.real(np.vdot(psi, apply_obs(psi, ob, n))) for ob in obs])


def expval_density(rho: np.ndarray, n: int, obs) -> np.ndarray:
    out = []
    for ob in obs:
        M, wires = obs_matrix(ob)
        # Tr(O rho): apply O to the ket side of rho, then trace
        r = apply_matrix(rho.reshape(-1), M, wires, 2 * n).reshape(2**n, 2**n)
        out.append(np.real(np.trace(r)))
    return np.array(out)


def measure_state(psi: np.ndarray, n: int, type: str, obs=()):
    if type == "state":
        return psi
    if type == "probs":
        return np.abs(psi) ** 2
    if type == "density":
        return np.outer(psi, psi.conj())
    if type == "expval":
        return expval_state(psi, n, obs)
    raise ValueError(f"Unknown measurement type: {type!r}")


def measure_density(rho: np.ndarray, n: int, type: str, obs=()):
    if type == "density":
        return rho
    if type == "probs":
        return np.real(np.diag(rho))
    if type == "expval":
        return expval_density(rho, n, obs)
    raise ValueError("Measurement type 'state' is not defined for mixed (noisy) circuits. Use 'density' instead.")


def execute(records, n: int, type: str, obs=(), init=None):
    """Reference semantics of Script.execute for one sample."""
    if any(r[0] in CHANNELS for r in records):
        return measure_density(simulate_mixed(records, n, init), n, type, obs)
    return measure_state(simulate_pure(records, n, init), n, type, obs)


# ---------------------------------------------------------------------------
# adjoint gradient (simulation.py:546-655), per recorded angle
# ---------------------------------------------------------------------------
def param_count(name: str) -> int:
    if name == "Rot":
        return 3
    if name in ("RX", "RY", "RZ", "ControlledPhaseShift", "PauliRot", "RXX", "RYY", "RZZ", "RZX",
                "ControlledPauliRot", "CRX", "CRY", "CRZ"):
        return 1
    return 0


def adjoint_grad(records, n: int, obs, ct=None, init=None) -> Tuple[np.ndarray, np.ndarray]:
    """(expvals, d(sum_o ct_o <O_o>)/d(angles)) in recording order of angles.

    lam = 2 sum_o ct_o O_o psi is the gradient w.r.t. the final state
    (d/dRe + i d/dIm); walking back, dL/dtheta = Re <lam | dU/dtheta | psi_in>.
    """
    psi = simulate_pure(records, n, init)
    ev = expval_state(psi, n, obs)
    ct = np.ones(len(obs)) if ct is None else np.asarray(ct, dtype=float)
    lam = np.zeros_like(psi)
    for c, ob in zip(ct, obs):
        lam = lam + 2.0 * c * apply_obs(psi, ob, n)
    grads: List[List[float]] = []
    for name, wires, params in reversed(list(records)):
        if name == "Barrier":
            continue
        U = gate_matrix(name, params, len(wires))
        psi = apply_matrix(psi, U.conj().T, list(wires), n)
        g = [float(np.real(np.vdot(lam, apply_matrix(psi, dU, list(wires), n))))
             for dU in gate_derivatives(name, params, len(wires))]
        grads.append(g)
        lam = apply_matrix(lam, U.conj().T, list(wires), n)
    flat = [v for g in reversed(grads) for v in g]
    return ev, np.array(flat)


def finite_difference(fn, x: np.ndarray, h: float = 1e-6) -> np.ndarray:
    """Central differences of a scalar function of a real vector."""
    x = np.asarray(x, dtype=float)
    g = np.zeros_like(x)
    for i in range(x.size):
        e = np.zeros_like(x)
        e.flat[i] = h
        g.flat[i] = (fn(x + e) - fn(x - e)) / (2 * h)
    return g


# ---------------------------------------------------------------------------
# the reference's plan (pass counts): _fuse, _fuse_runs, _compile_mixed
# ---------------------------------------------------------------------------
STRUCT_PERM = {"PauliX": (1, 0), "SWAP": (0, 2, 1, 3), "CX": (0, 1, 3, 2), "CCX": (0, 1, 2, 3, 4, 5, 7, 6),
               "CSWAP": (0, 1, 2, 3, 4, 6, 5, 7)}
STRUCT_DIAG = {"Id", "PauliZ", "S", "RZ", "CZ", "ControlledPhaseShift", "DiagonalQubitUnitary", "RZZ"}


def _kind(name: str) -> Optional[str]:
    if name in STRUCT_PERM:
        return "permutation"
    if name in STRUCT_DIAG:
        return "diagonal"
    return None


def fuse(records) -> List[Tuple[Tuple[int, ...], Optional[str]]]:
    """Blocks of jaqsi's _fuse (simulation.py:214-240): (wires, kind)."""
    fused: List[list] = []
    last: Dict[int, int] = {}
    for name, wires, params in records:
        if name == "Barrier":
            continue
        wires = tuple(wires)
        kind = _kind(name)
        i = last.get(wires[0])
        if i is not None and fused[i][0] == wires and all(last[w] == i for w in wires):
            a, b = fused[i][1], kind
            fused[i][1] = a if a == b else None
            continue
        fused.append([wires, kind])
        for w in wires:
            last[w] = len(fused) - 1
    return [(w, k) for w, k in fused]


def jaqsi_pass_count(records) -> int:
    """Entries of jaqsi's statevector plan (_fuse then _fuse_runs, :290-335)."""
    plan = 0
    run = 0
    kind = None
    for _, k in fuse(records):
        if k != kind:
            plan += 1 if run > 1 else run
            run = 0
            kind = k
        if k is None:
            plan += 1
        else:
            run += 1
    plan += 1 if run > 1 else run
    return plan


def jaqsi_mixed_pass_count(records, n: int) -> int:
    """Blocks of jaqsi's _compile_mixed (:348-381)."""
    superops = []
    for name, wires, params in records:
        if name == "Barrier":
            continue
        ket = tuple(wires)
        bra = tuple(w + n for w in wires)
        if name in CHANNELS or len(ket) <= 2:
            superops.append(("G", ket + bra, []))
        else:
            superops.append(("G", ket, []))
            superops.append(("G", bra, []))
    return len(fuse(superops))


def jaqsi_mixed_plan(records, n: int) -> List[Tuple[str, Tuple[int, ...], np.ndarray]]:
    """Fused superoperator blocks of jaqsi's _compile_mixed (:348-381) with
    their matrices, as ('dense', axes, S) entries on the 2n-axis density
    vector: sum_k kron(K, K*) for a channel, kron(U, U*) for a gate on at most
    two wires, U on the ket axes and U* on the bra axes for wider gates; then
    _fuse (:214-240) multiplies neighbours on identical axis tuples."""
    blocks: List[list] = []
    last: Dict[int, int] = {}

    def push(S, axes):
        i = last.get(axes[0])
        if i is not None and blocks[i][1] == axes and all(last.get(a) == i for a in axes):
            blocks[i][0] = S @ blocks[i][0]
            return
        blocks.append([S, axes])
        for a in axes:
            last[a] = len(blocks) - 1

    for name, wires, params in records:
        if name == "Barrier":
            continue
        ket = tuple(wires)
        bra = tuple(w + n for w in wires)
        if name in CHANNELS:
            push(sum(np.kron(K, K.conj()) for K in kraus(name, params)), ket + bra)
        else:
            U = gate_matrix(name, params, len(wires))
            if len(ket) <= 2:
                push(np.kron(U, U.conj()), ket + bra)
            else:
                push(U, ket)
                push(U.conj(), bra)
    return [("dense", axes, S) for S, axes in blocks]


# ---------------------------------------------------------------------------
# optax.adam restated (defaults of optax 0.2.8)
# ---------------------------------------------------------------------------
class Adam:
    """mu = (1-b1) g + b1 mu; nu = (1-b2) g^2 + b2 nu; bias-corrected;
    update = -lr mu_hat / (sqrt(nu_hat + eps_root) + eps)."""

    def __init__(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, eps_root: float = 0.0):
        self.lr, self.b1, self.b2, self.eps, self.eps_root = lr, b1, b2, eps, eps_root
        self.mu = None
        self.nu = None
        self.count = 0

    def update(self, g: np.ndarray) -> np.ndarray:
        g = np.asarray(g, dtype=np.float64)
        if self.mu is None:
            self.mu = np.zeros_like(g)
            self.nu = np.zeros_like(g)
        self.mu = (1 - self.b1) * g + self.b1 * self.mu
        self.nu = (1 - self.b2) * (g * g) + self.b2 * self.nu
        self.count += 1
        mu_hat = self.mu / (1 - self.b1**self.count)
        nu_hat = self.nu / (1 - self.b2**self.count)
        u = mu_hat / (np.sqrt(nu_hat + self.eps_root) + self.eps)
        return -self.lr * u


def adam_trajectory(value_and_grad, params: np.ndarray, lr: float, steps: int):
    """Losses after every step of plain Adam plus the final loss, and the
    final parameters (jaqsi/tests/test_training.py:15-30)."""
    opt = Adam(lr)
    p = np.asarray(params, dtype=np.float64).copy()
    losses = []
    for _ in range(steps):
        loss, g = value_and_grad(p)
        p = p + opt.update(g)
        losses.append(float(loss))
    losses.append(float(value_and_grad(p)[0]))
    return np.array(losses), p


# ---------------------------------------------------------------------------
# the reference's executable plan with matrices (simulation.py:214-335), for
# the timed CPU baseline (oracle/jqoracle.c executes it)
# ---------------------------------------------------------------------------
def _structure(name: str, k: int):
    if name in STRUCT_PERM:
        return ("perm", STRUCT_PERM[name])
    if name in STRUCT_DIAG:
        return ("diag", None)
    return (None, None)


def _fused_kind(a, b):
    if a[0] == "perm" and b[0] == "perm":
        return ("perm", tuple(a[1][i] for i in b[1]))
    if a[0] == "diag" and b[0] == "diag":
        return ("diag", None)
    return (None, None)


def compose_permutation(blocks, n: int) -> np.ndarray:
    """2^n int32 gather map of a run of permutation blocks (:243-267):
    out[o] = in[index[o]]."""
    o = np.arange(2**n, dtype=np.int64)
    index = o.copy()
    for _, wires, (_, perm) in blocks:
        k = len(wires)
        bits = [n - 1 - w for w in wires]
        col = np.zeros_like(o)
        mask = 0
        for i, b in enumerate(bits):
            col |= ((o >> b) & 1) << (k - 1 - i)
            mask |= 1 << b
        src_col = np.asarray(perm, dtype=np.int64)[col]
        src = o & ~mask
        for i, b in enumerate(bits):
            src |= ((src_col >> (k - 1 - i)) & 1) << b
        index = index[src]
    return index.astype(np.int32)


def jaqsi_plan(records, n: int, compose=None):
    """Entries ('dense', wires, U) | ('gather', index) | ('diag', wires, d) of
    jaqsi's statevector plan: _fuse then _fuse_runs.  ``compose(run, n)``
    builds a permutation run's gather map (default: compose_permutation;
    oracle/cplan.py passes the C version of the same fold)."""
    compose = compose or compose_permutation
    blocks: List[list] = []
    last: Dict[int, int] = {}
    for name, wires, params in records:
        if name == "Barrier":
            continue
        wires = tuple(wires)
        U = gate_matrix(name, params, len(wires))
        st = _structure(name, len(wires))
        i = last.get(wires[0])
        if i is not None and blocks[i][1] == wires and all(last[w] == i for w in wires):
            blocks[i][0] = U @ blocks[i][0]
            blocks[i][2] = _fused_kind(blocks[i][2], st)
            continue
        blocks.append([U, wires, st])
        for w in wires:
            last[w] = len(blocks) - 1
    plan = []
    run: List[list] = []
    kind = None

    def flush():
        if len(run) > 1 and kind == "perm":
            plan.append(("gather", compose(run, n)))
        elif len(run) > 1:
            ws = tuple(sorted({w for b in run for w in b[1]}))
            d = np.ones((2,) * len(ws), dtype=np.complex128)
            ax = {w: i for i, w in enumerate(ws)}
            for U, bw, _ in run:
                f = np.diag(U).reshape((2,) * len(bw) + (1,) * (len(ws) - len(bw)))
                d = d * np.moveaxis(f, tuple(range(len(bw))), tuple(ax[w] for w in bw))
            plan.append(("diag", ws, d.reshape(-1)))
        else:
            for U, bw, _ in run:
                plan.append(("dense", bw, U))
        run.clear()

    for b in blocks:
        k = b[2][0]
        if k != kind:
            flush()
            kind = k
        if k is None:
            plan.append(("dense", b[1], b[0]))
        else:
            run.append(b)
    flush()
    return plan


# ---------------------------------------------------------------------------
# pulse gates (jaqsi/evolution.py:195-264 Magnus schemes, :354-405 closed form)
# ---------------------------------------------------------------------------
def magnus_unitary(H_mats, fns, params, t0: float, t1: float, steps: int, order: int) -> np.ndarray:
    """The reference's fixed-step commutator-free Magnus integrators: the
    midpoint rule (order 2) or CFM4:2 with U <- exp(Om_b) exp(Om_a) U
    (order 4); coefficient functions take (params, t) with float t."""
    from scipy.linalg import expm

    A = [-1j * np.asarray(H, dtype=np.complex128) for H in H_mats]
    d = A[0].shape[0]
    h = (t1 - t0) / steps

    def Hat(t):
        return sum(complex(f(p, t)) * a for f, p, a in zip(fns, params, A))

    U = np.eye(d, dtype=np.complex128)
    s3 = np.sqrt(3.0)
    c1, c2, a1, a2 = 0.5 - s3 / 6, 0.5 + s3 / 6, 0.25 + s3 / 6, 0.25 - s3 / 6
    for n in range(steps):
        tn = t0 + n * h
        if order == 2:
            U = expm(h * Hat(tn + 0.5 * h)) @ U
        else:
            H1, H2 = Hat(tn + c1 * h), Hat(tn + c2 * h)
            U = expm(h * (a2 * H1 + a1 * H2)) @ expm(h * (a1 * H1 + a2 * H2)) @ U
    return U


def evolution_reference(H_mats, fns, params, t0: float, t1: float, rtol: float = 1e-12) -> np.ndarray:
    """dU/dt = -i sum_i f_i(p_i, t) H_i U, U(t0) = I, by an adaptive
    Dormand-Prince (order 8) solve at tight tolerances: an independent check
    of the Magnus schemes and the closed form."""
    from scipy.integrate import solve_ivp

    Hs = [np.asarray(H, dtype=np.complex128) for H in H_mats]
    d = Hs[0].shape[0]

    def rhs(t, y):
        U = y.reshape(d, d)
        Ht = sum(complex(f(p, t)) * H for f, p, H in zip(fns, params, Hs))
        return (-1j * Ht @ U).reshape(-1)

    sol = solve_ivp(rhs, (t0, t1), np.eye(d, dtype=np.complex128).reshape(-1), method="DOP853", rtol=rtol,
                    atol=rtol)
    return sol.y[:, -1].reshape(d, d)
