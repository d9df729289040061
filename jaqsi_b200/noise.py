"""Kraus noise channels (restates jaqsi/noise.py:32-465).

Recording any channel switches a circuit to density-matrix simulation.  The
Kraus operators are constants of the recorded circuit: the backend folds each
channel into a superoperator sum_k K (x) conj(K) when it builds the plan.
"""
from __future__ import annotations

from typing import List, Union

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200.gateset import Id, PauliX, PauliY, PauliZ
from jaqsi_b200.operations import Operation, _contract, cdtype


def _scalar(x) -> float:
    if isinstance(x, torch.Tensor):
        return float(x.detach().cpu())
    return float(x)


def _check_unit_interval(value, name: str) -> None:
    if not 0.0 <= _scalar(value) <= 1.0:
        raise ValueError(f"{name} must be in [0, 1].")


class KrausChannel(Operation):
    """Channel phi(rho) = sum_k K_k rho K_k^dagger (noise.py:32-120)."""

    def kraus_matrices(self) -> List[np.ndarray]:
        raise NotImplementedError

    @property
    def matrix(self):
        raise TypeError(
            f"{self.__class__.__name__} is a noise channel and has no single "
            "unitary matrix. Use apply_to_density() instead."
        )

    def apply_to_state(self, state, n_qubits):
        raise TypeError(
            f"{self.__class__.__name__} is a noise channel and cannot be "
            "applied to a pure statevector. Use execute(type='density') instead."
        )

    def apply_to_density(self, rho: torch.Tensor, n_qubits: int) -> torch.Tensor:
        k = len(self.wires)
        dim = 2**n_qubits
        bra = [w + n_qubits for w in self.wires]
        out = torch.zeros((dim, dim), dtype=cdtype())
        for K in self.kraus_matrices():
            Kt = torch.as_tensor(np.asarray(K), dtype=cdtype()).reshape((2,) * 2 * k)
            r = rho.reshape((2,) * 2 * n_qubits).to(cdtype())
            r = _contract(r, Kt, k, self.wires)
            r = _contract(r, Kt.conj(), k, bra)
            out = out + r.reshape(dim, dim)
        return out

    def _jq_lower(self):
        mats = [np.asarray(K, dtype=np.complex128) for K in self.kraus_matrices()]
        return L.JQ_K_CHANNEL, [], mats

    def _jq_static_key(self):
        mats = self._jq_lower()[2]
        return ("channel", tuple(m.tobytes() for m in mats))


class BitFlip(KrausChannel):
    """K0 = sqrt(1-p) I, K1 = sqrt(p) X (noise.py:123-158)."""

    _num_wires = 1
    _param_names = ("p",)

    def __init__(self, p, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(p, "p")
        self.p = p
        super().__init__(wires=wires)

    def kraus_matrices(self):
        p = _scalar(self.p)
        return [np.sqrt(1 - p) * Id._matrix, np.sqrt(p) * PauliX._matrix]


class PhaseFlip(KrausChannel):
    """K0 = sqrt(1-p) I, K1 = sqrt(p) Z (noise.py:161-196)."""

    _num_wires = 1
    _param_names = ("p",)

    def __init__(self, p, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(p, "p")
        self.p = p
        super().__init__(wires=wires)

    def kraus_matrices(self):
        p = _scalar(self.p)
        return [np.sqrt(1 - p) * Id._matrix, np.sqrt(p) * PauliZ._matrix]


class DepolarizingChannel(KrausChannel):
    """{sqrt(1-p) I, sqrt(p/3) X, sqrt(p/3) Y, sqrt(p/3) Z} (noise.py:199-237)."""

    _num_wires = 1
    _param_names = ("p",)

    def __init__(self, p, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(p, "p")
        self.p = p
        super().__init__(wires=wires)

    def kraus_matrices(self):
        p = _scalar(self.p)
        return [
            np.sqrt(1 - p) * Id._matrix,
            np.sqrt(p / 3) * PauliX._matrix,
            np.sqrt(p / 3) * PauliY._matrix,
            np.sqrt(p / 3) * PauliZ._matrix,
        ]


class AmplitudeDamping(KrausChannel):
    """K0 = diag(1, sqrt(1-g)), K1 = [[0, sqrt(g)], [0, 0]] (noise.py:240-277)."""

    _num_wires = 1
    _param_names = ("gamma",)

    def __init__(self, gamma, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(gamma, "gamma")
        self.gamma = gamma
        super().__init__(wires=wires)

    def kraus_matrices(self):
        g = _scalar(self.gamma)
        return [
            np.array([[1.0, 0.0], [0.0, np.sqrt(1 - g)]], dtype=np.complex128),
            np.array([[0.0, np.sqrt(g)], [0.0, 0.0]], dtype=np.complex128),
        ]


class PhaseDamping(KrausChannel):
    """K0 = diag(1, sqrt(1-g)), K1 = diag(0, sqrt(g)) (noise.py:280-316)."""

    _num_wires = 1
    _param_names = ("gamma",)

    def __init__(self, gamma, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(gamma, "gamma")
        self.gamma = gamma
        super().__init__(wires=wires)

    def kraus_matrices(self):
        g = _scalar(self.gamma)
        return [
            np.array([[1.0, 0.0], [0.0, np.sqrt(1 - g)]], dtype=np.complex128),
            np.array([[0.0, 0.0], [0.0, np.sqrt(g)]], dtype=np.complex128),
        ]


class ThermalRelaxationError(KrausChannel):
    """Simultaneous T1 relaxation and T2 dephasing (noise.py:319-431)."""

    _num_wires = 1
    _param_names = ("pe", "t1", "t2", "tg")

    def __init__(self, pe, t1, t2, tg, wires: Union[int, List[int]] = 0) -> None:
        _check_unit_interval(pe, "pe")
        if _scalar(t1) <= 0:
            raise ValueError("t1 must be > 0.")
        if _scalar(t2) <= 0:
            raise ValueError("t2 must be > 0.")
        if _scalar(t2) > 2 * _scalar(t1):
            raise ValueError("t2 must be <= 2·t1.")
        if _scalar(tg) < 0:
            raise ValueError("tg must be >= 0.")
        self.pe, self.t1, self.t2, self.tg = pe, t1, t2, tg
        super().__init__(wires=wires)

    def kraus_matrices(self):
        pe, t1, t2, tg = (_scalar(v) for v in (self.pe, self.t1, self.t2, self.tg))
        eT1 = np.exp(-tg / t1)
        p_reset = 1.0 - eT1
        eT2 = np.exp(-tg / t2)
        if t2 <= t1:
            pz = (1.0 - p_reset) * (1.0 - eT2 / eT1) / 2.0
            pr0 = (1.0 - pe) * p_reset
            pr1 = pe * p_reset
            pid = 1.0 - pz - pr0 - pr1
            c = np.complex128
            return [
                np.sqrt(pid) * np.eye(2, dtype=c),
                np.sqrt(pz) * np.array([[1, 0], [0, -1]], dtype=c),
                np.sqrt(pr0) * np.array([[1, 0], [0, 0]], dtype=c),
                np.sqrt(pr0) * np.array([[0, 1], [0, 0]], dtype=c),
                np.sqrt(pr1) * np.array([[0, 0], [1, 0]], dtype=c),
                np.sqrt(pr1) * np.array([[0, 0], [0, 1]], dtype=c),
            ]
        choi = np.array(
            [
                [1 - pe * p_reset, 0, 0, eT2],
                [0, pe * p_reset, 0, 0],
                [0, 0, (1 - pe) * p_reset, 0],
                [eT2, 0, 0, 1 - (1 - pe) * p_reset],
            ],
            dtype=np.complex128,
        )
        vals, vecs = np.linalg.eigh(choi)
        return [
            (np.sqrt(abs(vals[i])) * vecs[:, i].reshape(2, 2, order="F")).astype(np.complex128)
            for i in range(4)
        ]


class QubitChannel(KrausChannel):
    """Channel from user-supplied Kraus matrices (noise.py:434-465)."""

    def __init__(self, kraus_ops, wires: Union[int, List[int]] = 0) -> None:
        self._kraus_ops = [
            np.asarray(K.detach().cpu().numpy() if isinstance(K, torch.Tensor) else K, dtype=np.complex128)
            for K in kraus_ops
        ]
        super().__init__(wires=wires)

    def kraus_matrices(self):
        return self._kraus_ops
