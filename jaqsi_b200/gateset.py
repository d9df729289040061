"""Gate library (restates the matrices and structures of jaqsi/gateset.py).

Constant matrices are exact NumPy arrays; parametrised gates keep their angles
(Python floats or torch tensors) and lower to a device-built matrix, so a
recorded circuit never materialises per-gate tensors on the hot path.
"""
from __future__ import annotations

from functools import reduce
from typing import List, Optional, Union

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200.operations import GateStructure, Hermitian, Matrix, Operation, _as_real, cdtype


class Id(Operation):
    """Identity on any number of wires (gateset.py:32-60)."""

    _matrix = np.eye(2, dtype=np.complex128)
    _num_wires = None
    _structure = GateStructure(diagonal=True)
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)
        k = len(self.wires)
        if k > 1:
            self._matrix = np.eye(2**k, dtype=np.complex128)
            self._structure = GateStructure(diagonal=True)


class PauliX(Operation):
    _matrix = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    _num_wires = 1
    _structure = GateStructure(permutation=(1, 0))
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class PauliY(Operation):
    _matrix = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    _num_wires = 1
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class PauliZ(Operation):
    _matrix = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    _num_wires = 1
    _structure = GateStructure(diagonal=True)
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class H(Operation):
    _matrix = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
    _num_wires = 1
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class S(Operation):
    _matrix = np.array([[1, 0], [0, 1j]], dtype=np.complex128)
    _num_wires = 1
    _structure = GateStructure(diagonal=True)
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0) -> None:
        super().__init__(wires=wires)


class SWAP(Operation):
    _matrix = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
    _num_wires = 2
    _structure = GateStructure(permutation=(0, 2, 1, 3))
    is_unitary = True
    is_clifford = True

    def __init__(self, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class RandomUnitary(Operation):
    """Random Hermitian matrix applied as a gate (gateset.py:175-205).

    ``key`` is a ``torch.Generator`` or an integer seed (the reference takes a
    JAX PRNG key; the random stream is therefore not the reference's).
    """

    def __init__(self, wires, key, scale: float = 1.0, record: bool = True) -> None:
        wires_l = list(wires) if isinstance(wires, (list, tuple)) else [wires]
        dim = 2 ** len(wires_l)
        gen = key if isinstance(key, torch.Generator) else torch.Generator().manual_seed(int(key))
        a = torch.randn(dim, dim, generator=gen, dtype=torch.float64)
        b = torch.randn(dim, dim, generator=gen, dtype=torch.float64)
        A = torch.complex(a, b)
        Hm = (A + A.conj().T) / 2.0
        Hm = Hm * (scale / torch.linalg.norm(Hm))
        super().__init__(wires_l, matrix=Hm.numpy(), record=record)


class DiagonalQubitUnitary(Operation):
    """Diagonal unitary given by its diagonal (gateset.py:208-350)."""

    _param_names = ()
    is_unitary = True

    def __init__(self, diag, wires: Union[int, List[int]] = 0, generator=None, scale=None, **kwargs) -> None:
        self.diag = diag
        self._generator = generator
        self._scale = scale
        wires_l = list(wires) if isinstance(wires, (list, tuple)) else [wires]
        expected = 2 ** len(wires_l)
        if tuple(diag.shape) != (expected,):
            raise ValueError(
                f"DiagonalQubitUnitary expects {expected} diagonal entries for {len(wires_l)} wire(s), "
                f"got shape {tuple(diag.shape)}"
            )
        kwargs.setdefault("name", "DiagU")
        mat = torch.diag(diag) if isinstance(diag, torch.Tensor) else np.diag(np.asarray(diag, dtype=np.complex128))
        super().__init__(wires=wires, matrix=mat, **kwargs)
        self._structure = GateStructure(diagonal=True)

    def _jq_lower(self):
        if isinstance(self.diag, torch.Tensor):
            return L.JQ_K_MATRIX, [], self.diag
        return L.JQ_K_CONST, [], np.diag(np.asarray(self.diag, dtype=np.complex128))

    def decompose(self) -> List[Operation]:
        if self._generator is None:
            return super().decompose()
        k = len(self.wires)
        dim = 2**k
        marks = np.asarray(self._generator, dtype=float).reshape(-1)
        signs = np.array([[1 - 2 * ((j >> (k - 1 - i)) & 1) for j in range(dim)] for i in range(k)])
        ops: List[Operation] = []
        for mask in range(1, dim):
            chi = np.ones(dim)
            for i in range(k):
                if (mask >> i) & 1:
                    chi = chi * signs[i]
            alpha = float(marks @ chi) / dim
            if abs(alpha) < 1e-12:
                continue
            word = "".join("Z" if (mask >> i) & 1 else "I" for i in range(k))
            ops.append(PauliRot(2.0 * alpha * self._scale, word, wires=self.wires, record=False))
        return ops


class Barrier(Operation):
    """Visual separator; no effect on the state (gateset.py:353-380)."""

    _matrix = None

    def __init__(self, wires: Union[int, List[int]] = 0) -> None:
        super().__init__(wires=wires)

    def apply_to_state(self, state, n_qubits):
        return state

    def apply_to_density(self, rho, n_qubits):
        return rho


_PAULI_MATRICES = {
    "I": Id._matrix,
    "X": PauliX._matrix,
    "Y": PauliY._matrix,
    "Z": PauliZ._matrix,
}


def _pauli_tensor(word: str) -> np.ndarray:
    return reduce(np.kron, [_PAULI_MATRICES[c] for c in word])


def _pauli_masks(word: str):
    """X/Y and Z/Y position masks of a Pauli word; position i -> bit k-1-i."""
    k = len(word)
    px = pz = 0
    for i, ch in enumerate(word):
        bit = 1 << (k - 1 - i)
        if ch in "XY":
            px |= bit
        if ch in "ZY":
            pz |= bit
        if ch not in "IXYZ":
            raise ValueError(f"invalid Pauli letter {ch!r} in {word!r}")
    return px, pz


def _rot_matrix(theta, pauli: np.ndarray) -> torch.Tensor:
    """cos(theta/2) I - i sin(theta/2) P in torch (gateset.py:399-405)."""
    th = _as_real(theta)
    dim = pauli.shape[0]
    c = torch.cos(th / 2).to(cdtype())
    s = torch.sin(th / 2).to(cdtype())
    P = torch.as_tensor(pauli, dtype=cdtype())
    return c * torch.eye(dim, dtype=cdtype()) - 1j * s * P


def _make_rotation_gate(pauli_class, name: str, kind: int):
    pauli_mat = pauli_class._matrix

    class _RotationGate(Operation):
        __doc__ = f"Rotation about {name[1]}: {name}(t) = exp(-i t/2 {name[1]}) (gateset.py:408-451)."
        _num_wires = 1
        is_unitary = True
        _param_names = ("theta",)
        _structure = GateStructure(diagonal=pauli_class is PauliZ)
        _jq_param_kind = kind  # lowering fixed by the class (simulation._class_lowering)

        def __init__(self, theta, wires: Union[int, List[int]] = 0, **kwargs) -> None:
            self.theta = theta
            if kwargs or type(wires) is not int:
                super().__init__(wires=wires, **kwargs)
            else:  # one int wire, recorded: the circuit-recording hot path
                self._record_fast([wires])

        @property
        def matrix(self) -> torch.Tensor:
            return _rot_matrix(self.theta, pauli_mat)

        def _jq_lower(self):
            return kind, [self.theta], None

        def _jq_static_key(self):
            return (kind,)

        def generator(self) -> Operation:
            return pauli_class(wires=self.wires[0], record=False)

    _RotationGate.__name__ = name
    _RotationGate.__qualname__ = name
    return _RotationGate


RX = _make_rotation_gate(PauliX, "RX", L.JQ_K_RX)
RY = _make_rotation_gate(PauliY, "RY", L.JQ_K_RY)
RZ = _make_rotation_gate(PauliZ, "RZ", L.JQ_K_RZ)

_P0 = np.array([[1, 0], [0, 0]], dtype=np.complex128)
_P1 = np.array([[0, 0], [0, 1]], dtype=np.complex128)


def _make_controlled_gate(target_class, name: str):
    target_mat = target_class._matrix

    class _ControlledGate(Operation):
        __doc__ = f"Controlled-{target_class.__name__[5:]} (gateset.py:459-512)."
        _matrix = np.kron(_P0, Id._matrix) + np.kron(_P1, target_mat)
        _num_wires = 2
        is_unitary = True
        is_controlled = True
        _structure = GateStructure(
            permutation=(0, 1, 3, 2) if target_class is PauliX else (),
            diagonal=target_class is PauliZ,
            controls=1,
        )
        is_clifford = True

        def __init__(self, wires: List[int] = [0, 1], **kwargs) -> None:
            if kwargs or type(wires) is not list or len(wires) != 2 or type(wires[0]) is not int \
                    or type(wires[1]) is not int or wires[0] == wires[1]:
                super().__init__(wires=wires, **kwargs)  # (validates and raises)
            else:  # two distinct int wires, recorded: the circuit-recording hot path
                self._record_fast([wires[0], wires[1]])

        def decompose(self) -> List[Operation]:
            if name != "CZ":
                return super().decompose()
            c, t = self.wires
            return [H(wires=t, record=False), CX(wires=[c, t], record=False), H(wires=t, record=False)]

    _ControlledGate.__name__ = name
    _ControlledGate.__qualname__ = name
    return _ControlledGate


CX = _make_controlled_gate(PauliX, "CX")
CY = _make_controlled_gate(PauliY, "CY")
CZ = _make_controlled_gate(PauliZ, "CZ")


class CCX(Operation):
    """Toffoli (gateset.py:515-548)."""

    _matrix = np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 5, 7, 6]]
    is_controlled = True
    _num_wires = 3
    _structure = GateStructure(permutation=(0, 1, 2, 3, 4, 5, 7, 6), controls=2)
    is_unitary = True

    def __init__(self, wires: List[int] = [0, 1, 2], **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class CSWAP(Operation):
    """Fredkin (gateset.py:551-584)."""

    _matrix = np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 6, 5, 7]]
    is_controlled = True
    _num_wires = 3
    _structure = GateStructure(permutation=(0, 1, 2, 3, 4, 6, 5, 7), controls=1)
    is_unitary = True

    def __init__(self, wires: List[int] = [0, 1, 2], **kwargs) -> None:
        super().__init__(wires=wires, **kwargs)


class ControlledPhaseShift(Operation):
    """diag(1, 1, 1, e^{i phi}) (gateset.py:587-619)."""

    _num_wires = 2
    is_unitary = True
    _param_names = ("phi",)
    is_controlled = True

    def __init__(self, phi, wires: List[int] = [0, 1], **kwargs) -> None:
        self.phi = phi
        super().__init__(wires=wires, **kwargs)
        self._structure = GateStructure(diagonal=True, controls=1)

    @property
    def matrix(self) -> torch.Tensor:
        ph = torch.exp(1j * _as_real(self.phi).to(cdtype()))
        d = torch.stack([torch.ones((), dtype=cdtype())] * 3 + [ph])
        return torch.diag(d)

    def _jq_lower(self):
        return L.JQ_K_CPHASE, [self.phi], None

    def _jq_static_key(self):
        return (L.JQ_K_CPHASE,)


class Rot(Operation):
    """Rot(phi, theta, omega) = RZ(omega) RY(theta) RZ(phi) (gateset.py:622-667)."""

    _num_wires = 1
    is_unitary = True
    _param_names = ("phi", "theta", "omega")
    _jq_param_kind = L.JQ_K_ROT  # lowering fixed by the class (simulation._class_lowering)

    def __init__(self, phi, theta, omega, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        self.phi = phi
        self.theta = theta
        self.omega = omega
        if kwargs or type(wires) is not int:
            super().__init__(wires=wires, **kwargs)
        else:  # one int wire, recorded: the circuit-recording hot path
            self._record_fast([wires])

    @property
    def matrix(self) -> torch.Tensor:
        return (
            _rot_matrix(self.omega, PauliZ._matrix)
            @ _rot_matrix(self.theta, PauliY._matrix)
            @ _rot_matrix(self.phi, PauliZ._matrix)
        )

    def _jq_lower(self):
        return L.JQ_K_ROT, [self.phi, self.theta, self.omega], None

    def _jq_static_key(self):
        return (L.JQ_K_ROT,)

    def decompose(self) -> List[Operation]:
        w = self.wires[0]
        return [RZ(self.phi, wires=w, record=False), RY(self.theta, wires=w, record=False),
                RZ(self.omega, wires=w, record=False)]


class PauliRot(Operation):
    """exp(-i theta/2 P) for a Pauli word P (gateset.py:670-719)."""

    _param_names = ("theta",)
    is_unitary = True

    def __init__(self, theta, pauli_word: str, wires: Union[int, List[int]] = 0, **kwargs) -> None:
        self.theta = theta
        self.pauli_word = pauli_word
        super().__init__(wires=wires, **kwargs)
        if len(pauli_word) != len(self.wires):
            raise ValueError(f"Pauli word {pauli_word!r} does not match {len(self.wires)} wire(s)")
        self._px, self._pz = _pauli_masks(pauli_word)
        self._structure = GateStructure(diagonal=set(pauli_word) <= {"I", "Z"})

    @property
    def matrix(self) -> torch.Tensor:
        return _rot_matrix(self.theta, _pauli_tensor(self.pauli_word))

    def _jq_lower(self):
        return L.JQ_K_PAULIROT, [self.theta], None

    def _jq_static_key(self):
        return (L.JQ_K_PAULIROT, self.pauli_word, 0)

    def generator(self) -> Operation:
        return Hermitian(matrix=_pauli_tensor(self.pauli_word), wires=self.wires, record=False)


def _make_pauli_rotation_subclass(name: str, word: str):
    class _PauliRotSubclass(PauliRot):
        __doc__ = f"{name}(theta) = exp(-i theta/2 {word}) (gateset.py:722-758)."
        _num_wires = len(word)

        def __init__(self, theta, wires=None, **kwargs) -> None:
            if wires is None:
                wires = list(range(len(word)))
            super().__init__(theta, word, wires=wires, **kwargs)

    _PauliRotSubclass.__name__ = name
    _PauliRotSubclass.__qualname__ = name
    return _PauliRotSubclass


RXX = _make_pauli_rotation_subclass("RXX", "XX")
RYY = _make_pauli_rotation_subclass("RYY", "YY")
RZZ = _make_pauli_rotation_subclass("RZZ", "ZZ")
RZX = _make_pauli_rotation_subclass("RZX", "ZX")


class ControlledPauliRot(Operation):
    """PauliRot on the targets when all controls are |1> (gateset.py:764-829)."""

    _param_names = ("theta",)
    is_unitary = True
    is_controlled = True

    def __init__(self, theta, pauli_word: str, wires: List[int], n_controls: int = 1, **kwargs) -> None:
        self.theta = theta
        self.pauli_word = pauli_word
        self.n_controls = n_controls
        wires_l = [wires] if isinstance(wires, int) else list(wires)
        if len(wires_l) != n_controls + len(pauli_word):
            raise ValueError(
                f"ControlledPauliRot expects {n_controls + len(pauli_word)} wires "
                f"({n_controls} control + {len(pauli_word)} target), got {len(wires_l)}."
            )
        super().__init__(wires=wires_l, **kwargs)
        self._px, self._pz = _pauli_masks(pauli_word)
        self._structure = GateStructure(diagonal=set(pauli_word) <= {"I", "Z"}, controls=n_controls)

    @property
    def matrix(self) -> torch.Tensor:
        R = _rot_matrix(self.theta, _pauli_tensor(self.pauli_word))
        d_t = R.shape[0]
        dim = (2**self.n_controls) * d_t
        top = torch.eye(dim - d_t, dtype=cdtype())
        return torch.block_diag(top, R)

    def _jq_lower(self):
        return L.JQ_K_PAULIROT, [self.theta], None

    def _jq_static_key(self):
        return (L.JQ_K_PAULIROT, self.pauli_word, self.n_controls)

    def generator(self) -> Operation:
        P = _pauli_tensor(self.pauli_word)
        d_t = P.shape[0]
        dim = (2**self.n_controls) * d_t
        gen = np.zeros((dim, dim), dtype=np.complex128)
        gen[dim - d_t:, dim - d_t:] = P
        return Hermitian(matrix=gen, wires=self.wires, record=False)


def _make_controlled_rotation_subclass(name: str, axis: str):
    class _CRotation(ControlledPauliRot):
        __doc__ = f"Controlled R{axis} (gateset.py:832-890)."
        _num_wires = 2

        def __init__(self, theta, wires: List[int] = [0, 1], **kwargs) -> None:
            super().__init__(theta, axis, wires=wires, n_controls=1, **kwargs)

        def decompose(self) -> List[Operation]:
            c, t = self.wires
            th = self.theta
            if axis == "Z":
                return [RZ(th / 2, wires=t, record=False), CX(wires=[c, t], record=False),
                        RZ(-th / 2, wires=t, record=False), CX(wires=[c, t], record=False)]
            if axis == "X":
                return [H(wires=t, record=False), RZ(th / 2, wires=t, record=False), CX(wires=[c, t], record=False),
                        RZ(-th / 2, wires=t, record=False), CX(wires=[c, t], record=False), H(wires=t, record=False)]
            return [RX(np.pi / 2, wires=t, record=False), RZ(th / 2, wires=t, record=False),
                    CX(wires=[c, t], record=False), RZ(-th / 2, wires=t, record=False),
                    CX(wires=[c, t], record=False), RX(-np.pi / 2, wires=t, record=False)]

    _CRotation.__name__ = name
    _CRotation.__qualname__ = name
    return _CRotation


CRX = _make_controlled_rotation_subclass("CRX", "X")
CRY = _make_controlled_rotation_subclass("CRY", "Y")
CRZ = _make_controlled_rotation_subclass("CRZ", "Z")


def build_parity_observable(qubit_group: List[int]) -> Hermitian:
    """Z-parity observable on *qubit_group* (gateset.py:892-910), tagged with
    its Pauli word so the backend measures it without a dense matrix."""
    Z = PauliZ._matrix
    mat = reduce(np.kron, [Z] * len(qubit_group))
    obs = Hermitian(matrix=mat, wires=qubit_group, record=False)
    obs._pauli_label = "Z" * len(qubit_group)
    return obs
