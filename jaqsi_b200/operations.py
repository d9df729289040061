"""Operation model (restates the circuit-facing part of jaqsi/operations.py).

An :class:`Operation` records itself on the active tape when created
(jaqsi/operations.py:229-273).  Its matrix is a PyTorch tensor in the active
complex dtype; the simulation backend never builds it on the hot path, it
lowers each op to a compact descriptor (:meth:`Operation._jq_lower`) whose
matrix the GPU builds from the op's angles.
"""
from __future__ import annotations

import string
from functools import lru_cache, reduce
from typing import Callable, List, NamedTuple, Optional, Tuple, Union

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200.tape import _local as _tape_local
from jaqsi_b200.tape import active_tape, recording  # noqa: F401  (re-export)

Matrix = Union[np.ndarray, torch.Tensor]

_DEFAULT_DTYPE = [torch.complex128]


def set_default_dtype(dtype: torch.dtype) -> None:
    """Select complex64 or complex128 as the default simulation dtype.

    The reference picks complex128 iff ``jax_enable_x64`` is set
    (jaqsi/operations.py:30-43); here the choice is explicit, and
    ``Script.execute(dtype=...)`` overrides it per call.
    """
    if dtype not in (torch.complex64, torch.complex128):
        raise ValueError(f"dtype must be torch.complex64 or torch.complex128, got {dtype}")
    _DEFAULT_DTYPE[0] = dtype


def cdtype() -> torch.dtype:
    """The active complex dtype (complex128 unless changed)."""
    return _DEFAULT_DTYPE[0]


def rdtype(c: Optional[torch.dtype] = None) -> torch.dtype:
    """Real dtype matching complex dtype *c* (default: the active one)."""
    c = c or cdtype()
    return torch.float32 if c == torch.complex64 else torch.float64


def _as_real(x, like: Optional[torch.Tensor] = None) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(torch.float64)
    return torch.tensor(float(x), dtype=torch.float64)


def _to_tensor(m: Matrix, dtype: Optional[torch.dtype] = None) -> torch.Tensor:
    dtype = dtype or cdtype()
    if isinstance(m, torch.Tensor):
        return m.to(dtype)
    return torch.as_tensor(np.asarray(m), dtype=dtype)


@lru_cache(maxsize=256)
def _einsum_subscript(n: int, k: int, target_axes: Tuple[int, ...]) -> str:
    """Subscript contracting a (2,)*2k gate with axes *target_axes* of a rank-n
    tensor, restoring axis order (jaqsi/operations.py:46-77)."""
    letters = string.ascii_letters
    state_idx = list(letters[:n])
    contracted = [state_idx[ax] for ax in target_axes]
    new_out = [letters[n + i] for i in range(k)]
    result_idx = list(state_idx)
    for i, ax in enumerate(target_axes):
        result_idx[ax] = new_out[i]
    return "".join(new_out + contracted) + "," + "".join(state_idx) + "->" + "".join(result_idx)


def _contract(tensor: torch.Tensor, gate: torch.Tensor, k: int, axes) -> torch.Tensor:
    return torch.einsum(_einsum_subscript(tensor.dim(), k, tuple(axes)), gate, tensor)


class GateStructure(NamedTuple):
    """Static matrix guarantees (jaqsi/operations.py:176-185).

    ``permutation[i]`` is the input column of output row i; controls are the
    leading wires, active only when all are one.
    """

    permutation: Tuple[int, ...] = ()
    diagonal: bool = False
    controls: int = 0


class Operation:
    """Base class of gates, observables and channels (jaqsi/operations.py:188).

    Attributes:
        _matrix: class-level constant matrix (exact NumPy) or per-instance
            matrix (NumPy constant or torch tensor, possibly requiring grad).
        _num_wires: expected wire count (``None`` = any).
        _param_names: parameter attribute names, in order.
        is_unitary: whether the matrix is unitary; the adjoint gradient is
            used only when every op on the tape sets it (operations.py:223).
    """

    is_controlled = False
    _structure = GateStructure()
    is_clifford = False
    is_unitary = False

    _matrix: Optional[Matrix] = None
    _num_wires: Optional[int] = None
    _param_names: Tuple[str, ...] = ()

    def __init__(
        self,
        wires: Union[int, List[int]] = 0,
        matrix: Optional[Matrix] = None,
        record: bool = True,
        name: Optional[str] = None,
    ) -> None:
        # (hot: runs once per recorded op on every call of a circuit)
        self.name = name or self.__class__.__name__
        ws = list(wires) if isinstance(wires, (list, tuple)) else [wires]
        self._wires = ws
        nw = self._num_wires
        if nw is not None and len(ws) != nw:
            raise ValueError(f"{self.name} expects {nw} wire(s), got {len(ws)}: {ws}")
        if len(ws) > 1 and len(ws) != len(set(ws)):
            raise ValueError(f"{self.name} received duplicate wires: {ws}")
        if matrix is not None:
            self._matrix = matrix
            self._structure = GateStructure()
        if record:
            stack = getattr(_tape_local, "stack", None)
            if stack:
                stack[-1].append(self)

    def _record_fast(self, ws: List[int]) -> None:
        """Common tail of ``__init__`` for subclasses' hot path: class name, no
        instance matrix, recorded on the active tape.  *ws* is a fresh wire
        list the caller has already validated."""
        self.name = type(self).__name__
        self._wires = ws
        stack = getattr(_tape_local, "stack", None)
        if stack:
            stack[-1].append(self)

    # -- basic properties ----------------------------------------------------
    @property
    def wires(self) -> List[int]:
        return self._wires

    @wires.setter
    def wires(self, wires) -> None:
        self._wires = list(wires) if isinstance(wires, (list, tuple)) else [wires]

    @property
    def parameters(self) -> list:
        return [getattr(self, n) for n in self._param_names]

    def __repr__(self) -> str:
        params = self.parameters
        if params:
            txt = ", ".join(
                f"{float(v):.4f}" if isinstance(v, (float, np.floating)) or (isinstance(v, torch.Tensor) and v.numel() == 1)
                else str(v)
                for v in params
            )
            return f"{self.name}({txt}, wires={self.wires})"
        return f"{self.name}(wires={self.wires})"

    @property
    def matrix(self) -> torch.Tensor:
        """The op's matrix as a torch tensor in the active complex dtype."""
        if self._matrix is None:
            raise NotImplementedError(f"{self.__class__.__name__} does not define a matrix.")
        return _to_tensor(self._matrix)

    def decompose(self) -> List["Operation"]:
        raise NotImplementedError(f"{self.__class__.__name__} does not define a decomposition.")

    # -- lowering to the C ABI -----------------------------------------------------
    def _jq_lower(self):
        """(kind, angles, payload) describing how the device builds the matrix.

        ``payload`` is a NumPy constant (JQ_K_CONST) or a torch tensor
        (JQ_K_MATRIX, gathered per call so gradients reach it).
        """
        m = self._matrix
        if m is None:
            raise NotImplementedError(f"{self.__class__.__name__} does not define a matrix.")
        if isinstance(m, torch.Tensor):
            return L.JQ_K_MATRIX, [], m
        cls = self.__class__
        if m is cls._matrix:
            # class-constant matrix: converted once per class
            c = cls.__dict__.get("_jq_const")
            if c is None:
                c = np.asarray(m, dtype=np.complex128)
                cls._jq_const = c
            return L.JQ_K_CONST, [], c
        return L.JQ_K_CONST, [], np.asarray(m, dtype=np.complex128)

    def _jq_static_key(self):
        """Hashable part of the lowering that selects the execution plan."""
        cls = self.__class__
        if cls._matrix is not None and self._matrix is cls._matrix and not isinstance(self._matrix, torch.Tensor):
            return (cls.__name__,)
        kind, _, payload = self._jq_lower()
        if kind == L.JQ_K_CONST:
            if self.__class__._matrix is not None and self._matrix is self.__class__._matrix:
                return (self.__class__.__name__,)
            return ("const", payload.shape, payload.tobytes())
        return (kind,)

    # -- algebra (jaqsi/operations.py:367-532) ---------------------------------------
    def _update_tape_operation(self, op: "Operation") -> None:
        tape = active_tape()
        if tape is not None:
            if tape and tape[-1] is self:
                tape[-1] = op
            else:
                tape.append(op)

    def dagger(self) -> "Operation":
        """U^dagger on the same wires, replacing U on the tape if it was last."""
        mat = self.matrix.conj().transpose(-2, -1)
        op = Operation(wires=self.wires, matrix=mat, record=False)
        op.is_unitary = self.is_unitary
        st = self._structure
        perm = st.permutation
        if perm:
            perm = tuple(perm.index(i) for i in range(len(perm)))
        op._structure = st._replace(permutation=perm)
        self._update_tape_operation(op)
        return op

    def power(self, power: int) -> "Operation":
        mat = torch.linalg.matrix_power(self.matrix, power)
        op = Operation(wires=self.wires, matrix=mat, record=False)
        op.is_unitary = self.is_unitary
        self._update_tape_operation(op)
        return op

    def __mul__(self, other):
        if isinstance(other, Operation):
            return self.__matmul__(other)
        op = Operation(wires=self.wires, matrix=other * self.matrix, record=False)
        self._update_tape_operation(op)
        return op

    __rmul__ = __mul__

    def __add__(self, other: "Operation") -> "Operation":
        if sorted(self.wires) != sorted(other.wires):
            raise ValueError(
                "Can only add operations acting on the same set of wires, "
                f"got {self.wires} and {other.wires}"
            )
        return Operation(wires=self.wires, matrix=self.matrix + other.matrix, record=False)

    def prod(self, *ops: "Operation") -> "Operation":
        if not ops:
            return self
        all_ops = (self,) + ops
        all_wires: List[int] = []
        for op in all_ops:
            for w in op.wires:
                if w not in all_wires:
                    all_wires.append(w)
        n = len(all_wires)
        mat = _embed_matrix(all_ops[0].matrix, all_ops[0].wires, all_wires, n)
        for op in all_ops[1:]:
            mat = mat @ _embed_matrix(op.matrix, op.wires, all_wires, n)
        names = "*".join(op.name for op in all_ops)
        op = Operation(wires=all_wires, matrix=mat, name=f"Prod({names})", record=False)
        op.is_unitary = all(o.is_unitary for o in all_ops)
        return op

    def __matmul__(self, other):
        if not isinstance(other, Operation):
            return NotImplemented
        return self.prod(other)

    # -- dense helpers (test oracles of the reference: operations.py:534-644) --------
    def lifted_matrix(self, n_qubits: int) -> torch.Tensor:
        """The full 2^n x 2^n matrix of this op."""
        dim = 2**n_qubits
        eye = torch.eye(dim, dtype=cdtype())
        cols = [self.apply_to_state(eye[:, j], n_qubits) for j in range(dim)]
        return torch.stack(cols, dim=1)

    def apply_to_state(self, state: torch.Tensor, n_qubits: int) -> torch.Tensor:
        k = len(self.wires)
        gate = self.matrix.reshape((2,) * 2 * k)
        psi = state.reshape((2,) * n_qubits).to(gate.dtype)
        return _contract(psi, gate, k, self.wires).reshape(2**n_qubits)

    def apply_to_density(self, rho: torch.Tensor, n_qubits: int) -> torch.Tensor:
        k = len(self.wires)
        U = self.matrix.reshape((2,) * 2 * k)
        r = rho.reshape((2,) * 2 * n_qubits).to(U.dtype)
        r = _contract(r, U, k, self.wires)
        r = _contract(r, U.conj(), k, [w + n_qubits for w in self.wires])
        return r.reshape(2**n_qubits, 2**n_qubits)


def _embed_matrix(mat: torch.Tensor, op_wires, all_wires, n_total: int) -> torch.Tensor:
    """Tensor *mat* with identities on the missing wires and order the qubits
    as *all_wires* (jaqsi/operations.py:107-149)."""
    k = len(op_wires)
    if k == n_total and list(op_wires) == list(all_wires):
        return mat
    missing = [w for w in all_wires if w not in op_wires]
    full = mat
    for _ in missing:
        full = torch.kron(full, torch.eye(2, dtype=mat.dtype))
    current = list(op_wires) + missing
    if current != list(all_wires):
        perm = [current.index(w) for w in all_wires]
        t = full.reshape([2] * (2 * n_total))
        t = t.permute(perm + [p + n_total for p in perm])
        full = t.reshape(2**n_total, 2**n_total)
    return full


class Hermitian(Operation):
    """A Hermitian observable or gate given by its matrix (operations.py:647)."""

    def __init__(self, matrix: Matrix, wires: Union[int, List[int]] = 0, record: bool = True) -> None:
        if not isinstance(matrix, torch.Tensor):
            matrix = np.asarray(matrix, dtype=np.complex128)
        super().__init__(wires=wires, matrix=matrix, record=record)

    def __rmul__(self, coeff_fn):
        """``coeff_fn * Hermitian`` -> a one-term ParametrizedHamiltonian
        (jaqsi/operations.py:683-702)."""
        if isinstance(coeff_fn, Operation):
            return Operation.__mul__(self, coeff_fn)
        if not callable(coeff_fn):
            raise TypeError(f"Left operand of `* Hermitian` must be callable, got {type(coeff_fn)}")
        from jaqsi_b200.evolution import ParametrizedHamiltonian

        return ParametrizedHamiltonian(terms=[(coeff_fn, self._matrix, self.wires)])

    def evolve(self, name: Optional[str] = None, **odeint_kwargs):
        """Gate factory ``(t, wires=0) -> exp(-i t H)`` (jaqsi/operations.py:704-720)."""
        from jaqsi_b200.evolution import Evolution

        return Evolution.evolve(self, name=name, **odeint_kwargs)
