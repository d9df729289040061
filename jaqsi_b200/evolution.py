"""Pulse-level gates: time evolution under a parametrised Hamiltonian.

The reference's surface (jaqsi/evolution.py, jaqsi/operations.py:683-860):
``coeff_fn * Hermitian(H, wires)`` builds a :class:`ParametrizedHamiltonian`
``H(t) = sum_i f_i(p_i, t) H_i``; ``H.evolve(**options)`` returns a gate
factory ``(coeff_args, T) -> PendingEvolution``.  The gate's unitary
``U = T exp(-i int_{t0}^{t1} H(t) dt)`` is solved lazily: ``resolve_pending``
(jaqsi/evolution.py:730-773) solves every pending gate of a tape in batches,
and the simulation calls it before running the tape
(jaqsi/simulation.py:713).

Solvers (``solver=``, as in the reference, evolution.py:91):
- ``"magnus2"`` / ``"magnus4"``: the commutator-free Magnus schemes on
  ``magnus_steps`` fixed steps (midpoint rule; CFM4:2 of Blanes and Moan,
  exp(Omega_b) exp(Omega_a) per step).  All gates of a group run in one GPU
  launch (``jq_magnus_product``: one CTA per gate, exponentials by scaling
  and squaring, an ordered tree product); gradients w.r.t. the pulse
  parameters come from the kernel's reverse pass (``jq_magnus_product_grad``)
  chained through the coefficient functions by autograd.
- ``"dopri8"`` / ``"dopri5"`` (the reference's adaptive integrators): a single
  term with a concrete matrix is solved in closed form, as the reference does
  (evolution.py:354-405): ``U = V exp(-i lambda A) V^H`` with the pulse area
  ``A = int f dt`` from composite Gauss-Legendre quadrature; several terms run
  the 4th-order Magnus scheme on the finest grid the kernel takes
  (``DOPRI_MAGNUS_STEPS``) instead of an adaptive step-size controller.

Coefficient functions are called with torch tensors: ``f(params, t)`` with
``t`` a 1-D tensor of times (broadcasting), or, if that fails, one scalar
time at a time under ``torch.func.vmap``.
"""
from __future__ import annotations

import ctypes
import math
import threading
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200.operations import Operation, cdtype

__all__ = ["ParametrizedHamiltonian", "Evolution", "PendingEvolution", "resolve_pending"]

# Magnus steps used for adaptive-solver requests with several terms (the
# kernel's limit for 2x2 and 4x4 gates is 2048 sub-steps = 1024 CFM4 steps).
DOPRI_MAGNUS_STEPS = {2: 1024, 4: 1024, 8: 256}
# Composite Gauss-Legendre quadrature of the closed-form pulse area.
_GL_POINTS = 16
_GL_PANELS = 64


def _wlist(w) -> List[int]:
    return [int(w)] if isinstance(w, (int, np.integer)) else [int(x) for x in w]


def _as_matrix(H) -> torch.Tensor:
    if isinstance(H, torch.Tensor):
        return H.to(torch.complex128)
    return torch.as_tensor(np.asarray(H, dtype=np.complex128))


class ParametrizedHamiltonian:
    """``H(t) = sum_i f_i(params_i, t) H_i`` (jaqsi/operations.py:722-860)."""

    def __init__(self, terms: List[Tuple[Callable, Any, Union[int, List[int]]]]) -> None:
        if len(terms) == 0:
            raise ValueError("ParametrizedHamiltonian needs at least one term.")
        first_wires = _wlist(terms[0][2])
        for _, _, w in terms[1:]:
            if _wlist(w) != first_wires:
                raise ValueError(
                    "All terms of a ParametrizedHamiltonian must currently act on the same wires; got "
                    f"{_wlist(w)} vs. {first_wires}. Multi-wire broadcasting across terms is not yet supported."
                )
        first_shape = tuple(_as_matrix(terms[0][1]).shape)
        for _, H, _ in terms[1:]:
            if tuple(_as_matrix(H).shape) != first_shape:
                raise ValueError(
                    f"All term matrices must have the same shape; got {tuple(_as_matrix(H).shape)} vs. {first_shape}."
                )
        self._terms = tuple((fn, _as_matrix(H), _wlist(w)) for fn, H, w in terms)
        self.wires: List[int] = list(first_wires)

    @property
    def coeff_fns(self) -> Tuple[Callable, ...]:
        return tuple(fn for fn, _, _ in self._terms)

    @property
    def H_mats(self) -> Tuple[torch.Tensor, ...]:
        return tuple(H for _, H, _ in self._terms)

    @property
    def n_terms(self) -> int:
        return len(self._terms)

    def __add__(self, other: "ParametrizedHamiltonian") -> "ParametrizedHamiltonian":
        if not isinstance(other, ParametrizedHamiltonian):
            return NotImplemented
        return ParametrizedHamiltonian(terms=list(self._terms) + list(other._terms))

    def __neg__(self) -> "ParametrizedHamiltonian":
        return ParametrizedHamiltonian(
            terms=[((lambda f: lambda p, t: -f(p, t))(fn), H, w) for fn, H, w in self._terms])

    def __sub__(self, other: "ParametrizedHamiltonian") -> "ParametrizedHamiltonian":
        if not isinstance(other, ParametrizedHamiltonian):
            return NotImplemented
        return self + (-other)

    def evolve(self, name: Optional[str] = None, **odeint_kwargs) -> Callable:
        """Gate factory ``(coeff_args, T) -> Operation`` (Evolution.evolve)."""
        return Evolution.evolve(self, name=name, **odeint_kwargs)


# ---------------------------------------------------------------------------
# coefficient values and the GPU product of exponentials
# ---------------------------------------------------------------------------
def _coeff_values(fn: Callable, params, t: torch.Tensor) -> torch.Tensor:
    """fn(params, t) at every time of the 1-D tensor t, as complex128."""
    try:
        v = fn(params, t)
        v = torch.as_tensor(v)
        if v.shape != t.shape:
            v = v.expand(t.shape) if v.dim() == 0 else None
    except Exception:
        v = None
    if v is None:
        v = torch.func.vmap(lambda tt: torch.as_tensor(fn(params, tt)))(t)
    return v.to(device=t.device, dtype=torch.complex128)


class _MagnusProduct(torch.autograd.Function):
    """U[g] = prod_m expm(sum_i w[g, m, i] A[g, i]) on the GPU
    (jq_magnus_product; backward: jq_magnus_product_grad)."""

    @staticmethod
    def forward(ctx, A, w):
        G, nt, d, _ = A.shape
        M = w.shape[1]
        A = A.contiguous()
        w = w.contiguous()
        U = torch.empty((G, d, d), dtype=torch.complex128, device=w.device)
        st = ctypes.c_void_p(torch.cuda.current_stream(w.device).cuda_stream)
        L.check(L.lib().jq_magnus_product(G, d, nt, M, ctypes.c_void_p(A.data_ptr()), nt * d * d,
                                          ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(U.data_ptr()), st))
        ctx.save_for_backward(A, w)
        return U

    @staticmethod
    def backward(ctx, gU):
        A, w = ctx.saved_tensors
        G, nt, d, _ = A.shape
        M = w.shape[1]
        gU = gU.to(torch.complex128).contiguous()
        gw = torch.empty_like(w)
        st = ctypes.c_void_p(torch.cuda.current_stream(w.device).cuda_stream)
        L.check(L.lib().jq_magnus_product_grad(G, d, nt, M, ctypes.c_void_p(A.data_ptr()), nt * d * d,
                                               ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(gU.data_ptr()),
                                               ctypes.c_void_p(gw.data_ptr()), st))
        return None, gw


_SQ3 = math.sqrt(3.0)
# CFM4:2 nodes and weights (Blanes and Moan 2006), as jaqsi/evolution.py:239-243
_C1, _C2 = 0.5 - _SQ3 / 6.0, 0.5 + _SQ3 / 6.0
_A1, _A2 = 0.25 + _SQ3 / 6.0, 0.25 - _SQ3 / 6.0


def _magnus_weights(fns, params, t0, t1, n_steps: int, order: int, device) -> torch.Tensor:
    """w [M, n_terms]: the sub-step weights of one gate (M = n_steps for the
    midpoint rule, 2 n_steps for CFM4:2, sub-step 2k = Omega_a, 2k+1 = Omega_b)."""
    t0 = torch.as_tensor(t0, dtype=torch.float64, device=device)
    t1 = torch.as_tensor(t1, dtype=torch.float64, device=device)
    h = (t1 - t0) / n_steps
    k = torch.arange(n_steps, dtype=torch.float64, device=device)
    if order == 2:
        t = t0 + (k + 0.5) * h
        c = torch.stack([_coeff_values(f, p, t) for f, p in zip(fns, params)], dim=-1)  # [S, nt]
        return h * c
    ta = t0 + (k + _C1) * h
    tb = t0 + (k + _C2) * h
    c1 = torch.stack([_coeff_values(f, p, ta) for f, p in zip(fns, params)], dim=-1)
    c2 = torch.stack([_coeff_values(f, p, tb) for f, p in zip(fns, params)], dim=-1)
    wa = h * (_A1 * c1 + _A2 * c2)
    wb = h * (_A2 * c1 + _A1 * c2)
    return torch.stack([wa, wb], dim=1).reshape(2 * n_steps, len(fns))


def _gauss_legendre(device) -> Tuple[torch.Tensor, torch.Tensor]:
    x, wt = np.polynomial.legendre.leggauss(_GL_POINTS)
    return (torch.tensor(x, dtype=torch.float64, device=device), torch.tensor(wt, dtype=torch.float64, device=device))


def _pulse_area(fn, params, t0, t1, device) -> torch.Tensor:
    """int_{t0}^{t1} fn(params, t) dt by composite Gauss-Legendre quadrature."""
    x, wt = _gauss_legendre(device)
    t0 = torch.as_tensor(t0, dtype=torch.float64, device=device)
    t1 = torch.as_tensor(t1, dtype=torch.float64, device=device)
    panel = (t1 - t0) / _GL_PANELS
    starts = t0 + panel * torch.arange(_GL_PANELS, dtype=torch.float64, device=device)
    t = (starts[:, None] + panel * (x[None, :] + 1.0) / 2.0).reshape(-1)
    v = _coeff_values(fn, params, t).reshape(_GL_PANELS, _GL_POINTS)
    return (v * wt[None, :]).sum() * panel / 2.0


# ---------------------------------------------------------------------------
# gates
# ---------------------------------------------------------------------------
class PendingEvolution(Operation):
    """Time-evolution gate whose unitary is solved lazily
    (jaqsi/evolution.py:692-727): batched with the other pending gates of a
    tape by :func:`resolve_pending`, or alone on first access of ``matrix``."""

    is_unitary = True

    def __init__(self, wires, name, spec: tuple, params: tuple, t0, t1) -> None:
        super().__init__(wires=wires, name=name)
        self._matrix = None
        self._spec = spec      # (H_mats, coeff_fns, solver, steps, closed_form)
        self._params = params  # one parameter set per term
        self._t0, self._t1 = t0, t1

    @property
    def matrix(self) -> torch.Tensor:
        if self._matrix is None:
            resolve_pending([self])
        return self._matrix

    def _jq_lower(self):
        if self._matrix is None:
            resolve_pending([self])
        return super()._jq_lower()


class Evolution:
    """Gate factories for static and time-dependent Hamiltonians
    (jaqsi/evolution.py:28-690)."""

    _solver_defaults: dict = {
        "max_steps": 2**13,
        "throw": True,
        "solver": "dopri8",
        "magnus_steps": 256,
        "host_offload": False,
        "closed_form": True,
    }
    _valid_solvers = ("dopri8", "dopri5", "magnus2", "magnus4")
    _lock = threading.Lock()

    @classmethod
    def set_solver_defaults(cls, **kwargs) -> None:
        """Update the defaults of later ``evolve`` calls (keys as in
        ``_solver_defaults``; ``host_offload`` is accepted and has no
        effect: the solves run on the GPU)."""
        for k, v in kwargs.items():
            if k not in cls._solver_defaults:
                raise ValueError(f"Unknown solver default {k!r}")
            if k == "solver" and v not in cls._valid_solvers:
                raise ValueError(f"Unknown solver {v!r}; expected one of {cls._valid_solvers}")
            with cls._lock:
                cls._solver_defaults[k] = v

    @classmethod
    def _options(cls, kw: dict) -> Tuple[str, int, bool]:
        solver = str(kw.pop("solver", cls._solver_defaults["solver"]))
        if solver not in cls._valid_solvers:
            raise ValueError(f"Unknown solver {solver!r}; expected one of {cls._valid_solvers}")
        steps = int(kw.pop("magnus_steps", cls._solver_defaults["magnus_steps"]))
        closed = bool(kw.pop("closed_form", cls._solver_defaults["closed_form"]))
        for k in ("atol", "rtol", "max_steps", "throw"):  # adaptive-controller settings
            kw.pop(k, None)
        if kw:
            raise TypeError(f"unexpected solver options {sorted(kw)}")
        return solver, steps, closed

    @classmethod
    def evolve(cls, hamiltonian, name: Optional[str] = None, **odeint_kwargs) -> Callable:
        """Static Hermitian: ``(t, wires=0) -> exp(-i t H)``; parametrised
        Hamiltonian: ``(coeff_args, T) -> PendingEvolution``
        (jaqsi/evolution.py:407-443)."""
        from jaqsi_b200.operations import Hermitian

        if isinstance(hamiltonian, Hermitian):
            H = _as_matrix(hamiltonian.matrix)

            def _apply_static(t, wires=0) -> Operation:
                tt = torch.as_tensor(t, dtype=torch.float64)
                U = torch.linalg.matrix_exp(-1j * tt.to(torch.complex128) * H.to(tt.device))
                op = Operation(wires=wires, matrix=U, name=name)
                op.is_unitary = True
                return op

            return _apply_static
        if not isinstance(hamiltonian, ParametrizedHamiltonian):
            raise TypeError(f"evolve() expects a Hermitian or ParametrizedHamiltonian, got {type(hamiltonian)}")
        solver, steps, closed = cls._options(dict(odeint_kwargs))
        ph = hamiltonian
        dim = ph.H_mats[0].shape[0]
        if dim not in (2, 4, 8):
            raise ValueError(f"pulse gates act on 1 to 3 qubits (matrix dimension 2, 4 or 8), got {dim}")
        spec = (ph.H_mats, ph.coeff_fns, solver, steps, closed)

        def _apply(coeff_args, T) -> Operation:
            params = tuple(coeff_args) if isinstance(coeff_args, (list, tuple)) else (coeff_args,)
            if len(params) != ph.n_terms:
                raise ValueError(
                    f"Expected {ph.n_terms} parameter set(s) for a {ph.n_terms}-term ParametrizedHamiltonian, "
                    f"got {len(params)}.")
            Tt = torch.as_tensor(T, dtype=torch.float64) if not isinstance(T, torch.Tensor) else T
            if Tt.dim() == 0:
                t0, t1 = torch.zeros((), dtype=torch.float64), Tt
            else:
                t0, t1 = Tt[0], Tt[1]
            return PendingEvolution(ph.wires, name, spec, params, t0, t1)

        return _apply


# ---------------------------------------------------------------------------
# batched solve of a tape's pending gates
# ---------------------------------------------------------------------------
def _on_device(p, dev):
    if isinstance(p, torch.Tensor):
        return p.to(dev)
    if isinstance(p, (np.ndarray, list, tuple)):
        return torch.as_tensor(np.asarray(p, dtype=np.float64), device=dev)
    return p


def _closed_form(op: PendingEvolution, dev) -> torch.Tensor:
    """Single concrete term: U = V exp(-i lambda int f dt) V^H
    (jaqsi/evolution.py:354-405 integrates the same scalar pulse area)."""
    H = op._spec[0][0].detach().cpu().numpy()
    lam, V = np.linalg.eigh(H)
    area = _pulse_area(op._spec[1][0], _on_device(op._params[0], dev), op._t0, op._t1, dev)
    Vt = torch.as_tensor(V, dtype=torch.complex128, device=dev)
    phase = torch.exp(-1j * torch.as_tensor(lam, dtype=torch.float64, device=dev) * area)
    return (Vt * phase[None, :]) @ Vt.conj().T


def _group_key(op: PendingEvolution) -> tuple:
    H_mats, _, solver, steps, closed = op._spec
    dim, nt = int(H_mats[0].shape[0]), len(H_mats)
    if solver in ("dopri8", "dopri5") and closed and nt == 1:
        return ("closed",)
    order = 2 if solver == "magnus2" else 4
    n = steps if solver.startswith("magnus") else DOPRI_MAGNUS_STEPS[dim]
    return ("magnus", dim, nt, order, n)


def resolve_pending(tape: Sequence[Operation]) -> List[int]:
    """Solve every unresolved :class:`PendingEvolution` of *tape*: the gates of
    one Magnus group (matrix size, term count, scheme, step count) in one GPU
    launch, closed-form gates one by one.  Returns the group sizes
    (jaqsi/evolution.py:730-773)."""
    groups: Dict[tuple, List[PendingEvolution]] = {}
    for op in tape:
        if isinstance(op, PendingEvolution) and op._matrix is None:
            groups.setdefault(_group_key(op), []).append(op)
    if not groups:
        return []
    from jaqsi_b200.simulation import _device

    dev = _device()
    sizes = []
    for key, ops in groups.items():
        sizes.append(len(ops))
        if key[0] == "closed":
            for op in ops:
                op._matrix = _closed_form(op, dev)
            continue
        _, dim, nt, order, n = key
        A = torch.stack([torch.stack([-1j * H.to(dev) for H in op._spec[0]]) for op in ops])
        w = torch.stack([
            _magnus_weights(op._spec[1], tuple(_on_device(p, dev) for p in op._params), op._t0, op._t1, n, order,
                            dev)
            for op in ops
        ])
        U = _MagnusProduct.apply(A, w)
        for i, op in enumerate(ops):
            op._matrix = U[i]
    return sizes
