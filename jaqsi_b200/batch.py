"""Batched uneven instances: expectation values and full adjoint gradients of
many independent circuits (different qubit counts, depths and parameters) in
one CUDA-graph launch of libjqsim's ``jq_batch`` path.

This is the gradient-workload form of the reference's batched execution
(``Script.execute`` under vmap / shard_map, jaqsi/script.py:426-434 and
:87-125), for circuits that do not share one structure.  Instances with the
same structure share one plan.  Small instances run one per warp, mid-size
ones one per CTA with the whole state in shared memory, larger ones as
batched tile passes or, up to three qubits above the
per-CTA limit, one per thread-block cluster with the state split over the
cluster's shared memory; the split is autotunable (:meth:`BatchedGradients.autotune`).

Example::

    tapes = [(tape_i, n_i, [jq.PauliZ(0)]) for ...]
    bg = BatchedGradients(tapes, dtype=torch.complex64)
    expvals, grads = bg.run()            # concatenated over instances
    ev_i, g_i = bg.split(expvals, grads)[i]
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib as L
from .simulation import (Lowered, _device, _lower_obs, _resolve_dtype, _stream, get_plan, lower_tape)

__all__ = ["BatchedGradients"]


def _all_angles_trainable(lw: Lowered) -> Lowered:
    """The same lowering with every op that has angles marked as trainable, so
    the plan accumulates a gradient for every angle slot (float angles
    included)."""
    out = Lowered()
    out.angles = lw.angles
    out.mats = lw.mats
    out.unitary = lw.unitary
    keys = []
    for st in lw.statics:
        kind, wires, struct, angle_slot, mat_slot, mat_is_diag, px, pz, nctrl, payload, grad, unitary = st
        if angle_slot >= 0:
            grad = 1
        out.statics.append((kind, wires, struct, angle_slot, mat_slot, mat_is_diag, px, pz, nctrl, payload, grad,
                            unitary))
    for k, st in zip(lw.key, out.statics):
        skey, wires, struct, _, unitary, mat_is_diag = k
        keys.append((skey, wires, struct, st[10], unitary, mat_is_diag))
    out.key = ("all-trainable",) + tuple(keys)
    return out


class BatchedGradients:
    """Forward + adjoint of a fixed list of instances ``(tape, n_qubits, obs)``.

    Every instance must be a unitary statevector circuit whose parameters are
    angles (no matrix-valued arguments).  :meth:`run` returns the
    concatenated expectation values (``n_obs`` per instance) and gradients of
    ``sum_o ct_o <O_o>`` with respect to every angle of every instance, in
    recording order (``n_angles`` per instance).
    """

    def __init__(self, instances: Sequence[Tuple[list, int, list]], dtype=None, config: Optional[dict] = None,
                 tune: Optional[dict] = None):
        if len(instances) == 0:
            raise ValueError("BatchedGradients needs at least one instance")
        self.dtype = _resolve_dtype(dtype)
        self.device = _device()
        tune = dict(tune) if tune is not None else {"jit": -1}
        self._plans = []
        index = {}
        plan_of: List[int] = []
        values: List[float] = []
        self.n_angles: List[int] = []
        self.n_obs: List[int] = []
        for tape, n, obs in instances:
            lw = _all_angles_trainable(lower_tape(tape, n))
            if lw.mats:
                raise ValueError("BatchedGradients: matrix-valued gate arguments are not supported")
            if not lw.unitary:
                raise ValueError("BatchedGradients: noise channels need the density-matrix path")
            specs, okey = _lower_obs(list(obs), n)
            plan = get_plan(lw, specs, okey, n, L.JQ_STATEVECTOR, self.dtype, tune)
            key = id(plan)
            if key not in index:
                index[key] = len(self._plans)
                self._plans.append(plan)
            plan_of.append(index[key])
            values.extend(float(a) for a in lw.angles)
            self.n_angles.append(len(lw.angles))
            self.n_obs.append(len(specs))
        self._lib = L.lib()
        handles = (ctypes.c_void_p * len(self._plans))(*[p.handle for p in self._plans])
        po = (ctypes.c_int32 * len(plan_of))(*plan_of)
        cfg = None
        if config is not None:
            cfg = L.JqBatchConfig(**config)
        h = ctypes.c_void_p()
        L.check(self._lib.jq_batch_build(handles, len(self._plans), po, len(plan_of),
                                         ctypes.byref(cfg) if cfg is not None else None, ctypes.byref(h)))
        self.handle = h
        na = ctypes.c_int64()
        no = ctypes.c_int64()
        L.check(self._lib.jq_batch_info(self.handle, ctypes.byref(na), ctypes.byref(no), None, None))
        self.n_angles_total = na.value
        self.n_obs_total = no.value
        dev = self.device
        self.angles = torch.tensor(values if values else [0.0], dtype=torch.float64, device=dev)
        self.expval = torch.empty(max(self.n_obs_total, 1), dtype=torch.float64, device=dev)
        self.grad = torch.empty(max(self.n_angles_total, 1), dtype=torch.float64, device=dev)
        self.ct = None
        self._ws_bytes = int(self._lib.jq_batch_workspace_bytes(self.handle))
        self.workspace = torch.empty(max(self._ws_bytes, 1), dtype=torch.uint8, device=dev)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.jq_batch_free(h)
            except Exception:
                pass
            self.handle = None

    @property
    def config(self) -> dict:
        cfg = L.JqBatchConfig()
        L.check(self._lib.jq_batch_info(self.handle, None, None, None, ctypes.byref(cfg)))
        return cfg.as_dict()

    @property
    def classes(self) -> dict:
        """Instances per class under the current configuration."""
        nc = (ctypes.c_int32 * 4)()
        L.check(self._lib.jq_batch_info(self.handle, None, None, nc, None))
        return {"warp": nc[0], "cta": nc[1], "tile": nc[2], "cluster": nc[3]}

    def set_config(self, **config) -> None:
        cfg = L.JqBatchConfig(**{**self.config, **config})
        L.check(self._lib.jq_batch_set_config(self.handle, ctypes.byref(cfg)))

    def autotune(self) -> dict:
        """Time the candidate configurations on the current angles, keep the
        fastest and return it."""
        cfg = L.JqBatchConfig()
        L.check(self._lib.jq_batch_autotune(self.handle, ctypes.c_void_p(self.angles.data_ptr()),
                                            ctypes.c_void_p(self.expval.data_ptr()),
                                            ctypes.c_void_p(self.grad.data_ptr()),
                                            ctypes.c_void_p(self.workspace.data_ptr()), self._ws_bytes, _stream(),
                                            ctypes.byref(cfg)))
        return cfg.as_dict()

    def set_angles(self, angles: torch.Tensor) -> None:
        """New parameter values (same structure): float64 [n_angles total]."""
        a = torch.as_tensor(angles, dtype=torch.float64).reshape(-1)
        if a.numel() != self.n_angles_total:
            raise ValueError(f"expected {self.n_angles_total} angles, got {a.numel()}")
        self.angles[: a.numel()].copy_(a.to(self.device), non_blocking=True)

    def set_cotangents(self, ct: Optional[torch.Tensor]) -> None:
        """Weights ct of the observables (float64 [n_obs total]); None: all ones."""
        if ct is None:
            self.ct = None
            return
        c = torch.as_tensor(ct, dtype=torch.float64).reshape(-1)
        if c.numel() != self.n_obs_total:
            raise ValueError(f"expected {self.n_obs_total} cotangents, got {c.numel()}")
        if self.ct is None:
            self.ct = torch.empty(max(self.n_obs_total, 1), dtype=torch.float64, device=self.device)
        self.ct[: c.numel()].copy_(c.to(self.device), non_blocking=True)

    def run(self) -> Tuple[torch.Tensor, torch.Tensor]:
        """Expectation values [n_obs total] and gradients [n_angles total]
        (views of buffers the next run overwrites)."""
        vp = ctypes.c_void_p
        L.check(self._lib.jq_batch_run(self.handle, vp(self.angles.data_ptr()),
                                       vp(self.ct.data_ptr()) if self.ct is not None else None,
                                       vp(self.expval.data_ptr()), vp(self.grad.data_ptr()),
                                       vp(self.workspace.data_ptr()), self._ws_bytes, _stream()))
        return self.expval[: self.n_obs_total], self.grad[: self.n_angles_total]

    def split(self, expval: torch.Tensor, grad: torch.Tensor) -> List[Tuple[torch.Tensor, torch.Tensor]]:
        """Per-instance (expectation values, gradients)."""
        out = []
        eo = go = 0
        for no, na in zip(self.n_obs, self.n_angles):
            out.append((expval[eo: eo + no], grad[go: go + na]))
            eo += no
            go += na
        return out
