"""``Script``: record a circuit function and execute it on the GPU backend.

Keeps the reference surface ``Script(f, n_qubits).execute(type, obs, args=...,
kwargs=..., in_axes=..., shots=..., key=..., initial_state=..., fingerprint=...)``
(jaqsi/script.py:154-335).  Batched execution (``in_axes``) records the
circuit once per call under ``torch.func.vmap`` to gather every sample's
angles into one [batch, n_angles] tensor, then runs all samples in one set of
kernel launches (jaqsi/script.py:389-744 maps the same signature onto
``jax.vmap``).
"""
from __future__ import annotations

from typing import Any, Callable, Hashable, List, Optional, Tuple

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200 import simulation
from jaqsi_b200.operations import Operation, rdtype
from jaqsi_b200.tape import recording


def make_hashable(obj):
    """Recursively convert *obj* into a hashable form (jaqsi/script.py:18-32)."""
    if isinstance(obj, dict):
        return tuple(sorted((k, make_hashable(v)) for k, v in obj.items()))
    if isinstance(obj, (list, tuple)):
        return tuple(make_hashable(x) for x in obj)
    if isinstance(obj, set):
        return frozenset(make_hashable(x) for x in obj)
    return obj


def _as_arg(a):
    if isinstance(a, np.ndarray):
        return torch.as_tensor(a)
    return a


class Script:
    """Record and execute a quantum circuit defined by a Python function."""

    def __init__(self, f: Callable[..., None], n_qubits: Optional[int] = None) -> None:
        self.f = f
        self._n_qubits = n_qubits
        self._jit_cache: dict = {}

    def __getstate__(self) -> dict:
        return {**self.__dict__, "_jit_cache": {}}

    def record(self, *args, **kwargs) -> List[Operation]:
        """Run the circuit function and return its recorded ops."""
        with recording() as tape:
            self.f(*args, **kwargs)
        return tape

    def execute(
        self,
        type: str = "expval",
        obs: Optional[List[Operation]] = None,
        *,
        args: tuple = (),
        kwargs: Optional[dict] = None,
        in_axes: Optional[Tuple] = None,
        shots: Optional[int] = None,
        key=None,
        initial_state=None,
        fingerprint: Optional[Hashable] = None,
        dtype=None,
    ) -> torch.Tensor:
        """Execute the circuit and return measurement results.

        Same arguments and result shapes as jaqsi/script.py:226-335, plus
        ``dtype`` (torch.complex64 / torch.complex128).  ``key`` is an integer
        seed or a ``torch.Generator`` for shot sampling.
        """
        if obs is None:
            obs = []
        if kwargs is None:
            kwargs = {}
        if initial_state is not None:
            nd = initial_state.dim() if isinstance(initial_state, torch.Tensor) else np.ndim(initial_state)
            if in_axes is None and nd != 1:
                raise ValueError(f"initial_state must be a 1D statevector when in_axes is None; got ndim={nd}.")
            if in_axes is not None and nd not in (1, 2):
                raise ValueError(
                    f"Batched initial_state must be 1D (broadcast) or 2D (one state per sample); got ndim={nd}."
                )
        args = tuple(_as_arg(a) for a in args)
        with simulation.gc_paused():
            if in_axes is not None:
                return self._execute_batched(type, obs, args, kwargs, tuple(in_axes), shots, key, initial_state,
                                             fingerprint, dtype)
            tape = self.record(*args, **kwargs)
            n_qubits = self._n_qubits or simulation.infer_n_qubits(tape, obs)
            use_density = simulation.has_noise(tape)
            return simulation.simulate_and_measure(
                tape, n_qubits, type, obs, use_density, shots=shots, key=key, initial_state=initial_state,
                dtype=dtype
            )

    @staticmethod
    def _batch_size(args: tuple, in_axes: Tuple) -> int:
        for a, ax in zip(args, in_axes):
            if ax is not None:
                return a.shape[ax]
        return 1

    def _execute_batched(self, type, obs, args, kwargs, in_axes, shots, key, initial_state, fingerprint, dtype):
        if len(in_axes) != len(args):
            raise ValueError(
                f"in_axes has {len(in_axes)} entries but args has {len(args)}. "
                "Provide one in_axes entry per positional argument."
            )
        batch = self._batch_size(args, in_axes)
        dt = simulation._resolve_dtype(dtype)
        dev = simulation._device()
        holder = {}

        def gather(*sample_args):
            tape = self.record(*sample_args, **kwargs)
            lw = simulation.lower_tape(tape, self._n_qubits or simulation.infer_n_qubits(tape, obs))
            holder["tape"] = tape
            holder["lw"] = lw
            holder["n"] = self._n_qubits or simulation.infer_n_qubits(tape, obs)
            ang = (
                torch.stack([a.to(torch.float64).reshape(()) if isinstance(a, torch.Tensor)
                             else torch.tensor(float(a), dtype=torch.float64) for a in lw.angles])
                if lw.angles else torch.zeros(0, dtype=torch.float64)
            )
            mats = (
                torch.cat([m.to(torch.complex128).reshape(-1) for m in lw.mats])
                if lw.mats else torch.zeros(0, dtype=torch.complex128)
            )
            return ang, mats

        batched_any = any(ax is not None and isinstance(a, torch.Tensor) for a, ax in zip(args, in_axes))
        if batched_any:
            dims = tuple(ax if isinstance(a, torch.Tensor) else None for a, ax in zip(args, in_axes))
            ang_b, mats_b = torch.func.vmap(gather, in_dims=dims, randomness="error")(*args)
        else:
            ang, mats = gather(*args)
            ang_b = ang.unsqueeze(0).expand(batch, -1)
            mats_b = mats.unsqueeze(0).expand(batch, -1)
        tape, lw, n_qubits = holder["tape"], holder["lw"], holder["n"]
        use_density = simulation.has_noise(tape)
        simulation._check_type(type, use_density)
        exact = shots is None or type not in ("probs", "expval")
        mtype = type if exact else "probs"
        mode = L.JQ_DENSITY if use_density else L.JQ_STATEVECTOR
        specs, okey = simulation._lower_obs(obs if mtype == "expval" else [], n_qubits)
        plan = simulation.get_plan(lw, specs, okey, n_qubits, mode, dt)
        angles = ang_b.to(dev).contiguous() if lw.angles else None
        mats = mats_b.to(dev).contiguous() if lw.mats else None
        init, init_b = simulation._prepare_init(initial_state, n_qubits, dt, dev, batched_ok=True)
        res = self._run_chunked(plan, simulation._OUT[mtype], batch, angles, mats, init, init_b)
        if not exact:
            gen = simulation._generator(key, res.device)
            return torch.stack([
                simulation.sample_shots(res[b], n_qubits, type, obs, shots, gen) for b in range(batch)
            ])
        return simulation._finish(res, type, dt)

    @staticmethod
    def _run_chunked(plan, out_type, batch, angles, mats, init, init_b):
        """Run in chunks that fit in free device memory (jaqsi/memory.py:169-239)."""
        per = plan.workspace_bytes(1, 2 if not (plan.mode == L.JQ_STATEVECTOR and plan.unitary) else 1)
        per += plan.state_elems * (8 if plan.cdtype == torch.complex64 else 16) * 2
        free, _ = torch.cuda.mem_get_info()
        chunk = max(1, min(batch, int(0.6 * free // max(per, 1))))
        if chunk >= batch:
            return simulation.run_plan(plan, out_type, batch, angles, mats, init, init_b)
        outs = []
        for s in range(0, batch, chunk):
            e = min(batch, s + chunk)
            a = angles[s:e] if angles is not None else None
            m = mats[s:e] if mats is not None else None
            i = init[s:e] if (init is not None and init_b) else init
            outs.append(simulation.run_plan(plan, out_type, e - s, a, m, i, init_b))
        return torch.cat(outs)

    def draw(self, figure: str = "text", args: tuple = (), kwargs: Optional[dict] = None, **draw_kwargs: Any) -> str:
        """Plain-text drawing of the recorded ops (the reference also offers
        matplotlib/TikZ backends, jaqsi/script.py:746-818)."""
        if figure != "text":
            raise ValueError(f"Invalid figure mode: {figure!r}. Only 'text' is available in this backend.")
        tape = self.record(*args, **(kwargs or {}))
        n = self._n_qubits or simulation.infer_n_qubits(tape, [])
        lines = [f"{w}: " for w in range(n)]
        for op in tape:
            for w in range(n):
                lines[w] += (op.name if w in op.wires else "-" * len(op.name)) + "-"
        return "\n".join(lines)
