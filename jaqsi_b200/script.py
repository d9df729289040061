"""``Script``: record a circuit function and execute it on the GPU backend.

Keeps the reference surface ``Script(f, n_qubits).execute(type, obs, args=...,
kwargs=..., in_axes=..., shots=..., key=..., initial_state=..., fingerprint=...)``
(jaqsi/script.py:154-335).  Batched execution (``in_axes``) runs all samples
in one set of kernel launches (jaqsi/script.py:389-744 maps the same
signature onto ``jax.vmap``).

Call-signature cache.  The reference compiles a batched call once per
signature (``_jit_cache`` keyed on type, in_axes, argument shapes and
``fingerprint``, jaqsi/script.py:695-705) and then only feeds new argument
values.  ``Script`` does the same for every call, batched or not: the first
call of a signature records the circuit while watching its arguments, and if
every recorded angle is an element of an argument tensor (or a constant), it
keeps the lowered structure and the element indices.  Later calls with the
same signature skip the circuit function and gather the angles from the new
arguments with one index operation.  A circuit that reads an argument's value
into Python (a branch on it, ``float()``, ``.item()``), computes an angle from
arguments with tensor arithmetic, or passes per-call matrices is re-recorded on
every call, as before.  State read outside the arguments belongs in
``fingerprint``, as in the reference.  ``Script.cache_traces = False`` turns
the cache off.
"""
from __future__ import annotations

from typing import Any, Callable, Hashable, List, Optional, Tuple

import numpy as np
import torch
from torch.overrides import TorchFunctionMode

from jaqsi_b200 import _lib as L
from jaqsi_b200 import shard, simulation
from jaqsi_b200.operations import Operation, rdtype
from jaqsi_b200.tape import recording

# Tensor methods that hand an argument's value to Python code: a circuit that
# calls one of them on an argument-derived tensor may change its structure with
# the value, so its calls are not cached.
_VALUE_READS = frozenset(
    getattr(torch.Tensor, n)
    for n in ("__bool__", "__float__", "__int__", "__index__", "__complex__", "item", "tolist", "numpy",
              "__array__")
    if hasattr(torch.Tensor, n)
)
_NO_TRACE = object()


def _transformed(t: torch.Tensor) -> bool:
    """Whether t is wrapped by a torch.func transform (vmap, grad, jvp, ...)."""
    try:
        return bool(torch._C._functorch.is_functorch_wrapped_tensor(t))
    except AttributeError:  # pragma: no cover - older torch
        return False


def _tensors_in(x):
    if isinstance(x, torch.Tensor):
        yield x
    elif isinstance(x, (list, tuple)):
        for v in x:
            yield from _tensors_in(v)
    elif isinstance(x, dict):
        for v in x.values():
            yield from _tensors_in(v)


class _ArgWatch(TorchFunctionMode):
    """While a circuit records: marks every tensor computed from the call's
    argument tensors, and notes any read of such a tensor's value into Python."""

    def __init__(self, roots):
        super().__init__()
        self.ids = {id(t) for t in roots}
        self.keep = list(roots)  # keeps ids unique while recording
        self.value_read = False

    def __torch_function__(self, func, types, args=(), kwargs=None):
        kwargs = kwargs or {}
        tainted = any(id(t) in self.ids for t in _tensors_in((args, kwargs)))
        if tainted and func in _VALUE_READS:
            self.value_read = True
        out = func(*args, **kwargs)
        if tainted:
            for t in _tensors_in(out):
                self.ids.add(id(t))
                self.keep.append(t)
        return out


class _Trace:
    """Cached lowering of one call signature and where each angle comes from:
    slot positions and flat element indices per argument, plus constants."""

    __slots__ = ("lw", "n_qubits", "use_density", "n_angles", "parts", "cpos", "cval", "plans", "_dev")

    def __init__(self, lw, n_qubits, use_density, parts, cpos, cval):
        self.lw = lw
        self.n_qubits = n_qubits
        self.use_density = use_density
        self.n_angles = len(lw.angles)
        self.parts = parts  # [(arg index, slot positions, flat indices)]
        self.cpos, self.cval = cpos, cval
        self.plans: dict = {}
        self._dev: dict = {}
        lw.angles = []  # the first call's values are not kept

    def _idx(self, dev):
        d = self._dev.get(dev)
        if d is None:
            d = ([(i, torch.tensor(pos, dtype=torch.long, device=dev), torch.tensor(idx, dtype=torch.long))
                  for i, pos, idx in self.parts],
                 torch.tensor(self.cpos, dtype=torch.long, device=dev),
                 torch.tensor(self.cval, dtype=torch.float64, device=dev))
            self._dev[dev] = d
        return d

    def angles(self, args, dev, batch=None, in_axes=None):
        """float64 angles on `dev`: [n_angles], or [batch, n_angles] with
        each argument's batch axis from in_axes (None: broadcast)."""
        if self.n_angles == 0:
            return None
        parts, cpos, cval = self._idx(dev)
        if batch is None:
            if len(parts) == 1 and not self.cpos and len(parts[0][2]) == self.n_angles and self._ordered():
                i, _, idx = parts[0]
                return args[i].reshape(-1).index_select(0, idx.to(args[i].device)).to(dev, torch.float64)
            out = torch.zeros(self.n_angles, dtype=torch.float64, device=dev)
            if self.cpos:
                out = out.index_copy(0, cpos, cval)
            for i, pos, idx in parts:
                v = args[i].reshape(-1).index_select(0, idx.to(args[i].device)).to(dev, torch.float64)
                out = out.index_copy(0, pos, v)
            return out
        out = torch.zeros((batch, self.n_angles), dtype=torch.float64, device=dev)
        if self.cpos:
            out = out.index_copy(1, cpos, cval.expand(batch, -1))
        for i, pos, idx in parts:
            a, ax = args[i], in_axes[i]
            if ax is None:
                v = a.reshape(-1).index_select(0, idx.to(a.device)).to(dev, torch.float64).expand(batch, -1)
            else:
                v = a.movedim(ax, 0).reshape(batch, -1).index_select(1, idx.to(a.device)).to(dev, torch.float64)
            out = out.index_copy(1, pos, v)
        return out

    def _ordered(self):
        pos = self.parts[0][1]
        return all(p == k for k, p in enumerate(pos))


def _trace_recipe(angles, roots):
    """(parts, cpos, cval) when every tensor angle is one element of one
    contiguous root tensor (matched by storage and offset); None otherwise."""
    by_storage = {}
    for i, a in roots:
        if a.numel() and a.is_contiguous():
            by_storage.setdefault(a.untyped_storage().data_ptr(), []).append((i, a))
    parts: dict = {}
    cpos, cval = [], []
    for slot, v in enumerate(angles):
        if not isinstance(v, torch.Tensor):
            cpos.append(slot)
            cval.append(float(v))
            continue
        if v.numel() != 1 or v.is_complex():
            return None
        hit = None
        for i, a in by_storage.get(v.untyped_storage().data_ptr(), ()):
            off = v.storage_offset() - a.storage_offset()
            if a.dtype == v.dtype and 0 <= off < a.numel():
                if hit is not None:
                    return None
                hit = (i, off)
        if hit is None:
            return None
        p = parts.setdefault(hit[0], ([], []))
        p[0].append(slot)
        p[1].append(hit[1])
    return [(i, pos, idx) for i, (pos, idx) in sorted(parts.items())], cpos, cval


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

    cache_traces = True  # reuse the lowering of a call signature (module docstring)

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
            tkey = self._trace_key(type, args, kwargs, None, fingerprint, dtype, initial_state, shots)
            tr = self._jit_cache.get(tkey) if tkey is not None else None
            tape = None
            if tr is None and tkey is not None:
                tape, tr = self._new_trace(tkey, args, kwargs)
            if isinstance(tr, _Trace):
                dev = simulation._device()
                return simulation.execute_lowered(
                    tr.lw, self._trace_qubits(tr, obs), type, obs, tr.use_density, tr.angles(args, dev), None,
                    shots=shots, key=key, initial_state=initial_state, dtype=dtype, plans=tr.plans)
            if tape is None:
                tape = self.record(*args, **kwargs)
            n_qubits = self._n_qubits or simulation.infer_n_qubits(tape, obs)
            use_density = simulation.has_noise(tape)
            return simulation.simulate_and_measure(
                tape, n_qubits, type, obs, use_density, shots=shots, key=key, initial_state=initial_state,
                dtype=dtype
            )

    # ---- call-signature cache --------------------------------------------
    def _trace_key(self, mtype, args, kwargs, in_axes, fingerprint, dtype, initial_state, shots):
        """Cache key of a call, or None when the call is not cacheable."""
        if not self.cache_traces:
            return None
        sig = []
        for i, a in enumerate(args):
            if isinstance(a, torch.Tensor):
                if _transformed(a):
                    return None  # under a torch.func transform: record every call
                sig.append(("t", tuple(a.shape), a.dtype, a.device, a.requires_grad))
            elif a is None or isinstance(a, (bool, int, float, complex, str)):
                if in_axes is not None and in_axes[i] is not None:
                    return None
                sig.append(("v", a.__class__.__name__, a))
            else:
                return None
        if any(True for _ in _tensors_in(kwargs)):
            return None
        try:
            kw = make_hashable(kwargs)
            key = ("trace", mtype, tuple(sig), kw, in_axes, fingerprint, simulation._resolve_dtype(dtype),
                   None if initial_state is None else tuple(np.shape(initial_state)), shots is not None)
            hash(key)
        except TypeError:
            return None
        return key

    def _new_trace(self, tkey, rec_args, kwargs):
        """Record once while watching the argument tensors; cache a _Trace
        (or the marker that this signature is not cacheable)."""
        roots = [(i, a) for i, a in enumerate(rec_args) if isinstance(a, torch.Tensor)]
        watch = _ArgWatch([a for _, a in roots])
        with watch:
            tape = self.record(*rec_args, **kwargs)
        n_tape = simulation.infer_n_qubits(tape, [])
        lw = simulation.lower_tape(tape, max(n_tape, self._n_qubits or 0))
        tr = _NO_TRACE
        if not watch.value_read and not lw.mats:
            rec = _trace_recipe(lw.angles, roots)
            if rec is not None:
                tr = _Trace(lw, n_tape, simulation.has_noise(tape), *rec)
        self._jit_cache[tkey] = tr
        return tape, tr

    def _trace_qubits(self, tr, obs) -> int:
        if self._n_qubits:
            return self._n_qubits
        return max(tr.n_qubits, simulation.infer_n_qubits([], obs) if obs else 1)

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
        spec = shard.active()
        if spec is not None and shots is None and batch >= spec[2]:
            # this rank's rows of the batch, all-gathered (jaqsi_b200.shard)
            def local(largs, lbatch, linit):
                return self._execute_batched(type, obs, largs, kwargs, in_axes, None, key, linit, fingerprint,
                                             dtype)

            return shard.sharded_batch_call(local, args, in_axes, batch, *spec, initial_state=initial_state)
        dt = simulation._resolve_dtype(dtype)
        dev = simulation._device()
        tkey = self._trace_key(type, args, kwargs, in_axes, fingerprint, dtype, initial_state, shots)
        tr = self._jit_cache.get(tkey) if tkey is not None else None
        if tr is None and tkey is not None:
            # record one sample (contiguous slices of the batched arguments)
            sample = tuple(a.movedim(ax, 0)[0].contiguous() if ax is not None else a for a, ax in zip(args, in_axes))
            _, tr = self._new_trace(tkey, sample, kwargs)
        if isinstance(tr, _Trace):
            n_qubits = self._trace_qubits(tr, obs)
            return self._run_batched(tr.lw, n_qubits, tr.use_density, type, obs, batch,
                                     tr.angles(args, dev, batch, in_axes), None, shots, key, initial_state, dt, dev,
                                     tr.plans)
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
        return self._run_batched(lw, n_qubits, simulation.has_noise(tape), type, obs, batch,
                                 ang_b if lw.angles else None, mats_b if lw.mats else None, shots, key,
                                 initial_state, dt, dev, None)

    def _run_batched(self, lw, n_qubits, use_density, type, obs, batch, ang_b, mats_b, shots, key, initial_state,
                     dt, dev, plans):
        simulation._check_type(type, use_density)
        exact = shots is None or type not in ("probs", "expval")
        mtype = type if exact else "probs"
        mode = L.JQ_DENSITY if use_density else L.JQ_STATEVECTOR
        specs, okey = simulation._lower_obs(obs if mtype == "expval" else [], n_qubits)
        pk = (okey, n_qubits, mode, dt)
        plan = plans.get(pk) if plans is not None else None
        if plan is None:
            plan = simulation.get_plan(lw, specs, okey, n_qubits, mode, dt)
            if plans is not None:
                plans[pk] = plan
        angles = ang_b.to(dev).contiguous() if ang_b is not None else None
        mats = mats_b.to(dev).contiguous() if mats_b is not None else None
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
