"""Simulation layer: the drop-in for jaqsi/simulation.py on one B200.

A recorded tape is lowered to ``jq_op`` descriptors, compiled once per
structure into a ``jq_plan`` (cached like the reference's jit cache,
jaqsi/script.py:695-725) and executed by libjqsim through its C ABI.  Angles
and per-call matrices are gathered into one device tensor each, so gradients
flow back to the circuit's arguments through a single
``torch.autograd.Function`` whose backward is the GPU adjoint
(unitary statevector plans) or the checkpointed reverse pass (everything else).
"""
from __future__ import annotations

import contextlib
import ctypes
import gc
import math
import threading
from collections import OrderedDict
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from jaqsi_b200 import _lib as L
from jaqsi_b200.gateset import Barrier, Id, PauliX, PauliY, PauliZ
from jaqsi_b200.noise import KrausChannel
from jaqsi_b200.operations import Operation, cdtype, rdtype

_TYPES = ("state", "probs", "expval", "density")
_OUT = {"state": L.JQ_OUT_STATE, "probs": L.JQ_OUT_PROBS, "expval": L.JQ_OUT_EXPVAL, "density": L.JQ_OUT_DENSITY}


def infer_n_qubits(ops: List[Operation], obs: List[Operation]) -> int:
    """``max(wire) + 1`` over ops and observables (jaqsi/simulation.py:32-46)."""
    wires = set()
    for op in list(ops) + list(obs):
        wires.update(op.wires)
    return max(wires) + 1 if wires else 1


def has_noise(tape: List[Operation]) -> bool:
    """Whether the tape holds a Kraus channel (jaqsi/simulation.py:49-62)."""
    return any(isinstance(op, KrausChannel) for op in tape)


@contextlib.contextmanager
def gc_paused():
    """Pause Python's cyclic garbage collector for one circuit call.

    Recording a circuit allocates a few thousand short-lived container objects
    per call (ops, wire lists, angle views).  With the collector running they
    survive its young-generation passes while the tape is alive, are promoted
    into the oldest generation and every few calls trigger a full collection
    of the whole heap (tens of milliseconds with torch loaded).  They are all
    freed by reference counting when the call returns, so pausing the
    collector for the call changes only the timing.  The previous state is
    restored on exit (a collector that was already off stays off).
    """
    was = gc.isenabled()
    if was:
        gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError(
            "jaqsi_b200 executes circuits on a CUDA GPU (sm_100a) only; no CUDA device is available"
        )
    return torch.device("cuda", torch.cuda.current_device())


# ---------------------------------------------------------------------------
# observables
# ---------------------------------------------------------------------------
_PAULI_WORD_OF = {PauliX: "X", PauliY: "Y", PauliZ: "Z"}


def _concrete_matrix(ob: Operation) -> np.ndarray:
    m = ob._matrix
    if isinstance(m, torch.Tensor):
        m = m.detach().cpu().numpy()
    return np.asarray(m, dtype=np.complex128)


def _detect_pauli(m: np.ndarray):
    """(word masks over matrix bits, n_y, real coefficient) if *m* is a real
    multiple of a Pauli word, else None."""
    d = m.shape[0]
    k = d.bit_length() - 1
    nz = np.nonzero(np.abs(m[:, 0]) > 0)[0]
    if len(nz) != 1:
        return None
    x = int(nz[0])
    z = 0
    base = m[x, 0]
    for b in range(k):
        c = 1 << b
        v = m[c ^ x, c]
        if abs(v - base) < 1e-14 * max(1.0, abs(base)):
            continue
        if abs(v + base) < 1e-14 * max(1.0, abs(base)):
            z |= c
        else:
            return None
    ny = bin(x & z).count("1")
    ph = [1, 1j, -1, -1j][ny % 4]
    coeff = base / ph
    if abs(coeff.imag) > 1e-14 * max(1.0, abs(coeff)):
        return None
    coeff = float(coeff.real)
    ref = np.zeros_like(m)
    for c in range(d):
        sign = -1.0 if bin(c & z).count("1") % 2 else 1.0
        ref[c ^ x, c] = coeff * ph * sign
    if not np.allclose(ref, m, atol=1e-14, rtol=0):
        return None
    return x, z, ny, coeff


def _lower_obs(obs: Sequence[Operation], n: int):
    """jq_obs records (plus keep-alive buffers) and a cache key."""
    specs = []
    for ob in obs:
        wires = list(ob.wires)
        for w in wires:
            if w < 0 or w >= n:
                raise ValueError(f"observable wire {w} outside 0..{n - 1}")
        word = getattr(ob, "_pauli_label", None)
        coeff = 1.0
        if word is None and type(ob) in _PAULI_WORD_OF:
            word = _PAULI_WORD_OF[type(ob)]
        if word is None and isinstance(ob, Id):
            word = "I" * len(wires)
        if word is not None:
            x = z = 0
            ny = 0
            for i, ch in enumerate(word):
                bit = 1 << (n - 1 - wires[i])
                if ch in "XY":
                    x |= bit
                if ch in "ZY":
                    z |= bit
                ny += ch == "Y"
            specs.append(("P", x, z, ny, coeff, None, wires))
            continue
        m = _concrete_matrix(ob)
        det = _detect_pauli(m)
        if det is not None:
            xl, zl, ny, coeff = det
            k = len(wires)
            x = z = 0
            for i, w in enumerate(wires):
                pos = 1 << (k - 1 - i)
                if xl & pos:
                    x |= 1 << (n - 1 - w)
                if zl & pos:
                    z |= 1 << (n - 1 - w)
            specs.append(("P", x, z, ny, coeff, None, wires))
        else:
            if len(wires) > L.JQ_MAX_OP_WIRES:
                raise ValueError(f"observables on more than {L.JQ_MAX_OP_WIRES} wires are not supported")
            specs.append(("D", 0, 0, 0, 1.0, np.ascontiguousarray(m), wires))
    key = tuple(
        (s[0], s[1], s[2], s[3], s[4], tuple(s[6])) if s[0] == "P" else ("D", tuple(s[6]), s[5].tobytes())
        for s in specs
    )
    return specs, key


def _build_obs_array(specs):
    arr = (L.JqObs * max(1, len(specs)))()
    keep = []
    for i, (kind, x, z, ny, coeff, mat, wires) in enumerate(specs):
        o = arr[i]
        o.kind = L.JQ_OBS_PAULI if kind == "P" else L.JQ_OBS_DENSE
        o.n_wires = len(wires)
        for j, w in enumerate(wires[: L.JQ_MAX_OP_WIRES]):
            o.wires[j] = w
        o.x_mask, o.z_mask, o.n_y, o.coeff = x, z, ny, coeff
        if mat is not None:
            buf = np.ascontiguousarray(mat.astype(np.complex128)).view(np.float64)
            keep.append(buf)
            o.mat = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return arr, keep


# ---------------------------------------------------------------------------
# tape lowering
# ---------------------------------------------------------------------------
class Lowered:
    """Static structure of a tape (plan key + jq_op fields) and its per-call
    values (angles and matrices)."""

    __slots__ = ("key", "statics", "angles", "mats", "unitary")

    def __init__(self):
        self.key = None
        self.statics = []
        self.angles: list = []
        self.mats: list = []
        self.unitary = True


def _is_tensor(v) -> bool:
    return isinstance(v, torch.Tensor)


_CLASS_LOWERING: Dict[type, object] = {}


def _class_lowering(cls):
    """Lowering fields fixed by the op's class alone, or False.

    Two kinds of class qualify: parametrised gates that declare
    ``_jq_param_kind`` in their own class body (angles = their parameters in
    ``_param_names`` order, no payload), and gates whose matrix is a
    class-level constant with the default ``_jq_lower`` / ``_jq_static_key``.
    Either way an instance that keeps the class's matrix and structure lowers
    to (kind, static key, structure, unitary, parameter names, payload), and
    only its wires and angle values vary.  "skip" marks barriers.
    """
    if issubclass(cls, Barrier):
        return "skip"
    kind = cls.__dict__.get("_jq_param_kind")
    if kind is not None:
        return (kind, (kind,), cls._structure, bool(cls.is_unitary), tuple(cls._param_names), None)
    m = cls._matrix
    if (m is not None and not isinstance(m, torch.Tensor) and cls._jq_lower is Operation._jq_lower
            and cls._jq_static_key is Operation._jq_static_key):
        c = cls.__dict__.get("_jq_const")
        if c is None:
            c = np.asarray(m, dtype=np.complex128)
            cls._jq_const = c
        return (L.JQ_K_CONST, (cls.__name__,), cls._structure, bool(cls.is_unitary), (), c)
    return False


def _bad_wire(op, wires, n_qubits):
    bad = [w for w in wires if not (0 <= w < n_qubits)][0]
    return ValueError(f"{op.name}: wire {bad} outside 0..{n_qubits - 1}")


def lower_tape(tape: Sequence[Operation], n_qubits: int) -> Lowered:
    """Lower recorded ops to plan statics and per-call values.  Pending pulse
    gates are solved first, in batches (jaqsi/simulation.py:713)."""
    from jaqsi_b200.evolution import resolve_pending

    resolve_pending(tape)
    lw = Lowered()
    keys = []
    statics = lw.statics
    n_ang = 0
    n_mat = 0
    max_wires = L.JQ_MAX_OP_WIRES
    k_matrix, k_paulirot = L.JQ_K_MATRIX, L.JQ_K_PAULIROT
    tensor = torch.Tensor
    angles_out = lw.angles
    valid = frozenset(range(n_qubits))
    cache = _CLASS_LOWERING
    for op in tape:
        cls = op.__class__
        ent = cache.get(cls)
        if ent is None:
            ent = _class_lowering(cls)
            cache[cls] = ent
        if ent == "skip":
            continue
        wires = tuple(op._wires)
        if not valid.issuperset(wires):
            raise _bad_wire(op, wires, n_qubits)
        if len(wires) > max_wires:
            raise ValueError(f"{op.name}: gates on more than {max_wires} wires are not supported")
        d = op.__dict__
        if ent is not False and "_structure" not in d and "_matrix" not in d:
            kind, skey, st, unitary, pnames, payload = ent
            grad = 0
            angle_slot = -1
            if pnames:
                angle_slot = n_ang
                for nm in pnames:
                    a = d[nm] if nm in d else getattr(op, nm)
                    angles_out.append(a)
                    if isinstance(a, tensor):
                        grad = 1
                n_ang += len(pnames)
            keys.append((skey, wires, st, grad, unitary, 0))
            statics.append((kind, wires, st, angle_slot, -1, 0, 0, 0, st.controls, payload, grad, unitary))
            if not unitary:
                lw.unitary = False
            continue
        kind, angles, payload = op._jq_lower()
        st = op._structure
        unitary = bool(op.is_unitary)
        grad = 0
        angle_slot = -1
        mat_slot = -1
        mat_is_diag = 0
        if angles:
            angle_slot = n_ang
            n_ang += len(angles)
            angles_out.extend(angles)
            for a in angles:
                if isinstance(a, tensor):
                    grad = 1
                    break
        if kind == k_matrix:
            mat_slot = n_mat
            t = payload
            mat_is_diag = int(t.dim() == 1)
            n_mat += t.numel()
            lw.mats.append(t)
            grad = 1
        skey = op._jq_static_key()
        px = getattr(op, "_px", 0)
        pz = getattr(op, "_pz", 0)
        nctrl = getattr(op, "n_controls", 0) if kind == k_paulirot else st.controls
        keys.append((skey, wires, st, grad, unitary, mat_is_diag))
        statics.append((kind, wires, st, angle_slot, mat_slot, mat_is_diag, px, pz, nctrl, payload, grad, unitary))
        if not unitary:
            lw.unitary = False
    lw.key = tuple(keys)
    return lw


def _build_op_array(statics):
    arr = (L.JqOp * max(1, len(statics)))()
    keep = []
    for i, (kind, wires, st, angle_slot, mat_slot, mat_is_diag, px, pz, nctrl, payload, grad, unitary) in enumerate(statics):
        o = arr[i]
        o.kind = kind
        o.n_wires = len(wires)
        for j, w in enumerate(wires):
            o.wires[j] = w
        o.n_controls = int(nctrl)
        o.diagonal = int(bool(st.diagonal))
        if st.permutation:
            o.has_perm = 1
            for j, p in enumerate(st.permutation):
                o.perm[j] = int(p)
        o.angle_slot = angle_slot
        o.mat_slot = mat_slot
        o.mat_is_diag = mat_is_diag
        o.pauli_x, o.pauli_z = int(px), int(pz)
        o.grad = grad
        o.unitary = int(unitary)
        if kind == L.JQ_K_CONST:
            buf = np.ascontiguousarray(payload, dtype=np.complex128).view(np.float64)
            keep.append(buf)
            o.const_mat = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        elif kind == L.JQ_K_CHANNEL:
            buf = np.ascontiguousarray(np.stack(payload), dtype=np.complex128).view(np.float64)
            keep.append(buf)
            o.n_kraus = len(payload)
            o.const_mat = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return arr, keep


# ---------------------------------------------------------------------------
# plans
# ---------------------------------------------------------------------------
class Plan:
    """An immutable libjqsim execution plan (freed with the object)."""

    def __init__(self, statics, obs_specs, n_qubits: int, mode: int, dtype: torch.dtype, tune: Optional[dict] = None):
        ops, keep_ops = _build_op_array(statics)
        obs_arr, keep_obs = _build_obs_array(obs_specs)
        t = L.JqTune()
        for k, v in (tune or {}).items():
            setattr(t, k, int(v))
        handle = ctypes.c_void_p()
        lib = L.lib()
        L.check(
            lib.jq_plan_build(
                ops, len(statics), obs_arr, len(obs_specs), n_qubits, mode,
                L.JQ_C64 if dtype == torch.complex64 else L.JQ_C128, ctypes.byref(t), ctypes.byref(handle),
            )
        )
        self._lib = lib
        self.handle = handle
        info = L.JqPlanInfo()
        L.check(lib.jq_plan_get_info(handle, ctypes.byref(info)))
        self.info = info.as_dict()
        self.n_qubits = n_qubits
        self.mode = mode
        self.cdtype = dtype
        self.rdtype = rdtype(dtype)
        self.n_obs = len(obs_specs)
        self.state_elems = info.state_elems
        self.n_angles = info.n_angles
        self.n_mats = info.n_mats
        self.unitary = bool(info.unitary)
        del keep_ops, keep_obs  # the plan copied everything it needs

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.jq_plan_free(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = None

    def workspace_bytes(self, batch: int, with_grad: int = 0) -> int:
        return int(self._lib.jq_workspace_bytes(self.handle, batch, 0, with_grad))


_PLAN_CACHE: "OrderedDict[tuple, Plan]" = OrderedDict()
_PLAN_LOCK = threading.Lock()
PLAN_CACHE_SIZE = 256


def get_plan(lw: Lowered, obs_specs, obs_key, n_qubits: int, mode: int, dtype: torch.dtype,
             tune: Optional[dict] = None) -> Plan:
    """The plan of a lowered tape, memoised.  Observables are lowered only for
    expectation values, so a statevector plan with observables is built with
    ``expval_only``: trailing permutations and constant diagonals are then
    absorbed into Z-string observables (the state it leaves is the one before
    them; jaqsi measures the same values after them, simulation.py:777-801)."""
    if obs_specs and mode == L.JQ_STATEVECTOR and not (tune or {}).get("no_fuse"):
        tune = dict(tune or {}, expval_only=1)
    key = (lw.key, obs_key, n_qubits, mode, dtype, tuple(sorted((tune or {}).items())))
    with _PLAN_LOCK:
        plan = _PLAN_CACHE.get(key)
        if plan is not None:
            _PLAN_CACHE.move_to_end(key)
            return plan
    plan = Plan(lw.statics, obs_specs, n_qubits, mode, dtype, tune)
    with _PLAN_LOCK:
        _PLAN_CACHE[key] = plan
        while len(_PLAN_CACHE) > PLAN_CACHE_SIZE:
            _PLAN_CACHE.popitem(last=False)
    return plan


def _functorch_wrapped(t: torch.Tensor) -> bool:
    try:
        return bool(torch._C._functorch.is_functorch_wrapped_tensor(t))
    except AttributeError:  # pragma: no cover - older torch
        return False


def _view_gather(values: list, device: torch.device) -> Optional[torch.Tensor]:
    """One index op when every tensor angle is a one-element view of the same
    contiguous base tensor (the ``params[l, w, i]`` pattern); None otherwise.

    The views the circuit created are bypassed: gradients reach the base
    through a single scatter instead of one select-backward per angle.
    """
    base = None
    dtype = None
    pos, offs, fpos, fval = [], [], [], []
    tensor = torch.Tensor
    for i, v in enumerate(values):
        if isinstance(v, tensor):
            b = v._base
            if b is not base:
                # first tensor angle: the base is checked once (views made
                # under a torch.func transform carry no usable offsets)
                if base is not None or b is None or not b.is_floating_point() or not b.is_contiguous():
                    return None
                if _functorch_wrapped(v):
                    return None
                base, dtype = b, b.dtype
            if v.dtype is not dtype or v.numel() != 1:
                return None
            pos.append(i)
            offs.append(v.storage_offset())
        else:
            fpos.append(i)
            fval.append(float(v))
    if base is None:
        return None
    flat = base.reshape(-1)
    idx = torch.tensor(offs, dtype=torch.long)
    if base.storage_offset():
        idx -= base.storage_offset()
    idx = idx.to(flat.device, non_blocking=True)
    vals = flat.index_select(0, idx).to(torch.float64)
    if not fpos:
        return vals.to(device)
    full = torch.zeros(len(values), dtype=torch.float64)
    full[fpos] = torch.tensor(fval, dtype=torch.float64)
    full = full.to(vals.device)
    out = full.index_copy(0, torch.tensor(pos, dtype=torch.long).to(vals.device), vals)
    return out.to(device)


def gather_angles(values: list, device: torch.device) -> Optional[torch.Tensor]:
    """One float64 device tensor of the tape's angles (keeps autograd links)."""
    if not values:
        return None
    tensors = [v for v in values if isinstance(v, torch.Tensor)]
    if not tensors:
        return torch.tensor([float(v) for v in values], dtype=torch.float64).to(device, non_blocking=True)
    fast = _view_gather(values, device)
    if fast is not None:
        return fast
    devs = {t.device for t in tensors}
    home = tensors[0].device if len(devs) == 1 else device
    parts = [
        v.to(device=home, dtype=torch.float64).reshape(())
        if isinstance(v, torch.Tensor)
        else torch.tensor(float(v), dtype=torch.float64, device=home)
        for v in values
    ]
    return torch.stack(parts).to(device)


def gather_mats(values: list, device: torch.device) -> Optional[torch.Tensor]:
    if not values:
        return None
    parts = [v.resolve_conj().to(torch.complex128).reshape(-1).to(device) for v in values]
    return torch.cat(parts) if len(parts) > 1 else parts[0]


# ---------------------------------------------------------------------------
# execution
# ---------------------------------------------------------------------------
def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# init_batched flag: the initial state of a density plan is a density matrix
_INIT_DENSITY = 2


def _returns_state(plan: Plan, out_type: int) -> bool:
    return out_type == L.JQ_OUT_STATE or (out_type == L.JQ_OUT_DENSITY and plan.mode == L.JQ_DENSITY)


def _forward_launch(plan: Plan, out_type: int, batch: int, init_batched: int, angles, mats, init):
    """jq_forward into fresh (state, out) tensors."""
    dev = _device()
    dim = 1 << plan.n_qubits
    shape = (batch, dim, dim) if plan.mode == L.JQ_DENSITY else (batch, dim)
    state = torch.empty(shape, dtype=plan.cdtype, device=dev)
    out = None
    if out_type == L.JQ_OUT_EXPVAL:
        out = torch.empty((batch, plan.n_obs), dtype=torch.float64, device=dev)
    elif out_type == L.JQ_OUT_PROBS:
        out = torch.empty((batch, dim), dtype=plan.rdtype, device=dev)
    elif out_type == L.JQ_OUT_DENSITY and plan.mode == L.JQ_STATEVECTOR:
        out = torch.empty((batch, dim, dim), dtype=plan.cdtype, device=dev)
    wsb = plan.workspace_bytes(batch, 0)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    L.check(
        plan._lib.jq_forward(
            plan.handle, batch, _ptr(angles), _ptr(mats), _ptr(init), init_batched, out_type,
            _ptr(state), _ptr(out), _ptr(ws), wsb, _stream(),
        )
    )
    return state, out


class _Execute(torch.autograd.Function):
    """Forward = jq_forward; backward = jq_adjoint or jq_backward (through
    _ExecuteGrad); forward-mode derivatives (torch.func.jvp / jacfwd) through
    `jvp`.  The second output is the final state for the derivative rules
    (empty when the result is the state itself); run_plan drops it."""

    @staticmethod
    def forward(plan: Plan, out_type: int, batch: int, init_batched: int, angles, mats, init):
        state, out = _forward_launch(plan, out_type, batch, init_batched, angles, mats, init)
        if _returns_state(plan, out_type):
            return state, state.new_empty(0)
        return out, state

    @staticmethod
    def setup_context(ctx, inputs, output):
        plan, out_type, batch, init_batched, angles, mats, init = inputs
        res, aux = output
        state = res if aux.numel() == 0 else aux
        ctx.mark_non_differentiable(aux)
        ctx.plan, ctx.out_type, ctx.batch, ctx.init_batched = plan, out_type, batch, init_batched
        ctx.save_for_backward(angles, mats, init, state)
        ctx.save_for_forward(angles, mats, init, state)

    @staticmethod
    def backward(ctx, g, _g_aux):
        angles, mats, init, state = ctx.saved_tensors
        need = (angles is not None and ctx.needs_input_grad[4], mats is not None and ctx.needs_input_grad[5],
                init is not None and ctx.needs_input_grad[6])
        if not any(need):
            return None, None, None, None, None, None, None
        ga, gm, gi = _ExecuteGrad.apply(ctx.plan, ctx.out_type, ctx.batch, ctx.init_batched, need, angles, mats,
                                        init, state, g)
        return (None, None, None, None) + _shape_grads(ctx.init_batched, need, angles, mats, ga, gm, gi)

    @staticmethod
    def vmap(info, in_dims, plan, out_type, batch, init_batched, angles, mats, init):
        """Batched inputs become extra plan instances: vmap index v, instance
        b -> instance v * batch + b."""
        B = info.batch_size
        da, dm, di = in_dims[4], in_dims[5], in_dims[6]
        fold = _vmap_folder(B, batch)
        ang = None if angles is None else fold(angles, da, (angles.dim() - (da is not None)) == 1)
        mt = None if mats is None else fold(mats, dm, (mats.dim() - (dm is not None)) == 1)
        ini, ib = init, init_batched
        if init is not None and (di is not None or init_batched & 1):
            ini = fold(init, di, not init_batched & 1)
            ib = init_batched | 1
        res, aux = _Execute.apply(plan, out_type, B * batch, ib, ang, mt, ini)
        res = res.reshape((B, batch) + tuple(res.shape[1:]))
        if aux.numel():
            aux = aux.reshape((B, batch) + tuple(aux.shape[1:]))
            return (res, aux), (0, 0)
        return (res, aux), (0, None)

    @staticmethod
    def jvp(ctx, _t_plan, _t_out, _t_batch, _t_initb, t_angles, t_mats, t_init):
        """Tangent of the result: J v, with the rows of J from one batched
        reverse call (one instance per real output component).  jaqsi routes
        forward mode around its adjoint into plain autodiff
        (jaqsi/simulation.py:492-518); here the adjoint supplies the rows."""
        angles, mats, init, state = ctx.saved_tensors
        plan, out_type, batch = ctx.plan, ctx.out_type, ctx.batch
        return _jvp_by_rows(plan, out_type, batch, ctx.init_batched, angles, mats, init, state, t_angles, t_mats,
                            t_init), None


def _shape_grads(init_batched, need, angles, mats, ga, gm, gi):
    ga = ga if need[0] else None
    gm = gm if need[1] else None
    gi = gi if need[2] else None
    if gi is not None and not init_batched & 1:
        gi = gi.sum(0)
    if ga is not None and angles.dim() == 1:
        ga = ga[0]
    if gm is not None and mats.dim() == 1:
        gm = gm[0]
    return ga, gm, gi


def _grad_launch(plan: Plan, out_type: int, batch: int, init_batched: int, need, angles, mats, init, state, g):
    """Per-instance input gradients [batch, ...] for the output cotangent g."""
    dev = state.device
    lib = plan._lib
    g = g.contiguous()
    ct = g.to(torch.float64).contiguous() if out_type == L.JQ_OUT_EXPVAL else None
    ct_state = None
    if out_type != L.JQ_OUT_EXPVAL:
        ct_state = g.to(plan.rdtype if out_type == L.JQ_OUT_PROBS else plan.cdtype).contiguous()
    ga = torch.empty((batch, plan.n_angles), dtype=torch.float64, device=dev) if need[0] else None
    gm = torch.empty((batch, plan.n_mats), dtype=torch.complex128, device=dev) if need[1] else None
    gdim = plan.state_elems if init_batched & _INIT_DENSITY else 1 << plan.n_qubits
    gi = torch.empty((batch, gdim), dtype=plan.cdtype, device=dev) if need[2] else None
    use_adjoint = plan.mode == L.JQ_STATEVECTOR and plan.unitary
    wsb = plan.workspace_bytes(batch, 1 if use_adjoint else 2)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    if use_adjoint:
        L.check(
            lib.jq_adjoint(
                plan.handle, batch, _ptr(angles), _ptr(mats), _ptr(state), out_type, _ptr(ct),
                _ptr(ct_state), _ptr(ga), _ptr(gm), _ptr(gi), _ptr(ws), wsb, _stream(),
            )
        )
    else:
        L.check(
            lib.jq_backward(
                plan.handle, batch, _ptr(angles), _ptr(mats), _ptr(init), init_batched, out_type,
                _ptr(ct), _ptr(ct_state), _ptr(ga), _ptr(gm), _ptr(gi), _ptr(ws), wsb, _stream(),
            )
        )
    empty = torch.empty(0, device=dev)
    return (ga if ga is not None else empty, gm if gm is not None else empty, gi if gi is not None else empty)


class _ExecuteGrad(torch.autograd.Function):
    """The reverse call as its own Function so that torch.func transforms
    can batch it (`vmap`: jacrev's stacked cotangents become extra plan
    instances).  No second derivatives."""

    @staticmethod
    def forward(plan, out_type, batch, init_batched, need, angles, mats, init, state, g):
        return _grad_launch(plan, out_type, batch, init_batched, need, angles, mats, init, state, g)

    @staticmethod
    def setup_context(ctx, inputs, output):
        pass

    @staticmethod
    def backward(ctx, *grads):
        raise RuntimeError("second derivatives through a simulated circuit are not supported")

    @staticmethod
    def vmap(info, in_dims, plan, out_type, batch, init_batched, need, angles, mats, init, state, g):
        """Batched inputs (jacrev's stacked cotangents, or circuit inputs)
        become extra plan instances: vmap index v, instance b -> v * batch + b."""
        B = info.batch_size
        da, dm, di, ds, dg = in_dims[5:10]
        fold = _vmap_folder(B, batch)
        ang = None if angles is None else fold(angles, da, (angles.dim() - (da is not None)) == 1)
        mt = None if mats is None else fold(mats, dm, (mats.dim() - (dm is not None)) == 1)
        ini, ib = init, init_batched
        if init is not None and (di is not None or init_batched & 1):
            ini = fold(init, di, not init_batched & 1)
            ib = init_batched | 1
        ga, gm, gi = _ExecuteGrad.apply(plan, out_type, B * batch, ib, need, ang, mt, ini,
                                        fold(state, ds, False), fold(g, dg, False))

        def split(t):
            return t if t.numel() == 0 else t.reshape((B, batch) + tuple(t.shape[1:]))

        ga, gm, gi = split(ga), split(gm), split(gi)
        return (ga, gm, gi), (0 if ga.numel() else None, 0 if gm.numel() else None, 0 if gi.numel() else None)


def _vmap_folder(B: int, batch: int):
    """fold(t, d, shared): a tensor of a vmapped Function call (vmap dim d,
    None if unbatched) as [B * batch, ...] rows, one per plan instance; a
    per-index tensor that is `shared` by the batch's instances is repeated."""

    def fold(t, d, shared):
        if t is None:
            return None
        t = t.unsqueeze(0).expand((B,) + tuple(t.shape)) if d is None else t.movedim(d, 0)
        if shared:
            return t.unsqueeze(1).expand(B, batch, *t.shape[1:]).reshape(B * batch, *t.shape[1:]).contiguous()
        return t.reshape(B * batch, *t.shape[2:]).contiguous()

    return fold


# Forward-mode derivatives need one reverse instance per real output
# component; beyond this many amplitudes in flight they are refused.
_JVP_MAX_ELEMS = 1 << 28


def _jvp_by_rows(plan: Plan, out_type: int, batch: int, init_batched: int, angles, mats, init, state,
                 t_angles, t_mats, t_init):
    dim = 1 << plan.n_qubits
    if out_type == L.JQ_OUT_EXPVAL:
        shape, cplx = (plan.n_obs,), False
    elif out_type == L.JQ_OUT_PROBS:
        shape, cplx = (dim,), False
    elif out_type == L.JQ_OUT_STATE:
        shape, cplx = (dim,), True
    else:
        shape, cplx = (dim, dim), True
    n_out = int(np.prod(shape))
    rows = n_out * (2 if cplx else 1)
    if rows * batch * plan.state_elems > _JVP_MAX_ELEMS:
        raise NotImplementedError(
            f"forward-mode derivatives of this {'state' if cplx else 'output'} need {rows * batch} reverse passes "
            f"over {plan.state_elems}-element states; use reverse mode (backward / jacrev)")
    dev = state.device
    # cotangents: instance (b, r) has a one-hot cotangent on real component r
    eye = torch.eye(n_out, dtype=torch.float64, device=dev)
    ct = eye if not cplx else torch.cat([eye.to(plan.cdtype), 1j * eye.to(plan.cdtype)])
    ct = ct.reshape((rows,) + shape)
    g = ct.unsqueeze(0).expand((batch,) + tuple(ct.shape)).reshape((batch * rows,) + shape)

    def rep(t):
        return None if t is None else t.unsqueeze(1).expand((t.shape[0], rows) + tuple(t.shape[1:])).reshape(
            (t.shape[0] * rows,) + tuple(t.shape[1:]))

    ang2 = angles if angles is None or angles.dim() == 2 else angles.unsqueeze(0).expand(batch, -1)
    mat2 = mats if mats is None or mats.dim() == 2 else mats.unsqueeze(0).expand(batch, -1)
    ini2 = init if init is None or init_batched & 1 else init.unsqueeze(0).expand(batch, -1)
    need = (angles is not None and t_angles is not None, mats is not None and t_mats is not None,
            init is not None and t_init is not None)
    ga, gm, gi = _ExecuteGrad.apply(plan, out_type, batch * rows, 1 | (init_batched & _INIT_DENSITY), need,
                                    None if ang2 is None else rep(ang2).contiguous(),
                                    None if mat2 is None else rep(mat2).contiguous(),
                                    None if ini2 is None else rep(ini2).contiguous(), rep(state).contiguous(), g)
    tan = torch.zeros((batch, rows), dtype=torch.float64, device=dev)
    if need[0]:
        ta = t_angles if t_angles.dim() == 2 else t_angles.unsqueeze(0).expand(batch, -1)
        tan = tan + torch.einsum("bri,bi->br", ga.reshape(batch, rows, -1), ta.to(torch.float64))
    if need[1]:
        tm = t_mats if t_mats.dim() == 2 else t_mats.unsqueeze(0).expand(batch, -1)
        tan = tan + torch.einsum("bri,bi->br", gm.reshape(batch, rows, -1).conj(), tm.to(torch.complex128)).real
    if need[2]:
        ti = t_init if init_batched & 1 else t_init.unsqueeze(0).expand(batch, -1)
        tan = tan + torch.einsum("bri,bi->br", gi.reshape(batch, rows, -1).conj().to(torch.complex128),
                                 ti.to(torch.complex128)).real
    if cplx:
        tan = torch.complex(tan[:, :n_out], tan[:, n_out:])
    tan = tan.reshape((batch,) + shape)
    if out_type == L.JQ_OUT_EXPVAL:
        return tan
    rd = plan.rdtype if not cplx else plan.cdtype
    return tan.to(rd)


def run_plan(plan: Plan, out_type: int, batch: int, angles, mats, init, init_batched: int) -> torch.Tensor:
    """Execute *plan* for *batch* instances through the autograd Function."""
    return _Execute.apply(plan, out_type, batch, init_batched, angles, mats, init)[0]


def _prepare_init(initial_state, n_qubits: int, dtype: torch.dtype, device, batched_ok: bool):
    if initial_state is None:
        return None, 0
    t = initial_state if isinstance(initial_state, torch.Tensor) else torch.as_tensor(np.asarray(initial_state))
    t = t.to(device=device, dtype=dtype)
    dim = 2**n_qubits
    if t.dim() == 1:
        if t.numel() != dim:
            raise ValueError(f"initial_state has {t.numel()} amplitudes, expected {dim}")
        return t.contiguous(), 0
    if t.dim() == 2 and batched_ok:
        if t.shape[1] != dim:
            raise ValueError(f"initial_state rows have {t.shape[1]} amplitudes, expected {dim}")
        return t.contiguous(), 1
    raise ValueError(f"initial_state must be a 1D statevector; got ndim={t.dim()}.")


def _resolve_dtype(dtype) -> torch.dtype:
    if dtype is None:
        return cdtype()
    if dtype in (torch.complex64, "complex64", np.complex64):
        return torch.complex64
    if dtype in (torch.complex128, "complex128", np.complex128):
        return torch.complex128
    raise ValueError(f"unsupported dtype {dtype!r}")


def _check_type(type: str, use_density: bool) -> None:
    if type not in _TYPES:
        raise ValueError(f"Unknown measurement type: {type!r}")
    if use_density and type == "state":
        raise ValueError(
            "Measurement type 'state' is not defined for mixed (noisy) circuits. Use 'density' instead."
        )


def _finish(result: torch.Tensor, type: str, dtype: torch.dtype) -> torch.Tensor:
    if type == "expval":
        return result.to(rdtype(dtype))
    return result


def simulate_and_measure(
    tape: List[Operation],
    n_qubits: int,
    type: str,
    obs: List[Operation],
    use_density: bool,
    shots: Optional[int] = None,
    key=None,
    initial_state=None,
    adjoint: bool = True,
    dtype=None,
    tune: Optional[dict] = None,
) -> torch.Tensor:
    """Simulate *tape* and measure (jaqsi/simulation.py:658-732).

    ``adjoint`` is accepted for signature compatibility: the backward of a
    unitary statevector plan is always the adjoint method, every other plan
    uses the checkpointed reverse pass.  ``dtype`` selects complex64 or
    complex128 (default :func:`~jaqsi_b200.operations.cdtype`).
    """
    _check_type(type, use_density)
    dev = _device()
    lw = lower_tape(tape, n_qubits)
    return execute_lowered(lw, n_qubits, type, obs, use_density, gather_angles(lw.angles, dev),
                           gather_mats(lw.mats, dev), shots=shots, key=key, initial_state=initial_state,
                           dtype=dtype, tune=tune)


def execute_lowered(lw: Lowered, n_qubits: int, type: str, obs, use_density: bool, angles, mats,
                    shots: Optional[int] = None, key=None, initial_state=None, dtype=None,
                    tune: Optional[dict] = None, plans: Optional[dict] = None) -> torch.Tensor:
    """Run a lowered tape with its gathered angles / matrices (device
    tensors) and measure: the tail of simulate_and_measure.  ``plans``, when
    given, memoises the plan per (observables, mode, dtype, tune) for a
    caller that keeps one lowering across calls."""
    obs = list(obs or [])
    _check_type(type, use_density)
    dt = _resolve_dtype(dtype)
    dev = _device()
    exact = shots is None or type not in ("probs", "expval")
    mtype = type if exact else "probs"
    mode = L.JQ_DENSITY if use_density else L.JQ_STATEVECTOR
    specs, okey = _lower_obs(obs if mtype == "expval" else [], n_qubits)
    pk = (okey, n_qubits, mode, dt, tuple(sorted((tune or {}).items())))
    plan = plans.get(pk) if plans is not None else None
    if plan is None:
        plan = get_plan(lw, specs, okey, n_qubits, mode, dt, tune)
        if plans is not None:
            plans[pk] = plan
    init, init_b = _prepare_init(initial_state, n_qubits, dt, dev, batched_ok=False)
    res = run_plan(plan, _OUT[mtype], 1, angles, mats, init, init_b)[0]
    if not exact:
        return sample_shots(res, n_qubits, type, obs, shots, key)
    return _finish(res, type, dt)


def measure_state(state: torch.Tensor, n_qubits: int, type: str, obs: List[Operation], dtype=None) -> torch.Tensor:
    """Measure a given statevector (jaqsi/simulation.py:735-811).

    Runs an empty plan on the GPU from *state*; differentiable w.r.t. the
    state.  A leading batch dimension is allowed.
    """
    _check_type(type, False)
    dt = _resolve_dtype(dtype if dtype is not None else (state.dtype if state.is_complex() else None))
    dev = _device()
    st = state if isinstance(state, torch.Tensor) else torch.as_tensor(np.asarray(state))
    batched = st.dim() == 2
    batch = st.shape[0] if batched else 1
    st = st.reshape(batch, -1).to(device=dev, dtype=dt).contiguous()
    lw = lower_tape([], n_qubits)
    specs, okey = _lower_obs(obs if type == "expval" else [], n_qubits)
    plan = get_plan(lw, specs, okey, n_qubits, L.JQ_STATEVECTOR, dt)
    res = run_plan(plan, _OUT[type], batch, None, None, st, 1)
    res = _finish(res, type, dt)
    return res if batched else res[0]


def measure_density(rho: torch.Tensor, n_qubits: int, type: str, obs: List[Operation], dtype=None) -> torch.Tensor:
    """Measure a given density matrix (jaqsi/simulation.py:814-857)."""
    if type not in _TYPES:
        raise ValueError(f"Unknown measurement type: {type!r}")
    if type == "state":
        raise ValueError(
            "Measurement type 'state' is not defined for mixed (noisy) circuits. Use 'density' instead."
        )
    dim = 2**n_qubits
    r = rho if isinstance(rho, torch.Tensor) else torch.as_tensor(np.asarray(rho))
    dt = _resolve_dtype(dtype if dtype is not None else (r.dtype if r.is_complex() else None))
    r = r.to(dt)
    if type == "density":
        return r
    # an empty density plan run from rho: the GPU measurement kernels
    # (Pauli words and dense observables on the density, its diagonal)
    dev = _device()
    batched = r.dim() == 3
    batch = r.shape[0] if batched else 1
    if r.shape[-2:] != (dim, dim):
        raise ValueError(f"rho has shape {tuple(r.shape)}, expected (..., {dim}, {dim})")
    rr = r.reshape(batch, dim * dim).to(dev).contiguous()
    lw = lower_tape([], n_qubits)
    specs, okey = _lower_obs(obs if type == "expval" else [], n_qubits)
    plan = get_plan(lw, specs, okey, n_qubits, L.JQ_DENSITY, dt)
    res = _finish(run_plan(plan, _OUT[type], batch, None, None, rr, 1 | _INIT_DENSITY), type, dt)
    return res if batched else res[0]


# ---------------------------------------------------------------------------
# shots (jaqsi/simulation.py:860-917)
# ---------------------------------------------------------------------------
def _obs_diagonal(ob: Operation, n_qubits: int, device) -> torch.Tensor:
    """diag of the lifted observable as a length-2^n real vector."""
    dim = 2**n_qubits
    idx = torch.arange(dim, device=device)
    k = len(ob.wires)
    sub = torch.zeros(dim, dtype=torch.long, device=device)
    for i, w in enumerate(ob.wires):
        sub = sub | (((idx >> (n_qubits - 1 - w)) & 1) << (k - 1 - i))
    m = _concrete_matrix(ob) if not isinstance(ob, (PauliX, PauliY, PauliZ)) else type(ob)._matrix
    d = torch.as_tensor(np.real(np.diag(np.asarray(m))).copy(), dtype=torch.float64, device=device)
    return d[sub]


def _generator(key, device) -> torch.Generator:
    if isinstance(key, torch.Generator):
        return key
    g = torch.Generator(device=device)
    g.manual_seed(0 if key is None else int(key))
    return g


def sample_shots(probs: torch.Tensor, n_qubits: int, type: str, obs, shots: int, key) -> torch.Tensor:
    """Histogram of *shots* basis samples drawn from *probs* on the GPU
    (``jq_sample_shots``: inverse CDF over a float64 prefix sum).

    ``key`` is an integer seed (the same seed gives the same counts) or a
    ``torch.Generator`` (a seed is drawn from it); the draws are not the
    reference's JAX PRNG stream, only the same distribution.
    """
    if type not in ("probs", "expval"):
        raise ValueError(f"Shot simulation is only supported for 'probs' and 'expval', got {type!r}.")
    dim = 2**n_qubits
    p = probs.detach().to(torch.float64).contiguous()
    rows = p.reshape(-1, dim)
    if isinstance(key, torch.Generator):
        seed = int(torch.randint(0, 2**62, (1,), generator=key, device=key.device).item())
    else:
        seed = 0 if key is None else int(key) & 0xFFFFFFFFFFFFFFFF
    lib = L.lib()
    wsb = int(lib.jq_sample_workspace_bytes(rows.shape[0], dim))
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=p.device)
    counts = torch.empty((rows.shape[0], dim), dtype=torch.int32, device=p.device)
    L.check(lib.jq_sample_shots(_ptr(rows), rows.shape[0], dim, int(shots), seed, _ptr(counts), _ptr(ws), wsb,
                                _stream()))
    est = (counts.to(torch.float64) / shots).reshape(p.shape)  # shots < 2^31: int32 counts
    if type == "probs":
        return est.to(probs.dtype)
    vals = [est @ _obs_diagonal(ob, n_qubits, p.device) for ob in obs]
    if not vals:
        return torch.zeros(est.shape[:-1] + (0,), dtype=probs.dtype, device=p.device)
    return torch.stack(vals, dim=-1).to(probs.dtype)
