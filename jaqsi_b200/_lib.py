"""ctypes binding of libjqsim.so (declared in include/jqsim.h).

The library is loaded from the package directory; there is no fallback: a
missing or unloadable library raises ``RuntimeError`` on first use.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional

JQ_OK = 0
JQ_EINVAL = -1
JQ_ENOMEM = -2
JQ_ECUDA = -3
JQ_ETIMEOUT = -4
JQ_EABORT = -5
JQ_EUNSUPPORTED = -6

JQ_MAX_OP_WIRES = 6
JQ_MAX_QUBITS = 30
JQ_STATIC_WS_BYTES = 4 << 20

JQ_C64, JQ_C128 = 0, 1
JQ_STATEVECTOR, JQ_DENSITY = 0, 1
JQ_OUT_STATE, JQ_OUT_PROBS, JQ_OUT_EXPVAL, JQ_OUT_DENSITY = 0, 1, 2, 3

JQ_K_CONST = 0
JQ_K_MATRIX = 1
JQ_K_RX = 2
JQ_K_RY = 3
JQ_K_RZ = 4
JQ_K_ROT = 5
JQ_K_CPHASE = 6
JQ_K_PAULIROT = 7
JQ_K_CHANNEL = 8

JQ_OBS_PAULI = 0
JQ_OBS_DENSE = 1

EXPORTED = (
    "jq_plan_build",
    "jq_plan_free",
    "jq_plan_get_info",
    "jq_plan_block_passes",
    "jq_plan_jit_source",
    "jq_workspace_bytes",
    "jq_forward",
    "jq_forward_noalloc",
    "jq_sweep",
    "jq_adjoint",
    "jq_backward",
    "jq_sample_workspace_bytes",
    "jq_sample_shots",
    "jq_magnus_product",
    "jq_magnus_product_grad",
    "jq_batch_build",
    "jq_batch_free",
    "jq_batch_info",
    "jq_batch_workspace_bytes",
    "jq_batch_set_config",
    "jq_batch_run",
    "jq_batch_autotune",
    "jq_last_error",
    "jq_version",
)


class JqOp(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("n_wires", ctypes.c_int32),
        ("wires", ctypes.c_int32 * JQ_MAX_OP_WIRES),
        ("n_controls", ctypes.c_int32),
        ("diagonal", ctypes.c_int32),
        ("has_perm", ctypes.c_int32),
        ("perm", ctypes.c_int32 * (1 << JQ_MAX_OP_WIRES)),
        ("angle_slot", ctypes.c_int32),
        ("mat_slot", ctypes.c_int32),
        ("mat_is_diag", ctypes.c_int32),
        ("pauli_x", ctypes.c_uint32),
        ("pauli_z", ctypes.c_uint32),
        ("n_kraus", ctypes.c_int32),
        ("grad", ctypes.c_int32),
        ("unitary", ctypes.c_int32),
        ("const_mat", ctypes.POINTER(ctypes.c_double)),
    ]


class JqObs(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("n_wires", ctypes.c_int32),
        ("wires", ctypes.c_int32 * JQ_MAX_OP_WIRES),
        ("x_mask", ctypes.c_uint64),
        ("z_mask", ctypes.c_uint64),
        ("n_y", ctypes.c_int32),
        ("coeff", ctypes.c_double),
        ("mat", ctypes.POINTER(ctypes.c_double)),
    ]


class JqTune(ctypes.Structure):
    _fields_ = [
        ("tile_bits", ctypes.c_int32),
        ("tile_bits_adj", ctypes.c_int32),
        ("threads", ctypes.c_int32),
        ("no_fuse", ctypes.c_int32),
        ("ckpt_stride", ctypes.c_int32),
        ("jit", ctypes.c_int32),
        ("expval_only", ctypes.c_int32),
    ]


class JqPlanInfo(ctypes.Structure):
    _fields_ = [
        ("n_qubits", ctypes.c_int32),
        ("n_bits", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("dtype", ctypes.c_int32),
        ("n_ops", ctypes.c_int32),
        ("n_blocks", ctypes.c_int32),
        ("n_passes_fwd", ctypes.c_int32),
        ("n_passes_adj", ctypes.c_int32),
        ("n_tile_ops_fwd", ctypes.c_int32),
        ("tile_bits_fwd", ctypes.c_int32),
        ("tile_bits_adj", ctypes.c_int32),
        ("n_angles", ctypes.c_int32),
        ("n_mats", ctypes.c_int32),
        ("n_obs", ctypes.c_int32),
        ("unitary", ctypes.c_int32),
        ("state_elems", ctypes.c_int64),
        ("n_stages_fwd", ctypes.c_int32),
        ("n_smem_ops_fwd", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class JqBatchConfig(ctypes.Structure):
    _fields_ = [
        ("warp_max_qubits", ctypes.c_int32),
        ("cta_max_qubits", ctypes.c_int32),
        ("warp_threads", ctypes.c_int32),
        ("cta_threads", ctypes.c_int32),
        ("cluster_bits", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_LIB: Optional[ctypes.CDLL] = None
_LOCK = threading.Lock()
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libjqsim.so")


def _declare(lib: ctypes.CDLL) -> None:
    vp = ctypes.c_void_p
    i32 = ctypes.c_int
    lib.jq_plan_build.argtypes = [
        ctypes.POINTER(JqOp), i32, ctypes.POINTER(JqObs), i32, i32, i32, i32,
        ctypes.POINTER(JqTune), ctypes.POINTER(vp),
    ]
    lib.jq_plan_build.restype = i32
    lib.jq_plan_free.argtypes = [vp]
    lib.jq_plan_free.restype = i32
    lib.jq_plan_get_info.argtypes = [vp, ctypes.POINTER(JqPlanInfo)]
    lib.jq_plan_get_info.restype = i32
    lib.jq_plan_block_passes.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), i32]
    lib.jq_plan_block_passes.restype = i32
    lib.jq_plan_jit_source.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.jq_plan_jit_source.restype = ctypes.c_size_t
    lib.jq_workspace_bytes.argtypes = [vp, i32, i32, i32]
    lib.jq_workspace_bytes.restype = ctypes.c_size_t
    lib.jq_forward.argtypes = [vp, i32, vp, vp, vp, i32, i32, vp, vp, vp, ctypes.c_size_t, vp]
    lib.jq_forward.restype = i32
    lib.jq_forward_noalloc.argtypes = [vp, i32, vp, vp, vp, i32, i32, vp, vp, vp]
    lib.jq_forward_noalloc.restype = i32
    lib.jq_sweep.argtypes = [vp, i32, vp, vp, vp, vp, ctypes.c_size_t, vp]
    lib.jq_sweep.restype = i32
    lib.jq_adjoint.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    lib.jq_adjoint.restype = i32
    lib.jq_backward.argtypes = [vp, i32, vp, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    lib.jq_backward.restype = i32
    lib.jq_sample_workspace_bytes.argtypes = [i32, ctypes.c_int64]
    lib.jq_sample_workspace_bytes.restype = ctypes.c_size_t
    lib.jq_sample_shots.argtypes = [vp, i32, ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, vp, vp,
                                    ctypes.c_size_t, vp]
    lib.jq_sample_shots.restype = i32
    lib.jq_magnus_product.argtypes = [i32, i32, i32, i32, vp, ctypes.c_int64, vp, vp, vp]
    lib.jq_magnus_product.restype = i32
    lib.jq_magnus_product_grad.argtypes = [i32, i32, i32, i32, vp, ctypes.c_int64, vp, vp, vp, vp]
    lib.jq_magnus_product_grad.restype = i32
    lib.jq_batch_build.argtypes = [ctypes.POINTER(vp), i32, ctypes.POINTER(ctypes.c_int32), i32,
                                   ctypes.POINTER(JqBatchConfig), ctypes.POINTER(vp)]
    lib.jq_batch_build.restype = i32
    lib.jq_batch_free.argtypes = [vp]
    lib.jq_batch_free.restype = i32
    lib.jq_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                  ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(JqBatchConfig)]
    lib.jq_batch_info.restype = i32
    lib.jq_batch_workspace_bytes.argtypes = [vp]
    lib.jq_batch_workspace_bytes.restype = ctypes.c_size_t
    lib.jq_batch_set_config.argtypes = [vp, ctypes.POINTER(JqBatchConfig)]
    lib.jq_batch_set_config.restype = i32
    lib.jq_batch_run.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    lib.jq_batch_run.restype = i32
    lib.jq_batch_autotune.argtypes = [vp, vp, vp, vp, vp, ctypes.c_size_t, vp, ctypes.POINTER(JqBatchConfig)]
    lib.jq_batch_autotune.restype = i32
    lib.jq_last_error.argtypes = []
    lib.jq_last_error.restype = ctypes.c_char_p
    lib.jq_version.argtypes = []
    lib.jq_version.restype = ctypes.c_char_p


def lib() -> ctypes.CDLL:
    """The loaded libjqsim (raises ``RuntimeError`` if it cannot be loaded)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"libjqsim.so not found at {LIB_PATH}; build it with "
                    "`python -m jaqsi_b200.build` (nvcc, sm_100a)"
                )
            try:
                handle = ctypes.CDLL(LIB_PATH)
            except OSError as exc:  # pragma: no cover - depends on the machine
                raise RuntimeError(f"cannot load {LIB_PATH}: {exc}") from exc
            _declare(handle)
            _LIB = handle
    return _LIB


class JqError(RuntimeError):
    """A libjqsim call failed; ``status`` holds the negative status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libjqsim error {status}: {message}")
        self.status = status


def check(status: int) -> None:
    """Raise on a non-zero libjqsim status (ValueError for invalid input)."""
    if status == JQ_OK:
        return
    msg = lib().jq_last_error().decode(errors="replace")
    if status == JQ_EINVAL:
        raise ValueError(msg)
    if status == JQ_ENOMEM:
        raise MemoryError(msg)
    raise JqError(status, msg)
