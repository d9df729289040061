"""The reference's compiled statevector plan, executed by the oracle's OpenMP C
restatement (oracle/jqoracle.c).

TEST / BASELINE INFRASTRUCTURE ONLY: tests/ use it as the float64 checker of
large statevector sweeps, and bench.py times it as the reference arm and the
CPU baseline.  Nothing in the product imports it.

The plan is the one the reference builds (jaqsi/simulation.py:214-335, restated
by sim_np.jaqsi_plan): fused dense blocks, composed diagonals, and one 2^n
int32 gather map per run of permutations.  The gather maps are composed in C
(jqo_compose_perm, the fold of _compose_permutation, :243-267) and shared
between runs of identical structure only while building; each plan entry keeps
its own copy of the map, as the reference's compiled program holds one
constant per entry.  Running the plan is _run (:400-409): one full pass over
the state per entry.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence

import numpy as np

from oracle import sim_np as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libjqoracle.so")
_LIB = None
_DENSE, _GATHER, _DIAG = 0, 1, 2
MAXW = 32  # JQO_MAXW: wires of one plan entry


def lib() -> ctypes.CDLL:
    """The oracle's C library (built by oracle/Makefile on first use)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = ctypes.CDLL(LIB_PATH)
        for sfx, T in (("", ctypes.c_double), ("f", ctypes.c_float)):
            P = ctypes.POINTER(T)
            f = getattr(L, f"jqo_run_plan{sfx}")
            f.restype = ctypes.c_int
            f.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p, ctypes.c_void_p]
            e = getattr(L, f"jqo_expval_z{sfx}")
            e.restype = ctypes.c_double
            e.argtypes = [P, ctypes.c_int, ctypes.c_uint64]
            e = getattr(L, f"jqo_expval_z_dm{sfx}")
            e.restype = ctypes.c_double
            e.argtypes = [P, ctypes.c_int, ctypes.c_uint64]
            z = getattr(L, f"jqo_init_zero{sfx}")
            z.restype = None
            z.argtypes = [P, ctypes.c_int]
        L.jqo_compose_perm.restype = None
        L.jqo_compose_perm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p]
        L.jqo_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def compose_permutation_c(run, n: int, memo: Optional[dict] = None) -> np.ndarray:
    """Gather map of a permutation run, same result as
    sim_np.compose_permutation, folded block by block in C."""
    key = tuple((tuple(w), tuple(st[1])) for _, w, st in run)
    if memo is not None and key in memo:
        return memo[key].copy()
    L = lib()
    cur = np.arange(1 << n, dtype=np.int32)
    nxt = np.empty_like(cur)
    for _, wires, (_, perm) in run:
        bits = (ctypes.c_int * len(wires))(*[n - 1 - w for w in wires])
        pm = np.ascontiguousarray(perm, dtype=np.int32)
        L.jqo_compose_perm(n, len(wires), bits, pm.ctypes.data, cur.ctypes.data, nxt.ctypes.data)
        cur, nxt = nxt, cur
    if memo is not None:
        memo[key] = cur.copy()
    return cur


class ReferencePlan:
    """The reference's plan of one circuit, ready to run in C.

    mixed=False: the statevector plan (_compile, simulation.py:338-345) on n
    wires.  mixed=True: the density-matrix plan (_compile_mixed, :348-381) on
    the 2n-wire vector of the row-major density matrix (simulate_mixed,
    :443-473); `run` then returns the flat dim x dim matrix."""

    def __init__(self, records: Sequence, n: int, mixed: bool = False):
        memo: dict = {}
        self.n_qubits = n
        self.mixed = mixed
        self.n = 2 * n if mixed else n
        if mixed:
            self.entries = O.jaqsi_mixed_plan(records, n)
        else:
            self.entries = O.jaqsi_plan(records, n, compose=lambda run, nn: compose_permutation_c(run, nn, memo))
        m = len(self.entries)
        self.kind = np.zeros(m, dtype=np.int32)
        self.nw = np.zeros(m, dtype=np.int32)
        self.wires = np.zeros(MAXW * m, dtype=np.int32)
        self._keep: List[np.ndarray] = []
        data = (ctypes.c_void_p * m)()
        index = (ctypes.c_void_p * m)()
        for e, ent in enumerate(self.entries):
            if ent[0] == "gather":
                self.kind[e] = _GATHER
                arr = np.ascontiguousarray(ent[1], dtype=np.int32)
                index[e] = arr.ctypes.data
            else:
                self.kind[e] = _DENSE if ent[0] == "dense" else _DIAG
                ws = list(ent[1])
                if ent[0] == "dense" and len(ws) > 4:
                    raise ValueError("the C plan runner applies dense blocks of at most 4 wires")
                self.nw[e] = len(ws)
                self.wires[MAXW * e: MAXW * e + len(ws)] = ws
                arr = np.ascontiguousarray(np.asarray(ent[2], dtype=np.complex128).reshape(-1)).view(np.float64)
                data[e] = arr.ctypes.data
            self._keep.append(arr)
        self._data, self._index = data, index
        self.passes = m

    def run(self, dtype=np.complex128, init: Optional[np.ndarray] = None, bufs=None) -> np.ndarray:
        """Final state (complex64 or complex128) from |0..0> or `init`.
        `bufs` (two float arrays of 2 * 2^n, the run dtype's real type) are
        reused across calls when given (the timed baseline passes them)."""
        L = lib()
        single = np.dtype(dtype) == np.complex64
        rt = np.float32 if single else np.float64
        sfx = "f" if single else ""
        dim = 1 << self.n
        if bufs is None:
            bufs = (np.empty(2 * dim, dtype=rt), np.empty(2 * dim, dtype=rt))
        P = ctypes.POINTER(ctypes.c_float if single else ctypes.c_double)
        b0, b1 = (b.ctypes.data_as(P) for b in bufs)
        if init is None:
            getattr(L, f"jqo_init_zero{sfx}")(b0, self.n)
        else:
            bufs[0][:] = np.ascontiguousarray(init, dtype=dtype).view(rt)
        r = getattr(L, f"jqo_run_plan{sfx}")(b0, b1, self.n, self.passes, self.kind.ctypes.data,
                                             self.nw.ctypes.data, self.wires.ctypes.data,
                                             ctypes.cast(self._data, ctypes.c_void_p),
                                             ctypes.cast(self._index, ctypes.c_void_p))
        return bufs[r].view(np.complex64 if single else np.complex128)

    def expval_z(self, state: np.ndarray, zmasks: Sequence[int]) -> np.ndarray:
        """<Z-string> for each flat-index mask over the n qubits, accumulated
        in float64: measure_state's diagonal fast path
        (jaqsi/simulation.py:777-801) for a statevector, the trace against the
        diagonal of rho (:814-857) for a density matrix."""
        L = lib()
        single = state.dtype == np.complex64
        sfx = "f" if single else ""
        P = ctypes.POINTER(ctypes.c_float if single else ctypes.c_double)
        ptr = state.view(np.float32 if single else np.float64).ctypes.data_as(P)
        fn = getattr(L, f"jqo_expval_z_dm{sfx}" if self.mixed else f"jqo_expval_z{sfx}")
        return np.array([fn(ptr, self.n_qubits, ctypes.c_uint64(z)) for z in zmasks])


def z_masks(n: int) -> List[int]:
    """Flat-index masks of Z_i, i = 0..n-1."""
    return [1 << (n - 1 - i) for i in range(n)]


def zz_masks(n: int) -> List[int]:
    """Flat-index masks of Z_i Z_(i+1), i = 0..n-2 (wire 0 = most significant bit)."""
    return [(1 << (n - 1 - i)) | (1 << (n - 2 - i)) for i in range(n - 1)]


def threads() -> int:
    return int(lib().jqo_max_threads())
