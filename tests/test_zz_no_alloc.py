"""jq_forward_noalloc: the forward entry point for callers that cannot
allocate device memory (FFI hosts holding only raw device pointers, services
under a fixed device-memory budget).  Its workspace is a static 4 MiB device
array inside libjqsim, so the call itself allocates nothing.

Checked through the C ABI against jq_forward (caller-provided workspace) on
two calls in a row, with the device's free memory unchanged across each call,
plus its two rejections: a plan that is not yet resident
on the device and a workspace above the static limit.  Collected last so that
a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import jaqsi_b200 as jq
from jaqsi_b200 import _lib as L
from jaqsi_b200 import simulation as sim

pytestmark = pytest.mark.gpu

TOL = {torch.complex64: 1e-5, torch.complex128: 1e-10}


def _plan(n, layers, dtype, seed):
    ang = np.random.default_rng(seed).uniform(0, 2 * np.pi, (layers, n, 3))
    with jq.recording() as tape:
        for l in range(layers):
            for w in range(n):
                jq.RX(float(ang[l, w, 0]), wires=w)
                jq.Rot(float(ang[l, w, 1]), float(ang[l, w, 2]), 0.3, wires=w)
            for w in range(n):
                jq.CX(wires=[w, (w + 1) % n])
    obs = [jq.build_parity_observable([i, i + 1]) for i in range(n - 1)] + [jq.PauliX(0)]
    lw = sim.lower_tape(tape, n)
    specs, okey = sim._lower_obs(obs, n)
    # a private plan (not shared through the cache) so residency starts empty
    plan = sim.Plan(lw.statics, specs, n, L.JQ_STATEVECTOR, dtype)
    angles = sim.gather_angles(lw.angles, torch.device("cuda"))
    return plan, angles


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_noalloc_forward_matches_forward(dtype):
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    plan, angles = _plan(12, 4, dtype, seed=7)
    lib = plan._lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    # not yet resident on this device: rejected, nothing launched
    state = torch.empty((1, plan.state_elems), dtype=dtype, device=dev)
    out = torch.empty((1, plan.n_obs), dtype=torch.float64, device=dev)
    rc = lib.jq_forward_noalloc(plan.handle, 1, _vp(angles), None, None, 0, L.JQ_OUT_EXPVAL, _vp(state), _vp(out),
                                stream)
    assert rc == L.JQ_EINVAL
    assert b"not resident" in lib.jq_last_error()

    # reference: jq_forward with a caller-provided workspace
    wsb = plan.workspace_bytes(1, 0)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    ref_state = torch.empty_like(state)
    ref_out = torch.empty_like(out)
    L.check(lib.jq_forward(plan.handle, 1, _vp(angles), None, None, 0, L.JQ_OUT_EXPVAL, _vp(ref_state),
                           _vp(ref_out), _vp(ws), wsb, stream))

    # two calls in a row: the static workspace keeps the previous call's contents
    for _ in range(2):
        state.fill_(float("nan"))
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        L.check(lib.jq_forward_noalloc(plan.handle, 1, _vp(angles), None, None, 0, L.JQ_OUT_EXPVAL, _vp(state),
                                       _vp(out), stream))
        torch.cuda.synchronize()
        # the call itself took no device memory
        assert torch.cuda.mem_get_info()[0] == free_before
        np.testing.assert_allclose(out.cpu().numpy(), ref_out.cpu().numpy(), atol=TOL[dtype], rtol=0)
        np.testing.assert_allclose(state.cpu().numpy(), ref_state.cpu().numpy(), atol=TOL[dtype], rtol=0)


def test_noalloc_rejects_oversize_workspace():
    dev = torch.device("cuda", 0)
    plan, angles = _plan(8, 3, torch.complex128, seed=3)
    lib = plan._lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # make the plan resident with one ordinary call
    wsb = plan.workspace_bytes(1, 0)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    st = torch.empty((1, plan.state_elems), dtype=torch.complex128, device=dev)
    L.check(lib.jq_forward(plan.handle, 1, _vp(angles), None, None, 0, L.JQ_OUT_STATE, _vp(st), None, _vp(ws), wsb,
                           stream))
    per_instance = plan.workspace_bytes(1, 0)
    batch = L.JQ_STATIC_WS_BYTES // max(per_instance, 1) + 64
    assert plan.workspace_bytes(batch, 0) > L.JQ_STATIC_WS_BYTES
    rc = lib.jq_forward_noalloc(plan.handle, batch, _vp(angles), None, None, 0, L.JQ_OUT_STATE, _vp(st), None, stream)
    assert rc == L.JQ_ENOMEM
    assert b"static limit" in lib.jq_last_error()
