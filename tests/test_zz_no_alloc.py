"""The entry point that allocates nothing: aturan_buoy_ref_level_static.

It serves callers that may not allocate device memory -- an application whose memory pool owns
the GPU and hands the library only its own buffers, or a plugin run under a fixed device-memory
budget -- by keeping its scratch in a fixed array inside the library. These tests call it through
the C ABI on device buffers the test owns and compare it with the level means that
aturan_rk4_step computes through a context (same tree order; the sin(theta) weights are the
device's there and the host's here, so the two agree to rounding), on two calls in a row: the
second call finds the scratch holding the first call's contents and must give the same answer.

The file is named to be collected last, so a run that stops at the first failure has run every
other test; it passes alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

from aturan_b200 import api, params as P, state as S


def test_static_entry_point_rejects_grids_beyond_its_scratch():
    L = api.load_library()
    p = P.default_params()
    p.im = api.STATIC_MAX_IM + 1
    dummy = ctypes.c_void_p(1)
    rc = L.aturan_buoy_ref_level_static(ctypes.byref(p), dummy, dummy, dummy, None)
    assert rc == api.E_INVALID
    assert b"static scratch" in L.aturan_last_error(None)
    # a level whose cells a 32-bit index cannot count
    p = P.default_params()
    p.jm, p.km = 4096, 300000
    rc = L.aturan_buoy_ref_level_static(ctypes.byref(p), dummy, dummy, dummy, None)
    assert rc == api.E_INVALID
    assert b"level size" in L.aturan_last_error(None)


@pytest.mark.gpu
def test_static_entry_point_matches_context_twice():
    import torch
    torch.cuda.set_device(0)
    L = api.load_library()
    p = P.default_params()
    p.exact_reductions = 0                     # the context's tree order, which the static form uses
    st = S.synthetic_state(p, seed=4242)
    ctx = api.Context(p)
    ctx.upload_state(st)
    ctx.rk4_step()                             # its first kernel forms the level means from t, p_stat
    want = ctx.buoy_ref_level()
    ctx.close()

    t = torch.from_numpy(st["t"]).cuda()
    ps = torch.from_numpy(st["p_stat"]).cuda()
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((p.im,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.aturan_buoy_ref_level_static(ctypes.byref(p), ctypes.c_void_p(t.data_ptr()),
                                            ctypes.c_void_p(ps.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.aturan_last_error(None)
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        rel = np.abs(got - want).max() / np.abs(want).max()
        assert rel <= 1e-14, (call, rel)
