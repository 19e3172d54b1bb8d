"""GPU parity of one iteration of the reference's loop (aturan_iteration) against the oracle's
iteration, which reproduces the compiled reference's own Run() bit for bit
(tests/test_oracle_vs_ref.py::test_reference_loop).

FP64, 4 iterations (two odd: RK4 onward; two even: the full sequence), every module at the
reference's defaults, PressureSolverUran's sweep: every field finite, in every field 99.99 % of the
cells within 1e-10 of its maximum and at most 0.01 % beyond 1e-9 (the transcendental-dependent
modules -- saturation adjustment, MCA, precipitation, NH4SH equilibrium -- round CUDA's exp / log /
pow differently from glibc's in the last bit, which can move isolated cells; on the synthetic
state measured: none beyond 1.1e-12). Mixed form, 4 iterations, against the FP64 device
iteration: T and u within 1e-5 of their maxima, every field's 99.99th percentile within 1e-4.
"""
import numpy as np
import pytest

from aturan_b200 import fields as F, params as P, state as S

pytestmark = pytest.mark.gpu

NAMES = [n for n in F.NAMES if n not in F.PROJECTION]


def run_gpu(p, st, ip, n):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    for it in range(1, n + 1):
        ctx.iteration(it, ip)
    out = ctx.download_state(NAMES)
    ctx.close()
    return out


def stats(g, o, n):
    s = max(float(np.abs(o[n]).max()), 1e-300)
    d = np.abs(g[n] - o[n]) / s
    return float(d.max()), float(np.quantile(d, 0.9999)), float((d > 1e-9).mean())


def test_iteration_fp64_matches_oracle(oracle_lib):
    p, ip = P.default_params(), P.default_iter_params()
    st = S.synthetic_state(p, seed=123)
    g = run_gpu(p, st, ip, 4)
    for it in range(1, 5):
        oracle_lib.iteration(p, ip, st, it)
    for n in NAMES:
        assert np.all(np.isfinite(g[n])), n
        mx, q, frac = stats(g, st, n)
        assert q <= 1e-10 and frac <= 1e-4, (n, mx, q, frac)


def test_iteration_knobs_fp64(oracle_lib):
    """The shared red-black solver with its own sweeps, the p_dyn filter on all axes
    (DAMP_P_HORIZ 1), the MCA every second iteration, H2S precipitation off."""
    p, ip = P.default_params(12, 20, 33), P.default_iter_params()
    ip.press_kind, ip.max_sweeps = P.PRESS_RB_SHARED, 3
    ip.damp_p_horiz = 1.0
    ip.mca_stride = 2
    ip.precip.h2s = 0
    st = S.synthetic_state(p, seed=124)
    g = run_gpu(p, st, ip, 4)
    for it in range(1, 5):
        oracle_lib.iteration(p, ip, st, it)
    for n in NAMES:
        assert np.all(np.isfinite(g[n])), n
        mx, q, frac = stats(g, st, n)
        assert q <= 1e-10 and frac <= 1e-3, (n, mx, q, frac)


def test_iteration_mixed_against_fp64():
    ip = P.default_iter_params()
    p64, p32 = P.default_params(), P.default_params(precision=P.MIXED)
    st = S.synthetic_state(p64, seed=125)
    g64 = run_gpu(p64, st, ip, 4)
    g32 = run_gpu(p32, st, ip, 4)
    for n in ("t", "u"):
        assert stats(g32, g64, n)[0] <= 1e-5, (n, stats(g32, g64, n))
    for n in NAMES:
        assert np.all(np.isfinite(g32[n])), n
        assert stats(g32, g64, n)[1] <= 1e-4, (n, stats(g32, g64, n))


def test_iteration_rejects_before_launching():
    from aturan_b200.api import AturanError, Context, E_UNSUPPORTED
    p = P.default_params(9, 13, 17)
    ctx = Context(p)
    try:
        ip = P.default_iter_params()
        ip.turb.buoy = 1
        with pytest.raises(AturanError) as e:
            ctx.iteration(2, ip)
        assert e.value.code == E_UNSUPPORTED
    finally:
        ctx.close()
