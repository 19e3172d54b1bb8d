"""GPU parity of the turbulence closure (aturan_turbulence) against the oracle.

Bars: FP64 bit-exact in every value the closure writes (the oracle is pinned bit for bit to the
compiled reference in tests/test_oracle_vs_ref.py and by the golden digest below); fields it does
not write untouched. Mixed form (FP32 storage, FP64 arithmetic on the stored values): within 1e-5
of each field's maximum against the oracle run on the FP32-rounded inputs.
"""
import json
import os

import numpy as np
import pytest

from aturan_b200 import params as P, state as S
from tests.golden.make_golden import CASES, digest, turb_input
from tests.turb_case import TURB_OUT, turb_state

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
UNTOUCHED = ["t", "u", "w", "h2o", "p_dyn", "rho_mix", "massflux_h2s"]


def run_gpu(p, st, tp=None, names=()):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    ctx.turbulence(tp)
    out = ctx.download_state(list(names))
    ctx.close()
    return out


@pytest.mark.parametrize("shape", [(41, 181, 361), (9, 13, 17), (5, 5, 5)])
def test_turbulence_fp64_matches_oracle(oracle_lib, shape):
    p, tp = P.default_params(*shape), P.default_turb_params()
    st = turb_state(S.synthetic_state(p, seed=71), p, seed=72)
    g = run_gpu(p, st, tp, TURB_OUT + UNTOUCHED)
    st0 = S.copy_state(st)
    oracle_lib.turbulence(p, tp, st)
    for n in TURB_OUT:
        ne = np.count_nonzero(g[n] != st[n])
        assert ne == 0, (shape, n, ne, np.abs(g[n] - st[n]).max())
    for n in UNTOUCHED:
        assert np.array_equal(g[n], st0[n]), n


@pytest.mark.parametrize("knob", ["no_curvature", "open_phi"])
def test_turbulence_fp64_knobs(oracle_lib, knob):
    """TURB_CURV = 0 (no curvature terms) and the open phi seam (k from 1, plain neighbours, no
    seam copy)."""
    p, tp = P.default_params(12, 20, 33), P.default_turb_params()
    if knob == "no_curvature":
        tp.curv = 0
    else:
        tp.phi_periodic = 0
    st = turb_state(S.synthetic_state(p, seed=73), p, seed=74)
    g = run_gpu(p, st, tp, TURB_OUT)
    oracle_lib.turbulence(p, tp, st)
    for n in TURB_OUT:
        assert np.array_equal(g[n], st[n]), (knob, n)


def test_turbulence_reproduces_reference_golden():
    """The FP64 closure against the compiled reference's digests directly."""
    rec = GOLDEN["cases"]["turbulence"]
    p = P.default_params()
    st = turb_input(p, S.synthetic_state(p, seed=rec["seed"]), CASES["turbulence"]["seed"])
    g = run_gpu(p, st, None, list(rec["fields"]))
    for n, want in rec["fields"].items():
        assert digest(g[n]) == want["sha256"], n


def test_turbulence_mixed_matches_oracle(oracle_lib):
    p32 = P.default_params(precision=P.MIXED)
    p, tp = P.default_params(), P.default_turb_params()
    st = turb_state(S.synthetic_state(p, seed=75), p, seed=76)
    g = run_gpu(p32, st, tp, TURB_OUT)
    s = {n: a.astype(np.float32).astype(np.float64) for n, a in st.items()}
    oracle_lib.turbulence(p, tp, s)
    for n in TURB_OUT:
        d = np.abs(g[n] - s[n]).max() / np.abs(s[n]).max()
        assert d <= 1e-5, (n, d)


def test_turbulence_rejects_unsupported_knobs():
    from aturan_b200.api import AturanError, Context, E_UNSUPPORTED
    ctx = Context(P.default_params(9, 13, 17))
    try:
        for field, value in (("model", 0), ("turb_free", 0), ("clamp_pass", 0), ("buoy", 1), ("abl_taper", 1)):
            tp = P.default_turb_params()
            setattr(tp, field, value)
            with pytest.raises(AturanError) as e:
                ctx.turbulence(tp)
            assert e.value.code == E_UNSUPPORTED, field
    finally:
        ctx.close()
