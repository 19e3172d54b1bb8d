"""GPU parity of the passes after RK4 (aturan_post_step) against the oracle.

Bars: FP64 bit-exact in every written value for every knob set (the oracle is pinned bit for bit
to the compiled reference in tests/test_oracle_vs_ref.py and by the golden digest below), the
clamp's counts equal and its sums within 1e-12 (the summation order differs); fields the passes
do not write untouched. Mixed form (FP32 storage, FP64 arithmetic on the stored values): within
1e-6 of each field's maximum against the oracle run on the FP32-rounded inputs, the clamp's
counts equal.
"""
import json
import os

import numpy as np
import pytest

from aturan_b200 import params as P, state as S
from tests.golden.make_golden import CASES, digest, post_input
from tests.post_case import KNOB_SETS, POST_FIELDS, post_state

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
UNTOUCHED = ["tke", "dis", "p_dyn", "nue", "rho_mix", "tn", "h2on"]


def run_gpu(p, st, pp):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    added, cells = ctx.post_step(pp, sums=True)
    out = ctx.download_state(POST_FIELDS + UNTOUCHED)
    ctx.close()
    return out, added, cells


@pytest.mark.parametrize("shape", [(41, 181, 361), (9, 13, 17), (5, 5, 5)])
@pytest.mark.parametrize("knobs", list(KNOB_SETS))
def test_post_step_fp64_matches_oracle(oracle_lib, knobs, shape):
    p = P.default_params(*shape)
    st = post_state(S.synthetic_state(p, seed=51), p, seed=52)
    pp = KNOB_SETS[knobs][1]()
    g, ga, gc = run_gpu(p, st, pp)
    st0 = S.copy_state(st)
    oa, oc = oracle_lib.post_step(p, st, pp)
    for n in POST_FIELDS:
        ne = np.count_nonzero(~((g[n] == st[n]) | (np.isnan(g[n]) & np.isnan(st[n]))))
        assert ne == 0, (knobs, shape, n, ne)
    for n in UNTOUCHED:
        assert np.array_equal(g[n], st0[n]), n
    assert np.array_equal(gc, oc), (gc, oc)
    assert np.allclose(ga, oa, rtol=1e-12, atol=0.0), (ga, oa)
    if pp.species_clamp:
        assert gc.sum() > 0


def test_post_step_reproduces_reference_golden():
    """The FP64 passes against the compiled reference's digests directly (default knobs)."""
    rec = GOLDEN["cases"]["post_step"]
    p = P.default_params()
    st = post_input(p, S.synthetic_state(p, seed=rec["seed"]), CASES["post_step"]["seed"])
    g, _, _ = run_gpu(p, st, P.default_post_params())
    for n, want in rec["fields"].items():
        assert digest(g[n]) == want["sha256"], n


@pytest.mark.parametrize("knobs", ["defaults", "no_geo_balance_forms"])
def test_post_step_mixed_within_fp32_rounding(oracle_lib, knobs):
    p = P.default_params(precision=P.MIXED)
    st = post_state(S.synthetic_state(p, seed=53), p, seed=54)
    st32 = dict(st)                        # the passes' fields as the FP32 context stores them
    for n in POST_FIELDS:
        st32[n] = st[n].astype(np.float32).astype(np.float64)
    pp = KNOB_SETS[knobs][1]()
    g, ga, gc = run_gpu(p, st32, pp)
    p64 = P.default_params()
    oa, oc = oracle_lib.post_step(p64, st32, pp)
    for n in POST_FIELDS:
        ref = st32[n]
        scale = max(float(np.abs(ref).max()), 1e-30)
        assert np.abs(g[n] - ref).max() <= 1e-6 * scale, (knobs, n, np.abs(g[n] - ref).max() / scale)
    assert np.array_equal(gc, oc), (gc, oc)
    assert np.allclose(ga, oa, rtol=1e-5, atol=0.0), (ga, oa)


def test_iteration_sequence_matches_oracle(oracle_lib):
    """Two iterations of a driver's sequence -- aturan_step (GS pressure), aturan_post_step,
    aturan_restore_ncopies -- against the oracle's same calls, FP64, on the config-3 grid. Every
    prognostic field and n-copy, boundary planes included, within 1e-10 of its maximum: the
    saturation adjustment's last-bit exp/log differences (the one-step bar, 1e-11) carried
    through two iterations and the post passes."""
    from aturan_b200 import fields as F
    from aturan_b200.api import Context
    p = P.default_params(41, 91, 181)
    st = post_state(S.synthetic_state(p, seed=61), p, seed=62, nan=False)
    pp = P.default_post_params()
    ctx = Context(p)
    ctx.upload_state(st)
    for _ in range(2):
        ctx.step(P.PRESS_GS_LEX)
        ctx.post_step(pp)
        ctx.restore_ncopies(1.0)
        oracle_lib.step(p, st, P.PRESS_GS_LEX)
        oracle_lib.post_step(p, st, pp)
        for n in F.PROGNOSTIC:                     # restoreVar(1.0)
            st[n + "n"] = st[n].copy()
    names = F.PROGNOSTIC + F.NCOPIES + ["p_dyn"]
    g = ctx.download_state(names)
    ctx.close()
    for n in names:
        scale = max(float(np.abs(st[n]).max()), 1e-300)
        assert np.abs(g[n] - st[n]).max() <= 1e-10 * scale, (n, np.abs(g[n] - st[n]).max() / scale)


def test_post_step_rejects_bad_version():
    from aturan_b200.api import AturanError, Context, E_INVALID
    p = P.default_params(9, 13, 17)
    ctx = Context(p)
    pp = P.default_post_params()
    pp.abi_version = 99
    with pytest.raises(AturanError) as e:
        ctx.post_step(pp)
    ctx.close()
    assert e.value.code == E_INVALID
