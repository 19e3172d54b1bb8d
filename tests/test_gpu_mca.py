"""GPU parity of the moist convective adjustment (aturan_mca) against the oracle.

The oracle's restatement is pinned bit for bit to the compiled reference
(tests/test_oracle_vs_ref.py::test_mca). CUDA's exp/log round differently from the host libm in
the last bit, so, as for the saturation adjustment, values agree to 1e-11 of each field's maximum
except in columns where that last bit changes a stability decision or a solve's path. Those
columns are counted (a few per thousand are expected) and checked for sense: every value finite,
T within 2 K of the oracle's, every species within the range the oracle's column spans.
"""
import numpy as np
import pytest

from aturan_b200 import fields as F, params as P, state as S

pytestmark = pytest.mark.gpu

NAMES = ["t", "nh4sh"] + [n for g in F.GASES for n in F.GAS_FIELDS[g]]


def run_gpu(p, st):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    ctx.mca()
    g = ctx.download_state(NAMES)
    ctx.close()
    return g


def compare(p, g, o, tol, max_bad_frac):
    """Columns beyond tol of each field's maximum are counted; in them every value must be finite,
    T within 2 K (of the oracle's, in kelvin) and each species within its oracle column's range
    widened by 1 % of the field's maximum."""
    bad = np.zeros((p.jm, p.km), dtype=bool)
    for n in NAMES:
        assert np.all(np.isfinite(g[n])), n
        d = np.abs(g[n] - o[n])
        bad |= (d > tol * max(float(np.abs(o[n]).max()), 1e-300)).any(axis=0)
    nbad = int(bad.sum())
    assert nbad <= max_bad_frac * bad.size, f"{nbad} of {bad.size} columns beyond {tol}"
    if nbad:
        jj, kk = np.nonzero(bad)
        dT = np.abs(g["t"][:, jj, kk] - o["t"][:, jj, kk]) * p.t_ref
        assert dT.max() <= 2.0, dT.max()
        for n in NAMES[1:]:
            col_o = o[n][:, jj, kk]
            slack = 0.01 * max(float(np.abs(o[n]).max()), 1e-300)
            lo, hi = col_o.min(axis=0) - slack, col_o.max(axis=0) + slack
            assert np.all((g[n][:, jj, kk] >= lo) & (g[n][:, jj, kk] <= hi)), n
    return nbad


def test_mca_matches_oracle(oracle_lib):
    p = P.default_params()
    st = S.synthetic_state(p, seed=72)
    before = st["t"].copy()
    g = run_gpu(p, st)
    oracle_lib.mca(p, st)
    compare(p, g, st, 1e-11, 0.005)
    assert np.count_nonzero(g["t"] != before) > 100000


@pytest.mark.parametrize("shape", [(70, 13, 17), (190, 9, 9)])
def test_mca_deep_columns(oracle_lib, shape):
    """Columns deeper than one warp's 32 lanes (and, at 190 levels, than 48 KB of shared memory for
    four warps): each lane takes several levels."""
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=73)
    g = run_gpu(p, st)
    oracle_lib.mca(p, st)
    compare(p, g, st, 1e-11, 0.02)


def test_mca_mixed_matches_oracle(oracle_lib):
    """The mixed form (FP32 storage, T as an FP32 pair, FP64 arithmetic) against the oracle on the
    same FP32-rounded inputs: the column decisions see inputs that agree to the pair's precision,
    so the values agree to FP32 rounding outside the counted columns."""
    p32 = P.default_params(precision=P.MIXED)
    p = P.default_params()
    st = S.synthetic_state(p, seed=74)
    g = run_gpu(p32, st)
    s = {n: (a if n in ("t", "tn") else a.astype(np.float32).astype(np.float64)) for n, a in st.items()}
    oracle_lib.mca(p, s)
    compare(p, g, s, 1e-6, 0.01)
