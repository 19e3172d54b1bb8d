"""GPU parity of the moist convective adjustment (aturan_mca) against the oracle.

The oracle's restatement is pinned bit for bit to the compiled reference
(tests/test_oracle_vs_ref.py::test_mca). CUDA's exp/log round differently from the host libm in
the last bit, so, as for the saturation adjustment, values agree to 1e-11 of each field's maximum
except in columns where that last bit changes a stability decision or a solve's path; those
columns are counted and must be few.
"""
import numpy as np
import pytest

from aturan_b200 import fields as F, params as P, state as S

pytestmark = pytest.mark.gpu

NAMES = ["t", "nh4sh"] + [n for g in F.GASES for n in F.GAS_FIELDS[g]]


def test_mca_matches_oracle(oracle_lib):
    from aturan_b200.api import Context
    p = P.default_params()
    st = S.synthetic_state(p, seed=72)
    before = st["t"].copy()
    ctx = Context(p)
    ctx.upload_state(st)
    ctx.mca()
    g = ctx.download_state(NAMES)
    ctx.close()
    oracle_lib.mca(p, st)
    bad = np.zeros((p.jm, p.km), dtype=bool)
    for n in NAMES:
        d = np.abs(g[n] - st[n])
        bad |= (d > 1e-11 * max(float(np.abs(st[n]).max()), 1e-300)).any(axis=0)
    nbad = int(bad.sum())
    assert nbad <= 0.01 * bad.size, f"{nbad} of {bad.size} columns beyond 1e-11"
    assert np.count_nonzero(g["t"] != before) > 100000


def test_mca_refuses_mixed_and_deep_columns():
    from aturan_b200.api import AturanError, Context, E_UNSUPPORTED
    for p in (P.default_params(9, 13, 17, precision=P.MIXED), P.default_params(70, 13, 17)):
        ctx = Context(p)
        with pytest.raises(AturanError) as e:
            ctx.mca()
        ctx.close()
        assert e.value.code == E_UNSUPPORTED
