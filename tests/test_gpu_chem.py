"""GPU parity of the chemistry (aturan_chemistry) against the oracle.

Bars. Forcing (DiffMassFluxUran, the filters, ChemMassRateUran, FluxLimiterNH4SH, the filters):
FP64 bit-exact in every written value (the oracle is pinned bit for bit to the compiled reference
in tests/test_oracle_vs_ref.py and by the golden digest below), fields it does not write
untouched. NH4SH equilibrium: FP64 within 1e-12 of each field's maximum and the counts within 0.1 %
(the bisection's sign tests evaluate CUDA's pow, which may round differently from the host libm's
in the last bit, so a cell's root may land one bisection step away). Mixed form (FP32 storage, FP64
arithmetic on the stored values, T as an FP32 pair): within 1e-5 of each field's maximum against
the oracle run on the FP32-rounded inputs.
"""
import json
import os

import numpy as np
import pytest

from aturan_b200 import fields as F, params as P, state as S
from tests.chem_case import EQ_OUT, FORCING_OUT, chem_state
from tests.golden.make_golden import CASES, chem_input, digest

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
FORCING = 2
EQ = 1


def run_gpu(p, st, what, cp=None, names=()):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    counts = ctx.chemistry(what, cp, counts=True)
    out = ctx.download_state(list(names))
    ctx.close()
    return out, counts


def rounded32(st):
    """The state as the mixed context stores it: every field rounded to FP32 except t, which the
    temperature pair carries to ~2^-48."""
    return {n: (a if n in ("t", "tn") else a.astype(np.float32).astype(np.float64)) for n, a in st.items()}


@pytest.mark.parametrize("shape", [(41, 181, 361), (9, 13, 17)])
def test_forcing_fp64_matches_oracle(oracle_lib, shape):
    p, cp = P.default_params(*shape), P.default_chem_params()
    st = chem_state(S.synthetic_state(p, seed=61), p, seed=62)
    untouched = ["t", "nh3", "h2s", "nh4sh", "u", "p_dyn", "nue"]
    g, _ = run_gpu(p, st, FORCING, cp, FORCING_OUT + untouched)
    st0 = S.copy_state(st)
    oracle_lib.chem_forcing(p, cp, st)
    for n in FORCING_OUT:
        ne = np.count_nonzero(g[n] != st[n])
        assert ne == 0, (shape, n, ne, np.abs(g[n] - st[n]).max())
    for n in untouched:
        assert np.array_equal(g[n], st0[n]), n
    assert np.count_nonzero(st["fluxlim_nh4sh"]) > 0


@pytest.mark.parametrize("knob", ["minus_sign", "open_phi"])
def test_forcing_fp64_knobs(oracle_lib, knob):
    """difflux_plus = 0 (massflux = -difflux) and the open phi seam (phi_periodic = 0: k from 1,
    plain neighbours, filters without the ring)."""
    p, cp = P.default_params(12, 20, 33), P.default_chem_params()
    if knob == "minus_sign":
        cp.difflux_plus = 0
    else:
        cp.phi_periodic = 0
    st = chem_state(S.synthetic_state(p, seed=63), p, seed=64)
    g, _ = run_gpu(p, st, FORCING, cp, FORCING_OUT)
    oracle_lib.chem_forcing(p, cp, st)
    for n in FORCING_OUT:
        assert np.array_equal(g[n], st[n]), (knob, n)


def test_forcing_reproduces_reference_golden():
    """The FP64 forcing against the compiled reference's digests directly."""
    rec = GOLDEN["cases"]["chem_forcing"]
    p = P.default_params()
    st = chem_input(p, S.synthetic_state(p, seed=rec["seed"]), CASES["chem_forcing"]["seed"])
    g, _ = run_gpu(p, st, FORCING, None, list(rec["fields"]))
    for n, want in rec["fields"].items():
        assert digest(g[n]) == want["sha256"], n


@pytest.mark.parametrize("shape", [(41, 181, 361), (9, 13, 17)])
def test_nh4sh_eq_fp64_matches_oracle(oracle_lib, shape):
    p, cp = P.default_params(*shape), P.default_chem_params()
    st = chem_state(S.synthetic_state(p, seed=65), p, seed=66)
    g, (gf, gd) = run_gpu(p, st, EQ, cp, EQ_OUT + ["u", "massflux_h2s"])
    st0 = S.copy_state(st)
    of, od = oracle_lib.nh4sh_eq(p, cp, st)
    for n in EQ_OUT:
        d = np.abs(g[n] - st[n]).max() / np.abs(st[n]).max()
        assert d <= 1e-12, (shape, n, d)
    for n in ("u", "massflux_h2s"):
        assert np.array_equal(g[n], st0[n]), n
    assert abs(gf - of) <= max(2, of // 1000) and abs(gd - od) <= max(2, od // 1000), (gf, of, gd, od)
    if shape[0] == 41:
        assert of > 10000 and od > 10000, (of, od)


def test_chemistry_both_parts_in_order(oracle_lib):
    """what = NH4SH_EQ | FORCING runs the equilibrium first, then the forcing on its result."""
    p, cp = P.default_params(12, 20, 33), P.default_chem_params()
    st = chem_state(S.synthetic_state(p, seed=67), p, seed=68)
    g, _ = run_gpu(p, st, EQ | FORCING, cp, EQ_OUT + FORCING_OUT)
    oracle_lib.nh4sh_eq(p, cp, st)
    oracle_lib.chem_forcing(p, cp, st)
    for n in EQ_OUT + FORCING_OUT:
        d = np.abs(g[n] - st[n]).max() / max(np.abs(st[n]).max(), 1e-300)
        assert d <= 1e-10, (n, d)


@pytest.mark.parametrize("what", [EQ, FORCING])
def test_chemistry_mixed_matches_oracle(oracle_lib, what):
    """Each part alone on the same FP32-rounded inputs as the oracle. (Run back to back, the
    equilibrium's FP32-rounded NH4SH would feed the Superbee limiter, whose ratio of neighbour
    differences is ill-conditioned where NH4SH is nearly uniform: its output differs there by a few
    per cent of its maximum between an FP32 and an FP64 NH4SH, a property of the limiter, not of
    the arithmetic.)"""
    p32 = P.default_params(precision=P.MIXED)
    p, cp = P.default_params(), P.default_chem_params()
    st = chem_state(S.synthetic_state(p, seed=69), p, seed=70)
    names = EQ_OUT if what == EQ else FORCING_OUT
    g, (gf, gd) = run_gpu(p32, st, what, cp, names)
    s = rounded32(st)
    if what == EQ:
        of, od = oracle_lib.nh4sh_eq(p, cp, s)
        assert abs(gf - of) <= of // 100 and abs(gd - od) <= od // 100, (gf, of, gd, od)
    else:
        oracle_lib.chem_forcing(p, cp, s)
    for n in names:
        d = np.abs(g[n] - s[n]).max() / np.abs(s[n]).max()
        assert d <= 1e-5, (n, d)


def test_chemistry_rejects_unsupported_knobs():
    from aturan_b200.api import AturanError, Context, E_UNSUPPORTED
    p = P.default_params(9, 13, 17)
    ctx = Context(p)
    try:
        for field, value in (("nh4sh_eq", 0), ("difflux_laplacian", 0)):
            cp = P.default_chem_params()
            setattr(cp, field, value)
            with pytest.raises(AturanError) as e:
                ctx.chemistry(FORCING, cp)
            assert e.value.code == E_UNSUPPORTED, field
    finally:
        ctx.close()
