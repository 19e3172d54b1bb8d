"""GPU parity of the precipitation microphysics (aturan_precipitation) against the oracle.

Bars: FP64 within 1e-11 of each field's maximum (the saturation pressure's exp and log and the
collection terms' pow are CUDA's, which may round differently from the host libm's in the last
bit; every branch of the scheme is continuous in those values, so the difference stays at
rounding level); fields the call does not write untouched. Mixed form (FP32 storage, FP64
arithmetic on the stored values): within 1e-5 of each field's maximum against the oracle run on
the FP32-rounded inputs.
"""
import json
import os

import numpy as np
import pytest

from aturan_b200 import params as P, state as S
from tests.golden.make_golden import CASES, precip_input
from tests.precip_case import PRECIP_OUT, PRECIP_OUT_UNCOUPLED, precip_state

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
UNTOUCHED = ["t", "u", "p_dyn", "rho_mix", "nue", "massflux_h2s"]


def run_gpu(p, st, pp=None, names=()):
    from aturan_b200.api import Context
    ctx = Context(p)
    ctx.upload_state(st)
    ctx.precipitation(pp)
    out = ctx.download_state(list(names))
    ctx.close()
    return out


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("shape", [(41, 181, 361), (9, 13, 17)])
def test_precipitation_fp64_matches_oracle(oracle_lib, shape):
    p, pp = P.default_params(*shape), P.default_precip_params()
    st = precip_state(S.synthetic_state(p, seed=81), p, seed=82)
    g = run_gpu(p, st, pp, PRECIP_OUT_UNCOUPLED + UNTOUCHED)
    st0 = S.copy_state(st)
    oracle_lib.precipitation(p, pp, st)
    for n in PRECIP_OUT_UNCOUPLED:
        assert rel(g[n], st[n]) <= 1e-11, (shape, n, rel(g[n], st[n]))
    for n in UNTOUCHED:
        assert np.array_equal(g[n], st0[n]), n
    assert np.count_nonzero(g["Q_precip"]) > 0


@pytest.mark.parametrize("knob", ["uncoupled", "no_h2s"])
def test_precipitation_fp64_knobs(oracle_lib, knob):
    """The depletion written into the condensate fields (coupling 0), and H2S off with another
    rate scale."""
    p, pp = P.default_params(12, 20, 33), P.default_precip_params()
    if knob == "uncoupled":
        pp.coupling = 0
    else:
        pp.h2s = 0
        pp.rate_scale = 0.003
    st = precip_state(S.synthetic_state(p, seed=83), p, seed=84)
    g = run_gpu(p, st, pp, PRECIP_OUT_UNCOUPLED)
    oracle_lib.precipitation(p, pp, st)
    for n in PRECIP_OUT_UNCOUPLED:
        assert rel(g[n], st[n]) <= 1e-11, (knob, n, rel(g[n], st[n]))


def test_precipitation_near_reference_golden():
    """The FP64 scheme against the compiled reference's sampled values directly (the digests need
    bit equality, which CUDA's exp / log / pow do not promise)."""
    rec = GOLDEN["cases"]["precipitation"]
    p = P.default_params()
    st = precip_input(p, S.synthetic_state(p, seed=rec["seed"]), CASES["precipitation"]["seed"])
    g = run_gpu(p, st, None, list(rec["fields"]))
    for n, want in rec["fields"].items():
        a = g[n].ravel()
        scale = max(np.abs(a).max(), 1e-300)
        for idx, hx in want["samples"]:
            assert abs(a[idx] - float.fromhex(hx)) <= 1e-11 * scale, (n, idx, a[idx], hx)


def test_precipitation_mixed_matches_oracle(oracle_lib):
    p32 = P.default_params(precision=P.MIXED)
    p, pp = P.default_params(), P.default_precip_params()
    st = precip_state(S.synthetic_state(p, seed=85), p, seed=86)
    g = run_gpu(p32, st, pp, PRECIP_OUT)
    s = {n: (a if n in ("t", "tn") else a.astype(np.float32).astype(np.float64)) for n, a in st.items()}
    oracle_lib.precipitation(p, pp, s)
    for n in PRECIP_OUT:
        assert rel(g[n], s[n]) <= 1e-5, (n, rel(g[n], s[n]))
