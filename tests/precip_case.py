"""Seeded inputs for the precipitation microphysics, shared by the oracle-vs-reference test (CPU)
and the GPU parity test."""
import numpy as np

from aturan_b200 import fields as F

GASES = ["h2o", "nh3", "ch4", "h2s"]
S_FIELDS = [n for n in F.FORCING if n.startswith("S_precip")]
# every field the precipitation writes with the coupling on
PRECIP_OUT = ["Q_precip"] + S_FIELDS
# and with it off
PRECIP_OUT_UNCOUPLED = ["Q_precip"] + S_FIELDS + [n for g in GASES for n in (g, g + "_cloud", g + "_ice")]


def precip_state(st, p, seed):
    """st with cloud and ice in about 30 % of the cells of every condensable (up to half the
    vapour density, so warm cells pass the autoconversion threshold and cold ones rime), a few
    negative condensate values, and seeded values in Q_precip and the S_precip_* (which the call
    must zero); k = km-1 stays the copy of k = 0."""
    rng = np.random.default_rng(seed)
    s = {n: np.array(a, dtype=np.float64, copy=True) for n, a in st.items()}
    shape = (p.im, p.jm, p.km)
    for g in GASES:
        v = np.abs(s[g])
        for c in ("_cloud", "_ice"):
            a = np.where(rng.random(shape) < 0.3, v * rng.uniform(0.0, 0.5, shape), 0.0)
            a[rng.random(shape) < 0.002] = -1e-12
            s[g + c] = a
    for n in PRECIP_OUT:
        s[n] = rng.normal(0.0, 1e-3, shape)
    for n in PRECIP_OUT_UNCOUPLED:
        s[n][:, :, -1] = s[n][:, :, 0]
    return s
