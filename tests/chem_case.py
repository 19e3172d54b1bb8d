"""Seeded inputs for the chemistry (NH4SH equilibrium and the chemistry forcing), shared by the
oracle-vs-reference test (CPU) and the GPU parity test."""
import numpy as np

from aturan_b200 import fields as F

# the persistent fields the forcing reads on the boundary rows and overwrites inside
PERSISTENT = F.CHEM_STATE + ["massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "thermalmassflux"]
# every field the forcing writes
FORCING_OUT = ["rho_mix"] + PERSISTENT
# every field the equilibrium writes
EQ_OUT = ["t", "nh3", "h2s", "nh4sh"]


def chem_state(st, p, seed):
    """st with seeded values in the persistent chemistry fields (boundary rows included), NH4SH
    present in every cell and NH3 depleted a millionfold in a fifth of them, so that the
    equilibrium both forms NH4SH (where NH3 and H2S are supersaturated) and decomposes it (where
    NH3 is depleted); k = km-1 stays the copy of k = 0."""
    rng = np.random.default_rng(seed)
    s = {n: np.array(a, dtype=np.float64, copy=True) for n, a in st.items()}
    shape = (p.im, p.jm, p.km)
    scale = {"fluxlim_nh4sh": 1e-12, "thermalmassflux": 1e-3}
    for n in PERSISTENT:
        s[n] = rng.normal(0.0, scale.get(n, 1e-9), shape)
    s["nh4sh"] = np.abs(rng.normal(0.0, 1e-5, shape))
    m = rng.random(shape) < 0.2
    s["nh3"][m] *= 1e-6
    for n in PERSISTENT + ["nh4sh", "nh3"]:
        s[n][:, :, -1] = s[n][:, :, 0]
    return s
