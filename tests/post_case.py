"""Seeded inputs and knob sets for the passes after RK4 (filters, boundary passes, species clamp).

Shared by the oracle-vs-reference test (CPU) and the GPU parity test. A knob set is the ATURAN_*
environment the reference reads and the aturan_post_params that environment resolves to.
"""
import numpy as np

from aturan_b200 import fields as F, params as P

SPECIES = ["h2o", "h2o_cloud", "h2o_ice", "h2s", "h2s_cloud", "h2s_ice", "nh3", "nh3_cloud",
           "nh3_ice", "ch4", "ch4_cloud", "ch4_ice", "nh4sh"]
FLUXES = ["massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "thermalmassflux"]
# every field the passes write
POST_FIELDS = ["t", "u", "v", "w"] + SPECIES + FLUXES + F.CHEM_STATE


def post_state(st, p, seed, nan=True):
    """st with seeded fluxes, negative species values in ~1 % of the cells (boundary planes
    included) and (nan=True) two NaNs, so the floor and the clamp have work."""
    rng = np.random.default_rng(seed)
    s = {n: np.array(a, dtype=np.float64, copy=True) for n, a in st.items()}
    shape = (p.im, p.jm, p.km)
    for n in FLUXES:
        s[n] = rng.normal(0.0, 1e-3, shape)
    for n in SPECIES:
        a = s[n]
        scale = max(float(np.abs(a).max()), 1e-12)
        m = rng.random(shape) < 0.01
        a[m] = -scale * rng.random(int(m.sum()))
    if nan:
        s["h2o"][p.im // 2, p.jm // 2, p.km // 2] = np.nan
        s["nh3_ice"][0, p.jm // 3, p.km // 4] = np.nan
    for n in F.CHEM_STATE:                     # drawn last: the draws above keep their values
        s[n] = rng.normal(0.0, 1e-9, shape)
    return s


def _pp(**kw):
    pp = P.default_post_params(geo_balance=kw.pop("geo_balance", True))
    for k, v in kw.items():
        setattr(pp, k, v)
    return pp


# name -> (environment of the reference, the post params it resolves to)
KNOB_SETS = {
    "defaults": ({}, lambda: _pp()),
    "no_geo_balance_forms": ({"ATURAN_GEO_BALANCE": "0", "ATURAN_BC_RADIUS_COPY": "3", "ATURAN_BC_BOTTOM_FORM": "1",
                              "ATURAN_BC_POLE_COPY": "1", "ATURAN_BC_TOP_TAPER": "2", "ATURAN_BC_RADIUS_POSITIVE": "2",
                              "ATURAN_DAMP_T_VERT": "0.5", "ATURAN_DAMP_T_HORIZ": "0.7", "ATURAN_BC_LID_U": "0"},
                             lambda: _pp(geo_balance=False, radius_form=3, bottom_form=1, pole_form=1, top_taper=2,
                                         radius_positive=2, damp_t_vert=0.5, damp_t_horiz=0.7, lid_u=0)),
    "cubic_lid_open_phi": ({"ATURAN_BC_LID_VW": "3", "ATURAN_BC_TOP_TAPER": "1", "ATURAN_DAMP_T_J": "1",
                            "ATURAN_BC_PHI_PERIODIC": "0", "ATURAN_SPECIES_CLAMP": "0", "ATURAN_BC_RADIUS_POSITIVE": "0",
                            "ATURAN_VEL_SHAPIRO": "0.3", "ATURAN_BC_RADIUS_COPY": "1"},
                           lambda: _pp(lid_vw=3, top_taper=1, damp_t_j=1, phi_periodic=0, species_clamp=0,
                                       radius_positive=0, vel_shapiro=0.3, radius_form=1)),
}
