"""Field ids of the C ABI (include/aturan_b200.h, enum aturan_field), with the reference's names.

The names are the cUranusModel member names (planet/cUranusModel.h:1356-1553); the hydrostatic
split vectors p_baro, p_b0, p_bfollow are flat [(i*jm + j)*km + k] vectors there
(cUranusModel.h:1482-1495) and are exchanged here as 3-D fields of the same logical layout.
"""

PROGNOSTIC = [
    "t", "u", "v", "w",
    "ch4", "ch4_cloud", "ch4_ice",
    "h2o", "h2o_cloud", "h2o_ice",
    "h2s", "h2s_cloud", "h2s_ice",
    "nh3", "nh3_cloud", "nh3_ice",
    "nh4sh", "tke", "dis",
]
NCOPIES = [n + "n" for n in PROGNOSTIC]
PRESSURE = ["p_dyn", "p_hydro", "p_stat"]
FORCING = [
    "nue", "thermalmassflux", "Q_precip",
    "S_precip_ch4", "S_precip_ch4_cloud", "S_precip_ch4_ice",
    "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice",
    "S_precip_h2s", "S_precip_h2s_cloud", "S_precip_h2s_ice",
    "S_precip_nh3", "S_precip_nh3_cloud", "S_precip_nh3_ice",
    "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh",
    "rho_mix", "tke_source", "dis_source",
]
HYDRO = ["p_baro", "p_b0", "p_bfollow"]
PROJECTION = ["rhs_u", "rhs_v", "rhs_w", "aux_u", "aux_v", "aux_w"]
# The chemistry's diffusive tendencies (cUranusModel.h:1401-1403), persistent between iterations.
CHEM_STATE = ["difflux_h2s", "difflux_nh3", "difflux_nh4sh"]
# The turbulence closure's shear production (cUranusModel.h:358), a diagnostic it writes.
TURB_DIAG = ["prod"]

NAMES = PROGNOSTIC + NCOPIES + PRESSURE + FORCING + HYDRO + PROJECTION + CHEM_STATE + TURB_DIAG
NFIELDS = len(NAMES)
ID = {n: i for i, n in enumerate(NAMES)}
NPROG = len(PROGNOSTIC)

# The condensables of the saturation adjustment in the iteration loop's order
# (planet/cUranusModel.cpp:998-1027) and their (vapour, cloud, ice) fields.
GASES = ["h2o", "h2s", "nh3", "ch4"]
GAS_FIELDS = {g: (g, g + "_cloud", g + "_ice") for g in GASES}

# Fields every path reads or writes; what a full step touches.
STATE_FIELDS = NAMES

assert NFIELDS == 76, NFIELDS
assert ID["tn"] == 19 and ID["p_dyn"] == 38 and ID["nue"] == 41
assert ID["p_baro"] == 63 and ID["rhs_u"] == 66 and ID["difflux_h2s"] == 72
