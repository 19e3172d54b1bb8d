"""The `aturan_params` struct of include/aturan_b200.h as a ctypes Structure, and its defaults.

The defaults are the values the reference holds after its own initialisation on the
41 x 181 x 361 grid with no ATURAN_* variable set:

* grid and config scalars: planet/cUranusModel.cpp:336-351, planet/cUranusDefaults.cpp.inc;
* mixture properties r_mix, R_mix, cp_mix, mue_mix and the densities r_h2, r_he, r_ch4 after
  ThermalPropertiesUran and the T-anchor rescale (cUranusModel.cpp:498-526) -- written as exact
  hexadecimal doubles because they are computed, not typed, by the reference;
* the resolved knob defaults of the path (cUranusModel.h:116-117, 521-597, 1438-1498;
  RHS_Uran_Turb.cpp:208-672; PressureSolver.h:168-237; SaturationAdjustment.h:283-302);
* per-gas constants as SaturationAdjustmentUran::run passes them (SaturationAdjustmentUran.cpp:
  222-238: H2S has no ice set and uses its liquid one).
"""
import ctypes
import math

ABI_VERSION = 1
FP64, MIXED = 0, 1
PRESS_GS_LEX, PRESS_RB_SHARED, PRESS_RB_SOR, PRESS_RB_LINE = 0, 1, 2, 3


class Gas(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "t_0", "t_00", "ep", "lv", "ls", "C", "L0", "R", "del_alf", "del_bet",
        "C_i", "L0_i", "del_alf_i", "del_bet_i")]


_INT_FIELDS = (
    "abi_version", "im", "jm", "km", "precision", "turb_active", "coriolis_full",
    "cp_h2_mode", "cp_gas", "cp_dyn", "press_consistent", "press_incr", "rigid_lid",
    "satadj_conserve", "satadj_newton", "satadj_evap", "satadj_ice_entry",
    "satadj_bergeron", "satadj_freeze", "satadj_dry_exit", "local_rho", "nh4sh_sync",
    "exact_reductions")
_DBL_FIELDS = (
    "r0", "dr", "the0", "dthe", "phi0", "dphi", "dt", "metric_R_km", "sinthe_min",
    "L_atm", "u_0", "t_ref", "g", "omega", "re", "pr",
    "Coriolis", "centrifugal", "buoyancy", "chemical_reaction", "R_ref", "p_ref",
    "r_mix", "R_mix", "cp_mix", "mue_mix",
    "r_h2", "r_he", "r_ch4", "cp_h2", "cp_he", "cp_ch4",
    "sc_ch4", "sc_h2o", "sc_h2s", "sc_nh3", "sc_nh4sh",
    "alpha_sponge", "r_p_nh4sh", "rho_cond_nh4sh",
    "turb_coupling", "precip_coupling", "tmf_scale", "cent_mom", "pbaro_follow",
    "t_min_K", "t_max_K", "p_dyn_cap", "satadj_stop_tol", "satadj_entry_tol")


class Params(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_int32) for n in _INT_FIELDS]
                + [("reserved_i", ctypes.c_int32 * 7)]
                + [(n, ctypes.c_double) for n in _DBL_FIELDS]
                + [("reserved_d", ctypes.c_double * 6), ("gas", Gas * 4)])

    def copy(self):
        p = Params()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(Params))
        return p

    @property
    def shape(self):
        return (self.im, self.jm, self.km)


_H = float.fromhex
# (t_0, t_00, ep, lv, ls, C, L0, R, del_alf, del_bet, C_i, L0_i, del_alf_i, del_bet_i)
# cUranusModel.h:880-906 (t_0, t_00), :1092-1098 (ep), :1101-1115 (lv, ls), :1143-1192 (sets)
GAS_DEFAULTS = {
    "h2o": (273.15, 210.15, 8.1253, 2.5009e6, 2.8339e6, 25.096, 3148.2, 461.52, 0.0, -8.7e-3,
            28.418, 3567.3, 0.0, -8.7e-3),
    "h2s": (187.65, 140.0, 14.5192, 5.5e5, 7.45e5, 17.064, 747.0, 243.96, 0.0, -2.9e-3,
            17.064, 747.0, 0.0, -2.9e-3),
    "nh3": (195.5, 140.0, 7.6752, 1.3720e6, 1.8320e6, 27.863, 2016.0, 488.21, -0.888, 0.0,
            34.948, 2692.5, -0.888, 0.0),
    "ch4": (90.69, 67.36, 7.6752, 5.11e5, 5.11e5, 1.627, 553.1, 518.28, 1.002, -4.1e-3,
            1.627, 553.1, 1.002, -4.1e-3),
}

DEFAULTS = dict(
    abi_version=ABI_VERSION, im=41, jm=181, km=361, precision=FP64,
    turb_active=1, coriolis_full=1, cp_h2_mode=2, cp_gas=1, cp_dyn=1,
    press_consistent=1, press_incr=1, rigid_lid=1,
    satadj_conserve=1, satadj_newton=1, satadj_evap=1, satadj_ice_entry=0,
    satadj_bergeron=2, satadj_freeze=1, satadj_dry_exit=1, local_rho=1, nh4sh_sync=1,
    exact_reductions=1,
    r0=1.0, dr=0.025, the0=0.0, dthe=1.0 / (180.0 / math.pi), phi0=0.0,
    dphi=1.0 / (180.0 / math.pi), dt=0.001, metric_R_km=25362.0, sinthe_min=0.4,
    L_atm=225.0, u_0=100.0, t_ref=76.4, g=8.69, omega=0.000101, re=1000.0, pr=0.69,
    Coriolis=1.0, centrifugal=1.0, buoyancy=1.0, chemical_reaction=1.0, R_ref=3.61491, p_ref=1.0,
    r_mix=_H("0x1.d296ea433d4a6p+1"), R_mix=_H("0x1.31fad52a5899ap+11"),
    cp_mix=_H("0x1.0f59f37b7f291p+13"), mue_mix=_H("0x1.5e6b31135aa58p-17"),
    r_h2=_H("0x1.e0c778070069fp+0"), r_he=_H("0x1.2eb67afaed4c3p-2"),
    r_ch4=_H("0x1.a6e858fcad66bp-2"), cp_h2=14.32e3, cp_he=5.19e3, cp_ch4=2.232e3,
    sc_ch4=0.99, sc_h2o=0.61, sc_h2s=0.94, sc_nh3=0.61, sc_nh4sh=0.7,
    alpha_sponge=10.0, r_p_nh4sh=1.0e-5, rho_cond_nh4sh=1170.0,
    turb_coupling=1.0, precip_coupling=1.0, tmf_scale=0.0, cent_mom=0.0, pbaro_follow=64.0,
    t_min_K=7.5, t_max_K=2000.0, p_dyn_cap=0.2, satadj_stop_tol=1.0e-3, satadj_entry_tol=0.0,
)


def default_params(im=None, jm=None, km=None, precision=FP64):
    """The reference's defaults; a different grid keeps every constant (degrees per cell are
    rescaled so the grid still spans 0..180 deg in theta and 0..360 deg in phi)."""
    p = Params()
    for k, v in DEFAULTS.items():
        setattr(p, k, v)
    for n, g in enumerate(("h2o", "h2s", "nh3", "ch4")):
        for fname, val in zip([f[0] for f in Gas._fields_], GAS_DEFAULTS[g]):
            setattr(p.gas[n], fname, val)
    if im is not None:
        p.im = im
    if jm is not None:
        p.jm = jm
        p.dthe = (180.0 / (jm - 1)) / (180.0 / math.pi)
    if km is not None:
        p.km = km
        p.dphi = (360.0 / (km - 1)) / (180.0 / math.pi)
    if im is not None and im != 41:
        p.dr = 1.0 / (im - 1)
    p.precision = precision
    return p


def params_from_ref(ref):
    """Params carrying the scalars of an initialised reference model (oracle/ref.py)."""
    p = default_params()
    for k in ("r_mix", "R_mix", "cp_mix", "mue_mix", "r_h2", "r_he", "r_ch4", "cp_h2", "cp_he",
              "cp_ch4", "dt", "L_atm", "u_0", "t_ref", "g", "omega", "re", "pr", "Coriolis",
              "centrifugal", "buoyancy", "chemical_reaction", "R_ref", "p_ref", "sc_ch4",
              "sc_h2o", "sc_h2s", "sc_nh3", "sc_nh4sh", "alpha_sponge", "r_p_nh4sh",
              "rho_cond_nh4sh"):
        setattr(p, k, ref.scalar(k))
    p.turb_active = int(ref.scalar("turb_active"))
    p.nh4sh_sync = int(ref.scalar("nh4sh_eq"))
    for n, g in enumerate(("h2o", "h2s", "nh3", "ch4")):
        G = p.gas[n]
        for fld, key in (("t_0", "t_0_"), ("t_00", "t_00_"), ("ep", "ep_"), ("lv", "lv_"),
                         ("ls", "ls_"), ("C", "C_"), ("L0", "L0_"), ("R", "R_"),
                         ("del_alf", "del_alf_"), ("del_bet", "del_bet_")):
            setattr(G, fld, ref.scalar(key + g))
        if g == "h2s":
            G.C_i, G.L0_i, G.del_alf_i, G.del_bet_i = G.C, G.L0, G.del_alf, G.del_bet
        else:
            G.C_i = ref.scalar(f"C_{g}_ice")
            G.L0_i = ref.scalar(f"L0_{g}_ice")
            G.del_alf_i = ref.scalar(f"del_alf_{g}_ice")
            G.del_bet_i = ref.scalar(f"del_bet_{g}_ice")
    return p


class PostParams(ctypes.Structure):
    """aturan_post_params: the knobs of the passes after RungeKuttaUran (cUranusModel.cpp:1218-1248)."""
    _fields_ = ([(n, ctypes.c_int32) for n in (
        "abi_version", "damp_t_j", "radius_form", "bottom_form", "pole_form", "lid_u", "top_taper",
        "lid_vw", "radius_positive", "phi_periodic", "species_clamp")]
        + [("reserved_i", ctypes.c_int32 * 5)]
        + [(n, ctypes.c_double) for n in ("damp_t_horiz", "damp_t_vert", "vel_shapiro")]
        + [("reserved_d", ctypes.c_double * 5)])

    def copy(self):
        c = PostParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(self))
        return c


def default_post_params(geo_balance=True):
    """The values the reference's ATURAN_* knobs take with the environment unset (ATURAN_GEO_BALANCE
    defaults to 1, cUranusModel.h:1467-1469); geo_balance=False gives those of GEO_BALANCE=0."""
    pp = PostParams()
    pp.abi_version = ABI_VERSION
    pp.damp_t_j = 0 if geo_balance else 1             # cUranusModel.cpp:1216-1217
    pp.radius_form = 0                                # cUranusModel.h:406
    pp.bottom_form = 0                                # cUranusModel.h:409
    pp.pole_form = 0                                  # cUranusModel.h:405
    pp.lid_u = 1                                      # BC_LID_U = BC_RIGID_LID, cUranusModel.h:403
    pp.top_taper = 0                                  # cUranusModel.h:404
    pp.lid_vw = 2 if geo_balance else 0               # BC_Uran.h:155
    pp.radius_positive = 1                            # BC_Uran.h:92
    pp.phi_periodic = 1                               # cUranusModel.h:412
    pp.species_clamp = 1                              # BC_Uran.h:111
    pp.damp_t_horiz = 1.0                             # cUranusModel.cpp:1214-1215
    pp.damp_t_vert = 0.0                              # cUranusModel.cpp:1204-1205
    pp.vel_shapiro = 0.0 if geo_balance else 1.0      # cUranusModel.cpp:1229-1230
    return pp


# aturan_chem_params' doubles in their order, and the reference's values (cUranusModel.h:997-999,
# 1076-1087, 1135-1140; c_mix as ThermalPropertiesUran sums it; ATPhys.h:104's polar floor)
CHEM_SCALARS = ("m_nh3", "m_h2s", "m_nh4sh", "c_mix", "D_nh4sh", "DT_nh4sh", "cp_nh3", "cp_h2s",
                "cp_nh4sh", "k_nh3", "k_h2s", "k_nh4sh", "polar_floor")
CHEM_DEFAULTS = dict(m_nh3=17.03052, m_h2s=34.08088, m_nh4sh=51.1114, c_mix=float.fromhex("0x1.12b14645f7a58p+0"),
                     D_nh4sh=1.45e-9, DT_nh4sh=1.45e-9, cp_nh3=2.19e3, cp_h2s=2.24e3, cp_nh4sh=2.00e3,
                     k_nh3=0.02102, k_h2s=0.013, k_nh4sh=0.02102, polar_floor=0.4)


class ChemParams(ctypes.Structure):
    """aturan_chem_params: the chemistry's constants and knobs (planet/ChemistryUran.h)."""
    _fields_ = ([(n, ctypes.c_int32) for n in (
        "abi_version", "nh4sh_eq", "difflux_plus", "difflux_laplacian", "phi_periodic")]
        + [("reserved_i", ctypes.c_int32 * 3)]
        + [(n, ctypes.c_double) for n in CHEM_SCALARS]
        + [("reserved_d", ctypes.c_double * 5)])


def default_chem_params():
    """The reference's values with its ATURAN_* knobs unset."""
    cp = ChemParams()
    cp.abi_version = ABI_VERSION
    cp.nh4sh_eq = 1                                   # ChemistryUran.h:134-137
    cp.difflux_plus = 1                               # ChemistryUran.h:64-65
    cp.difflux_laplacian = 1                          # ChemistryUran.h:292-293
    cp.phi_periodic = 1                               # cUranusModel.h:412
    for n, v in CHEM_DEFAULTS.items():
        setattr(cp, n, v)
    return cp


def chem_params_from_ref(ref):
    """The chemistry params read from the initialised reference model."""
    cp = default_chem_params()
    for n in CHEM_SCALARS:
        setattr(cp, n, ref.chem_scalar(n))
    cp.nh4sh_eq = int(ref.chem_scalar("nh4sh_eq"))
    cp.phi_periodic = int(ref.chem_scalar("phi_periodic"))
    return cp


class TurbParams(ctypes.Structure):
    """aturan_turb_params: the turbulence closure's knobs (planet/Turbulence.h)."""
    _fields_ = ([(n, ctypes.c_int32) for n in (
        "abi_version", "model", "turb_free", "clamp_pass", "curv", "buoy", "abl_taper", "phi_periodic")]
        + [(n, ctypes.c_double) for n in ("nue_max", "k_bg", "nue_air")]
        + [("reserved_d", ctypes.c_double * 5)])


TURB_K_OMEGA_SST = 2


def default_turb_params():
    """The reference's values with its ATURAN_* knobs unset (Turbulence.h:123-180, the constructor's
    nue_gas, Uranus's turb_default_buoy 0, turb_model k_omega_SST)."""
    tp = TurbParams()
    tp.abi_version = ABI_VERSION
    tp.model = TURB_K_OMEGA_SST
    tp.turb_free = 1
    tp.clamp_pass = 1
    tp.curv = 1
    tp.buoy = 0
    tp.abl_taper = 0
    tp.phi_periodic = 1
    tp.nue_max = 1.0e5
    tp.k_bg = 1.0
    tp.nue_air = 1.8e-5
    return tp


def turb_params_from_ref(ref):
    """The turbulence knobs read from the initialised reference model."""
    tp = default_turb_params()
    for n in ("model", "turb_free", "clamp_pass", "curv", "buoy", "abl_taper", "phi_periodic"):
        setattr(tp, n, int(ref.turb_scalar(n)))
    tp.nue_max = ref.turb_scalar("nue_max")
    tp.k_bg = ref.turb_scalar("k_bg")
    return tp


class PrecipParams(ctypes.Structure):
    """aturan_precip_params: the precipitation's knobs (planet/Precipitation.h)."""
    _fields_ = ([(n, ctypes.c_int32) for n in ("abi_version", "coupling", "h2s")]
                + [("reserved_i", ctypes.c_int32 * 5)]
                + [("rate_scale", ctypes.c_double)]
                + [("reserved_d", ctypes.c_double * 7)])


def default_precip_params():
    """The reference's values with its ATURAN_* knobs unset (Precipitation.h:164-167,
    cUranusModel.h:276-279 and :610)."""
    pp = PrecipParams()
    pp.abi_version = ABI_VERSION
    pp.coupling = 1
    pp.h2s = 1
    pp.rate_scale = 0.00071
    return pp


def precip_params_from_ref(ref):
    """The precipitation knobs read from the initialised reference model."""
    pp = default_precip_params()
    pp.coupling = int(ref.precip_scalar("coupling"))
    pp.h2s = int(ref.precip_scalar("h2s"))
    pp.rate_scale = ref.precip_scalar("rate_scale")
    return pp


class IterParams(ctypes.Structure):
    """aturan_iter_params: one iteration of the model's loop (cUranusModel.cpp:952-1296)."""
    _fields_ = ([(n, ctypes.c_int32) for n in (
        "abi_version", "press_kind", "max_sweeps", "chemistry", "precipitation", "turbulence", "mca_stride")]
        + [("reserved_i", ctypes.c_int32 * 5)]
        + [(n, ctypes.c_double) for n in ("omega", "tol", "damp_p_horiz")]
        + [("reserved_d", ctypes.c_double * 5)]
        + [("post", PostParams), ("chem", ChemParams), ("turb", TurbParams), ("precip", PrecipParams)])


def default_iter_params(geo_balance=True):
    """The reference's loop with its ATURAN_* knobs unset: PressureSolverUran's sweep, the radial
    p_dyn filter only (DAMP_P_HORIZ 0 with GEO_BALANCE, cUranusModel.cpp:979-980), chemistry,
    precipitation, turbulence and the MCA every iteration on."""
    ip = IterParams()
    ip.abi_version = ABI_VERSION
    ip.press_kind = PRESS_GS_LEX
    ip.max_sweeps = 1
    ip.chemistry = 1
    ip.precipitation = 1
    ip.turbulence = 1
    ip.mca_stride = 1
    ip.omega = 1.0
    ip.tol = 0.0
    ip.damp_p_horiz = 0.0 if geo_balance else 1.0
    ip.post = default_post_params(geo_balance)
    ip.chem = default_chem_params()
    ip.turb = default_turb_params()
    ip.precip = default_precip_params()
    return ip
