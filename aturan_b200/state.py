"""Seeded synthetic states of the 41 x 181 x 361 shell (or any grid), FP64, host-side numpy.

The reference publishes no dataset for this path (its NetCDF files are read by no code), so the
inputs are seeded synthetic fields with the reference's shapes, magnitudes and structure:

* `synthetic_state(p, seed)` builds a state from scratch: a dry adiabat from 17.3 bar under an
  isothermal top whose temperature runs parabolically from the poles (t_pole) to the equator
  (t_equator) as InitVariables_Uran.cpp:35-47 does; a hydrostatic p_stat; the retrograde /
  prograde zonal jet template of the benchmark; vapour densities decaying with a seeded scale
  height; seeded cloud and ice in a subset of cells (so that every branch of the saturation
  adjustment runs: melt, freeze, evaporation, Bergeron, condensation, dry exit); smooth seeded
  pressure and projection fields; and the pointwise RHS inputs at the magnitudes the reference's
  initialised model holds.
* `perturb(base, p, seed)` applies the benchmark's perturbation recipe to a given base state
  (for example the reference's own initialised state).

Every field follows the seam convention: k = km-1 is a copy of k = 0.
"""
import math

import numpy as np

from . import fields as F


def coords(p):
    """rad.z and the.z as lib/Array_1D.cpp:50-60 builds them (a running sum)."""
    rad = np.empty(p.im)
    rad[0] = p.r0
    for l in range(1, p.im):
        rad[l] = rad[l - 1] + p.dr
    the = np.empty(p.jm)
    the[0] = p.the0
    for l in range(1, p.jm):
        the[l] = the[l - 1] + p.dthe
    return rad, the


def _seam(a):
    a[..., -1] = a[..., 0]
    return a


def _smooth(rng, shape, amp, modes=4):
    """A smooth seeded field: a few low-order sinusoids in (r, theta, phi)."""
    im, jm, km = shape
    z = np.linspace(0.0, 1.0, im)[:, None, None]
    th = np.linspace(0.0, math.pi, jm)[None, :, None]
    ph = np.linspace(0.0, 2.0 * math.pi, km)[None, None, :]
    out = np.zeros(shape)
    for _ in range(modes):
        a = rng.normal() * amp
        m = rng.integers(1, 5)
        n = rng.integers(0, 4)
        l = rng.integers(0, 3)
        out += a * np.sin(m * th + rng.uniform(0, 6.3)) * np.cos(n * ph + rng.uniform(0, 6.3)) \
            * np.cos(l * math.pi * z + rng.uniform(0, 6.3))
    return out


def jet_template(lat_deg, u_0):
    """Zonal wind [nondimensional]: -A cos(3 lat) with A = 100 m/s for |lat| < 30 deg and 250 m/s
    beyond: -100 m/s at the equator, +250 m/s at +-60 deg, 0 at the poles."""
    A = np.where(np.abs(lat_deg) < 30.0, 100.0, 250.0)
    return -A * np.cos(np.radians(3.0 * lat_deg)) / u_0


F_DEEP = {"ch4": 0.023, "h2s": 1.0e-4, "nh3": 1.0e-5, "h2o": 1.0e-3}
H_SCALE_KM = 50.0


def _species_vapour(rng, p, rho, z_km):
    out = {}
    for g in ("ch4", "h2o", "h2s", "nh3"):
        H = H_SCALE_KM * (1.0 + 0.1 * rng.normal())
        out[g] = F_DEEP[g] * np.exp(-z_km / H)[:, None, None] * rho
    return out


def synthetic_state(p, seed=20261203, condensate=True):
    rng = np.random.default_rng(seed)
    im, jm, km = p.im, p.jm, p.km
    shape = (im, jm, km)
    rad, the = coords(p)
    lat = 90.0 - np.degrees(the)
    z_km = np.arange(im) * (p.L_atm / (im - 1))
    t_pole, t_eq = 49.15, 60.65
    x = np.arange(jm) * (2.0 / (jm - 1))
    T_top = (t_pole - t_eq) * (x * x - 2.0 * x) + t_pole
    T_bot = 194.0
    lapse = p.g / 1.0e4 * 1.0e3                      # K/km for cp ~ 1e4 J/(kg K)
    T = np.maximum(T_bot - lapse * z_km[:, None], T_top[None, :])          # [K], (im, jm)
    R = p.R_ref * 1.0e3
    ps = np.empty((im, jm))
    ps[0] = 17.3
    for i in range(1, im):
        Tm = 0.5 * (T[i] + T[i - 1])
        ps[i] = ps[i - 1] * np.exp(-p.g * (z_km[i] - z_km[i - 1]) * 1.0e3 / (R * Tm))
    T3 = np.repeat(T[:, :, None], km, axis=2) * (1.0 + 1.0e-3 * rng.normal(size=shape))
    ps3 = np.repeat(ps[:, :, None], km, axis=2)
    rho = ps3 * 1.0e5 / (p.R_mix * T3)

    s = {}
    s["t"] = T3 / p.t_ref
    s["p_stat"] = ps3
    s["rho_mix"] = rho.copy()
    w = np.repeat(jet_template(lat, p.u_0)[None, :, None], im, axis=0)
    s["w"] = np.broadcast_to(w, shape) + rng.normal(0.0, 0.1, shape) / p.u_0
    s["u"] = rng.normal(0.0, 0.1, shape) / p.u_0 * 1.0e-2
    s["v"] = rng.normal(0.0, 0.1, shape) / p.u_0
    vap = _species_vapour(rng, p, rho, z_km)
    for g in ("ch4", "h2o", "h2s", "nh3"):
        c = vap[g] * (1.0 + 0.05 * rng.normal(size=shape))
        cloud = np.zeros(shape)
        ice = np.zeros(shape)
        if condensate:
            sel_c = rng.random(shape) < 0.2
            sel_i = rng.random(shape) < 0.2
            cloud[sel_c] = c[sel_c] * rng.uniform(0.0, 0.5, sel_c.sum())
            ice[sel_i] = c[sel_i] * rng.uniform(0.0, 0.5, sel_i.sum())
            neg = rng.random(shape) < 0.005
            cloud[neg] = -1.0e-12
            # a band of supersaturation: vapour raised 30x in some columns
            band = (rng.random((1, jm, km)) < 0.1) & (np.arange(im)[:, None, None] > 5)
            c = np.where(band, c * 30.0, c)
        s[g] = c
        s[g + "_cloud"] = cloud
        s[g + "_ice"] = ice
    s["nh4sh"] = np.abs(1.0e-8 * (1.0 + rng.normal(size=shape))) * rho
    s["tke"] = 1.0e-4 * (1.0 + 0.1 * rng.random(shape))
    s["dis"] = 2.3282 * (1.0 + 0.1 * rng.random(shape))

    s["p_dyn"] = 16.0 + _smooth(rng, shape, 5.0) + 0.01 * rng.normal(size=shape)
    s["p_hydro"] = _smooth(rng, shape, 1.0)
    s["p_baro"] = _smooth(rng, shape, 2.0)
    s["p_b0"] = _smooth(rng, shape, 0.5)
    s["p_bfollow"] = _smooth(rng, shape, 0.01)

    s["nue"] = 4.19e-5 * (1.0 + 0.05 * rng.normal(size=shape))
    s["thermalmassflux"] = 0.05 + 0.05 * rng.normal(size=shape)
    s["Q_precip"] = 0.05 * rng.random(shape)
    for nm in F.FORCING:
        if nm.startswith("S_precip"):
            s[nm] = 1.0e-6 * rng.normal(size=shape)
    for nm in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh"):
        s[nm] = 1.0e-7 * rng.normal(size=shape)
    s["fluxlim_nh4sh"] = 1.0e-14 * rng.normal(size=shape)
    s["tke_source"] = 2.0e-5 * rng.normal(size=shape)
    s["dis_source"] = -0.17 + 0.05 * rng.normal(size=shape)

    for nm in ("rhs_u", "rhs_v", "rhs_w"):
        s[nm] = _smooth(rng, shape, 1.0e-2) + 1.0e-3 * rng.normal(size=shape)
    for nm, r in (("aux_u", "rhs_u"), ("aux_v", "rhs_v"), ("aux_w", "rhs_w")):
        s[nm] = s[r] + _smooth(rng, shape, 1.0e-2)

    for q in F.PROGNOSTIC:
        s[q + "n"] = s[q].copy()
    for q in ("un", "vn", "wn"):
        s[q] = s[q] * (1.0 + 1.0e-6 * rng.normal(size=shape))
    # drawn last, so that every field above keeps the values it had before these were held
    for nm in F.CHEM_STATE:
        s[nm] = 1.0e-9 * rng.normal(size=shape)
    s["prod"] = np.abs(1.0e-4 * rng.normal(size=shape))

    out = {}
    for n in F.NAMES:
        a = np.ascontiguousarray(np.array(s[n], dtype=np.float64))
        out[n] = _seam(a)
    return out


def perturb(base, p, seed=20261203, forcing_noise=True):
    """The benchmark's perturbation of a base state (interior cells; k = km-1 follows k = 0):
    T x (1 + 1e-3 N); zonal wind = jet template + N(0, 0.1 m/s); u, v = N(0, 0.1 m/s); vapour
    densities f_deep exp(-z / H) rho_local with a seeded H around 50 km, cloud and ice zero.
    forcing_noise adds seeded values to the pointwise RHS inputs the reference's initial state
    holds at zero (precipitation, chemistry sources), so every term of the RHS is exercised."""
    rng = np.random.default_rng(seed)
    s = {n: np.array(a, dtype=np.float64, copy=True) for n, a in base.items()}
    im, jm, km = p.im, p.jm, p.km
    shape = (im, jm, km)
    rad, the = coords(p)
    lat = 90.0 - np.degrees(the)
    z_km = np.arange(im) * (p.L_atm / (im - 1))
    I = (slice(1, im - 1), slice(1, jm - 1), slice(0, km - 1))
    s["t"][I] = s["t"][I] * (1.0 + 1.0e-3 * rng.normal(size=s["t"][I].shape))
    w = jet_template(lat, p.u_0)[None, :, None] + rng.normal(0.0, 0.1, shape) / p.u_0
    s["w"][I] = w[I]
    s["u"][I] = (rng.normal(0.0, 0.1, shape) / p.u_0)[I]
    s["v"][I] = (rng.normal(0.0, 0.1, shape) / p.u_0)[I]
    rho = s["p_stat"] * 1.0e5 / (p.R_mix * s["t"] * p.t_ref)
    vap = _species_vapour(rng, p, rho, z_km)
    for g in ("ch4", "h2o", "h2s", "nh3"):
        s[g][I] = vap[g][I]
        s[g + "_cloud"][I] = 0.0
        s[g + "_ice"][I] = 0.0
    if forcing_noise:
        s["Q_precip"] = 0.05 * rng.random(shape)
        for nm in F.FORCING:
            if nm.startswith("S_precip"):
                s[nm] = 1.0e-6 * rng.normal(size=shape)
        for nm in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh"):
            s[nm] = 1.0e-7 * rng.normal(size=shape)
        for nm in ("rhs_u", "rhs_v", "rhs_w"):
            s[nm] = _smooth(rng, shape, 1.0e-2) + 1.0e-3 * rng.normal(size=shape)
        for nm, r in (("aux_u", "rhs_u"), ("aux_v", "rhs_v"), ("aux_w", "rhs_w")):
            s[nm] = s[r] + _smooth(rng, shape, 1.0e-2)
    for q in F.PROGNOSTIC:
        s[q + "n"] = s[q].copy()
    for n in s:
        if s[n].ndim == 3:
            _seam(s[n])
    return s


def copy_state(s):
    return {n: a.copy() for n, a in s.items()}


# ---- the isolated Poisson solve's input: a smoothed random velocity field and its divergence ----

def _box3(a):
    """One pass of the 3x3x3 box filter over (r, theta, phi) on the km-1 distinct meridians:
    periodic in phi, the end rows repeated in r and theta (a clamped stencil). Separable: the
    mean of three neighbours along each axis in turn."""
    a = (np.roll(a, 1, axis=2) + a + np.roll(a, -1, axis=2)) / 3.0
    for ax in (0, 1):
        n = a.shape[ax]
        lo = np.take(a, np.r_[0, 0:n - 1], axis=ax)
        hi = np.take(a, np.r_[1:n, n - 1], axis=ax)
        a = (lo + a + hi) / 3.0
    return a


def poisson_velocity(p, seed=20261205, passes=3):
    """(u, v, w): iid N(0, 1) values on every cell of the shell (km-1 distinct meridians, k = km-1
    the seam copy of k = 0), smoothed by `passes` passes of the 3x3x3 box filter."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(3):
        a = rng.standard_normal((p.im, p.jm, p.km - 1))
        for _ in range(passes):
            a = _box3(a)
        out.append(_seam(np.ascontiguousarray(np.concatenate([a, a[:, :, :1]], axis=2))))
    return tuple(out)


def poisson_source(p, u, v, w):
    """The shared solver's pressure source for aux = (u, v, w), FP64 on the host: the boundary rows
    that prepareProjectionBoundaries sets (Pressure_Uran.cpp:30-146: the lid's aux_u = 0, or the
    cubic extrapolation without the rigid lid; cubic radial ends of v, w; cubic polar rows of u
    with v = w = 0 there; the seam copy), then the centred divergence
    du/dr + dv/dtheta / rm + dw/dphi / (rm sin theta) (PressureSolver.h:448-459, no obstacle) and
    its clamp at den * p_dyn_cap with the non-finite guard (:481-487) on the interior. Returns the
    source on [im][jm][km], zero outside the interior. Same operations in the same order as the
    C code, so the values are the same bits as the oracle's."""
    import math
    im, jm, km = p.im, p.jm, p.km
    au, av, aw = (np.array(x, dtype=np.float64, copy=True) for x in (u, v, w))
    J, K = slice(1, jm - 1), slice(0, km - 1)

    def cub0(X):
        return X[3, J, K] - 3.0 * X[2, J, K] + 3.0 * X[1, J, K]

    def cub1(X):
        return X[im - 4, J, K] - 3.0 * X[im - 3, J, K] + 3.0 * X[im - 2, J, K]
    if p.rigid_lid:
        au[0, J, K] = 0.0
        au[im - 1, J, K] = 0.0
    else:
        au[0, J, K], au[im - 1, J, K] = cub0(au), cub1(au)
    for X in (av, aw):
        X[0, J, K], X[im - 1, J, K] = cub0(X), cub1(X)
    Ii = slice(1, im - 1)
    au[Ii, 0, K] = au[Ii, 3, K] - 3.0 * au[Ii, 2, K] + 3.0 * au[Ii, 1, K]
    au[Ii, jm - 1, K] = au[Ii, jm - 4, K] - 3.0 * au[Ii, jm - 3, K] + 3.0 * au[Ii, jm - 2, K]
    for X in (av, aw):
        X[Ii, 0, K] = 0.0
        X[Ii, jm - 1, K] = 0.0
    for X in (au, av, aw):
        _seam(X)
    rad, the = coords(p)
    st = np.array([max(math.sin(t), p.sinthe_min) for t in the])
    st[st == 0.0] = 1.0e-5
    R_km = p.metric_R_km
    rm = rad + (R_km / p.L_atm - 1.0) if R_km > 0.0 else rad.copy()
    inv_dr2, inv_dthe2, inv_dphi2 = 1.0 / (p.dr * p.dr), 1.0 / (p.dthe * p.dthe), 1.0 / (p.dphi * p.dphi)
    inv_2dr, inv_2dthe, inv_2dphi = 1.0 / (2.0 * p.dr), 1.0 / (2.0 * p.dthe), 1.0 / (2.0 * p.dphi)
    rm2 = (rm * rm)[:, None]
    inv_rm2 = 1.0 / rm2
    inv_rm2sinthe2 = inv_rm2 / (st * st)[None, :]
    num1 = 1.0 * inv_dr2
    num2 = inv_rm2 * inv_dthe2
    num3 = inv_rm2sinthe2 * inv_dphi2
    den = 2.0 * num1 + 2.0 * num2 + 2.0 * num3                       # (im, jm)
    inv_rm = (1.0 / rm)[:, None]
    inv_rmsinthe = 1.0 / (rm[:, None] * st[None, :])
    k = np.arange(km - 1)
    ke = np.where(k + 1 >= km - 1, k + 1 - (km - 1), k + 1)
    kw = np.where(k - 1 < 0, k - 1 + (km - 1), k - 1)
    Jj = slice(1, jm - 1)
    du = (au[2:, Jj, :km - 1] - au[:-2, Jj, :km - 1]) * inv_2dr
    dv = (av[Ii, 2:, :km - 1] - av[Ii, :-2, :km - 1]) * inv_2dthe
    dw = (aw[Ii, Jj][:, :, ke] - aw[Ii, Jj][:, :, kw]) * inv_2dphi
    with np.errstate(invalid="ignore", over="ignore"):
        div = du * 1.0 + dv * inv_rm[Ii, :, None] + dw * inv_rmsinthe[Ii, Jj, None]
    smax = (den[Ii, Jj] * p.p_dyn_cap)[:, :, None]
    div = np.where(np.isfinite(div), div, 0.0)
    div = np.where(div > smax, smax, np.where(div < -smax, -smax, div))
    src = np.zeros((im, jm, km))
    src[Ii, Jj, :km - 1] = div
    return src
