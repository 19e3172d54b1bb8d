"""Test infrastructure: a torch FP64 restatement of the dry part of one RK4 step (t, u, v, w), used
as the reference for the hand-written adjoint through torch.autograd. Only tests import it.

It follows the same reference code as oracle/aturan_oracle.c, restricted to the fields that the
temperature and the velocities depend on:
  * planet/RungeKutta_Uran_Turb.cpp:18-37   buoyancy reference level (sin-theta weighted mean),
  * planet/RungeKutta_Uran_Turb.cpp:62-177  hydrostatic column integral with PBARO_FOLLOW,
  * planet/RHS_Uran_Turb.cpp:92-788         rhs of t, u, v, w (transport, diffusion, Coriolis,
                                            centrifugal, pressure work with cp(T), sponge,
                                            hydrostatic-split gradients),
  * planet/RungeKutta_Uran_Turb.cpp:242-403 the four stages and the clamped final update.
Its forward is checked against the C restatement (which is bit-identical to the compiled
reference) in tests/test_dry_ref.py; its arithmetic order is not the reference's, so it agrees to
rounding, not bit for bit. Inputs t, u, v, w are the state AND its start-of-step copies (the step
runs right after the n-copy sync).
"""
import numpy as np
import torch

from aturan_b200.state import coords

CP_T_LO, CP_T_HI, CP_DT = 5.0, 1500.0, 0.5


def _metric_radius(p, r):
    return r + (p.metric_R_km / p.L_atm - 1.0) if p.metric_R_km > 0.0 else r


def _coriolis_scale(p):
    return (p.L_atm * 1.0e3 if p.coriolis_full else p.L_atm) / p.u_0


class DryStep:
    """dry = DryStep(p, fixed, oracle); t1, u1, v1, w1 = dry(t, u, v, w) on torch FP64 tensors of
    shape (im, jm, km). `fixed` holds p_dyn, p_stat, p_baro, p_b0, p_bfollow, nue and, when present,
    thermalmassflux and Q_precip (numpy)."""

    def __init__(self, p, fixed, oracle):
        self.p = p
        im, jm, km = p.im, p.jm, p.km
        T = lambda a: torch.tensor(np.array(a, dtype=np.float64))
        self.pdyn, self.pstat = T(fixed["p_dyn"]), T(fixed["p_stat"])
        self.pbaro, self.pb0, self.pbf = T(fixed["p_baro"]), T(fixed["p_b0"]), T(fixed["p_bfollow"])
        self.nue = T(fixed["nue"])
        # the frozen pointwise inputs of rhs_t (RHS_Uran_Turb.cpp:503-557)
        zero = np.zeros((im, jm, km))
        self.tmf_f = T(fixed.get("thermalmassflux", zero))
        self.qp_f = T(fixed.get("Q_precip", zero))
        rad, the = coords(p)
        self.rm_i = T(np.array([_metric_radius(p, r) for r in rad]))
        self.wsin = T(np.sin(the))
        self.cor_j = T(p.Coriolis * _coriolis_scale(p) * 2.0 * p.omega * np.abs(np.sin(the)))
        # cp(T): the affine gas combination of a 0.5 K linear table commutes with the interpolation,
        # so the table of cp_lapse at the nodes interpolates to the same function
        n = int((CP_T_HI - CP_T_LO) / CP_DT) + 1
        self.cp_nodes = T(np.array([oracle.cp_lapse(p, CP_T_LO + i * CP_DT) for i in range(n)]))
        # per-(i,j) geometry of the interior (RungeKutta_Uran_Turb.cpp:258-283)
        ii, jj = np.arange(1, im - 1), np.arange(1, jm - 1)
        rm = np.array([_metric_radius(p, rad[i]) for i in ii])[:, None, None]
        s = np.abs(np.sin(the[jj]))[None, :, None]
        sinthe = np.maximum(p.sinthe_min, s)
        costhe = np.cos(the[jj])[None, :, None]
        g = {}
        g["inv_rm"] = 1.0 / rm
        g["inv_rm2"] = 1.0 / (rm * rm)
        g["inv_rmsinthe"] = 1.0 / (rm * sinthe)
        g["inv_rm2sinthe"] = g["inv_rm2"] / sinthe
        g["inv_rm2sinthe2"] = g["inv_rm2"] / (sinthe * sinthe)
        g["costhe_inv_rm2sinthe"] = costhe * g["inv_rm2sinthe"]
        g["costhe"] = costhe + 0 * rm
        g["cotanthe"] = (costhe / sinthe) + 0 * rm
        g["v_metric"] = (1.0 + costhe / (sinthe * sinthe)) * g["inv_rm2"]
        sinthe_bf = np.sqrt(np.maximum(0.0, 1.0 - costhe * costhe))
        g["sinthe_bf"] = sinthe_bf + 0 * rm
        scale_cen = p.L_atm * p.L_atm / (p.u_0 * p.u_0)
        cenf = 1.0 * p.centrifugal * p.cent_mom * scale_cen
        g["cent_rad"] = cenf * p.omega * p.omega * rm * sinthe_bf * sinthe_bf
        g["cent_the"] = cenf * p.omega * p.omega * rm * sinthe_bf * costhe
        frac = (ii - (im - 1) * 3 // 4) / ((im - 1) // 4)
        frac = np.maximum(frac, 0.0)[:, None, None]
        g["sponge"] = p.alpha_sponge * frac * frac + 0 * s
        self.geo = {k: T(np.broadcast_to(v, (im - 2, jm - 2, 1))) for k, v in g.items()}
        N = km - 1
        self.ke = torch.tensor([(k + 1) % N for k in range(N)])
        self.kw = torch.tensor([(k - 1) % N for k in range(N)])

    # ---- cp(T) (CpH2.h:77-84, 122-134) ----
    def cp_lapse(self, TK):
        Tc = TK.clamp(CP_T_LO, CP_T_HI)
        x = (Tc - CP_T_LO) / CP_DT
        i = torch.clamp(x.detach().floor().long(), max=self.cp_nodes.numel() - 2)
        f = x - i.to(x.dtype)
        a, b = self.cp_nodes[i], self.cp_nodes[i + 1]
        return a + f * (b - a)

    def _stencil(self, F):
        c = F[1:-1, 1:-1, :-1]
        N = self.p.km - 1
        rp, rm = F[2:, 1:-1, :N], F[:-2, 1:-1, :N]
        tp, tm = F[1:-1, 2:, :N], F[1:-1, :-2, :N]
        pe, pw = F[1:-1, 1:-1, :N][:, :, self.ke], F[1:-1, 1:-1, :N][:, :, self.kw]
        p = self.p
        i2dr, i2dt, i2dp = 1.0 / (2.0 * p.dr), 1.0 / (2.0 * p.dthe), 1.0 / (2.0 * p.dphi)
        idr2, idt2, idp2 = 1.0 / (p.dr * p.dr), 1.0 / (p.dthe * p.dthe), 1.0 / (p.dphi * p.dphi)
        return dict(c=c, d1r=(rp - rm) * i2dr, d2r=(rp - 2.0 * c + rm) * idr2,
                    d1t=(tp - tm) * i2dt, d2t=(tp - 2.0 * c + tm) * idt2,
                    d1p=(pe - pw) * i2dp, d2p=(pe - 2.0 * c + pw) * idp2)

    def hydro(self, T, V, W):
        p = self.p
        rR = p.r_mix * p.R_mix
        valid = T > 0.0
        Ts = torch.where(valid, T, torch.ones_like(T))
        b = torch.where(valid, p.g * self.pstat / (rR * Ts * p.t_ref), torch.zeros_like(T))
        w = self.wsin[None, :, None] * valid.to(T.dtype)
        ref = (w * b).sum(dim=(1, 2)) / w.sum(dim=(1, 2))
        nd_rel = p.g * (p.L_atm * 1.0e3) / (p.u_0 * p.u_0)
        fb = torch.where(valid, -nd_rel * p.buoyancy * (b - ref[:, None, None]) / ref[:, None, None],
                         torch.zeros_like(T))
        met = (V * V + W * W) / self.rm_i[:, None, None] + self.cor_j[None, :, None] * W

        def cumtrapz(F):
            inc = 0.5 * (F[:-1] + F[1:]) * p.dr
            return torch.cat([torch.zeros_like(F[:1]), torch.cumsum(inc, dim=0)], dim=0)

        if p.pbaro_follow > 0.0:
            Pm, Pb = cumtrapz(met), cumtrapz(fb)
            pbf = self.pbf + (Pb - self.pb0 - self.pbf) / p.pbaro_follow
            return Pm + Pb + self.pbaro - pbf, ref
        return cumtrapz(fb + met) + self.pbaro, ref

    def rhs(self, X, ph):
        """rhs of t, u, v, w on the interior (im-2, jm-2, km-1) from the full stage inputs."""
        p, g = self.p, self.geo
        T, U, V, W = X
        sT, sU, sV, sW = self._stencil(T), self._stencil(U), self._stencil(V), self._stencil(W)
        u, v, w = sU["c"], sV["c"], sW["c"]
        N = p.km - 1
        P = self.pdyn
        dpdr = (P[2:, 1:-1, :N] - P[:-2, 1:-1, :N]) / (2.0 * p.dr)
        dpdthe = (P[1:-1, 2:, :N] - P[1:-1, :-2, :N]) / (2.0 * p.dthe)
        Pc = P[1:-1, 1:-1, :N]
        dpdphi = (Pc[:, :, self.ke] - Pc[:, :, self.kw]) / (2.0 * p.dphi)
        PHc = ph[1:-1, 1:-1, :N]
        dphdthe = (ph[1:-1, 2:, :N] - ph[1:-1, :-2, :N]) / (2.0 * p.dthe) * g["inv_rm"]
        dphdphi = (PHc[:, :, self.ke] - PHc[:, :, self.kw]) / (2.0 * p.dphi) * g["inv_rmsinthe"]

        two_omega = 2.0 * p.omega
        cor_rad = -two_omega * g["sinthe_bf"] * w
        cor_the = -two_omega * g["costhe"] * w
        cor_phi = two_omega * (g["costhe"] * v + g["sinthe_bf"] * u)
        scale_p = 1.0e5 / (p.r_mix * p.u_0 * p.u_0)
        ce = p.u_0 * p.u_0 / (p.cp_mix * p.t_ref)
        scale_cor = _coriolis_scale(p)
        v_invrm, w_invrs = v * g["inv_rm"], w * g["inv_rmsinthe"]

        pressure_t = ce * scale_p * (u * dpdr + v_invrm * dpdthe + w_invrs * dpdphi)
        tc = sT["c"]
        if p.cp_dyn:
            pos = tc > 0.0
            cpv = self.cp_lapse(torch.where(pos, tc, torch.ones_like(tc)) * p.t_ref)
            pressure_t = torch.where(pos, pressure_t * (p.cp_mix / cpv), pressure_t)

        def transport(s):
            return u * s["d1r"] + v_invrm * s["d1t"] + w_invrs * s["d1p"]

        tr_t = transport(sT)
        tr_u = transport(sU)
        tr_v = transport(sV) + (u * v - w * w * g["cotanthe"]) * g["inv_rm"]
        tr_w = transport(sW) + (w * u + v * w * g["cotanthe"]) * g["inv_rm"]
        two_inv_rm = 2.0 * g["inv_rm"]

        def diff_scalar(s):
            return (s["d2r"] + s["d1r"] * two_inv_rm + s["d2t"] * g["inv_rm2"]
                    + s["d1t"] * g["costhe_inv_rm2sinthe"] + s["d2p"] * g["inv_rm2sinthe2"])

        dif_t = diff_scalar(sT)
        dif_u = (sU["d2r"] + 2.0 * u * g["inv_rm2"] + sU["d2t"] * g["inv_rm2"] + 4.0 * sU["d1r"] * g["inv_rm"]
                 + sU["d1t"] * g["costhe_inv_rm2sinthe"] + sU["d2p"] * g["inv_rm2sinthe2"])
        dif_v = (diff_scalar(sV) - g["v_metric"] * v + 2.0 * sU["d1t"] * g["inv_rm2"]
                 - sW["d1p"] * 2.0 * g["costhe"] * g["inv_rm2sinthe2"])
        dif_w = (diff_scalar(sW) - g["v_metric"] * w + 2.0 * sU["d1p"] * g["inv_rm2sinthe"]
                 + sV["d1p"] * 2.0 * g["costhe"] * g["inv_rm2sinthe2"])

        nue = self.nue[1:-1, 1:-1, :N]
        if p.turb_coupling != 0.0:
            nue_t = torch.where(torch.isfinite(nue), p.turb_coupling * nue.clamp(min=0.0), torch.zeros_like(nue))
        else:
            nue_t = torch.zeros_like(nue)
        nue_t_s = nue_t / 0.9
        re_eff = p.re
        tmf = (p.tmf_scale * p.chemical_reaction * self.tmf_f[1:-1, 1:-1, :N] if p.tmf_scale != 0.0
               else torch.zeros_like(nue))
        precip_t = torch.zeros_like(nue)
        if p.precip_coupling != 0.0 and p.r_mix > 0.0 and p.cp_mix > 0.0:
            precip_t = (p.precip_coupling * self.qp_f[1:-1, 1:-1, :N] * (p.L_atm * 1.0e3)
                        / (p.r_mix * p.cp_mix * p.u_0 * p.t_ref))
            precip_t = torch.where(torch.isfinite(precip_t), precip_t.clamp(-0.5, 0.5), torch.zeros_like(nue))
        r_t = pressure_t - tr_t + dif_t / (p.re * p.pr) + dif_t * nue_t_s - tmf + precip_t
        r_u = (-dpdr * scale_p - tr_u + dif_u / re_eff + dif_u * nue_t
               - 0.0 * p.Coriolis * scale_cor * cor_rad + g["cent_rad"] - g["sponge"] * u)
        r_v = (-dpdthe * scale_p * g["inv_rm"] - dphdthe - tr_v + dif_v / re_eff + dif_v * nue_t
               - p.Coriolis * scale_cor * cor_the + g["cent_the"])
        r_w = (-dpdphi * scale_p * g["inv_rmsinthe"] - dphdphi - tr_w + dif_w / re_eff + dif_w * nue_t
               - p.Coriolis * scale_cor * cor_phi)
        return [r_t, r_u, r_v, r_w]

    def __call__(self, t, u, v, w):
        p = self.p
        N = p.km - 1
        Y = [t, u, v, w]
        ph, _ = self.hydro(t, v, w)
        dt = p.dt
        X = Y
        acc = None
        for stage in range(4):
            c_in = 0.5 * dt if stage in (0, 1) else (dt if stage == 2 else 0.0)
            wgt = 1.0 if stage in (0, 3) else 2.0
            k = self.rhs(X, ph)
            acc = [wgt * r for r in k] if acc is None else [a + wgt * r for a, r in zip(acc, k)]
            if stage < 3:
                X = []
                for q in range(4):
                    full = Y[q].clone()
                    full[1:-1, 1:-1, :N] = Y[q][1:-1, 1:-1, :N] + c_in * k[q]
                    X.append(full)
        out = []
        tmin, tmax = p.t_min_K / p.t_ref, p.t_max_K / p.t_ref
        for q in range(4):
            full = Y[q].clone()
            y = Y[q][1:-1, 1:-1, :N] + dt * acc[q] / 6.0
            if q == 0:
                y = y.clamp(tmin, tmax)
            full[1:-1, 1:-1, :N] = y
            out.append(full)
        return out


SPECIES = ("ch4", "ch4_cloud", "ch4_ice", "h2o", "h2o_cloud", "h2o_ice",
           "h2s", "h2s_cloud", "h2s_ice", "nh3", "nh3_cloud", "nh3_ice")


class MoistRK4Step(DryStep):
    """The same RK4 step over t, u, v, w and the twelve condensable species
    (planet/RHS_Uran_Turb.cpp:790-850): each species is carried by u, v, w and diffused with
    1/(Sc Re) + nue_t/0.9, plus its frozen forcing (the precipitation source S_precip_<species>
    times the precipitation coupling; H2S and NH3 vapour also the mass flux times the chemical
    reaction switch). `fixed` additionally holds S_precip_* and massflux_h2s / massflux_nh3."""

    def __init__(self, p, fixed, oracle):
        super().__init__(p, fixed, oracle)
        T = lambda a: torch.tensor(np.array(a, dtype=np.float64))
        N = p.km - 1
        zero = np.zeros((p.im, p.jm, p.km))
        self.sp_forc = []
        for n in SPECIES:
            f = p.precip_coupling * T(fixed.get("S_precip_" + n, zero))[1:-1, 1:-1, :N]
            if n in ("h2s", "nh3"):
                f = f + p.chemical_reaction * T(fixed.get("massflux_" + n, zero))[1:-1, 1:-1, :N]
            self.sp_forc.append(f)
        sc = {"ch4": p.sc_ch4, "h2o": p.sc_h2o, "h2s": p.sc_h2s, "nh3": p.sc_nh3}
        self.sp_sc_re = [sc[n.split("_")[0]] * p.re for n in SPECIES]

    def rhs(self, X, ph):
        r = super().rhs(X[:4], ph)
        p, g = self.p, self.geo
        N = p.km - 1
        U, V, W = X[1], X[2], X[3]
        u, v, w = U[1:-1, 1:-1, :N], V[1:-1, 1:-1, :N], W[1:-1, 1:-1, :N]
        v_invrm, w_invrs = v * g["inv_rm"], w * g["inv_rmsinthe"]
        nue = self.nue[1:-1, 1:-1, :N]
        if p.turb_coupling != 0.0:
            nue_t = torch.where(torch.isfinite(nue), p.turb_coupling * nue.clamp(min=0.0), torch.zeros_like(nue))
        else:
            nue_t = torch.zeros_like(nue)
        nue_t_s = nue_t / 0.9
        two_inv_rm = 2.0 * g["inv_rm"]
        for q in range(len(SPECIES)):
            s = self._stencil(X[4 + q])
            transport = u * s["d1r"] + v_invrm * s["d1t"] + w_invrs * s["d1p"]
            diffusion = (s["d2r"] + s["d1r"] * two_inv_rm + s["d2t"] * g["inv_rm2"]
                         + s["d1t"] * g["costhe_inv_rm2sinthe"] + s["d2p"] * g["inv_rm2sinthe2"])
            r.append(-transport + diffusion / self.sp_sc_re[q] + diffusion * nue_t_s + self.sp_forc[q])
        return r

    def __call__(self, *Y):
        p = self.p
        N = p.km - 1
        Y = list(Y)
        nf = len(Y)
        ph, _ = self.hydro(Y[0], Y[2], Y[3])
        dt = p.dt
        X = Y
        acc = None
        for stage in range(4):
            c_in = 0.5 * dt if stage in (0, 1) else (dt if stage == 2 else 0.0)
            wgt = 1.0 if stage in (0, 3) else 2.0
            k = self.rhs(X, ph)
            acc = [wgt * r for r in k] if acc is None else [a + wgt * r for a, r in zip(acc, k)]
            if stage < 3:
                X = []
                for q in range(nf):
                    full = Y[q].clone()
                    full[1:-1, 1:-1, :N] = Y[q][1:-1, 1:-1, :N] + c_in * k[q]
                    X.append(full)
        out = []
        tmin, tmax = p.t_min_K / p.t_ref, p.t_max_K / p.t_ref
        for q in range(nf):
            full = Y[q].clone()
            y = Y[q][1:-1, 1:-1, :N] + dt * acc[q] / 6.0
            if q == 0:
                y = y.clamp(tmin, tmax)
            full[1:-1, 1:-1, :N] = y
            out.append(full)
        return out
