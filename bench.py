"""Throughput of the ATURAN dynamical-core step on B200: cell-steps/s at 41 x 181 x 361.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--press gs|rb|sor]

A step is one pass of the hot path over the synthetic seeded state: the pressure solve, the four
saturation adjustments (H2O, H2S, NH3, CH4), the n-copy sync and the RK4 step -- the in-scope
calls of one even iteration of cUranusModel::Run (planet/cUranusModel.cpp:967-1123). The
headline workload is the mixed-precision full step (FP32 state and stencils, FP64 pressure and
saturation-adjustment Newton iteration); --precision fp64 runs the plain FP64 path.

One process per GPU (torchrun for N > 1). The path has no exchange step at this grid size, so
ranks run independent replicas (weak scaling); NCCL carries only the barrier and the max of the
per-rank times. Rank 0 prints one JSON line.

--impl reference times the reference's own CPU implementation (the compiled unmodified sources
in oracle/_ref, all host threads; the C restatement in oracle/ when that was not built) on the
same workload; under torchrun only rank 0 runs it.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 41 * 181 * 361          # the metric's N: stored cells of the shell
METRIC = "cell-steps/s at 41x181x361"

# Algorithmic words per stored cell of one RK4 stage launch (fused RHS + stage update: stage
# input, start-of-step copies, accumulator, pressure pair, pointwise inputs; writes acc and the
# next stage input) and of the step's other kernels.
STAGE_WORDS = (81, 119, 119, 106)
STEP_OTHER_WORDS = {"hydro": 11, "satadj": 28, "gs_per_sweep": 3, "gs_source": 5}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons polled through NVML back to back (a 2 ms sleep between polls)
    while the timed region runs; each poll takes three NVML queries, so a region of a few tens of
    milliseconds sees only a few samples (`samples` in the result says how many). Falls back to
    nvidia-smi (100 ms period) when NVML is not importable. Reads only."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.sm, self.mx, self.reasons = [], [], set()
        self.proc = None
        self.nv = None
        self.run = False
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            try:
                import torch
                pr = torch.cuda.get_device_properties(index)
                bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
                h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv, self.h = nv, h
            self.bits = [(n, getattr(nv, attr, val)) for n, attr, val in self.REASONS]
        except Exception:
            self.nv = None

    def _poll(self):
        nv = self.nv
        while self.run:
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                self.mx.append(float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h) if hasattr(
                    nv, "nvmlDeviceGetCurrentClocksEventReasons") else nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for n, bit in self.bits:
                    if r & bit:
                        self.reasons.add(n)
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        if self.nv is not None:
            # the launching thread holds the GIL between its API calls; a short switch interval
            # lets the poller in every ~2 ms instead of every 5 ms or less often
            self.si = sys.getswitchinterval()
            sys.setswitchinterval(1e-4)
            self.run = True
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        try:
            self.rows = []
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.nv is not None:
            self.run = False
            self.t.join(timeout=2)
            sys.setswitchinterval(self.si)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                    "sm_max_mhz": max(self.mx) if self.mx else None,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = [n for n, _, _ in self.REASONS]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def adjoint_timing(api, P, S, torch, reps=5):
    """Device time of one taped FP64 RK4 step and of its hand-written adjoint on the full grid
    (41x181x361), CUDA events on the context's stream, after two warm-up pairs."""
    p = P.default_params(precision=P.FP64)
    ctx = api.Context(p)
    ctx.upload_state(S.synthetic_state(p, seed=20261206))
    ctx.tape(True)
    stream = torch.cuda.ExternalStream(ctx.stream)
    g = torch.Generator(device="cuda").manual_seed(5)
    ybar = [torch.randn(p.shape, dtype=torch.float64, device="cuda", generator=g) for _ in range(4)]
    xbar = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    yp, xp = [t.data_ptr() for t in ybar], [t.data_ptr() for t in xbar]
    for _ in range(2):
        ctx.rk4_step()
        ctx.rk4_adjoint(yp, xp)
    ctx.synchronize()
    fwd = adj = 0.0
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        ctx.rk4_step()
        e[1].record(stream)
        ctx.rk4_adjoint(yp, xp)
        e[2].record(stream)
        e[2].synchronize()
        fwd += e[0].elapsed_time(e[1])
        adj += e[1].elapsed_time(e[2])
    out = {"fwd_ms": fwd / reps, "adj_ms": adj / reps, "adj_over_fwd": adj / fwd, "precision": "fp64",
           "grid": [p.im, p.jm, p.km],
           "what": "forward = aturan_rk4_step with the tape on (level means, hydrostatic integral, 4 stages, "
                   "tape copies); adjoint = aturan_rk4_adjoint (4 reverse stages, hydrostatic and level-mean "
                   "adjoints, layout copies in and out)"}
    # the full steps the multi-step gradients chain (aturan_b200.autograd): the pressure solve to a
    # residual and its transposed solve included, dry and moist
    press = dict(kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=200, tol=1e-8)
    abar_in = [torch.randn(p.shape, dtype=torch.float64, device="cuda", generator=g) for _ in range(3)]
    abar_out = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
    pbar = torch.empty(p.shape, dtype=torch.float64, device="cuda")
    ai, ao = [t.data_ptr() for t in abar_in], [t.data_ptr() for t in abar_out]
    ybar16 = [torch.randn(p.shape, dtype=torch.float64, device="cuda", generator=g) for _ in range(16)]
    xbar16 = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in range(16)]
    y16, x16 = [t.data_ptr() for t in ybar16], [t.data_ptr() for t in xbar16]
    torch.cuda.synchronize()

    def dry_fwd():
        ctx.pressure(**press)
        ctx.rk4_step()

    def dry_adj():
        ctx.rk4_adjoint_ex(yp, ai, xp, pbar.data_ptr())
        ctx.pressure_adjoint(pbar.data_ptr(), ao, press["kind"], press["omega"], press["max_sweeps"], press["tol"])

    def moist_fwd():
        ctx.restore_ncopies(1.0)
        ctx.pressure(**press)
        ctx.satadj(0xF, count=False)
        ctx.sync_ncopies()
        ctx.rk4_step()

    def moist_adj():
        ctx.moist_adjoint(y16, ai, x16, pbar.data_ptr())
        ctx.pressure_adjoint(pbar.data_ptr(), ao, press["kind"], press["omega"], press["max_sweeps"], press["tol"])

    def pair(fwd_fn, adj_fn, n=3):
        for _ in range(2):
            fwd_fn()
            adj_fn()
        ctx.synchronize()
        f_ = a_ = 0.0
        for _ in range(n):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            fwd_fn()
            e[1].record(stream)
            adj_fn()
            e[2].record(stream)
            e[2].synchronize()
            f_ += e[0].elapsed_time(e[1])
            a_ += e[1].elapsed_time(e[2])
        return f_ / n, a_ / n

    try:
        f_, a_ = pair(dry_fwd, dry_adj)
        out["dry_full_step"] = {"fwd_ms": f_, "adj_ms": a_, "adj_over_fwd": a_ / f_,
                                "what": "forward = aturan_pressure (RB_LINE to 1e-8, taped) + aturan_rk4_step; adjoint "
                                        "= aturan_rk4_adjoint_ex (aux adjoint in, p_dyn adjoint out) + "
                                        "aturan_pressure_adjoint (the transposed solve to 1e-8)"}
        ctx.tape(2)
        f_, a_ = pair(moist_fwd, moist_adj)
        out["moist_full_step"] = {"fwd_ms": f_, "adj_ms": a_, "adj_over_fwd": a_ / f_,
                                  "what": "forward = restoreVar + aturan_pressure (RB_LINE to 1e-8) + aturan_satadj "
                                          "(4 gases) + n-copy sync + aturan_rk4_step, moist tape; adjoint = "
                                          "aturan_moist_adjoint (RK4 over t, u, v, w and the 12 species, the "
                                          "adjustment's implicit adjoint) + aturan_pressure_adjoint"}
    finally:
        ctx.close()
    return out


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def press_args(name):
    from aturan_b200 import params as P
    if name == "gs":
        return dict(kind=P.PRESS_GS_LEX, omega=1.0, max_sweeps=1, tol=0.0), "GS_LEX: one lexicographic sweep (PressureSolverUran)"
    if name == "rb":
        return dict(kind=P.PRESS_RB_SHARED, omega=1.0, max_sweeps=1, tol=0.0), "RB_SHARED: one red-black sweep (PressureSolver)"
    if name == "line":
        return dict(kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=50, tol=1e-6), "RB_LINE to relative residual 1e-6, omega 1.0"
    return dict(kind=P.PRESS_RB_SOR, omega=1.8, max_sweeps=400, tol=1e-6), "RB_SOR to relative residual 1e-6, omega 1.8"


# The two launches of one RK4 stage, timed together (the roofline's "kernel").
STAGE_KERNELS = {"mixed": "RK4 stage: rk_stage_pair_kernel (momentum + T) + rk_scalar_pair_kernel (15 scalars)",
                 "fp64": "RK4 stage: rk_stage_kernel (momentum + T) + rk_scalar_async_kernel (15 scalars)"}


def algorithmic_stage_bytes(precision):
    """Average algorithmic bytes per RK4 stage launch over the shell's stored cells."""
    total = 0.0
    for w in STAGE_WORDS:
        if precision == "fp64":
            total += w * 8
        else:          # FP32 storage except the FP64 pressure pair read by every stage
            total += (w - 2) * 4 + 2 * 8
    return total / 4 * N_CELLS


def step_alg_bytes(precision, press, sweeps, N=N_CELLS):
    """Algorithmic bytes of one full step (every value each kernel must read or write once, per
    stored cell; FP32 words of 4 B in the mixed form except the FP64 pressure family):
      RK4 stages   the stage words above (81 + 119 + 119 + 106 per cell)
      prelude      level means (t, p_stat) and hydrostatic integral (t, p_stat, v, w; p_baro, p_b0,
                   p_bfollow read, p_hydro and p_bfollow written: FP64)
      satadj+sync  t, p_stat, rho_mix, 12 species read; t, 12 species written; their 13 n-copies and
                   nh4sh's (read and written) by the fused sync; the mixed form adds the temperature
                   pair's low parts (t read and written, tn written)
      pressure     RB_LINE / RB_SOR: aux_u, v, w read and the FP64 source written; per sweep p and the
                   source read, p written (FP32 correction sweeps in the mixed form); per residual check
                   p and the source read (the mixed form also writes r and e in FP32); per column
                   correction p read and written; the mixed form's refinement p += e. GS_LEX: the
                   source (5 words) and one sweep (3 words)
    sweeps: the pressure sweeps of each timed step (aturan_pressure_last)."""
    mixed = precision == "mixed"
    e = 4 if mixed else 8
    rk = sum(((w - 2) * 4 + 2 * 8) if mixed else w * 8 for w in STAGE_WORDS)
    prelude = 6 * e + 5 * 8
    sat = 43 * e + (3 * 4 if mixed else 0)
    S = statistics.mean(sweeps) if sweeps else 0.0
    if press in ("line", "sor"):
        every = 8 if press == "line" else 16
        corr = math.ceil(S / every) if S else 0
        if mixed:
            inner = 2 if press == "line" else 48
            refine = math.ceil(S / inner) if S else 0
            pres = (3 * e + 8) + S * 3 * 4 + (refine + 1) * (2 * 8 + 2 * 4) + refine * (4 + 2 * 8) + corr * 2 * 4
        else:
            checks = (S + 1) if press == "line" else (math.ceil(S / 16) + 1)
            pres = (3 * e + 8) + S * 3 * 8 + checks * 2 * 8 + corr * 2 * 8
    else:
        pres = 5 * 8 + 3 * 8 * max(S, 1.0)
    out = {"rk4": rk * N, "prelude": prelude * N, "satadj_sync": sat * N, "pressure": pres * N}
    out["total"] = sum(out.values())
    return out


def post_step_bytes(p, pp, e):
    """Algorithmic bytes of one aturan_post_step with knobs pp and storage e bytes per value: every
    value the passes must read or write once (the padding never counts)."""
    im, jm, km = p.im, p.jm, p.km
    N = im * jm * km
    b = 0
    if pp.damp_t_horiz != 0.0:
        b += 2 * N                                   # t along k (and j): read and write
        if pp.damp_t_j:
            b += 2 * N
    if pp.damp_t_vert != 0.0:
        b += 2 * N
    if pp.vel_shapiro != 0.0:
        b += 3 * 3 * 2 * N                           # u, v, w along k, j, i
    nrad, nphi, nthx, nthz, nsp = 25, 24, 16, 9, 13
    b += nrad * 6 * jm * km                          # radius: planes 1, 2, im-2, im-3 read, 0 and im-1 written
    b += (nthx * 6 + nthz * 2) * im * km             # theta: rows 1, 2, jm-2, jm-3 read, 0 and jm-1 written
    b += nphi * 2 * im * jm                          # phi: k = 0 read, k = km-1 written
    if pp.species_clamp:
        b += nsp * N                                 # every species value read (writes: the clipped few)
    return b * e


def post_step_timing(api, P, S, torch, precision, calls=20):
    """aturan_post_step with the reference's default knobs at 41x181x361: device time per call (CUDA
    events on the context's stream, mean over `calls` after 3 warm-up calls), its algorithmic bytes
    and GB/s, and the compiled reference's same passes on the host cores when it is present."""
    prec = P.MIXED if precision == "mixed" else P.FP64
    p = P.default_params(precision=prec)
    pp = P.default_post_params()
    ctx = api.Context(p)
    ctx.upload_state(S.synthetic_state(p, seed=20261205))
    s = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(3):
        ctx.post_step(pp)
    ctx.synchronize()
    ctx.profile(False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(calls):
        ctx.post_step(pp)
    e1.record(s)
    e1.synchronize()
    launches = ctx.profile_read()["post"][0] // calls
    ctx.close()
    ms = e0.elapsed_time(e1) / calls
    alg = post_step_bytes(p, pp, 4 if precision == "mixed" else 8)
    peak, peak_kind = peaks()
    out = {"ms": ms, "launches": launches, "alg_bytes": alg, "achieved_gbs": alg / (ms / 1e3) / 1e9,
           "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_source": f"{peak_kind} hbm_gbs",
           "what": "t filter along k, radius/theta/phi boundary passes with the species floor and lid v, w, "
                   "species clamp (the reference's default knobs), 41x181x361; 20 calls, state > L2"}
    try:
        from oracle import ref as R
        if R.available():
            m = R.Ref.get_instance()
            m.post_step(pp)
            t0 = time.perf_counter()
            for _ in range(5):
                m.post_step(pp)
            out["cpu_reference_ms"] = (time.perf_counter() - t0) / 5 * 1e3
            out["cpu_reference_cores"] = os.cpu_count()
    except Exception as ex:               # reported, never silently replaced
        out["cpu_reference_ms"] = f"{type(ex).__name__}: {ex}"
    return out


def chem_bytes(p, e, changed, tpair):
    """Algorithmic bytes of one aturan_chemistry(NH4SH_EQ | FORCING) with storage e bytes per value:
    the equilibrium reads t, p_stat, nh3, h2s, nh4sh once and writes t, nh3, h2s, nh4sh in the
    `changed` cells; the forcing reads t, p_stat, the three species, u, v, w once and writes
    rho_mix, thermalmassflux, difflux_* (3), massflux_* (3) and fluxlim_nh4sh once, and each of the
    eight filtered fields is read and written once more by its filter (the three axes fused, the
    minimum). tpair: t carries a second FP32 word (the mixed form's pair)."""
    N = p.im * p.jm * p.km
    tw = 4 if tpair else 0
    eq = N * (5 * e + tw) + changed * (4 * e + tw)
    forcing = N * (8 * e + tw) + N * 9 * e + 8 * 2 * N * e
    return eq + forcing


def chem_timing(api, P, S, torch, precision, calls=10):
    """aturan_chemistry (NH4SH equilibrium and forcing, the reference's knobs) at 41x181x361: device
    time per call (CUDA events on the context's stream, mean over `calls` on a freshly uploaded
    state each, after one warm-up call), its algorithmic bytes and GB/s, and the compiled
    reference's same calls on the host cores when it is present."""
    prec = P.MIXED if precision == "mixed" else P.FP64
    p = P.default_params(precision=prec)
    st = S.synthetic_state(p, seed=20261207)
    ctx = api.Context(p)
    s = torch.cuda.ExternalStream(ctx.stream)
    ctx.upload_state(st)
    nf, nd = ctx.chemistry(counts=True)
    ms = []
    for _ in range(calls):
        ctx.upload_state(st)
        ctx.synchronize()
        ctx.profile(False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.chemistry()
        e1.record(s)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = ctx.profile_read()["chem"][0]
    ctx.close()
    m = statistics.median(ms)
    alg = chem_bytes(p, 4 if precision == "mixed" else 8, nf + nd, precision == "mixed")
    peak, peak_kind = peaks()
    out = {"ms": m, "launches": launches, "alg_bytes": alg, "achieved_gbs": alg / (m / 1e3) / 1e9,
           "frac": alg / (m / 1e3) / 1e9 / peak, "peak_source": f"{peak_kind} hbm_gbs",
           "cells_formed": nf, "cells_decomposed": nd,
           "what": "NH4SH equilibrium + chemistry forcing (rho_mix, thermal mass flux, D lap(c), filters, mass "
                   f"rates, Superbee limiter, filters), {precision}, 41x181x361, synthetic state; median of {calls}"}
    try:
        from oracle import ref as R
        if R.available():
            m_ = R.Ref.get_instance()
            m_.load(st)
            t0 = time.perf_counter()
            m_.chem_eq()
            m_.chem_forcing()
            out["cpu_reference_ms"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference_cores"] = os.cpu_count()
    except Exception as ex:               # reported, never silently replaced
        out["cpu_reference_ms"] = f"{type(ex).__name__}: {ex}"
    return out


def iteration_timing(api, P, S, torch, precision, pa, iters=8):
    """aturan_iteration at 41x181x361 with the state resident: device time per iteration over
    iterations 5..4+iters (even and odd alternating, as the loop runs them), with the MCA every
    iteration (the reference's default) and without it, and the per-kind device times of the
    first (events on the streams each kind runs on)."""
    prec = P.MIXED if precision == "mixed" else P.FP64
    p = P.default_params(precision=prec)
    st = S.synthetic_state(P.default_params(), seed=20261208)
    out = {"what": f"one iteration of the reference's loop on the device, {precision}, 41x181x361, the "
                   f"bench's pressure solve; mean over {iters} iterations"}
    for mca in (1, 0):
        ip = P.default_iter_params()
        ip.press_kind, ip.omega, ip.max_sweeps, ip.tol = pa["kind"], pa["omega"], pa["max_sweeps"], pa["tol"]
        ip.mca_stride = mca
        ctx = api.Context(p)
        ctx.upload_state(st)
        s = torch.cuda.ExternalStream(ctx.stream)
        for it in range(1, 5):
            ctx.iteration(it, ip)
        ctx.synchronize()
        ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for it in range(5, 5 + iters):
            ctx.iteration(it, ip)
        e1.record(s)
        e1.synchronize()
        prof = ctx.profile_read()
        ctx.close()
        key = "with_mca" if mca else "without_mca"
        out[key] = {"ms_per_iteration": e0.elapsed_time(e1) / iters,
                    "kinds_ms_per_iteration": {k: v[1] / iters for k, v in prof.items() if v[0]}}
    return out


def mca_timing(api, P, S, torch, reps=3, grid=(41, 181, 361), reference=True):
    """aturan_mca (FP64, default knobs) on a seeded synthetic state in which most columns are
    unstable: device time of one call on the freshly uploaded state (CUDA events on the context's
    stream, median of `reps`, after one warm-up call), and the compiled reference's same call on
    the host cores when it is present (full grid only)."""
    p = P.default_params(*grid)
    st = S.synthetic_state(p, seed=72)
    ctx = api.Context(p)
    s = torch.cuda.ExternalStream(ctx.stream)
    ms = []
    for r in range(reps + 1):
        ctx.upload_state(st)
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.mca()
        e1.record(s)
        e1.synchronize()
        if r > 0:
            ms.append(e0.elapsed_time(e1))
    ctx.close()
    out = {"ms": statistics.median(ms), "columns": p.jm * p.km,
           "what": "moist convective adjustment, FP64, %dx%dx%d, synthetic state (seed 72), one call per upload" % grid}
    if not reference:
        return out
    try:
        from oracle import ref as R
        if R.available():
            m = R.Ref.get_instance()
            m.load(st)
            t0 = time.perf_counter()
            m.mca()
            out["cpu_reference_ms"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference_cores"] = os.cpu_count()
    except Exception as ex:               # reported, never silently replaced
        out["cpu_reference_ms"] = f"{type(ex).__name__}: {ex}"
    return out


POISSON_OMEGAS = (1.0, 1.5, 1.6, 1.7, 1.8, 1.9)


def poisson_timing(api, P, S, torch, tol=1e-8, omegas=POISSON_OMEGAS):
    """The isolated Poisson solve at 41x181x361: the source is the shared solver's divergence
    (with its boundary rows and clamp) of a seeded N(0, 1) velocity field smoothed by 3 passes of a
    3x3x3 box filter (aturan_b200.state.poisson_velocity / poisson_source, FP64); Lc x = src from
    x = 0 to a relative L2 residual of `tol` through aturan_pressure_solve, for point red-black SOR
    and radial-line red-black SOR at every omega, in an FP64 context (FP64 sweeps) and in a mixed
    context (FP32 sweeps inside FP64 iterative refinement; the same FP64 source and solution).
    Per case: the status, sweeps, the achieved residual, device time (CUDA events on the context's
    stream around the synchronous call) and the sweeps' algorithmic bytes (p read, src read, p
    written per sweep: 3 words per stored cell) against the HBM peak. The iterate and the source
    (43 MB in FP64) fit in L2, so that fraction can pass 1."""
    p = P.default_params()
    u, v, w = S.poisson_velocity(p, seed=20261205)
    src = S.poisson_source(p, u, v, w)
    bd = torch.tensor(src, device="cuda")
    xd = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    peak, peak_kind = peaks()
    N = p.im * p.jm * p.km
    out = {"what": "Lc x = div(smoothed N(0,1) velocity) at 41x181x361 from x = 0 to a relative residual of "
                   f"{tol:g}; aturan_pressure_solve; FP64 context = FP64 sweeps, mixed context = FP32 sweeps "
                   "in FP64 refinement", "tol": tol, "cases": [], "peak_source": f"{peak_kind} hbm_gbs"}
    solves = {}
    for prec_name, prec in (("fp64", P.FP64), ("mixed", P.MIXED)):
        ctx = api.Context(P.default_params(precision=prec))
        s = torch.cuda.ExternalStream(ctx.stream)
        for kind_name, kind, cap in (("rb_sor", P.PRESS_RB_SOR, 6000), ("rb_line", P.PRESS_RB_LINE, 400)):
            for om in omegas:
                for rep in range(2):               # the first call warms the kernels up
                    xd.zero_()
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(s)
                    rc, sweeps, res = ctx.pressure_solve(bd.data_ptr(), xd.data_ptr(), kind, False, om, cap, tol)
                    e1.record(s)
                    e1.synchronize()
                ms = e0.elapsed_time(e1)
                word = 8 if prec_name == "fp64" else 4
                alg = 3 * word * N * sweeps
                out["cases"].append({"kind": kind_name, "precision": prec_name, "omega": om,
                                     "converged": rc == 0, "sweeps": sweeps, "resid": res, "ms": ms,
                                     "sweep_alg_gbs": alg / (ms / 1e3) / 1e9,
                                     "sweep_frac": alg / (ms / 1e3) / 1e9 / peak})
                if rc == 0 and om in (1.0, 1.8):
                    solves[(prec_name, kind_name, om)] = xd.clone()
        ctx.close()
    # the mixed solution against the FP64 one (interior, up to the free constant of the
    # all-Neumann problem), for the fastest case of each kind
    I = (slice(1, p.im - 1), slice(1, p.jm - 1), slice(0, p.km - 1))
    agree = {}
    for kind_name, om in (("rb_sor", 1.8), ("rb_line", 1.0)):
        a, b = solves.get(("mixed", kind_name, om)), solves.get(("fp64", kind_name, om))
        if a is not None and b is not None:
            d = (a - b)[I]
            d = d - d.mean()
            bb = b[I] - b[I].mean()
            agree[f"{kind_name}_omega{om}"] = float(d.abs().max() / bb.abs().max())
    out["mixed_vs_fp64_solution"] = agree
    best = {}
    for c in out["cases"]:
        key = f"{c['kind']}_{c['precision']}"
        if c["converged"] and (key not in best or c["ms"] < best[key]["ms"]):
            best[key] = {"omega": c["omega"], "sweeps": c["sweeps"], "ms": c["ms"]}
    out["best"] = best
    return out


def cpu_reference_step_time(nsteps, press, budget_s=120.0):
    """Time the reference's own step on the host cores after one untimed warm-up step; at most
    nsteps steps and no more than fit in budget_s. Returns (seconds/step, kind, cores, note, n)."""
    from oracle import ref as R
    from aturan_b200 import params as P, state as S
    cores = os.cpu_count() or 1
    p = P.default_params()
    if R.available():
        m = R.Ref.get_instance()
        m.load(S.perturb(m.state(), p, seed=20261204))

        def one():
            if press == "rb":
                m.pressure_rb(1)
            else:
                m.pressure_gs()
            for g in range(4):
                m.satadj(g)
            m.sync_ncopies()
            m.rk4()
        kind = "reference"
        what = f"the compiled reference (oracle/_ref, -O3, OpenMP {cores} threads) on its own initialised state, perturbed"
    else:
        from oracle import Oracle
        O = Oracle()
        O.set_threads(cores)
        st = S.synthetic_state(p, seed=20261204)
        pk = P.PRESS_RB_SHARED if press == "rb" else P.PRESS_GS_LEX

        def one():
            O.step(p, st, pk)
        kind = "port"
        what = f"the C restatement (oracle/, OpenMP {cores} threads) on the synthetic state"
    t0 = time.perf_counter()
    one()                                          # warm-up, also the time estimate
    t_warm = time.perf_counter() - t0
    n = max(1, min(nsteps, int(budget_s / max(t_warm, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(n):
        one()
    dt = (time.perf_counter() - t0) / n
    ptxt = ("1 red-black sweep (PressureSolver)" if press == "rb" else
            "1 lexicographic GS sweep (PressureSolverUran, the reference's default; the reference has no "
            "solve to a residual, so this is its step for every GPU pressure kind)")
    return dt, kind, cores, f"{n} full steps (pressure: {ptxt} + 4 SatAdj + sync + RK4) of {what}, 41x181x361", n


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    dt, kind, cores, note, n = cpu_reference_step_time(max(1, args.steps), args.press)
    value = N_CELLS / dt
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": world, "steps": n, "warmup": 1, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "dynamical-core full step (pressure + 4 SatAdj + n-copy sync + RK4), 41x181x361, "
                               "FP64 on the host cores",
                   "grid": [41, 181, 361], "cells": N_CELLS,
                   # the solve the reference ran: it has no solve to a residual, so every pressure kind
                   # other than the shared red-black sweep times its default lexicographic GS sweep
                   "pressure": "rb" if args.press == "rb" else "gs"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": kind, "sample": note},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--press", default="line", choices=["gs", "rb", "sor", "line"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the RK4 adjoint / forward timing")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--profile-run", action="store_true",
                    help="only the warm-up and the K timed steps (for ncu); prints a short line")
    ap.add_argument("--grid", default="41x181x361", help="IxJxK of the shell (profiling cases)")
    ap.add_argument("--post-step", action="store_true",
                    help="only the passes after RK4 (aturan_post_step): prints the post_step object")
    ap.add_argument("--mca", action="store_true",
                    help="only the moist convective adjustment (aturan_mca): prints the mca object")
    ap.add_argument("--iteration", action="store_true",
                    help="only the full iteration of the model's loop (aturan_iteration): prints the iteration object")
    ap.add_argument("--poisson", action="store_true",
                    help="only the isolated Poisson solve (omega sweep, FP64 and mixed): prints the poisson object")
    args = ap.parse_args()
    rank, world, local = dist_env()

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)

    from aturan_b200 import api, params as P, replicas, state as S
    if args.mca:
        if rank == 0:
            grid = tuple(int(x) for x in args.grid.lower().split("x"))
            print(json.dumps({"mca": mca_timing(api, P, S, torch, grid=grid,
                                                reference=grid == (41, 181, 361))}), flush=True)
        return
    if args.iteration:
        if rank == 0:
            print(json.dumps({"iteration": iteration_timing(api, P, S, torch, args.precision,
                                                            press_args(args.press)[0]),
                              "precision": args.precision}), flush=True)
        return
    if args.poisson:
        if rank == 0:
            print(json.dumps({"poisson": poisson_timing(api, P, S, torch)}), flush=True)
        return
    if args.post_step:
        if rank == 0:
            print(json.dumps({"post_step": post_step_timing(api, P, S, torch, args.precision),
                              "precision": args.precision}), flush=True)
        return
    prec = P.MIXED if args.precision == "mixed" else P.FP64
    gi, gj, gk = (int(x) for x in args.grid.lower().split("x"))
    p = P.default_params(gi, gj, gk, precision=prec)
    st = S.synthetic_state(p, seed=replicas.replica_seed(20261203, rank))
    ctx = api.Context(p)
    ctx.upload_state(st)
    pa, press_note = press_args(args.press)

    def step():
        ctx.step(**pa)

    W = max(3, args.warmup)
    for _ in range(W):
        step()
    ctx.synchronize()
    if args.profile_run:
        for _ in range(args.steps):
            step()
        ctx.synchronize()
        print(json.dumps({"profile_run": True, "grid": args.grid, "precision": args.precision,
                          "steps": args.steps, "warmup": W}), flush=True)
        ctx.close()
        return
    stream = torch.cuda.ExternalStream(ctx.stream)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed region: K steps, device time on the context's stream, max over ranks ----
    K = args.steps
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.profile(timing=False)
    e0.record(stream)
    for _ in range(K):
        step()
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = sum(v[0] for v in ctx.profile_read().values())
    ms_max = replicas.max_over_ranks(ms, dist, device="cuda")
    value = replicas.throughput(N_CELLS, K, world, ms_max / 1e3)

    # ---- per-kernel device times of the same steps (event-bracketed pass) ----
    ctx.profile(timing=True)
    sweeps = []
    for _ in range(K):
        step()
        sweeps.append(ctx.pressure_last()[0])      # the step's pressure sweeps (a host-side value)
    prof = ctx.profile_read()
    n_stage, ms_stage = prof["rk_stage"]          # 2 launches per stage
    avg_stage_ms = ms_stage / (4 * K)
    alg = algorithmic_stage_bytes(args.precision)
    peak, peak_kind = peaks()
    achieved = alg / (avg_stage_ms / 1e3) / 1e9
    step_alg = step_alg_bytes(args.precision, args.press, sweeps)
    step_roof = {"achieved": step_alg["total"] / (ms_max / K / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": step_alg["total"] / (ms_max / K / 1e3) / 1e9 / peak, "alg_bytes_per_step": step_alg,
                 "sweeps_per_step": statistics.mean(sweeps) if sweeps else None,
                 "what": "every kernel of the step: the algorithmic bytes of the RK4 stages, the level means "
                         "and hydrostatic integral, the saturation adjustment with its fused n-copy sync, and "
                         "the pressure solve with its actual sweep count, divided by ms_per_step"}
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"rk_stage_{args.precision}_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_launch")
        except Exception:
            traffic = None

    # ---- end to end through the C ABI with host buffers ----
    from aturan_b200 import fields as F
    # what a CPU driver hands the drop-in every step: the prognostic fields
    # and the pointwise RHS inputs its CPU modules (chemistry, precipitation, turbulence closure,
    # boundary conditions, filters) changed; the n-copies, p_dyn, p_hydro, p_bfollow and the
    # constant fields stay resident. Back: the new prognostic fields, p_dyn, p_hydro and the
    # projection fields.
    in_names = F.PROGNOSTIC + F.FORCING
    out_names = F.PROGNOSTIC + ["p_dyn", "p_hydro"] + F.PROJECTION
    pinned = {n: torch.from_numpy(np.ascontiguousarray(st[n])).pin_memory() for n in in_names}
    outs = {n: torch.empty(p.shape, dtype=torch.float64).pin_memory() for n in out_names}
    in_ptrs = [pinned[n].data_ptr() for n in in_names]
    out_ptrs = [outs[n].data_ptr() for n in out_names]
    barrier()
    E = max(1, args.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(E):
        ctx.upload_many(in_names, in_ptrs)          # aturan_upload_many: one wait for all fields
        step()
        ctx.download_many(out_names, out_ptrs)      # aturan_download_many
    e2e_s = time.perf_counter() - t0
    e2e_step_value = replicas.throughput(N_CELLS, E, world, replicas.max_over_ranks(e2e_s, dist, device="cuda"))
    fbytes = p.im * p.jm * p.km * 8
    e2e_step = {"value": e2e_step_value, "unit": "cell-steps/s", "h2d_bytes_per_step": len(in_names) * fbytes,
                "d2h_bytes_per_step": len(out_names) * fbytes, "steps": E,
                "what": "aturan_step alone, the host modules of the loop kept on the CPU: their inputs to the "
                        "RHS up and the step's outputs down every step"}

    # the drop-in with every module of the loop on the device (aturan_chemistry, _precipitation,
    # _turbulence, _mca, _post_step): the forcing the step reads is formed and kept on the device,
    # so what crosses PCIe every step is the state a host driver owns -- the prognostic fields up
    # (the n-copies then set from them on the device, restoreVar's copy) and the new prognostic
    # fields with p_dyn back
    in_loop = F.PROGNOSTIC
    out_loop = F.PROGNOSTIC + ["p_dyn"]
    in_ptrs_l = [pinned[n].data_ptr() for n in in_loop]
    out_ptrs_l = [outs[n].data_ptr() for n in out_loop]
    barrier()
    t0 = time.perf_counter()
    for _ in range(E):
        ctx.upload_many(in_loop, in_ptrs_l)
        ctx.restore_ncopies(1.0)
        step()
        ctx.download_many(out_loop, out_ptrs_l)
    e2e_loop_s = time.perf_counter() - t0
    e2e_value = replicas.throughput(N_CELLS, E, world, replicas.max_over_ranks(e2e_loop_s, dist, device="cuda"))

    # ---- accuracy of the mixed step against the FP64 step (which matches the FP64 oracle) ----
    accuracy = None
    if args.precision == "mixed" and rank == 0:
        accuracy = mixed_accuracy(api, P, S, F, pa, torch)
        if pa["tol"] > 0.0:
            # the same comparison with both solves taken to 1e-9, so that the solve tolerance (two
            # different iterates each within tol of the solution) does not mask the arithmetic
            tight = dict(pa, tol=1e-9, max_sweeps=max(pa["max_sweeps"], 100))
            acc9 = mixed_accuracy(api, P, S, F, tight, torch, steps=(1, 10))
            accuracy["solve_tol_1e-9"] = {k: acc9[k] for k in ("step1", "step10", "step10_p99.99")}

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        try:
            adjoint = adjoint_timing(api, P, S, torch)
        except Exception as ex:          # reported, never silently replaced
            adjoint = {"error": f"{type(ex).__name__}: {ex}"}

    post = None
    if rank == 0 and not args.no_adjoint:
        try:
            post = post_step_timing(api, P, S, torch, args.precision)
        except Exception as ex:          # reported, never silently replaced
            post = {"error": f"{type(ex).__name__}: {ex}"}

    chem = None
    if rank == 0 and not args.no_adjoint:
        try:
            chem = chem_timing(api, P, S, torch, args.precision)
        except Exception as ex:          # reported, never silently replaced
            chem = {"error": f"{type(ex).__name__}: {ex}"}

    iteration = None
    if rank == 0 and not args.no_adjoint:
        try:
            iteration = iteration_timing(api, P, S, torch, args.precision, pa)
        except Exception as ex:          # reported, never silently replaced
            iteration = {"error": f"{type(ex).__name__}: {ex}"}

    poisson = None
    if rank == 0 and not args.no_adjoint:
        try:
            poisson = poisson_timing(api, P, S, torch)
        except Exception as ex:          # reported, never silently replaced
            poisson = {"error": f"{type(ex).__name__}: {ex}"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            dt, kind, cores, note, _ = cpu_reference_step_time(max(1, args.cpu_steps), args.press, budget_s=30.0)
            cpu = {"value": N_CELLS / dt, "unit": "cell-steps/s", "cores": cores, "kind": kind, "sample": note}
        except Exception as ex:          # reported, never silently replaced
            cpu = {"value": None, "unit": "cell-steps/s", "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "mixed" else "f64",
            "data": "synthetic seeded state (aturan_b200.state.synthetic_state)",
            "config": {"workload": f"dynamical-core full step: pressure ({press_note}) + 4 SatAdj + n-copy sync + RK4, "
                                   f"41x181x361, {args.precision}",
                       "grid": [41, 181, 361], "cells": N_CELLS, "precision": args.precision,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (working set > 1.5 GB), no flush"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": STAGE_KERNELS[args.precision], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs", "avg_launch_ms": avg_stage_ms,
                         "alg_bytes_per_launch": alg, "step": step_roof},
            "kernels_ms_per_step": {k: v[1] / K for k, v in prof.items()},
            "kernels_ms_note": "device time per kind from events on the stream each kind runs on; the "
                               "saturation adjustment and the n-copy sync run on a second stream beside the "
                               "pressure solve, so the satadj, copy and rb entries overlap in time",
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": len(in_loop) * fbytes,
                    "d2h_bytes_per_step": len(out_loop) * fbytes, "steps": E,
                    "what": "aturan_step through the C ABI with the prognostic state up from pinned host memory "
                            "(n-copies set from it on the device) and the new state with p_dyn back every step; "
                            "the forcing fields resident, formed on the device by the loop's other modules"},
            "e2e_step_only": e2e_step,
            "clocks": clk,
            "adjoint": adjoint,
            "post_step": post,
            "chemistry": chem,
            "iteration": iteration,
            "poisson": poisson,
            "cpu_baseline": cpu,
        }
        if accuracy is not None:
            line["accuracy_vs_fp64"] = accuracy
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def mixed_accuracy(api, P, S, F, pa, torch, steps=(1, 10, 200)):
    """The mixed step against the FP64 step (which matches the FP64 oracle) from the same state,
    each step followed by the reference's restoreVar (n-copies <- state) as its iteration loop does:
    per-field max |mixed - fp64| / max |fp64| over the interior after 1, 10 and 200 steps (and the
    99.99th percentile of the same ratio over cells, and the norm-wise ||mixed - fp64||_2 / ||fp64||_2),
    and both step times (CUDA events on each
    context's stream, median over steps 2..10, each step timed alone and waited for; and 30 steps
    back to back after step 200, as ms_per_step is taken). A third context times the FP64 step with tree-ordered
    level means (exact_reductions = 0): still within 1e-11 of the reference, and the fastest FP64
    step, so the fair denominator of the speed-up."""
    p64 = P.default_params(precision=P.FP64)
    p64t = P.default_params(precision=P.FP64)
    p64t.exact_reductions = 0
    p32 = P.default_params(precision=P.MIXED)
    st = S.synthetic_state(p64, seed=99)
    c64, c32, c64t = api.Context(p64), api.Context(p32), api.Context(p64t)
    c64.upload_state(st)
    c32.upload_state(st)
    c64t.upload_state(st)
    s64, s32 = torch.cuda.ExternalStream(c64.stream), torch.cuda.ExternalStream(c32.stream)
    s64t = torch.cuda.ExternalStream(c64t.stream)
    I = (slice(1, p64.im - 1), slice(1, p64.jm - 1), slice(0, p64.km - 1))
    out, t64, t32, t64t = {}, [], [], []
    done = 0

    def timed(ctx, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(**pa)
        e1.record(stream)
        e1.synchronize()
        ctx.restore_ncopies(1.0)          # the reference's restoreVar between iterations
        return e0.elapsed_time(e1)

    for n in steps:
        while done < n:
            a, b = timed(c64, s64), timed(c32, s32)
            c = timed(c64t, s64t) if done < 10 else None
            done += 1
            if 2 <= done <= 10:
                t64.append(a)
                t32.append(b)
                t64t.append(c)
        errs, p9999, l2 = {}, {}, {}
        for f in F.PROGNOSTIC + ["p_dyn"]:
            a, b = c32.download(f)[I], c64.download(f)[I]
            s = np.abs(b).max()
            d = np.abs(a - b) / (s if s > 0 else 1.0)
            errs[f] = float(d.max())
            p9999[f] = float(np.quantile(d, 0.9999))
            nb = float(np.linalg.norm(b))
            l2[f] = float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)
        out[f"step{n}"] = errs
        out[f"step{n}_p99.99"] = p9999
        out[f"step{n}_rel_l2"] = l2
        if n == 10:
            # the FP64 step with tree-ordered level sums against the bit-exact one: two FP64 paths
            # that differ by rounding only (~1e-13 in the level means), so what separates them
            # after 10 steps is the reference algorithm's own sensitivity (threshold tests)
            tre, trq = {}, {}
            for f in ("t", "u", "v", "w", "p_dyn"):
                a, b = c64t.download(f)[I], c64.download(f)[I]
                s_ = np.abs(b).max()
                d = np.abs(a - b) / (s_ if s_ > 0 else 1.0)
                tre[f] = float(d.max())
                trq[f] = float(np.quantile(d, 0.9999))
            out["fp64_tree_vs_fp64_step10"] = {"max": tre, "p99.99": trq}
    # the same three steps back to back (each followed by restoreVar, no host wait between
    # steps), as ms_per_step times the bench's step: 30 steps per context after the comparison
    def steady(ctx, stream, n=30):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.synchronize()
        e0.record(stream)
        for _ in range(n):
            ctx.step(**pa)
            ctx.restore_ncopies(1.0)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n
    st64, st32, st64t = steady(c64, s64), steady(c32, s32), steady(c64t, s64t)
    out["steady_ms_per_step"] = {"fp64": st64, "fp64_tree": st64t, "mixed": st32,
                                 "what": "30 steps back to back per context (restoreVar after each), CUDA "
                                         "events around all 30: the timing ms_per_step uses"}
    out["mixed_speedup_over_fp64_steady"] = st64 / st32
    out["mixed_speedup_over_fp64_tree_steady"] = st64t / st32
    c64.close()
    c32.close()
    c64t.close()
    m64, m32, m64t = statistics.median(t64), statistics.median(t32), statistics.median(t64t)
    out["fp64_ms_per_step"] = m64
    out["fp64_tree_ms_per_step"] = m64t
    out["mixed_ms_per_step"] = m32
    out["mixed_speedup_over_fp64"] = m64 / m32
    out["mixed_speedup_over_fp64_tree"] = m64t / m32
    return out


if __name__ == "__main__":
    main()
