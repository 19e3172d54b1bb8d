"""Python face of the C ABI (include/aturan_b200.h) over ctypes.

`Context` mirrors the reference's call sites on the hot path:

    ctx.pressure(kind)      PressureSolverUran(m).run() / PressureSolver<cUranusModel>(m).run()
    ctx.satadj(mask)        SaturationAdjustmentUran(m).run(gas, ...) x 4, in the loop's order
    ctx.sync_ncopies()      the ATURAN_RK_SCALAR_SYNC=2 copy after the adjustments
    ctx.rk4_step()          cUranusModel::RungeKuttaUran()
    ctx.step(kind)          the in-scope calls of one even iteration of cUranusModel::Run

State lives on the device; `upload`/`download` move whole fields as FP64 [i][j][k] arrays.
There is no CPU fallback: without the built library or a CUDA device the calls raise.
"""
import ctypes
import os

import numpy as np

from . import fields as F
from .params import (ChemParams, IterParams, Params, PostParams, PrecipParams, TurbParams, default_chem_params,
                     default_iter_params, default_params, default_post_params, default_precip_params,
                     default_turb_params)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaturan_b200.so")

OK, NOT_CONVERGED = 0, 1
E_INVALID, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_NONFINITE = -1, -2, -3, -4, -5
_NAMES = {0: "ok", 1: "not converged", -1: "invalid argument", -2: "unsupported", -3: "CUDA error",
          -4: "out of device memory", -5: "non-finite value"}

# Every entry point the header declares, with its ctypes signature.
SIGNATURES = {
    "aturan_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_ctx_create": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_ctx_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "aturan_upload": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "aturan_download": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "aturan_upload_device": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "aturan_download_device": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "aturan_download_buoy_ref": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_upload_many": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "aturan_download_many": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
                             ctypes.c_int),
    "aturan_pressure_last": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_rk4_step": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_tape": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "aturan_restore_ncopies": ([ctypes.c_void_p, ctypes.c_double], ctypes.c_int),
    "aturan_pressure_solve": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                               ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                              ctypes.c_int),
    "aturan_rk4_adjoint": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_rk4_adjoint_ex": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p], ctypes.c_int),
    "aturan_moist_adjoint": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p], ctypes.c_int),
    "aturan_set_heating": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "aturan_pressure_adjoint": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_pressure": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                         ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_satadj": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_sync_ncopies": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_step": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "aturan_sync": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "aturan_profile": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "aturan_profile_read": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "aturan_buoy_ref_level_static": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p], ctypes.c_int),
    "aturan_post_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_post_step": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_mca": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_chem_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_chemistry": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
                         ctypes.c_int),
    "aturan_turb_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_turbulence": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_precip_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_precipitation": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "aturan_iter_params_default": ([ctypes.c_void_p], ctypes.c_int),
    "aturan_iteration": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
}

CHEM_NH4SH_EQ, CHEM_FORCING = 1, 2

STATIC_MAX_IM, STATIC_MAX_JM, STATIC_MAX_LEVEL_CELLS = 512, 4096, 1 << 30

KERNEL_KINDS = ["rk_stage", "satadj", "gs", "rb", "hydro", "copy", "adjoint", "post", "mca", "chem", "turb", "precip"]
NSPECIES = 13

_LIB = None


def load_library(path=LIB_PATH):
    """Load libaturan_b200.so (built in-tree by `make -C aturan_b200/csrc`)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C aturan_b200/csrc` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


class AturanError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


def library_default_params():
    p = Params()
    rc = load_library().aturan_params_default(ctypes.byref(p))
    assert rc == 0
    return p


def library_default_post_params():
    pp = PostParams()
    rc = load_library().aturan_post_params_default(ctypes.byref(pp))
    assert rc == 0
    return pp


def library_default_chem_params():
    cp = ChemParams()
    rc = load_library().aturan_chem_params_default(ctypes.byref(cp))
    assert rc == 0
    return cp


def library_default_turb_params():
    tp = TurbParams()
    rc = load_library().aturan_turb_params_default(ctypes.byref(tp))
    assert rc == 0
    return tp


def library_default_precip_params():
    pp = PrecipParams()
    rc = load_library().aturan_precip_params_default(ctypes.byref(pp))
    assert rc == 0
    return pp


def library_default_iter_params():
    ip = IterParams()
    rc = load_library().aturan_iter_params_default(ctypes.byref(ip))
    assert rc == 0
    return ip


class Context:
    """One device-resident model state and its stream (aturan_ctx)."""

    def __init__(self, params=None):
        self.L = load_library()
        self.p = (params if params is not None else default_params()).copy()
        h = ctypes.c_void_p()
        rc = self.L.aturan_ctx_create(ctypes.byref(self.p), ctypes.byref(h))
        if rc != 0:
            raise AturanError(rc, "aturan_ctx_create failed")
        self.h = h
        self.shape = (self.p.im, self.p.jm, self.p.km)

    def _check(self, rc, what):
        if rc < 0:
            msg = self.L.aturan_last_error(self.h)
            raise AturanError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.aturan_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- fields ----
    def upload(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.shape, (name, a.shape)
        self._check(self.L.aturan_upload(self.h, F.ID[name], a.ctypes.data), f"upload {name}")

    def download(self, name, out=None):
        a = out if out is not None else np.empty(self.shape)
        self._check(self.L.aturan_download(self.h, F.ID[name], a.ctypes.data), f"download {name}")
        return a

    def upload_state(self, state):
        for n, a in state.items():
            if n in F.ID:
                self.upload(n, a)

    def download_state(self, names=F.NAMES):
        return {n: self.download(n) for n in names}

    def upload_device(self, name, ptr):
        self._check(self.L.aturan_upload_device(self.h, F.ID[name], ctypes.c_void_p(ptr)), f"upload_device {name}")

    def download_device(self, name, ptr):
        self._check(self.L.aturan_download_device(self.h, F.ID[name], ctypes.c_void_p(ptr)), f"download_device {name}")

    def buoy_ref_level(self):
        a = np.empty(self.p.im)
        self._check(self.L.aturan_download_buoy_ref(self.h, a.ctypes.data), "buoy_ref")
        return a

    # ---- the path ----
    def rk4_step(self):
        self._check(self.L.aturan_rk4_step(self.h), "rk4_step")

    def restore_ncopies(self, coeff=1.0):
        """aturan_restore_ncopies: the reference's restoreVar(coeff) after a step."""
        self._check(self.L.aturan_restore_ncopies(self.h, float(coeff)), "restore_ncopies")

    def post_step(self, pp=None, sums=False):
        """aturan_post_step: the filters, boundary passes and species clamp that follow the RK4 step
        (cUranusModel.cpp:1218-1248), with pp's knobs (default: the reference's defaults). With
        sums=True returns this call's clipped sum and count per species (synchronizes)."""
        pp = default_post_params() if pp is None else pp
        if not sums:
            self._check(self.L.aturan_post_step(self.h, ctypes.byref(pp), None, None), "post_step")
            return None
        added = np.zeros(NSPECIES)
        cells = np.zeros(NSPECIES, dtype=np.int64)
        self._check(self.L.aturan_post_step(self.h, ctypes.byref(pp), added.ctypes.data, cells.ctypes.data),
                    "post_step")
        return added, cells

    def mca(self):
        """aturan_mca: the moist convective adjustment (ConvectiveAdjustment.h:402-849), default knobs."""
        self._check(self.L.aturan_mca(self.h), "mca")

    def iteration(self, iter_n, ip=None):
        """aturan_iteration: iteration number iter_n (from 1) of the model's loop
        (cUranusModel.cpp:952-1296) with ip's knobs (default: the reference's)."""
        ip = default_iter_params() if ip is None else ip
        self._check(self.L.aturan_iteration(self.h, ctypes.byref(ip), int(iter_n)), "iteration")

    def precipitation(self, pp=None):
        """aturan_precipitation: the three-category scheme of H2O, NH3, CH4 and H2S
        (Precipitation<cUranusModel>::run, cUranusModel.cpp:1037) with pp's knobs (default: the
        reference's)."""
        pp = default_precip_params() if pp is None else pp
        self._check(self.L.aturan_precipitation(self.h, ctypes.byref(pp)), "precipitation")

    def turbulence(self, tp=None):
        """aturan_turbulence: the k-omega SST closure (Turbulence<cUranusModel>::run,
        cUranusModel.cpp:1270) with tp's knobs (default: the reference's)."""
        tp = default_turb_params() if tp is None else tp
        self._check(self.L.aturan_turbulence(self.h, ctypes.byref(tp)), "turbulence")

    def chemistry(self, what=CHEM_NH4SH_EQ | CHEM_FORCING, cp=None, counts=False):
        """aturan_chemistry: the NH4SH equilibrium (cUranusModel.cpp:1034) and/or the chemistry
        forcing (cUranusModel.cpp:1074-1087) with cp's constants (default: the reference's). With
        counts=True returns (cells that formed NH4SH, cells that decomposed it) (synchronizes)."""
        cp = default_chem_params() if cp is None else cp
        if not counts:
            self._check(self.L.aturan_chemistry(self.h, ctypes.byref(cp), int(what), None, None), "chemistry")
            return None
        nf, nd = ctypes.c_long(), ctypes.c_long()
        self._check(self.L.aturan_chemistry(self.h, ctypes.byref(cp), int(what), ctypes.byref(nf),
                                            ctypes.byref(nd)), "chemistry")
        return nf.value, nd.value

    def tape(self, on=True):
        """aturan_tape: keep (or free) what the adjoint needs from the following RK4 steps; on=True
        or 1 the dry tape (aturan_rk4_adjoint), 2 the moist tape (aturan_moist_adjoint)."""
        mode = 0 if not on else (2 if on == 2 else 1)
        self._check(self.L.aturan_tape(self.h, mode), "tape")

    def rk4_adjoint(self, ybar_ptrs, xbar_ptrs):
        """aturan_rk4_adjoint on device pointers (t, u, v, w order) to contiguous FP64 arrays."""
        yb = (ctypes.c_void_p * 4)(*[ctypes.c_void_p(int(x)) for x in ybar_ptrs])
        xb = (ctypes.c_void_p * 4)(*[ctypes.c_void_p(int(x)) for x in xbar_ptrs])
        self._check(self.L.aturan_rk4_adjoint(self.h, yb, xb), "rk4_adjoint")

    def rk4_adjoint_ex(self, ybar_ptrs, auxbar_ptrs, xbar_ptrs, pbar_ptr, heatbar_ptr=None):
        """aturan_rk4_adjoint_ex: auxbar_ptrs (3, or None) in; pbar_ptr, heatbar_ptr (or None) out."""
        yb = (ctypes.c_void_p * 4)(*[ctypes.c_void_p(int(x)) for x in ybar_ptrs])
        xb = (ctypes.c_void_p * 4)(*[ctypes.c_void_p(int(x)) for x in xbar_ptrs])
        ab = (ctypes.c_void_p * 3)(*[ctypes.c_void_p(int(x)) for x in auxbar_ptrs]) if auxbar_ptrs else None
        opt = lambda x: ctypes.c_void_p(int(x)) if x else None
        self._check(self.L.aturan_rk4_adjoint_ex(self.h, yb, ab, xb, opt(pbar_ptr), opt(heatbar_ptr)), "rk4_adjoint_ex")

    def moist_adjoint(self, ybar_ptrs, auxbar_ptrs, xbar_ptrs, pbar_ptr, heatbar_ptr=None):
        """aturan_moist_adjoint: ybar_ptrs / xbar_ptrs 16 device pointers (t, u, v, w and the twelve
        condensable species in field order); auxbar_ptrs (3, or None) in; pbar_ptr, heatbar_ptr (or
        None) out."""
        yb = (ctypes.c_void_p * 16)(*[ctypes.c_void_p(int(x)) for x in ybar_ptrs])
        xb = (ctypes.c_void_p * 16)(*[ctypes.c_void_p(int(x)) for x in xbar_ptrs])
        ab = (ctypes.c_void_p * 3)(*[ctypes.c_void_p(int(x)) for x in auxbar_ptrs]) if auxbar_ptrs else None
        opt = lambda x: ctypes.c_void_p(int(x)) if x else None
        self._check(self.L.aturan_moist_adjoint(self.h, yb, ab, xb, opt(pbar_ptr), opt(heatbar_ptr)), "moist_adjoint")

    def set_heating(self, ptr, on_device=True):
        """aturan_set_heating: a [jm][km] FP64 heating rate in K/s (device or host pointer), None removes it."""
        self._check(self.L.aturan_set_heating(self.h, ctypes.c_void_p(int(ptr)) if ptr else None,
                                              1 if on_device else 0), "set_heating")

    def pressure_adjoint(self, pbar_ptr, auxbar_ptrs, kind=3, omega=1.0, max_sweeps=200, tol=1e-10):
        """aturan_pressure_adjoint; (rc, sweeps, resid)."""
        ab = (ctypes.c_void_p * 3)(*[ctypes.c_void_p(int(x)) for x in auxbar_ptrs])
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self._check(self.L.aturan_pressure_adjoint(self.h, int(kind), float(omega), int(max_sweeps), float(tol),
                                                        ctypes.c_void_p(int(pbar_ptr)), ab, ctypes.byref(s),
                                                        ctypes.byref(r)), "pressure_adjoint")
        return rc, s.value, r.value

    def pressure_solve(self, b_ptr, x_ptr, kind=3, transposed=False, omega=1.0, max_sweeps=200, tol=1e-10):
        """aturan_pressure_solve on device pointers: Lc x = b (or Lc^T x = b); (rc, sweeps, resid)."""
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self._check(self.L.aturan_pressure_solve(self.h, int(kind), 1 if transposed else 0, float(omega),
                                                      int(max_sweeps), float(tol), ctypes.c_void_p(int(b_ptr)),
                                                      ctypes.c_void_p(int(x_ptr)), ctypes.byref(s), ctypes.byref(r)),
                         "pressure_solve")
        return rc, s.value, r.value

    def upload_many(self, names, ptrs, on_device=False):
        """aturan_upload_many: field names and host (or device) pointers of FP64 [i][j][k] arrays."""
        n = len(names)
        ids = (ctypes.c_int * n)(*[F.ID[x] for x in names])
        ps = (ctypes.c_void_p * n)(*[ctypes.c_void_p(int(x)) for x in ptrs])
        self._check(self.L.aturan_upload_many(self.h, n, ids, ps, 1 if on_device else 0), "upload_many")

    def download_many(self, names, ptrs, on_device=False):
        """aturan_download_many into host (or device) pointers of FP64 [i][j][k] arrays."""
        n = len(names)
        ids = (ctypes.c_int * n)(*[F.ID[x] for x in names])
        ps = (ctypes.c_void_p * n)(*[ctypes.c_void_p(int(x)) for x in ptrs])
        self._check(self.L.aturan_download_many(self.h, n, ids, ps, 1 if on_device else 0), "download_many")

    def pressure_last(self):
        """aturan_pressure_last: (sweeps, residual) of the last pressure solve."""
        s = ctypes.c_int()
        r = ctypes.c_double()
        self._check(self.L.aturan_pressure_last(self.h, ctypes.byref(s), ctypes.byref(r)), "pressure_last")
        return s.value, r.value

    def pressure(self, kind=0, omega=1.0, max_sweeps=1, tol=0.0):
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self._check(self.L.aturan_pressure(self.h, int(kind), float(omega), int(max_sweeps), float(tol),
                                                ctypes.byref(s), ctypes.byref(r)), "pressure")
        return rc, s.value, r.value

    def satadj(self, gas_mask=0xF, count=True):
        na, nn = ctypes.c_long(), ctypes.c_long()
        if count:
            self._check(self.L.aturan_satadj(self.h, int(gas_mask), ctypes.byref(na), ctypes.byref(nn)), "satadj")
            return na.value, nn.value
        self._check(self.L.aturan_satadj(self.h, int(gas_mask), None, None), "satadj")
        return None

    def sync_ncopies(self):
        self._check(self.L.aturan_sync_ncopies(self.h), "sync_ncopies")

    def step(self, kind=0, omega=1.0, max_sweeps=1, tol=0.0):
        return self._check(self.L.aturan_step(self.h, int(kind), float(omega), int(max_sweeps), float(tol)), "step")

    def profile(self, timing=True):
        """Reset the per-class launch counters (and event timing when timing=True)."""
        self._check(self.L.aturan_profile(self.h, 1 if timing else 0), "profile")

    def profile_read(self):
        """{kind: (launches, ms)} since the last profile()."""
        n = len(KERNEL_KINDS)
        ms = (ctypes.c_double * n)()
        la = (ctypes.c_long * n)()
        self._check(self.L.aturan_profile_read(self.h, ms, la, n), "profile_read")
        return {k: (la[q], ms[q]) for q, k in enumerate(KERNEL_KINDS)}

    def synchronize(self):
        self._check(self.L.aturan_sync(self.h), "sync")

    @property
    def stream(self):
        return self.L.aturan_stream(self.h)
