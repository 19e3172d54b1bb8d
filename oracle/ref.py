"""ctypes wrapper of the compiled reference (oracle/_ref/libaturan_ref_v{2,3}.so).

TEST INFRASTRUCTURE. The shared library is the reference's own C++ sources compiled unmodified
(oracle/Makefile, target `ref`) with oracle/ref/ref_harness.cpp exposing a C ABI over one
cUranusModel. It exists on machines where it was built from the reference tree; callers check
`available()` and skip otherwise. One model per process: the reference keeps its knobs in
function-local statics and its model is a process-wide singleton.
"""
import ctypes
import os

import numpy as np

from aturan_b200 import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
VEC_FIELDS = ("p_baro", "p_b0", "p_bfollow")


def _cpu_has(flag):
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    return flag in line.split()
    except OSError:
        pass
    return False


def lib_path():
    v3 = os.path.join(REF_DIR, "libaturan_ref_v3.so")
    v2 = os.path.join(REF_DIR, "libaturan_ref_v2.so")
    if os.path.exists(v3) and _cpu_has("avx2") and _cpu_has("fma") and _cpu_has("bmi2"):
        return v3
    if os.path.exists(v2):
        return v2
    return None


def available():
    return lib_path() is not None


_SINGLETON = None


class Ref:
    """The reference model, initialised once per process (Run() with nm = 0)."""

    def __init__(self, outdir="/tmp/aturan_ref_out", quiet=True, loop_iterations=0, path=None):
        path = path or lib_path()
        if path is None:
            raise RuntimeError("compiled reference not found under oracle/_ref")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_char_p]
        for fn in ("ref_get", "ref_set", "ref_get_vec"):
            getattr(L, fn).argtypes = [ctypes.c_char_p, vp]
        L.ref_set_vec.argtypes = [ctypes.c_char_p, vp, ctypes.c_long]
        L.ref_vec_size.argtypes = [ctypes.c_char_p]
        L.ref_vec_size.restype = ctypes.c_long
        L.ref_scalar.argtypes = [ctypes.c_char_p, vp]
        L.ref_cp_lapse.argtypes = [ctypes.c_double]
        L.ref_cp_lapse.restype = ctypes.c_double
        L.ref_pressure_shared.argtypes = [ctypes.c_int]
        L.ref_satadj.argtypes = [ctypes.c_int]
        L.ref_hydro.argtypes = [ctypes.c_int]
        if hasattr(L, "ref_damp_wiggles"):       # a harness built before the post-step entry points lacks them
            L.ref_damp_wiggles.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
            L.ref_clamp_species.argtypes = [vp, vp]
        if hasattr(L, "ref_chem_scalar"):
            L.ref_chem_scalar.argtypes = [ctypes.c_char_p, vp]
        if hasattr(L, "ref_turb_scalar"):
            L.ref_turb_scalar.argtypes = [ctypes.c_char_p, vp]
        if hasattr(L, "ref_precip_scalar"):
            L.ref_precip_scalar.argtypes = [ctypes.c_char_p, vp]
        L.ref_set_quiet(1 if quiet else 0)
        self.L = L
        self.path = path
        im, jm, km = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.ref_dims(ctypes.byref(im), ctypes.byref(jm), ctypes.byref(km))
        self.shape = (im.value, jm.value, km.value)
        os.makedirs(outdir, exist_ok=True)
        if loop_iterations > 0:
            # Run() with that many iterations of the model's own loop after its initialisation
            L.ref_create_loop.argtypes = [ctypes.c_char_p, ctypes.c_int]
            assert L.ref_create_loop(outdir.encode(), int(loop_iterations)) == 0
        else:
            assert L.ref_create(outdir.encode()) == 0

    @classmethod
    def get_instance(cls):
        global _SINGLETON
        if _SINGLETON is None:
            _SINGLETON = cls()
        return _SINGLETON

    def scalar(self, name):
        d = ctypes.c_double()
        assert self.L.ref_scalar(name.encode(), ctypes.byref(d)) == 0, name
        return d.value

    def get(self, name):
        a = np.empty(self.shape)
        if name in VEC_FIELDS or name == "buoy_ref_level":
            n = self.L.ref_vec_size(name.encode())
            v = np.empty(n)
            assert self.L.ref_get_vec(name.encode(), v.ctypes.data) == 0
            return v.reshape(self.shape) if name in VEC_FIELDS else v
        assert self.L.ref_get(name.encode(), a.ctypes.data) == 0, name
        return a

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if name in VEC_FIELDS:
            assert self.L.ref_set_vec(name.encode(), a.ctypes.data, a.size) == 0
            return
        assert a.shape == self.shape, (name, a.shape)
        assert self.L.ref_set(name.encode(), a.ctypes.data) == 0, name

    def state(self, names=F.NAMES):
        return {n: self.get(n) for n in names}

    def load(self, state):
        for n, a in state.items():
            if n in F.ID:
                self.set(n, a)

    def coords(self):
        rad = np.empty(self.shape[0])
        the = np.empty(self.shape[1])
        self.L.ref_coords(rad.ctypes.data_as(ctypes.c_void_p), the.ctypes.data_as(ctypes.c_void_p))
        return rad, the

    def cp_lapse(self, T):
        return self.L.ref_cp_lapse(float(T))

    def rk4(self):
        assert self.L.ref_rk4() == 0

    def hydro(self, advance=True):
        assert self.L.ref_hydro(int(advance)) == 0

    def pressure_gs(self):
        assert self.L.ref_pressure_uran() == 0

    def pressure_rb(self, sweeps):
        assert self.L.ref_pressure_shared(int(sweeps)) == 0

    def satadj(self, gas):
        assert self.L.ref_satadj(int(gas)) == 0

    def sync_ncopies(self):
        assert self.L.ref_sync_ncopies() == 0

    def geo_balance(self):
        return bool(self.L.ref_geo_balance())

    def post_step(self, pp):
        """cUranusModel.cpp:1218-1248 on the loaded state: the t and velocity filters with pp's
        axes and strengths (the values the model's own knobs take must be passed), then bcRadius,
        bcTheta, bcPhi and clampNegativeSpecies with the reference's own knobs. Returns this call's
        clipped sums and counts per species."""
        L = self.L
        if pp.damp_t_horiz != 0.0:
            assert L.ref_damp_wiggles(b"t", 0, int(pp.damp_t_j), 1, float(pp.damp_t_horiz)) == 0
        if pp.damp_t_vert != 0.0:
            assert L.ref_damp_wiggles(b"t", 1, 0, 0, float(pp.damp_t_vert)) == 0
        if pp.vel_shapiro != 0.0:
            for n in (b"u", b"v", b"w"):
                assert L.ref_damp_wiggles(n, 1, 1, 1, float(pp.vel_shapiro)) == 0
        assert L.ref_bc_radius() == 0 and L.ref_bc_theta() == 0 and L.ref_bc_phi() == 0
        added, cells = np.zeros(13), np.zeros(13, dtype=np.int64)
        n = L.ref_clamp_species(added.ctypes.data, cells.ctypes.data)
        assert n in (0, 13), n
        return added, cells

    def mca(self):
        """MoistConvectiveAdjustment as the model's loop calls it (cUranusModel.cpp:1276-1292)."""
        assert self.L.ref_mca() == 0

    def chem_eq(self):
        """ChemistryUran::EquilibriumNH4SH("loop") (cUranusModel.cpp:1034)."""
        assert self.L.ref_chem_eq() == 0

    def chem_forcing(self):
        """DiffMassFluxUran, the filters, ChemMassRateUran, FluxLimiterNH4SH and the filters
        (cUranusModel.cpp:1074-1087)."""
        assert self.L.ref_chem_forcing() == 0

    def chem_scalar(self, name):
        d = ctypes.c_double()
        assert self.L.ref_chem_scalar(name.encode(), ctypes.byref(d)) == 0, name
        return d.value

    def turbulence(self):
        """Turbulence<cUranusModel>::run (cUranusModel.cpp:1270)."""
        assert self.L.ref_turbulence() == 0

    def turb_scalar(self, name):
        d = ctypes.c_double()
        assert self.L.ref_turb_scalar(name.encode(), ctypes.byref(d)) == 0, name
        return d.value

    def precipitation(self):
        """Precipitation<cUranusModel>::run (cUranusModel.cpp:1037)."""
        assert self.L.ref_precipitation() == 0

    def precip_scalar(self, name):
        d = ctypes.c_double()
        assert self.L.ref_precip_scalar(name.encode(), ctypes.byref(d)) == 0, name
        return d.value
