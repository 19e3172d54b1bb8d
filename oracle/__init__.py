"""CPU oracle of the aturan_b200 hot path -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

`Oracle` wraps liboracle.so, the plain-C restatement of the reference's FP64 algorithm
(aturan_oracle.c, which cites the reference file:line each function follows). `oracle.ref`
wraps the compiled reference itself (oracle/_ref, built from the reference's own sources).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this package, and
only to check or to time the reference's CPU path; the product never routes through it.

Parity of the restatement is pinned against the compiled reference in
tests/test_oracle_vs_ref.py (bit equality) and against the committed fixtures in tests/golden/.
"""
import ctypes
import os
import subprocess

import numpy as np

from aturan_b200 import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def reference_tree():
    """Where the reference's sources lie: $ATURAN_REF, else the REF default of oracle/Makefile."""
    env = os.environ.get("ATURAN_REF")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as fh:
        for line in fh:
            if line.startswith("REF") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    return ""


def build(quiet=True):
    """Compile liboracle.so (and, when the reference tree is present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.check_call(["make", "-C", HERE, "liboracle.so"], stdout=out)
    ref = reference_tree()
    if ref and os.path.isdir(os.path.join(ref, "planet")):
        subprocess.check_call(["make", "-C", HERE, "-j8", "ref", f"REF={ref}"], stdout=out)


def field_ptrs(state):
    """A (double* [NFIELDS]) array over a dict of C-contiguous float64 arrays; missing = NULL."""
    arr = (ctypes.c_void_p * F.NFIELDS)()
    for name, a in state.items():
        if name not in F.ID:
            continue
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], name
        arr[F.ID[name]] = a.ctypes.data
    return arr


class Oracle:
    def __init__(self, path=LIB_PATH):
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, P = ctypes.c_void_p, ctypes.c_void_p
        for fn, args, res in (
            ("oracle_buoy_ref", [P, vp, vp], ctypes.c_int),
            ("oracle_hydro", [P, vp, vp, ctypes.c_int], ctypes.c_int),
            ("oracle_rk4", [P, vp, vp], ctypes.c_int),
            ("oracle_pressure_gs", [P, vp], ctypes.c_int),
            ("oracle_pressure_rb", [P, vp, ctypes.c_int], ctypes.c_int),
            ("oracle_pressure_sor", [P, vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_int, vp, vp], ctypes.c_int),
            ("oracle_pressure_line", [P, vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, vp, vp], ctypes.c_int),
            ("oracle_pressure_source", [P, vp, vp], ctypes.c_int),
            ("oracle_pressure_source_compat", [P, vp, vp], ctypes.c_int),
            ("oracle_pressure_residual", [P, vp, vp], ctypes.c_double),
            ("oracle_laplace_apply", [P, vp, vp, ctypes.c_int], ctypes.c_int),
            ("oracle_solve", [P, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                              vp, vp], ctypes.c_int),
            ("oracle_satadj", [P, vp, ctypes.c_int, vp, vp], ctypes.c_int),
            ("oracle_sync_ncopies", [P, vp], ctypes.c_int),
            ("oracle_step", [P, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                             ctypes.c_double, vp], ctypes.c_int),
            ("oracle_cp_lapse", [P, ctypes.c_double], ctypes.c_double),
            ("oracle_rhs_cell", [P, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            ("oracle_set_threads", [ctypes.c_int], None),
            ("oracle_post_step", [P, vp, P, vp, vp], ctypes.c_int),
            ("oracle_mca", [P, vp], ctypes.c_int),
            ("oracle_nh4sh_eq", [P, P, vp, vp], ctypes.c_int),
            ("oracle_chem_forcing", [P, P, vp], ctypes.c_int),
            ("oracle_turbulence", [P, P, vp], ctypes.c_int),
            ("oracle_precipitation", [P, P, vp], ctypes.c_int),
            ("oracle_iteration", [P, P, vp, ctypes.c_int], ctypes.c_int),
        ):
            f = getattr(L, fn)
            f.argtypes = args
            f.restype = res
        self.L = L

    @staticmethod
    def _p(p):
        return ctypes.cast(ctypes.pointer(p), ctypes.c_void_p)

    def set_threads(self, n):
        self.L.oracle_set_threads(int(n))

    def rk4(self, p, state):
        ref = np.zeros(p.im)
        assert self.L.oracle_rk4(self._p(p), field_ptrs(state), ref.ctypes.data) == 0
        return ref

    def buoy_ref(self, p, state):
        ref = np.zeros(p.im)
        assert self.L.oracle_buoy_ref(self._p(p), field_ptrs(state), ref.ctypes.data) == 0
        return ref

    def hydro(self, p, state, ref_level, advance=True):
        ref_level = np.ascontiguousarray(ref_level, dtype=np.float64)
        assert self.L.oracle_hydro(self._p(p), field_ptrs(state), ref_level.ctypes.data, int(advance)) == 0

    def pressure_gs(self, p, state):
        assert self.L.oracle_pressure_gs(self._p(p), field_ptrs(state)) == 0

    def pressure_rb(self, p, state, sweeps):
        assert self.L.oracle_pressure_rb(self._p(p), field_ptrs(state), int(sweeps)) == 0

    def pressure_sor(self, p, state, omega, max_sweeps, tol, check_every=1):
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self.L.oracle_pressure_sor(self._p(p), field_ptrs(state), float(omega), int(max_sweeps),
                                        float(tol), int(check_every), ctypes.addressof(s),
                                        ctypes.addressof(r))
        return rc, s.value, r.value

    def pressure_line(self, p, state, omega, max_iter, tol):
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self.L.oracle_pressure_line(self._p(p), field_ptrs(state), float(omega), int(max_iter), float(tol),
                                         ctypes.addressof(s), ctypes.addressof(r))
        return rc, s.value, r.value

    def laplace_apply(self, p, x, transposed=False):
        """Lc x or Lc^T x (the folded pressure operator) on the interior."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(p.shape)
        assert self.L.oracle_laplace_apply(self._p(p), x.ctypes.data, out.ctypes.data, int(transposed)) == 0
        return out

    def solve(self, p, b, x, transposed=False, line=True, omega=1.0, max_iter=200, tol=1e-10):
        """Solve Lc x = b or Lc^T x = b (b made compatible), x updated in place; (rc, iters, resid)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        assert x.flags.c_contiguous and x.dtype == np.float64
        s = ctypes.c_int()
        r = ctypes.c_double()
        rc = self.L.oracle_solve(self._p(p), b.ctypes.data, x.ctypes.data, int(transposed), int(line), float(omega),
                                 int(max_iter), float(tol), ctypes.addressof(s), ctypes.addressof(r))
        return rc, s.value, r.value

    def pressure_source(self, p, state):
        src = np.zeros(p.shape)
        assert self.L.oracle_pressure_source(self._p(p), field_ptrs(state), src.ctypes.data) == 0
        return src

    def pressure_source_compat(self, p, state):
        src = np.zeros(p.shape)
        assert self.L.oracle_pressure_source_compat(self._p(p), field_ptrs(state), src.ctypes.data) == 0
        return src

    def pressure_residual(self, p, state, src):
        return self.L.oracle_pressure_residual(self._p(p), field_ptrs(state), src.ctypes.data)

    def satadj(self, p, state, gas):
        na, nn = ctypes.c_long(), ctypes.c_long()
        assert self.L.oracle_satadj(self._p(p), field_ptrs(state), int(gas), ctypes.addressof(na),
                                    ctypes.addressof(nn)) == 0
        return na.value, nn.value

    def sync_ncopies(self, p, state):
        assert self.L.oracle_sync_ncopies(self._p(p), field_ptrs(state)) == 0

    def step(self, p, state, press_kind=0, omega=1.0, max_sweeps=1, tol=0.0):
        ref = np.zeros(p.im)
        assert self.L.oracle_step(self._p(p), field_ptrs(state), int(press_kind), float(omega),
                                  int(max_sweeps), float(tol), ref.ctypes.data) == 0
        return ref

    def cp_lapse(self, p, T):
        return self.L.oracle_cp_lapse(self._p(p), float(T))

    def rhs_cell(self, p, state, i, j, k):
        out = np.zeros(22)
        assert self.L.oracle_rhs_cell(self._p(p), field_ptrs(state), i, j, k, out.ctypes.data) == 0
        return out

    def post_step(self, p, state, pp):
        """The passes after RK4 (filters, boundary passes, species clamp) on the state in place;
        returns this call's clipped sums and counts per species."""
        added, cells = np.zeros(13), np.zeros(13, dtype=np.int64)
        assert self.L.oracle_post_step(self._p(p), field_ptrs(state), self._p(pp), added.ctypes.data,
                                       cells.ctypes.data) == 0
        return added, cells

    def mca(self, p, state):
        """The moist convective adjustment (default knobs) on the state in place."""
        assert self.L.oracle_mca(self._p(p), field_ptrs(state)) == 0

    def nh4sh_eq(self, p, cp, state):
        """EquilibriumNH4SH("loop") on the state in place; returns (cells formed, cells decomposed)."""
        c = np.zeros(2, dtype=np.int64)
        assert self.L.oracle_nh4sh_eq(self._p(p), self._p(cp), field_ptrs(state), c.ctypes.data) == 0
        return int(c[0]), int(c[1])

    def chem_forcing(self, p, cp, state):
        """The chemistry forcing sequence (rho_mix, thermalmassflux, difflux_*, massflux_*,
        fluxlim_nh4sh) on the state in place."""
        assert self.L.oracle_chem_forcing(self._p(p), self._p(cp), field_ptrs(state)) == 0

    def turbulence(self, p, tp, state):
        """Turbulence<cUranusModel>::run (k-omega SST, default knobs) on the state in place."""
        assert self.L.oracle_turbulence(self._p(p), self._p(tp), field_ptrs(state)) == 0

    def precipitation(self, p, pp, state):
        """Precipitation<cUranusModel>::run (H2O, NH3, CH4, H2S) on the state in place."""
        assert self.L.oracle_precipitation(self._p(p), self._p(pp), field_ptrs(state)) == 0

    def iteration(self, p, ip, state, iter_n):
        """One iteration (number iter_n, from 1) of the model's loop on the state in place."""
        assert self.L.oracle_iteration(self._p(p), self._p(ip), field_ptrs(state), int(iter_n)) == 0
