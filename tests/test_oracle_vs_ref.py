"""The oracle restatement against the compiled reference (oracle/_ref), bit for bit.

The reference is the unmodified C++ compiled from its own sources; its model is initialised
once (Run() with nm = 0). Each test loads the same state into both, runs the reference routine
and the oracle function, and requires every output FP64 value to be identical. Skipped where the
reference has not been built (it needs the reference tree).
"""
import numpy as np
import pytest

from aturan_b200 import fields as F, params as P, state as S

pytestmark = pytest.mark.slow


@pytest.fixture(scope="module")
def base_state(ref_model):
    return ref_model.state()


def assert_same(a, b, names):
    for n in names:
        x, y = a[n], b[n]
        ne = np.count_nonzero(x != y)
        assert ne == 0, f"{n}: {ne} cells differ, max |d| = {np.abs(x - y).max()}"


def test_params_are_the_references(ref_model):
    p, pr = P.default_params(), P.params_from_ref(ref_model)
    for name, _ in P.Params._fields_:
        if name in ("gas", "reserved_i", "reserved_d"):
            continue
        assert getattr(p, name) == getattr(pr, name), name
    for n in range(4):
        for name, _ in P.Gas._fields_:
            assert getattr(p.gas[n], name) == getattr(pr.gas[n], name), (n, name)


def test_coordinates(ref_model):
    rad, the = ref_model.coords()
    r2, t2 = S.coords(P.default_params())
    assert np.array_equal(rad, r2) and np.array_equal(the, t2)


def test_cp_lapse(ref_model, oracle_lib):
    p = P.default_params()
    for T in [1.0, 5.0, 5.25, 49.3, 76.4, 150.0, 233.7, 1499.75, 1500.0, 2500.0]:
        assert ref_model.cp_lapse(T) == oracle_lib.cp_lapse(p, T), T


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_satadj_sequence(ref_model, oracle_lib, base_state, source):
    p = P.default_params()
    st = S.perturb(base_state, p, seed=11) if source == "reference_init" else S.synthetic_state(p, seed=12)
    ref_model.load(st)
    for g, gas in enumerate(F.GASES):
        ref_model.satadj(g)
        oracle_lib.satadj(p, st, g)
        names = ["t"] + list(F.GAS_FIELDS[gas])
        assert_same(ref_model.state(names), st, names)


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_rk4(ref_model, oracle_lib, base_state, source):
    p = P.default_params()
    st = S.perturb(base_state, p, seed=21) if source == "reference_init" else S.synthetic_state(p, seed=22)
    ref_model.load(st)
    ref_model.rk4()
    lev = oracle_lib.rk4(p, st)
    names = F.PROGNOSTIC + ["p_hydro", "p_bfollow"] + F.PROJECTION
    assert_same(ref_model.state(names), st, names)
    assert np.array_equal(ref_model.get("buoy_ref_level"), lev)


def test_pressure_gs(ref_model, oracle_lib, base_state):
    p = P.default_params()
    st = S.perturb(base_state, p, seed=31)
    ref_model.load(st)
    ref_model.pressure_gs()
    oracle_lib.pressure_gs(p, st)
    names = ["p_dyn", "aux_u", "aux_v", "aux_w"]
    assert_same(ref_model.state(names), st, names)


@pytest.mark.parametrize("sweeps", [1, 4])
def test_pressure_rb(ref_model, oracle_lib, base_state, sweeps):
    p = P.default_params()
    st = S.perturb(base_state, p, seed=40 + sweeps)
    ref_model.load(st)
    ref_model.pressure_rb(sweeps)
    oracle_lib.pressure_rb(p, st, sweeps)
    names = ["p_dyn"] + F.PROJECTION
    assert_same(ref_model.state(names), st, names)


def test_full_step(ref_model, oracle_lib, base_state):
    """cUranusModel.cpp:967-1123, in-scope calls: GS pressure, SatAdj x4, n-copy sync, RK4."""
    p = P.default_params()
    st = S.perturb(base_state, p, seed=51)
    ref_model.load(st)
    ref_model.pressure_gs()
    for g in range(4):
        ref_model.satadj(g)
    ref_model.sync_ncopies()
    ref_model.rk4()
    oracle_lib.step(p, st, P.PRESS_GS_LEX)
    names = F.PROGNOSTIC + F.NCOPIES + ["p_dyn", "p_hydro", "p_bfollow"] + F.PROJECTION
    assert_same(ref_model.state(names), st, names)


def test_post_step(ref_model, oracle_lib, base_state):
    """The passes after RK4 with the reference's default knobs (cUranusModel.cpp:1218-1248): t
    filter, boundary passes (with the species floor and the lid v, w) and the species clamp; every
    written value identical, the clamp's counts equal and its sums equal up to the order of the
    reference's OpenMP reduction."""
    from tests.post_case import KNOB_SETS, POST_FIELDS, post_state
    p = P.default_params()
    st = post_state(S.perturb(base_state, p, seed=41), p, seed=42)
    pp = KNOB_SETS["defaults"][1]()
    assert bool(pp.lid_vw == 2) == ref_model.geo_balance()
    ref_model.load(st)
    ra, rc = ref_model.post_step(pp)
    oa, oc = oracle_lib.post_step(p, st, pp)
    assert_same(ref_model.state(POST_FIELDS), st, POST_FIELDS)
    assert np.array_equal(rc, oc) and rc.sum() > 0
    assert np.allclose(ra, oa, rtol=1e-12, atol=0.0)


POST_KNOBS = ["no_geo_balance_forms", "cubic_lid_open_phi"]
PHYSICS_KNOBS = ["chem_minus_open_phi", "turb_no_curv_open_phi", "precip_uncoupled", "precip_no_h2s"]


@pytest.fixture(scope="module")
def knob_children():
    """Every knob set's child process started at once, each with its share of the host's cores
    (a child spends most of its time in the reference's serial initialisation), and waited for
    together: {(child script, knob set): (return code, stdout, stderr)}."""
    import os
    import subprocess
    import sys
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference (oracle/_ref) not present")
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    from tests.post_case import KNOB_SETS as POST_SETS
    from _physics_knobs_child import KNOB_SETS as PHYS_SETS
    jobs = [("_post_knobs_child.py", k, POST_SETS[k][0]) for k in POST_KNOBS]
    jobs += [("_physics_knobs_child.py", k, PHYS_SETS[k][0]) for k in PHYSICS_KNOBS]
    threads = str(max(1, (os.cpu_count() or 1) // len(jobs)))
    procs = {}
    for script, k, knob_env in jobs:
        env = dict(os.environ, **knob_env)
        env["OMP_NUM_THREADS"] = threads
        procs[(script, k)] = subprocess.Popen([sys.executable, os.path.join(here, script), k], env=env,
                                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    out = {}
    for key, pr in procs.items():
        try:
            so, se = pr.communicate(timeout=1800)
        except subprocess.TimeoutExpired:
            pr.kill()
            so, se = pr.communicate()
        out[key] = (pr.returncode, so, se)
    return out


@pytest.mark.parametrize("knobs", POST_KNOBS)
def test_post_step_knob_sets(knobs, knob_children):
    """Other knob values (forms, taper, lid, floor, filters, an open phi seam): the reference reads
    them from its environment once per process, so each set runs in a child process with that
    environment; the child requires bit equality as above."""
    rc, so, se = knob_children[("_post_knobs_child.py", knobs)]
    assert rc == 0 and "OK" in so, so[-2000:] + se[-2000:]


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_mca(ref_model, oracle_lib, base_state, source):
    """The moist convective adjustment (ConvectiveAdjustment.h:402-849) as the model's loop calls
    it, default knobs: every value it writes (t, the twelve condensables, nh4sh) identical. Both
    states have most columns unstable somewhere, so segments form, mix, settle and grow."""
    p = P.default_params()
    st = S.perturb(base_state, p, seed=71) if source == "reference_init" else S.synthetic_state(p, seed=72)
    names = ["t", "nh4sh"] + [n for g in F.GASES for n in F.GAS_FIELDS[g]]
    before = {n: st[n].copy() for n in names}
    ref_model.load(st)
    ref_model.mca()
    oracle_lib.mca(p, st)
    assert_same(ref_model.state(names), st, names)
    assert np.count_nonzero(st["t"] != before["t"]) > 100000


def test_chem_params_are_the_references(ref_model):
    cp, cr = P.default_chem_params(), P.chem_params_from_ref(ref_model)
    for name, _ in P.ChemParams._fields_:
        if name in ("reserved_i", "reserved_d"):
            continue
        assert getattr(cp, name) == getattr(cr, name), name
    assert ref_model.chem_scalar("coord_stretching") == 0.0


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_nh4sh_equilibrium(ref_model, oracle_lib, base_state, source):
    """EquilibriumNH4SH("loop") (ChemistryUran.h:210-275): t, nh3, h2s, nh4sh identical in every
    cell; NH4SH both forms and decomposes in many cells."""
    from tests.chem_case import EQ_OUT, chem_state
    p, cp = P.default_params(), P.default_chem_params()
    base = S.perturb(base_state, p, seed=81) if source == "reference_init" else S.synthetic_state(p, seed=82)
    st = chem_state(base, p, seed=83)
    ref_model.load(st)
    ref_model.chem_eq()
    nf, nd = oracle_lib.nh4sh_eq(p, cp, st)
    assert_same(ref_model.state(EQ_OUT), st, EQ_OUT)
    assert nf > 10000 and nd > 10000, (nf, nd)


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_chem_forcing(ref_model, oracle_lib, base_state, source):
    """DiffMassFluxUran, the filters, ChemMassRateUran, FluxLimiterNH4SH and the filters
    (cUranusModel.cpp:1074-1087), on persistent fields whose boundary rows hold seeded values:
    every value written identical."""
    from tests.chem_case import FORCING_OUT, chem_state
    p, cp = P.default_params(), P.default_chem_params()
    base = S.perturb(base_state, p, seed=84) if source == "reference_init" else S.synthetic_state(p, seed=85)
    st = chem_state(base, p, seed=86)
    ref_model.load(st)
    ref_model.chem_forcing()
    oracle_lib.chem_forcing(p, cp, st)
    assert_same(ref_model.state(FORCING_OUT), st, FORCING_OUT)
    assert np.count_nonzero(st["fluxlim_nh4sh"]) > 100000


def test_turb_params_are_the_references(ref_model):
    tp, tr = P.default_turb_params(), P.turb_params_from_ref(ref_model)
    for name, _ in P.TurbParams._fields_:
        if name == "reserved_d":
            continue
        assert getattr(tp, name) == getattr(tr, name), name
    assert ref_model.turb_scalar("active") == 1.0 and ref_model.turb_scalar("bc_turb_active") == 0.0


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_turbulence(ref_model, oracle_lib, base_state, source):
    """Turbulence<cUranusModel>::run (k-omega SST, default knobs): every value it writes (tke, dis,
    nue, prod, tke_source, dis_source, and tken, disn at the seam and the edges) identical."""
    from tests.turb_case import TURB_OUT, turb_state
    p, tp = P.default_params(), P.default_turb_params()
    base = S.perturb(base_state, p, seed=91) if source == "reference_init" else S.synthetic_state(p, seed=92)
    st = turb_state(base, p, seed=93)
    ref_model.load(st)
    ref_model.turbulence()
    oracle_lib.turbulence(p, tp, st)
    assert_same(ref_model.state(TURB_OUT), st, TURB_OUT)
    assert np.count_nonzero(st["prod"] > 0) > 100000


def test_precip_params_are_the_references(ref_model):
    pp, pr = P.default_precip_params(), P.precip_params_from_ref(ref_model)
    for name in ("coupling", "h2s", "rate_scale"):
        assert getattr(pp, name) == getattr(pr, name), name


@pytest.mark.parametrize("source", ["reference_init", "synthetic"])
def test_precipitation(ref_model, oracle_lib, base_state, source):
    """Precipitation<cUranusModel>::run (H2O, NH3, CH4, H2S, default knobs): Q_precip and the twelve
    S_precip_* identical in every cell; at least two species precipitate in many cells (H2O, whose
    ice-autoconversion band lies above the domain's temperatures, does not)."""
    from tests.precip_case import PRECIP_OUT, precip_state
    p, pp = P.default_params(), P.default_precip_params()
    base = S.perturb(base_state, p, seed=95) if source == "reference_init" else S.synthetic_state(p, seed=96)
    st = precip_state(base, p, seed=97)
    ref_model.load(st)
    ref_model.precipitation()
    oracle_lib.precipitation(p, pp, st)
    assert_same(ref_model.state(PRECIP_OUT), st, PRECIP_OUT)
    active = [g for g in ("h2o", "nh3", "ch4", "h2s")
              if np.count_nonzero(st["S_precip_" + g + "_cloud"]) + np.count_nonzero(st["S_precip_" + g + "_ice"]) > 1000]
    assert len(active) >= 2, active
    assert np.count_nonzero(st["Q_precip"]) > 1000


@pytest.mark.parametrize("knobs", PHYSICS_KNOBS)
def test_physics_knob_sets(knobs, knob_children):
    """Other knob values of the chemistry (massflux = -difflux, the open phi seam), the turbulence
    closure (no curvature terms, the open seam) and the precipitation (the depletion written into the
    condensate fields; no H2S and another rate scale), each in a child process with that environment;
    the child requires bit equality of every written value."""
    rc, so, se = knob_children[("_physics_knobs_child.py", knobs)]
    assert rc == 0 and "OK" in so, so[-2000:] + se[-2000:]


def test_reference_loop(ref_model, oracle_lib, base_state, tmp_path):
    """The reference's own loop: Run() with 4 iterations after its initialisation (in a child
    process, a fresh model) against the oracle's iteration applied 4 times to the initialised state
    (iterations 1 and 3 odd: RK4 onward; 2 and 4 even: the full sequence). Every field the loop
    carries is identical, which pins the iteration's composition and order as well as its parts."""
    import os
    import subprocess
    import sys
    p, ip = P.default_params(), P.default_iter_params()
    n = 4
    out = tmp_path / "loop.npz"
    child = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_loop_child.py")
    r = subprocess.run([sys.executable, child, str(n), str(out)], capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    got = dict(np.load(out))
    st = {k: np.array(v, copy=True) for k, v in base_state.items()}
    for it in range(1, n + 1):
        oracle_lib.iteration(p, ip, st, it)
    names = [m for m in F.NAMES if m not in F.PROJECTION]
    bad = {m: int(np.count_nonzero(got[m] != st[m])) for m in names if not np.array_equal(got[m], st[m])}
    assert not bad, bad
    assert not np.array_equal(got["t"], base_state["t"])
