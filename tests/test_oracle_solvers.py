"""The oracle's to-residual Poisson solvers (point and line red-black SOR with the column-uniform
correction). The reference has no converged solve to compare with (it sweeps a fixed count), so
these are pinned to the reference through its own sweep: a converged solution must be a fixed
point of PressureSolver<cUranusModel>::run's red-black sweep (PressureSolver.h:318-495), which the
oracle reproduces bit for bit (tests/test_golden.py, case pressure_rb3)."""
import numpy as np
import pytest

from aturan_b200 import params as P, state as S


def case(shape=(21, 37, 73), seed=40):
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=seed)
    st["p_dyn"][:] = 0.0
    return p, st


def interior_centered(a):
    x = a[1:-1, 1:-1, :-1]
    return x - x.mean()


def test_point_and_line_reach_tolerance_and_agree(oracle_lib):
    p, st = case()
    a, b = S.copy_state(st), S.copy_state(st)
    rc, sweeps, res = oracle_lib.pressure_sor(p, a, 1.8, 3000, 1e-10, 16)
    assert rc == 0 and res <= 1e-10 and sweeps < 3000
    rc, its, res = oracle_lib.pressure_line(p, b, 1.0, 200, 1e-10)
    assert rc == 0 and res <= 1e-10 and its <= 10, its
    # the all-Neumann equation fixes p up to a constant: compare without it
    da, db = interior_centered(a["p_dyn"]), interior_centered(b["p_dyn"])
    assert np.abs(da - db).max() <= 1e-8 * np.abs(db).max()


def test_converged_solution_is_a_fixed_point_of_the_reference_sweep(oracle_lib):
    p, st = case(seed=41)
    rc, its, res = oracle_lib.pressure_line(p, st, 1.0, 200, 1e-11)
    assert rc == 0
    moved = S.copy_state(st)
    oracle_lib.pressure_rb(p, moved, 1)
    # what is left is the compatibility shift of the source (a few 1e-5 of it) divided by the
    # operator's diagonal
    scale = np.abs(st["p_dyn"]).max()
    assert np.abs(moved["p_dyn"] - st["p_dyn"]).max() <= 1e-7 * scale


def test_cap_reports_not_converged(oracle_lib):
    p, st = case(seed=42)
    rc, its, res = oracle_lib.pressure_line(p, st, 1.0, 1, 1e-14)
    assert rc == 1 and its == 1 and res > 1e-14
    p, st = case(seed=42)
    rc, sweeps, res = oracle_lib.pressure_sor(p, st, 1.8, 5, 1e-14, 16)
    assert rc == 1 and sweeps == 5


@pytest.mark.parametrize("kind", [P.PRESS_RB_SOR, P.PRESS_RB_LINE])
def test_step_with_converged_solvers_agree(oracle_lib, kind):
    """The whole step with either solver (their solutions differ only by the constant, which no
    gradient sees)."""
    p, st = case(shape=(12, 20, 33), seed=43)
    ref = S.copy_state(st)
    oracle_lib.step(p, ref, P.PRESS_RB_LINE, 1.0, 100, 1e-11)
    got = S.copy_state(st)
    omega = 1.8 if kind == P.PRESS_RB_SOR else 1.0
    oracle_lib.step(p, got, kind, omega, 5000, 1e-11)
    for n in ("t", "u", "v", "w"):
        scale = np.abs(ref[n]).max()
        assert np.abs(got[n] - ref[n]).max() <= 1e-9 * scale, n


# ---- the transposed operator and its solve (the pressure solve's adjoint) ----

def _interior_random(p, rng):
    a = np.zeros(p.shape)
    a[1:-1, 1:-1, :-1] = rng.standard_normal((p.im - 2, p.jm - 2, p.km - 1))
    return a


def test_transposed_operator_is_the_transpose(oracle_lib):
    p = P.default_params(13, 21, 33)
    rng = np.random.default_rng(11)
    x, y = _interior_random(p, rng), _interior_random(p, rng)
    a = float((oracle_lib.laplace_apply(p, x) * y).sum())
    b = float((x * oracle_lib.laplace_apply(p, y, transposed=True)).sum())
    assert abs(a - b) <= 1e-13 * abs(a)


@pytest.mark.parametrize("line", [True, False])
def test_adjoint_solve_dot_product(oracle_lib, line):
    """<Lc^-1 s, g> = <s, Lc^-T g> for compatible s and g: the transposed solve is the adjoint of
    the forward solve (the free constant of p and the free multiple of y y of the adjoint solution
    drop out against the compatible partners)."""
    p = P.default_params(21, 37, 73)
    rng = np.random.default_rng(12)
    s, g = _interior_random(p, rng), _interior_random(p, rng)
    x, lam = np.zeros(p.shape), np.zeros(p.shape)
    om = 1.0 if line else 1.8
    rc1, it1, _ = oracle_lib.solve(p, s, x, False, line, om, 3000, 1e-10)
    rc2, it2, _ = oracle_lib.solve(p, g, lam, True, line, om, 3000, 1e-10)
    assert rc1 == 0 and rc2 == 0
    assert abs(it1 - it2) <= (1 if line else 16)           # same convergence for both systems
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    yi = np.ones(p.im); yi[[1, -2]] = 1.5
    yj = np.ones(p.jm); yj[[1, -2]] = 1.5
    W = (yi[:, None, None] * yj[None, :, None] * np.ones(p.km)[None, None, :])[I]
    sc = s[I] - (W * s[I]).sum() / W.sum()
    gc = g[I] - g[I].mean()
    lhs, rhs = float((x[I] * gc).sum()), float((sc * lam[I]).sum())
    assert abs(lhs - rhs) <= 1e-8 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("shape,rigid", [((12, 20, 33), 1), ((41, 91, 181), 1), ((9, 13, 17), 0)])
def test_poisson_source_is_the_shared_solvers(oracle_lib, shape, rigid):
    """The isolated Poisson solve's right-hand side (aturan_b200.state.poisson_source: the
    divergence of PressureSolver.h:448-487 after prepareProjectionBoundaries) is the oracle's
    pressure source, which is pinned to the compiled reference, bit for bit."""
    from aturan_b200 import fields as F
    p = P.default_params(*shape)
    p.rigid_lid = rigid
    u, v, w = S.poisson_velocity(p, seed=5)
    src = S.poisson_source(p, u, v, w)
    st = {n: np.zeros(p.shape) for n in F.PROJECTION}
    st["aux_u"], st["aux_v"], st["aux_w"] = u.copy(), v.copy(), w.copy()
    assert np.array_equal(src, oracle_lib.pressure_source(p, st))


def test_poisson_velocity_is_smoothed_and_periodic():
    p = P.default_params(12, 20, 33)
    u, v, w = S.poisson_velocity(p, seed=7)
    for a in (u, v, w):
        assert a.shape == p.shape and np.array_equal(a[..., -1], a[..., 0])
        # 3 passes of a 3x3x3 mean shrink unit-variance noise well below 1
        assert 0.02 < a.std() < 0.3
    u2, _, _ = S.poisson_velocity(p, seed=7)
    assert np.array_equal(u, u2)
