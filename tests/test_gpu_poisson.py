"""The isolated Poisson solve (the benchmark's config of the pressure equation alone): the source is
the shared solver's divergence of a seeded smoothed random velocity field
(aturan_b200.state.poisson_source, bit-equal to the oracle's source, tests/test_oracle_solvers.py),
solved to a relative residual through aturan_pressure_solve in an FP64 context (FP64 sweeps) and in
a mixed context (FP32 sweeps inside FP64 iterative refinement).

The reference has no solve to a residual; the pins are the CPU restatement's iteration counts and
the CPU operator's own residual of the GPU solution (oracle_laplace_apply), which must meet the
tolerance whatever precision the sweeps ran in."""
import numpy as np
import pytest

from aturan_b200 import params as P, state as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _compatible(p, b):
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    yi = np.ones(p.im); yi[[1, -2]] = 1.5
    yj = np.ones(p.jm); yj[[1, -2]] = 1.5
    W = (yi[:, None, None] * yj[None, :, None] * np.ones(p.km)[None, None, :])[I]
    return b[I] - (W * b[I]).sum() / W.sum()


def _solve(p, prec, b, kind, omega, tol, cap):
    from aturan_b200 import api
    q = P.default_params(p.im, p.jm, p.km, precision=prec)
    ctx = api.Context(q)
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc, its, res = ctx.pressure_solve(bd.data_ptr(), xd.data_ptr(), kind, False, omega, cap, tol)
    ctx.close()
    return rc, its, res, xd.cpu().numpy()


@pytest.fixture(scope="module")
def case():
    p = P.default_params(41, 91, 181)
    u, v, w = S.poisson_velocity(p, seed=20261205)
    return p, S.poisson_source(p, u, v, w)


@pytest.mark.parametrize("kind,omega", [(P.PRESS_RB_LINE, 1.0), (P.PRESS_RB_SOR, 1.8), (P.PRESS_RB_SOR, 1.5)])
def test_fp64_solve_matches_the_cpu_restatement(oracle_lib, case, kind, omega):
    p, b = case
    line = kind == P.PRESS_RB_LINE
    rc, its, res, x = _solve(p, P.FP64, b, kind, omega, 1e-8, 6000)
    x_ref = np.zeros(p.shape)
    rc2, its2, res2 = oracle_lib.solve(p, b, x_ref, False, line, omega, 6000, 1e-8)
    assert rc == 0 and rc2 == 0 and res <= 1e-8
    assert abs(its - its2) <= (1 if line else 16), (its, its2)
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    bc = _compatible(p, b)
    rel = np.linalg.norm(bc - oracle_lib.laplace_apply(p, x)[I]) / np.linalg.norm(bc)
    assert rel <= 2e-8, rel
    d = x[I] - x_ref[I]
    d -= d.mean()
    xr = x_ref[I] - x_ref[I].mean()
    assert np.abs(d).max() <= 1e-6 * np.abs(xr).max()


@pytest.mark.parametrize("kind,omega", [(P.PRESS_RB_LINE, 1.0), (P.PRESS_RB_SOR, 1.8)])
def test_mixed_solve_reaches_the_fp64_residual(oracle_lib, case, kind, omega):
    """FP32 sweeps inside FP64 refinement: the FP64 residual (checked here with the CPU operator)
    still reaches 1e-8, and the solution is the FP64 solve's to the tolerance's size."""
    p, b = case
    rc, its, res, x = _solve(p, P.MIXED, b, kind, omega, 1e-8, 6000)
    assert rc == 0 and res <= 1e-8, (rc, res)
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    bc = _compatible(p, b)
    rel = np.linalg.norm(bc - oracle_lib.laplace_apply(p, x)[I]) / np.linalg.norm(bc)
    assert rel <= 2e-8, rel
    rc64, _, _, x64 = _solve(p, P.FP64, b, kind, omega, 1e-8, 6000)
    assert rc64 == 0
    d = x[I] - x64[I]
    d -= d.mean()
    xr = x64[I] - x64[I].mean()
    assert np.abs(d).max() <= 1e-6 * np.abs(xr).max()


def test_mixed_transposed_solve(oracle_lib):
    """The transposed system in a mixed context: Lc^T x = b (b made zero-mean) to 1e-8, checked
    with the CPU's transposed operator."""
    p = P.default_params(21, 37, 73)
    rng = np.random.default_rng(73)
    b = np.zeros(p.shape)
    b[1:-1, 1:-1, :-1] = rng.standard_normal((p.im - 2, p.jm - 2, p.km - 1))
    from aturan_b200 import api
    ctx = api.Context(P.default_params(21, 37, 73, precision=P.MIXED))
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc, its, res = ctx.pressure_solve(bd.data_ptr(), xd.data_ptr(), P.PRESS_RB_LINE, True, 1.0, 400, 1e-8)
    ctx.close()
    assert rc == 0 and res <= 1e-8
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    bc = b[I] - b[I].mean()
    x = xd.cpu().numpy()
    rel = np.linalg.norm(bc - oracle_lib.laplace_apply(p, x, True)[I]) / np.linalg.norm(bc)
    assert rel <= 2e-8, rel
