"""The hand-written adjoint of the RK4 step (aturan_rk4_adjoint via aturan_b200.autograd) against
(1) torch.autograd through the FP64 torch restatement of the dry step (oracle/dry_ref.py, whose
forward matches the C restatement to 1e-12, tests/test_dry_ref.py), as a full vector-Jacobian
product with random cotangents, and (2) central finite differences of the GPU forward in seeded
random directions of (T, zonal-wind template) on the 41 x 91 x 181 grid, loss = mean T^2 on the
last integrated layer i = im - 2."""
import numpy as np
import pytest
import torch

from aturan_b200 import api, params as P, state as S
from aturan_b200.autograd import DryRK4Step, DryStepper, DRY

pytestmark = pytest.mark.gpu

FIXED = ("p_dyn", "p_stat", "p_baro", "p_b0", "p_bfollow", "nue", "thermalmassflux", "Q_precip")


def make(shape, seed):
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=seed)
    ctx = api.Context(p)
    ctx.upload_state(st)
    return p, st, ctx


@pytest.mark.parametrize("shape,seed", [((12, 20, 33), 61), ((21, 37, 73), 62)])
def test_adjoint_matches_torch_autograd(oracle_lib, shape, seed):
    from oracle.dry_ref import DryStep
    p, st, ctx = make(shape, seed)
    stepper = DryStepper(ctx)
    x = [torch.tensor(st[n], device="cuda", requires_grad=True) for n in DRY]
    y = DryRK4Step.apply(stepper, *x)
    rng = np.random.default_rng(seed)
    ybar = [torch.tensor(rng.standard_normal(p.shape), device="cuda") for _ in DRY]
    g_gpu = torch.autograd.grad(y, x, ybar)
    ctx.close()

    ref = DryStep(p, {n: st[n] for n in FIXED}, oracle_lib)
    xc = [torch.tensor(st[n], requires_grad=True) for n in DRY]
    yc = ref(*xc)
    for a, b in zip(y, yc):                       # the same forward
        assert (a.detach().cpu() - b.detach()).abs().max() <= 1e-11 * b.detach().abs().max()
    g_ref = torch.autograd.grad(yc, xc, [g.cpu() for g in ybar])
    for n, a, b in zip(DRY, g_gpu, g_ref):
        a = a.cpu()
        err = float((a - b).abs().max() / b.abs().max())
        assert err < 1e-9, (n, err)


def template_to_rows(tmpl, p):
    """The 181-point (1 degree) zonal-wind template on the grid's rows: linear in latitude."""
    lat_t = torch.linspace(-90.0, 90.0, tmpl.numel(), dtype=torch.float64, device=tmpl.device)
    _, the = S.coords(p)
    lat = torch.tensor(90.0 - np.degrees(the), device=tmpl.device)
    x = (lat + 90.0) / 180.0 * (tmpl.numel() - 1)
    i0 = torch.clamp(x.floor().long(), 0, tmpl.numel() - 2)
    f = x - i0.to(x.dtype)
    assert lat_t.numel() == tmpl.numel()
    return tmpl[i0] * (1.0 - f) + tmpl[i0 + 1] * f


def test_adjoint_finite_differences_config3():
    p, st, ctx = make((41, 91, 181), 20261206)
    stepper = DryStepper(ctx)
    x0 = [torch.tensor(st[n], device="cuda") for n in DRY]
    tmpl0 = torch.zeros(181, dtype=torch.float64, device="cuda")

    def loss(T, tmpl):
        w = x0[3] + (template_to_rows(tmpl, p) / p.u_0)[None, :, None]
        y = DryRK4Step.apply(stepper, T, x0[1], x0[2], w)
        return (y[0][p.im - 2, 1:-1, :-1] ** 2).mean()

    T = x0[0].clone().requires_grad_(True)
    tm = tmpl0.clone().requires_grad_(True)
    L = loss(T, tm)
    gT, gtm = torch.autograd.grad(L, (T, tm))
    rng = np.random.default_rng(20261206)
    worst = 0.0
    with torch.no_grad():
        for _ in range(32):
            dT = torch.tensor(rng.standard_normal(p.shape), device="cuda") * 1e-3 * float(x0[0].abs().max())
            dtm = torch.tensor(rng.standard_normal(181), device="cuda")          # m/s
            h = 1e-3
            lp = loss(x0[0] + h * dT, tmpl0 + h * dtm)
            lm = loss(x0[0] - h * dT, tmpl0 - h * dtm)
            fd = float((lp - lm) / (2 * h))
            an = float((gT * dT).sum() + (gtm * dtm).sum())
            worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    ctx.close()
    assert worst <= 1e-4, worst


def test_adjoint_requires_tape_and_fp64():
    p = P.default_params(9, 13, 17)
    ctx = api.Context(p)
    ctx.upload_state(S.synthetic_state(p, seed=3))
    t = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(api.AturanError):
        ctx.rk4_adjoint([t.data_ptr()] * 4, [t.data_ptr()] * 4)
    ctx.close()
    pm = P.default_params(9, 13, 17, precision=P.MIXED)
    cm = api.Context(pm)
    with pytest.raises(api.AturanError):
        cm.tape(True)
    cm.close()


# ---- the pressure solve's adjoint: the transposed folded operator (aturan_pressure_solve) ----

def _interior(p, rng):
    a = np.zeros(p.shape)
    a[1:-1, 1:-1, :-1] = rng.standard_normal((p.im - 2, p.jm - 2, p.km - 1))
    return a


@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("kind", [P.PRESS_RB_LINE, P.PRESS_RB_SOR])
def test_pressure_solve_matches_oracle(oracle_lib, kind, transposed):
    p = P.default_params(21, 37, 73)
    rng = np.random.default_rng(71)
    b = _interior(p, rng)
    line = kind == P.PRESS_RB_LINE
    om = 1.0 if line else 1.8
    ctx = api.Context(p)
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc, its, res = ctx.pressure_solve(bd.data_ptr(), xd.data_ptr(), kind, transposed, om, 3000, 1e-10)
    ctx.close()
    x_ref = np.zeros(p.shape)
    rc2, its2, res2 = oracle_lib.solve(p, b, x_ref, transposed, line, om, 3000, 1e-10)
    assert rc == 0 and rc2 == 0 and res <= 1e-10
    assert abs(its - its2) <= (1 if line else 16), (its, its2)
    # the CPU operator's residual of the GPU solution, against the compatible right-hand side
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    x = xd.cpu().numpy()
    Lx = oracle_lib.laplace_apply(p, x, transposed)[I]
    if transposed:
        bc = b[I] - b[I].mean()
    else:
        yi = np.ones(p.im); yi[[1, -2]] = 1.5
        yj = np.ones(p.jm); yj[[1, -2]] = 1.5
        W = (yi[:, None, None] * yj[None, :, None] * np.ones(p.km)[None, None, :])[I]
        bc = b[I] - (W * b[I]).sum() / W.sum()
    rel = np.linalg.norm(bc - Lx) / np.linalg.norm(bc)
    assert rel <= 2e-10, rel


@pytest.mark.parametrize("kind", [P.PRESS_RB_LINE, P.PRESS_RB_SOR])
def test_pressure_adjoint_dot_product(kind):
    """<Lc^-1 s, g> = <s, Lc^-T g> for compatible s, g on the GPU (41 x 91 x 181)."""
    p = P.default_params(41, 91, 181)
    rng = np.random.default_rng(72)
    I = (slice(1, -1), slice(1, -1), slice(0, -1))
    s, g = _interior(p, rng), _interior(p, rng)
    yi = np.ones(p.im); yi[[1, -2]] = 1.5
    yj = np.ones(p.jm); yj[[1, -2]] = 1.5
    W = (yi[:, None, None] * yj[None, :, None] * np.ones(p.km)[None, None, :])[I]
    s[I] -= (W * s[I]).sum() / W.sum()
    g[I] -= g[I].mean()
    om = 1.0 if kind == P.PRESS_RB_LINE else 1.8
    ctx = api.Context(p)
    sd, gd = torch.tensor(s, device="cuda"), torch.tensor(g, device="cuda")
    xd = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    ld = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc1, _, _ = ctx.pressure_solve(sd.data_ptr(), xd.data_ptr(), kind, False, om, 5000, 1e-10)
    rc2, _, _ = ctx.pressure_solve(gd.data_ptr(), ld.data_ptr(), kind, True, om, 5000, 1e-10)
    ctx.close()
    assert rc1 == 0 and rc2 == 0
    x, lam = xd.cpu().numpy(), ld.cpu().numpy()
    lhs, rhs = float((x[I] * g[I]).sum()), float((s[I] * lam[I]).sum())
    assert abs(lhs - rhs) <= 1e-8 * abs(lhs), (lhs, rhs)


# ---- the whole dry step (pressure solve + RK4) and a checkpointed multi-step adjoint ----

def _full_setup(shape, seed, tol=1e-11):
    from aturan_b200.autograd import DryFullStepper
    p, st, ctx = make(shape, seed)
    stepper = DryFullStepper(ctx, kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=200, tol=tol)
    xs = [torch.tensor(st[n], device="cuda") for n in DRY]
    aux = [torch.tensor(st[n], device="cuda") for n in ("aux_u", "aux_v", "aux_w")]
    return p, ctx, stepper, xs, aux


def test_rollout_checkpointing_is_exact():
    """Checkpointing recomputes the same deterministic forward: gradients identical for any
    checkpoint spacing."""
    from aturan_b200.autograd import rollout_gradient
    p, ctx, stepper, xs, aux = _full_setup((21, 37, 73), 81)
    loss = lambda x: (x[0][p.im - 2, 1:-1, :-1] ** 2).mean()
    L1, g1, a1 = rollout_gradient(stepper, xs, aux, 3, 1, loss)
    L3, g3, a3 = rollout_gradient(stepper, xs, aux, 3, 3, loss)
    L2, g2, a2 = rollout_gradient(stepper, xs, aux, 3, 2, loss)
    ctx.close()
    assert float(L1) == float(L3) == float(L2)
    for a, b, c in zip(g1 + a1, g3 + a3, g2 + a2):
        assert torch.equal(a, b) and torch.equal(a, c)


def test_rollout_gradient_finite_differences():
    """Three dry steps with the pressure solve inside (line SOR to 1e-11 from p = 0), checkpoints
    every 2 steps, on the 41 x 91 x 181 grid: the adjoint gradient with respect to the initial
    T, u and aux_u against central differences in 8 seeded directions."""
    from aturan_b200.autograd import rollout_gradient
    p, ctx, stepper, xs, aux = _full_setup((41, 91, 181), 82)
    loss = lambda x: (x[0][p.im - 2, 1:-1, :-1] ** 2).mean() + (x[1][p.im // 2, 1:-1, :-1] ** 2).mean()
    L, gx, ga = rollout_gradient(stepper, xs, aux, 3, 2, loss)

    def run(xs_, aux_):
        x, a = xs_, aux_
        with torch.no_grad():
            for _ in range(3):
                x, a = stepper.forward(x, a)
        return float(loss(x))

    rng = np.random.default_rng(82)
    worst = 0.0
    for _ in range(8):
        dT = torch.tensor(rng.standard_normal(p.shape), device="cuda") * 1e-3 * float(xs[0].abs().max())
        du = torch.tensor(rng.standard_normal(p.shape), device="cuda") * 1e-3 * float(xs[1].abs().max())
        da = torch.tensor(rng.standard_normal(p.shape), device="cuda") * 1e-3 * float(aux[0].abs().max())
        h = 1e-2
        xp = [xs[0] + h * dT, xs[1] + h * du, xs[2], xs[3]]
        xm = [xs[0] - h * dT, xs[1] - h * du, xs[2], xs[3]]
        ap = [aux[0] + h * da, aux[1], aux[2]]
        am = [aux[0] - h * da, aux[1], aux[2]]
        fd = (run(xp, ap) - run(xm, am)) / (2 * h)
        an = float((gx[0] * dT).sum() + (gx[1] * du).sum() + (ga[0] * da).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    ctx.close()
    assert worst <= 1e-4, worst


def test_config4_dry_heating_gradient():
    """A dry form of the 50-step checkpointed adjoint: 41 x 181 x 361, FP64, pressure solved to a
    residual each step, checkpoints every 10 steps, a seeded heating field H(theta, phi) ~ N(0,
    1e-5 K/s) in the temperature tendency; loss = sin(theta)-weighted mean T over |lat| <= 5 deg
    minus over |lat| >= 85 deg (all interior levels and meridians) after 50 steps; its gradient
    with respect to H against central differences in 3 seeded directions. (The moist, mixed form
    is tests/test_gpu_moist_adjoint.py::test_config4_moist_mixed_heating_gradient.)"""
    from aturan_b200.autograd import DryFullStepper, rollout_gradient
    p = P.default_params()
    st = S.synthetic_state(p, seed=20261207)
    for n in ("ch4", "ch4_cloud", "ch4_ice", "h2o", "h2o_cloud", "h2o_ice", "h2s", "h2s_cloud", "h2s_ice",
              "nh3", "nh3_cloud", "nh3_ice", "nh4sh"):
        st[n][:] = 0.0                                  # dry
    ctx = api.Context(p)
    ctx.upload_state(st)
    stepper = DryFullStepper(ctx, kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=100, tol=1e-10)
    xs = [torch.tensor(st[n], device="cuda") for n in DRY]
    aux = [torch.tensor(st[n], device="cuda") for n in ("aux_u", "aux_v", "aux_w")]
    rng = np.random.default_rng(20261207)
    H = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
    _, the = S.coords(p)
    lat = 90.0 - np.degrees(the)
    wj = np.abs(np.sin(the))
    eq = torch.tensor(np.where(np.abs(lat) <= 5.0, wj, 0.0), device="cuda")
    po = torch.tensor(np.where(np.abs(lat) >= 85.0, wj, 0.0), device="cuda")

    def loss(x):
        T = x[0][1:-1, :, :-1]                          # interior levels, every meridian
        return ((T * eq[None, :, None]).sum() / (eq.sum() * T.shape[0] * T.shape[2])
                - (T * po[None, :, None]).sum() / (po.sum() * T.shape[0] * T.shape[2]))

    L, gx, ga, gH = rollout_gradient(stepper, xs, aux, 50, 10, loss, heat=H)

    def run(Hx):
        x, a = xs, aux
        with torch.no_grad():
            for _ in range(50):
                x, a = stepper.forward(x, a, Hx)
        return float(loss(x))

    worst = 0.0
    for _ in range(3):
        d = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
        h = 1.0
        fd = (run(H + h * d) - run(H - h * d)) / (2 * h)
        an = float((gH * d).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    ctx.close()
    assert worst <= 1e-4, worst


@pytest.mark.parametrize("rigid_lid", [1, 0])
def test_pressure_adjoint_directional(rigid_lid):
    """aturan_pressure_adjoint against central differences of the pressure call itself (aux ->
    p_dyn: boundary rows, divergence, compatibility shift, solve, boundary passes), with the rigid
    lid (aux_u = 0 on the radial boundary rows) and without it (cubic extrapolation)."""
    p = P.default_params(21, 37, 73)
    p.rigid_lid = rigid_lid
    st = S.synthetic_state(p, seed=93)
    ctx = api.Context(p)
    ctx.upload_state(st)
    ctx.tape(True)
    aux0 = [torch.tensor(st[n], device="cuda") for n in ("aux_u", "aux_v", "aux_w")]
    zero = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    out = torch.empty(p.shape, dtype=torch.float64, device="cuda")

    def solve(aux):
        torch.cuda.synchronize()
        for n, a in zip(("aux_u", "aux_v", "aux_w"), aux):
            ctx.upload_device(n, a.contiguous().data_ptr())
        ctx.upload_device("p_dyn", zero.data_ptr())
        ctx.pressure(P.PRESS_RB_LINE, omega=1.0, max_sweeps=200, tol=1e-11)
        ctx.download_device("p_dyn", out.data_ptr())
        return out.clone()

    rng = np.random.default_rng(93)
    pbar = torch.tensor(rng.standard_normal(p.shape), device="cuda")
    pbar -= pbar.mean()                                 # the solve leaves p's constant free
    d = [torch.tensor(rng.standard_normal(p.shape), device="cuda") * 1e-2 * float(a.abs().max()) for a in aux0]
    h = 1e-2
    fd = float(((solve([a + h * x for a, x in zip(aux0, d)]) - solve([a - h * x for a, x in zip(aux0, d)]))
                * pbar).sum()) / (2 * h)
    solve(aux0)                                         # tapes the call the adjoint reverses
    abar = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    ctx.pressure_adjoint(pbar.data_ptr(), [a.data_ptr() for a in abar], P.PRESS_RB_LINE, 1.0, 200, 1e-11)
    ctx.close()
    an = float(sum((a * x).sum() for a, x in zip(abar, d)))
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
