"""The moist step's adjoint (aturan_tape(ctx, 2), aturan_moist_adjoint, MoistFullStepper):
(1) the RK4 step's adjoint over t, u, v, w and the twelve condensable species against
torch.autograd through the torch FP64 restatement (oracle/dry_ref.py MoistRK4Step, whose forward
matches the C restatement to 1e-12: tests/test_dry_ref.py); (2) the saturation adjustment's
implicit adjoint against central differences of the oracle's adjustment taken to its root
(aturan_params.satadj_stop_tol = 1e-13), cell by cell; (3) a three-step moist trajectory with the
pressure solve inside against central differences of the GPU forward with the adjustment taken to
its root."""
import numpy as np
import pytest
import torch

from aturan_b200 import api, params as P, state as S
from aturan_b200.autograd import MOIST

pytestmark = pytest.mark.gpu

SPECIES = MOIST[4:]
FIXED = ("p_dyn", "p_stat", "p_baro", "p_b0", "p_bfollow", "nue", "thermalmassflux", "Q_precip") \
    + tuple("S_precip_" + n for n in SPECIES) + ("massflux_h2s", "massflux_nh3")


def _ptrs(ts):
    return [t.data_ptr() for t in ts]


@pytest.mark.parametrize("shape,seed", [((12, 20, 33), 63), ((21, 37, 73), 64)])
def test_moist_rk4_adjoint_matches_torch_autograd(oracle_lib, shape, seed):
    """No adjustment in the taped step: aturan_moist_adjoint is the RK4 step's adjoint over the
    sixteen fields; a full vector-Jacobian product with random cotangents on every field."""
    from oracle.dry_ref import MoistRK4Step
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=seed)
    ctx = api.Context(p)
    ctx.upload_state(st)
    ctx.tape(2)
    ctx.restore_ncopies(1.0)                      # the start-of-step copies are the state
    ctx.rk4_step()
    rng = np.random.default_rng(seed)
    ybar = [torch.tensor(rng.standard_normal(p.shape), device="cuda") for _ in MOIST]
    xbar = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in MOIST]
    torch.cuda.synchronize()
    ctx.moist_adjoint(_ptrs(ybar), None, _ptrs(xbar), None)
    out = ctx.download_state(list(MOIST))
    ctx.close()

    ref = MoistRK4Step(p, {n: st[n] for n in FIXED}, oracle_lib)
    xc = [torch.tensor(st[n], requires_grad=True) for n in MOIST]
    yc = ref(*xc)
    for n, b in zip(MOIST, yc):                   # the same forward
        b = b.detach().numpy()
        assert np.abs(out[n] - b).max() <= 1e-11 * max(np.abs(b).max(), 1e-300), n
    g_ref = torch.autograd.grad(yc, xc, [g.cpu() for g in ybar])
    for n, a, b in zip(MOIST, xbar, g_ref):
        a = a.cpu()
        err = float((a - b).abs().max() / b.abs().max())
        assert err < 1e-9, (n, err)


def _oracle_adjust(oracle_lib, p, st):
    s = S.copy_state(st)
    for g in range(4):
        oracle_lib.satadj(p, s, g)
    return s


def test_satadj_implicit_adjoint_matches_finite_differences(oracle_lib):
    """The adjustment alone: a taped step whose RK4 has dt = 1e-20 (the identity to rounding, so
    its adjoint passes the cotangents through) after an adjustment of all four gases with the
    stopping test at 1e-13 (the passes reach the root the implicit adjoint differentiates). Per
    cell, the directional derivative sum_f ybar_f dF_f(x; d) from central differences of the
    oracle's adjustment against sum_f xbar_f d_f, in three seeded directions (each field perturbed
    in proportion to its own magnitude, so no value changes sign); the cells whose branch (the
    entry decision or the phases present at the root) changes within the step, where the
    derivative jumps, are counted and allowed up to 1 %."""
    shape = (12, 20, 33)
    p = P.default_params(*shape)
    p.dt = 1.0e-20
    p.satadj_stop_tol = 1.0e-13
    st = S.synthetic_state(P.default_params(*shape), seed=65)
    ctx = api.Context(p)
    ctx.upload_state(st)
    ctx.tape(2)
    ctx.restore_ncopies(1.0)
    ctx.satadj(0xF, count=False)
    ctx.sync_ncopies()
    ctx.rk4_step()
    rng = np.random.default_rng(65)
    names = ("t",) + SPECIES
    ybar = [torch.tensor(rng.standard_normal(p.shape) if n in names else np.zeros(p.shape), device="cuda")
            for n in MOIST]
    xbar = [torch.empty(p.shape, dtype=torch.float64, device="cuda") for _ in MOIST]
    torch.cuda.synchronize()
    ctx.moist_adjoint(_ptrs(ybar), None, _ptrs(xbar), None)
    gpu_after = ctx.download_state(list(names))
    ctx.close()
    yb = {n: g.cpu().numpy() for n, g in zip(MOIST, ybar)}
    xb = {n: g.cpu().numpy() for n, g in zip(MOIST, xbar)}
    base = _oracle_adjust(oracle_lib, p, st)
    for n in names:                                   # the same forward (CUDA's exp / log aside)
        gas = [m for m in names if m.split("_")[0] == n.split("_")[0]]
        scale = max(max(np.abs(base[m]).max() for m in gas), 1e-300)
        assert np.abs(gpu_after[n] - base[n]).max() <= 1e-9 * scale, n
    h = 1.0e-6
    for rep in range(3):
        d = {n: rng.standard_normal(p.shape) * np.abs(st[n]) for n in names}
        sp, sm = S.copy_state(st), S.copy_state(st)
        for n in names:
            sp[n] = st[n] + h * d[n]
            sm[n] = st[n] - h * d[n]
        fp, fm = _oracle_adjust(oracle_lib, p, sp), _oracle_adjust(oracle_lib, p, sm)
        fd = sum(yb[n] * (fp[n] - fm[n]) / (2 * h) for n in names)
        ad = sum(xb[n] * d[n] for n in names)
        scale = sum(np.abs(yb[n] * (fp[n] - fm[n]) / (2 * h)) + np.abs(xb[n] * d[n]) for n in names)
        bad = np.abs(fd - ad) > 1e-5 * scale + 1e-300
        assert bad.mean() <= 0.01, (rep, int(bad.sum()), bad.size)
        # where it agrees, it agrees closely, and the changed cells are most of the grid
        good = ~bad
        assert np.all(np.abs(fd - ad)[good] <= 1e-5 * scale[good] + 1e-300)
    changed = sum(np.abs(base[n] - st[n]) > 0 for n in names) > 0
    assert changed.mean() > 0.3


def _moist_setup(shape, seed, stop_tol=None):
    from aturan_b200.autograd import MoistFullStepper
    p = P.default_params(*shape)
    if stop_tol is not None:
        p.satadj_stop_tol = stop_tol
    st = S.synthetic_state(P.default_params(*shape), seed=seed)
    ctx = api.Context(p)
    ctx.upload_state(st)
    stepper = MoistFullStepper(ctx, kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=200, tol=1e-11)
    xs = [torch.tensor(st[n], device="cuda") for n in MOIST]
    aux = [torch.tensor(st[n], device="cuda") for n in ("aux_u", "aux_v", "aux_w")]
    return p, ctx, stepper, xs, aux


def test_moist_rollout_checkpointing_is_exact():
    from aturan_b200.autograd import rollout_gradient
    p, ctx, stepper, xs, aux = _moist_setup((21, 37, 73), 83)
    loss = lambda x: (x[0][p.im - 2, 1:-1, :-1] ** 2).mean()
    L1, g1, a1 = rollout_gradient(stepper, xs, aux, 3, 1, loss)
    L3, g3, a3 = rollout_gradient(stepper, xs, aux, 3, 3, loss)
    ctx.close()
    assert float(L1) == float(L3)
    for a, b in zip(g1 + a1, g3 + a3):
        assert torch.equal(a, b)


def test_moist_rollout_heating_gradient_finite_differences():
    """Three moist steps (pressure to 1e-11, the adjustment of four gases taken to its root, RK4)
    on 21 x 37 x 73 with a seeded heating field; loss = mean T of the interior after the last step
    minus mean T at mid-depth; gradient with respect to the heating and to the initial H2O vapour
    against central differences in 4 seeded directions."""
    from aturan_b200.autograd import rollout_gradient
    p, ctx, stepper, xs, aux = _moist_setup((21, 37, 73), 84, stop_tol=1e-13)
    rng = np.random.default_rng(84)
    H = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
    loss = lambda x: x[0][1:-1, 1:-1, :-1].mean() - x[0][p.im // 2, 1:-1, :-1].mean()
    L, gx, ga, gH = rollout_gradient(stepper, xs, aux, 3, 2, loss, heat=H)
    iv = MOIST.index("h2o")

    def run(Hx, xs_):
        x, a = xs_, aux
        with torch.no_grad():
            for _ in range(3):
                x, a = stepper.forward(x, a, Hx)
        return float(loss(x))

    worst = 0.0
    for _ in range(4):
        dH = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
        dv = torch.tensor(rng.standard_normal(p.shape), device="cuda") * xs[iv].abs() * 1e-3
        h = 1e-3
        xp = list(xs); xm = list(xs)
        xp[iv] = xs[iv] + h * dv
        xm[iv] = xs[iv] - h * dv
        fd = (run(H + h * dH, xp) - run(H - h * dH, xm)) / (2 * h)
        an = float((gH * dH).sum() + (gx[iv] * dv).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    ctx.close()
    assert worst <= 1e-4, worst


def test_moist_adjoint_needs_the_moist_tape():
    p = P.default_params(9, 13, 17)
    ctx = api.Context(p)
    ctx.upload_state(S.synthetic_state(p, seed=4))
    ctx.tape(True)
    ctx.rk4_step()
    t = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(api.AturanError):
        ctx.moist_adjoint([t.data_ptr()] * 16, None, [t.data_ptr()] * 16, None)
    ctx.tape(2)
    ctx.rk4_step()
    with pytest.raises(api.AturanError):
        ctx.rk4_adjoint([t.data_ptr()] * 4, [t.data_ptr()] * 4)
    ctx.close()


def test_config4_moist_mixed_heating_gradient():
    """The 50-step checkpointed adjoint with moist physics: 41 x 181 x 361, the synthetic state's
    four condensables, the pressure solved to a residual each step, the adjustment of four gases,
    checkpoints every 10 steps, a seeded heating field H(theta, phi) ~ N(0, 1e-5 K/s); loss = the
    sin(theta)-weighted mean T over |lat| <= 5 deg minus over |lat| >= 85 deg after step 50.
      * FP64 with the adjustment a continuous map (stopping test 1e-13, so the passes reach the
        root; no entry band, so no cell jumps between left alone and adjusted): the adjoint
        gradient with respect to H against central differences of the same forward in 3 seeded
        directions. With the reference's 1e-3 entry band the forward is discontinuous: over 5-50
        steps the central differences move by 1-30 % with the step size while the adjoint stays
        put (an FP64 run with the band, measured);
      * the reference's stopping test (1e-3): the mixed-precision trajectory (FP32 state and
        stencils, FP64 pressure refinement and adjustment; its checkpoints held as the mixed state)
        reversed by the FP64 adjoint about FP64 steps restarted from those checkpoints, against the
        FP64 reference gradient (FP64 trajectory, FP64 adjoint)."""
    from aturan_b200.autograd import MoistFullStepper, rollout_gradient
    p = P.default_params()
    st = S.synthetic_state(p, seed=20261208)
    rng = np.random.default_rng(20261208)
    H = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
    _, the = S.coords(p)
    lat = 90.0 - np.degrees(the)
    wj = np.abs(np.sin(the))
    eq = torch.tensor(np.where(np.abs(lat) <= 5.0, wj, 0.0), device="cuda")
    po = torch.tensor(np.where(np.abs(lat) >= 85.0, wj, 0.0), device="cuda")

    def loss(x):
        T = x[0][1:-1, :, :-1]
        return ((T * eq[None, :, None]).sum() / (eq.sum() * T.shape[0] * T.shape[2])
                - (T * po[None, :, None]).sum() / (po.sum() * T.shape[0] * T.shape[2]))

    xs = [torch.tensor(st[n], device="cuda") for n in MOIST]
    aux = [torch.tensor(st[n], device="cuda") for n in ("aux_u", "aux_v", "aux_w")]
    press = dict(kind=P.PRESS_RB_LINE, omega=1.0, max_sweeps=100, tol=1e-10)

    # (1) FP64 at the root: gradient against finite differences
    pr = P.default_params()
    pr.satadj_stop_tol = 1e-13
    pr.satadj_entry_tol = -1.0
    cr = api.Context(pr)
    cr.upload_state(st)
    sr = MoistFullStepper(cr, **press)
    L, gx, ga, gH = rollout_gradient(sr, xs, aux, 50, 10, loss, heat=H)

    def run(Hx):
        x, a = xs, aux
        with torch.no_grad():
            for _ in range(50):
                x, a = sr.forward(x, a, Hx)
        return float(loss(x))

    worst = 0.0
    for _ in range(3):
        d = torch.tensor(1e-5 * rng.standard_normal((p.jm, p.km)), device="cuda")
        h = 1e-2
        fd = (run(H + h * d) - run(H - h * d)) / (2 * h)
        an = float((gH * d).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    cr.close()
    print("config4 moist FD worst", worst)
    assert worst <= 1e-3, worst

    # (2) the reference's stopping test: the mixed trajectory against the FP64 reference gradient
    c64 = api.Context(p)
    c64.upload_state(st)
    s64 = MoistFullStepper(c64, **press)
    L64, _, _, g64 = rollout_gradient(s64, xs, aux, 50, 10, loss, heat=H)
    c32 = api.Context(P.default_params(precision=P.MIXED))
    c32.upload_state(st)
    f32 = MoistFullStepper(c32, tape=False, **press)
    L32, _, _, g32 = rollout_gradient(s64, xs, aux, 50, 10, loss, heat=H, forward_stepper=f32)
    c32.close()
    c64.close()
    rel = float((g32 - g64).norm() / g64.norm())
    rel_max = float((g32 - g64).abs().max() / g64.abs().max())
    dl = abs(float(L32) - float(L64)) / abs(float(L64))
    print("config4 mixed vs FP64: gradient rel L2", rel, "max", rel_max, "loss", dl)
    assert dl <= 1e-5, dl
    assert rel <= 1e-3 and rel_max <= 1e-2, (rel, rel_max)
