"""torch.autograd binding of the RK4 step's hand-written adjoint (aturan_tape / aturan_rk4_adjoint).

DryRK4Step maps the dry prognostic fields (t, u, v, w) before one RK4 step to the same fields
after it, on CUDA FP64 tensors of shape (im, jm, km) in the reference's logical [i][j][k] layout.
Every other input of the step (p_dyn, p_stat, p_baro, p_b0, p_bfollow, the forcing, the other
prognostic fields) is held at the values the context had when the stepper was made: each call
re-uploads them, so calls are independent. The forward runs aturan_rk4_step on the context with the
tape on; the backward runs aturan_rk4_adjoint, the reverse of that step (no autograd tape of its
own: the kernels are the adjoint).
"""
import torch

from . import fields as F

DRY = ("t", "u", "v", "w")
# fields a step changes that the dry tendencies read: restored before every forward
_RESTORE = ("p_bfollow",)


class DryStepper:
    """Holds an FP64 aturan_b200.api.Context and the fixed inputs of the step."""

    def __init__(self, ctx, tape=True):
        if not torch.cuda.is_available():
            raise RuntimeError("DryStepper needs a CUDA device")
        self.ctx = ctx
        self.shape = (ctx.p.im, ctx.p.jm, ctx.p.km)
        self.saved = {n: torch.empty(self.shape, dtype=torch.float64, device="cuda") for n in _RESTORE}
        self.n_forward = 0                     # id of the step the tape holds
        torch.cuda.synchronize()
        for n, t in self.saved.items():
            ctx.download_device(n, t.data_ptr())
        if tape:
            ctx.tape(True)

    def forward(self, xs):
        ctx = self.ctx
        xs = [x.detach().contiguous() for x in xs]
        torch.cuda.synchronize()
        for n, t in self.saved.items():
            ctx.upload_device(n, t.data_ptr())
        for n, x in zip(DRY, xs):              # the state and its start-of-step copy
            ctx.upload_device(n, x.data_ptr())
            ctx.upload_device(n + "n", x.data_ptr())
        ctx.rk4_step()
        self.n_forward += 1
        out = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in DRY]
        for n, o in zip(DRY, out):
            ctx.download_device(n, o.data_ptr())
        return out

    def backward(self, ybar):
        ybar = [torch.zeros(self.shape, dtype=torch.float64, device="cuda") if g is None else g.contiguous()
                for g in ybar]
        xbar = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in DRY]
        torch.cuda.synchronize()
        self.ctx.rk4_adjoint([g.data_ptr() for g in ybar], [x.data_ptr() for x in xbar])
        return xbar


class DryRK4Step(torch.autograd.Function):
    """t1, u1, v1, w1 = DryRK4Step.apply(stepper, t, u, v, w)."""

    @staticmethod
    def forward(fctx, stepper, t, u, v, w):
        fctx.stepper = stepper
        out = tuple(stepper.forward([t, u, v, w]))
        fctx.step_id = stepper.n_forward
        return out

    @staticmethod
    def backward(fctx, *ybar):
        if fctx.step_id != fctx.stepper.n_forward:
            raise RuntimeError("DryRK4Step: the tape holds a later step; run backward before the next forward")
        xbar = fctx.stepper.backward(list(ybar))
        return (None, *xbar)


assert all(n in F.ID for n in DRY + tuple(n + "n" for n in DRY) + _RESTORE)
assert tuple(F.PROGNOSTIC[:4]) == DRY


AUX = ("aux_u", "aux_v", "aux_w")


class DryFullStepper(DryStepper):
    """One full dry step with the pressure solve inside: (t, u, v, w, aux_u, aux_v, aux_w) ->
    the same after it. The step solves the pressure equation from the aux fields (the projection
    outputs of the previous step's RK4) with kind/omega/tol (RB_SOR or RB_LINE, from p_dyn = 0 so
    that the result does not depend on an earlier call) and runs the RK4 step, whose stage 3
    writes the next aux. The saturation adjustment is the identity on a dry state and is not run.
    Backward: aturan_rk4_adjoint_ex (the state's and p_dyn's adjoints from the outputs', the aux
    outputs' adjoint entering at stage 3), then aturan_pressure_adjoint (p_dyn's adjoint back to
    the aux inputs'). Only the aux interior enters the next solve; boundary rows get no gradient."""

    def __init__(self, ctx, kind=3, omega=1.0, max_sweeps=200, tol=1e-10, tape=True):
        super().__init__(ctx, tape)
        self.press = (kind, omega, max_sweeps, tol)
        self.zero = torch.zeros(self.shape, dtype=torch.float64, device="cuda")

    def forward(self, xs, aux, heat=None):
        """heat: an optional [jm][km] heating rate in K/s (aturan_set_heating) held for the step."""
        ctx = self.ctx
        xs = [x.detach().contiguous() for x in xs]
        aux = [a.detach().contiguous() for a in aux]
        if heat is not None:
            heat = heat.detach().contiguous()
        torch.cuda.synchronize()
        ctx.set_heating(heat.data_ptr() if heat is not None else None)
        self.heated = heat is not None
        for n, t in self.saved.items():
            ctx.upload_device(n, t.data_ptr())
        ctx.upload_device("p_dyn", self.zero.data_ptr())
        for n, x in zip(DRY, xs):
            ctx.upload_device(n, x.data_ptr())
            ctx.upload_device(n + "n", x.data_ptr())
        for n, a in zip(AUX, aux):
            ctx.upload_device(n, a.data_ptr())
        kind, omega, ms, tol = self.press
        ctx.pressure(kind, omega=omega, max_sweeps=ms, tol=tol)
        ctx.rk4_step()
        self.n_forward += 1
        out = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in DRY + AUX]
        for n, o in zip(DRY + AUX, out):
            ctx.download_device(n, o.data_ptr())
        return out[:4], out[4:]

    def backward(self, ybar, auxbar):
        """(xbar, abar), or (xbar, abar, hbar) when the step had a heating field."""
        z = lambda g: torch.zeros(self.shape, dtype=torch.float64, device="cuda") if g is None else g.contiguous()
        ybar = [z(g) for g in ybar]
        auxbar = [z(g) for g in auxbar]
        xbar = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in DRY]
        pbar = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        abar = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in AUX]
        hbar = torch.empty(self.shape[1:], dtype=torch.float64, device="cuda") if self.heated else None
        torch.cuda.synchronize()
        self.ctx.rk4_adjoint_ex([g.data_ptr() for g in ybar], [g.data_ptr() for g in auxbar],
                                [x.data_ptr() for x in xbar], pbar.data_ptr(),
                                hbar.data_ptr() if hbar is not None else None)
        kind, omega, ms, tol = self.press
        self.ctx.pressure_adjoint(pbar.data_ptr(), [a.data_ptr() for a in abar], kind, omega, ms, tol)
        return (xbar, abar) if hbar is None else (xbar, abar, hbar)


class DryFullStep(torch.autograd.Function):
    """t1, u1, v1, w1, au1, av1, aw1 = DryFullStep.apply(stepper, t, u, v, w, au, av, aw)."""

    @staticmethod
    def forward(fctx, stepper, t, u, v, w, au, av, aw):
        fctx.stepper = stepper
        xs, aux = stepper.forward([t, u, v, w], [au, av, aw])
        fctx.step_id = stepper.n_forward
        return tuple(xs + aux)

    @staticmethod
    def backward(fctx, *gr):
        if fctx.step_id != fctx.stepper.n_forward:
            raise RuntimeError("DryFullStep: the tape holds a later step; run backward before the next forward")
        xbar, abar = fctx.stepper.backward(list(gr[:4]), list(gr[4:]))
        return (None, *xbar, *abar)


MOIST = tuple(F.PROGNOSTIC[:16])           # t, u, v, w and the twelve condensable species


class MoistFullStepper(DryFullStepper):
    """One full moist step in the reference's order, the saturation adjustment inside:
    (t, u, v, w, twelve condensable species, aux_u, aux_v, aux_w) -> the same after it. The step
    solves the pressure equation from the aux fields (from p_dyn = 0), adjusts the four gases
    (aturan_satadj), sets the start-of-step copies to the adjusted state (aturan_sync_ncopies) and
    runs the RK4 step. Backward: aturan_moist_adjoint (the RK4 step's adjoint over the sixteen
    fields, then the adjustment's implicit adjoint), then aturan_pressure_adjoint. The other scalar
    fields (NH4SH, k, epsilon), p_stat, the forcing and the hydrostatic split are held at the
    context's values. tape=False makes a forward-only stepper, e.g. on a mixed-precision context
    (rollout_gradient's forward_stepper)."""

    def __init__(self, ctx, kind=3, omega=1.0, max_sweeps=200, tol=1e-10, tape=True):
        super().__init__(ctx, kind, omega, max_sweeps, tol, tape=False)
        if tape:
            ctx.tape(2)
        self.others = {n: torch.empty(self.shape, dtype=torch.float64, device="cuda")
                       for n in F.PROGNOSTIC[16:]}
        torch.cuda.synchronize()
        for n, t in self.others.items():
            ctx.download_device(n, t.data_ptr())

    def forward(self, xs, aux, heat=None):
        ctx = self.ctx
        xs = [x.detach().contiguous() for x in xs]
        aux = [a.detach().contiguous() for a in aux]
        if heat is not None:
            heat = heat.detach().contiguous()
        torch.cuda.synchronize()
        ctx.set_heating(heat.data_ptr() if heat is not None else None)
        self.heated = heat is not None
        for n, t in self.saved.items():
            ctx.upload_device(n, t.data_ptr())
        for n, t in self.others.items():
            ctx.upload_device(n, t.data_ptr())
        ctx.upload_device("p_dyn", self.zero.data_ptr())
        for n, x in zip(MOIST, xs):
            ctx.upload_device(n, x.data_ptr())
        for n, a in zip(AUX, aux):
            ctx.upload_device(n, a.data_ptr())
        ctx.restore_ncopies(1.0)               # every start-of-step copy is the step's input
        kind, omega, ms, tol = self.press
        ctx.pressure(kind, omega=omega, max_sweeps=ms, tol=tol)
        ctx.satadj(0xF, count=False)
        ctx.sync_ncopies()                     # the adjusted scalars' copies (RK_SCALAR_SYNC)
        ctx.rk4_step()
        self.n_forward += 1
        out = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in MOIST + AUX]
        for n, o in zip(MOIST + AUX, out):
            ctx.download_device(n, o.data_ptr())
        return out[:16], out[16:]

    def backward(self, ybar, auxbar):
        z = lambda g: torch.zeros(self.shape, dtype=torch.float64, device="cuda") if g is None else g.contiguous()
        ybar = [z(g) for g in ybar]
        auxbar = [z(g) for g in auxbar]
        xbar = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in MOIST]
        pbar = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        abar = [torch.empty(self.shape, dtype=torch.float64, device="cuda") for _ in AUX]
        hbar = torch.empty(self.shape[1:], dtype=torch.float64, device="cuda") if self.heated else None
        torch.cuda.synchronize()
        self.ctx.moist_adjoint([g.data_ptr() for g in ybar], [g.data_ptr() for g in auxbar],
                               [x.data_ptr() for x in xbar], pbar.data_ptr(),
                               hbar.data_ptr() if hbar is not None else None)
        kind, omega, ms, tol = self.press
        self.ctx.pressure_adjoint(pbar.data_ptr(), [a.data_ptr() for a in abar], kind, omega, ms, tol)
        return (xbar, abar) if hbar is None else (xbar, abar, hbar)


def rollout_gradient(stepper, xs0, aux0, nsteps, every, loss_fn, heat=None, forward_stepper=None):
    """Loss after nsteps DryFullStepper steps from (xs0, aux0) and its gradient with respect to
    xs0 and aux0, by the hand-written adjoint with checkpointing: the forward keeps the inputs of
    every `every`-th step; the backward recomputes a segment's step inputs from its checkpoint,
    then re-runs each step (which tapes it) right before its adjoint, last step first. Memory:
    (nsteps / every + every) step inputs; cost about three forward passes plus the adjoints.
    loss_fn maps the final (t, u, v, w) to a scalar tensor (differentiated by torch.autograd).
    With heat (a [jm][km] heating rate held over the trajectory) the gradient with respect to it,
    summed over the steps, is returned too.
    forward_stepper (e.g. a forward-only MoistFullStepper on a mixed-precision context) runs the
    trajectory itself: the loss and the checkpoints are its, while each segment is recomputed from
    its checkpoint, taped and reversed by `stepper` (FP64): the adjoint of the mixed trajectory
    linearised about FP64 steps restarted from its checkpoints."""
    fwd = forward_stepper if forward_stepper is not None else stepper
    ck = {0: ([x.detach() for x in xs0], [a.detach() for a in aux0])}
    xs, aux = ck[0]
    with torch.no_grad():
        for n in range(nsteps):
            xs, aux = fwd.forward(xs, aux, heat)
            if (n + 1) % every == 0 and n + 1 < nsteps:
                ck[n + 1] = (xs, aux)
    xf = [x.detach().requires_grad_(True) for x in xs]
    loss = loss_fn(xf)
    ybar = list(torch.autograd.grad(loss, xf, allow_unused=True))
    ybar = [torch.zeros_like(x) if g is None else g for x, g in zip(xf, ybar)]
    abar = [torch.zeros_like(a) for a in aux]
    hsum = None if heat is None else torch.zeros_like(heat)
    for start in sorted(ck, reverse=True):
        end = min(start + every, nsteps)
        inputs = [ck[start]]
        with torch.no_grad():
            for _ in range(start, end - 1):
                inputs.append(stepper.forward(*inputs[-1], heat))
        for n in reversed(range(start, end)):
            stepper.forward(*inputs[n - start], heat)      # tapes step n
            out = stepper.backward(ybar, abar)
            ybar, abar = out[0], out[1]
            if heat is not None:
                hsum += out[2]
    if heat is None:
        return loss.detach(), ybar, abar
    return loss.detach(), ybar, abar, hsum
