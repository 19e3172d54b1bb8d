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

    def __init__(self, ctx):
        if not torch.cuda.is_available():
            raise RuntimeError("DryStepper needs a CUDA device")
        self.ctx = ctx
        self.shape = (ctx.p.im, ctx.p.jm, ctx.p.km)
        self.saved = {n: torch.empty(self.shape, dtype=torch.float64, device="cuda") for n in _RESTORE}
        self.n_forward = 0                     # id of the step the tape holds
        torch.cuda.synchronize()
        for n, t in self.saved.items():
            ctx.download_device(n, t.data_ptr())
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
