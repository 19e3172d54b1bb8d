"""The torch FP64 restatement of the dry RK4 step (the adjoint's gradient reference) against the C
restatement, which is bit-identical to the compiled reference: same t, u, v, w after one step to
rounding."""
import numpy as np
import pytest
import torch

from aturan_b200 import params as P, state as S
from oracle.dry_ref import DryStep

FIXED = ("p_dyn", "p_stat", "p_baro", "p_b0", "p_bfollow", "nue", "thermalmassflux", "Q_precip")


@pytest.mark.parametrize("shape,seed", [((12, 20, 33), 51), ((21, 37, 73), 52)])
def test_dry_step_matches_oracle(oracle_lib, shape, seed):
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=seed)
    dry = DryStep(p, {n: st[n] for n in FIXED}, oracle_lib)
    x = [torch.tensor(st[n]) for n in ("t", "u", "v", "w")]
    out = dry(*x)
    ref = S.copy_state(st)
    for n in ("t", "u", "v", "w"):                 # the step's start-of-step copies are the state
        ref[n + "n"][:] = ref[n]
    oracle_lib.rk4(p, ref)
    for n, o in zip(("t", "u", "v", "w"), out):
        a, b = o.numpy(), ref[n]
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err < 1e-12, (n, err)


def test_dry_step_gradient_is_finite_difference_consistent(oracle_lib):
    """torch.autograd through the restatement agrees with central differences (a check of the
    restatement's differentiability; the GPU adjoint is compared against this gradient)."""
    p = P.default_params(12, 20, 33)
    st = S.synthetic_state(p, seed=53)
    dry = DryStep(p, {n: st[n] for n in FIXED}, oracle_lib)
    x = [torch.tensor(st[n], requires_grad=True) for n in ("t", "u", "v", "w")]

    def loss(xs):
        t1 = dry(*xs)[0]
        return (t1[p.im - 2, 1:-1, :-1] ** 2).mean()

    L = loss(x)
    grads = torch.autograd.grad(L, x)
    rng = np.random.default_rng(7)
    for _ in range(3):
        d = [torch.tensor(rng.standard_normal(p.shape)) * (1e-3 * float(xi.detach().abs().max()) + 1e-12)
             for xi in x]
        h = 1e-3
        with torch.no_grad():
            lp = loss([xi + h * di for xi, di in zip(x, d)])
            lm = loss([xi - h * di for xi, di in zip(x, d)])
        fd = float((lp - lm) / (2 * h))
        an = float(sum((g * di).sum() for g, di in zip(grads, d)))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-30), (fd, an)


MOIST_FIXED = FIXED + tuple("S_precip_" + n for n in ("ch4", "ch4_cloud", "ch4_ice", "h2o", "h2o_cloud", "h2o_ice",
                                                     "h2s", "h2s_cloud", "h2s_ice", "nh3", "nh3_cloud", "nh3_ice")) \
    + ("massflux_h2s", "massflux_nh3")


@pytest.mark.parametrize("shape,seed", [((12, 20, 33), 54), ((21, 37, 73), 55)])
def test_moist_step_matches_oracle(oracle_lib, shape, seed):
    """The moist restatement (t, u, v, w and the twelve condensable species) against the C
    restatement's RK4 step."""
    from oracle.dry_ref import MoistRK4Step, SPECIES
    p = P.default_params(*shape)
    st = S.synthetic_state(p, seed=seed)
    names = ("t", "u", "v", "w") + SPECIES
    step = MoistRK4Step(p, {n: st[n] for n in MOIST_FIXED}, oracle_lib)
    out = step(*[torch.tensor(st[n]) for n in names])
    ref = S.copy_state(st)
    for n in names + ("nh4sh", "tke", "dis"):
        ref[n + "n"][:] = ref[n]
    oracle_lib.rk4(p, ref)
    for n, o in zip(names, out):
        a, b = o.numpy(), ref[n]
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
        assert err < 1e-12, (n, err)
