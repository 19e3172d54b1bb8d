"""Seeded inputs for the turbulence closure, shared by the oracle-vs-reference test (CPU) and the
GPU parity test."""
import numpy as np

# every field the closure writes
TURB_OUT = ["tke", "dis", "nue", "prod", "tke_source", "dis_source", "tken", "disn"]


def turb_state(st, p, seed):
    """st with k* spread around the background floor k_bg / u_0^2 (about 2 % of the cells negative),
    omega* around the background value (about 2 % below the floor dis_min, some negative), and
    seeded values in every other field the closure writes, so that the clamps, the floors, the caps
    and the edge copies all act; k = km-1 stays the copy of k = 0."""
    rng = np.random.default_rng(seed)
    s = {n: np.array(a, dtype=np.float64, copy=True) for n, a in st.items()}
    shape = (p.im, p.jm, p.km)
    k_bg = 1.0 / (p.u_0 * p.u_0)
    s["tke"] = k_bg * (0.5 + 3.0 * rng.random(shape))
    s["tke"][rng.random(shape) < 0.02] *= -1.0
    s["dis"] = 2.33 * (0.5 + rng.random(shape))
    low = rng.random(shape) < 0.02
    s["dis"][low] = rng.normal(0.0, 1e-10, int(low.sum()))
    for n in ("nue", "prod", "tke_source", "dis_source"):
        s[n] = rng.normal(0.0, 1e-3, shape)
    s["tken"] = s["tke"] * (1.0 + 1e-3 * rng.normal(size=shape))
    s["disn"] = s["dis"] * (1.0 + 1e-3 * rng.normal(size=shape))
    for n in TURB_OUT:
        s[n][:, :, -1] = s[n][:, :, 0]
    return s
