"""Child process of tests/test_oracle_vs_ref.py::test_physics_knob_sets: the reference reads its
knobs from the environment once per process, so each knob set of the chemistry, the turbulence
closure and the precipitation runs in a process of its own. Loads the reference's initialised
state with the row's seeded inputs, runs the reference's routine and the oracle's with the params
that environment resolves to, and exits 0 when every written value is identical."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from aturan_b200 import fields as F, params as P, state as S  # noqa: E402
from oracle import Oracle, ref  # noqa: E402

# name -> (environment of the reference, row)
KNOB_SETS = {
    "chem_minus_open_phi": ({"ATURAN_CHEM_DIFFLUX_PLUS": "0", "ATURAN_BC_PHI_PERIODIC": "0"}, "chem"),
    "turb_no_curv_open_phi": ({"ATURAN_TURB_CURV": "0", "ATURAN_BC_PHI_PERIODIC": "0"}, "turb"),
    "precip_uncoupled": ({"ATURAN_PRECIP_COUPLING": "0"}, "precip"),
    "precip_no_h2s": ({"ATURAN_PRECIP_H2S": "0", "ATURAN_PRECIP_SCALE": "0.003"}, "precip"),
}


def main(name):
    env, row = KNOB_SETS[name]
    for k, v in env.items():
        assert os.environ.get(k) == v, (k, os.environ.get(k))
    r = ref.Ref()
    O = Oracle()
    p = P.default_params()
    base = S.perturb(r.state([n for n in F.NAMES if n not in ref.VEC_FIELDS]), p, seed=45)
    if row == "chem":
        from tests.chem_case import EQ_OUT, FORCING_OUT, chem_state
        cp = P.chem_params_from_ref(r)
        cp.difflux_plus = 0 if env.get("ATURAN_CHEM_DIFFLUX_PLUS") == "0" else 1
        assert cp.phi_periodic == 0
        st = chem_state(base, p, seed=46)
        r.load(st)
        r.chem_eq()
        r.chem_forcing()
        O.nh4sh_eq(p, cp, st)
        O.chem_forcing(p, cp, st)
        names = EQ_OUT + FORCING_OUT
    elif row == "turb":
        from tests.turb_case import TURB_OUT, turb_state
        tp = P.turb_params_from_ref(r)
        assert tp.curv == 0 and tp.phi_periodic == 0
        st = turb_state(base, p, seed=47)
        r.load(st)
        r.turbulence()
        O.turbulence(p, tp, st)
        names = TURB_OUT
    else:
        from tests.precip_case import PRECIP_OUT_UNCOUPLED, precip_state
        pp = P.precip_params_from_ref(r)
        st = precip_state(base, p, seed=48)
        r.load(st)
        r.precipitation()
        O.precipitation(p, pp, st)
        names = PRECIP_OUT_UNCOUPLED
    got = r.state(names)
    bad = [n for n in names if not np.array_equal(got[n], st[n], equal_nan=True)]
    assert not bad, bad
    print("OK", name)


if __name__ == "__main__":
    main(sys.argv[1])
