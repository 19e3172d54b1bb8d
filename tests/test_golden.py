"""The oracle restatement reproduces the compiled reference's golden digests bit for bit.

tests/golden/golden.json was made by tests/golden/make_golden.py from the compiled reference on
seeded synthetic states; this test needs only the oracle, so it pins it on any machine.
"""
import json
import os

import numpy as np
import pytest

from aturan_b200 import params as P, state as S
from tests.golden.make_golden import CASES, digest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def oracle_runner(O, name, p, st):
    lev = None
    if name == "satadj4":
        for g in range(4):
            O.satadj(p, st, g)
    elif name == "rk4":
        lev = O.rk4(p, st)
    elif name == "pressure_gs":
        O.pressure_gs(p, st)
    elif name == "pressure_rb3":
        O.pressure_rb(p, st, 3)
    elif name == "step_gs":
        lev = O.step(p, st, P.PRESS_GS_LEX)
    elif name == "mca":
        O.mca(p, st)
    elif name == "post_step":
        from tests.golden.make_golden import post_input
        st = post_input(p, st, CASES[name]["seed"])
        O.post_step(p, st, P.default_post_params())
    elif name.startswith("chem_"):
        from tests.golden.make_golden import chem_input
        st = chem_input(p, st, CASES[name]["seed"])
        if name == "chem_eq":
            O.nh4sh_eq(p, P.default_chem_params(), st)
        else:
            O.chem_forcing(p, P.default_chem_params(), st)
    elif name == "turbulence":
        from tests.golden.make_golden import turb_input
        st = turb_input(p, st, CASES[name]["seed"])
        O.turbulence(p, P.default_turb_params(), st)
    elif name == "precipitation":
        from tests.golden.make_golden import precip_input
        st = precip_input(p, st, CASES[name]["seed"])
        O.precipitation(p, P.default_precip_params(), st)
    out = dict(st)
    if lev is not None:
        out["buoy_ref_level"] = lev
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_golden(oracle_lib, name):
    rec = GOLDEN["cases"][name]
    p = P.default_params()
    st = S.synthetic_state(p, seed=rec["seed"])
    out = oracle_runner(oracle_lib, name, p, st)
    for fname, want in rec["fields"].items():
        a = np.ascontiguousarray(out[fname]).ravel()
        for idx, hx in want["samples"]:
            assert a[idx] == float.fromhex(hx) or (np.isnan(a[idx]) and np.isnan(float.fromhex(hx))), \
                (name, fname, idx, a[idx], hx)
        assert digest(out[fname]) == want["sha256"], (name, fname)
