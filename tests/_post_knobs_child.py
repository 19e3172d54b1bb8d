"""Child process of tests/test_oracle_vs_ref.py::test_post_step_knob_sets: the reference reads its
knobs from the environment once per process, so each knob set runs in a process of its own.
Loads the reference's initialised state with the post-step inputs, runs the reference's passes
and the oracle's, and exits 0 when every written value is identical."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from aturan_b200 import fields as F, params as P, state as S  # noqa: E402
from oracle import Oracle, ref  # noqa: E402
from tests.post_case import KNOB_SETS, POST_FIELDS, post_state  # noqa: E402


def main(name):
    env, mk = KNOB_SETS[name]
    for k, v in env.items():
        assert os.environ.get(k) == v, (k, os.environ.get(k))
    r = ref.Ref()
    p = P.default_params()
    # the hydrostatic split vectors are empty without GEO_BALANCE, and the passes do not read them
    st = post_state(S.perturb(r.state([n for n in F.NAMES if n not in ref.VEC_FIELDS]), p, seed=43), p, seed=44)
    pp = mk()
    r.load(st)
    ra, rc = r.post_step(pp)
    oa, oc = Oracle().post_step(p, st, pp)
    got = r.state(POST_FIELDS)
    bad = [n for n in POST_FIELDS if not np.array_equal(got[n], st[n], equal_nan=True)]
    assert not bad, bad
    assert np.array_equal(rc, oc), (rc, oc)
    assert np.allclose(ra, oa, rtol=1e-12, atol=0.0), (ra, oa)
    print("OK", name)


if __name__ == "__main__":
    main(sys.argv[1])
