"""Child process of tests/test_gpu_dropin.py: the reference's own initialised model (the compiled
reference with the driver glue, oracle/_ref/libaturan_ref_glue.so) runs N iterations of its loop on
the GPU through libaturan_b200 (glue_run: upload, aturan_iteration x N, download into the model's
fields); the oracle runs the same N iterations on the same initialised state. Prints one JSON line
of per-field agreement and exits 0."""
import faulthandler
import json
import os
import sys

faulthandler.enable()

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from aturan_b200 import fields as F, params as P  # noqa: E402
from oracle import Oracle, ref  # noqa: E402

GLUE = os.path.join(ROOT, "oracle", "_ref", "libaturan_ref_glue.so")


def main(n, precision):
    print("loading the reference with the glue", file=sys.stderr, flush=True)
    r = ref.Ref(path=GLUE)
    print("reference initialised", file=sys.stderr, flush=True)
    names = [m for m in F.NAMES if m not in F.PROJECTION]
    st = r.state(F.NAMES)                    # every field the oracle's iteration reads or writes
    p = P.params_from_ref(r)
    ip = P.default_iter_params()
    rc = r.L.glue_run(int(n), int(precision))
    assert rc == 0, rc
    g = r.state(names)
    O = Oracle()
    for it in range(1, n + 1):
        O.iteration(p, ip, st, it)
    out = {}
    for m in names:
        s = max(float(np.abs(st[m]).max()), 1e-300)
        d = np.abs(g[m] - st[m]) / s
        out[m] = [float(d.max()), float(np.quantile(d, 0.9999)), float((d > 1e-9).mean()),
                  bool(np.all(np.isfinite(g[m])))]
    print(json.dumps(out))


if __name__ == "__main__":
    main(int(sys.argv[1]), int(sys.argv[2]))
