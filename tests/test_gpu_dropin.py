"""The drop-in on the reference's own model: the compiled reference (oracle/_ref, built from its
unmodified sources) with the driver glue oracle/ref/b200_glue.cpp, compiled against the reference's
headers as a maintainer would add it, runs iterations 1-4 of its loop on the GPU through
libaturan_b200 (glue_run: aturan_params and aturan_iter_params built from the model, the model's
Arrays uploaded, aturan_iteration four times, the Arrays downloaded); the oracle, whose iteration
reproduces the reference's own Run() bit for bit (tests/test_oracle_vs_ref.py::test_reference_loop),
runs the same four iterations on the same initialised state. Runs in a child process (one reference
model per process). Needs the glue library, which the reference tree builds (oracle/Makefile glue).

Bar (FP64): every field finite; in every field 99.99 % of the cells within 1e-9 of the field's
maximum and at most 0.1 % beyond it (the last-bit differences of CUDA's exp/log/pow in the
saturation adjustment, the MCA and the precipitation move a few isolated cells further, as their
own tests count).
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GLUE = os.path.join(ROOT, "oracle", "_ref", "libaturan_ref_glue.so")


def test_reference_model_through_the_glue():
    if not os.path.exists(GLUE):
        pytest.skip("driver glue library (oracle/_ref/libaturan_ref_glue.so) not built")
    child = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_dropin_child.py")
    r = subprocess.run([sys.executable, child, "4", "0"], capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    worst = sorted(res.items(), key=lambda kv: -kv[1][0])[:6]
    for name, (mx, q9999, frac, finite) in res.items():
        assert finite, name
        assert q9999 <= 1e-9 and frac <= 1e-3, (name, mx, q9999, frac, worst)
