"""Child process of tests/test_oracle_vs_ref.py::test_reference_loop: runs the compiled reference's
Run() with N iterations of its own loop after its initialisation (a fresh model per process) and
saves the resulting fields to an .npz file for the parent to compare."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from aturan_b200 import fields as F  # noqa: E402
from oracle import ref  # noqa: E402


def main(n, path):
    r = ref.Ref(loop_iterations=n)
    np.savez(path, **r.state(F.NAMES))
    print("OK", n)


if __name__ == "__main__":
    main(int(sys.argv[1]), sys.argv[2])
