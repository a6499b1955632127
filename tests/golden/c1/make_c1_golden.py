"""Generates tests/golden/c1/bump2d_c1_5000.npz: the 192 x 64 circular-arc bump
channel (JST, RK4, local time step at CFL 2.0, uniform inlet start; the
``cases.bump2d()`` defaults) advanced 5000 iterations by the reference solver
built from its own sources (oracle/_ref/ref_harness, see
oracle/refbuild/Makefile, with -ffp-contract=off).

The fixture holds the final conservative state, the residual-norm history and
the physical time. The case files themselves are not stored: ``cases.bump2d()``
rebuilds them deterministically.

Run from the repository root after the reference build exists:
    python tests/golden/c1/make_c1_golden.py
"""

from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

from cturbobfm_b200 import cases  # noqa: E402
from oracle import oracle  # noqa: E402

N_ITER = 5000
OUT = os.path.join(HERE, "bump2d_c1_5000.npz")


def main():
    if not oracle.ref_available():
        raise SystemExit("the reference build (oracle/_ref) is missing: run oracle.build() with the reference present")
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    with tempfile.TemporaryDirectory() as d:
        ini = cases.bump2d().write(d)
        ref = oracle.ref_harness("steps", ini, N_ITER, timeout=3600.0)
    assert ref["iterations"] == N_ITER
    np.savez_compressed(OUT, n_iter=N_ITER, state=ref["state"], lognorm=ref["lognorm"], time=ref["time"],
                        shape=ref["shape"])
    print("wrote", OUT)


if __name__ == "__main__":
    main()
