"""Regenerates the oracle fixtures in this directory.

* ``c1_z.json`` / ``c2_z.json`` — Z(w) of the 4-turn spiral (240 filaments,
  10 frequencies) and the 40-leg meander (2,400 filaments, 32 frequencies)
  from the CPU oracle (oracle/fh_oracle.cpp, the C++ restatement of the
  reference's dense path).  The oracle itself is pinned to the reference's
  known answers in ``known_answers.json`` (tests/test_oracle_known_answers.py).
* ``c1_fill_sample.json`` — a sample of C1 partial inductances with their
  method ids, for a fill check that needs no oracle run.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from fasterhenry_b200 import fixtures as F  # noqa: E402
from oracle import oracle as O  # noqa: E402


def z_fixture(name, deck, freqs):
    s = O.System(deck)
    z = s.sweep(freqs)
    doc = {"deck": deck.name, "counts": s.counts, "frequencies_hz": freqs,
           "z_re": z.real.tolist(), "z_im": z.imag.tolist(),
           "generator": "oracle System.sweep (FP64, blocked LU PANEL 32)"}
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(doc, f, indent=1)


def main():
    d1, f1 = F.c1_spiral()
    z_fixture("c1_z.json", d1, f1)
    d2, f2 = F.c2_meander()
    z_fixture("c2_z.json", d2, f2)
    fil, _ = O.discretize(d1)
    L, meth = O.fill(fil, methods=True)
    rng = np.random.default_rng(7)
    idx = rng.choice(len(fil), size=(64, 2))
    rows = [[int(i), int(j), float(L[i, j]), int(meth[i, j])] for i, j in idx]
    with open(os.path.join(HERE, "c1_fill_sample.json"), "w") as f:
        json.dump({"deck": d1.name, "entries": rows, "generator": "oracle fill"}, f, indent=1)


if __name__ == "__main__":
    main()
