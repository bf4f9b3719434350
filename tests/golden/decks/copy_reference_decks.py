"""Copies the reference's own deck fixtures (fasterhenry-cli/tests/data/) into
this folder, byte for byte, so the tests can pin the deck reader to them on
machines without the reference checkout.  Run from the repository root with
the reference at REFERENCE (default /root/reference):

    python tests/golden/decks/copy_reference_decks.py

The files are small self-authored decks of the reference project:
spiral.inp / spiral.json (the round-trip pair of
fasterhenry-cli/tests/roundtrip.rs:18-40), twobar.inp (the two-port SPICE
fixture) and the ground-plane decks plane_*.inp.
"""
import os
import shutil
import sys

NAMES = ["spiral.inp", "spiral.json", "twobar.inp", "plane_fasthenry.inp", "plane_extension.inp",
         "plane_decay_rect.inp", "plane_decay_extension.inp"]


def main():
    ref = os.environ.get("REFERENCE", "/root/reference")
    src = os.path.join(ref, "fasterhenry-cli", "tests", "data")
    here = os.path.dirname(os.path.abspath(__file__))
    for name in NAMES:
        shutil.copyfile(os.path.join(src, name), os.path.join(here, name))
        print("copied", name)
    return 0


if __name__ == "__main__":
    sys.exit(main())
