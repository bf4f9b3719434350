"""Copies the reference's own deck fixtures (fasterhenry-cli/tests/data/) into
this folder, byte for byte, so the tests can pin the deck reader to them on
machines without the reference checkout.  Run from the repository root with
the reference at REFERENCE (default /root/reference):

    python tests/golden/decks/copy_reference_decks.py

The files are small self-authored decks of the reference project:
spiral.inp / spiral.json (the round-trip pair of
fasterhenry-cli/tests/roundtrip.rs:18-40), twobar.inp (the two-port SPICE
fixture) and the ground-plane decks plane_*.inp.  It also writes the two
```json example documents of docs/input-format.md, in order, as
input_format_example_0.json (the minimal one) and input_format_example_1.json
(the documented pins of fasterhenry-cli/tests/input_format_doc.rs).
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
    with open(os.path.join(ref, "docs", "input-format.md")) as f:
        lines = f.read().splitlines()
    blocks, block = [], None
    for line in lines:
        if block is None and line.rstrip() == "```json":
            block = []
        elif block is not None and line.rstrip() == "```":
            blocks.append("\n".join(block) + "\n")
            block = None
        elif block is not None:
            block.append(line)
    for k, text in enumerate(blocks):
        name = "input_format_example_%d.json" % k
        with open(os.path.join(here, name), "w") as f:
            f.write(text)
        print("wrote", name)
    return 0


if __name__ == "__main__":
    sys.exit(main())
