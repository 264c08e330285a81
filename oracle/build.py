"""Builds the test-side checkers (test infrastructure; nothing here ships in the library).

    python -m oracle.build

  oracle/_build/liboracle.so  the C restatement of the reference algorithm (otmap_oracle.c)
  oracle/_ref/libotref.so     the reference library compiled from its own sources, when a
                              reference checkout is found (see reference_root)
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def reference_root() -> str | None:
    """The reference checkout: $OTMAP_REFERENCE, else a directory named `reference` beside
    this repository's root. None when neither holds the reference's otlib/ sources."""
    for cand in (os.environ.get("OTMAP_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "otlib")):
            return os.path.abspath(cand)
    return None


def _run(cmd):
    r = subprocess.run(cmd, cwd=ROOT, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("command failed: " + " ".join(cmd))
    return r.stdout


def build(reference: bool = True) -> None:
    _run(["make", "-C", HERE, "oracle"])
    ref_root = reference_root()
    if reference and ref_root:
        _run(["make", "-C", HERE, "ref", f"REF={ref_root}", "-j8"])


if __name__ == "__main__":
    build()
    print(os.path.join(HERE, "_ref", "libotref.so"))
