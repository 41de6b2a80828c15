"""Generate ``tests/golden/example_userxy1.npz`` from the reference's own
example case (``example/userxy1`` of the reference: the configuration files
of its documented smoke run ``./imcom config_example S 1.d-3 1.d-6`` and the
FITS images they name, including the truth image
``ideal_output.example.fits``).

The fixture stores every file's bytes unchanged (one uint8 array per file
name), so a test can write the directory back out and run the library's own
configuration and FITS readers on it.  ``unpack(dest)`` does that.

Usage: ``python tests/golden/make_example_fixture.py <reference root>`` (the
directory holding the reference's ``example/``; required).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "example_userxy1.npz")
CONFIG = "config_example"


def main(root: str) -> None:
    src = os.path.join(root, "example", "userxy1")
    out = {}
    for name in sorted(os.listdir(src)):
        raw = open(os.path.join(src, name), "rb").read()  # symlinks followed
        out[name] = np.frombuffer(raw, dtype=np.uint8)
    np.savez_compressed(FIXTURE, **out)


def unpack(dest: str) -> str:
    """Write the example directory into `dest`; returns the main config path."""
    with np.load(FIXTURE) as z:
        for name in z.files:
            with open(os.path.join(dest, name), "wb") as f:
                f.write(z[name].tobytes())
    return os.path.join(dest, CONFIG)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_example_fixture.py <reference root>")
    main(sys.argv[1])
