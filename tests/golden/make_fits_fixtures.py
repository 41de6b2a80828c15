"""Generate ``tests/golden/fits_examples.npz`` from the reference's example
FITS files (example/fits/*.example.fits of the reference, written by its
CFITSIO/IDL tooling).

For each of three images -- an input exposure (32 x 32), an input x-coordinate
map with half-pixel values (32 x 32) and the ideal output (65 x 65, whose
data block ends part-way through a 2880-byte record) -- the fixture keeps the
primary header record (2880 bytes), the image as decoded here with numpy
alone (big-endian float64 after the header, axis 1 fastest) and the SHA-256
of the file's data records (the data and its zero padding).  The FITS tests
rebuild each file from these, read it with the library and write it back.

Usage: ``python tests/golden/make_fits_fixtures.py <reference root>`` (the
directory holding the reference's ``example/fits``; required).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ("test1", "x2", "ideal_output")


def decode(raw: bytes):
    cards = [raw[i:i + 80].decode("ascii") for i in range(0, 2880, 80)]
    kv = {c[:8].strip(): c[10:30].strip() for c in cards if c[8:10] == "= "}
    assert kv["SIMPLE"] == "T" and kv["BITPIX"] == "-64" and kv["NAXIS"] == "2"
    assert any(c.startswith("END ") for c in cards)  # one header record
    n1, n2 = int(kv["NAXIS1"]), int(kv["NAXIS2"])
    data = np.frombuffer(raw[2880:2880 + 8 * n1 * n2], dtype=">f8").astype(np.float64)
    return data.reshape((n1, n2), order="F")


def main(root: str) -> None:
    out = {}
    for name in FILES:
        raw = open(os.path.join(root, "example", "fits", f"{name}.example.fits"), "rb").read()
        assert len(raw) % 2880 == 0
        out[f"{name}_header"] = np.frombuffer(raw[:2880], dtype=np.uint8)
        out[f"{name}_image"] = decode(raw)
        out[f"{name}_data_sha256"] = np.array(hashlib.sha256(raw[2880:]).hexdigest())
    np.savez_compressed(os.path.join(HERE, "fits_examples.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fits_fixtures.py <reference root>")
    main(sys.argv[1])
