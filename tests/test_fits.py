"""FITS images without CFITSIO (imcom_b200/csrc/fits.cpp), on CPU.

The library's writer is checked against an independent decoder written here
(header cards, 2880-byte blocks, big-endian data), and its reader against
files built here by hand in every BITPIX, with BSCALE / BZERO, BLANK and NaN
pixels (undefined pixels read as -666, the reference's null value,
imcom_io.f90:366), headers longer than one block and D exponents.  Sizes
that do not match, missing and malformed files are errors, where the
reference stops (imcom_io.f90:382-393).  Files written by the reference's own
tooling (its example inputs, tests/golden/fits_examples.npz) read back bit for
bit and are written again with the same keys, values, data and padding.
"""
import hashlib
import os

import numpy as np
import pytest

from imcom_b200 import fits
from imcom_b200._lib import ImcomError

IMCOM_ERR_FITS = 10
EXAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fits_examples.npz")


def cards_of(raw):
    out = []
    for i in range(0, len(raw), 80):
        c = raw[i:i + 80].decode("ascii")
        out.append(c)
        if c.startswith("END "):
            break
    return out


def decode(path):
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    cards = cards_of(raw)
    kv = {}
    for c in cards:
        if c[8:10] == "= ":
            kv[c[:8].strip()] = c[10:].split("/")[0].strip()
    start = (len(cards) * 80 + 2879) // 2880 * 2880
    naxes = [int(kv[f"NAXIS{a + 1}"]) for a in range(int(kv["NAXIS"]))]
    count = int(np.prod(naxes))
    data = np.frombuffer(raw[start:start + 8 * count], dtype=">f8")
    return cards, kv, data.reshape(naxes, order="F"), raw[start + 8 * count:]


def hand_file(path, bitpix, values, extra=(), naxes=None, comments=0):
    """A FITS file built here: the given cards, then big-endian data."""
    values = np.asarray(values)
    naxes = naxes or list(values.shape)

    def card(k, v):
        return f"{k:<8}= {v:>20}".ljust(80)
    hdr = [card("SIMPLE", "T"), card("BITPIX", str(bitpix)), card("NAXIS", str(len(naxes)))]
    hdr += [card(f"NAXIS{a + 1}", str(n)) for a, n in enumerate(naxes)]
    hdr += [card(k, v) for k, v in extra]
    hdr += [f"COMMENT   card {i} of a long header".ljust(80) for i in range(comments)]
    hdr += ["END".ljust(80)]
    h = "".join(hdr).encode("ascii")
    h += b" " * ((-len(h)) % 2880)
    dt = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}[bitpix]
    d = np.asarray(values, dtype=dt).ravel(order="F").tobytes()
    d += b"\0" * ((-len(d)) % 2880)
    with open(path, "wb") as f:
        f.write(h + d)


def test_writer_layout(tmp_path):
    a = np.asfortranarray(np.arange(35, dtype=float).reshape(5, 7, order="F") * 0.25 - 3)
    p = str(tmp_path / "a.fits")
    fits.write(p, a)
    cards, kv, data, pad = decode(p)
    assert cards[0].startswith("SIMPLE  =") and cards[0][29] == "T"
    assert [c[:8].strip() for c in cards] == ["SIMPLE", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2",
                                              "EXTEND", "END"]
    assert kv["BITPIX"] == "-64" and kv["NAXIS"] == "2"
    assert kv["NAXIS1"] == "5" and kv["NAXIS2"] == "7"
    for c in cards[:-1]:
        assert len(c) == 80 and c[10:30].rstrip() == c[10:30].rstrip().rjust(20).rstrip()
        assert c[10:30].strip() and c[29] != " "  # value ends in column 30
    assert np.array_equal(data, a)
    assert set(pad) <= {0}


@pytest.mark.parametrize("shape", [(1, 1), (3, 1000), (361, 8), (16, 16)])
def test_round_trip_is_bit_exact(tmp_path, shape):
    rng = np.random.default_rng(shape[0] * shape[1])
    a = rng.standard_normal(shape) * np.logspace(-300, 300, shape[0] * shape[1]).reshape(shape)
    flat = a.reshape(-1)
    flat[:4] = [0.0, -0.0, 5e-324, -1.7976931348623157e308][:flat.size]
    p = str(tmp_path / "r.fits")
    fits.write(p, a)
    assert fits.size(p) == (shape[0], shape[1], -64)
    b = fits.read(p)
    assert b.shape == shape and b.flags.f_contiguous
    assert np.array_equal(np.asarray(a).view(np.uint64), b.view(np.uint64))


def test_cube_layout(tmp_path):
    c = np.asfortranarray(np.arange(60, dtype=float).reshape(3, 4, 5, order="F"))
    p = str(tmp_path / "c.fits")
    fits.write_cube(p, c)
    cards, kv, data, _ = decode(p)
    assert kv["NAXIS"] == "3" and (kv["NAXIS1"], kv["NAXIS2"], kv["NAXIS3"]) == ("3", "4", "5")
    assert np.array_equal(data, c)


def test_reads_every_bitpix_with_scaling_and_nulls(tmp_path):
    v16 = np.array([[1, -2, 7], [300, -32768, 5]], dtype=np.int16)
    p = str(tmp_path / "i16.fits")
    hand_file(p, 16, v16, extra=[("BSCALE", "2.5D0"), ("BZERO", "-1.0"), ("BLANK", "-32768")])
    got = fits.read(p)
    want = -1.0 + 2.5 * v16.astype(float)
    want[v16 == -32768] = -666.0
    assert np.array_equal(got, want)

    v8 = np.array([[0, 255], [17, 128]], dtype=np.uint8)
    p8 = str(tmp_path / "u8.fits")
    hand_file(p8, 8, v8)
    assert np.array_equal(fits.read(p8), v8.astype(float))

    v32 = np.array([[2 ** 31 - 1], [-(2 ** 31)]], dtype=np.int32)
    p32 = str(tmp_path / "i32.fits")
    hand_file(p32, 32, v32, extra=[("BZERO", "2147483648")])
    assert np.array_equal(fits.read(p32), v32.astype(float) + 2147483648.0)

    v64 = np.array([[2 ** 40, -5]], dtype=np.int64)
    p64 = str(tmp_path / "i64.fits")
    hand_file(p64, 64, v64)
    assert np.array_equal(fits.read(p64), v64.astype(float))

    vf = np.array([[1.5, np.nan], [-2.25, 3e38]], dtype=np.float32)
    pf = str(tmp_path / "f32.fits")
    hand_file(pf, -32, vf)
    want = vf.astype(float)
    want[np.isnan(want)] = -666.0
    assert np.array_equal(fits.read(pf), want)

    vd = np.array([[np.nan, 1.0]])
    pd = str(tmp_path / "f64.fits")
    hand_file(pd, -64, vd)
    assert np.array_equal(fits.read(pd), [[-666.0, 1.0]])


@pytest.mark.parametrize("bitpix,extra", [(-64, ()), (-64, (("BSCALE", "0.5"), ("BZERO", "3"))),
                                          (-32, ()), (16, (("BLANK", "7"),))])
def test_reads_span_chunks(tmp_path, bitpix, extra):
    """300 x 1001 values: more than two of the reader's 131072-value chunks
    and a ragged last one, through the in-place (8-byte) and staged paths."""
    rng = np.random.default_rng(abs(bitpix) + len(extra))
    shape = (300, 1001)
    if bitpix == 16:
        v = rng.integers(-300, 300, shape).astype(np.int16)
    else:
        v = rng.standard_normal(shape).astype(np.float32 if bitpix == -32 else np.float64)
        v.reshape(-1)[[0, 131071, 131072, 262144, v.size - 1]] = np.nan
    p = str(tmp_path / "big.fits")
    hand_file(p, bitpix, v, extra=list(extra))
    kv = dict(extra)
    want = float(kv.get("BZERO", 0)) + float(kv.get("BSCALE", 1)) * v.astype(np.float64)
    null = np.isnan(want) if bitpix < 0 else v == int(kv["BLANK"])
    want[null] = -666.0
    got = fits.read(p)
    assert np.array_equal(got, want)


def test_long_header_and_one_axis(tmp_path):
    v = np.arange(10, dtype=float)
    p = str(tmp_path / "long.fits")
    hand_file(p, -64, v, comments=60)  # the header spans three blocks
    assert fits.size(p) == (10, 1, -64)
    assert np.array_equal(fits.read(p)[:, 0], v)


def test_overwrite_replaces_the_file(tmp_path):
    p = str(tmp_path / "o.fits")
    fits.write(p, np.ones((100, 100)))
    fits.write(p, np.full((2, 3), 7.0))
    assert fits.size(p) == (2, 3, -64)
    assert np.array_equal(fits.read(p), np.full((2, 3), 7.0))


def test_errors(tmp_path):
    p = str(tmp_path / "e.fits")
    fits.write(p, np.zeros((4, 5)))
    with pytest.raises(ImcomError) as e:
        fits.read(p, shape=(5, 4))
    assert e.value.status == IMCOM_ERR_FITS and "NAXIS1" in str(e.value)
    with pytest.raises(ImcomError) as e:
        fits.size(str(tmp_path / "missing.fits"))
    assert e.value.status == IMCOM_ERR_FITS
    bad = tmp_path / "bad.fits"
    bad.write_bytes(b"NOT A FITS FILE".ljust(2880))
    with pytest.raises(ImcomError, match="SIMPLE"):
        fits.size(str(bad))
    trunc = tmp_path / "trunc.fits"
    raw = open(p, "rb").read()
    trunc.write_bytes(raw[:2880 + 40])
    with pytest.raises(ImcomError, match="end early"):
        fits.read(str(trunc))
    noend = tmp_path / "noend.fits"
    noend.write_bytes(raw[:80 * 3])
    with pytest.raises(ImcomError, match="END"):
        fits.size(str(noend))


@pytest.mark.parametrize("name", ["test1", "x2", "ideal_output"])
def test_reference_example_files(tmp_path, name):
    """The reference's example inputs (written by its CFITSIO tooling): the
    library reads them bit for bit, and its writer reproduces every card's
    key and value columns, the header padding and the data records byte for
    byte (only the card comments differ)."""
    gold = np.load(EXAMPLES)
    header = gold[f"{name}_header"].tobytes()
    image = np.asfortranarray(gold[f"{name}_image"])
    data = image.ravel(order="F").astype(">f8").tobytes()
    data += b"\0" * ((-len(data)) % 2880)
    assert hashlib.sha256(data).hexdigest() == str(gold[f"{name}_data_sha256"])
    p = tmp_path / f"{name}.fits"
    p.write_bytes(header + data)
    assert fits.size(str(p)) == (image.shape[0], image.shape[1], -64)
    got = fits.read(str(p))
    assert np.array_equal(got.view(np.uint64), image.view(np.uint64))
    q = str(tmp_path / "again.fits")
    fits.write(q, got)
    again = open(q, "rb").read()
    assert len(again) == len(header) + len(data) and again[2880:] == data
    for i in range(36):
        ref, card = header[80 * i:80 * i + 80], again[80 * i:80 * i + 80]
        assert card[:30] == ref[:30]
        if ref.startswith(b"END "):
            break
    assert again[80 * i:2880] == header[80 * i:2880]
