"""The FITS maps the drop-in write_map (and so MLmap/MTmap) writes, checked card
by card with a parser of this file that shares nothing with the library's own
reader, against the layout the reference's write_map gets from CFITSIO
(mappraiser/src/iofiles.c:19-52): a primary array with no data (BITPIX 16,
NAXIS 0, EXTEND, the creation DATE), then a binary table of 12 nside^2 rows
whose one column SIGNAL is 8-byte doubles (format 1D; integer maps are
converted into it), PIXTYPE HEALPIX, ORDERING, NSIDE, COORDSYS and the
coordinate-system comment.  Host code only: no GPU."""
import re

import numpy as np
import pytest


def _cards(block_bytes):
    assert len(block_bytes) % 2880 == 0
    text = block_bytes.decode("ascii")
    return [text[i:i + 80] for i in range(0, len(text), 80)]


def _parse(path):
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    hdus, pos = [], 0
    for _ in range(2):
        cards = []
        while True:
            blk = _cards(raw[pos:pos + 2880])
            pos += 2880
            cards += blk
            if any(c.startswith("END ") or c.rstrip() == "END" for c in blk):
                break
        keys = []
        for c in cards:
            assert len(c) == 80 and all(32 <= ord(ch) < 127 for ch in c)
            key = c[:8].rstrip()
            if key == "END":
                break
            if c[8:10] == "= ":
                val = c[10:].split(" / ")[0].strip()
                keys.append((key, val))
            else:
                keys.append((key, c[8:].rstrip()))
        hdus.append(keys)
    return hdus, raw[pos:]


@pytest.mark.parametrize("kind", ["double", "int"])
@pytest.mark.parametrize("nest", [1, 0])
def test_write_map_layout(tmp_path, kind, nest):
    import midapack_b200 as mb
    nside = 4
    npix = 12 * nside * nside
    rng = np.random.default_rng(2)
    data = rng.standard_normal(npix) if kind == "double" else rng.integers(-5, 1000, npix).astype(np.int32)
    path = str(tmp_path / "m.fits")
    mb.lib().write_map(data.ctypes.data, 82 if kind == "double" else 31, nside, path.encode(),
                       b"\x01" if nest else b"\x00", b"G")
    (prim, ext), payload = _parse(path)
    pk = [k for k, _ in prim]
    assert pk[:4] == ["SIMPLE", "BITPIX", "NAXIS", "EXTEND"]
    d = dict(prim)
    assert d["SIMPLE"] == "T" and d["BITPIX"] == "16" and d["NAXIS"] == "0" and d["EXTEND"] == "T"
    assert re.fullmatch(r"'\d{4}-\d\d-\d\dT\d\d:\d\d:\d\d'", d["DATE"])
    ek = [k for k, _ in ext]
    assert ek[:8] == ["XTENSION", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2", "PCOUNT", "GCOUNT", "TFIELDS"]
    e = dict(ext)
    assert e["XTENSION"] == "'BINTABLE'" and e["BITPIX"] == "8" and e["NAXIS"] == "2"
    assert e["NAXIS1"] == "8" and e["NAXIS2"] == str(npix) and e["PCOUNT"] == "0" and e["GCOUNT"] == "1"
    assert e["TFIELDS"] == "1" and e["TTYPE1"].strip("'").strip() == "SIGNAL"
    assert e["TFORM1"].strip("'").strip() == "1D"
    assert e["EXTNAME"].strip("'").strip() == "BINTABLE" and e["PIXTYPE"].strip("'").strip() == "HEALPIX"
    assert e["ORDERING"].strip("'").strip() == ("NESTED" if nest else "RING")
    assert e["NSIDE"] == str(nside) and e["COORDSYS"].strip("'").strip() == "G"
    assert any(k == "COMMENT" and "Galactic" in v for k, v in ext)
    vals = np.frombuffer(payload, dtype=">f8", count=npix)
    np.testing.assert_array_equal(vals, data.astype(np.float64))
    assert not any(payload[8 * npix:])  # zero padding to the 2880-byte block
