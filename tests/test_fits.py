"""FITS map output (lt_write_fits): the reference's primary-image layout, read back with
the package's reader.  CPU only (host code)."""
import numpy as np

from lenstool_hpc_b200.fits import read_fits, write_fits


def test_fits_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.normal(0., 10., (37, 53))
    img[3, 4] = 1e30
    frame = (-100., 100., -50., 75.)
    p = tmp_path / "map.fits"
    write_fits(p, img, frame)
    raw = p.read_bytes()
    assert len(raw) % 2880 == 0
    hdr, data = read_fits(p)
    # the reference's keywords, in its order (src/module_writeFits.cpp:113-206)
    assert hdr["_order"][:6] == ["SIMPLE", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2", "EXTEND"]
    assert hdr["_order"][6:] == ["BZERO", "BSCALE", "CRVAL1", "CRPIX1", "CDELT1", "CUNIT1", "CTYPE1", "CRVAL2",
                                 "CRPIX2", "CDELT2", "CUNIT2", "CTYPE2", "ORIGIN", "DATE"]
    assert hdr["SIMPLE"] is True and hdr["BITPIX"] == -32 and hdr["NAXIS1"] == 53 and hdr["NAXIS2"] == 37
    assert hdr["CRVAL1"] == -100. and hdr["CRPIX1"] == 1. and hdr["CRVAL2"] == -50.
    # float keywords carry 7 significant digits of the float32 value (cfitsio's format)
    assert hdr["CDELT1"] == float("%.7G" % np.float32(200. / 52))
    assert hdr["CDELT2"] == float("%.7G" % np.float32(125. / 36))
    assert hdr["CUNIT1"] == "arcsec" and hdr["CTYPE2"] == "LINEAR" and hdr["ORIGIN"] == "JPK-SOFT"
    assert np.array_equal(data, img.astype(np.float32))
    # every header card is 80 printable ASCII characters
    head = raw[:raw.index(b"END" + b" " * 77) + 80]
    assert len(head) % 80 == 0 and all(32 <= b < 127 for b in head)


def test_fits_rejects_bad_input(tmp_path):
    import pytest
    import lenstool_hpc_b200 as lt
    with pytest.raises(lt.LensError):
        write_fits(tmp_path / "x.fits", np.zeros((1, 5)), (0., 1., 0., 1.))
    with pytest.raises(lt.LensError):
        write_fits(tmp_path / "no" / "such" / "dir.fits", np.zeros((4, 4)), (0., 1., 0., 1.))


def _independent_read(raw: bytes):
    """A minimal reader written from the FITS standard alone (not the package's): 80-byte
    cards in 2880-byte blocks up to END, then NAXIS2 x NAXIS1 big-endian IEEE values of
    BITPIX -32, scaled by BSCALE and BZERO."""
    cards = {}
    pos = 0
    while True:
        card = raw[pos:pos + 80].decode("ascii")
        pos += 80
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= ":
            val = card[10:].split("/")[0].strip()
            cards[key] = val.strip("'").strip() if val.startswith("'") else val
    pos = (pos + 2879) // 2880 * 2880
    nx, ny = int(cards["NAXIS1"]), int(cards["NAXIS2"])
    assert int(cards["BITPIX"]) == -32
    data = np.frombuffer(raw[pos:pos + 4 * nx * ny], dtype=">f4").reshape(ny, nx)
    return cards, data.astype(np.float64) * float(cards.get("BSCALE", 1.)) + float(cards.get("BZERO", 0.))


def test_fits_independent_reader(tmp_path):
    """The written file read by a reader independent of the package's: the same image,
    keyword values and a data block padded to 2880 bytes."""
    rng = np.random.default_rng(4)
    img = rng.normal(0., 3., (29, 41))
    frame = (-20., 20., -10., 18.)
    p = tmp_path / "map.fits"
    write_fits(p, img, frame)
    raw = p.read_bytes()
    cards, data = _independent_read(raw)
    assert cards["SIMPLE"] == "T" and int(cards["NAXIS"]) == 2
    assert float(cards["CRVAL1"]) == -20. and float(cards["CRVAL2"]) == -10.
    assert np.array_equal(data, img.astype(np.float32).astype(np.float64))
    hdr, data2 = read_fits(p)
    assert np.array_equal(data2, data.astype(np.float32))
