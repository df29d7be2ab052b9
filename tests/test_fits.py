"""FITS cube writer (CPU): header cards and data read back with a minimal
parser of the FITS standard (2880-byte blocks, 80-character cards, big-endian
IEEE floats)."""
import math

import numpy as np

from mtb.fits import FitsCube


def read_fits(path):
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    cards, i = {}, 0
    while True:
        c = raw[i:i + 80].decode("ascii")
        i += 80
        if c.startswith("END"):
            break
        if c[8:10] == "= ":
            v = c[10:].strip()
            if v.startswith("'"):
                v = v[1:v.index("'", 1)].strip()     # quoted string (may contain '/')
            else:
                v = v.split("/")[0].strip()
            cards[c[:8].strip()] = v
    start = (i + 2879) // 2880 * 2880
    shape = [int(cards["NAXIS%d" % k]) for k in range(int(cards["NAXIS"]), 0, -1)]
    data = np.frombuffer(raw[start:start + 4 * int(np.prod(shape))], ">f4").reshape(shape)
    return cards, data


def test_fits_cube_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    nx, ny, nch = 48, 32, 3
    dl = 2.0 / 3600 * math.pi / 180
    freqs = np.array([1.3e9, 1.4e9, 1.5e9])
    imgs = rng.standard_normal((nch, 4, ny, nx)).astype(np.float32)
    path = tmp_path / "cube.fits"
    with FitsCube(path, nx, ny, freqs, dl, ra_deg=120.5, dec_deg=-45.25, telescope="MeerKAT",
                  obs_mjd=60000.5) as f:
        for c in (2, 0, 1):                    # any order
            f.write(c, imgs[c])
    cards, data = read_fits(path)
    assert cards["SIMPLE"] == "T" and int(cards["BITPIX"]) == -32
    assert [int(cards["NAXIS%d" % k]) for k in (1, 2, 3, 4)] == [nx, ny, 4, nch]
    assert cards["CTYPE1"] == "RA---SIN" and cards["CTYPE2"] == "DEC--SIN"
    assert cards["CTYPE3"] == "STOKES" and cards["CTYPE4"] == "FREQ"
    assert math.isclose(float(cards["CDELT1"]), -2.0 / 3600, rel_tol=1e-12)
    assert math.isclose(float(cards["CDELT2"]), 2.0 / 3600, rel_tol=1e-12)
    assert float(cards["CRPIX1"]) == nx // 2 + 1 and float(cards["CRPIX2"]) == ny // 2 + 1
    assert float(cards["CRVAL1"]) == 120.5 and float(cards["CRVAL2"]) == -45.25
    assert float(cards["CRVAL3"]) == 1 and float(cards["CDELT3"]) == 1
    assert float(cards["CRVAL4"]) == 1.3e9 and float(cards["CDELT4"]) == 1e8
    assert cards["BUNIT"] == "JY/BEAM" and cards["TELESCOP"] == "MeerKAT"
    assert cards["DATE-OBS"].startswith("2023-02-25T12:00:00")
    assert np.array_equal(data, imgs)


def test_fits_single_stokes(tmp_path):
    img = np.arange(20, dtype=np.float32).reshape(1, 4, 5)
    path = tmp_path / "i.fits"
    with FitsCube(path, 5, 4, [1.4e9], 1e-5, stokes="I") as f:
        f.write(0, img)
    cards, data = read_fits(path)
    assert int(cards["NAXIS3"]) == 1 and int(cards["NAXIS4"]) == 1
    assert np.array_equal(data[0], img)


def test_fits_header_matches_expected_cards(tmp_path):
    """Every card of tests/golden/fits_header_iv_nonuniform.json: the header
    the reference's ImageManager::createFITS writes (ImageManager.cpp:68-108,
    132-188) for two circular polarisations (Stokes I, V) and a non-uniform
    channel list, restated card by card.  Numbers to 1e-12 relative."""
    import json
    import os
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fits_header_iv_nonuniform.json")))
    i = fx["input"]
    arcsec = math.pi / (180 * 3600)
    path = tmp_path / "iv.fits"
    imgs = np.random.default_rng(1).standard_normal((len(i["freqs_hz"]), 2, i["ny"], i["nx"])).astype(np.float32)
    with FitsCube(path, i["nx"], i["ny"], i["freqs_hz"], i["l_increment_arcsec"] * arcsec,
                  m_increment=i["m_increment_arcsec"] * arcsec, stokes=i["stokes"], ra_deg=i["ra_deg"],
                  dec_deg=i["dec_deg"], telescope=i["telescope"], observer=i["observer"],
                  obs_mjd=i["obs_mjd"]) as f:
        for c in range(len(i["freqs_hz"])):
            f.write(c, imgs[c])
    cards, data = read_fits(path)
    for key, want in fx["cards"].items():
        assert key in cards, key
        v = want["value"]
        if isinstance(v, str):
            assert cards[key] == v, (key, cards[key], v)
        else:
            assert math.isclose(float(cards[key]), float(v), rel_tol=1e-12, abs_tol=1e-300), (key, cards[key], v)
    for key in fx["present"]:
        assert key in cards, key
    # channel planes in list order, each [Stokes][m][l]
    assert data.shape == (4, 2, i["ny"], i["nx"]) and np.array_equal(data, imgs)


def test_fits_stokes_axis_codes(tmp_path):
    """The Stokes axis is linear in the FITS codes of the list
    ConfigurationManager.cpp:137-154 builds: I (1 pol), I Q (2 linear),
    I V (2 circular), I Q U V (4)."""
    for stokes, crval, cdelt in (("I", 1, 1), ("IQ", 1, 1), ("IV", 1, 3), ("IQUV", 1, 1)):
        path = tmp_path / ("s_%s.fits" % stokes)
        with FitsCube(path, 4, 4, [1.4e9], 1e-5, stokes=stokes) as f:
            f.write(0, np.zeros((len(stokes), 4, 4), np.float32))
        cards, _ = read_fits(path)
        assert int(cards["NAXIS3"]) == len(stokes)
        assert float(cards["CRVAL3"]) == crval and float(cards["CDELT3"]) == cdelt
