"""The FITS binary-table reader / writer that feeds survey catalogs to the device."""
import numpy as np
import pytest


def test_round_trip_and_layout(tmp_path):
    from cosmonpc_b200 import fits

    rng = np.random.default_rng(0)
    cols = {"RA": rng.random(777) * 360, "Z": rng.random(777).astype(np.float32),
            "ID": np.arange(777, dtype=np.int64), "FLAG": rng.integers(0, 5, 777).astype(np.int16),
            "N": rng.integers(0, 9, 777).astype(np.int32), "B": rng.integers(0, 255, 777).astype(np.uint8)}
    p = tmp_path / "t.fits"
    fits.write_table(str(p), cols)
    assert p.stat().st_size % fits.BLOCK == 0
    t = fits.open_table(str(p))
    assert t.nrows == 777 and t.row_bytes == 8 + 4 + 8 + 2 + 4 + 1
    assert [t.columns[c].offset for c in cols] == [0, 8, 12, 20, 22, 26]
    r = t.read_columns(list(cols))
    for k, v in cols.items():
        np.testing.assert_array_equal(r[k], v)
    rows = np.asarray(t.rows())
    assert rows.shape == (777, t.row_bytes)
    # big-endian on disk
    assert rows[5, 0:8].tobytes() == np.array([cols["RA"][5]], dtype=">f8").tobytes()
    sub = t.read_columns(["Z"], rows=np.arange(10, 20))
    np.testing.assert_array_equal(sub["Z"], cols["Z"][10:20])


def test_header_scaling_and_hdu_choice(tmp_path):
    from cosmonpc_b200 import fits

    # hand-written table with TZERO/TSCAL on an int16 column
    cards = [fits._card("XTENSION", "BINTABLE"), fits._card("BITPIX", 8), fits._card("NAXIS", 2),
             fits._card("NAXIS1", 10), fits._card("NAXIS2", 3), fits._card("PCOUNT", 0),
             fits._card("GCOUNT", 1), fits._card("TFIELDS", 2), fits._card("TTYPE1", "A"),
             fits._card("TFORM1", "1D"), fits._card("TTYPE2", "S"), fits._card("TFORM2", "I"),
             fits._card("TSCAL2", 0.5), fits._card("TZERO2", 32768.0)]
    data = np.zeros(3, dtype=[("A", ">f8"), ("S", ">i2")])
    data["A"] = [1.5, -2.0, 3.25]
    data["S"] = [-32768, 0, 100]
    p = tmp_path / "s.fits"
    with open(p, "wb") as f:
        f.write(fits._header_bytes([fits._card("SIMPLE", True), fits._card("BITPIX", 8), fits._card("NAXIS", 0),
                                    fits._card("EXTEND", True)]))
        f.write(fits._header_bytes(cards))
        b = data.tobytes()
        f.write(b + b"\0" * ((-len(b)) % fits.BLOCK))
    t = fits.open_table(str(p))
    r = t.read_columns(["A", "S"])
    np.testing.assert_array_equal(r["A"], [1.5, -2.0, 3.25])
    np.testing.assert_array_equal(r["S"], 32768.0 + 0.5 * np.array([-32768, 0, 100]))
    assert len(fits.hdu_list(str(p))) == 2


def test_rejects_non_fits(tmp_path):
    from cosmonpc_b200 import fits

    p = tmp_path / "x.fits"
    p.write_bytes(b"X" * 2880)
    with pytest.raises(ValueError):
        fits.open_table(str(p))


def test_weight_rules_follow_reference():
    from cosmonpc_b200 import _lib, survey

    names = ["RA", "DEC", "Z", "WEIGHT_FKP", "WEIGHT_SYSTOT", "WEIGHT_NOZ", "WEIGHT_CP"]
    assert survey._weight_rule(names + ["WEIGHT"], {"scheme": "boss", "name_alias": "X"}, "data") == \
        (_lib.W_COLUMN, "WEIGHT")
    assert survey._weight_rule(names, {"scheme": None, "name_alias": None}, "data") == (_lib.W_ONE, None)
    assert survey._weight_rule(names, {"scheme": "boss", "name_alias": None}, "data")[0] == _lib.W_BOSS
    assert survey._weight_rule(names, {"scheme": "boss", "name_alias": None}, "randoms")[0] == _lib.W_ONE
    assert survey._weight_rule(names, {"scheme": "eboss", "name_alias": None}, "data")[0] == _lib.W_EBOSS
    assert survey._weight_rule(names, {"scheme": None, "name_alias": "WEIGHT_CP"}, "data") == \
        (_lib.W_COLUMN, "WEIGHT_CP")
    with pytest.raises(ValueError, match="DESI"):
        survey._weight_rule(names, {"scheme": "desi", "name_alias": None}, "data")
    with pytest.raises(AssertionError):
        survey._weight_rule(names, {"scheme": "sdss", "name_alias": None}, "data")


def test_oracle_comoving_distance_against_quadrature():
    from scipy.integrate import quad

    from oracle.survey import comoving_distance

    h, om = 0.6766, 0.31
    z = np.array([0.0, 0.01, 0.2, 0.5, 0.8, 1.5, 3.0])
    ref = np.array([quad(lambda t: 1 / np.sqrt(om * (1 + t) ** 3 + 1 - om), 0, zi, epsabs=1e-15, epsrel=1e-13)[0]
                    for zi in z]) * 299792.458 / (100 * h) * h
    np.testing.assert_allclose(comoving_distance(z, h, om), ref, rtol=1e-13, atol=1e-10)
