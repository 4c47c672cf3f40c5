"""Calibration-solutions files: the hyperdrive FITS format
(solutions/hyperdrive.rs) and the AO binary format (solutions/ao.rs),
written and read back as the reference's own tests do
(solutions/tests.rs:13-317), the FITS layer against the standard's block and
card rules and against an independent writer (astropy-written FITS files
of the reference's test tree, tests/golden/fits_srclists.json).  No GPU."""

import base64
import json
import math
import struct
from pathlib import Path

import numpy as np
import pytest

from mwa_hyperdrive_b200 import fits
from mwa_hyperdrive_b200 import solutions as S

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "fits_srclists.json").read_text())["lists"]


def make_solutions(ntb=2, ntiles=128, nch=768):
    """The reference's test solutions (solutions/tests.rs:13-100): Jones
    (1.01+1.02i, 1.03+1.04i, 1.05+1.06i, 1.07+1.08i) x 1, 2, 3, ...; tiles
    3-4 and chanblocks 5-7 NaN."""
    v = np.arange(1.0, ntb * ntiles * nch + 1).reshape(ntb, ntiles, nch, 1)
    dj = v * np.array([1.01, 1.02, 1.03, 1.04, 1.05, 1.06, 1.07, 1.08])
    dj[:, 3:5] = np.nan
    dj[:, :, 5:8] = np.nan
    nbl = ntiles * (ntiles - 1) // 2
    return S.CalibrationSolutions(
        di_jones=dj, flagged_tiles=[3, 4], flagged_chanblocks=[5, 6, 7],
        chanblock_freqs=np.array([(i + 10) * 10.0 for i in range(nch)]), obsid=1090008640,
        start_timestamps=[1090008640.0, 1090008650.0], end_timestamps=[1090008650.0, 1090008660.0],
        average_timestamps=[1090008645.0, 1090008655.0], max_iterations=30, stop_threshold=1e-10,
        min_threshold=1e-5, raw_data_corrections=S.RawDataCorrections("cotter2014", True, False, False),
        tile_names=[f"tile{i:03d}" for i in range(ntiles)], dipole_gains=np.ones((ntiles, 32)),
        dipole_delays=np.zeros((ntiles, 16), np.uint32), beam_file=None,
        calibration_results=np.full((ntb, nch), 1e-6), baseline_weights=np.arange(nbl, dtype=np.float64),
        uvw_min=82.0, uvw_max=math.inf, freq_centroid=182e6, modeller="CPU")


def same_jones(a, b):
    nan = np.isnan(a).any(axis=-1)
    assert np.array_equal(nan, np.isnan(b).any(axis=-1))
    np.testing.assert_array_equal(a[~nan], b[~nan])


def test_fits_round_trip_with_metadata(tmp_path):
    s = make_solutions()
    p = tmp_path / "sols.fits"
    S.write_solutions(s, p)
    r = S.read_solutions(p)
    same_jones(s.di_jones, r.di_jones)
    assert r.raw_data_corrections == s.raw_data_corrections
    assert r.max_iterations == 30 and r.stop_threshold == 1e-10 and r.min_threshold == 1e-5
    assert r.flagged_tiles == [3, 4] and r.flagged_chanblocks == [5, 6, 7]
    assert r.start_timestamps == s.start_timestamps and r.end_timestamps == s.end_timestamps
    assert r.average_timestamps == s.average_timestamps
    np.testing.assert_array_equal(r.chanblock_freqs, s.chanblock_freqs)
    np.testing.assert_array_equal(r.baseline_weights, s.baseline_weights)
    assert r.tile_names == s.tile_names
    np.testing.assert_array_equal(r.dipole_gains, s.dipole_gains)
    np.testing.assert_array_equal(r.dipole_delays, s.dipole_delays)
    np.testing.assert_array_equal(r.calibration_results, s.calibration_results)
    assert r.obsid == 1090008640 and r.modeller == "CPU"
    assert r.uvw_min == 82.0 and r.uvw_max == math.inf
    assert r.freq_centroid == pytest.approx(182e6, rel=1e-15)


def test_fits_round_trip_without_metadata(tmp_path):
    """solutions/tests.rs:110-190: only the Jones matrices and the flags."""
    full = make_solutions()
    s = S.CalibrationSolutions(di_jones=full.di_jones, flagged_tiles=[3, 4], flagged_chanblocks=[5, 6, 7])
    p = tmp_path / "sols.fits"
    S.write_fits(s, p)
    r = S.read_fits(p)
    same_jones(s.di_jones, r.di_jones)
    assert r.flagged_tiles == [3, 4] and r.flagged_chanblocks == [5, 6, 7]
    for k in ("raw_data_corrections", "max_iterations", "stop_threshold", "min_threshold", "start_timestamps",
              "end_timestamps", "average_timestamps", "chanblock_freqs", "baseline_weights", "tile_names",
              "calibration_results", "uvw_min", "uvw_max", "freq_centroid", "modeller", "obsid"):
        assert getattr(r, k) is None, k


def test_fits_layout(tmp_path):
    """2880-byte blocks, 80-column ASCII cards, mandatory keywords first and
    in order, data big-endian with NAXIS1 the fastest axis."""
    s = make_solutions(ntb=1, ntiles=4, nch=3)
    s.beam_file = "/a/very/long/path/" + "x" * 120 + "/mwa_full_embedded_element_pattern.h5"
    p = tmp_path / "sols.fits"
    S.write_fits(s, p)
    b = p.read_bytes()
    assert len(b) % 2880 == 0
    assert all(32 <= c < 127 for c in b[:2880])
    cards = [b[i:i + 80].decode() for i in range(0, 2880, 80)]
    assert [c[:8].strip() for c in cards[:4]] == ["SIMPLE", "BITPIX", "NAXIS", "EXTEND"]
    prim, hdus = fits.decode(b)
    assert prim["BEAMFILE"] == s.beam_file  # CONTINUE long string
    sol = fits.find(hdus, "SOLUTIONS")
    assert [sol.header[f"NAXIS{i}"] for i in range(1, 5)] == [8, 3, 4, 1]
    assert sol.header["BITPIX"] == -64
    # the first element of the image sits right after its header, big-endian
    off = b.index(b"XTENSION= 'IMAGE   '")
    hdr_end = off + 2880 * ((len(sol.header.encode())) // 2880)
    assert struct.unpack(">d", b[hdr_end:hdr_end + 8])[0] == s.di_jones[0, 0, 0, 0]
    cb = fits.find(hdus, "CHANBLOCKS")
    assert cb.columns == [("Index", "J"), ("Flag", "1X"), ("Freq", "D")]
    tl = fits.find(hdus, "TILES")
    assert [c[0] for c in tl.columns] == ["Antenna", "Flag", "TileName", "DipoleGains", "DipoleDelays"]


def test_ao_round_trip(tmp_path):
    s = make_solutions(ntb=2, ntiles=16, nch=24)
    p = tmp_path / "sols.bin"
    S.write_solutions(s, p)
    b = p.read_bytes()
    assert b[:7] == b"MWAOCAL" and b[7:16] == bytes(9)
    assert struct.unpack("<4I2d", b[16:48]) == (2, 16, 24, 4, 1090008640.0, 1090008660.0)
    assert len(b) == 48 + 2 * 16 * 24 * 64
    r = S.read_solutions(p)
    same_jones(s.di_jones, r.di_jones)
    assert r.flagged_tiles == [3, 4] and r.flagged_chanblocks == [5, 6, 7]
    assert r.start_timestamps == [1090008640.0] and r.end_timestamps == [1090008660.0]
    assert r.average_timestamps == [1090008650.0]


def test_bad_files(tmp_path):
    p = tmp_path / "x.bin"
    p.write_bytes(b"NOTOCAL" + bytes(41))
    with pytest.raises(S.SolutionsError):
        S.read_ao(p)
    with pytest.raises(S.SolutionsError):
        S.read_solutions(tmp_path / "x.txt")
    with pytest.raises(S.SolutionsError):
        S.write_solutions(make_solutions(1, 4, 3), tmp_path / "x.uvfits")


@pytest.mark.parametrize("stem", ["jack", "lobes", "gleam"])
def test_fits_reader_on_an_independent_writer(stem):
    """Binary tables written by astropy (the reference's FITS source lists):
    every HDU decodes, column widths add up to NAXIS1, and the values agree
    with the YAML list holding the same sources."""
    b = base64.b64decode(GOLDEN[stem]["fits_base64"])
    prim, hdus = fits.decode(b)
    assert prim["SIMPLE"] is True
    for h in hdus:
        assert h.kind == "BINTABLE"
        rows = h.header["NAXIS2"]
        for name, _ in h.columns:
            assert len(h.data[name]) == rows
    if stem == "jack":
        import yaml

        y = yaml.safe_load(GOLDEN[stem]["yaml"])
        t = hdus[0].data
        for k, src in enumerate(t["UNQ_SOURCE_ID"]):
            comp = y[src][int(t["NAME"][k].rsplit("_C", 1)[1])]
            assert comp["ra"] == pytest.approx(t["RA"][k], abs=1e-12)
            assert comp["dec"] == pytest.approx(t["DEC"][k], abs=1e-12)
        shp = hdus[1].data
        assert list(shp["N1"][:3]) == [0, 0, 1] and list(shp["N2"][:3]) == [0, 1, 0]
