"""Hyperdrive-format source lists: the reader and writer against the
reference's own test files (tests/golden/srclist_files.json, generated from
the reference tree by tests/golden/make_golden.py), round trips, and the
reader's checks.  No GPU."""

import json
import math
from pathlib import Path

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import srclist_io as io

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "srclist_files.json").read_text())["lists"]


@pytest.mark.parametrize("name,fmt", [("hyperdrive_srclist.yaml", "yaml"), ("hyperdrive_srclist.json", "json")])
def test_reference_lists_read_and_write_back_to_the_same_text(name, fmt):
    """The reference's write tests produce these files' text from an in-code
    list (general_tests.rs:731-779); reading them and writing them again
    must give the same text."""
    g = GOLDEN[name]
    s = io.parse_source_list(g["text"], fmt)
    assert len(s) == g["num_sources"]
    assert sum(len(src.components) for src in s.values()) == g["num_components"]
    out = io.to_yaml(s) if fmt == "yaml" else io.to_json(s)
    assert out == g["text"] if fmt == "json" else out.strip() == g["text"].strip()


def test_reference_list_contents():
    s = io.parse_source_list(GOLDEN["hyperdrive_srclist.yaml"]["text"])
    a, b = s["super_sweet_source1"], s["super_sweet_source2"]
    c = a.components[0]
    assert c.ra == math.radians(10.0) and c.dec == math.radians(-27.0)
    assert isinstance(c.comp_type, sl.Point)
    assert [f.freq for f in c.flux_type.fds] == [150e6, 170e6]
    assert (c.flux_type.fds[1].q, c.flux_type.fds[1].u, c.flux_type.fds[1].v) == (1.0, 2.0, 3.0)
    g, sh = b.components
    assert isinstance(g.comp_type, sl.Gaussian)
    assert g.comp_type.maj == math.radians(20.0) / 3600.0 and g.comp_type.pa == math.radians(75.0)
    assert isinstance(g.flux_type, sl.PowerLaw) and g.flux_type.si == -0.8
    assert isinstance(sh.comp_type, sl.Shapelet)
    assert [(k.n1, k.n2, k.value) for k in sh.comp_type.coeffs] == [(0, 1, 0.5)]
    assert isinstance(sh.flux_type, sl.CurvedPowerLaw) and sh.flux_type.q == 0.2
    assert io.parse_source_list(GOLDEN["hyperdrive_srclist.json"]["text"], "json") == s


def close(a: sl.SourceList, b: sl.SourceList) -> bool:
    """Equal up to the last bit of the degree <-> radian conversions."""
    if list(a.keys()) != list(b.keys()):
        return False

    def flat(x):
        return json.dumps(io.to_mapping(x), sort_keys=True)

    fa, fb = json.loads(flat(a)), json.loads(flat(b))

    def cmp(u, v):
        if isinstance(u, dict):
            return u.keys() == v.keys() and all(cmp(u[k], v[k]) for k in u)
        if isinstance(u, list):
            return len(u) == len(v) and all(cmp(p, q) for p, q in zip(u, v))
        if isinstance(u, float):
            return math.isclose(u, v, rel_tol=1e-13, abs_tol=1e-12)
        return u == v

    return cmp(fa, fb)


def test_all_kinds_round_trip():
    """general_tests.rs:369-385: nine sources of every component and flux
    type survive a write/read round trip (the file writes 150 MHz as 150e6,
    which YAML 1.1 readers see as text; it must still read as a number)."""
    s = io.parse_source_list(GOLDEN["srclist_all_kinds.yaml"]["text"])
    assert len(s) == 9
    assert s["point-list"].components[0].flux_type.fds[0].freq == 150e6
    for text, fmt in [(io.to_yaml(s), "yaml"), (io.to_json(s), "json")]:
        assert close(io.parse_source_list(text, fmt), s)


def random_list(seed):
    rng = np.random.default_rng(seed)
    out = sl.SourceList()
    for k in range(12):
        comps = []
        for _ in range(int(rng.integers(1, 4))):
            ra, dec = float(rng.uniform(0, 2 * math.pi)), float(rng.uniform(-math.pi / 2, math.pi / 2))
            fd = sl.FluxDensity(float(rng.uniform(1e8, 3e8)), float(rng.lognormal()), float(rng.normal() * 0.1), 0.0,
                                float(rng.normal() * 0.01))
            ft = [sl.PowerLaw(float(rng.normal(-0.8, 0.2)), fd), sl.CurvedPowerLaw(-0.7, fd, float(rng.normal(0, 0.2))),
                  sl.FluxList([fd, sl.FluxDensity(fd.freq * 1.3, fd.i * 0.8)])][k % 3]
            ct = [sl.Point(), sl.Gaussian(1e-4, 5e-5, 0.3),
                  sl.Shapelet(1e-4, 5e-5, 0.3, [sl.ShapeletCoeff(int(rng.integers(0, 6)), int(rng.integers(0, 6)),
                                                                  float(rng.normal())) for _ in range(4)])][k % 3]
            comps.append(sl.SourceComponent(ra, dec, ct, ft))
        out[f"src{k:02d}"] = sl.Source(comps)
    return out


@pytest.mark.parametrize("fmt", ["yaml", "json"])
def test_round_trip_files(tmp_path, fmt):
    s = random_list(3)
    p = tmp_path / f"list.{fmt}"
    io.write_source_list(s, p)
    t = io.read_source_list(p)
    assert close(t, s)
    io.write_source_list(s, p, num_sources=5)
    assert list(io.read_source_list(p).keys()) == list(s.keys())[:5]


@pytest.mark.parametrize("bad", [
    "a:\n- ra: 360.0\n  dec: 0.0\n  comp_type: point\n  flux_type:\n    list:\n    - freq: 1.0e8\n      i: 1.0\n",
    "a:\n- ra: 10.0\n  dec: -91.0\n  comp_type: point\n  flux_type:\n    list:\n    - freq: 1.0e8\n      i: 1.0\n",
    "a:\n- ra: 10.0\n  dec: 0.0\n  comp_type: disc\n  flux_type:\n    list:\n    - freq: 1.0e8\n      i: 1.0\n",
    "a:\n- ra: 10.0\n  dec: 0.0\n  comp_type: point\n  flux_type:\n    list: []\n",
    "a: []\n",
])
def test_reader_rejects_bad_lists(bad):
    with pytest.raises(io.SourceListError):
        io.parse_source_list(bad)
