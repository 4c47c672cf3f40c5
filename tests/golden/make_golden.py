"""Regenerate the golden fixtures in this directory from the reference's own
known-answer tests.

Run in an environment that has the mwa_hyperdrive source tree (pass its root
as argv[1] or in HDC_REFERENCE_DIR); the outputs are committed so that nothing reads the reference at
test time.

* model_kats.json  -- expected no-beam visibilities (f32, epsilon 0 in the
  reference) from src/model/tests/mod.rs: the zenith / off-zenith list,
  power-law and curved-power-law cases (lines 351-444, 600-731, 887-1018), the
  two-component Gaussian and shapelet cases (1393-1569) and the shapelet UVWs
  (1530-1568).  Values are parsed from the Rust source text.
* srclist_files.json -- the reference's hyperdrive-format source-list test
  files (YAML and JSON) with their source and component counts.
* fits_srclists.json -- the reference's FITS-format source lists (written by
  astropy through test_files/gen_fits_srclists.py), base64, with the YAML
  lists that hold the same sources; they check the FITS reader against an
  independent FITS writer.
* ref_struct_layouts.json -- sizeof/offsetof of every drop-in FFI struct
  measured by compiling layout_probe.py's probe against the reference's
  src/gpu/types.h (FP64 build), and the parameter types of the reference's
  drop-in C functions as defined in src/gpu/{model,peel,utils}.cu.
* uvfits_sdc3.json -- the content of the reference's one uvfits test file
  (test_files/sdc3/sdc3_0000.uvfits: one timestep, one channel, XX only, one
  cross-correlation, 512 stations of SKA-Low with ARRAYX/Y/Z zero as casacore
  writes them) as its primary header card images, the group's values, and the
  AN table's keywords and the three columns a reader uses (ANNAME, STABXYZ,
  NOSTA), so that the test can rebuild the file; with the reference's expected
  values from src/io/read/uvfits/tests.rs:909-958 (test_sdc3).
* shapelet_basis_samples.json -- samples of the shapelet basis table produced
  by the reference's generator script src/model/make_shapelet_basis_values.py
  (imported, its gen_shape_basis evaluated at the sampled points), plus the
  reference's own table KATs (src/model/shapelets.rs:44-59).
"""

import importlib.util
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

CPLX = re.compile(r"Complex::new\(\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\)")
UVW = re.compile(r"UVW\s*\{\s*u:\s*([-+0-9.eE]+),\s*v:\s*([-+0-9.eE]+),\s*w:\s*([-+0-9.eE]+),?\s*\}")
IDENT = re.compile(r"Jones::identity\(\)(?:\s*\*\s*([-+0-9.eE]+))?")


def fn_body(src: str, name: str) -> str:
    start = src.index(f"fn {name}(")
    end = src.index("\n}\n", start)
    return src[start:end]


def parse_rows(body: str, nbl: int = 3):
    """Rows of Jones (as [re, im] * 4) for a test function that states its
    expectation per frequency row (`let expected_*` blocks)."""
    rows = []
    blocks = re.split(r"let expected", body)[1:]
    for blk in blocks:
        blk = blk.split("assert_abs_diff_eq")[0]
        cs = CPLX.findall(blk)
        if cs:
            vals = [[float(a), float(b)] for a, b in cs]
            assert len(vals) % 4 == 0
            jones = [vals[i : i + 4] for i in range(0, len(vals), 4)]
            rows.extend(jones[i : i + nbl] for i in range(0, len(jones), nbl))
        else:
            m = IDENT.search(blk)
            assert m, blk[:200]
            s = float(m.group(1)) if m.group(1) else 1.0
            j = [[s, 0.0], [0.0, 0.0], [0.0, 0.0], [s, 0.0]]
            rows.append([j] * nbl)
    return rows


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    src = (ref / "src/model/tests/mod.rs").read_text()
    out = {
        "source": "src/model/tests/mod.rs (mwa_hyperdrive 0.8.0)",
        "obs": {
            "phase_centre_deg": [0.0, -27.0],
            "off_phase_centre_deg": [1.0, -27.0],
            "freqs_hz": [150e6, 175e6, 200e6],
            "lst_rad": 0.0,
            "xyzs": [[0.0, 1.0, 0.0], [0.0, -1.0, 0.0], [1.0, 0.0, 0.0]],
        },
        "cases": {},
    }
    for name in [
        "test_list_zenith_visibilities",
        "test_list_off_zenith_visibilities",
        "test_power_law_zenith_visibilities",
        "test_power_law_off_zenith_visibilities",
        "test_curved_power_law_zenith_visibilities",
        "test_curved_power_law_off_zenith_visibilities",
        "test_multiple_gaussian_components",
    ]:
        rows = parse_rows(fn_body(src, name))
        assert len(rows) == 3 and all(len(r) == 3 for r in rows), name
        out["cases"][name] = rows

    body = fn_body(src, "test_multiple_shapelet_components")
    vis_part, uvw_part = body.split("assert_abs_diff_eq!(expected, vis", 1)
    cs = [[float(a), float(b)] for a, b in CPLX.findall(vis_part)]
    jones = [cs[i : i + 4] for i in range(0, len(cs), 4)]
    out["cases"]["test_multiple_shapelet_components"] = [jones[i : i + 3] for i in range(0, 9, 3)]
    uvws = [[float(a), float(b), float(c)] for a, b, c in UVW.findall(uvw_part)]
    assert len(uvws) == 6
    out["shapelet_uvws_bl_comp"] = [uvws[i : i + 2] for i in range(0, 6, 2)]
    (HERE / "model_kats.json").write_text(json.dumps(out, indent=1))

    # Shapelet basis: evaluate the reference generator's basis function.
    spec = importlib.util.spec_from_file_location("mk", ref / "src/model/make_shapelet_basis_values.py")
    gen_src = (ref / "src/model/make_shapelet_basis_values.py").read_text()
    # Import only the function definition (the script body writes files).
    ns: dict = {}
    exec(gen_src.split("max_x = 50")[0], ns)
    gen = ns["gen_shape_basis"]
    xlocs = np.linspace(-50, 50, 10001)
    rng = np.random.default_rng(7)
    samples = []
    for n in [0, 1, 2, 3, 5, 8, 13, 21, 40, 70, 100]:
        vals = gen(n, xlocs, beta=1.0)
        idx = sorted(set(rng.integers(3500, 6500, size=24).tolist() + [5000, 5001, 4999, 0, 10000]))
        for i in idx:
            samples.append([n, int(i), float(vals[i])])
    (HERE / "shapelet_basis_samples.json").write_text(
        json.dumps(
            {
                "source": "src/model/make_shapelet_basis_values.py gen_shape_basis; KATs src/model/shapelets.rs:44-59",
                "kat": {"index_5000": 1.0, "index_5001": 0.99995, "eps_5000": 1e-10, "eps_5001": 1e-8},
                "samples_n_index_value": samples,
            },
            indent=0,
        )
    )
    del spec

    # Source-list file-format vectors: the reference's hyperdrive YAML and JSON
    # test lists (whose text its write tests reproduce from an in-code list,
    # src/srclist/general_tests.rs:711-779) and the all-kinds list
    # (general_tests.rs:369-385: 9 sources survive a write/read round trip),
    # with their contents as a YAML-independent reader sees them.
    import yaml

    tf = ref / "test_files"
    lists = {}
    for name in ["hyperdrive_srclist.yaml", "hyperdrive_srclist.json", "srclist_all_kinds.yaml"]:
        text = (tf / name).read_text()
        parsed = json.loads(text) if name.endswith(".json") else yaml.safe_load(text)
        lists[name] = {"text": text, "num_sources": len(parsed),
                       "num_components": sum(len(v) for v in parsed.values())}
    (HERE / "srclist_files.json").write_text(
        json.dumps({"source": "test_files/{hyperdrive_srclist.yaml,hyperdrive_srclist.json,srclist_all_kinds.yaml}",
                    "lists": lists}, indent=1))

    # FITS files from an independent writer (astropy), and the YAML twins of
    # their sources.
    import base64

    fl = {}
    for stem in ["jack", "gleam", "lobes"]:
        fl[stem] = {"fits_base64": base64.b64encode((tf / f"{stem}.fits").read_bytes()).decode("ascii"),
                    "yaml": (tf / f"{stem}.yaml").read_text() if (tf / f"{stem}.yaml").exists() else None}
    (HERE / "fits_srclists.json").write_text(
        json.dumps({"source": "test_files/{jack,gleam,lobes}.{fits,yaml}", "lists": fl}, indent=1))


def layouts(ref_root: str) -> None:
    spec = importlib.util.spec_from_file_location("layout_probe", HERE / "layout_probe.py")
    lp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(lp)
    gpu = Path(ref_root) / "src" / "gpu"
    protos = {}
    for f in ["model.cu", "peel.cu", "utils.cu"]:
        protos.update(lp.prototypes((gpu / f).read_text()))
    (HERE / "ref_struct_layouts.json").write_text(json.dumps(
        {"source": "src/gpu/types.h (FP64 build), src/gpu/{model,peel,utils}.cu definitions",
         "layouts": lp.probe(gpu / "types.h"), "prototypes": protos}, indent=1) + "\n")


def uvfits_sdc3(ref_root):
    """The sdc3 uvfits file's headers, data and AN rows (see the module
    docstring), read with this package's FITS layer."""
    sys.path.insert(0, str(HERE.parents[1]))
    from mwa_hyperdrive_b200 import fits

    path = Path(ref_root) / "test_files" / "sdc3" / "sdc3_0000.uvfits"
    raw = path.read_bytes()
    h, hdus = fits.decode(raw)
    cards = []
    for k in range(0, len(h.encode()), 80):
        c = h.encode()[k:k + 80].decode("ascii")
        if c.strip():
            cards.append(c)
    # the AN table's keywords (its column definitions are rebuilt from the
    # three columns a reader needs) and rows; the FQ table is not needed
    an = fits.find(hdus, "AIPS AN")
    hc = [an.header.encode()[k:k + 80].decode("ascii") for k in range(0, len(an.header.encode()), 80)]
    skip = ("XTENSION", "BITPIX", "NAXIS", "PCOUNT", "GCOUNT", "TFIELDS", "TTYPE", "TFORM", "TUNIT", "EXTNAME", "END")
    keys = [c for c in hc if c.strip() and not c.startswith(skip)]
    tables = [{"name": "AIPS AN", "cards": keys,
               "columns": [["ANNAME", "8A"], ["STABXYZ", "3D"], ["NOSTA", "1J"]],
               "data": {"ANNAME": list(an.data["ANNAME"]), "STABXYZ": np.asarray(an.data["STABXYZ"]).tolist(),
                        "NOSTA": np.asarray(an.data["NOSTA"]).tolist()}}]
    groups = [x for x in hdus if x.kind == "GROUPS"][0]
    (HERE / "uvfits_sdc3.json").write_text(json.dumps({
        "source": "test_files/sdc3/sdc3_0000.uvfits; expected values: src/io/read/uvfits/tests.rs:909-958",
        "primary_cards": cards, "groups": groups.data.astype(np.float64).tolist(), "tables": tables,
        "expected": {"num_timestamps": 1, "num_fine_chans": 1, "longitude_deg": 116.76372382627274,
                     "latitude_deg": -26.824419317822766, "height_m": -10.401579822123448, "epsilon": 1e-8,
                     "polarisations": "XX", "flagged_tiles": list(range(2, 512)),
                     "vis_xx": [-8.517027, -7.5777674], "weight": 1.0}}) + "\n")


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HDC_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_golden.py <mwa_hyperdrive source root> (or set HDC_REFERENCE_DIR)")
    main(root)
    layouts(root)
    uvfits_sdc3(root)
