"""Hyperdrive-format sky-model source lists (YAML and JSON): read, write,
and the brightness veto that orders a list for the predictor.

File layout (srclist/hyperdrive/read.rs:14-51, write.rs:16-69, with the
serde field layout of srclist/types/components/mod.rs:21-128 and
flux_density/mod.rs:18-150): a mapping of source name -> list of
components; a component is ``ra``, ``dec`` [deg], ``comp_type`` (``point``,
or ``gaussian`` / ``shapelet`` with ``maj``, ``min`` [arcsec], ``pa`` [deg]
and, for shapelets, ``coeffs`` of ``n1``, ``n2``, ``value``) and
``flux_type`` (``list`` of flux densities, ``power_law`` {``si``, ``fd``},
``curved_power_law`` {``si``, ``fd``, ``q``}); a flux density is ``freq``
[Hz], ``i`` and the nonzero ones of ``q``, ``u``, ``v`` [Jy].  In memory
(:mod:`srclist`) positions, sizes and angles are radians.

The writers reproduce the reference's output text (block-style YAML with
sequences at their key's indentation; JSON with two-space indentation and a
final newline), so a list written here reads back identically in either
implementation.
"""

from __future__ import annotations

import json
import math
import re
from pathlib import Path
from typing import Optional, Union

import numpy as np

from . import srclist as sl


class SourceListError(ValueError):
    """A source list that cannot be read or written."""


# ----------------------------------------------------------------- reading
def _num(x, what: str) -> float:
    # YAML 1.1 loaders read "150e6" (no dot, unsigned exponent) as a string;
    # the reference's YAML 1.2 reader takes it as a number, and so do we
    try:
        return float(x)
    except (TypeError, ValueError):
        raise SourceListError(f"{what}: expected a number, got {x!r}") from None


def _fd(d: dict) -> sl.FluxDensity:
    if not isinstance(d, dict) or "freq" not in d or "i" not in d:
        raise SourceListError(f"a flux density needs freq and i: {d!r}")
    return sl.FluxDensity(_num(d["freq"], "freq"), _num(d["i"], "i"), _num(d.get("q", 0.0), "q"),
                          _num(d.get("u", 0.0), "u"), _num(d.get("v", 0.0), "v"))


def _flux_type(d):
    if not isinstance(d, dict) or len(d) != 1:
        raise SourceListError(f"flux_type must be one of list, power_law, curved_power_law: {d!r}")
    (kind, body), = d.items()
    if kind == "list":
        if not isinstance(body, list) or not body:
            raise SourceListError("a flux-density list needs at least one entry")
        return sl.FluxList(sorted((_fd(x) for x in body), key=lambda f: f.freq))
    if kind == "power_law":
        return sl.PowerLaw(_num(body["si"], "si"), _fd(body["fd"]))
    if kind == "curved_power_law":
        return sl.CurvedPowerLaw(_num(body["si"], "si"), _fd(body["fd"]), _num(body["q"], "q"))
    raise SourceListError(f"unknown flux type {kind!r}")


def _comp_type(d):
    if d == "point":
        return sl.Point()
    if not isinstance(d, dict) or len(d) != 1:
        raise SourceListError(f"comp_type must be point, gaussian or shapelet: {d!r}")
    (kind, body), = d.items()
    # arcsec -> rad as the reference orders it (degrees to radians, then / 3600)
    maj = math.radians(_num(body["maj"], "maj")) / 3600.0
    mn = math.radians(_num(body["min"], "min")) / 3600.0
    pa = math.radians(_num(body["pa"], "pa"))
    if kind == "gaussian":
        return sl.Gaussian(maj, mn, pa)
    if kind == "shapelet":
        coeffs = [sl.ShapeletCoeff(int(c["n1"]), int(c["n2"]), _num(c["value"], "value")) for c in body["coeffs"]]
        for c in coeffs:
            if not (0 <= c.n1 <= 255 and 0 <= c.n2 <= 255):
                raise SourceListError(f"shapelet coefficient orders must fit in a byte: {c}")
        return sl.Shapelet(maj, mn, pa, coeffs)
    raise SourceListError(f"unknown component type {kind!r}")


def from_mapping(obj) -> sl.SourceList:
    """A :class:`srclist.SourceList` from the parsed YAML/JSON mapping; RA must
    lie in [0, 360) and Dec in [-90, 90] degrees (read.rs:20-28)."""
    if not isinstance(obj, dict):
        raise SourceListError("a hyperdrive source list is a mapping of source names to components")
    out = sl.SourceList()
    for name, comps in obj.items():
        if not isinstance(comps, list) or not comps:
            raise SourceListError(f"source {name!r} has no components")
        cs = []
        for c in comps:
            ra = math.radians(_num(c["ra"], "ra"))
            dec = math.radians(_num(c["dec"], "dec"))
            if not (0.0 <= ra < 2.0 * math.pi):
                raise SourceListError(f"source {name!r}: RA {math.degrees(ra)} deg is outside [0, 360)")
            if not (-0.5 * math.pi <= dec <= 0.5 * math.pi):
                raise SourceListError(f"source {name!r}: Dec {math.degrees(dec)} deg is outside [-90, 90]")
            cs.append(sl.SourceComponent(ra, dec, _comp_type(c["comp_type"]), _flux_type(c["flux_type"])))
        out[str(name)] = sl.Source(cs)
    return out


def read_source_list(source: Union[str, Path], fmt: Optional[str] = None) -> sl.SourceList:
    """Read a hyperdrive YAML or JSON source list from a path (format from
    the suffix unless ``fmt`` is "yaml" or "json")."""
    path = Path(source)
    fmt = fmt or ("json" if path.suffix.lower() == ".json" else "yaml")
    text = path.read_text()
    return parse_source_list(text, fmt)


def parse_source_list(text: str, fmt: str = "yaml") -> sl.SourceList:
    if fmt == "json":
        obj = json.loads(text)
    elif fmt == "yaml":
        import yaml

        obj = yaml.safe_load(text)
    else:
        raise SourceListError(f"unknown source-list format {fmt!r}")
    return from_mapping(obj)


# ----------------------------------------------------------------- writing
def _float_text(x: float) -> str:
    """A float as the reference's serialiser prints it: shortest round-trip
    digits, ".0" on integral values, exponents without "+" or leading zeros."""
    x = float(x)
    if math.isnan(x) or math.isinf(x):
        raise SourceListError("source lists hold finite numbers only")
    s = repr(x)
    if "e" in s:
        mant, exp = s.split("e")
        s = f"{mant}e{int(exp)}"
    return s


def _fd_map(f: sl.FluxDensity) -> dict:
    d = {"freq": f.freq, "i": f.i}
    for k in ("q", "u", "v"):
        if getattr(f, k) != 0.0:
            d[k] = getattr(f, k)
    return d


def _comp_map(c: sl.SourceComponent) -> dict:
    t = c.comp_type
    if isinstance(t, sl.Point):
        ct = "point"
    else:
        body = {"maj": math.degrees(t.maj) * 3600.0, "min": math.degrees(t.min) * 3600.0, "pa": math.degrees(t.pa)}
        if isinstance(t, sl.Shapelet):
            body["coeffs"] = [{"n1": int(k.n1), "n2": int(k.n2), "value": k.value} for k in t.coeffs]
            ct = {"shapelet": body}
        else:
            ct = {"gaussian": body}
    f = c.flux_type
    if isinstance(f, sl.FluxList):
        ft = {"list": [_fd_map(x) for x in sorted(f.fds, key=lambda y: y.freq)]}
    elif isinstance(f, sl.PowerLaw):
        ft = {"power_law": {"si": f.si, "fd": _fd_map(f.fd)}}
    elif isinstance(f, sl.CurvedPowerLaw):
        ft = {"curved_power_law": {"si": f.si, "fd": _fd_map(f.fd), "q": f.q}}
    else:
        raise SourceListError(f"unknown flux type {f!r}")
    return {"ra": math.degrees(c.ra), "dec": math.degrees(c.dec), "comp_type": ct, "flux_type": ft}


def to_mapping(source_list: sl.SourceList, num_sources: Optional[int] = None) -> dict:
    names = list(source_list.keys())
    if num_sources is not None:
        names = names[:num_sources]
    return {n: [_comp_map(c) for c in source_list[n].components] for n in names}


_PLAIN = re.compile(r"^[A-Za-z_][A-Za-z0-9_.+\-]*$")


def _yaml_scalar(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return _float_text(v)
    s = str(v)
    # names that YAML would read as something else are quoted
    if _PLAIN.match(s) and s.lower() not in ("true", "false", "null", "yes", "no", "on", "off", "~"):
        return s
    return json.dumps(s)


def _yaml_lines(v, indent: int, out: list) -> None:
    pad = " " * indent
    if isinstance(v, dict):
        for k, x in v.items():
            if isinstance(x, dict):
                out.append(f"{pad}{_yaml_scalar(k)}:")
                _yaml_lines(x, indent + 2, out)
            elif isinstance(x, list):
                out.append(f"{pad}{_yaml_scalar(k)}:")
                _yaml_lines(x, indent, out)  # block sequences sit at their key's indentation
            else:
                out.append(f"{pad}{_yaml_scalar(k)}: {_yaml_scalar(x)}")
    elif isinstance(v, list):
        for x in v:
            if isinstance(x, dict):
                sub: list = []
                _yaml_lines(x, indent + 2, sub)
                sub[0] = pad + "- " + sub[0][indent + 2:]
                out.extend(sub)
            else:
                out.append(f"{pad}- {_yaml_scalar(x)}")
    else:
        out.append(pad + _yaml_scalar(v))


def to_yaml(source_list: sl.SourceList, num_sources: Optional[int] = None) -> str:
    out: list = []
    _yaml_lines(to_mapping(source_list, num_sources), 0, out)
    return "\n".join(out) + "\n"


def _json_text(v, indent: int) -> str:
    pad, inner = " " * indent, " " * (indent + 2)
    if isinstance(v, dict):
        items = [f"{inner}{json.dumps(str(k))}: {_json_text(x, indent + 2)}" for k, x in v.items()]
        return "{\n" + ",\n".join(items) + "\n" + pad + "}" if items else "{}"
    if isinstance(v, list):
        items = [inner + _json_text(x, indent + 2) for x in v]
        return "[\n" + ",\n".join(items) + "\n" + pad + "]" if items else "[]"
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return _float_text(v)
    return json.dumps(v)


def to_json(source_list: sl.SourceList, num_sources: Optional[int] = None) -> str:
    return _json_text(to_mapping(source_list, num_sources), 0) + "\n"


def write_source_list(source_list: sl.SourceList, path: Union[str, Path], fmt: Optional[str] = None,
                      num_sources: Optional[int] = None) -> None:
    """Write ``source_list`` (or its first ``num_sources`` sources) as YAML
    or JSON (format from the suffix unless given)."""
    path = Path(path)
    fmt = fmt or ("json" if path.suffix.lower() == ".json" else "yaml")
    if fmt not in ("yaml", "json"):
        raise SourceListError(f"unknown source-list format {fmt!r}")
    path.write_text(to_json(source_list, num_sources) if fmt == "json" else to_yaml(source_list, num_sources))


# -------------------------------------------------------------------- veto
DEFAULT_ELEVATION_LIMIT_DEG = 0.0
DEFAULT_CUTOFF_DISTANCE_DEG = 180.0  # no distance cut unless asked for
DEFAULT_VETO_THRESHOLD_JY = 0.01


def veto_sources(source_list: sl.SourceList, phase_centre, lst_rad: float, array_latitude_rad: float,
                 freqs_hz, beam: str = "none", num_sources: Optional[int] = None,
                 source_dist_cutoff_deg: float = DEFAULT_CUTOFF_DISTANCE_DEG,
                 veto_threshold: float = DEFAULT_VETO_THRESHOLD_JY,
                 min_elevation_deg: float = DEFAULT_ELEVATION_LIMIT_DEG, fee_beam=None) -> sl.SourceList:
    """veto_sources (srclist/veto.rs:44-188): a new list without the sources
    that have a component below the elevation limit or farther than the
    cutoff from the phase centre, or whose beam-attenuated brightness (XX +
    YY, summed over components) falls below ``veto_threshold`` Jy at any of
    ``freqs_hz``; sorted brightest first (by that smallest brightness) and cut
    to the first ``num_sources``.  The brightness is computed on the GPU
    (hdc_source_brightness).  Raises if fewer than ``num_sources`` remain.
    The predictor then models the list in reverse, dimmest first.  ``beam`` is
    "none", "analytic" or "fee"; for "fee", ``fee_beam`` is a
    :class:`mwa_hyperdrive_b200.fee.FeeBeam` prepared for one tile with the
    observation's ideal delays and unit gains at ``freqs_hz`` (the reference
    asks its beam for no tile, beam/fee.rs:287-292)."""
    import ctypes

    from . import _lib

    names = list(source_list.keys())
    if not names:
        return sl.SourceList()
    comps, owner = [], []
    for k, n in enumerate(names):
        for c in source_list[n].components:
            comps.append(c)
            owner.append(k)
    sky = sl.SkyModelArrays.from_components(comps)
    comp_source = np.ascontiguousarray(owner, np.int32)
    freqs = np.ascontiguousarray(freqs_hz, np.float64)
    out = np.zeros(len(names))
    beams = {"none": 0, "analytic": 1}
    if beam == "fee":
        if fee_beam is None:
            raise SourceListError('beam "fee" needs fee_beam')
        rc = _lib.lib().hdc_source_brightness_fee(ctypes.byref(sky.struct()), comp_source.ctypes.data, len(names),
                                                  freqs.ctypes.data, freqs.size, float(lst_rad),
                                                  float(array_latitude_rad), _lib.RADec(*phase_centre),
                                                  fee_beam.handle, math.radians(source_dist_cutoff_deg),
                                                  math.radians(min_elevation_deg), out.ctypes.data)
        _lib.check(rc, "hdc_source_brightness_fee")
    elif beam in beams:
        rc = _lib.lib().hdc_source_brightness(ctypes.byref(sky.struct()), comp_source.ctypes.data, len(names),
                                              freqs.ctypes.data, freqs.size, float(lst_rad), float(array_latitude_rad),
                                              _lib.RADec(*phase_centre), beams[beam],
                                              math.radians(source_dist_cutoff_deg), math.radians(min_elevation_deg),
                                              out.ctypes.data)
        _lib.check(rc, "hdc_source_brightness")
    else:
        raise SourceListError(f"unknown beam {beam!r}")
    keep = [(out[k], n) for k, n in enumerate(names) if out[k] >= 0.0 and out[k] >= veto_threshold]
    keep.sort(key=lambda t: -t[0])  # brightest first
    if num_sources is not None:
        if num_sources > len(keep):
            raise SourceListError(f"asked for {num_sources} sources but only {len(keep)} survive the veto")
        keep = keep[:num_sources]
    result = sl.SourceList()
    for _, n in keep:
        result[n] = source_list[n]
    return result
