"""A small FITS reader and writer (FITS standard 4.0): header cards with the
CONTINUE long-string and HIERARCH long-keyword conventions (as cfitsio
writes them), IMAGE extensions and BINTABLE extensions
with fixed-width columns (L, X, B, I, J, K, E, D, A, with repeat counts).
Enough for the hyperdrive calibration-solutions files
(solutions/hyperdrive.rs) and FITS source lists; no compression, no
variable-length arrays, no scaling keywords.

Data are big-endian on disk; images come back as C-ordered numpy arrays with
the FITS axes reversed (NAXIS1 fastest), as cfitsio presents them.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

BLOCK = 2880
CARD = 80


class FitsError(ValueError):
    pass


# ----------------------------------------------------------------- cards
def _fmt_value(v) -> str:
    """A value field: logical/number right-justified to column 30, strings
    quoted from column 11 (at least 8 characters inside the quotes)."""
    if isinstance(v, bool):
        return f"{'T' if v else 'F':>20}"
    if isinstance(v, (int, np.integer)):
        return f"{int(v):>20}"
    if isinstance(v, (float, np.floating)):
        v = float(v)
        if not math.isfinite(v):
            raise FitsError("FITS header values cannot be NaN or infinite")
        t = repr(v).upper()
        if "E" in t:
            mant, exp = t.split("E")
            if "." not in mant:
                mant += ".0"
            t = f"{mant}E{exp}"
        elif "." not in t:
            t += ".0"
        return f"{t:>20}"
    s = str(v).replace("'", "''")
    return f"'{s:<8}'"


class Header:
    """Ordered FITS header: (key, value, comment) records plus COMMENT and
    HISTORY lines."""

    def __init__(self):
        self.records: List[Tuple[str, object, Optional[str]]] = []

    def set(self, key: str, value, comment: Optional[str] = None) -> None:
        key = key.upper()
        for i, (k, _, _) in enumerate(self.records):
            if k == key and k not in ("COMMENT", "HISTORY"):
                self.records[i] = (key, value, comment)
                return
        self.records.append((key, value, comment))

    def comment(self, text: str) -> None:
        self.records.append(("COMMENT", text, None))

    def get(self, key: str, default=None):
        key = key.upper()
        for k, v, _ in self.records:
            if k == key:
                return v
        return default

    def __contains__(self, key: str) -> bool:
        return any(k == key.upper() for k, _, _ in self.records)

    def __getitem__(self, key: str):
        key = key.upper()
        for k, v, _ in self.records:
            if k == key:
                return v
        raise KeyError(key)

    # -- encoding
    def encode(self) -> bytes:
        cards: List[str] = []
        for key, value, comment in self.records:
            if key in ("COMMENT", "HISTORY"):
                text = str(value)
                for i in range(0, max(len(text), 1), 72):
                    cards.append(f"{key:<8}{text[i:i + 72]}")
                continue
            if len(key) > 8:  # the HIERARCH convention, as cfitsio writes longer names
                card = f"HIERARCH {key} = {_fmt_value(value).strip()}"
                if comment:
                    card += f" / {comment}"
                if len(card) > CARD:
                    raise FitsError(f"keyword {key!r} and its value do not fit one card")
                cards.append(card)
                continue
            if isinstance(value, str) and len(_fmt_value(value)) + 10 > CARD:
                cards.extend(_long_string_cards(key, value, comment))
                continue
            card = f"{key:<8}= {_fmt_value(value)}"
            if comment:
                card += f" / {comment}"
            if len(card) > CARD:
                card = card[:CARD]
            cards.append(card)
        cards.append("END")
        text = "".join(f"{c:<80}" for c in cards)
        pad = (-len(text)) % BLOCK
        return (text + " " * pad).encode("ascii")

    @staticmethod
    def decode(buf: bytes, pos: int) -> Tuple["Header", int]:
        h = Header()
        pending: Optional[List] = None  # [key, value, comment] of a string ending in '&'
        while True:
            if pos + BLOCK > len(buf):
                raise FitsError("truncated header")
            block = buf[pos:pos + BLOCK].decode("ascii", errors="replace")
            pos += BLOCK
            done = False
            for k in range(0, BLOCK, CARD):
                card = block[k:k + CARD]
                key = card[:8].strip()
                if key == "END":
                    done = True
                    break
                if key == "CONTINUE" and pending is not None:
                    s, _ = _parse_string(card[8:].strip())
                    pending[1] = pending[1][:-1] + s
                    if not pending[1].endswith("&"):
                        h.records.append(tuple(pending))
                        pending = None
                    continue
                if pending is not None:
                    h.records.append(tuple(pending))
                    pending = None
                if key == "HIERARCH" and "=" in card:
                    name, _, rest = card[8:].partition("=")
                    value, comment = _parse_value(rest)
                    h.records.append((name.strip().upper(), value, comment))
                    continue
                if key in ("COMMENT", "HISTORY", ""):
                    if key:
                        h.records.append((key, card[8:].rstrip(), None))
                    continue
                if card[8:10] != "= ":
                    continue
                value, comment = _parse_value(card[10:])
                if isinstance(value, str) and value.endswith("&"):
                    pending = [key, value, comment]
                else:
                    h.records.append((key, value, comment))
            if done:
                break
        if pending is not None:
            pending[1] = pending[1][:-1]
            h.records.append(tuple(pending))
        return h, pos


def _long_string_cards(key: str, value: str, comment: Optional[str]) -> List[str]:
    """The CONTINUE convention (as cfitsio's fits_write_key_longstr): pieces
    of at most 67 characters once quotes are doubled, each but the last
    ending in '&'; a doubled quote is never split."""
    pieces: List[str] = []
    cur, room = "", 66  # one place kept for the '&'
    for ch in value:
        e = "''" if ch == "'" else ch
        if len(cur) + len(e) > room:
            pieces.append(cur)
            cur = ""
        cur += e
    pieces.append(cur)
    pieces = [p + "&" for p in pieces[:-1]] + [pieces[-1]]
    cards = [f"{key:<8}= '{pieces[0]}'"]
    cards += [f"CONTINUE  '{p}'" for p in pieces[1:]]
    if comment:
        cards[-1] = (cards[-1] + f" / {comment}")[:CARD]
    return cards


def _parse_string(t: str) -> Tuple[str, str]:
    if not t.startswith("'"):
        raise FitsError(f"bad string value {t!r}")
    out, i = [], 1
    while i < len(t):
        if t[i] == "'":
            if i + 1 < len(t) and t[i + 1] == "'":
                out.append("'")
                i += 2
                continue
            break
        out.append(t[i])
        i += 1
    rest = t[i + 1:]
    c = rest.split("/", 1)
    return "".join(out).rstrip(), (c[1].strip() if len(c) > 1 else "")


def _parse_value(t: str):
    t = t.strip()
    if t.startswith("'"):
        return _parse_string(t)
    v, _, c = t.partition("/")
    v = v.strip()
    c = c.strip() or None
    if v == "T":
        return True, c
    if v == "F":
        return False, c
    if v == "":
        return None, c
    try:
        return int(v), c
    except ValueError:
        pass
    try:
        return float(v.replace("D", "E")), c
    except ValueError:
        return v, c


# -------------------------------------------------------------- columns
_TYPES = {"L": ("u1", 1), "B": ("u1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8), "E": (">f4", 4),
          "D": (">f8", 8)}


def _parse_tform(tform: str) -> Tuple[int, str]:
    tform = tform.strip()
    i = 0
    while i < len(tform) and tform[i].isdigit():
        i += 1
    repeat = int(tform[:i]) if i else 1
    code = tform[i:i + 1]
    if code not in _TYPES and code not in ("A", "X"):
        raise FitsError(f"unsupported TFORM {tform!r}")
    return repeat, code


def _width(repeat: int, code: str) -> int:
    if code == "A":
        return repeat
    if code == "X":
        return (repeat + 7) // 8
    return repeat * _TYPES[code][1]


@dataclass
class Column:
    name: str
    tform: str
    data: object  # numpy array [rows] or [rows, repeat]; list of str for 'A'; bool array for 'X'/'L'


@dataclass
class HDU:
    header: Header
    data: object = None  # numpy array (IMAGE) or Dict[str, array] (BINTABLE)
    kind: str = "IMAGE"
    columns: List[Tuple[str, str]] = field(default_factory=list)  # BINTABLE (name, tform)

    @property
    def name(self) -> str:
        return str(self.header.get("EXTNAME", "")).strip()


def _encode_column(col: Column, rows: int) -> np.ndarray:
    repeat, code = _parse_tform(col.tform)
    w = _width(repeat, code)
    out = np.zeros((rows, w), np.uint8)
    if code == "A":
        for r, s in enumerate(col.data):
            b = str(s).encode("ascii")[:repeat]
            out[r, :len(b)] = np.frombuffer(b, np.uint8)
    elif code == "X":
        bits = np.asarray(col.data, bool).reshape(rows, -1)
        out[:] = np.packbits(bits, axis=1, bitorder="big")[:, :w]
    elif code == "L":
        v = np.asarray(col.data, bool).reshape(rows, repeat)
        out[:] = np.where(v, ord("T"), ord("F")).astype(np.uint8)
    else:
        dt = _TYPES[code][0]
        v = np.ascontiguousarray(np.asarray(col.data).reshape(rows, repeat).astype(dt))
        out[:] = v.view(np.uint8).reshape(rows, w)
    return out


def _decode_column(raw: np.ndarray, tform: str):
    repeat, code = _parse_tform(tform)
    rows = raw.shape[0]
    if code == "A":
        return [bytes(r).split(b"\0", 1)[0].decode("ascii", errors="replace").rstrip() for r in raw]
    if code == "X":
        bits = np.unpackbits(raw, axis=1, bitorder="big")[:, :repeat].astype(bool)
        return bits[:, 0] if repeat == 1 else bits
    if code == "L":
        v = raw == ord("T")
        return v[:, 0] if repeat == 1 else v
    dt = np.dtype(_TYPES[code][0])
    v = np.ascontiguousarray(raw).view(dt).reshape(rows, repeat).astype(dt.newbyteorder("="))
    return v[:, 0] if repeat == 1 else v


# -------------------------------------------------------------- writing
def primary_header() -> Header:
    h = Header()
    h.set("SIMPLE", True, "file does conform to FITS standard")
    h.set("BITPIX", 8, "number of bits per data pixel")
    h.set("NAXIS", 0, "number of data axes")
    h.set("EXTEND", True, "FITS dataset may contain extensions")
    return h


def image_hdu(name: str, data: np.ndarray) -> HDU:
    data = np.asarray(data)
    bitpix = {np.dtype(np.float64): -64, np.dtype(np.float32): -32, np.dtype(np.int32): 32,
              np.dtype(np.int16): 16, np.dtype(np.uint8): 8, np.dtype(np.int64): 64}[data.dtype]
    h = Header()
    h.set("XTENSION", "IMAGE", "IMAGE extension")
    h.set("BITPIX", bitpix, "number of bits per data pixel")
    h.set("NAXIS", data.ndim, "number of data axes")
    for i, n in enumerate(reversed(data.shape)):
        h.set(f"NAXIS{i + 1}", int(n), f"length of data axis {i + 1}")
    h.set("PCOUNT", 0, "required keyword; must = 0")
    h.set("GCOUNT", 1, "required keyword; must = 1")
    h.set("EXTNAME", name, "name of this HDU")
    return HDU(h, data, "IMAGE")


def table_hdu(name: str, columns: Sequence[Column], rows: int) -> HDU:
    h = Header()
    widths = [_width(*_parse_tform(c.tform)) for c in columns]
    h.set("XTENSION", "BINTABLE", "binary table extension")
    h.set("BITPIX", 8, "8-bit bytes")
    h.set("NAXIS", 2, "2-dimensional binary table")
    h.set("NAXIS1", int(sum(widths)), "width of table in bytes")
    h.set("NAXIS2", int(rows), "number of rows in table")
    h.set("PCOUNT", 0, "size of special data area")
    h.set("GCOUNT", 1, "one data group (required keyword)")
    h.set("TFIELDS", len(columns), "number of fields in each row")
    for i, c in enumerate(columns):
        h.set(f"TTYPE{i + 1}", c.name, f"label for field {i + 1}")
        h.set(f"TFORM{i + 1}", c.tform, "data format of field")
    h.set("EXTNAME", name, "name of this binary table extension")
    data = {c.name: c.data for c in columns}
    return HDU(h, data, "BINTABLE", [(c.name, c.tform) for c in columns])


def _pad(b: bytes, fill: bytes = b"\0") -> bytes:
    return b + fill * ((-len(b)) % BLOCK)


def encode(primary: Header, hdus: Sequence[HDU], primary_data: Optional[np.ndarray] = None) -> bytes:
    """The file's bytes: the primary header (and its data -- e.g. random
    groups [GCOUNT][PCOUNT + values] -- big-endian) then each extension."""
    out = [primary.encode()]
    if primary_data is not None:
        a = np.asarray(primary_data)
        out.append(_pad(np.ascontiguousarray(a.astype(a.dtype.newbyteorder(">"))).tobytes()))
    for hdu in hdus:
        out.append(hdu.header.encode())
        if hdu.kind == "IMAGE":
            a = np.asarray(hdu.data)
            out.append(_pad(np.ascontiguousarray(a.astype(a.dtype.newbyteorder(">"))).tobytes()))
        else:
            rows = int(hdu.header["NAXIS2"])
            cols = [_encode_column(Column(n, t, hdu.data[n]), rows) for n, t in hdu.columns]
            table = np.concatenate(cols, axis=1) if cols else np.zeros((rows, 0), np.uint8)
            out.append(_pad(np.ascontiguousarray(table).tobytes()))
    return b"".join(out)


def write(path: Union[str, Path], primary: Header, hdus: Sequence[HDU],
          primary_data: Optional[np.ndarray] = None) -> None:
    Path(path).write_bytes(encode(primary, hdus, primary_data))


# -------------------------------------------------------------- reading
_BITPIX = {8: "u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def decode(buf: bytes) -> Tuple[Header, List[HDU]]:
    pos = 0
    hdus: List[HDU] = []
    primary = None
    while pos < len(buf):
        if not buf[pos:pos + 8].strip(b" \0"):
            break  # trailing padding
        h, pos = Header.decode(buf, pos)
        naxis = int(h.get("NAXIS", 0))
        dims = [int(h[f"NAXIS{i + 1}"]) for i in range(naxis)]
        bitpix = int(h["BITPIX"])
        # random groups (uvfits): NAXIS1 = 0, each of GCOUNT groups holds
        # PCOUNT parameters then the product of NAXIS2.. values
        groups = h.get("GROUPS") is True and naxis >= 1 and dims[0] == 0
        gsize = int(h.get("PCOUNT", 0)) + ((int(np.prod(dims[1:])) if groups else int(np.prod(dims))) if dims else 0)
        nbytes = (abs(bitpix) // 8) * int(h.get("GCOUNT", 1)) * gsize
        raw = buf[pos:pos + nbytes]
        if len(raw) < nbytes:
            raise FitsError("truncated data")
        pos += nbytes + ((-nbytes) % BLOCK)
        xt = str(h.get("XTENSION", "")).strip()
        if primary is None:
            if h.get("SIMPLE") is not True:
                raise FitsError("not a FITS file (no SIMPLE = T)")
            primary = h
            if groups:
                # [GCOUNT][PCOUNT + values]; parameters unscaled (PSCAL / PZERO are the caller's)
                hdus.append(HDU(h, np.frombuffer(raw, _BITPIX[bitpix]).reshape(int(h.get("GCOUNT", 1)), gsize).astype(
                    np.dtype(_BITPIX[bitpix]).newbyteorder("=")), "GROUPS"))
            elif dims:
                hdus.append(HDU(h, np.frombuffer(raw, _BITPIX[bitpix]).reshape(dims[::-1]).astype(
                    np.dtype(_BITPIX[bitpix]).newbyteorder("=")), "PRIMARY"))
            continue
        if xt == "BINTABLE":
            nfields = int(h["TFIELDS"])
            rowlen, rows = dims[0], dims[1]
            table = np.frombuffer(raw[:rowlen * rows], np.uint8).reshape(rows, rowlen)
            data, cols, off = {}, [], 0
            for i in range(nfields):
                name = str(h.get(f"TTYPE{i + 1}", f"col{i + 1}")).strip()
                tform = str(h[f"TFORM{i + 1}"]).strip()
                w = _width(*_parse_tform(tform))
                data[name] = _decode_column(table[:, off:off + w], tform)
                cols.append((name, tform))
                off += w
            hdus.append(HDU(h, data, "BINTABLE", cols))
        else:
            arr = None
            if dims:
                arr = np.frombuffer(raw, _BITPIX[bitpix]).reshape(dims[::-1]).astype(
                    np.dtype(_BITPIX[bitpix]).newbyteorder("="))
            hdus.append(HDU(h, arr, "IMAGE"))
    if primary is None:
        raise FitsError("empty file")
    return primary, hdus


def read(path: Union[str, Path]) -> Tuple[Header, List[HDU]]:
    return decode(Path(path).read_bytes())


def find(hdus: Sequence[HDU], name: str) -> Optional[HDU]:
    for h in hdus:
        if h.name.upper() == name.upper():
            return h
    return None
