"""Sky-model source-list types: the host-side mirror of mwa_hyperdrive's
``srclist/types`` (components/mod.rs:21-128, flux_density/mod.rs:18-150,
source/mod.rs, source_list/mod.rs:71).

A :class:`SourceList` is an ordered mapping of source name -> :class:`Source`;
a source holds :class:`SourceComponent` s.  :meth:`SourceList.to_sky_model`
flattens components into the struct-of-arrays :class:`SkyModelArrays` that the
C ABI (``HdcSkyModel`` in ``include/hdc.h``) consumes, in the reference's
modelling order: sources reversed, components in order
(model/cpu.rs:86-93, model/gpu.rs:600-606).
"""

from __future__ import annotations

import ctypes
import math
from collections import OrderedDict
from dataclasses import dataclass, field
from typing import Iterable, List, Optional, Sequence

import numpy as np

POINT, GAUSSIAN, SHAPELET = 0, 1, 2
FLUX_LIST, FLUX_POWER_LAW, FLUX_CURVED_POWER_LAW = 0, 1, 2


@dataclass
class FluxDensity:
    """Stokes flux densities [Jy] at ``freq`` [Hz] (flux_density/mod.rs:18-42)."""

    freq: float
    i: float
    q: float = 0.0
    u: float = 0.0
    v: float = 0.0


@dataclass
class PowerLaw:
    """S = fd * (nu / fd.freq)^si."""

    si: float
    fd: FluxDensity


@dataclass
class CurvedPowerLaw:
    """S = fd * (nu / fd.freq)^si * exp(q ln(nu / fd.freq)^2)."""

    si: float
    fd: FluxDensity
    q: float


@dataclass
class FluxList:
    """Flux densities at several frequencies, sorted by frequency."""

    fds: List[FluxDensity]


@dataclass
class ShapeletCoeff:
    n1: int
    n2: int
    value: float


@dataclass
class Point:
    pass


@dataclass
class Gaussian:
    maj: float  # [rad]
    min: float  # [rad]
    pa: float  # [rad]


@dataclass
class Shapelet:
    maj: float
    min: float
    pa: float
    coeffs: List[ShapeletCoeff] = field(default_factory=list)


@dataclass
class SourceComponent:
    ra: float  # [rad]
    dec: float  # [rad]
    comp_type: object
    flux_type: object


@dataclass
class Source:
    components: List[SourceComponent]


class SourceList(OrderedDict):
    """Ordered source name -> Source (source_list/mod.rs:71, an IndexMap)."""

    def to_sky_model(self, reverse: bool = True) -> "SkyModelArrays":
        srcs = list(self.values())
        if reverse:
            srcs = srcs[::-1]
        comps = [c for s in srcs for c in s.components]
        return SkyModelArrays.from_components(comps)


class HdcSkyModel(ctypes.Structure):
    """ctypes twin of ``HdcSkyModel`` in include/hdc.h."""

    _fields_ = [
        ("num_components", ctypes.c_int),
        ("comp_type", ctypes.POINTER(ctypes.c_int)),
        ("ra", ctypes.POINTER(ctypes.c_double)),
        ("dec", ctypes.POINTER(ctypes.c_double)),
        ("maj", ctypes.POINTER(ctypes.c_double)),
        ("min", ctypes.POINTER(ctypes.c_double)),
        ("pa", ctypes.POINTER(ctypes.c_double)),
        ("flux_type", ctypes.POINTER(ctypes.c_int)),
        ("si", ctypes.POINTER(ctypes.c_double)),
        ("q", ctypes.POINTER(ctypes.c_double)),
        ("fd_start", ctypes.POINTER(ctypes.c_int)),
        ("fd_count", ctypes.POINTER(ctypes.c_int)),
        ("fds", ctypes.POINTER(ctypes.c_double)),
        ("coeff_start", ctypes.POINTER(ctypes.c_int)),
        ("coeff_count", ctypes.POINTER(ctypes.c_int)),
        ("coeff_n1", ctypes.POINTER(ctypes.c_int)),
        ("coeff_n2", ctypes.POINTER(ctypes.c_int)),
        ("coeff_value", ctypes.POINTER(ctypes.c_double)),
    ]


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class SkyModelArrays:
    """Struct-of-arrays sky model (one row per component, modelling order)."""

    def __init__(self, comp_type, ra, dec, maj, mn, pa, flux_type, si, q, fd_start, fd_count, fds, coeff_start,
                 coeff_count, coeff_n1, coeff_n2, coeff_value):
        self.comp_type = np.ascontiguousarray(comp_type, dtype=np.int32)
        self.ra = np.ascontiguousarray(ra, dtype=np.float64)
        self.dec = np.ascontiguousarray(dec, dtype=np.float64)
        self.maj = np.ascontiguousarray(maj, dtype=np.float64)
        self.min = np.ascontiguousarray(mn, dtype=np.float64)
        self.pa = np.ascontiguousarray(pa, dtype=np.float64)
        self.flux_type = np.ascontiguousarray(flux_type, dtype=np.int32)
        self.si = np.ascontiguousarray(si, dtype=np.float64)
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.fd_start = np.ascontiguousarray(fd_start, dtype=np.int32)
        self.fd_count = np.ascontiguousarray(fd_count, dtype=np.int32)
        self.fds = np.ascontiguousarray(np.asarray(fds, dtype=np.float64).reshape(-1, 5))
        self.coeff_start = np.ascontiguousarray(coeff_start, dtype=np.int32)
        self.coeff_count = np.ascontiguousarray(coeff_count, dtype=np.int32)
        self.coeff_n1 = np.ascontiguousarray(coeff_n1, dtype=np.int32)
        self.coeff_n2 = np.ascontiguousarray(coeff_n2, dtype=np.int32)
        self.coeff_value = np.ascontiguousarray(coeff_value, dtype=np.float64)
        # ctypes dislikes NULL for zero-length arrays in some paths; keep >=1
        for name in ("fds", "coeff_n1", "coeff_n2", "coeff_value"):
            a = getattr(self, name)
            if a.size == 0:
                setattr(self, name + "_buf", np.zeros(5 if name == "fds" else 1, dtype=a.dtype))
            else:
                setattr(self, name + "_buf", a)
        self._struct: Optional[HdcSkyModel] = None

    @property
    def num_components(self) -> int:
        return int(self.ra.size)

    @staticmethod
    def from_components(comps: Sequence[SourceComponent]) -> "SkyModelArrays":
        n = len(comps)
        ct = np.zeros(n, np.int32)
        ra = np.zeros(n)
        dec = np.zeros(n)
        maj = np.zeros(n)
        mn = np.zeros(n)
        pa = np.zeros(n)
        ft = np.zeros(n, np.int32)
        si = np.zeros(n)
        q = np.zeros(n)
        fd_start = np.zeros(n, np.int32)
        fd_count = np.zeros(n, np.int32)
        fds: List[List[float]] = []
        cs = np.zeros(n, np.int32)
        cc = np.zeros(n, np.int32)
        n1: List[int] = []
        n2: List[int] = []
        cv: List[float] = []
        for k, c in enumerate(comps):
            ra[k], dec[k] = c.ra, c.dec
            t = c.comp_type
            if isinstance(t, Point):
                ct[k] = POINT
            elif isinstance(t, Gaussian):
                ct[k] = GAUSSIAN
                maj[k], mn[k], pa[k] = t.maj, t.min, t.pa
            elif isinstance(t, Shapelet):
                ct[k] = SHAPELET
                maj[k], mn[k], pa[k] = t.maj, t.min, t.pa
                cs[k] = len(cv)
                cc[k] = len(t.coeffs)
                for co in t.coeffs:
                    n1.append(int(co.n1))
                    n2.append(int(co.n2))
                    cv.append(float(co.value))
            else:
                raise TypeError(f"unknown component type {t!r}")
            f = c.flux_type
            fd_start[k] = len(fds)
            if isinstance(f, FluxList):
                ft[k] = FLUX_LIST
                if not f.fds:
                    raise ValueError("a flux-density list needs at least one entry")
                prev = -math.inf
                for e in f.fds:
                    if e.freq < prev:
                        raise ValueError("The list of flux densities used for estimation were not sorted")
                    prev = e.freq
                    fds.append([e.freq, e.i, e.q, e.u, e.v])
                fd_count[k] = len(f.fds)
            elif isinstance(f, PowerLaw):
                ft[k] = FLUX_POWER_LAW
                si[k] = f.si
                fds.append([f.fd.freq, f.fd.i, f.fd.q, f.fd.u, f.fd.v])
                fd_count[k] = 1
            elif isinstance(f, CurvedPowerLaw):
                ft[k] = FLUX_CURVED_POWER_LAW
                si[k], q[k] = f.si, f.q
                fds.append([f.fd.freq, f.fd.i, f.fd.q, f.fd.u, f.fd.v])
                fd_count[k] = 1
            else:
                raise TypeError(f"unknown flux type {f!r}")
        return SkyModelArrays(ct, ra, dec, maj, mn, pa, ft, si, q, fd_start, fd_count, np.array(fds).reshape(-1, 5),
                              cs, cc, n1, n2, cv)

    def select(self, mask: np.ndarray) -> "SkyModelArrays":
        """Sub-model of the components where ``mask`` is true (order kept)."""
        idx = np.nonzero(np.asarray(mask))[0]
        fds, n1, n2, cv = [], [], [], []
        fs, fc, cs, cc = [], [], [], []
        for k in idx:
            fs.append(len(fds))
            fc.append(self.fd_count[k])
            fds.extend(self.fds[self.fd_start[k]: self.fd_start[k] + self.fd_count[k]].tolist())
            cs.append(len(cv))
            cc.append(self.coeff_count[k])
            a, b = self.coeff_start[k], self.coeff_start[k] + self.coeff_count[k]
            n1.extend(self.coeff_n1[a:b].tolist())
            n2.extend(self.coeff_n2[a:b].tolist())
            cv.extend(self.coeff_value[a:b].tolist())
        return SkyModelArrays(self.comp_type[idx], self.ra[idx], self.dec[idx], self.maj[idx], self.min[idx],
                              self.pa[idx], self.flux_type[idx], self.si[idx], self.q[idx], fs, fc,
                              np.array(fds).reshape(-1, 5), cs, cc, n1, n2, cv)

    def struct(self) -> HdcSkyModel:
        if self._struct is None:
            s = HdcSkyModel()
            s.num_components = self.num_components
            s.comp_type = _p(self.comp_type, ctypes.c_int)
            s.ra = _p(self.ra, ctypes.c_double)
            s.dec = _p(self.dec, ctypes.c_double)
            s.maj = _p(self.maj, ctypes.c_double)
            s.min = _p(self.min, ctypes.c_double)
            s.pa = _p(self.pa, ctypes.c_double)
            s.flux_type = _p(self.flux_type, ctypes.c_int)
            s.si = _p(self.si, ctypes.c_double)
            s.q = _p(self.q, ctypes.c_double)
            s.fd_start = _p(self.fd_start, ctypes.c_int)
            s.fd_count = _p(self.fd_count, ctypes.c_int)
            s.fds = _p(self.fds_buf, ctypes.c_double)
            s.coeff_start = _p(self.coeff_start, ctypes.c_int)
            s.coeff_count = _p(self.coeff_count, ctypes.c_int)
            s.coeff_n1 = _p(self.coeff_n1_buf, ctypes.c_int)
            s.coeff_n2 = _p(self.coeff_n2_buf, ctypes.c_int)
            s.coeff_value = _p(self.coeff_value_buf, ctypes.c_double)
            self._struct = s
        return self._struct


def radec_deg(ra_deg: float, dec_deg: float):
    return math.radians(ra_deg), math.radians(dec_deg)
