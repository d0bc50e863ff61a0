"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle restates the reference crate's CPU algorithm in plain C
(``oracle/dioptrin_oracle.c``). Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import this module; the product
package ``dioptrin_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdioptrin_oracle.so")

UNITS = {"2th_rad": 0, "2th_deg": 1, "q_A^-1": 2, "q_nm^-1": 3}
DTYPES = {np.dtype(np.uint16): 0, np.dtype(np.uint32): 1, np.dtype(np.int32): 2,
          np.dtype(np.float32): 3, np.dtype(np.float64): 4}


class Poni(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "pixel1", "pixel2", "distance", "poni1", "poni2", "rot1", "rot2", "rot3",
        "wavelength")]


class _Lut(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("nnz", C.c_int64),
                ("row_ptr", C.POINTER(C.c_int64)), ("col", C.POINTER(C.c_int64)),
                ("w", C.POINTER(C.c_double)), ("hist_min", C.c_double),
                ("hist_step", C.c_double)]


@dataclass
class Lut:
    """A CSR table copied out of the oracle: row_ptr, col (int64), w (f64 or None)."""
    row_ptr: np.ndarray
    col: np.ndarray
    w: Optional[np.ndarray]
    hist_min: float
    hist_step: float

    @property
    def n_rows(self) -> int:
        return len(self.row_ptr) - 1

    def bins(self) -> np.ndarray:
        out = np.empty(self.n_rows)
        _lib().or_bins(self.n_rows, self.hist_min, self.hist_step, _dp(out))
        return out

    def _c(self) -> _Lut:
        lut = _Lut()
        lut.n_rows = self.n_rows
        lut.nnz = len(self.col)
        self._keep = (np.ascontiguousarray(self.row_ptr, np.int64),
                      np.ascontiguousarray(self.col, np.int64),
                      None if self.w is None else np.ascontiguousarray(self.w, np.float64))
        lut.row_ptr = self._keep[0].ctypes.data_as(C.POINTER(C.c_int64))
        lut.col = self._keep[1].ctypes.data_as(C.POINTER(C.c_int64))
        lut.w = (None if self._keep[2] is None
                 else self._keep[2].ctypes.data_as(C.POINTER(C.c_double)))
        lut.hist_min = self.hist_min
        lut.hist_step = self.hist_step
        return lut


_LIB = None


def build() -> str:
    """Compile the oracle with its Makefile (a few seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        d, i64, i = C.c_double, C.c_int64, C.c_int
        pd, pu8 = P(C.c_double), P(C.c_uint8)
        lib.or_sample_positions.argtypes = [P(Poni), i64, i64, pd, pd, pd]
        lib.or_centres.argtypes = [P(Poni), i64, i64, i, i, d, pd, pd, pd, pd, pd, pd]
        lib.or_corners.argtypes = [P(Poni), i64, i64, i, pd, pd]
        lib.or_tth_chi_at.argtypes = [P(Poni), pd, pd, i64, pd, pd]
        lib.or_convert_unit.argtypes = [i, d, d]
        lib.or_convert_unit.restype = d
        lib.or_min_max_step.argtypes = [pd, i64, i64, pd, pd, pd]
        lib.or_bins.argtypes = [i64, d, d, pd]
        lib.or_build_ps1d.argtypes = [P(Poni), i64, i64, i, i64, i, d, d, P(_Lut)]
        lib.or_ps1d_fractions.argtypes = [P(Poni), i64, i64, i, i64, d, d, i, P(_Lut)]
        lib.or_build_counting1d.argtypes = [pd, i64, i64, i, d, d, P(_Lut)]
        lib.or_split1d.argtypes = [pd, i64, d, d, d, d, i, d, P(C.c_int64), pd, i64]
        lib.or_bslz4_decode.argtypes = [C.c_void_p, i64, i, i64, C.c_void_p]
        lib.or_grid2d_new.argtypes = [i64, i64, d, d, d, d, P(Grid2d)]
        lib.or_grid2d_bin.argtypes = [P(Grid2d), d, d]
        lib.or_grid2d_bin.restype = i64
        lib.or_grid2d_for.argtypes = [P(Poni), i64, i64, i, i64, i, i64, i64, i, d, d, i, d, d,
                                      P(Grid2d)]
        lib.or_pyfai_split2d.argtypes = [pd, P(Grid2d), d, P(C.c_int64), pd, i64]
        lib.or_build_2d.argtypes = [P(Poni), i64, i64, i, i64, i, P(Grid2d), P(_Lut)]
        lib.or_pyfai_radial_range.argtypes = [P(Poni), i64, i64, i, pd, pd]
        lib.or_build_pf1d.argtypes = [P(Poni), i64, i64, i, i64, i, d, d, P(_Lut)]
        lib.or_build_ss1d.argtypes = [P(Poni), i64, i64, i, i64, i64, i, d, d, P(_Lut)]
        lib.or_compact.argtypes = [P(_Lut), pu8, P(_Lut)]
        lib.or_denominators.argtypes = [P(_Lut), pd, pd]
        lib.or_integrate_strict.argtypes = [P(_Lut), pd, pd, i, pd, pd]
        lib.or_row_sums.argtypes = [P(_Lut), pd, pd, pd]
        lib.or_raw_sums.argtypes = [P(_Lut), pu8, pd, pd, pd, pd, pd, pd]
        lib.or_azimuthal_std.argtypes = [P(_Lut), pu8, pd, pd, pd, pd, pd, pd]
        lib.or_integrate_frames_mt.argtypes = [P(_Lut), pd, P(_Lut), pu8, pd, C.c_void_p, i,
                                               i64, i64, i, i, i, pd, pd, pd]
        lib.or_lut_free.argtypes = [P(_Lut)]
        _LIB = lib
    return _LIB


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u8(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def poni(**kw) -> Poni:
    p = Poni()
    for k, v in kw.items():
        setattr(p, k, float(v))
    return p


def _take(lut: _Lut) -> Lut:
    n = lut.n_rows
    row_ptr = np.ctypeslib.as_array(lut.row_ptr, (n + 1,)).copy()
    nnz = int(row_ptr[-1])
    col = (np.ctypeslib.as_array(lut.col, (nnz,)).copy() if nnz
           else np.zeros(0, np.int64))
    w = None
    if lut.w:
        w = np.ctypeslib.as_array(lut.w, (nnz,)).copy() if nnz else np.zeros(0)
    out = Lut(row_ptr, col, w, lut.hist_min, lut.hist_step)
    _lib().or_lut_free(C.byref(lut))
    return out


def sample_positions(p: Poni, dim1: int, dim2: int):
    n = dim1 * dim2
    x, y, z = np.empty(n), np.empty(n), np.empty(n)
    _lib().or_sample_positions(C.byref(p), dim1, dim2, _dp(x), _dp(y), _dp(z))
    return x, y, z


def centres(p: Poni, dim1: int, dim2: int, unit: str = "2th_rad",
            polarization_factor: Optional[float] = None) -> dict:
    n = dim1 * dim2
    out = {k: np.empty(n) for k in ("tth", "radial", "chi", "sa", "pol", "norm")}
    _lib().or_centres(C.byref(p), dim1, dim2, UNITS[unit],
                      0 if polarization_factor is None else 1,
                      0.0 if polarization_factor is None else float(polarization_factor),
                      *(_dp(out[k]) for k in ("tth", "radial", "chi", "sa", "pol", "norm")))
    return out


def corners(p: Poni, dim1: int, dim2: int, unit: str = "2th_rad"):
    n = (dim1 + 1) * (dim2 + 1)
    r, c = np.empty(n), np.empty(n)
    _lib().or_corners(C.byref(p), dim1, dim2, UNITS[unit], _dp(r), _dp(c))
    return r, c


def tth_chi_at(p: Poni, d1: np.ndarray, d2: np.ndarray):
    d1 = np.ascontiguousarray(d1, np.float64)
    d2 = np.ascontiguousarray(d2, np.float64)
    t, c = np.empty(len(d1)), np.empty(len(d1))
    _lib().or_tth_chi_at(C.byref(p), _dp(d1), _dp(d2), len(d1), _dp(t), _dp(c))
    return t, c


def min_max_step(data: np.ndarray, n_points: int):
    data = np.ascontiguousarray(data, np.float64)
    lo, hi, st = C.c_double(), C.c_double(), C.c_double()
    _lib().or_min_max_step(_dp(data), len(data), n_points, C.byref(lo), C.byref(hi),
                           C.byref(st))
    return lo.value, hi.value, st.value


def build_ps1d(p: Poni, dim1: int, dim2: int, n_points: int, unit: str = "2th_rad",
               radial_range=None) -> Lut:
    lut = _Lut()
    rr = radial_range or (0.0, 0.0)
    rc = _lib().or_build_ps1d(C.byref(p), dim1, dim2, UNITS[unit], n_points,
                              1 if radial_range else 0, rr[0], rr[1], C.byref(lut))
    if rc:
        raise MemoryError("oracle ps1d build failed")
    return _take(lut)


class Grid2d(C.Structure):
    """IntegrationGrid2d (integration/grid.rs:26-47)."""
    _fields_ = [("n_radial", C.c_int64), ("n_azimuthal", C.c_int64), ("r0", C.c_double),
                ("r1", C.c_double), ("a0", C.c_double), ("a1", C.c_double),
                ("clamp_radial_end", C.c_int), ("clamp_index_rounding", C.c_int),
                ("clamp_radial_outside", C.c_int), ("clamp_azimuthal_outside", C.c_int),
                ("pyfai", C.c_int)]

    def bin(self, radial: float, azimuthal: float):
        b = _lib().or_grid2d_bin(C.byref(self), radial, azimuthal)
        return None if b < 0 else int(b)

    def radial_centres(self):
        step = (self.r1 - self.r0) / self.n_radial
        return np.array([self.r0 + (i + 0.5) * step for i in range(self.n_radial)])

    def azimuthal_centres(self):
        step = (self.a1 - self.a0) / self.n_azimuthal
        return np.array([self.a0 + (i + 0.5) * step for i in range(self.n_azimuthal)])


METHOD_CODES = {"counting": 0, "pixel_split": 1, "pyfai_full": 2, "supersampled": 3}


def grid2d(n_radial: int, n_azimuthal: int, radial_range, azimuthal_range) -> Grid2d:
    g = Grid2d()
    if _lib().or_grid2d_new(n_radial, n_azimuthal, radial_range[0], radial_range[1],
                            azimuthal_range[0], azimuthal_range[1], C.byref(g)):
        raise ValueError("invalid 2D grid")
    return g


def grid2d_for(p: Poni, dim1: int, dim2: int, method: str, n_radial: int, n_azimuthal: int,
               unit: str = "2th_rad", n_ss: int = 1, radial_range=None,
               azimuthal_range=None) -> Grid2d:
    g = Grid2d()
    rr = radial_range or (0.0, 0.0)
    ar = azimuthal_range or (0.0, 0.0)
    if _lib().or_grid2d_for(C.byref(p), dim1, dim2, METHOD_CODES[method], n_ss, UNITS[unit],
                            n_radial, n_azimuthal, 1 if radial_range else 0, rr[0], rr[1],
                            1 if azimuthal_range else 0, ar[0], ar[1], C.byref(g)):
        raise ValueError("invalid 2D grid")
    return g


def pyfai_split2d(poly, g: Grid2d, sign: float = 1.0):
    """pyfai_split::split: list of (bin, weight), or None for the fallback."""
    flat = np.ascontiguousarray(np.asarray(poly, np.float64).ravel())
    bins = np.zeros(4096, np.int64)
    w = np.zeros(4096)
    m = _lib().or_pyfai_split2d(_dp(flat), C.byref(g), sign,
                                bins.ctypes.data_as(C.POINTER(C.c_int64)), _dp(w), 4096)
    if m == -1:
        return None
    if m < 0:
        raise ValueError("raster exceeds the oracle buffer")
    return [(int(bins[k]), float(w[k])) for k in range(m)]


def build_2d(p: Poni, dim1: int, dim2: int, method: str, g: Grid2d, unit: str = "2th_rad",
             n_ss: int = 1) -> Lut:
    lut = _Lut()
    if _lib().or_build_2d(C.byref(p), dim1, dim2, METHOD_CODES[method], n_ss, UNITS[unit],
                          C.byref(g), C.byref(lut)):
        raise MemoryError("oracle 2D build failed")
    return _take(lut)


def bslz4_decode(chunk: bytes, dtype, n_elems: int) -> np.ndarray:
    """Decode one Bitshuffle/LZ4 chunk into n_elems elements of dtype."""
    dt = np.dtype(dtype)
    out = np.zeros(n_elems, dt)
    buf = np.frombuffer(bytes(chunk), np.uint8)
    if _lib().or_bslz4_decode(buf.ctypes.data, len(buf), dt.itemsize, n_elems, out.ctypes.data):
        raise ValueError("malformed Bitshuffle/LZ4 chunk")
    return out


def split1d(poly, n_points: int, radial_range, azimuthal_range=(-math.pi, math.pi),
            sector: bool = False, sign: float = 1.0):
    """pyFAI full splitting of one quadrilateral (pyFAI corner order, (radial,
    chi) pairs): list of (bin, weight)."""
    flat = np.ascontiguousarray(np.asarray(poly, np.float64).ravel())
    bins = np.zeros(256, np.int64)
    w = np.zeros(256)
    m = _lib().or_split1d(_dp(flat), n_points, radial_range[0], radial_range[1],
                          azimuthal_range[0], azimuthal_range[1], 1 if sector else 0, sign,
                          bins.ctypes.data_as(C.POINTER(C.c_int64)), _dp(w), 256)
    if m < 0:
        raise ValueError("pixel spans more bins than the oracle buffer")
    return [(int(bins[k]), float(w[k])) for k in range(m)]


def pyfai_radial_range(p: Poni, dim1: int, dim2: int, unit: str = "2th_rad"):
    lo, hi = C.c_double(), C.c_double()
    _lib().or_pyfai_radial_range(C.byref(p), dim1, dim2, UNITS[unit], C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def build_pf1d(p: Poni, dim1: int, dim2: int, n_points: int, unit: str = "2th_rad",
               radial_range=None) -> Lut:
    lut = _Lut()
    rr = radial_range or (0.0, 0.0)
    rc = _lib().or_build_pf1d(C.byref(p), dim1, dim2, UNITS[unit], n_points,
                              1 if radial_range else 0, rr[0], rr[1], C.byref(lut))
    if rc == -2:
        raise ValueError("pyFAI-compatible splitting exceeds the 64-million-entry bound")
    if rc == -3:
        raise ValueError("invalid pyFAI full-splitting grid")
    if rc:
        raise MemoryError("oracle pyfai_full build failed")
    return _take(lut)


def ps1d_fractions(p: Poni, dim1: int, dim2: int, n_points: int, min: float, step: float,
                   clamp_low: bool = False, unit: str = "2th_rad") -> Lut:
    lut = _Lut()
    rc = _lib().or_ps1d_fractions(C.byref(p), dim1, dim2, UNITS[unit], n_points, min, step,
                                  1 if clamp_low else 0, C.byref(lut))
    if rc:
        raise MemoryError("oracle ps1d fractions failed")
    return _take(lut)


def build_counting1d(radial: np.ndarray, n_points: int, radial_range=None) -> Lut:
    radial = np.ascontiguousarray(radial, np.float64)
    lut = _Lut()
    rr = radial_range or (0.0, 0.0)
    rc = _lib().or_build_counting1d(_dp(radial), len(radial), n_points,
                                    1 if radial_range else 0, rr[0], rr[1], C.byref(lut))
    if rc:
        raise MemoryError("oracle counting build failed")
    return _take(lut)


def build_ss1d(p: Poni, dim1: int, dim2: int, n_points: int, n_ss: int,
               unit: str = "2th_rad", radial_range=None) -> Lut:
    lut = _Lut()
    rr = radial_range or (0.0, 0.0)
    rc = _lib().or_build_ss1d(C.byref(p), dim1, dim2, UNITS[unit], n_points, n_ss,
                              1 if radial_range else 0, rr[0], rr[1], C.byref(lut))
    if rc:
        raise MemoryError("oracle ss1d build failed")
    return _take(lut)


def compact(lut: Lut, mask: Optional[np.ndarray]) -> Lut:
    out = _Lut()
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8).ravel()
    src = lut._c()
    if _lib().or_compact(C.byref(src), _u8(m), C.byref(out)):
        raise MemoryError("oracle compaction failed")
    return _take(out)


def denominators(lut: Lut, norm: np.ndarray) -> np.ndarray:
    norm = np.ascontiguousarray(norm, np.float64)
    den = np.empty(lut.n_rows)
    src = lut._c()
    _lib().or_denominators(C.byref(src), _dp(norm), _dp(den))
    return den


def integrate_strict(lut: Lut, den: np.ndarray, signal: np.ndarray, errors: bool = True):
    signal = np.ascontiguousarray(signal, np.float64).ravel()
    y, e = np.empty(lut.n_rows), np.empty(lut.n_rows)
    src = lut._c()
    _lib().or_integrate_strict(C.byref(src), _dp(np.ascontiguousarray(den, np.float64)),
                               _dp(signal), 1 if errors else 0, _dp(y), _dp(e))
    return y, (e if errors else None)


def row_sums(lut: Lut, signal: np.ndarray):
    signal = np.ascontiguousarray(signal, np.float64).ravel()
    s, v = np.empty(lut.n_rows), np.empty(lut.n_rows)
    src = lut._c()
    _lib().or_row_sums(C.byref(src), _dp(signal), _dp(s), _dp(v))
    return s, v


def raw_sums(lut: Lut, mask: Optional[np.ndarray], norm: np.ndarray, signal: np.ndarray):
    """(S, N, V, C) per row over the entries whose pixel is unmasked
    (row(), src/lut/prepared.rs:1011-1118, strict order)."""
    signal = np.ascontiguousarray(signal, np.float64).ravel()
    norm = np.ascontiguousarray(norm, np.float64).ravel()
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8).ravel()
    out = [np.empty(lut.n_rows) for _ in range(4)]
    src = lut._c()
    _lib().or_raw_sums(C.byref(src), _u8(m), _dp(norm), _dp(signal), *[_dp(o) for o in out])
    return tuple(out)


def azimuthal_std(lut: Lut, mask: Optional[np.ndarray], norm: np.ndarray,
                  signal: np.ndarray, variance: Optional[np.ndarray] = None):
    signal = np.ascontiguousarray(signal, np.float64).ravel()
    norm = np.ascontiguousarray(norm, np.float64).ravel()
    var = None if variance is None else np.ascontiguousarray(variance, np.float64).ravel()
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8).ravel()
    y, e, s = np.empty(lut.n_rows), np.empty(lut.n_rows), np.empty(lut.n_rows)
    src = lut._c()
    _lib().or_azimuthal_std(C.byref(src), _u8(m), _dp(norm), _dp(signal), _dp(var),
                            _dp(y), _dp(e), _dp(s))
    return y, (e if variance is not None else None), s


def integrate_frames_mt(table: Lut, den: np.ndarray, full: Lut, mask, norm, frames: np.ndarray,
                        errors: bool, azimuthal_std: bool, threads: int):
    """Frames (n, dim1, dim2) of u16/u32/i32/f32/f64, integrated frame-parallel."""
    frames = np.ascontiguousarray(frames)
    n = frames.shape[0]
    npix = int(np.prod(frames.shape[1:]))
    nb = table.n_rows
    oi, os_, od = np.empty((n, nb)), np.empty((n, nb)), np.empty((n, nb))
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8).ravel()
    t_c, f_c = table._c(), full._c()
    rc = _lib().or_integrate_frames_mt(
        C.byref(t_c), _dp(np.ascontiguousarray(den, np.float64)), C.byref(f_c), _u8(m),
        _dp(np.ascontiguousarray(norm, np.float64)), frames.ctypes.data_as(C.c_void_p),
        DTYPES[frames.dtype], npix, n, 1 if errors else 0, 1 if azimuthal_std else 0,
        int(threads), _dp(oi), _dp(os_) if errors else None,
        _dp(od) if azimuthal_std else None)
    if rc:
        raise MemoryError("oracle frame integration failed")
    return oi, (os_ if errors else None), (od if azimuthal_std else None)
