"""Python surface of the B200 integration path, mirroring the reference's
Python bindings (dioptrin.pyi: ``Integrator`` :337, ``batch1d`` :845,
``batch1d_iter`` :906, ``Cuda1dPlan`` :1358) so existing callers keep working.

Every integration runs on the GPU through libdioptrin_b200.so; there is no
CPU path. Without a usable device the calls raise ``CudaUnavailableError``,
as the reference's CUDA plans do.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
from dataclasses import dataclass
from typing import Iterable, Iterator, Optional, Sequence, Union

import numpy as np

from . import _native as N
from ._native import CudaUnavailableError

_DTYPES = {np.dtype(np.uint16): 0, np.dtype(np.uint32): 1, np.dtype(np.int32): 2,
           np.dtype(np.float32): 3, np.dtype(np.float64): 4}


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Poni:
    """Calibration (src/poni.rs:13-24), SI units, radians."""
    pixel1: float = 0.0
    pixel2: float = 0.0
    distance: float = 0.0
    poni1: float = 0.0
    poni2: float = 0.0
    rot1: float = 0.0
    rot2: float = 0.0
    rot3: float = 0.0
    wavelength: float = 0.0

    _KEYS = {"PixelSize1": "pixel1", "PixelSize2": "pixel2", "Distance": "distance",
             "Poni1": "poni1", "Poni2": "poni2", "Rot1": "rot1", "Rot2": "rot2",
             "Rot3": "rot3", "Wavelength": "wavelength"}

    @classmethod
    def load(cls, path: str) -> "Poni":
        """Parse a v1 or v2 PONI file (Poni::load, src/poni.rs:79-137)."""
        poni = cls()
        with open(path) as f:
            for line in f:
                if line.lstrip().startswith("#") or ":" not in line:
                    continue
                key, value = (s.strip() for s in line.split(":", 1))
                if key in cls._KEYS:
                    setattr(poni, cls._KEYS[key], float(value))
                elif key == "Detector_config":
                    cfg = json.loads(value)
                    if not isinstance(cfg, dict):
                        raise ValueError("Detector_config must be a JSON object")
                    for k in ("pixel1", "pixel2"):
                        if cfg.get(k) is not None:
                            setattr(poni, k, float(cfg[k]))
        if poni.pixel1 == 0.0 or poni.pixel2 == 0.0:
            raise ValueError(f"{path}: missing pixel sizes (pixel1/pixel2) in PONI file")
        return poni

    @classmethod
    def from_dict(cls, d: dict) -> "Poni":
        return cls(**{k: float(d.get(k, 0.0)) for k in (
            "pixel1", "pixel2", "distance", "poni1", "poni2", "rot1", "rot2", "rot3",
            "wavelength")})

    def _c(self) -> N.Geometry:
        g = N.Geometry()
        for k in ("pixel1", "pixel2", "distance", "poni1", "poni2", "rot1", "rot2", "rot3",
                  "wavelength"):
            setattr(g, k, float(getattr(self, k)))
        return g


class IntegrationResult:
    """One integrated pattern (src/python/results.rs); lists like the
    reference, with ``*_array`` NumPy views."""

    def __init__(self, radial, intensity, errors=None, azimuthal_std=None, azimuthal=None,
                 n_radial=None, n_azimuthal=None):
        self.radial_array = None if radial is None else np.asarray(radial)
        self.intensity_array = np.asarray(intensity)
        self.errors_array = None if errors is None else np.asarray(errors)
        self.azimuthal_std_array = None if azimuthal_std is None else np.asarray(azimuthal_std)
        self.azimuthal_array = None if azimuthal is None else np.asarray(azimuthal)
        self.n_radial = n_radial
        self.n_azimuthal = n_azimuthal

    radial = property(lambda s: None if s.radial_array is None else s.radial_array.tolist())
    intensity = property(lambda s: s.intensity_array.tolist())
    errors = property(lambda s: None if s.errors_array is None else s.errors_array.tolist())
    azimuthal_std = property(
        lambda s: None if s.azimuthal_std_array is None else s.azimuthal_std_array.tolist())
    azimuthal = property(
        lambda s: None if s.azimuthal_array is None else s.azimuthal_array.tolist())


class IntermediateResult1d:
    """Sums before division (IntermediateResult1d, src/lut/integrate.rs:372-379):
    per bin sum_signal = sum w*s, sum_norm = sum w*norm, sum_variance =
    sum w^2*max(s,0) (None unless requested) and count = sum w. ``bins`` is the
    radial axis (the bin index order of a 2D plan's rows otherwise)."""

    def __init__(self, bins, sum_signal, sum_norm, sum_variance, count):
        self.bins = np.asarray(bins)
        self.sum_signal = np.asarray(sum_signal)
        self.sum_norm = np.asarray(sum_norm)
        self.sum_variance = None if sum_variance is None else np.asarray(sum_variance)
        self.count = np.asarray(count)


class BatchResult:
    """One batch item (dioptrin.pyi:243-275)."""

    def __init__(self, filename: str, result: Optional[IntegrationResult] = None,
                 error: Optional[str] = None):
        self.filename = filename
        self.result = result
        self.error = error

    def is_ok(self) -> bool:
        return self.error is None

    def is_err(self) -> bool:
        return self.error is not None


def _frame_array(image) -> np.ndarray:
    if isinstance(image, (str, bytes, os.PathLike)):
        raise TypeError("file inputs are decoded by the caller; pass a 2D NumPy array")
    a = np.asarray(image)
    if a.dtype not in _DTYPES:
        raise TypeError(f"unsupported dtype {a.dtype}; expected float64, float32, uint16, "
                        "uint32 or int32")
    if a.ndim != 2 or a.size == 0:
        raise ValueError("image must be a non-empty 2D array")
    if not a.flags.c_contiguous:
        raise ValueError("image must be C-contiguous")
    return a


_BSLZ4_DTYPES = {"uint16": N.DG_U16, "u16": N.DG_U16, "uint32": N.DG_U32, "u32": N.DG_U32,
                 "int32": N.DG_I32, "i32": N.DG_I32}


def _bslz4_dtype(dtype) -> int:
    key = np.dtype(dtype).name if not isinstance(dtype, str) else dtype
    if key not in _BSLZ4_DTYPES:
        raise TypeError(f"dtype must be 'uint16', 'uint32' or 'int32', got {dtype!r}")
    return _BSLZ4_DTYPES[key]


def _chunk_buffers(chunks) -> list:
    """uint8 views of a list or tuple of byte buffers (python/cuda.rs:897-913)."""
    if not isinstance(chunks, (list, tuple)):
        raise TypeError(f"chunks must be a list or tuple of byte buffers, got "
                        f"{type(chunks).__name__}")
    out = []
    for c in chunks:
        try:
            m = memoryview(c)
        except TypeError as e:
            raise TypeError(f"chunk must support the byte buffer protocol: {e}") from None
        if not m.c_contiguous:
            raise ValueError("chunk buffer must be C contiguous")
        out.append(np.frombuffer(m.cast("B") if m.format != "B" or m.ndim != 1 else m,
                                 np.uint8))
    return out


def bslz4_compress(frame: np.ndarray, block_bytes: int = 0) -> bytes:
    """One raw HDF5 Bitshuffle/LZ4 chunk of a uint16, uint32 or int32 frame,
    written by the library's host encoder (block_bytes 0: 8192-byte blocks)."""
    a = np.ascontiguousarray(frame)
    _bslz4_dtype(a.dtype)
    cap = N.lib().dg_bslz4_bound(a.size, a.itemsize, block_bytes)
    if cap < 0:
        raise ValueError("invalid Bitshuffle/LZ4 arguments")
    out = np.empty(cap, np.uint8)
    n = C.c_int64(0)
    N.check(N.lib().dg_bslz4_compress(a.ctypes.data, a.size, a.itemsize, block_bytes,
                                      out.ctypes.data, cap, C.byref(n)))
    return out[:n.value].tobytes()


class _PinnedHost:
    """Page-locked host memory from dg_host_alloc, freed with its last view."""

    def __init__(self, device: int, nbytes: int):
        p = C.c_void_p()
        N.check(N.lib().dg_host_alloc(int(device), int(nbytes), C.byref(p)))
        self.ptr, self.nbytes = p.value, int(nbytes)

    def __del__(self):
        ptr, self.ptr = getattr(self, "ptr", None), None
        if ptr:
            try:
                N.lib().dg_host_free(C.c_void_p(ptr))
            except Exception:
                pass


def alloc_pinned(shape, dtype, device: int = 0) -> np.ndarray:
    """A writable NumPy array in page-locked host memory: host-memory calls
    copy from it by DMA, without the driver's staging copy."""
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) * dt.itemsize
    owner = _PinnedHost(device, max(n, 1))
    buf = (C.c_uint8 * max(n, 1)).from_address(owner.ptr)
    buf._owner = owner
    return np.frombuffer(buf, np.uint8)[:n].view(dt).reshape(shape)


def is_pinned(a) -> bool:
    """Whether an array's memory is page-locked (is_pinned_host,
    src/integration/cuda/device.rs:1055-1078)."""
    ptr = a.ctypes.data if isinstance(a, np.ndarray) else int(a)
    return bool(N.lib().dg_host_is_pinned(C.c_void_p(ptr)))


_INPUT_ORDERS = {"detector": 0, "flip_vertical": 1}


class Cuda1dPlan:
    """A fixed-mask table resident in HBM (src/integration/cuda.rs:374-618).

    Created by ``Integrator.prepare_cuda1d``. Calls on one plan are serialised
    (a lock in the library); separate plans may run concurrently. The plan is
    a snapshot: later changes to the Integrator do not affect it."""

    def __init__(self, handle, shape, n_points, precision, device, n_azimuthal=0):
        self._h = handle
        self.shape = tuple(shape)
        self.n_points = n_points
        self.n_azimuthal = n_azimuthal
        self.precision = precision
        self.device = device
        info = self.info()
        self.table_entries = info.table_entries
        self.max_batch_frames = info.max_batch_frames
        rad = np.empty(n_points)
        N.check(N.lib().dg_plan_radial(self._h, _dp(rad), n_points))
        self._radial = rad
        dev = N.DeviceInfo()
        N.check(N.lib().dg_device_info_get(device, C.byref(dev)))
        self.device_name = dev.name.decode()

    @property
    def radial(self) -> list:
        return self._radial.tolist()

    @property
    def radial_array(self) -> np.ndarray:
        return self._radial

    @property
    def handle(self):
        return self._h

    def info(self) -> N.PlanInfo:
        info = N.PlanInfo()
        N.check(N.lib().dg_plan_query(self._h, C.byref(info)))
        return info

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().dg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export_table(self, which: int = 0):
        """(row_ptr, col, weight, denominator) of the masked (0) or unmasked
        (1, needs keep_tables) table, for parity checks."""
        info = self.info()
        nnz = info.table_entries if which == 0 else info.full_entries
        nb = self.n_points * max(1, self.n_azimuthal)
        rp = np.empty(nb + 1, np.int64)
        col = np.empty(max(nnz, 1), np.int32)
        w = np.empty(max(nnz, 1))
        den = np.empty(nb) if which == 0 else None
        N.check(N.lib().dg_plan_export_table(
            self._h, which, rp.ctypes.data_as(C.POINTER(C.c_int64)),
            col.ctypes.data_as(C.POINTER(C.c_int32)), _dp(w), _dp(den)))
        return rp, col[:nnz], w[:nnz], den

    def integrate_stack(self, stack: np.ndarray, errors: bool = False,
                        azimuthal_std: bool = False):
        """Integrate (n, dim1, dim2) frames; returns (I, sigma, std) arrays of
        shape (n, n_bins), sigma/std None when not requested."""
        stack = np.ascontiguousarray(stack)
        if stack.dtype not in _DTYPES:
            raise TypeError(f"unsupported dtype {stack.dtype}")
        if stack.ndim == 2:
            stack = stack[None]
        if tuple(stack.shape[1:]) != self.shape:
            raise ValueError(f"frames of shape {stack.shape[1:]} do not match plan {self.shape}")
        n = stack.shape[0]
        nb = self.n_points * max(1, self.n_azimuthal)
        flags = (N.DG_ERRORS if errors else 0) | (N.DG_AZIMUTHAL_STD if azimuthal_std else 0)
        oi = np.empty((n, nb))
        os_ = np.empty((n, nb)) if errors else None
        od = np.empty((n, nb)) if azimuthal_std else None
        N.check(N.lib().dg_integrate(self._h, stack.ctypes.data, _DTYPES[stack.dtype], n, flags,
                                     _dp(oi), _dp(os_), _dp(od)))
        return oi, os_, od

    def autotune(self, frames, *, errors: bool = False, azimuthal_std: bool = False):
        """Time every lane mapping of the gather on `frames` (a CUDA tensor
        of shape (n, dim1, dim2) on the plan's device) and keep the fastest
        for this plan. Returns (mapping index, [launch ms of every mapping])."""
        if getattr(frames, "is_cuda", False) is not True:
            raise TypeError("autotune takes device-resident frames (a CUDA tensor)")
        import torch
        codes = {torch.uint16: 0, torch.uint32: 1, torch.int32: 2, torch.float32: 3,
                 torch.float64: 4}
        if frames.dtype not in codes:
            raise TypeError(f"unsupported dtype {frames.dtype}")
        frames = frames.contiguous()
        if tuple(frames.shape[-2:]) != self.shape:
            raise ValueError(f"frames of shape {tuple(frames.shape[-2:])} do not match plan "
                             f"{self.shape}")
        n = frames.numel() // (self.shape[0] * self.shape[1])
        flags = (N.DG_ERRORS if errors else 0) | (N.DG_AZIMUTHAL_STD if azimuthal_std else 0)
        count = C.c_int32(0)
        N.check(N.lib().dg_plan_variant(self._h, -1, None, C.byref(count)))
        v, ms = C.c_int32(0), (C.c_double * count.value)()
        stream = torch.cuda.current_stream(frames.device).cuda_stream
        N.check(N.lib().dg_plan_autotune(self._h, C.c_void_p(frames.data_ptr()),
                                         codes[frames.dtype], n, flags, C.c_void_p(stream),
                                         C.byref(v), ms, count.value))
        return v.value, list(ms)

    @property
    def gather_variant(self) -> int:
        cur = C.c_int32(0)
        N.check(N.lib().dg_plan_variant(self._h, -1, C.byref(cur), None))
        return cur.value

    @gather_variant.setter
    def gather_variant(self, v: int) -> None:
        N.check(N.lib().dg_plan_variant(self._h, int(v), None, None))

    def integrate_bslz4_stack(self, chunks, dtype: str = "uint32", errors: bool = False,
                              azimuthal_std: bool = False):
        """Decode raw HDF5 Bitshuffle/LZ4 chunks (one per frame) on the GPU
        and integrate them (Cuda1dPlan::integrate_bslz4,
        src/integration/cuda.rs:554-564); returns (I, sigma, std) arrays of
        shape (n, n_bins) as integrate_stack does."""
        code = _bslz4_dtype(dtype)
        bufs = _chunk_buffers(chunks)
        n = len(bufs)
        nb = self.n_points * max(1, self.n_azimuthal)
        flags = (N.DG_ERRORS if errors else 0) | (N.DG_AZIMUTHAL_STD if azimuthal_std else 0)
        oi = np.empty((n, nb))
        os_ = np.empty((n, nb)) if errors else None
        od = np.empty((n, nb)) if azimuthal_std else None
        if n == 0:
            return oi, os_, od
        ptrs = (C.c_void_p * n)(*[b.ctypes.data for b in bufs])
        lens = (C.c_int64 * n)(*[b.nbytes for b in bufs])
        N.check(N.lib().dg_integrate_bslz4(self._h, ptrs, lens, n, code, flags, _dp(oi),
                                           _dp(os_), _dp(od)))
        return oi, os_, od

    def batch1d_bslz4(self, chunks, dtype: str = "uint32", *, errors: bool = False) -> list:
        """Python Cuda1dPlan.batch1d_bslz4 (src/python/cuda.rs:880-930):
        `chunks` is a list or tuple of byte buffers (bytes, bytearray,
        memoryview, C-contiguous uint8 arrays), one raw chunk per frame."""
        i, s, _ = self.integrate_bslz4_stack(chunks, dtype, errors)
        return [IntegrationResult(self._radial, i[k], None if s is None else s[k])
                for k in range(len(i))]

    def _stack_and_masks(self, frames, masks):
        stack = np.ascontiguousarray(frames)
        if stack.dtype not in _DTYPES:
            raise TypeError(f"unsupported dtype {stack.dtype}")
        if stack.ndim == 2:
            stack = stack[None]
        if tuple(stack.shape[1:]) != self.shape:
            raise ValueError(f"frames of shape {stack.shape[1:]} do not match plan {self.shape}")
        if masks is None:
            return stack, None, 0
        m = np.ascontiguousarray(masks)
        if m.dtype == np.bool_:
            m = m.view(np.uint8)
        if m.dtype != np.uint8:
            raise TypeError(f"masks must be uint8 (or bool), got {m.dtype}")
        if m.shape == self.shape:
            return stack, m, 0
        if m.shape != stack.shape:
            raise ValueError(f"masks of shape {m.shape} match neither the plan {self.shape} "
                             f"nor the frames {stack.shape}")
        return stack, m, self.shape[0] * self.shape[1]

    def integrate_dynamic_stack(self, frames, masks, errors: bool = False):
        """Integrate frames with per-frame masks (MaskMode::Dynamic,
        src/integration/dynamic.rs:159-196): `masks` is one (dim1, dim2)
        uint8 mask for every frame or one per frame; nonzero masks a pixel.
        Denominators are summed over each frame's unmasked entries. Returns
        (I, sigma) arrays of shape (n, n_bins), sigma None unless errors."""
        if masks is None:
            raise ValueError("per-frame masks are required")
        stack, m, stride = self._stack_and_masks(frames, masks)
        n = stack.shape[0]
        nb = self.n_points * max(1, self.n_azimuthal)
        oi = np.empty((n, nb))
        os_ = np.empty((n, nb)) if errors else None
        N.check(N.lib().dg_integrate_dynamic(self._h, stack.ctypes.data, _DTYPES[stack.dtype], n,
                                             m.ctypes.data, stride,
                                             N.DG_ERRORS if errors else 0, _dp(oi), _dp(os_)))
        return oi, os_

    def integrate_raw_stack(self, frames, masks=None, with_variance: bool = False) -> list:
        """Raw sums of every frame (Integrator::integrate1d_raw*,
        src/integration/methods.rs:299-360) as IntermediateResult1d; masks
        None uses the plan's own mask, else per-frame masks as in
        integrate_dynamic_stack."""
        stack, m, stride = self._stack_and_masks(frames, masks)
        n = stack.shape[0]
        nb = self.n_points * max(1, self.n_azimuthal)
        out = [np.empty((n, nb)) for _ in range(4)]
        if not with_variance:
            out[2] = None
        N.check(N.lib().dg_integrate_raw(self._h, stack.ctypes.data, _DTYPES[stack.dtype], n,
                                         None if m is None else m.ctypes.data, stride,
                                         N.DG_ERRORS if with_variance else 0, _dp(out[0]),
                                         _dp(out[1]), _dp(out[2]), _dp(out[3])))
        bins = self._radial if not self.n_azimuthal else np.arange(nb, dtype=np.float64)
        return [IntermediateResult1d(bins, out[0][k], out[1][k],
                                     None if out[2] is None else out[2][k], out[3][k])
                for k in range(n)]

    def integrate1d_raw(self, image, *, with_variance: bool = False,
                        mask=None) -> IntermediateResult1d:
        return self.integrate_raw_stack(_frame_array(image), mask, with_variance)[0]

    def alloc_pinned_batch(self, n_frames: int, dtype=None) -> np.ndarray:
        """Python Cuda1dPlan.alloc_pinned_batch (src/python/cuda.rs:808-870): a
        writable (n_frames, dim1, dim2) array in page-locked host memory
        (float32 unless dtype is given) for readers to decode into; integrating
        from it copies by DMA."""
        dt = np.dtype("float32" if dtype is None else dtype)
        if dt not in _DTYPES:
            raise TypeError(f"dtype must be native uint16, uint32, int32, float32 or float64, "
                            f"got {dt}")
        if n_frames < 0:
            raise ValueError("n_frames must not be negative")
        return alloc_pinned((int(n_frames),) + self.shape, dt, self.device)

    def integrate1d(self, image: np.ndarray, *, errors: bool = False,
                    azimuthal_std: bool = False) -> IntegrationResult:
        a = _frame_array(image)
        i, s, d = self.integrate_stack(a, errors, azimuthal_std)
        return IntegrationResult(self._radial, i[0], None if s is None else s[0],
                                 None if d is None else d[0])

    def batch1d(self, images, *, errors: bool = False,
                azimuthal_std: bool = False) -> list:
        if isinstance(images, np.ndarray) and images.ndim == 3:
            stack = images
        else:
            arrays = [_frame_array(a) for a in images]
            if not arrays:
                return []
            if len({a.dtype for a in arrays}) > 1:
                raise TypeError("all images of one call must have the same dtype")
            stack = np.stack(arrays)
        i, s, d = self.integrate_stack(stack, errors, azimuthal_std)
        return [IntegrationResult(self._radial, i[k], None if s is None else s[k],
                                  None if d is None else d[k]) for k in range(len(i))]


class Cuda2dPlan(Cuda1dPlan):
    """A fixed-mask 2D table resident in HBM (src/integration/cuda.rs:620-870,
    dioptrin.pyi:1463-1520): bins are the rows a * n_radial + r of an
    n_azimuthal x n_radial cake."""

    def __init__(self, handle, shape, n_radial, n_azimuthal, precision, device,
                 axes_given: bool):
        super().__init__(handle, shape, n_radial, precision, device, n_azimuthal)
        az = np.empty(n_azimuthal)
        N.check(N.lib().dg_plan_azimuthal(self._h, _dp(az), n_azimuthal))
        self._azimuthal = az
        self._axes_given = axes_given

    @property
    def n_radial(self) -> int:
        return self.n_points

    @property
    def azimuthal(self) -> list:
        return self._azimuthal.tolist()

    @property
    def azimuthal_array(self) -> np.ndarray:
        return self._azimuthal

    def _result(self, i, s) -> IntegrationResult:
        return IntegrationResult(self._radial if self._axes_given else None, i, s,
                                 azimuthal=self._azimuthal if self._axes_given else None,
                                 n_radial=self.n_points, n_azimuthal=self.n_azimuthal)

    def integrate2d(self, image: np.ndarray, *, errors: bool = False) -> IntegrationResult:
        a = _frame_array(image)
        i, s, _ = self.integrate_stack(a, errors)
        return self._result(i[0], None if s is None else s[0])

    def batch2d(self, images, *, errors: bool = False) -> list:
        if isinstance(images, np.ndarray) and images.ndim == 3:
            stack = images
        else:
            arrays = [_frame_array(a) for a in images]
            if not arrays:
                return []
            if len({a.dtype for a in arrays}) > 1:
                raise TypeError("all images of one call must have the same dtype")
            stack = np.stack(arrays)
        i, s, _ = self.integrate_stack(stack, errors)
        return [self._result(i[k], None if s is None else s[k]) for k in range(len(i))]

    def batch2d_bslz4(self, chunks, dtype: str = "uint32", *, errors: bool = False) -> list:
        """Python Cuda2dPlan.batch2d_bslz4 (src/python/cuda.rs:1076-1125)."""
        i, s, _ = self.integrate_bslz4_stack(chunks, dtype, errors)
        return [self._result(i[k], None if s is None else s[k]) for k in range(len(i))]

    def batch2d_bslz4_stack(self, chunks, dtype: str = "uint32", *, errors: bool = False):
        """Python Cuda2dPlan.batch2d_bslz4_stack (src/python/cuda.rs:1176-1256):
        one (n_frames, n_azimuthal, n_radial) float64 array, or (intensity,
        errors) with errors=True."""
        i, s, _ = self.integrate_bslz4_stack(chunks, dtype, errors)
        shape = (len(i), self.n_azimuthal, self.n_points)
        return (i.reshape(shape), s.reshape(shape)) if errors else i.reshape(shape)

    def integrate1d(self, *a, **k):
        raise TypeError("a 2D plan integrates with integrate2d")

    batch1d = integrate1d
    batch1d_bslz4 = integrate1d


class Dynamic1dPlan:
    """A geometry-only table for frames with their own masks
    (src/integration/dynamic.rs:9-16; Python Dynamic1dPlan,
    src/python/dynamic.rs:9-50), resident on the device."""

    def __init__(self, plan: Cuda1dPlan):
        self._plan = plan

    @property
    def shape(self):
        return self._plan.shape

    @property
    def n_points(self) -> int:
        return self._plan.n_points

    @property
    def shared_plan_id(self) -> int:
        return int(self._plan.handle or 0)

    @property
    def cuda_plan(self) -> Cuda1dPlan:
        return self._plan

    def worker(self, num_threads: int = 1) -> "Dynamic1dWorker":
        if num_threads <= 0:
            raise ValueError("num_threads must be positive")
        return Dynamic1dWorker(self._plan)

    def close(self) -> None:
        self._plan.close()


class Dynamic1dWorker:
    """Dynamic1dWorker (src/python/dynamic.rs:52-110): integrates a frame
    with its complete uint8 mask; calls share the plan and keep no state."""

    def __init__(self, plan: Cuda1dPlan):
        self._plan = plan

    def integrate1d(self, image, mask=None, *, errors: bool = False,
                    azimuthal_std: bool = False) -> IntegrationResult:
        a = _frame_array(image)
        if tuple(a.shape) != self._plan.shape:
            raise ValueError("image shape does not match prepared plan")
        if azimuthal_std:
            raise ValueError("azimuthal_std is not available on the device with per-frame masks")
        if mask is None:
            mask = np.zeros(self._plan.shape, np.uint8)
        i, s = self._plan.integrate_dynamic_stack(a, mask, errors)
        return IntegrationResult(self._plan.radial_array, i[0], None if s is None else s[0])

    def batch1d(self, images, masks, *, errors: bool = False) -> list:
        """Many frames with one mask each (or one shared (dim1, dim2) mask)."""
        i, s = self._plan.integrate_dynamic_stack(images, masks, errors)
        return [IntegrationResult(self._plan.radial_array, i[k], None if s is None else s[k])
                for k in range(len(i))]


class BatchIterator(Iterator[BatchResult]):
    """Streaming results in input order (src/batch/bounded.rs:172-420,
    dioptrin.pyi:277-335): frames are gathered into device batches of up to
    ``read_ahead`` as they arrive from the source."""

    def __init__(self, integrator: "Integrator", images, n_points: int, errors: bool,
                 azimuthal_std: bool, read_ahead: int = 32):
        self._it = iter(images)
        self._int = integrator
        self._n = n_points
        self._errors = errors
        self._std = azimuthal_std
        self._read_ahead = max(1, read_ahead)
        self._pending: list = []
        self.total = len(images) if hasattr(images, "__len__") else 0
        self.completed = 0
        self._index = 0
        self._error: Optional[BaseException] = None

    @property
    def progress(self) -> Optional[float]:
        return None if not self.total else self.completed / self.total

    def __iter__(self) -> "BatchIterator":
        return self

    def _refill(self) -> None:
        frames = []
        while len(frames) < self._read_ahead:
            try:
                item = next(self._it)
            except StopIteration:
                break
            except BaseException as e:  # surfaced at this item's position
                self._error = e
                break
            frames.append(_frame_array(item))
        if frames:
            names = [f"array_{self._index + k}" for k in range(len(frames))]
            self._index += len(frames)
            results = self._int._batch_arrays(frames, self._n, self._errors, self._std)
            self._pending.extend(BatchResult(n, r) for n, r in zip(names, results))

    def __next__(self) -> BatchResult:
        if not self._pending and self._error is None:
            self._refill()
        if self._pending:
            self.completed += 1
            return self._pending.pop(0)
        if self._error is not None:
            e, self._error = self._error, None
            raise e
        raise StopIteration


class Integrator:
    """Azimuthal integrator (src/integration.rs:278-573; Python class
    src/python/integrator.rs:186). Integration runs on one CUDA device through
    device-resident plans cached per image shape and bin count."""

    def __init__(self, poni_path: Optional[str] = None, method: Optional[str] = None,
                 polarization_factor: Optional[float] = None, n_ss: Optional[int] = None,
                 unit: Optional[str] = None, radial_range=None, *, fast_math: bool = True,
                 mask_mode: str = "fixed", sparse_layout: str = "csc", device: int = 0,
                 precision: str = "f32_compensated", poni: Optional[Poni] = None):
        self.poni = poni if poni is not None else Poni.load(poni_path)
        self._method = "pixel_split"
        self._n_ss = 5
        self.set_method(method or "pixel_split", n_ss)
        self._pol = None
        self.set_polarization_factor(polarization_factor)
        self._unit = "2th_rad"
        self.set_unit(unit or "2th_rad")
        self._radial_range = None
        if radial_range is not None:
            lo, hi = (float(v) for v in radial_range)
            if not (np.isfinite(lo) and np.isfinite(hi) and lo < hi):
                raise ValueError("radial_range must be finite with min < max")
            self._radial_range = (lo, hi)
        if mask_mode not in ("fixed", "dynamic"):
            raise ValueError("mask_mode must be 'fixed' or 'dynamic'")
        if mask_mode != "fixed":
            raise ValueError("the device integrator requires mask_mode fixed")
        if sparse_layout not in ("csc", "csr"):
            raise ValueError("sparse_layout must be 'csc' or 'csr'")
        if precision not in N.PRECISIONS:
            raise ValueError(f"unknown CUDA precision {precision!r}; expected \"f32\", "
                             "\"f32_compensated\" or \"f64\"")
        self.fast_math = fast_math  # accepted for compatibility; the device order is fixed
        self.mask_mode = mask_mode
        self.sparse_layout = sparse_layout
        self.device = device
        self.precision = precision
        self._mask: Optional[np.ndarray] = None
        self._plans: dict = {}
        self._lock = threading.Lock()

    @classmethod
    def from_poni_dict(cls, poni_dict: dict, method=None, polarization_factor=None, n_ss=None,
                       unit=None, radial_range=None, **kw) -> "Integrator":
        return cls(None, method, polarization_factor, n_ss, unit, radial_range,
                   poni=Poni.from_dict(poni_dict), **kw)

    # -- configuration (src/integration.rs:319-510) --
    def set_method(self, method: str, n_ss: Optional[int] = None) -> None:
        if method not in N.METHODS:
            raise ValueError(f"unknown method {method!r}")
        if n_ss is not None and n_ss <= 0:
            raise ValueError("n_ss must be positive")
        self._method = method
        if n_ss is not None:
            self._n_ss = int(n_ss)
        self._invalidate()

    @property
    def method(self) -> str:
        return self._method

    def set_polarization_factor(self, factor: Optional[float]) -> None:
        if factor is not None and not (-1.0 <= factor <= 1.0):
            raise ValueError("polarization_factor must lie in [-1, 1]")
        self._pol = None if factor is None else float(factor)
        self._invalidate()

    def set_unit(self, unit: str) -> None:
        if unit not in N.UNITS:
            raise ValueError(f"unknown unit {unit!r}")
        if unit.startswith("q") and not self.poni.wavelength > 0:
            raise ValueError("a q unit needs a positive PONI wavelength")
        self._unit = unit
        self._invalidate()

    def get_unit(self) -> str:
        return self._unit

    def set_radial_range(self, radial_range) -> None:
        self._radial_range = None if radial_range is None else tuple(map(float, radial_range))
        self._invalidate()

    def set_mask(self, mask: Optional[np.ndarray]) -> None:
        if mask is None:
            self.clear_mask()
            return
        if isinstance(mask, (str, bytes, os.PathLike)):
            raise TypeError("mask files are decoded by the caller; pass a 2D array")
        m = np.ascontiguousarray(np.asarray(mask) != 0, np.uint8)
        if m.ndim != 2:
            raise ValueError("mask must be 2D")
        self._mask = m
        self._invalidate()

    def clear_mask(self) -> None:
        self._mask = None
        self._invalidate()

    def _invalidate(self) -> None:
        plans = getattr(self, "_plans", None)
        if plans:
            for p in plans.values():
                p.close()
            plans.clear()

    # -- plans --
    def _method_struct(self, precision: str, device: int, max_batch_bytes: int,
                       keep_tables: bool, input_order: str = "detector") -> N.Method:
        if input_order not in _INPUT_ORDERS:
            raise ValueError(f"input_order must be 'detector' or 'flip_vertical', got "
                             f"{input_order!r}")
        m = N.Method()
        m.kind = N.METHODS[self._method]
        m.n_ss = self._n_ss
        m.unit = N.UNITS[self._unit]
        m.has_polarization = 0 if self._pol is None else 1
        m.polarization_factor = 0.0 if self._pol is None else self._pol
        m.has_radial_range = 0 if self._radial_range is None else 1
        if self._radial_range is not None:
            m.radial_min, m.radial_max = self._radial_range
        m.precision = N.PRECISIONS[precision]
        m.device = device
        m.max_batch_bytes = max_batch_bytes
        m.flags = (N.DG_PLAN_KEEP_TABLES if keep_tables else 0) | (
            N.DG_PLAN_FLIP_VERTICAL if input_order == "flip_vertical" else 0)
        return m

    def prepare_cuda1d(self, shape, n_points: int, *, precision: str = "f32_compensated",
                       device: int = 0, max_batch_bytes: Optional[int] = None,
                       keep_tables: bool = False, input_order: str = "detector") -> Cuda1dPlan:
        """Integrator::prepare_cuda1d (src/integration/cuda.rs:1089): the
        table is built on the device and kept there. input_order
        "flip_vertical" takes frames bottom row first
        (Cuda1dOptions::with_input_order, cuda.rs:174-182)."""
        if precision not in N.PRECISIONS:
            raise ValueError(f"unknown CUDA precision {precision!r}")
        if device < 0:
            raise OverflowError("device must be non-negative")
        dim1, dim2 = (int(v) for v in shape)
        if max_batch_bytes is not None and max_batch_bytes <= 0:
            raise ValueError("max_batch_bytes must be positive")
        if self._mask is not None and self._mask.shape != (dim1, dim2):
            raise ValueError(f"image shape ({dim1}, {dim2}) does not match mask shape "
                             f"{self._mask.shape}")
        m = self._method_struct(precision, device, max_batch_bytes or 0, keep_tables,
                                input_order)
        h = C.c_void_p()
        mask = (None if self._mask is None
                else self._mask.ctypes.data_as(C.POINTER(C.c_uint8)))
        N.check(N.lib().dg_plan_create(C.byref(self.poni._c()), C.byref(m), mask, dim1, dim2,
                                       int(n_points), 0, None, C.byref(h)))
        return Cuda1dPlan(h, (dim1, dim2), int(n_points), precision, device)

    def prepare_cuda2d(self, shape, n_radial: int, n_azimuthal: Optional[int] = None, *,
                       azimuthal_range=None, azimuthal_bracket: Optional[float] = None,
                       precision: str = "f32_compensated", device: int = 0,
                       max_batch_bytes: Optional[int] = None,
                       keep_tables: bool = False, input_order: str = "detector") -> Cuda2dPlan:
        """Integrator::prepare_cuda2d (src/integration/cuda.rs:1111-1157): the
        2D table on the shared grid of the method (default or explicit radial
        and azimuthal edges) is built on the device and kept there."""
        if azimuthal_bracket is not None:
            raise NotImplementedError("azimuthal_bracket rows are not supported by this build; "
                                      "give n_azimuthal and azimuthal_range")
        if n_azimuthal is None:
            raise ValueError("give n_azimuthal")
        if n_radial <= 0 or n_azimuthal <= 0:
            raise ValueError("n_radial and n_azimuthal must be positive")
        if n_radial * n_azimuthal > 2147483647:
            raise ValueError(f"2D bin count ({n_radial} x {n_azimuthal}) must be in "
                             "1..=2147483647")
        if precision not in N.PRECISIONS:
            raise ValueError(f"unknown CUDA precision {precision!r}")
        if device < 0:
            raise OverflowError("device must be non-negative")
        if max_batch_bytes is not None and max_batch_bytes <= 0:
            raise ValueError("max_batch_bytes must be positive")
        dim1, dim2 = (int(v) for v in shape)
        if self._mask is not None and self._mask.shape != (dim1, dim2):
            raise ValueError(f"image shape ({dim1}, {dim2}) does not match mask shape "
                             f"{self._mask.shape}")
        m = self._method_struct(precision, device, max_batch_bytes or 0, keep_tables,
                                input_order)
        h = C.c_void_p()
        mask = (None if self._mask is None
                else self._mask.ctypes.data_as(C.POINTER(C.c_uint8)))
        rng = None
        if azimuthal_range is not None:
            rng = (C.c_double * 2)(float(azimuthal_range[0]), float(azimuthal_range[1]))
        N.check(N.lib().dg_plan_create(C.byref(self.poni._c()), C.byref(m), mask, dim1, dim2,
                                       int(n_radial), int(n_azimuthal), rng, C.byref(h)))
        axes = azimuthal_range is not None or self._radial_range is not None
        return Cuda2dPlan(h, (dim1, dim2), int(n_radial), int(n_azimuthal), precision, device,
                          axes)

    def integrate2d(self, image, n_radial: int, n_azimuthal: Optional[int] = None,
                    errors: bool = False, azimuthal_range=None, *,
                    azimuthal_bracket: Optional[float] = None) -> IntegrationResult:
        """Integrator.integrate2d (dioptrin.pyi:660-730): a flat cake of
        n_azimuthal x n_radial bins (row a * n_radial + r)."""
        a = _frame_array(image)
        key = ("2d", a.shape, int(n_radial), n_azimuthal,
               None if azimuthal_range is None else tuple(float(v) for v in azimuthal_range))
        with self._lock:
            p = self._plans.get(key)
            if p is None:
                p = self.prepare_cuda2d(a.shape, n_radial, n_azimuthal,
                                        azimuthal_range=azimuthal_range,
                                        azimuthal_bracket=azimuthal_bracket,
                                        precision=self.precision, device=self.device)
                self._plans[key] = p
        return p.integrate2d(a, errors=errors)

    def integrate2d_on_azimuthal_range(self, image, n_radial: int, n_azimuthal: int,
                                       azimuthal_range, errors: bool = False) -> IntegrationResult:
        """Integrator::integrate2d_on_azimuthal_range (src/integration/grid.rs:439)."""
        return self.integrate2d(image, n_radial, n_azimuthal, errors, azimuthal_range)

    def prepare_dynamic1d(self, shape, n_points: int, *, precision: str = "f32_compensated",
                          device: int = 0, max_batch_bytes: Optional[int] = None,
                          input_order: str = "detector") -> "Dynamic1dPlan":
        """Integrator::prepare_dynamic1d (src/integration/dynamic.rs:29-65): one
        geometry table without the stored mask, for frames that each bring
        their complete mask. Built and kept on the device."""
        saved = self._mask
        self._mask = None
        try:
            plan = self.prepare_cuda1d(shape, n_points, precision=precision, device=device,
                                       max_batch_bytes=max_batch_bytes, input_order=input_order)
        finally:
            self._mask = saved
        return Dynamic1dPlan(plan)

    def integrate1d_raw(self, image, n_points: int) -> IntermediateResult1d:
        """Integrator::integrate1d_raw (src/integration/methods.rs:318-326)."""
        a = _frame_array(image)
        return self._plan(a.shape, n_points).integrate1d_raw(a)

    def integrate1d_raw_with_variance(self, image, n_points: int) -> IntermediateResult1d:
        """Integrator::integrate1d_raw_with_variance (methods.rs:329-337)."""
        a = _frame_array(image)
        return self._plan(a.shape, n_points).integrate1d_raw(a, with_variance=True)

    def _plan(self, shape, n_points: int) -> Cuda1dPlan:
        key = (tuple(shape), int(n_points))
        with self._lock:
            p = self._plans.get(key)
            if p is None:
                p = self.prepare_cuda1d(shape, n_points, precision=self.precision,
                                        device=self.device)
                self._plans[key] = p
            return p

    # -- integration (src/integration/methods.rs) --
    def integrate1d(self, image, n_points: int, errors: bool = False, *,
                    azimuthal_std: bool = False) -> IntegrationResult:
        if n_points <= 0:
            raise ValueError("n_points must be positive")
        a = _frame_array(image)
        return self._plan(a.shape, n_points).integrate1d(a, errors=errors,
                                                         azimuthal_std=azimuthal_std)

    def integrate1d_with_errors(self, image, n_points: int) -> IntegrationResult:
        return self.integrate1d(image, n_points, True)

    def integrate1d_with_azimuthal_std(self, image, n_points: int,
                                       errors: bool = False) -> IntegrationResult:
        return self.integrate1d(image, n_points, errors, azimuthal_std=True)

    def _batch_arrays(self, arrays: Sequence[np.ndarray], n_points: int, errors: bool,
                      azimuthal_std: bool) -> list:
        out: list = [None] * len(arrays)
        groups: dict = {}
        for k, a in enumerate(arrays):
            groups.setdefault((a.shape, a.dtype), []).append(k)
        for (shape, _), idx in groups.items():
            plan = self._plan(shape, n_points)
            res = plan.batch1d(np.stack([arrays[k] for k in idx]), errors=errors,
                               azimuthal_std=azimuthal_std)
            for k, r in zip(idx, res):
                out[k] = r
        return out

    def batch1d(self, images, n_points: int, errors: bool = False,
                num_workers: Optional[int] = None, num_threads: Optional[int] = None, *,
                azimuthal_std: bool = False) -> list:
        """Integrator.batch1d (src/python/integrator.rs:1867): arrays are
        integrated as device batches; results keep the input order."""
        if isinstance(images, (str, bytes, os.PathLike)):
            raise TypeError("images must be a list; wrap one path in a list")
        if n_points <= 0:
            raise ValueError("n_points must be positive")
        arrays = [_frame_array(a) for a in images]
        results = self._batch_arrays(arrays, n_points, errors, azimuthal_std)
        return [BatchResult(f"array_{k}", r) for k, r in enumerate(results)]

    def batch1d_iter(self, images, n_points: int, errors: bool = False,
                     num_workers: Optional[int] = None, num_threads: Optional[int] = None, *,
                     azimuthal_std: bool = False) -> BatchIterator:
        """Integrator.batch1d_iter (src/python/integrator.rs:2211)."""
        if isinstance(images, (str, bytes, os.PathLike)):
            raise TypeError("images must be a list or iterable; wrap one path in a list")
        if n_points <= 0:
            raise ValueError("n_points must be positive")
        if isinstance(images, list):
            for a in images:
                _frame_array(a)
        return BatchIterator(self, images, n_points, errors, azimuthal_std,
                             read_ahead=num_workers or 32)


def cuda_info(device: int = 0) -> dict:
    """cuda_info (src/integration/cuda.rs:262-329) as a dict."""
    try:
        info = N.DeviceInfo()
        st = N.lib().dg_device_info_get(device, C.byref(info))
    except CudaUnavailableError as e:
        return {"compiled": False, "available": False, "reason": str(e), "device": device}
    if st != N.DG_OK:
        return {"compiled": True, "available": False, "reason": N.last_error(), "device": device}
    return {"compiled": True, "available": True, "reason": None, "device": device,
            "device_name": info.name.decode(), "compute_capability": (info.cc_major,
                                                                      info.cc_minor),
            "sm_count": info.sm_count, "total_memory_bytes": info.total_memory_bytes,
            "driver_version": info.driver_version}


def cuda_available(device: int = 0) -> bool:
    return bool(cuda_info(device).get("available"))
