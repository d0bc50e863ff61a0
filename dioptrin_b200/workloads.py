"""Detector workloads used by the tests and the benchmark: seeded synthetic
stand-ins with the shapes, geometries, masks and value distributions of the
five benchmark configurations (Pilatus-1M-, Eiger-4M- and Eiger-9M-shaped
detectors). No external dataset is read.

Expected-intensity images are built on the host with NumPy (powder rings at
chosen 2-theta on a background, bright texture spots on ring pixels); Poisson
sampling of many frames is done on the GPU with torch when frames are needed
there (``frames_torch``), or with NumPy for small CPU cases.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class Workload:
    name: str
    dim1: int
    dim2: int
    pixel: float
    distance: float
    poni1: float
    poni2: float
    rot1: float = 0.0
    rot2: float = 0.0
    rot3: float = 0.0
    wavelength: float = 1e-10
    method: str = "pixel_split"
    n_ss: Optional[int] = None
    n_points: int = 1000
    polarization_factor: Optional[float] = None
    dtype: str = "uint32"
    errors: bool = True
    azimuthal_std: bool = False
    n_frames: int = 1
    n_azimuthal: int = 0  # > 0: a 2D cake of n_azimuthal x n_points bins
    azimuthal_range: Optional[tuple] = None
    kind: str = "counts"  # expected_image kind of the frames
    gaps: tuple = ()  # (module rows, module cols, module h, module w, gap h, gap w)
    dead_fraction: float = 0.0
    seed: int = 20261203

    @property
    def shape(self):
        return (self.dim1, self.dim2)

    def poni_dict(self) -> dict:
        return dict(pixel1=self.pixel, pixel2=self.pixel, distance=self.distance,
                    poni1=self.poni1, poni2=self.poni2, rot1=self.rot1, rot2=self.rot2,
                    rot3=self.rot3, wavelength=self.wavelength)

    def mask(self) -> np.ndarray:
        """Module gaps plus seeded dead pixels; nonzero = masked."""
        m = np.zeros(self.shape, np.uint8)
        if self.gaps:
            mr, mc, mh, mw, gh, gw = self.gaps
            rows = np.ones(self.dim1, bool)
            cols = np.ones(self.dim2, bool)
            for r in range(mr):
                rows[r * (mh + gh): r * (mh + gh) + mh] = False
            for c in range(mc):
                cols[c * (mw + gw): c * (mw + gw) + mw] = False
            m[rows, :] = 1
            m[:, cols] = 1
        if self.dead_fraction > 0:
            rng = np.random.default_rng(self.seed + 7)
            m[rng.random(self.shape) < self.dead_fraction] = 1
        return m

    def tth(self) -> np.ndarray:
        """Approximate centre 2-theta per pixel, for drawing rings (not the
        integration geometry)."""
        i = (np.arange(self.dim1) + 0.5) * self.pixel - self.poni1
        j = (np.arange(self.dim2) + 0.5) * self.pixel - self.poni2
        d1, d2 = np.meshgrid(i, j, indexing="ij")
        c1, s1 = math.cos(self.rot1), math.sin(self.rot1)
        c2, s2 = math.cos(self.rot2), math.sin(self.rot2)
        L = self.distance
        x = d1 * c2 - L * (c1 * s2)
        y = d2 * c1 - L * (-s1)
        z = d1 * s2 - d2 * c2 * s1 + L * c1 * c2
        return np.arctan2(np.sqrt(x * x + y * y), z)


PILATUS_1M = Workload(
    name="pilatus1m_ps1250", dim1=1043, dim2=981, pixel=172e-6, distance=0.200,
    poni1=0.0897, poni2=0.0844, wavelength=0.4e-10, n_points=1250, polarization_factor=0.99,
    dtype="int32", errors=True, n_frames=256, gaps=(5, 2, 195, 487, 17, 7))

EIGER_4M = Workload(
    name="eiger4m_ps2000_b256", dim1=2167, dim2=2070, pixel=75e-6, distance=0.15,
    poni1=(2167 / 2 + 40) * 75e-6, poni2=(2070 / 2 - 25) * 75e-6, rot1=0.02, rot2=-0.01,
    wavelength=0.3e-10, n_points=2000, dtype="uint32", errors=True, azimuthal_std=True,
    n_frames=256, gaps=(4, 2, 514, 1030, 37, 10), dead_fraction=0.02)

EIGER_4M_F32 = Workload(
    name="eiger4m_ps3000_f32", dim1=2167, dim2=2070, pixel=75e-6, distance=0.15,
    poni1=(2167 / 2 + 40) * 75e-6, poni2=(2070 / 2 - 25) * 75e-6, rot1=0.02, rot2=-0.01,
    wavelength=0.3e-10, n_points=3000, dtype="float32", errors=True, azimuthal_std=True,
    n_frames=128, kind="precision", gaps=(4, 2, 514, 1030, 37, 10), dead_fraction=0.02)

EIGER_9M = Workload(
    name="eiger9m_ss4", dim1=3269, dim2=3110, pixel=75e-6, distance=0.25,
    poni1=0.5 * 3269 * 75e-6, poni2=40 * 75e-6, rot1=0.05, wavelength=0.3e-10,
    method="supersampled", n_ss=4, n_points=1000, dtype="uint16", errors=False,
    n_frames=64, gaps=(6, 3, 514, 1030, 37, 10))

# Eiger-9M-shaped 2D cakes: 1000 radial x 360 azimuthal bins over (-pi, pi),
# beam near one edge so the chi seam crosses the detector.
EIGER_9M_2D_SS4 = Workload(
    name="eiger9m_2d_ss4", dim1=3269, dim2=3110, pixel=75e-6, distance=0.25,
    poni1=0.5 * 3269 * 75e-6, poni2=40 * 75e-6, rot1=0.05, wavelength=0.3e-10,
    method="supersampled", n_ss=4, n_points=1000, n_azimuthal=360,
    azimuthal_range=(-math.pi, math.pi), dtype="uint16", errors=True, n_frames=64,
    gaps=(6, 3, 514, 1030, 37, 10))

EIGER_9M_2D_PF = Workload(
    name="eiger9m_2d_pyfai", dim1=3269, dim2=3110, pixel=75e-6, distance=0.25,
    poni1=0.5 * 3269 * 75e-6, poni2=40 * 75e-6, rot1=0.05, wavelength=0.3e-10,
    method="pyfai_full", n_points=1000, n_azimuthal=360, azimuthal_range=(-math.pi, math.pi),
    dtype="uint16", errors=True, n_frames=64, gaps=(6, 3, 514, 1030, 37, 10))

WORKLOADS = {w.name: w for w in (PILATUS_1M, EIGER_4M, EIGER_4M_F32, EIGER_9M, EIGER_9M_2D_SS4,
                                 EIGER_9M_2D_PF)}


def expected_image(w: Workload, kind: str = "counts") -> np.ndarray:
    """Expected intensity (float64) before Poisson sampling.

    counts: background plus Gaussian rings (FWHM 0.05 deg) at seeded 2-theta
    with log-uniform amplitudes; the Eiger workloads add 1% low-frequency
    background modulation and texture spots (10-100x the ring on 1% of ring
    pixels). precision: 1e6 background with 1e-3 Gaussian relative variation
    and rings of amplitude 1e2.
    """
    rng = np.random.default_rng(w.seed)
    tth = np.degrees(w.tth())
    if kind == "precision":
        img = 1e6 * (1.0 + 1e-3 * rng.standard_normal(w.shape))
        for c in rng.uniform(2.0, 30.0, 20):
            img += 1e2 * np.exp(-0.5 * ((tth - c) / (0.05 / 2.3548)) ** 2)
        return img
    if w.name.startswith("pilatus"):
        bg, n_rings, lo, hi, amp = 50.0, 12, 2.0, 25.0, (200.0, 5000.0)
    elif w.name.startswith("eiger4m"):
        bg, n_rings, lo, hi, amp = 1e4, 20, 2.0, 33.0, (500.0, 5000.0)
    else:
        bg, n_rings, lo, hi, amp = 200.0, 20, 2.0, 30.0, (200.0, 2000.0)
    img = np.full(w.shape, bg)
    if w.name.startswith("eiger4m"):
        yy, xx = np.meshgrid(np.linspace(0, 1, w.dim1), np.linspace(0, 1, w.dim2),
                             indexing="ij")
        img *= 1.0 + 0.01 * np.sin(2 * np.pi * 1.3 * yy) * np.cos(2 * np.pi * 0.7 * xx)
    centres = rng.uniform(lo, hi, n_rings)
    amps = np.exp(rng.uniform(np.log(amp[0]), np.log(amp[1]), n_rings))
    sigma = 0.05 / 2.3548
    rings = np.zeros(w.shape)
    for c, a in zip(centres, amps):
        rings += a * np.exp(-0.5 * ((tth - c) / sigma) ** 2)
    if w.name.startswith("eiger4m"):
        ring_px = rings > 0.1 * rings.max()
        spots = ring_px & (rng.random(w.shape) < 0.01)
        rings[spots] *= rng.uniform(10.0, 100.0, int(spots.sum()))
    return img + rings


def frames_numpy(w: Workload, n: int, kind: str = "counts") -> np.ndarray:
    """n seeded frames in the workload's dtype (host memory)."""
    lam = expected_image(w, kind)
    rng = np.random.default_rng(w.seed + 1)
    dt = np.dtype(w.dtype)
    out = np.empty((n,) + w.shape, dt)
    for k in range(n):
        if kind == "precision":
            out[k] = (lam * (1.0 + 1e-3 * rng.standard_normal(w.shape))).astype(dt)
        else:
            f = rng.poisson(lam)
            out[k] = f.astype(dt)
    if w.gaps and np.issubdtype(dt, np.signedinteger):
        out[:, w.mask().astype(bool) & _gap_mask(w)] = -1
    return out


def _gap_mask(w: Workload) -> np.ndarray:
    g = Workload(**{**w.__dict__, "dead_fraction": 0.0})
    return g.mask().astype(bool)


def frames_torch(w: Workload, n: int, device: str = "cuda", kind: str = "counts"):
    """n seeded frames generated on the device (torch Poisson sampling)."""
    import torch

    lam = torch.from_numpy(expected_image(w, kind)).to(device=device, dtype=torch.float32)
    gen = torch.Generator(device=device)
    gen.manual_seed(w.seed + 1)
    dt = {"uint16": torch.uint16, "uint32": torch.uint32, "int32": torch.int32,
          "float32": torch.float32, "float64": torch.float64}[w.dtype]
    out = torch.empty((n,) + w.shape, dtype=dt, device=device)
    gaps = torch.from_numpy(_gap_mask(w)).to(device) if w.gaps else None
    for k in range(n):
        if kind == "precision":
            f = lam * (1.0 + 1e-3 * torch.randn(w.shape, generator=gen, device=device))
        else:
            f = torch.poisson(lam, generator=gen)
        if dt in (torch.uint16, torch.uint32):
            out[k] = f.to(torch.int64).to(dt)
        else:
            out[k] = f.to(dt)
        if gaps is not None and dt == torch.int32:
            out[k][gaps] = -1
    return out
