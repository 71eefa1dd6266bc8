"""Seeded synthetic inputs for the Fourier central-slice path (numpy, host side).

No public dataset is involved: volumes, slices and orientations are generated from a seed with the
shapes and value distributions of the workloads this library is measured on.

* Volumes: rfft grids D x H x (W/2+1), complex64, value (a + ib)/sqrt(2) with a, b ~ N(0,1), times
  the amplitude 1/max(|f|, 1/64) where f is the voxel's fftfreq norm.
* Slices: complex Gaussian times the envelope exp(-B f^2 / 4) (pixel size 1), f the 2-D fftfreq norm.
* Orientations: uniform on SO(3) from normalised 4-D Gaussian quaternions, composed into matrices in
  float64 and then cast to float32.
"""
from __future__ import annotations

import numpy as np


def index2frequency(i: np.ndarray, n: int, centered: bool) -> np.ndarray:
    if centered:
        return i - n // 2
    return np.where(i < (n + 1) // 2, i, i - n)


def grid_fftfreq_norm(shape3: tuple, centered: bool) -> np.ndarray:
    """|fftfreq| of every element of a D x H x (W/2+1) rfft grid (depth and height (non-)centered)."""
    D, H, W = shape3
    fz = index2frequency(np.arange(D), D, centered) / D
    fy = index2frequency(np.arange(H), H, centered) / H
    fx = np.arange(W // 2 + 1) / W
    return np.sqrt(fz[:, None, None] ** 2 + fy[None, :, None] ** 2 + fx[None, None, :] ** 2)


def slice_fftfreq_norm(shape2: tuple, centered: bool) -> np.ndarray:
    H, W = shape2
    fy = index2frequency(np.arange(H), H, centered) / H
    fx = np.arange(W // 2 + 1) / W
    return np.sqrt(fy[:, None] ** 2 + fx[None, :] ** 2)


def complex_gaussian(rng: np.random.Generator, shape: tuple) -> np.ndarray:
    a = rng.standard_normal(shape, dtype=np.float32)
    b = rng.standard_normal(shape, dtype=np.float32)
    return ((a + 1j * b) * np.float32(1 / np.sqrt(2))).astype(np.complex64)


def make_volume(n: int | tuple, seed: int = 0, centered: bool = True) -> np.ndarray:
    """rfft volume of shape (1, D, H, W/2+1), complex64, amplitude 1/max(|f|, 1/64)."""
    shape3 = (n, n, n) if isinstance(n, int) else tuple(n)
    rng = np.random.default_rng(seed)
    D, H, W = shape3
    v = complex_gaussian(rng, (D, H, W // 2 + 1))
    amp = 1.0 / np.maximum(grid_fftfreq_norm(shape3, centered), 1.0 / 64)
    return (v * amp.astype(np.float32))[None].astype(np.complex64)


def make_slices(count: int, n: int | tuple, seed: int = 1, bfactor: float = 100.0,
                centered: bool = False) -> np.ndarray:
    """rfft slices of shape (B, 1, H, W/2+1), complex64, complex Gaussian x exp(-B f^2 / 4)."""
    H, W = (n, n) if isinstance(n, int) else tuple(n)
    rng = np.random.default_rng(seed)
    s = complex_gaussian(rng, (count, H, W // 2 + 1))
    env = np.exp(-bfactor * slice_fftfreq_norm((H, W), centered) ** 2 / 4).astype(np.float32)
    return (s * env)[:, None].astype(np.complex64)


def random_quaternions(count: int, seed: int = 2) -> np.ndarray:
    """Uniform SO(3) quaternions, float64, stored z, y, x, w."""
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def quaternion_to_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrices (float64) of z,y,x,w quaternions, acting on (z, y, x) column vectors."""
    z, y, x, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    tx, ty, tz = 2 * x, 2 * y, 2 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    m = np.empty((q.shape[0], 3, 3))
    m[:, 0, 0] = 1 - (txx + tyy)
    m[:, 0, 1] = tyz + twx
    m[:, 0, 2] = txz - twy
    m[:, 1, 0] = tyz - twx
    m[:, 1, 1] = 1 - (txx + tzz)
    m[:, 1, 2] = txy + twz
    m[:, 2, 0] = txz + twy
    m[:, 2, 1] = txy - twz
    m[:, 2, 2] = 1 - (tyy + tzz)
    return m


def random_rotations(count: int, seed: int = 2) -> np.ndarray:
    """Uniform SO(3) rotation matrices (count, 3, 3), composed in float64, returned as float32."""
    return quaternion_to_matrix(random_quaternions(count, seed)).astype(np.float32)


def rotate_y(angles_rad: np.ndarray) -> np.ndarray:
    """Matrices rotating (z, y, x) vectors about the y axis (float64)."""
    c, s = np.cos(angles_rad), np.sin(angles_rad)
    m = np.zeros((len(angles_rad), 3, 3))
    m[:, 0, 0] = c
    m[:, 0, 2] = -s
    m[:, 1, 1] = 1
    m[:, 2, 0] = s
    m[:, 2, 2] = c
    return m


def rotate_z(angles_rad: np.ndarray) -> np.ndarray:
    c, s = np.cos(angles_rad), np.sin(angles_rad)
    m = np.zeros((len(angles_rad), 3, 3))
    m[:, 0, 0] = 1
    m[:, 1, 1] = c
    m[:, 1, 2] = s
    m[:, 2, 1] = -s
    m[:, 2, 2] = c
    return m


def scale_matrices(count: int, scale: tuple, seed: int | None = None, jitter: float = 0.0) -> np.ndarray:
    """(count, 2, 2) float32 diagonal (H, W) scaling matrices, optionally with seeded jitter."""
    m = np.zeros((count, 2, 2), dtype=np.float64)
    m[:, 0, 0] = scale[0]
    m[:, 1, 1] = scale[1]
    if jitter:
        rng = np.random.default_rng(seed)
        m += rng.uniform(-jitter, jitter, size=m.shape)
    return m.astype(np.float32)
