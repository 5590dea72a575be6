"""Device tables for the table integrands, and the seeded synthetic tables
of the benchmark workloads.

Tables are FP64 torch tensors on the context's device; the C structs
(cub_interp2d, cub_spline1d, cub_lclt_tables, cub_table7) point into them, so
a table object must outlive every integration that uses it.

Synthetic data (no network, no physics tables are shipped):

* ``table7_data(seed)`` -- the 7-D workload: a 512-knot cubic spline on
  [0, 1] with positive log-normal-shaped values, a 128 x 128 bilinear grid on
  [0, 1]^2 from a seeded sum of 2-D Gaussians plus a floor, sigma = 0.25, and
  ``table7_offsets(count, seed)`` mu offsets uniform in [-1, 1].
* ``lclt_data(seed)`` -- an LC_LT-shaped table set: 22 lt knots
  (geometric, 1..160) x 5 zt knots (0.1..0.3), smooth tau, mu, sigma, fmsk,
  fprj of the magnitudes the reference's cluster model uses.
"""
from __future__ import annotations

import ctypes as C

import numpy as np


class CInterp2D(C.Structure):
    _fields_ = [("xs", C.c_void_p), ("ys", C.c_void_p), ("zs", C.c_void_p), ("nx", C.c_int),
                ("ny", C.c_int)]


class CSpline1D(C.Structure):
    _fields_ = [("xs", C.c_void_p), ("ys", C.c_void_p), ("y2", C.c_void_p), ("n", C.c_int)]


class CLcLtTables(C.Structure):
    _fields_ = [("t", CInterp2D * 5)]


class CTable7(C.Structure):
    _fields_ = [("spline", CSpline1D), ("grid", CInterp2D), ("sigma", C.c_double)]


def table7_data(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    sx = np.linspace(0.0, 1.0, 512)
    # log-normal shape in x0, positive everywhere
    sy = np.exp(-(np.log(0.05 + sx) - np.log(0.35)) ** 2 / (2 * 0.6 ** 2)) + 0.05
    gx = np.linspace(0.0, 1.0, 128)
    gy = np.linspace(0.0, 1.0, 128)
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    gz = np.full_like(X, 0.2)
    for _ in range(8):
        w = rng.uniform(0.5, 1.5)
        cx, cy = rng.uniform(0.0, 1.0, 2)
        s = rng.uniform(0.1, 0.3)
        gz += w * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    return {"spline_x": sx, "spline_y": sy, "grid_x": gx, "grid_y": gy, "grid_z": gz,
            "sigma": 0.25}


def table7_offsets(count: int, seed: int = 1) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, count)


def lclt_data(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    lt = np.geomspace(1.0, 160.0, 22)
    zt = np.linspace(0.1, 0.3, 5)
    L, Z = np.meshgrid(lt, zt, indexing="ij")
    wob = 1 + 0.02 * rng.standard_normal(L.shape)  # seeded small roughness
    tau = 0.8 / (1.0 + 0.02 * L) * wob
    mu = np.log(L) * (1.0 + 0.5 * Z)
    sigma = 0.3 + 0.2 * Z + 0.02 * np.log(L)
    fmsk = 0.05 + 0.3 * Z
    fprj = 0.1 + 0.2 * L / (L + 20.0)
    return {"xs": lt, "ys": zt, "z": [tau, mu, sigma, fmsk, fprj]}


class DeviceTables:
    """FP64 copies of host arrays on a CUDA device (kept alive here)."""

    def __init__(self, device: int = 0):
        import torch

        self._torch = torch
        self._device = torch.device("cuda", device)
        self._keep = []

    def put(self, a) -> int:
        t = self._torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(self._device)
        self._keep.append(t)
        return t.data_ptr()


class Table7(DeviceTables):
    """The 7-D integrand's spline and grid on the device."""

    def __init__(self, data: dict, device: int = 0):
        super().__init__(device)
        from . import spline_second_derivatives

        y2 = spline_second_derivatives(data["spline_x"], data["spline_y"])
        gz = np.asarray(data["grid_z"], dtype=np.float64)
        self.c = CTable7(
            CSpline1D(self.put(data["spline_x"]), self.put(data["spline_y"]), self.put(y2),
                      len(data["spline_x"])),
            CInterp2D(self.put(data["grid_x"]), self.put(data["grid_y"]), self.put(gz.ravel()),
                      gz.shape[0], gz.shape[1]),
            float(data["sigma"]))
        self.data = data


class LcLtTables(DeviceTables):
    """The five LC_LT tables on the device (one shared grid)."""

    def __init__(self, data: dict, device: int = 0):
        super().__init__(device)
        xs, ys = self.put(data["xs"]), self.put(data["ys"])
        nx, ny = len(data["xs"]), len(data["ys"])
        self.c = CLcLtTables()
        for q in range(5):
            self.c.t[q] = CInterp2D(xs, ys, self.put(np.asarray(data["z"][q]).ravel()), nx, ny)
        self.data = data
