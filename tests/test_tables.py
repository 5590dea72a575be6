"""Table integrands on the CPU: the oracle's FP64 Interp2D, spline and the
LC_LT / 7-D table integrands, and the library's host spline solver."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "old-gpuintegration_b200"))


def test_table_cell_convention(oracle):
    """The cell left of the first knot >= t (the reference's SmallNearestN,
    GPUQuadInterp2D.cu:50-67), clamped to the table."""
    xs = np.array([0.0, 1.0, 2.5, 4.0, 7.0])
    L = oracle.lib()
    cell = lambda t: L.orc_table_cell(xs.ctypes.data_as(C.POINTER(C.c_double)), 5, t)
    assert cell(-3.0) == 0 and cell(0.0) == 0 and cell(0.5) == 0
    assert cell(1.0) == 0  # on a knot: the cell to its left
    assert cell(1.0000001) == 1 and cell(2.5) == 1 and cell(6.9) == 3
    assert cell(7.0) == 3 and cell(100.0) == 3


def test_bilinear_reproduces_bilinear_functions(oracle):
    """z = a + b x + c y + d x y is reproduced on any rectilinear grid,
    inside the table and (by linear extrapolation) outside it."""
    rng = np.random.default_rng(4)
    xs = np.sort(rng.uniform(0, 10, 9))
    ys = np.sort(rng.uniform(-2, 3, 6))
    a, b, c, d = 0.3, -1.2, 2.0, 0.7
    z = a + b * xs[:, None] + c * ys[None, :] + d * xs[:, None] * ys[None, :]
    t = oracle.interp2d(xs, ys, z)
    for x, y in rng.uniform([-2, -4], [12, 5], (200, 2)):
        want = a + b * x + c * y + d * x * y
        assert abs(oracle.interp2d_eval(t, x, y) - want) <= 1e-11 * (1 + abs(want))


def test_spline_second_derivatives_library_matches_oracle(cub, oracle):
    rng = np.random.default_rng(8)
    xs = np.cumsum(rng.uniform(0.05, 0.3, 40))
    ys = np.sin(xs) + 0.1 * xs
    lib = cub.spline_second_derivatives(xs, ys)
    ora = oracle.spline_second_derivs(xs, ys)
    assert lib[0] == 0 and lib[-1] == 0
    assert np.allclose(lib, ora, rtol=1e-13, atol=1e-13)


def test_spline_accuracy(oracle):
    xs = np.linspace(0, 1, 41)
    s = oracle.spline1d(xs, np.sin(3 * xs))
    for t in np.linspace(0.02, 0.98, 37):
        assert abs(oracle.spline_eval(s, t) - np.sin(3 * t)) < 2e-5
    # linear data is reproduced exactly by a natural spline
    s1 = oracle.spline1d(xs, 2 * xs - 1)
    assert abs(oracle.spline_eval(s1, 0.3141) - (2 * 0.3141 - 1)) < 1e-14


def test_lclt_oracle_converges(oracle):
    from cubature import tables as T

    d = T.lclt_data(0)
    f = oracle.make_lclt(d["xs"], d["ys"], d["z"], [1.0, 0.1, 0.0], [100.0, 0.3, 6.0])
    R = oracle.Rule(3)
    r5 = R.integrate_reference(f, 1e-5, 1e-12)
    r6 = R.integrate_reference(f, 1e-6, 1e-12)
    assert r5["status"] == r6["status"] == 0
    assert abs(r5["value"] - r6["value"]) <= 2e-5 * abs(r6["value"])
    # the integrand is a density in lc times smooth terms: positive value
    assert r6["value"] > 0


def test_table7_oracle_converges(oracle):
    from cubature import tables as T

    d = T.table7_data(0)
    off = T.table7_offsets(2)
    R = oracle.Rule(7)
    for o in off:
        f = oracle.make_table7(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"],
                               d["grid_z"], d["sigma"], o)
        r = R.integrate_reference(f, 1e-4, 1e-12, phase1_cap=1 << 28)
        g = R.integrate_global(f, 1e-4, 1e-12)
        assert r["status"] == 0 and g["status"] == 0
        assert abs(r["value"] - g["value"]) <= 3e-4 * abs(g["value"])


def test_synthetic_tables_are_seeded_and_positive():
    from cubature import tables as T

    a, b = T.table7_data(0), T.table7_data(0)
    assert np.array_equal(a["grid_z"], b["grid_z"]) and a["grid_z"].shape == (128, 128)
    assert a["spline_x"].shape == (512,) and (a["spline_y"] > 0).all() and (a["grid_z"] > 0).all()
    o = T.table7_offsets(256)
    assert o.shape == (256,) and o.min() >= -1 and o.max() <= 1
    L = T.lclt_data(0)
    assert L["xs"].shape == (22,) and L["ys"].shape == (5,) and len(L["z"]) == 5
