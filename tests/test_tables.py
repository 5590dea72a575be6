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


def _table7_bruteforce(oracle, d, offset, n=40):
    """The 7-D table integral by tensor Gauss-Legendre: the spline with 4
    points per knot cell (exact for its cubics), the bilinear grid by its
    trapezoid sum, the 4-D kernel with n points per axis."""
    sx, sy = d["spline_x"], d["spline_y"]
    sp = oracle.spline1d(sx, sy)
    xg, wg = np.polynomial.legendre.leggauss(4)
    s_int = 0.0
    for i in range(len(sx) - 1):
        a, b = sx[i], sx[i + 1]
        for x, w in zip(0.5 * (b - a) * xg + 0.5 * (a + b), 0.5 * (b - a) * wg):
            s_int += w * oracle.spline_eval(sp, x)
    gx, gy, gz = d["grid_x"], d["grid_y"], d["grid_z"]
    g_int = np.sum(np.outer(np.diff(gx), np.diff(gy)) / 4 *
                   (gz[:-1, :-1] + gz[1:, :-1] + gz[:-1, 1:] + gz[1:, 1:]))
    x, w = np.polynomial.legendre.leggauss(n)
    x, w = 0.5 * x + 0.5, 0.5 * w
    X3, X4, X5, X6 = np.meshgrid(x, x, x, x, indexing="ij")
    W = np.einsum("i,j,k,l->ijkl", w, w, w, w)
    r = 4 * X3 - (offset + 2 * X4 + 0.1 * (X5 + X6))
    k_int = np.sum(W * np.exp(-r * r / (2 * d["sigma"] ** 2)))
    return s_int * g_int * k_int


def test_table7_exact_matches_bruteforce(oracle):
    """The closed form of the 7-D table integral agrees with a tensor
    Gauss-Legendre evaluation of the same integrand to 1e-13."""
    from cubature import tables as T

    d = T.table7_data(0)
    for o in list(T.table7_offsets(256)[:2]) + [-1.0, 1.0]:
        ex = oracle.table7_exact(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"],
                                 d["grid_z"], d["sigma"], o)
        bf = _table7_bruteforce(oracle, d, o)
        assert abs(ex - bf) <= 1e-13 * abs(ex), (o, ex, bf)


def test_table7_exact_fixture(oracle):
    """tests/golden/table7_exact.json (tests/golden/make_table7_exact.py)
    holds the closed-form values of all 256 benchmark offsets; the oracle
    reproduces them, and its adaptive integration agrees at epsrel 1e-4."""
    import json
    from pathlib import Path

    from cubature import tables as T

    fx = json.loads((Path(__file__).resolve().parent / "golden" / "table7_exact.json").read_text())
    d = T.table7_data(0)
    offs = T.table7_offsets(256)
    assert np.array_equal(np.array(fx["offsets"]), offs)
    for i in (0, 17, 255):
        ex = oracle.table7_exact(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"],
                                 d["grid_z"], d["sigma"], offs[i])
        assert ex == fx["exact"][i]
    f = oracle.make_table7(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"], d["grid_z"],
                           d["sigma"], offs[0])
    g = oracle.Rule(7).integrate_global(f, 1e-4, 1e-12)
    assert g["status"] == 0
    assert abs(g["value"] - fx["exact"][0]) <= 1e-4 * abs(fx["exact"][0])
