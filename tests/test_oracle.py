"""CPU tests of the oracle (oracle/cuhre_oracle.c): the rule's algebra, the
analytic integrals, and the reference algorithm's invariants.

The reference repository ships no tests or golden vectors, so the rule is
pinned by its own known answers (exactness degrees, point counts, weight
sums, null-rule normalisation restated here independently) and the full
algorithm by analytic integrals and by outputs of the reference engine run
on a B200 (test_golden.py)."""
import itertools
import math

import numpy as np
import pytest


def monomials(n, deg):
    for c in itertools.combinations_with_replacement(range(n), deg):
        p = np.zeros(n, dtype=int)
        for i in c:
            p[i] += 1
        yield p


def exact_centered(p):
    # integral of prod (x_i - 1/2)^p_i over [0,1]^n
    return float(np.prod([(0.5 ** (k + 1) - (-0.5) ** (k + 1)) / (k + 1) for k in p]))


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 7, 8, 10])
def test_point_counts(oracle, n):
    R = oracle.Rule(n)
    g, s = R.points()
    t = R.tables()
    # quad/quad.h:83-85 and GPUQuadRule.cu:123-131
    assert R.npoints == 1 + 8 * n + 6 * n * (n - 1) + 4 * n * (n - 1) * (n - 2) // 3 + 2 ** n
    assert R.npoints == oracle.npoints(n)
    assert list(np.bincount(s, minlength=9)) == list(t["count"])
    assert list(t["count"]) == [1, 2 * n, 2 * n, 2 * n, 2 * n, 2 * n * (n - 1), 4 * n * (n - 1),
                                4 * n * (n - 1) * (n - 2) // 3, 2 ** n]
    # all points distinct and inside the box
    assert len({tuple(r) for r in np.round(g, 15)}) == R.npoints
    assert np.all(np.abs(g) < 0.5)


def test_known_point_counts(oracle):
    assert [oracle.npoints(n) for n in range(2, 11)] == [33, 77, 153, 273, 453, 717, 1105, 1689,
                                                          2605]


@pytest.mark.parametrize("n", [2, 3, 4])
def test_degree9_exact_all_monomials(oracle, n):
    R = oracle.Rule(n)
    g, s = R.points()
    w = R.tables()["wt"][s]
    x = -g  # x_local - 1/2
    for deg in range(0, 10):
        for p in monomials(n, deg):
            v = np.prod(x ** p, axis=1)
            assert abs(np.dot(w[:, 0], v) - exact_centered(p)) < 1e-14
            # null rules vanish through degrees 7, 7, 5, 3
            for r, top in ((1, 7), (2, 7), (3, 5), (4, 3)):
                if deg <= top:
                    assert abs(np.dot(w[:, r], v)) < 1e-13, (deg, r, p)


@pytest.mark.parametrize("n", [5, 8])
def test_degree9_exact_sampled(oracle, n):
    R = oracle.Rule(n)
    g, s = R.points()
    w = R.tables()["wt"][s, 0]
    rng = np.random.default_rng(n)
    for deg in range(0, 10):
        for _ in range(25):
            p = rng.multinomial(deg, np.ones(n) / n)
            assert abs(np.dot(w, np.prod((-g) ** p, axis=1)) - exact_centered(p)) < 1e-14
    # degree 10 is not integrated exactly
    p = np.zeros(n, dtype=int)
    p[0] = 10
    assert abs(np.dot(w, np.prod((-g) ** p, axis=1)) - exact_centered(p)) > 1e-9


@pytest.mark.parametrize("n", [2, 5, 8])
def test_null_rule_tables_restated(oracle, n):
    """Scale/Norm restated from the weight table (GPUQuadRule.cu:209-227)."""
    t = oracle.Rule(n).tables()
    wt, cnt = t["wt"], t["count"]
    for k in range(9):
        for q in range(1, 4):
            scale = 100.0 if wt[k, q] == 0 else -wt[k, q + 1] / wt[k, q]
            norm = 1.0 / sum(cnt[x] * abs(wt[x, q + 1] + scale * wt[x, q]) for x in range(9))
            assert t["scale"][k, q] == scale
            assert t["norm"][k, q] == norm


def test_rule_order_fourth_difference(oracle):
    """Points 1..4n are (+a e_d, -a e_d) of sets 1 and 2 per axis."""
    n = 5
    g, s = oracle.Rule(n).points()
    for d in range(n):
        for k, off in ((1, 1), (2, 1 + 2 * n)):
            plus, minus = g[off + 2 * d], g[off + 2 * d + 1]
            assert s[off + 2 * d] == k and s[off + 2 * d + 1] == k
            assert plus[d] > 0 and minus[d] == -plus[d]
            assert np.count_nonzero(plus) == 1


GENZ = [
    ("gaussian", [3.0, 5.0, 7.0], [0.3, 0.5, 0.6]),
    ("oscillatory", [1.1, 0.7, 1.5], [0.3, 0.0, 0.0]),
    ("corner_peak", [0.5, 1.0, 2.0], [0.0, 0.0, 0.0]),
    ("product_peak", [5.0, 10.0, 3.0], [0.2, 0.5, 0.7]),
    ("continuous", [2.0, 3.0, 1.0], [0.4, 0.5, 0.3]),
    ("discontinuous", [1.0, 2.0, 0.5], [0.6, 0.4, 0.0]),
]


@pytest.mark.parametrize("fam,a,u", GENZ)
def test_analytic_vs_quadrature(oracle, fam, a, u):
    """orc_exact against a tensor Gauss-Legendre quadrature (2-D; 3-D for the
    smooth families), split at the kinks and jumps."""
    smooth = fam in ("oscillatory", "corner_peak")
    n = 3 if smooth else 2
    a, u = a[:n], u[:n]
    f = oracle.make_integrand(fam, n, a, u)
    xs, ws = np.polynomial.legendre.leggauss(20 if smooth else 80)
    # split [0,1] at the kink/jump points for the nonsmooth families
    cuts = sorted({0.0, 1.0, *[v for v in u if 0 < v < 1]})
    pts, wts = [], []
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        pts.extend(lo + (hi - lo) * (xs + 1) / 2)
        wts.extend((hi - lo) * ws / 2)
    pts, wts = np.array(pts), np.array(wts)
    total = 0.0
    for idx in itertools.product(range(len(pts)), repeat=n):
        total += np.prod(wts[list(idx)]) * oracle.eval_integrand(f, pts[list(idx)])
    assert abs(total - oracle.exact(f)) < 1e-9 * max(1.0, abs(total))


def test_config1_reference_algorithm(oracle):
    """5-D Gaussian a=5 at epsrel 1e-3 (the small configuration)."""
    f = oracle.make_integrand("gaussian", 5, 5.0, 0.5)
    R = oracle.Rule(5)
    r = R.integrate_reference(f, 1e-3, 1e-12)
    ex = (math.sqrt(math.pi) / 5 * math.erf(2.5)) ** 5
    assert abs(oracle.exact(f) - ex) < 1e-16
    assert r["status"] == 0
    assert abs(r["value"] - ex) <= 1e-3 * ex
    assert r["error"] <= 1e-3 * abs(r["value"])
    assert r["phase2_regions"] == 0
    # neval = nregions * points in phase 1
    assert r["neval"] == r["nregions"] * 273


@pytest.mark.parametrize("fam,a,u", [("oscillatory", 1.1, 0.3), ("corner_peak", 0.5, 0.0)])
def test_config2_reference_algorithm(oracle, fam, a, u):
    f = oracle.make_integrand(fam, 8, a, u)
    r = oracle.Rule(8).integrate_reference(f, 1e-6, 1e-12)
    ex = oracle.exact(f)
    assert r["status"] == 0
    assert abs(r["value"] - ex) <= 1e-6 * abs(ex)


def test_split_layout(oracle):
    lo, ln = oracle.initial_grid(3)
    n = lo.shape[1]
    act = np.zeros(n, dtype=np.int32)
    act[[1, 5, 7]] = 1
    axis = np.array([i % 3 for i in range(n)], dtype=np.int32)
    clo, cln = oracle.split(lo, ln, act, axis)
    assert clo.shape == (3, 6)
    for j, i in enumerate([1, 5, 7]):
        ax = axis[i]
        for c in (0, 1):
            col = j + 3 * c
            for d in range(3):
                if d == ax:
                    assert cln[d, col] == ln[d, i] / 2
                    assert clo[d, col] == lo[d, i] + c * ln[d, i] / 2
                else:
                    assert cln[d, col] == ln[d, i] and clo[d, col] == lo[d, i]


def test_initial_grid(oracle):
    for n, d in ((2, 4), (4, 4), (5, 2), (8, 2)):
        lo, ln = oracle.initial_grid(n)
        assert lo.shape == (n, d ** n)
        assert np.all(ln == 1.0 / d)
        # every cell appears once; dimension 0 varies fastest
        assert lo[0, 1] == 1.0 / d and lo[1, 1] == 0.0
        assert len({tuple(c) for c in lo.T}) == d ** n


def test_phase2_box_refines(oracle):
    """A leftover box refined depth-first meets its own tolerance."""
    f = oracle.make_integrand("product_peak", 3, [20.0, 20.0, 20.0], [0.5, 0.5, 0.5])
    R = oracle.Rule(3)
    res, err, nreg, failed = R.phase2_box(f, [0.25, 0.25, 0.25], [0.5, 0.5, 0.5], 1e-7, 1e-12)
    assert failed == 0 and nreg >= 2
    assert err <= 1e-7 * abs(res)
    # at 1e-8 the 2048-bisection cap is hit: the box is reported as failed
    _, _, nreg, failed = R.phase2_box(f, [0.25, 0.25, 0.25], [0.5, 0.5, 0.5], 1e-8, 1e-12)
    assert failed == 1 and nreg == 2049
    # the whole-cube phase-2 run agrees with the analytic integral
    res, err, nreg, failed = R.phase2_box(f, [0, 0, 0], [1, 1, 1], 1e-8, 1e-14, 20000)
    assert failed == 0 and abs(res - oracle.exact(f)) <= 1e-8 * abs(res)


def test_sequential_cuhre(oracle):
    f = oracle.make_integrand("gaussian", 4, [4.0, 5.0, 6.0, 3.0], [0.4, 0.5, 0.6, 0.5])
    r = oracle.Rule(4).cuhre_sequential(f, 1e-6, 1e-14)
    assert r["status"] == 0
    assert abs(r["value"] - oracle.exact(f)) <= 1e-6 * oracle.exact(f)


def test_reference_phase2_path(oracle):
    """Force phase 2 with a small phase-1 cap; the result still converges."""
    f = oracle.make_integrand("product_peak", 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4])
    R = oracle.Rule(4)
    r = R.integrate_reference(f, 1e-6, 1e-12, phase1_cap=512)
    assert r["phase2_regions"] >= 512
    assert r["status"] == 0
    assert abs(r["value"] - oracle.exact(f)) <= 2e-6 * oracle.exact(f)
    # neval bookkeeping of GPUKernelquad.cu:887-888
    full = R.integrate_reference(f, 1e-6, 1e-12)
    assert full["status"] == 0


def test_unit_box_is_the_default(oracle):
    """An explicit [0,1]^n box reproduces the default domain bit for bit."""
    R = oracle.Rule(4)
    a, u = [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4]
    r0 = R.integrate_reference(oracle.make_integrand("product_peak", 4, a, u), 1e-6, 1e-12)
    r1 = R.integrate_reference(oracle.make_integrand("product_peak", 4, a, u, lo=0.0, hi=1.0),
                               1e-6, 1e-12)
    assert r0 == r1


@pytest.mark.parametrize("fam", ["gaussian", "product_peak"])
def test_box_integration(oracle, fam):
    """Integration over a non-unit box (the reference's Volume) against the
    closed form over that box, by both CPU engines."""
    lo, hi = [-0.5, 0.25, 1.0], [0.75, 2.0, 1.5]
    f = oracle.make_integrand(fam, 3, [3.0, 5.0, 4.0], [0.1, 0.9, 1.2], lo=lo, hi=hi)
    ex = oracle.exact(f)
    assert math.isfinite(ex) and ex > 0
    R = oracle.Rule(3)
    r = R.integrate_reference(f, 1e-8, 1e-14)
    assert r["status"] == 0
    assert abs(r["value"] - ex) <= 1e-8 * ex
    s = R.cuhre_sequential(f, 1e-8, 1e-14)
    assert s["status"] == 0
    assert abs(s["value"] - ex) <= 1e-8 * ex
