"""GPU parity tests: the CUDA path against the CPU oracle on the same
inputs, through the C ABI.

Tolerances (FP64 throughout):
  * region value: |avg_gpu - avg_cpu| <= 1e-13 * |avg_cpu| + 1e-300
  * region error: |err_gpu - err_cpu| <= 1e-12 * |avg_cpu| + 1e-12 * err_cpu
    (the null rules difference nearly equal sums, so the error is compared
    on the scale of the value, not of itself);
  * split axis and active flag: identical, except regions whose top two
    fourth differences are within 1e-9 (relative) or whose error ratio is
    within 1e-8 of 1 -- there the last bit of exp/cos decides;
  * scan/compact/bisect: bit-exact;
  * full integrations: the oracle's region count, evaluation count and
    status exactly, |I_gpu - I_cpu| <= 1e-12 |I| (rounding of different
    summation orders), and both within their error estimates of the
    analytic value.  Integrals that enter the depth-first second phase
    compare their values within 2 epsrel and their region counts within
    0.5% (the two sides order their heap pops of equal keys differently).
"""
import math
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FAMILY_PARAMS = {
    "gaussian": (lambda n, r: (r.uniform(2, 8, n), r.uniform(0.2, 0.8, n))),
    "oscillatory": (lambda n, r: (r.uniform(0.5, 2.0, n), np.full(n, r.uniform()))),
    "corner_peak": (lambda n, r: (r.uniform(0.2, 1.5, n), np.zeros(n))),
    "product_peak": (lambda n, r: (np.exp(r.uniform(0, np.log(30), n)), r.uniform(0.1, 0.9, n))),
    "continuous": (lambda n, r: (r.uniform(1, 5, n), r.uniform(0.2, 0.8, n))),
    "discontinuous": (lambda n, r: (r.uniform(0.2, 1.0, n), r.uniform(0.3, 0.9, n))),
    "cossum": (lambda n, r: (np.ones(n), np.zeros(n))),
}


def refined_list(oracle, n, rounds, seed, frac=0.5):
    """Initial grid plus `rounds` random bisections: dyadic boxes as the
    engine sees them."""
    rng = np.random.default_rng(seed)
    lo, ln = oracle.initial_grid(n)
    for _ in range(rounds):
        m = lo.shape[1]
        act = (rng.uniform(size=m) < frac).astype(np.int32)
        act[0] = 1
        ax = rng.integers(0, n, size=m).astype(np.int32)
        clo, cln = oracle.split(lo, ln, act, ax)
        keep = act == 0
        lo = np.concatenate([lo[:, keep], clo], axis=1)
        ln = np.concatenate([ln[:, keep], cln], axis=1)
    return np.ascontiguousarray(lo), np.ascontiguousarray(ln)


def assert_within(got, want, bound, label):
    """Element-wise |got - want| <= bound, reporting the worst region."""
    bad = ~(np.abs(got - want) <= bound)
    if bad.any():
        i = int(np.argmax(np.where(bad, np.abs(got - want) / np.maximum(bound, 1e-300), 0)))
        raise AssertionError(f"{label}: {int(bad.sum())} regions out of tolerance; worst #{i}: "
                             f"got {got[i]!r} want {want[i]!r} bound {bound[i]!r}")


def compare_regions(o, g, label):
    avg_c, err_c, mag = o["avg"], o["err"], o["mag"]
    avg_g, err_g, ax_g, act_g = [t.cpu().numpy() for t in g]
    # rounding scale: |avg| plus the L1 magnitude of the rule sum (matters
    # where the integrand cancels over a region)
    scale = np.abs(avg_c) + mag
    assert_within(avg_g, avg_c, 1e-13 * scale + 1e-300, ("avg",) + tuple(label))
    assert_within(err_g, err_c, 1e-12 * scale + 1e-12 * err_c + 1e-300, ("err",) + tuple(label))
    clear_axis = o["margin"] > 1e-9
    assert np.array_equal(ax_g[clear_axis], o["axis"][clear_axis]), label
    clear_ratio = np.abs(o["ratio"] - 1) > 1e-8
    assert np.array_equal(act_g[clear_ratio], o["active"][clear_ratio]), label
    return int((~clear_axis).sum()), int((~clear_ratio).sum())


@pytest.mark.parametrize("family", sorted(FAMILY_PARAMS))
@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_rule_eval_matches_oracle(cub, oracle, ctx, family, n):
    rng = np.random.default_rng(zlib.crc32(f"{family}-{n}".encode()))
    a, u = FAMILY_PARAMS[family](n, rng)
    rounds = {2: 6, 3: 5, 5: 4, 8: 2}[n]
    lo, ln = refined_list(oracle, n, rounds, seed=n)
    f_c = oracle.make_integrand(family, n, a, u)
    f_g = cub.Integrand(family, n, list(a), list(u))
    for eps in (1e-3, 1e-6):
        o = oracle.Rule(n).phase1_eval(f_c, lo, ln, eps, 1e-12)
        dlo = torch.from_numpy(lo).cuda()
        dln = torch.from_numpy(ln).cuda()
        g = cub.rule_eval(f_g, dlo, dln, eps, 1e-12)
        torch.cuda.synchronize()
        compare_regions(o, g, (family, n, eps))


@pytest.mark.parametrize("family,n", [("product_peak", 5), ("gaussian", 8), ("oscillatory", 6)])
def test_rule_eval_large_list(cub, oracle, ctx, family, n):
    """A list long enough for the thread-per-region kernel (>= 148*512)."""
    rng = np.random.default_rng(7)
    a, u = FAMILY_PARAMS[family](n, rng)
    lo, ln = refined_list(oracle, n, 30 if n == 5 else 24, seed=3, frac=0.15)
    while lo.shape[1] < 80000:
        lo = np.concatenate([lo, lo], axis=1)
        ln = np.concatenate([ln, ln], axis=1)
    lo, ln = np.ascontiguousarray(lo[:, :80000]), np.ascontiguousarray(ln[:, :80000])
    f_c = oracle.make_integrand(family, n, a, u)
    o = oracle.Rule(n).phase1_eval(f_c, lo, ln, 1e-5, 1e-12)
    g = cub.rule_eval(cub.Integrand(family, n, list(a), list(u)), torch.from_numpy(lo).cuda(),
                      torch.from_numpy(ln).cuda(), 1e-5, 1e-12)
    torch.cuda.synchronize()
    compare_regions(o, g, (family, n))


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("n", [2, 5, 8])
def test_split_bit_exact(cub, oracle, ctx, layout, n):
    rng = np.random.default_rng(n + 10 * layout)
    lo, ln = refined_list(oracle, n, 3, seed=n)
    m = lo.shape[1]
    act = (rng.uniform(size=m) < 0.4).astype(np.int32)
    ax = rng.integers(0, n, size=m).astype(np.int32)
    clo, cln = oracle.split(lo, ln, act, ax)
    glo, gln = cub.split(torch.from_numpy(lo).cuda(), torch.from_numpy(ln).cuda(),
                         torch.from_numpy(act).cuda(), torch.from_numpy(ax).cuda(), layout=layout)
    glo, gln = glo.cpu().numpy(), gln.cpu().numpy()
    k = clo.shape[1] // 2
    if layout == 1:  # adjacent children -> reference layout
        order = np.concatenate([np.arange(0, 2 * k, 2), np.arange(1, 2 * k, 2)])
        glo, gln = glo[:, order], gln[:, order]
    assert glo.shape == clo.shape
    assert np.array_equal(glo, clo) and np.array_equal(gln, cln)


def test_split_empty_and_all(cub, oracle, ctx):
    lo, ln = oracle.initial_grid(3)
    z = np.zeros(lo.shape[1], dtype=np.int32)
    glo, _ = cub.split(torch.from_numpy(lo).cuda(), torch.from_numpy(ln).cuda(),
                       torch.from_numpy(z).cuda(), torch.from_numpy(z).cuda())
    assert glo.shape[1] == 0
    one = np.ones(lo.shape[1], dtype=np.int32)
    glo, gln = cub.split(torch.from_numpy(lo).cuda(), torch.from_numpy(ln).cuda(),
                         torch.from_numpy(one).cuda(), torch.from_numpy(z).cuda())
    clo, cln = oracle.split(lo, ln, one, z)
    assert np.array_equal(glo.cpu().numpy(), clo) and np.array_equal(gln.cpu().numpy(), cln)


def test_reduce(cub, ctx):
    rng = np.random.default_rng(0)
    for n in (1, 31, 1000, 300001):
        avg = rng.normal(size=n)
        err = rng.uniform(size=n) * 1e-3
        act = (rng.uniform(size=n) < 0.3).astype(np.int32)
        out = cub.reduce(torch.from_numpy(avg).cuda(), torch.from_numpy(err).cuda(),
                         torch.from_numpy(act).cuda()).cpu().numpy()
        fin = act == 0
        ref = [math.fsum(avg), math.fsum(err), math.fsum(avg[fin]), math.fsum(err[fin])]
        scale = [np.abs(avg).sum(), err.sum(), np.abs(avg).sum(), err.sum()]
        for q in range(4):
            assert abs(out[q] - ref[q]) <= 1e-13 * scale[q]


CASES = [
    # (family, ndim, a, u, epsrel) -- configuration 1, configuration 2, others
    ("gaussian", 5, 5.0, 0.5, 1e-3),
    ("oscillatory", 8, 1.1, 0.3, 1e-6),
    ("corner_peak", 8, 0.5, 0.0, 1e-6),
    ("gaussian", 3, [4.0, 6.0, 5.0], [0.3, 0.5, 0.6], 1e-7),
    ("product_peak", 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4], 1e-5),
    ("continuous", 2, [3.0, 4.0], [0.4, 0.6], 1e-5),
    ("cossum", 6, 1.0, 0.0, 1e-4),
]


def _compare_full(r_g, r_c, exact, epsrel, label, count_tol=5e-3):
    assert r_g.status == r_c["status"], label
    if r_c.get("phase2_regions", 0) == 0:
        assert r_g.nregions == r_c["nregions"], (label, r_g.nregions, r_c["nregions"])
        assert r_g.neval == r_c["neval"], label
        assert abs(r_g.integral - r_c["value"]) <= 1e-12 * abs(r_c["value"]) + 1e-300, label
    else:
        assert abs(r_g.integral - r_c["value"]) <= 2 * epsrel * abs(r_c["value"]) + 1e-15, label
        assert abs(r_g.nregions - r_c["nregions"]) <= count_tol * r_c["nregions"] + 4, label
    if r_c["status"] == 0:
        assert abs(r_g.integral - exact) <= max(10 * r_g.error, 2 * epsrel * abs(exact)), label


@pytest.mark.parametrize("family,n,a,u,epsrel", CASES)
def test_integrate_matches_oracle(cub, oracle, ctx, family, n, a, u, epsrel):
    f_c = oracle.make_integrand(family, n, a, u)
    r_c = oracle.Rule(n).integrate_reference(f_c, epsrel, 1e-12)
    r_g = ctx.integrate(cub.Integrand(family, n, a, u), epsrel, 1e-12)
    _compare_full(r_g, r_c, oracle.exact(f_c), epsrel, (family, n))
    # the GPUcuhre mirror gives the same answer
    q = cub.GPUcuhre(n).integrate(cub.Integrand(family, n, a, u), epsrel, 1e-12)
    assert q.integral == r_g.integral and q.nregions == r_g.nregions


def test_integrate_phase2_matches_oracle(cub, oracle, ctx):
    """A small phase-1 cap sends leftover boxes through the depth-first
    second phase on both sides."""
    n, a, u, eps = 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4], 1e-6
    f_c = oracle.make_integrand("product_peak", n, a, u)
    r_c = oracle.Rule(n).integrate_reference(f_c, eps, 1e-12, phase1_cap=512)
    assert r_c["phase2_regions"] > 0
    r_g = ctx.integrate(cub.Integrand("product_peak", n, a, u), eps, 1e-12,
                        cub.options(phase1_cap=512))
    _compare_full(r_g, r_c, oracle.exact(f_c), eps, "phase2", count_tol=0.05)


def test_phase2_failed_boxes_counted(cub, oracle, ctx):
    """Boxes that hit the bisection cap are counted in the status, as the
    reference's errorFlag counts failed phase-2 blocks (GPUKernelquad.cu:891)."""
    n, eps = 3, 1e-9
    a, u = [40.0, 40.0, 40.0], [0.37, 0.52, 0.61]
    f_c = oracle.make_integrand("product_peak", n, a, u)
    r_c = oracle.Rule(n).integrate_reference(f_c, eps, 1e-14, phase1_cap=64, phase2_max=64)
    r_g = ctx.integrate(cub.Integrand("product_peak", n, a, u), eps, 1e-14,
                        cub.options(phase1_cap=64, phase2_max_regions=64))
    assert r_c["status"] > 0
    assert abs(r_g.status - r_c["status"]) <= max(2, 0.05 * r_c["status"])
    assert abs(r_g.integral - r_c["value"]) <= 1e-6 * abs(r_c["value"])


def test_batch_matches_single(cub, oracle, ctx):
    rng = np.random.default_rng(3)
    n, eps = 6, 1e-4
    params, singles = [], []
    for k in range(6):
        a = np.exp(rng.uniform(0, np.log(20), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
        singles.append(ctx.integrate(cub.Integrand("product_peak", n, list(a), list(u)), eps,
                                     1e-12))
    batch = ctx.integrate_batch("product_peak", n, params, eps, 1e-12)
    for b, s in zip(batch, singles):
        # the batched path loads parameters from memory instead of kernel
        # arguments, which may change FMA contraction in the last bit
        assert abs(b.integral - s.integral) <= 1e-13 * abs(s.integral)
        assert abs(b.error - s.error) <= 1e-10 * abs(s.error)
        assert b.nregions == s.nregions and b.status == s.status


def test_grouped_breadth_batch_equals_one_group(cub, ctx):
    """A breadth-policy batch of 1100 integrals under a small region capacity
    runs as a 256-integral probe group and groups sized from its peak (plus
    reruns in smaller groups if one still overflows).  Integrals share no
    arithmetic, but the group size decides which kernel evaluates an
    iteration (the persistent kernel for short lists, the multi-launch rule
    kernel for long ones), and the two sum a region's points in different
    orders: results agree with the default-capacity run to that rounding."""
    rng = np.random.default_rng(11)
    n, count, eps = 4, 1100, 1e-4
    params = [cub.make_params(n, list(np.exp(rng.uniform(0, np.log(20), n))),
                              list(rng.uniform(0.1, 0.9, n))) for _ in range(count)]
    whole = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                                cub.options(policy=cub.POLICY_BREADTH))
    ctx.reset_stats()
    grouped = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                                  cub.options(policy=cub.POLICY_BREADTH, max_slots=1 << 19))
    assert ctx.stats()["persistent_launches"] + ctx.stats()["eval_launches"] > 0
    for k, (g, w) in enumerate(zip(grouped, whole)):
        assert g.status == w.status, k
        assert abs(g.integral - w.integral) <= 1e-3 * eps * abs(w.integral) + 1e-15, k
        assert abs(g.nregions - w.nregions) <= 0.01 * w.nregions + 4, k
    assert all(r.status == 0 for r in whole)


def test_batch_matches_oracle(cub, oracle, ctx):
    rng = np.random.default_rng(5)
    n, eps = 6, 1e-4
    params, refs = [], []
    for k in range(5):
        a = np.exp(rng.uniform(0, np.log(50), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
        f_c = oracle.make_integrand("product_peak", n, a, u)
        refs.append((oracle.Rule(n).integrate_reference(f_c, eps, 1e-12), oracle.exact(f_c)))
    out = ctx.integrate_batch("product_peak", n, params, eps, 1e-12)
    for r_g, (r_c, ex) in zip(out, refs):
        _compare_full(r_g, r_c, ex, eps, "batch")


def test_batch_generator_misses_are_the_algorithms_own(cub, oracle, ctx):
    """Product peaks of the 4096-integral batch generator (6-D, a_i
    log-uniform in [1, 50], u_i uniform in [0.1, 0.9], seed = index) whose
    breadth-first results miss the analytic value by more than epsrel while
    reporting status 0 (seeds 26, 80, 206, 663, 1190: 1.2e-5 .. 3.3e-4
    relative).  The oracle's restatement of the reference algorithm gives
    the same region count and the same value to rounding: the miss is the
    degree-9 rule's optimistic error estimate on these sharp peaks, not the
    engine."""
    import math

    seeds = [26, 80, 206, 663, 1190]
    n, eps = 6, 1e-5
    params, cases = [], []
    for k in seeds:
        rng = np.random.default_rng(k)
        a = np.exp(rng.uniform(math.log(1.0), math.log(50.0), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
        cases.append((a, u))
    out = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                              cub.options(policy=cub.POLICY_BREADTH))
    R = oracle.Rule(n)
    for r_g, (a, u), k in zip(out, cases, seeds):
        f_c = oracle.make_integrand("product_peak", n, a, u)
        r_c = R.integrate_reference(f_c, eps, 1e-12, phase1_cap=1 << 28)
        ex = oracle.exact(f_c)
        assert r_g.status == r_c["status"] == 0, k
        assert r_g.nregions == r_c["nregions"], k
        assert abs(r_g.integral - r_c["value"]) <= 1e-12 * abs(ex), k
        assert abs(r_g.integral - ex) > eps * abs(ex), k  # the documented miss


def test_breadth_policy_converges(cub, oracle, ctx):
    f = cub.Integrand("product_peak", 5, [20.0, 30.0, 10.0, 25.0, 15.0],
                      [0.3, 0.5, 0.7, 0.45, 0.6])
    r = ctx.integrate(f, 1e-6, 1e-12, cub.options(policy=cub.POLICY_BREADTH))
    ex = oracle.exact(oracle.make_integrand("product_peak", 5, f.a, f.u))
    assert r.status == 0
    assert abs(r.integral - ex) <= 2e-6 * ex


def test_repeatable(cub, ctx):
    """Fixed-order reductions: two runs give bit-identical results."""
    f = cub.Integrand("corner_peak", 8, 0.5, 0.0)
    r1 = ctx.integrate(f, 1e-6, 1e-12)
    r2 = ctx.integrate(f, 1e-6, 1e-12)
    assert r1 == r2


PERSIST_CASES = [
    ("gaussian", 5, 5.0, 0.5, 1e-3),
    ("corner_peak", 8, 0.5, 0.0, 1e-6),
    ("product_peak", 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4], 1e-5),
    ("oscillatory", 3, [3.0, 2.0, 4.0], 0.2, 1e-8),
]


@pytest.mark.parametrize("family,n,a,u,epsrel", PERSIST_CASES)
def test_persistent_matches_multilaunch(cub, oracle, ctx, family, n, a, u, epsrel):
    """The persistent kernel (block- or warp-per-region evaluation, device-side
    loop) and one launch per step agree."""
    f = cub.Integrand(family, n, a, u)
    rp = ctx.integrate(f, epsrel, 1e-12, cub.options(persistent=True))
    rm = ctx.integrate(f, epsrel, 1e-12, cub.options(persistent=False))
    assert rp.status == rm.status
    assert abs(rp.integral - rm.integral) <= 1e-3 * epsrel * abs(rm.integral) + 1e-15
    assert abs(rp.nregions - rm.nregions) <= 0.01 * rm.nregions + 4
    ctx.reset_stats()
    ctx.integrate(f, epsrel, 1e-12, cub.options(persistent=True))
    st = ctx.stats()
    assert st["persistent_launches"] >= 1


def test_persistent_hands_over_and_back(cub, oracle, ctx):
    """A small hand-over length makes the run alternate between the two
    drivers; the result does not change."""
    f = cub.Integrand("product_peak", 5, [20.0, 30.0, 10.0, 25.0, 15.0],
                      [0.3, 0.5, 0.7, 0.45, 0.6])
    ra = ctx.integrate(f, 1e-5, 1e-12, cub.options(persistent=False))
    ctx.reset_stats()
    rb = ctx.integrate(f, 1e-5, 1e-12, cub.options(persistent=True, persistent_max_n=256))
    st = ctx.stats()
    assert st["persistent_launches"] >= 1 and st["eval_launches"] >= 1
    assert rb.status == ra.status
    assert abs(rb.integral - ra.integral) <= 1e-8 * abs(ra.integral)
    assert abs(rb.nregions - ra.nregions) <= 0.01 * ra.nregions + 4
    fo = oracle.make_integrand("product_peak", 5, f.a, f.u)
    assert abs(rb.integral - oracle.exact(fo)) <= 2e-5 * oracle.exact(fo)


def test_persistent_batch(cub, oracle, ctx):
    rng = np.random.default_rng(9)
    n, eps = 6, 1e-4
    params, refs = [], []
    for k in range(7):
        a = np.exp(rng.uniform(0, np.log(50), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
        refs.append(oracle.Rule(n).integrate_reference(
            oracle.make_integrand("product_peak", n, a, u), eps, 1e-12))
    rp = ctx.integrate_batch("product_peak", n, params, eps, 1e-12, cub.options(persistent=True))
    rm = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                             cub.options(persistent=False))
    for p, m, o in zip(rp, rm, refs):
        # the reference algorithm's own answer (its error estimate can be
        # optimistic for sharp peaks, so compare with the oracle, not the
        # analytic value)
        assert p.status == m.status == o["status"]
        assert abs(p.integral - o["value"]) <= 1e-3 * eps * abs(o["value"])
        assert abs(p.nregions - o["nregions"]) <= 0.01 * o["nregions"] + 4
        assert abs(p.nregions - m.nregions) <= 0.01 * m.nregions + 4


def _peak_batch(cub, n, count, seed):
    rng = np.random.default_rng(seed)
    params = []
    for _ in range(count):
        a = np.exp(rng.uniform(0, np.log(30), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
    return params


@pytest.mark.parametrize("count", [5, 48])
def test_persistent_batch_sizes(cub, ctx, count):
    """Batches decided by one warp (up to 32 integrals) and integral by
    integral (more than 32) give the answers of one launch per step."""
    n, eps = 4, 1e-5
    params = _peak_batch(cub, n, count, 21 + count)
    ctx.reset_stats()
    rp = ctx.integrate_batch("product_peak", n, params, eps, 1e-12, cub.options(persistent=True))
    assert ctx.stats()["persistent_iterations"] >= 2
    rm = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                             cub.options(persistent=False))
    for p, m in zip(rp, rm):
        assert p.status == m.status
        assert abs(p.integral - m.integral) <= 1e-3 * eps * abs(m.integral) + 1e-15
        assert abs(p.nregions - m.nregions) <= 0.01 * m.nregions + 4


@pytest.mark.parametrize("count", [3, 40])
def test_persistent_phase2_handoff(cub, ctx, count):
    """Integrals handed to the depth-first phase inside the persistent kernel
    get the same leftover boxes, hence the same results, as with one launch
    per step."""
    n, eps = 5, 1e-6
    params = _peak_batch(cub, n, count, 5 + count)
    opts = dict(phase1_cap=256)
    ctx.reset_stats()
    rp = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                             cub.options(persistent=True, **opts))
    st = ctx.stats()
    assert st["persistent_iterations"] >= 1 and st["phase2_boxes"] > 0
    rm = ctx.integrate_batch("product_peak", n, params, eps, 1e-12,
                             cub.options(persistent=False, **opts))
    for p, m in zip(rp, rm):
        assert p.status == m.status
        assert abs(p.integral - m.integral) <= 1e-3 * eps * abs(m.integral) + 1e-15
        assert abs(p.nregions - m.nregions) <= 0.01 * m.nregions + 4


BOX_CASES = [
    ("gaussian", 3, [3.0, 5.0, 4.0], [0.1, 0.9, 1.2], [-0.5, 0.25, 1.0], [0.75, 2.0, 1.5], 1e-8),
    ("product_peak", 5, [8.0, 12.0, 6.0, 10.0, 9.0], [0.3, 1.6, -0.5, 0.4, 2.0],
     [-1.0, 1.0, -2.0, 0.0, 1.5], [1.0, 2.5, 0.5, 0.5, 2.5], 1e-6),
]


@pytest.mark.parametrize("family,n,a,u,lo,hi,epsrel", BOX_CASES)
def test_integrate_box_matches_oracle(cub, oracle, ctx, family, n, a, u, lo, hi, epsrel):
    """Integration over a non-unit FP64 box (the reference's Volume) against
    the oracle over the same box and the closed form."""
    f_c = oracle.make_integrand(family, n, a, u, lo=lo, hi=hi)
    r_c = oracle.Rule(n).integrate_reference(f_c, epsrel, 1e-14)
    r_g = ctx.integrate(cub.Integrand(family, n, a, u), epsrel, 1e-14, lo=lo, hi=hi)
    _compare_full(r_g, r_c, oracle.exact(f_c), epsrel, ("box", family, n))
    q = cub.GPUcuhre(n).integrate(cub.Integrand(family, n, a, u), epsrel, 1e-14, vol=(lo, hi))
    assert q.integral == r_g.integral and q.nregions == r_g.nregions


def test_unit_box_is_the_default(cub, ctx):
    """An explicit [0,1]^n box reproduces the unit-cube entry point bit for
    bit (same grid arithmetic)."""
    f = cub.Integrand("product_peak", 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4])
    r0 = ctx.integrate(f, 1e-6, 1e-12)
    r1 = ctx.integrate(f, 1e-6, 1e-12, lo=0.0, hi=1.0)
    assert (r1.integral, r1.error, r1.nregions, r1.status) == \
        (r0.integral, r0.error, r0.nregions, r0.status)


def test_batch_box_matches_single(cub, oracle, ctx):
    rng = np.random.default_rng(17)
    n, eps = 4, 1e-6
    params, los, his, singles = [], [], [], []
    for k in range(6):
        a = np.exp(rng.uniform(0, np.log(20), n))
        u = rng.uniform(-1, 2, n)
        lo = rng.uniform(-1, 0.5, n)
        hi = lo + rng.uniform(0.5, 2.0, n)
        params.append(cub.make_params(n, list(a), list(u)))
        los.append(list(lo))
        his.append(list(hi))
        singles.append(ctx.integrate(cub.Integrand("product_peak", n, list(a), list(u)), eps,
                                     1e-14, lo=list(lo), hi=list(hi)))
        ex = oracle.exact(oracle.make_integrand("product_peak", n, a, u, lo=lo, hi=hi))
        assert abs(singles[-1].integral - ex) <= 2 * eps * ex
    batch = ctx.integrate_batch("product_peak", n, params, eps, 1e-14, lo=los, hi=his)
    for b, s in zip(batch, singles):
        assert abs(b.integral - s.integral) <= 1e-13 * abs(s.integral)
        assert b.nregions == s.nregions and b.status == s.status


def test_box_rejects_empty_box(cub, ctx):
    f = cub.Integrand("gaussian", 3, 4.0, 0.5)
    with pytest.raises(cub.CubatureError):
        ctx.integrate(f, 1e-6, 1e-12, lo=[0.0, 0.0, 1.0], hi=[1.0, 1.0, 1.0])


def test_reference_style_functor_front_end(oracle):
    """A functor written the reference's way (double x[], int dim), compiled
    against the C++ front end (quad::GPUcuhre, quad::Volume) as a caller of
    the reference would: same answers as the oracle, unit cube and box."""
    import json
    import subprocess
    from pathlib import Path

    exe = Path(__file__).resolve().parents[1] / "old-gpuintegration_b200" / "examples" / \
        "ref_api_example"
    assert exe.exists(), "build the examples with old-gpuintegration_b200/build.py"
    eps, lo, hi = 1e-7, -0.5, 1.5
    out = subprocess.run([str(exe), repr(eps), repr(lo), repr(hi)], capture_output=True,
                         text=True, timeout=120, check=True).stdout
    rows = [json.loads(line) for line in out.splitlines() if line.startswith("{")]
    assert [r["box"] for r in rows] == [False, True]
    a, u = [8.0, 12.0, 6.0], [0.3, 0.6, 0.5]
    for r in rows:
        box = dict(lo=lo, hi=hi) if r["box"] else {}
        f_c = oracle.make_integrand("product_peak", 3, a, u, **box)
        r_c = oracle.Rule(3).integrate_reference(f_c, eps, 1e-14)
        assert r["flag"] == r_c["status"] == 0
        assert abs(r["integral"] - r_c["value"]) <= 2 * eps * abs(r_c["value"])
        assert abs(r["integral"] - oracle.exact(f_c)) <= 2 * eps * oracle.exact(f_c)
        assert abs(r["nregions"] - r_c["nregions"]) <= 0.02 * r_c["nregions"] + 4
        if r_c["phase2_regions"] == 0:
            assert r["neval"] == r["nregions"] * oracle.Rule(3).npoints


def test_lclt_matches_oracle(cub, oracle, ctx):
    """The reference's LC_LT integrand (FP64 tables) over its 3-D box."""
    from cubature import tables as T

    d = T.lclt_data(0)
    lo, hi = [1.0, 0.1, 0.0], [100.0, 0.3, 6.0]
    eps = 1e-6
    f_c = oracle.make_lclt(d["xs"], d["ys"], d["z"], lo, hi)
    r_c = oracle.Rule(3).integrate_reference(f_c, eps, 1e-12)
    tab = T.LcLtTables(d, 0)
    r_g = ctx.integrate_lclt(tab, lo, hi, eps, 1e-12)
    _compare_full(r_g, r_c, r_c["value"], eps, "lclt")


def test_table7_batch_matches_oracle(cub, oracle, ctx):
    """The 7-D spline x bilinear x Gaussian-kernel integrand, one mu offset
    per integral, breadth-first with the reference's classification."""
    from cubature import tables as T

    d = T.table7_data(0)
    offs = T.table7_offsets(3)
    eps = 1e-4
    tab = T.Table7(d, 0)
    out = ctx.integrate_table7_batch(tab, offs, eps, 1e-12,
                                     cub.options(policy=cub.POLICY_BREADTH))
    R = oracle.Rule(7)
    for r_g, o in zip(out, offs):
        f_c = oracle.make_table7(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"],
                                 d["grid_z"], d["sigma"], o)
        r_c = R.integrate_reference(f_c, eps, 1e-12, phase1_cap=1 << 28)
        _compare_full(r_g, r_c, r_c["value"], eps, ("table7", o))


def test_table7_batch_at_stated_epsrel_vs_closed_form(cub, ctx):
    """The table workload at its stated epsrel 1e-6 (breadth-first, the
    reference's classification, epsabs 1e-12), four of the 256 benchmark
    offsets, against the closed-form FP64 values of
    tests/golden/table7_exact.json (tests/golden/make_table7_exact.py):
    every integral converges (status 0) and its reported error estimate
    covers the distance to the closed form.  That distance is a few times
    epsrel |I|: the reference's per-region test lets a region finish on
    epsabs alone, and over ~2e7 regions those allowances add up (a tighter
    epsabs of 1e-15 makes the per-region relative test refine the kernel's
    tails without end: 2.5e8 regions and no convergence)."""
    import json
    from pathlib import Path

    from cubature import tables as T

    fx = json.loads((Path(__file__).resolve().parent / "golden" / "table7_exact.json").read_text())
    pick = [0, 85, 170, 255]
    offs = [fx["offsets"][i] for i in pick]
    eps = 1e-6
    tab = T.Table7(T.table7_data(0), 0)
    out = ctx.integrate_table7_batch(tab, offs, eps, 1e-12,
                                     cub.options(policy=cub.POLICY_BREADTH))
    for r_g, i in zip(out, pick):
        exact = fx["exact"][i]
        assert r_g.status == 0, (i, r_g)
        assert abs(r_g.integral - exact) <= r_g.error, (i, r_g.integral, exact, r_g.error)
        assert abs(r_g.integral - exact) <= 5 * eps * abs(exact), (i, r_g.integral, exact)


def test_autotune_picks_a_working_tiling(cub, ctx):
    """The autotuner returns one of its candidates, and the batch integrated
    with it gives the default options' answers."""
    n, eps = 5, 1e-5
    params = [cub.make_params(n, list(a), list(u)) for a, u in
              ((a, u) for a, u in _peak_params_np(n, 12, 4))]
    best, ms = ctx.autotune_batch("product_peak", n, params, eps, 1e-12)
    assert ms > 0 and best.persistent_max_r in (0, 1, 2, 4, 8) and best.lanes in (0, 1, 8, 32)
    tuned = ctx.integrate_batch("product_peak", n, params, eps, 1e-12, best)
    ref = ctx.integrate_batch("product_peak", n, params, eps, 1e-12)
    for t, r in zip(tuned, ref):
        assert t.status == r.status
        assert abs(t.integral - r.integral) <= 1e-3 * eps * abs(r.integral)


def _peak_params_np(n, count, seed):
    rng = np.random.default_rng(seed)
    return [(np.exp(rng.uniform(0, np.log(20), n)), rng.uniform(0.1, 0.9, n))
            for _ in range(count)]


def test_mixed_batch_matches_single_family(cub, ctx):
    """Integrands of different families in one call give the answers of
    separate calls (same functors; parameters read from memory may change
    FMA contraction in the last bit)."""
    cases = [("oscillatory", 8, 1.1, 0.3), ("corner_peak", 8, 0.5, 0.0)]
    fs = [cub.Integrand(f, n, a, u) for f, n, a, u in cases]
    mixed = ctx.integrate_mixed(fs, 1e-6, 1e-12)
    for f, m in zip(fs, mixed):
        s = ctx.integrate(f, 1e-6, 1e-12)
        assert m.status == s.status and m.nregions == s.nregions
        assert abs(m.integral - s.integral) <= 1e-13 * abs(s.integral)
    fams = [("gaussian", [4.0, 6.0, 5.0, 3.0], [0.3, 0.5, 0.6, 0.4]),
            ("product_peak", [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4]),
            ("continuous", [3.0, 4.0, 2.0, 5.0], [0.4, 0.6, 0.5, 0.5]),
            ("cossum", 1.0, 0.0)]
    fs = [cub.Integrand(f, 4, a, u) for f, a, u in fams]
    mixed = ctx.integrate_mixed(fs, 1e-6, 1e-12)
    for f, m in zip(fs, mixed):
        s = ctx.integrate_batch(f.family, 4, [f.params()], 1e-6, 1e-12)[0]
        assert m.status == s.status and m.nregions == s.nregions
        assert abs(m.integral - s.integral) <= 1e-13 * abs(s.integral) + 1e-15


def _same(r, s, exact, label):
    assert r.status == s.status and r.nregions == s.nregions and r.neval == s.neval, label
    assert r.iterations == s.iterations, label
    if exact:
        assert r.integral == s.integral and r.error == s.error, label
    else:
        assert abs(r.integral - s.integral) <= 1e-13 * abs(s.integral) + 1e-300, label
        assert abs(r.error - s.error) <= 1e-12 * abs(s.integral) + 1e-12 * s.error, label


def test_graph_replays_match_direct_calls(cub, ctx):
    """The default workload's two integrals captured once in a CUDA graph
    and replayed with new parameters each call give the direct calls'
    results (parameters read from device memory instead of kernel
    arguments may change FMA contraction in the last bit)."""
    g = ctx.graph([("oscillatory", 8, 1), ("corner_peak", 8, 1)])
    try:
        for a_osc, u_osc, a_cp in [(1.1, 0.3, 0.5), (0.9, 0.7, 0.8), (1.1, 0.3, 0.5)]:
            fs = [cub.Integrand("oscillatory", 8, a_osc, u_osc),
                  cub.Integrand("corner_peak", 8, a_cp, 0.0)]
            got = g.launch(fs, 1e-6, 1e-12)
            for f, r in zip(fs, got):
                _same(r, ctx.integrate(f, 1e-6, 1e-12), False, f.family)
        assert g.info() == (3, 0)
    finally:
        g.close()


def test_graph_batch_entries_equal_batch_calls(cub, ctx):
    """Batch entries (the same parameter source as cub_integrate_batch)
    reproduce cub_integrate_batch bit for bit, per-integral tolerances
    included, on two replays in a row."""
    rng = np.random.default_rng(5)
    g = ctx.graph([("product_peak", 4, 16), ("gaussian", 3, 2)])
    try:
        for rep in range(2):
            pp = [cub.Integrand("product_peak", 4, list(np.exp(rng.uniform(0, np.log(30), 4))),
                                list(rng.uniform(0.1, 0.9, 4))) for _ in range(16)]
            ga = [cub.Integrand("gaussian", 3, list(rng.uniform(2, 8, 3)),
                                list(rng.uniform(0.2, 0.8, 3))) for _ in range(2)]
            er = list(rng.choice([1e-4, 1e-5], 18))
            got = g.launch(pp + ga, er, 1e-12)
            want = ctx.integrate_batch("product_peak", 4, [f.params() for f in pp], er[:16],
                                       [1e-12] * 16)
            want += ctx.integrate_batch("gaussian", 3, [f.params() for f in ga], er[16:],
                                        [1e-12] * 2)
            for k, (r, s) in enumerate(zip(got, want)):
                _same(r, s, True, f"rep {rep} integral {k}")
        assert g.info() == (2, 0)
    finally:
        g.close()


def test_graph_finishes_through_batch_call(cub, ctx):
    """An entry whose list outgrows the persistent limit inside the replay
    is finished by cub_integrate_batch; the result is that call's."""
    opts = cub.options(persistent_max_n=512)
    f = cub.Integrand("product_peak", 6, 25.0, 0.4)
    g = ctx.graph([("product_peak", 6, 1)], opts)
    try:
        r = g.launch([f], 1e-6, 1e-12)[0]
        assert g.info() == (1, 1)
        s = ctx.integrate_batch("product_peak", 6, [f.params()], 1e-6, 1e-12, opts)[0]
        _same(r, s, True, "rerun")
        assert r.nregions > 512
    finally:
        g.close()


def test_graph_finishes_phase2_through_batch_call(cub, ctx):
    """Under the reference policy an entry whose integrals hand boxes to
    phase 2 is finished by cub_integrate_batch (phase 2 is not part of the
    graph); results equal that call's."""
    opts = cub.options(phase1_cap=256)
    fs = [cub.Integrand("product_peak", 4, a, 0.45) for a in (20.0, 30.0)]
    g = ctx.graph([("product_peak", 4, 2)], opts)
    try:
        for rep in range(2):
            got = g.launch(fs, 1e-7, 1e-12)
            want = ctx.integrate_batch("product_peak", 4, [f.params() for f in fs], 1e-7, 1e-12,
                                       opts)
            for r, s in zip(got, want):
                _same(r, s, True, f"rep {rep}")
        assert g.info() == (2, 2)
        ctx.reset_stats()
        ctx.integrate_batch("product_peak", 4, [f.params() for f in fs], 1e-7, 1e-12, opts)
        assert ctx.stats()["phase2_boxes"] > 0
    finally:
        g.close()


def test_graph_rejects_oversized_grid(cub, ctx):
    """The initial grid must fit one persistent launch."""
    with pytest.raises(cub.CubatureError) as e:
        ctx.graph([("gaussian", 8, 4)], cub.options(persistent_max_n=512))
    assert e.value.code == cub.ERR_UNSUPPORTED
    with pytest.raises(cub.CubatureError):
        ctx.graph([("gaussian", 1, 4)])


REPLICATED_CASES = [
    ("oscillatory", 8, 1.1, 0.3, 1e-6),
    ("corner_peak", 8, 0.5, 0.0, 1e-6),
    ("gaussian", 5, 5.0, 0.5, 1e-3),
    ("gaussian", 3, [4.0, 6.0, 5.0], [0.3, 0.5, 0.6], 1e-7),
    ("product_peak", 4, [8.0, 12.0, 6.0, 10.0], [0.3, 0.6, 0.5, 0.4], 1e-5),
    ("continuous", 2, [3.0, 4.0], [0.4, 0.6], 1e-5),
    ("cossum", 6, 1.0, 0.0, 1e-4),
]


def _same_bits(a, b, label):
    assert (a.integral == b.integral and a.error == b.error and a.nregions == b.nregions
            and a.neval == b.neval and a.status == b.status and a.iterations == b.iterations), \
        (label, a, b)


@pytest.mark.parametrize("family,n,a,u,epsrel", REPLICATED_CASES)
def test_replicated_kernel_bit_identical(cub, ctx, family, n, a, u, epsrel):
    """The replicated-decision kernel (batches of at most 32 integrals on
    short lists) and the persistent kernel compute the same rule sums in the
    same order and take the same decisions: identical results, bit for
    bit, including runs whose lists outgrow the replicated kernel's range
    and continue in the other drivers."""
    f = cub.Integrand(family, n, a, u)
    for max_n in (0, 96):
        o_rep = cub.options(persistent_max_n=max_n)
        o_old = cub.options(persistent_max_n=max_n, replicated=False)
        r1 = ctx.integrate(f, epsrel, 1e-12, o_rep)
        r2 = ctx.integrate(f, epsrel, 1e-12, o_old)
        _same_bits(r1, r2, (family, n, max_n))


def test_replicated_kernel_bit_identical_batches(cub, ctx):
    """Small batches (one list, several integrals, uneven difficulty), the
    reference policy with a phase-1 cap that hands boxes to phase 2, and
    non-unit boxes: the two kernels agree bit for bit."""
    rng = np.random.default_rng(7)
    n = 5
    params = [cub.make_params(n, list(np.exp(rng.uniform(0, np.log(20), n))),
                              list(rng.uniform(0.2, 0.8, n))) for _ in range(12)]
    for opts in ({}, {"phase1_cap": 2048}, {"policy": cub.POLICY_BREADTH}):
        r1 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12, cub.options(**opts))
        r2 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12,
                                 cub.options(replicated=False, **opts))
        for k, (x, y) in enumerate(zip(r1, r2)):
            _same_bits(x, y, (opts, k))
    lo = [[-1.0] * 3, [0.0, 0.5, 0.0]]
    hi = [[1.0] * 3, [2.0, 1.5, 0.5]]
    gp = [cub.make_params(3, [2.0, 3.0, 1.5], [0.2, 0.9, 0.1])] * 2
    r1 = ctx.integrate_batch("gaussian", 3, gp, 1e-7, 1e-12, lo=lo, hi=hi)
    r2 = ctx.integrate_batch("gaussian", 3, gp, 1e-7, 1e-12, cub.options(replicated=False),
                             lo=lo, hi=hi)
    for x, y in zip(r1, r2):
        _same_bits(x, y, "box")


@pytest.mark.parametrize("world", [1, 2, 3])
def test_split_second_phase_matches_whole_integral(cub, oracle, ctx, world):
    """One integral's leftover boxes cut into `world` contiguous shares
    (cub_integrate_shard), the shares run one after another on this GPU and
    combined as the all-reduce of cubature.parallel.integrate_split does:
    the single-call result -- the same region and evaluation counts and
    status, the same value and error to rounding."""
    from cubature import parallel as P

    f = cub.Integrand("product_peak", 4, [30.0, 40.0, 20.0, 35.0], [0.3, 0.6, 0.5, 0.4])
    opts = cub.options(phase1_cap=512)
    whole = ctx.integrate(f, 1e-7, 1e-12, opts)
    shares = [ctx.integrate_shard(f, 1e-7, 1e-12, r, world, opts) for r in range(world)]
    p1 = shares[0][0]
    assert all(s[0] == p1 for s in shares)  # every rank's first phase is the same
    value = p1.integral + sum(s[1].integral for s in shares)
    error = p1.error + sum(s[1].error for s in shares)
    nreg = p1.nregions + sum(s[1].nregions for s in shares)
    neval = p1.neval + sum(s[1].neval for s in shares)
    failed = sum(s[1].status for s in shares)
    status = 0 if error <= max(1e-7 * abs(value), 1e-12) else failed
    assert (nreg, neval, status) == (whole.nregions, whole.neval, whole.status)
    assert abs(value - whole.integral) <= 1e-12 * abs(whole.integral)
    assert abs(error - whole.error) <= 1e-12 * abs(whole.integral)
    # the oracle cuts its leftover list in the reference's order (first
    # children, then second children), as the engine's shares do: the same
    # first phase, and shares of the same boxes (regions within the heap-tie
    # tolerance of the second phase)
    fc = oracle.make_integrand("product_peak", 4, [30.0, 40.0, 20.0, 35.0], [0.3, 0.6, 0.5, 0.4])
    for r in range(world):
        q1, qp = oracle.Rule(4).integrate_reference_shard(fc, 1e-7, 1e-12, r, world,
                                                          phase1_cap=512)
        assert q1["nregions"] == p1.nregions and qp["phase2_regions"] > 0
        assert abs(qp["nregions"] - shares[r][1].nregions) <= 5e-3 * qp["nregions"], r
    # world 1 through the combiner is the plain result
    if world == 1:
        res = P.integrate_split(lambda r, w: ctx.integrate_shard(f, 1e-7, 1e-12, r, w, opts),
                                1e-7, 1e-12)
        assert res.nregions == whole.nregions and res.status == whole.status


def test_device_loop_bit_identical(cub, ctx):
    """Long lists run their iterations as one graph launch with a
    conditional loop (bind, rule, partials, decide, scan, split, advance,
    test) instead of host-launched chains: the same kernels in the same
    order, so results are identical bit for bit -- a batch of 64 6-D
    product peaks whose lists outgrow the persistent kernel (breadth policy
    and the reference policy with phase-2 hand-over), a single 8-D corner
    peak under a small persistent limit, a breadth batch under a small
    capacity whose loop leaves to grow the buffers, and the 7-D table
    integrand."""
    rng = np.random.default_rng(21)
    n = 6
    params = [cub.make_params(n, list(np.exp(rng.uniform(0, np.log(50), n))),
                              list(rng.uniform(0.1, 0.9, n))) for _ in range(64)]
    for opts in ({"policy": cub.POLICY_BREADTH}, {"phase1_cap": 8192},
                 {"policy": cub.POLICY_BREADTH, "max_slots": 1 << 18}):
        ctx.reset_stats()
        r1 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12, cub.options(**opts))
        loops = ctx.stats()["device_loops"]
        r2 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12,
                                 cub.options(device_loop=False, **opts))
        assert loops > 0, opts
        for k, (x, y) in enumerate(zip(r1, r2)):
            _same_bits(x, y, (opts, k))
    f = cub.Integrand("corner_peak", 8, 0.5, 0.0)
    ctx.reset_stats()
    r1 = ctx.integrate(f, 1e-7, 1e-12, cub.options(persistent_max_n=64))
    assert ctx.stats()["device_loops"] > 0
    r2 = ctx.integrate(f, 1e-7, 1e-12, cub.options(persistent_max_n=64, device_loop=False))
    _same_bits(r1, r2, "corner peak")
    # a table integrand (its source carries device table pointers)
    from cubature import tables as T

    tab = T.Table7(T.table7_data(0), 0)
    offs = T.table7_offsets(3)
    ctx.reset_stats()
    t1 = ctx.integrate_table7_batch(tab, offs, 1e-4, 1e-12, cub.options(policy=cub.POLICY_BREADTH))
    assert ctx.stats()["device_loops"] > 0
    t2 = ctx.integrate_table7_batch(tab, offs, 1e-4, 1e-12,
                                    cub.options(policy=cub.POLICY_BREADTH, device_loop=False))
    for k, (x, y) in enumerate(zip(t1, t2)):
        _same_bits(x, y, ("table7", k))


def test_device_loop_config3_batch_bit_identical(cub, ctx):
    """The whole 4096-integral batch of the configuration-3 generator (6-D
    product peaks, seed = index, epsrel 1e-5, breadth policy): its
    long-list stretches run as device-driven loops and give the host
    loop's results bit for bit, integral by integral."""
    n, count = 6, 4096
    params = []
    for k in range(count):
        rng = np.random.default_rng(k)
        a = np.exp(rng.uniform(np.log(1.0), np.log(50.0), n))
        u = rng.uniform(0.1, 0.9, n)
        params.append(cub.make_params(n, list(a), list(u)))
    ctx.reset_stats()
    r1 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12,
                             cub.options(policy=cub.POLICY_BREADTH))
    assert ctx.stats()["device_loops"] > 0
    r2 = ctx.integrate_batch("product_peak", n, params, 1e-5, 1e-12,
                             cub.options(policy=cub.POLICY_BREADTH, device_loop=False))
    for k, (x, y) in enumerate(zip(r1, r2)):
        _same_bits(x, y, ("config 3", k))
