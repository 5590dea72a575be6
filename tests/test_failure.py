"""Failure detection, provoked on purpose and without a GPU fault.

* Non-finite integrand values.  An integrand that overflows to +inf in part
  of the box (exp(800 x_0 + ...) beyond x_0 ~ 0.885) makes the iteration's
  value sum non-finite.  The engine and the oracle stop that integral with
  status CUB_STATUS_NONFINITE instead of summing inf/NaN into a converged
  result; other integrals of the same batch are unaffected.  (The
  reference does not detect this: a NaN error fails no region test there,
  GPUQuadPhases.cu:63-74.)
* A grid-barrier wait that runs out.  The persistent kernels' grid barrier
  is a bounded spin.  A test option keeps one block from arriving, and a
  short spin limit makes every other block's wait give up within
  milliseconds: every block returns, the call reports CUB_ERR_TIMEOUT, and
  the context stays usable (the next call on it gives the normal result).
  No wait is unbounded and nothing faults; the held block itself waits with
  the same limit.
"""
import pytest

NONFINITE = 1 << 30
OVERFLOW = ("discontinuous", 3, [800.0, 1.0, 1.0], [1.0, 1.0, 1.0])


def test_oracle_flags_nonfinite(oracle):
    fam, n, a, u = OVERFLOW
    r = oracle.Rule(n).integrate_reference(oracle.make_integrand(fam, n, a, u), 1e-6, 1e-12)
    assert r["status"] == oracle.STATUS_NONFINITE == NONFINITE
    assert r["nregions"] > 0


@pytest.mark.gpu
def test_engine_flags_nonfinite_like_the_oracle(cub, oracle, ctx):
    fam, n, a, u = OVERFLOW
    r_c = oracle.Rule(n).integrate_reference(oracle.make_integrand(fam, n, a, u), 1e-6, 1e-12)
    r_g = ctx.integrate(cub.Integrand(fam, n, a, u), 1e-6, 1e-12)
    assert r_g.status == r_c["status"] == NONFINITE
    assert r_g.nregions == r_c["nregions"] and r_g.neval == r_c["neval"]


@pytest.mark.gpu
@pytest.mark.parametrize("policy", ["reference", "breadth"])
def test_nonfinite_integral_leaves_batch_neighbours_alone(cub, oracle, ctx, policy):
    fam, n, _, u = OVERFLOW
    avals = [[2.0, 1.0, 1.0], [800.0, 1.0, 1.0], [1.5, 0.5, 2.0]]
    params = [cub.make_params(n, a, u) for a in avals]
    pol = cub.POLICY_BREADTH if policy == "breadth" else cub.POLICY_REFERENCE
    out = ctx.integrate_batch(fam, n, params, 1e-6, 1e-12, cub.options(policy=pol))
    assert out[1].status == NONFINITE
    for k in (0, 2):
        f_c = oracle.make_integrand(fam, n, avals[k], u)
        ex = oracle.exact(f_c)
        assert out[k].status == 0
        assert abs(out[k].integral - ex) <= 2e-6 * abs(ex)


@pytest.mark.gpu
@pytest.mark.parametrize("replicated", [True, False], ids=["replicated", "persistent"])
def test_barrier_timeout_is_reported_and_context_survives(cub, ctx, replicated):
    f = cub.Integrand("corner_peak", 8, 0.5, 0.0)
    held = cub.options(barrier_spins=20000, test_hold_block=0, replicated=replicated)
    with pytest.raises(cub.CubatureError) as e:
        ctx.integrate(f, 1e-6, 1e-12, held)
    assert e.value.code == cub.ERR_TIMEOUT
    r = ctx.integrate(f, 1e-6, 1e-12, cub.options(replicated=replicated))
    assert r.status == 0 and r.nregions == 1554
