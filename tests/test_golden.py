"""Golden vectors from the reference engine itself.

tests/golden/ref_phase1_*.npz hold the per-region outputs of the
reference's INTEGRATE_GPU_PHASE1 (GPUQuadPhases.cu:38-79), compiled from
its own sources (oracle/ref_driver) and run on a B200 by
tests/golden/make_golden.py, on deterministic dyadic region lists.
tests/golden/ref_integrate.json (when present) holds full
GPUcuhre::integrate outputs.

CPU tests pin the oracle to these; the gpu-marked tests check the CUDA path
against them directly.  Tolerances as in test_gpu_parity.py: values within
1e-13 of the rounding scale (|avg| + L1 magnitude of the rule sum), split
axes and active flags identical except at near-ties.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
PHASE1 = sorted(GOLDEN.glob("ref_phase1_*.npz"))
INTEGRATE = GOLDEN / "ref_integrate.json"


def load(fn):
    z = np.load(fn)
    return {k: z[k] for k in z.files}


def check_against_reference(z, avg, err, axis, active, o, label):
    scale = np.abs(o["avg"]) + o["mag"]
    assert np.all(np.abs(avg - z["avg"]) <= 1e-13 * scale), label
    assert np.all(np.abs(err - z["err"]) <= 1e-12 * (scale + o["err"])), label
    clear = o["margin"] > 1e-9
    assert np.array_equal(axis[clear], z["axis"][clear]), label
    clear_r = np.abs(o["ratio"] - 1) > 1e-8
    assert np.array_equal(active[clear_r], z["active"][clear_r]), label


def test_golden_files_present():
    assert len(PHASE1) >= 5


@pytest.mark.parametrize("fn", PHASE1, ids=[p.stem for p in PHASE1])
def test_oracle_matches_reference_phase1(oracle, fn):
    z = load(fn)
    n = int(z["ndim"])
    f = oracle.make_integrand(str(z["family"]), n, z["a"], z["u"])
    o = oracle.Rule(n).phase1_eval(f, z["lo"], z["len"], float(z["epsrel"]), float(z["epsabs"]))
    check_against_reference(z, o["avg"], o["err"], o["axis"], o["active"], o, fn.stem)


def test_golden_axis_coverage(oracle):
    """The axis comparison is not vacuous: across the golden lists most
    regions have a clear split axis (symmetric integrands tie by design)."""
    clear = total = 0
    for fn in PHASE1:
        z = load(fn)
        n = int(z["ndim"])
        f = oracle.make_integrand(str(z["family"]), n, z["a"], z["u"])
        o = oracle.Rule(n).phase1_eval(f, z["lo"], z["len"], float(z["epsrel"]),
                                       float(z["epsabs"]))
        clear += int(np.sum(o["margin"] > 1e-9))
        total += len(o["margin"])
    assert clear > 0.5 * total


@pytest.mark.gpu
@pytest.mark.parametrize("fn", PHASE1, ids=[p.stem for p in PHASE1])
def test_cuda_matches_reference_phase1(cub, oracle, ctx, fn):
    import torch

    z = load(fn)
    n = int(z["ndim"])
    fam = str(z["family"])
    f = oracle.make_integrand(fam, n, z["a"], z["u"])
    o = oracle.Rule(n).phase1_eval(f, z["lo"], z["len"], float(z["epsrel"]), float(z["epsabs"]))
    g = cub.rule_eval(cub.Integrand(fam, n, list(z["a"]), list(z["u"])),
                      torch.from_numpy(np.ascontiguousarray(z["lo"])).cuda(),
                      torch.from_numpy(np.ascontiguousarray(z["len"])).cuda(),
                      float(z["epsrel"]), float(z["epsabs"]))
    avg, err, axis, active = [t.cpu().numpy() for t in g]
    check_against_reference(z, avg, err, axis, active, o, fn.stem)


def integrate_cases():
    if not INTEGRATE.exists():
        return []
    return json.loads(INTEGRATE.read_text())


def phase2_case(rec):
    """The reference's run reached its second phase (leftover boxes)."""
    if rec.get("phase2_boxes") is not None:
        return rec["phase2_boxes"] > 0
    return "phase2" in rec["name"]


@pytest.mark.parametrize("rec", [r for r in integrate_cases() if not phase2_case(r)],
                         ids=lambda r: r["name"])
def test_oracle_matches_reference_integrate(oracle, rec):
    """Runs that finish in the first phase: the oracle reproduces the
    reference's region count exactly, its status, and its value to rounding
    (including the reference's per-region epsabs test, which can report
    status 0 with an error estimate above the tolerance, case
    cornerpeak6_epsabs)."""
    n = rec["ndim"]
    f = oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"])
    r = oracle.Rule(n).integrate_reference(f, rec["epsrel"], rec["epsabs"])
    assert r["phase2_regions"] == 0
    assert r["nregions"] == rec["nregions"]
    assert r["neval"] == rec["neval"]
    assert r["status"] == rec["errorFlag"]
    assert abs(r["value"] - rec["integral"]) <= 1e-13 * abs(rec["integral"])
    # the null rules difference nearly equal sums: compare on the value scale
    assert abs(r["error"] - rec["error"]) <= 1e-13 * abs(rec["integral"]) + 1e-6 * rec["error"]


@pytest.mark.parametrize("rec", [r for r in integrate_cases()
                                 if phase2_case(r) and not r.get("estimate_miss")],
                         ids=lambda r: r["name"])
def test_reference_phase2_deviation(oracle, rec):
    """Runs that reach the second phase.  The reference keeps up to 128
    subregions of a leftover box in shared memory and, once full, spills to
    a device-malloc'ed pool and pulls back an approximate top 64
    (GPUQuadPhases.cu:184-420); on these golden cases its value moves away
    from the analytic integral by far more than its own error estimate.  The
    oracle refines the exact maximum-error subregion: same failed-box count
    and region count within 0.2%, and a value within its estimate."""
    n = rec["ndim"]
    f = oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"])
    r = oracle.Rule(n).integrate_reference(f, rec["epsrel"], rec["epsabs"])
    exact = oracle.exact(f)
    assert r["phase2_regions"] > 0
    assert r["status"] == rec["errorFlag"]
    assert abs(r["nregions"] - rec["nregions"]) <= 2e-3 * rec["nregions"]
    ours = abs(r["value"] - exact)
    theirs = abs(rec["integral"] - exact)
    assert ours <= max(r["error"], rec["epsrel"] * abs(exact))
    assert theirs > 10 * rec["error"]  # the documented deviation


@pytest.mark.parametrize("rec", [r for r in integrate_cases() if r.get("rerun")],
                         ids=lambda r: r["name"])
def test_reference_phase2_does_not_repeat(oracle, rec):
    """A second run of tests/golden/make_golden.py on the same B200 gave the
    reference's second phase different values, region counts and, on the
    failing case, a different failed-box count (58, then 61): its
    shared-memory pool spills to device-malloc'ed memory and pulls back an
    approximate top 64 from work that blocks share, so its result depends on
    timing.  The oracle (exact heap) returns the same result every time."""
    rr = rec["rerun"]
    assert (rr["integral"], rr["nregions"]) != (rec["integral"], rec["nregions"])
    n = rec["ndim"]
    f = oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"])
    R = oracle.Rule(n)
    a, b = R.integrate_reference(f, rec["epsrel"], rec["epsabs"]), \
        R.integrate_reference(f, rec["epsrel"], rec["epsabs"])
    assert a == b


@pytest.mark.parametrize("rec", [r for r in integrate_cases() if r.get("estimate_miss")],
                         ids=lambda r: r["name"])
def test_reference_engine_misses_like_the_oracle(oracle, rec):
    """Seeds of the 4096-integral product-peak generator (6-D, epsrel 1e-5)
    whose results miss the analytic value by more than epsrel with status
    0.  The reference engine misses them too (3.3e-4 and 3.8e-4 relative,
    errorFlag 0): the degree-9 rule's error estimate is optimistic on these
    sharp peaks.  On seed 206 the oracle's two-phase result equals the
    reference's to the last digit, with the same region count; on seed 1190
    the reference's approximate second phase lands further off."""
    n = rec["ndim"]
    f = oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"])
    r = oracle.Rule(n).integrate_reference(f, rec["epsrel"], rec["epsabs"])
    exact = oracle.exact(f)
    assert rec["errorFlag"] == 0 and r["status"] == 0
    assert abs(rec["integral"] - exact) > rec["epsrel"] * abs(exact)
    assert abs(r["value"] - exact) > rec["epsrel"] * abs(exact)
    assert abs(r["nregions"] - rec["nregions"]) <= 1e-3 * rec["nregions"]
    if rec["name"].endswith("seed206"):
        assert r["value"] == rec["integral"] and r["nregions"] == rec["nregions"]


@pytest.mark.gpu
@pytest.mark.parametrize("rec", integrate_cases(), ids=lambda r: r["name"])
def test_cuda_integrate_vs_reference(cub, oracle, ctx, rec):
    """The CUDA engine against the reference engine's own integrate().
    Runs that finish in the first phase give the reference's results
    exactly: the same region count, evaluation count and status, and the
    same value to rounding (the engines sum the rule in different orders;
    on every golden case no region's classification sits close enough to
    its threshold for that to flip it).  Second-phase runs agree in status
    and land within their error estimate of the analytic value (where the
    reference does not, see test_reference_phase2_deviation)."""
    n = rec["ndim"]
    r = ctx.integrate(cub.Integrand(rec["family_name"], n, rec["a"], rec["u"]), rec["epsrel"],
                      rec["epsabs"])
    exact = oracle.exact(oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"]))
    assert r.status == rec["errorFlag"]
    if not phase2_case(rec):
        assert r.nregions == rec["nregions"]
        assert r.neval == rec["neval"]
        assert abs(r.integral - rec["integral"]) <= 1e-12 * abs(rec["integral"])
        assert abs(r.error - rec["error"]) <= 1e-12 * abs(rec["integral"]) + 1e-6 * rec["error"]
    elif rec.get("estimate_miss"):
        # the rule's own miss (test_reference_engine_misses_like_the_oracle):
        # the engine lands where the oracle's two-phase run does
        o = oracle.Rule(n).integrate_reference(
            oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"]), rec["epsrel"],
            rec["epsabs"])
        assert abs(r.nregions - o["nregions"]) <= 5e-3 * o["nregions"]
        assert abs(r.integral - o["value"]) <= 2 * rec["epsrel"] * abs(o["value"])
    else:
        assert abs(r.nregions - rec["nregions"]) <= 5e-3 * rec["nregions"]
        assert abs(r.integral - exact) <= max(r.error, rec["epsrel"] * abs(exact))
