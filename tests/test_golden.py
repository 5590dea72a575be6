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


@pytest.mark.parametrize("rec", integrate_cases(), ids=lambda r: r["name"])
def test_oracle_matches_reference_integrate(oracle, rec):
    """Full two-phase runs: value within 2 epsrel, same status, region counts
    close (the reference's phase 2 keeps an approximate top-64 pool once a
    box has 128 subregions, the oracle the exact maximum)."""
    n = rec["ndim"]
    f = oracle.make_integrand(rec["family_name"], n, rec["a"], rec["u"])
    r = oracle.Rule(n).integrate_reference(f, rec["epsrel"], rec["epsabs"])
    assert abs(r["value"] - rec["integral"]) <= 2 * rec["epsrel"] * abs(rec["integral"]) + 1e-15
    if rec["errorFlag"] == 0:
        assert r["status"] == 0
    else:
        assert r["status"] > 0
    assert abs(r["nregions"] - rec["nregions"]) <= 0.05 * rec["nregions"] + 4
