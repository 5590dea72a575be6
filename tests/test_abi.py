"""CPU tests of the C ABI: the library loads, exports every function
include/cubature.h declares, validates arguments before touching a device,
and its host-side rule tables are bit-identical to the oracle's."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "cubature.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cub_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_expected(cub):
    assert declared_functions() == sorted(cub.EXPORTS)


def test_library_exports_all(cub):
    lib = cub.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(cub.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (cub_\w+)", out))
    assert set(declared_functions()) <= exported


def test_version_and_defaults(cub):
    assert cub.load_library().cub_version() >= 1
    o = cub.options()
    assert o.policy == cub.POLICY_REFERENCE
    assert o.phase1_cap == 1 << 14  # FIRST_PHASE_MAXREGIONS, quad/quad.h:21
    assert o.max_iters == 100  # GPUKernelquad.cu:631
    assert o.phase2_max_regions == 2048  # MAX_GLOBALPOOL_SIZE, quad/quad.h:9


@pytest.mark.parametrize("n", [2, 3, 5, 8, 12, 16])
def test_rule_tables_match_oracle(cub, oracle, n):
    t = cub.rule_tables(n)
    o = oracle.Rule(n).tables()
    assert np.array_equal(t["wt"], o["wt"])
    assert np.array_equal(t["scale"][:, 1:4], o["scale"][:, 1:4])
    assert np.array_equal(t["norm"][:, 1:4], o["norm"][:, 1:4])
    assert np.array_equal(t["count"], o["count"])


def test_invalid_arguments_fail_cleanly(cub):
    lib = cub.load_library()
    assert lib.cub_rule_tables(1, None, None, None, None) == cub.ERR_INVALID
    assert "ndim" in cub.last_error()
    p = cub.make_params(3)
    rc = lib.cub_rule_eval(99, 3, C.byref(p), 10, None, None, 10, 1e-3, 0.0, None, None, None,
                           None, None)
    assert rc == cub.ERR_INVALID and "family" in cub.last_error()
    rc = lib.cub_rule_eval(1, 9, C.byref(p), 10, None, None, 10, 1e-3, 0.0, None, None, None,
                           None, None)
    assert rc == cub.ERR_INVALID and "ndim" in cub.last_error()
    rc = lib.cub_rule_eval(1, 3, C.byref(p), 10, None, None, 10, 1e-3, 0.0, None, None, None,
                           None, None)
    assert rc == cub.ERR_INVALID
    assert lib.cub_split(3, 10, None, None, 5, None, None, None, None, 0, 0, None, None, 0,
                         None) == cub.ERR_INVALID


def test_no_device_reports_error(cub):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(cub.CubatureError):
        cub.Context(0)


def test_graph_arguments_checked_before_the_device(cub):
    """The graph entry points reject missing arguments without a device."""
    lib = cub.load_library()
    fams = (C.c_int * 1)(cub.family_id("gaussian"))
    dims = (C.c_int * 1)(3)
    cnts = (C.c_int * 1)(1)
    h = C.c_void_p()
    assert lib.cub_graph_create(None, 1, fams, dims, cnts, None, C.byref(h)) == cub.ERR_INVALID
    assert lib.cub_graph_launch(None, None, None, None, None) == cub.ERR_INVALID
    assert lib.cub_graph_info(None, None, None) == cub.ERR_INVALID
    lib.cub_graph_destroy(None)
