"""The table integrands against the reference's own quad::Interp2D
(GPUQuadInterp2D.cu:50-106) and LC_LT integrand (lc_lt_t.h:18-52).

tests/golden/make_golden.py --only tables ran the reference's Interp2D
(compiled from its sources by oracle/ref_driver) on a B200 over five
LC_LT-shaped tables rounded to FP32 (the reference holds its tables in FP32
textures), at query points on every knot, inside the table and below its
first knots; and integrated the reference engine on its LC_LT integrand
over two boxes.  Fixtures: tests/golden/ref_interp2d_lclt.npz,
tests/golden/ref_lclt.json.

Tolerances.  The reference reads FP32 knots and values, forms the cell
widths' product in FP32 and returns its result as an FP32 float, so a value
can differ from an FP64 evaluation of the same tables by two FP32
roundings: |ours - ref| <= 2.5e-7 |ref| (observed: at most 1.1e-7 on every
table).  Its LC_LT integrand carries those FP32 values into FP64
arithmetic, so whole integrations agree in status and to 2 epsrel
(observed: 8e-9 and 5e-8), but not in region count: the FP32 jitter of the
reference's integrand (~1e-7 of its value) enters its null-rule error
estimates, so at epsrel 1e-5..1e-6 it refines about twice as many regions
(33524 and 41660 against the FP64 oracle's 15878 and 7470).
"""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
INTERP = GOLDEN / "ref_interp2d_lclt.npz"
LCLT = GOLDEN / "ref_lclt.json"

HOST_SRC = r"""
#include <cmath>
#include <cstdio>
#include <vector>

#include "cubature/tables.cuh"

// argv: in.bin out.bin.  in: int32 rows, cols, nq; rows xs; cols ys;
// rows*cols z (row-major); nq qx; nq qy (all doubles).  out: nq values.
int main(int argc, char** argv) {
  FILE* in = std::fopen(argv[1], "rb");
  int h[3];
  if (!in || std::fread(h, sizeof(int), 3, in) != 3) return 2;
  const int rows = h[0], cols = h[1], nq = h[2];
  std::vector<double> xs(rows), ys(cols), z((size_t)rows * cols), qx(nq), qy(nq), out(nq);
  bool ok = std::fread(xs.data(), 8, rows, in) == (size_t)rows &&
            std::fread(ys.data(), 8, cols, in) == (size_t)cols &&
            std::fread(z.data(), 8, z.size(), in) == z.size() &&
            std::fread(qx.data(), 8, nq, in) == (size_t)nq &&
            std::fread(qy.data(), 8, nq, in) == (size_t)nq;
  std::fclose(in);
  if (!ok) return 2;
  cubature::Interp2D t{xs.data(), ys.data(), z.data(), rows, cols, {}, {}};
  for (int i = 0; i < nq; ++i) out[i] = t(qx[i], qy[i]);
  FILE* o = std::fopen(argv[2], "wb");
  std::fwrite(out.data(), 8, nq, o);
  std::fclose(o);
  return 0;
}
"""


def load():
    z = np.load(INTERP)
    return {k: z[k] for k in z.files}


def host_interp(tmp_path, xs, ys, z, qx, qy):
    """The library's Interp2D (include/cubature/tables.cuh) built for the
    host with g++ and evaluated at the query points."""
    gxx, nvcc = shutil.which("g++"), shutil.which("nvcc")
    if not gxx or not nvcc:
        pytest.skip("needs g++ and the CUDA headers")
    cuda_inc = Path(nvcc).resolve().parent.parent / "include"
    src, exe = tmp_path / "interp.cpp", tmp_path / "interp"
    if not exe.exists():
        src.write_text(HOST_SRC)
        subprocess.run([gxx, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{cuda_inc}",
                        str(src), "-o", str(exe)], check=True, capture_output=True, text=True)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as fh:
        np.array([len(xs), len(ys), len(qx)], dtype=np.int32).tofile(fh)
        for a in (xs, ys, z, qx, qy):
            np.ascontiguousarray(a, dtype=np.float64).tofile(fh)
    subprocess.run([str(exe), str(fin), str(fout)], check=True)
    return np.fromfile(fout, dtype=np.float64)


def test_fixture_shapes():
    d = load()
    assert d["z"].shape == (5, len(d["xs"]), len(d["ys"])) == (5, 22, 5)
    assert d["interp"].shape == (5, len(d["qx"]))
    assert d["xs"].dtype == np.float32 and np.all(np.isfinite(d["interp"]))


def test_library_interp2d_matches_reference(tmp_path):
    d = load()
    for q in range(5):
        ours = host_interp(tmp_path, d["xs"], d["ys"], d["z"][q], d["qx"], d["qy"])
        dev = np.abs(ours - d["interp"][q])
        tol = 2.5e-7 * np.abs(d["interp"][q])
        assert np.all(dev <= tol), (q, int(np.argmax(dev - tol)), float(dev.max()))


def test_oracle_interp2d_matches_reference(oracle):
    d = load()
    for q in range(5):
        t = oracle.interp2d(d["xs"], d["ys"], d["z"][q])
        ours = np.array([oracle.interp2d_eval(t, x, y) for x, y in zip(d["qx"], d["qy"])])
        assert np.all(np.abs(ours - d["interp"][q]) <= 2.5e-7 * np.abs(d["interp"][q])), q


def lclt_cases():
    return json.loads(LCLT.read_text()) if LCLT.exists() else []


@pytest.mark.parametrize("rec", lclt_cases(), ids=lambda r: r["name"])
def test_oracle_lclt_matches_reference(oracle, rec):
    d = load()
    f = oracle.make_lclt(d["xs"], d["ys"], list(d["z"]), rec["lo"], rec["hi"])
    r = oracle.Rule(3).integrate_reference(f, rec["epsrel"], rec["epsabs"])
    assert r["status"] == rec["errorFlag"]
    assert abs(r["value"] - rec["integral"]) <= 2 * rec["epsrel"] * abs(rec["integral"])


@pytest.mark.gpu
@pytest.mark.parametrize("rec", lclt_cases(), ids=lambda r: r["name"])
def test_cuda_lclt_matches_reference(cub, ctx, rec):
    from cubature import tables as T

    d = load()
    data = {"xs": d["xs"].astype(np.float64), "ys": d["ys"].astype(np.float64),
            "z": [d["z"][q].astype(np.float64) for q in range(5)]}
    tab = T.LcLtTables(data, 0)
    r = ctx.integrate_lclt(tab, rec["lo"], rec["hi"], rec["epsrel"], rec["epsabs"])
    assert r.status == rec["errorFlag"]
    assert abs(r.integral - rec["integral"]) <= 2 * rec["epsrel"] * abs(rec["integral"])
