"""The hinted knot lookup of include/cubature/tables.cuh, built for the host
with g++: for ascending knots -- uniform, jittered or geometric -- and any
hint (the host's, a wrong one, none), it returns the cell of the binary
search, so the uniform-table shortcut never changes a result."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

SRC = r"""
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "cubature/tables.cuh"

using cubature::KnotHint;
using cubature::table_cell;

int main() {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  long checked = 0, bad = 0;
  for (int trial = 0; trial < 3000; ++trial) {
    const int n = 2 + (int)(U(rng) * 200);
    const int kind = trial % 3;  // uniform, jittered, geometric
    const double a = -5 + 10 * U(rng), w = 0.1 + 10 * U(rng);
    std::vector<double> xs(n);
    for (int i = 0; i < n; ++i) {
      if (kind == 0)
        xs[i] = a + i * (w / (n - 1));
      else if (kind == 1)
        xs[i] = a + (i + 0.45 * (U(rng) - 0.5)) * (w / (n - 1));
      else
        xs[i] = a + w * (std::pow(1.05, i) - 1);
    }
    KnotHint hints[3];
    hints[0].x0 = xs[0];
    hints[0].inv_dx = (n - 1) / (xs[n - 1] - xs[0]);
    hints[1].x0 = xs[0] + w * (U(rng) - 0.5);
    hints[1].inv_dx = (n - 1) / w * (0.3 + 2 * U(rng));
    for (int q = 0; q < 400; ++q) {
      double t;
      const int k = (int)(U(rng) * n);
      switch (q % 4) {
        case 0: t = xs[k]; break;
        case 1: t = a - w + 3 * w * U(rng); break;
        case 2: t = std::nextafter(xs[k], U(rng) < 0.5 ? -1e300 : 1e300); break;
        default: t = U(rng) < 0.5 ? -INFINITY : INFINITY; break;
      }
      const int want = table_cell(xs.data(), n, t);
      for (const KnotHint& h : hints) {
        ++checked;
        if (table_cell(xs.data(), n, t, h) != want) ++bad;
      }
    }
  }
  std::printf("%ld %ld\n", checked, bad);
  return bad != 0;
}
"""


def test_hinted_cell_equals_binary_search(tmp_path):
    gxx, nvcc = shutil.which("g++"), shutil.which("nvcc")
    if not gxx or not nvcc:
        pytest.skip("needs g++ and the CUDA headers")
    cuda_inc = Path(nvcc).resolve().parent.parent / "include"
    src = tmp_path / "cell.cpp"
    src.write_text(SRC)
    exe = tmp_path / "cell"
    subprocess.run([gxx, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{cuda_inc}", str(src),
                    "-o", str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    checked, bad = map(int, out.stdout.split())
    assert checked == 3000 * 400 * 3 and bad == 0
