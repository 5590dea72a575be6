"""Closed-form values of the 7-D table integrand for the benchmark's 256
mu offsets (oracle.table7_exact on cubature.tables.table7_data(0) and
table7_offsets(256)), written to tests/golden/table7_exact.json.

    python tests/golden/make_table7_exact.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "old-gpuintegration_b200"))

import oracle as O  # noqa: E402
from cubature import tables as T  # noqa: E402


def main() -> int:
    d = T.table7_data(0)
    offs = T.table7_offsets(256)
    vals = [O.table7_exact(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"], d["grid_z"],
                           d["sigma"], float(o)) for o in offs]
    out = {"data_seed": 0, "offsets_seed": 1, "sigma": d["sigma"],
           "offsets": [float(o) for o in offs], "exact": vals}
    (Path(__file__).resolve().parent / "table7_exact.json").write_text(json.dumps(out, indent=0))
    return 0


if __name__ == "__main__":
    sys.exit(main())
