"""Extract the reference's own published benchmark outputs into a fixture.

``specs/001-sph-fluid-sim/benchmark-results.md`` holds the tables that the
reference's harness printed (``backend/reference-tests/src/benchmarks.rs``):

* T086 dam break: T*, the simulated front Z*_sim and the experimental Z*_ref
  it was compared with, per snapshot;
* T087 hydrostatic: depth, the simulated band pressure P_sim and rho g depth.

They are the only outputs of the reference's simulator in its tree, so the
parity tests compare the CUDA path and the oracle with them. The values are
taken number for number from those tables (nothing is recomputed); run

    python tests/golden/make_reference_tables.py /path/to/reference

to regenerate ``tests/golden/reference_benchmarks.json``.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = "specs/001-sph-fluid-sim/benchmark-results.md"


def _block(text: str, header: str) -> list[str]:
    """The fenced results block that follows ``header``."""
    start = text.index(header)
    fence = text.index("```", start)
    end = text.index("```", fence + 3)
    return text[fence + 3:end].strip().splitlines()


def parse(text: str) -> dict:
    num = r"[-+]?\d+(?:\.\d+)?"
    dam = dict(t_star=[], z_star_sim=[], z_star_ref=[])
    for line in _block(text, "## T086"):
        m = re.match(rf"\s*({num})\s+({num})\s+({num})\s+({num})%\s+OK\s*$", line)
        if m:
            dam["t_star"].append(float(m.group(1)))
            dam["z_star_sim"].append(float(m.group(2)))
            dam["z_star_ref"].append(float(m.group(3)))
    hyd = dict(depth=[], p_sim=[], p_ana=[])
    for line in _block(text, "## T087"):
        m = re.match(rf"\s*({num})\s+(N/A|{num})\s+({num})\s+", line)
        if m:
            hyd["depth"].append(float(m.group(1)))
            hyd["p_sim"].append(None if m.group(2) == "N/A" else float(m.group(2)))
            hyd["p_ana"].append(float(m.group(3)))
    return {"source": SOURCE, "dam_break_2d": dam, "hydrostatic_hires": hyd}


def main(ref_root: str) -> None:
    text = open(os.path.join(ref_root, SOURCE)).read()
    out = parse(text)
    assert len(out["dam_break_2d"]["t_star"]) == 8, out["dam_break_2d"]
    assert len(out["hydrostatic_hires"]["depth"]) == 10, out["hydrostatic_hires"]
    with open(os.path.join(HERE, "reference_benchmarks.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
