"""Write a model-local swarm_runtime.cu that runs the reference's time loop with the B200 collision
path.

A GameDev model directory may ship its own swarm_runtime.cu, which the reference's build compiles
in place of src/swarm/swarm_runtime.cu (Makefile:302-309).  This script derives that file from the
reference's own swarm_runtime.cu, read where it lies, with three edits and nothing else changed:

  * after `#include <_col_chain.cuh>` it includes gd_bridge.cuh (the C ABI behind the model's own
    constants);
  * the body of the `evolve_collisions` lambda (swarm_runtime.cu:357-471: the non-finite screen,
    the geometry epoch, the search and evolve_local_collisions) becomes one call,
    gd_bridge_evolve_collisions(dev_particle, dev_rngstate, duration, total_dust_mass,
    col_geom_valid), which keeps the lambda's contract: the same screen and exit, the geometry
    rebuilt only after invalidate_col_geometry(), every owner advanced by `duration`;
  * the controller reset at output boundaries (swarm_runtime.cu:490-496) calls
    gd_bridge_reset_controller().

The written file is a build product (it holds the reference's program around the edits), so it is
written into a build directory, never into this repository.

    usage: python make_runtime.py <reference swarm_runtime.cu> <out swarm_runtime.cu>
"""

from __future__ import annotations

import sys
from pathlib import Path

LAMBDA = "auto evolve_collisions = [&](real duration)"
INCLUDE = "#include <_col_chain.cuh>"
RESET = "std::fill(local.state.begin(), local.state.end(), col_bath_state{});"
BODY = """{
        // the B200 collision path (libgd_b200, mod/gd_bridge/gd_bridge.cuh)
        gd_bridge_evolve_collisions(dev_particle, dev_rngstate, duration, total_dust_mass, col_geom_valid);
    }"""


def _matching_brace(text: str, open_at: int) -> int:
    """Index of the brace closing the one at open_at, skipping comments and literals."""
    depth, i, n = 0, open_at, len(text)
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            i = text.find("\n", i)
            if i < 0:
                break
            continue
        if text.startswith("/*", i):
            i = text.find("*/", i) + 2
            continue
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise SystemExit("unbalanced braces in the evolve_collisions lambda")


def patch(source: str) -> str:
    for anchor in (LAMBDA, INCLUDE, RESET):
        if source.count(anchor) != 1:
            raise SystemExit(f"expected exactly one occurrence of: {anchor}")
    out = source.replace(INCLUDE, INCLUDE + "\n#include <gd_bridge.cuh>  // the B200 collision path", 1)
    start = out.index(LAMBDA)
    open_at = out.index("{", start + len(LAMBDA))
    close_at = _matching_brace(out, open_at)
    out = out[:open_at] + BODY + out[close_at + 1:]
    out = out.replace(RESET, "gd_bridge_reset_controller();  // the B200 path's per-group controller memory", 1)
    return out


def main(argv):
    if len(argv) != 3:
        raise SystemExit(__doc__)
    src, dst = Path(argv[1]), Path(argv[2])
    dst.parent.mkdir(parents=True, exist_ok=True)
    dst.write_text(patch(src.read_text()))


if __name__ == "__main__":
    main(sys.argv)
