"""Regenerate tests/golden/states.json from the CPU oracle:

    python tests/golden/make_golden.py

The oracle is pinned to the reference's own unit tests; these fixtures then
pin complete trajectories of small seeded systems (counts and SHA-256 digests
of positions, velocities, forces, images, ghost origins, neighbor lists, swap
records, registered columns and the box after each case's steps), so the oracle and the CUDA path
are both checked against committed data."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import CASES, build, state_digest  # noqa: E402


def main():
    out = {}
    for name in CASES:
        s, steps = build(oracle.OracleSystem, name,
                         attach=lambda o, probe: o.set_column_probe(**probe))
        s.step(steps)
        out[name] = state_digest(s)
    with open(os.path.join(HERE, "states.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
