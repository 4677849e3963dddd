#!/usr/bin/env python3
"""Generates tests/golden/golden.json from the reference pin.

The pin (oracle/_ref/libmpm_ref.so) is the reference's own WGSL compute
shaders (shaders.js), rewritten to C++ syntax by oracle/wgsl2cpp.py and run on
the host in dispatch order.  For every scenario in tests/scenarios.py this
records the SHA-256 of each state array after every substep, plus a few
summary numbers.  Run it where the reference checkout exists:

    MPM_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py

(without MPM_REFERENCE_DIR, oracle/Makefile's default location is used).

The GPU box has no reference checkout; the committed JSON carries the pin there.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "mls-mpm_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
import scenarios  # noqa: E402
from runner import cpu_run, diff_report  # noqa: E402


def main():
    O.build_oracle()
    if not O.ref_available():
        raise SystemExit("reference pin not built (needs the reference checkout)")
    out = {"source": "reference WGSL (shaders.js) via oracle/wgsl2cpp.py", "scenarios": {}}
    for name, make in scenarios.SCENARIOS.items():
        sc = make()
        steps = []
        # the pin one thread wide: its diffuse free-list pops are in particle
        # order only then (the canonical order the oracle and the GPU keep)
        for s, (ref, orc) in enumerate(zip(cpu_run(sc, "ref", threads=1), cpu_run(sc, "oracle", threads=8))):
            bad = diff_report(ref, orc)
            if bad:
                raise SystemExit(f"oracle != reference pin in {name} substep {s}: {bad}")
            rec = {"digest": O.digest(ref)}
            if ref["pos"].shape[0]:
                rec["pos_sum"] = float(np.float64(ref["pos"][:, :3]).sum())
            rec["mass_sum"] = int(ref["cell_mass"].astype(np.int64).sum())
            if "top" in ref:
                rec["alive"] = int(sc.diffuse_max - ref["top"][0])
            steps.append(rec)
        out["scenarios"][name] = {"substeps": sc.substeps, "n": sc.scene.n, "grid": list(sc.scene.grid),
                                  "diffuse_max": sc.diffuse_max, "steps": steps}
        print(f"{name}: {sc.substeps} substeps, n={sc.scene.n}", file=sys.stderr)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
