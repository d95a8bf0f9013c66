"""Generates the golden fixtures of the decision step from the reference's own CPU simulator (the oracle,
oracle/_ref/librsref.so, built from the reference's sources by oracle/Makefile).

For each case: the synthetic world (rsx_build_static) and seeded start states (rsx_make_states) of this library,
controls from rsx.decision_controls, and the oracle's decisions.  Stored per case: sha256 of the StaticData words, of
the start states, and per decision the sha256 of (result words, then every arena's tick-boundary words).  GPU tests
compare the kernels' outputs with these when the oracle library is not present.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "rocketsim-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import rsx  # noqa: E402
from conftest import Oracle  # noqa: E402

CASES = [
    # name, world seed, presets, mix, n arenas, decisions, state seed, control seed
    ("kickoff_octane_1024x100", 7, (0, 0), rsx.MIX_KICKOFF, 1024, 100, 11, 21),
    ("mixed_octane_256x40", 7, (0, 0), rsx.MIX_HEADLINE, 256, 40, 12, 22),
    ("mixed_dominus_merc_128x30", 7, (1, 5), rsx.MIX_HEADLINE, 128, 30, 13, 23),
    ("contact_heavy_breakout_plank_128x30", 7, (3, 2), rsx.MIX_CONTACT_HEAVY, 128, 30, 14, 24),
]


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run_case(orc, name, wseed, presets, mix, n, decisions, sseed, cseed):
    sd = rsx.build_static(wseed, *presets)
    st = rsx.make_states(sd, n, sseed, mix)
    rec = {"name": name, "world_seed": wseed, "presets": list(presets), "mix": list(mix), "n": n, "decisions": decisions,
           "state_seed": sseed, "control_seed": cseed, "static_sha": sha(sd), "init_sha": sha(st), "per_decision": []}
    for d in range(decisions):
        ctl = rsx.decision_controls(cseed, d, n)
        res = orc.run(st, sd, ctl)
        st[:, rsx.TICK_WORDS:] = 0
        rec["per_decision"].append(sha(res, st[:, :rsx.TICK_WORDS]))
    return rec


def main():
    orc = Oracle()
    out = [run_case(orc, *c) for c in CASES]
    with open(os.path.join(ROOT, "tests", "golden", "decisions.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()
