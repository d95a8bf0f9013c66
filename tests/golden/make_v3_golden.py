"""Pins the V3 dump format in the repository: sha256 of the arena dumps that oracle/v3dump.py (the Python restatement
of the reference's crates/rocketsim-cuda/src/dump.rs) writes for a fixed set of synthetic states — start states, after
decisions, and in the middle of a tick with contact records — and of the static dump of a fixed StaticData padded to
the importer's sizes.  tests/test_v3dump.py regenerates them with both implementations and compares.

  python tests/golden/make_v3_golden.py     # writes tests/golden/v3dump.json
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rocketsim-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    import rsx
    import v3dump as O
    from test_v3dump import _full_static, golden_states

    out = {"arena": [], "static": None}
    for label, s, sd in golden_states(rsx):
        t = O.empty_template()
        t.update({"config_hash": 0x1234, "ball_other_set": True})
        b = O.write_arena(s, sd, t)
        out["arena"].append({"case": label, "bytes": len(b), "sha256": hashlib.sha256(b).hexdigest()})
    sb, cfg = O.write_static(_full_static(rsx))
    out["static"] = {"bytes": len(sb), "sha256": hashlib.sha256(sb).hexdigest(), "config_hash": f"{cfg:016x}"}
    with open(os.path.join(HERE, "v3dump.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out)[:400])


if __name__ == "__main__":
    main()
