"""Turn one run of the reference-kernel harness into a committed fixture.

    make -C oracle ref                                  # builds oracle/_ref/ref_harness
    oracle/_ref/ref_harness 14 <dir>                    # on a B200
    python tests/golden/make_ref_fixtures.py <dir> tests/golden/ref_logn14.json [--merge]

The harness writes manifest.txt: per array its name, length, 64-bit digest
(tests/golden/refgen.py:digest) and first values, and raw copies of small
arrays (prime lists, RNG key). tests/test_golden_ref.py regenerates the
seeded inputs, runs the CPU oracle on them and compares digests.
"""
import json
import os
import sys

import numpy as np


def main(src, dst, merge=False):
    out = {"source": "kunpBFV kernels compiled for sm_100a, run on a B200 by oracle/ref_harness", "arrays": {}}
    if merge and os.path.exists(dst):  # keep the committed arrays; a repeated array must agree
        with open(dst) as f:
            out = json.load(f)
    with open(os.path.join(src, "manifest.txt")) as f:
        for line in f:
            parts = line.split()
            name, count, dig = parts[0], int(parts[1]), int(parts[2])
            if name in out["arrays"]:
                assert out["arrays"][name]["digest"] == dig, f"{name}: this run disagrees with the committed fixture"
            out["arrays"][name] = {"count": count, "digest": dig, "head": [int(x) for x in parts[3:]]}
            raw = os.path.join(src, name + ".bin")
            if os.path.exists(raw) and count <= 64:
                out[name] = [int(x) for x in np.fromfile(raw, dtype=np.uint64)]
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(out['arrays'])} arrays")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], "--merge" in sys.argv[3:])
