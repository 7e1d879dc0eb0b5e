"""Turn one run of the reference-kernel harness into committed fixtures.

    make -C oracle ref                                  # builds oracle/_ref/ref_harness
    oracle/_ref/ref_harness 14 <dir>                    # on a B200
    python tests/golden/make_ref_fixtures.py <dir> tests/golden/ref_logn14.json

The fixture keeps, per array the harness wrote, its length, SHA-256 and first
values, plus the context's prime lists; tests/test_golden_ref.py regenerates
the seeded inputs (refgen.py), runs the CPU oracle on them and compares hashes.
"""
import hashlib
import json
import os
import sys

import numpy as np


def main(src, dst):
    arrays = {}
    with open(os.path.join(src, "manifest.txt")) as f:
        for line in f:
            name, count = line.split()
            a = np.fromfile(os.path.join(src, name + ".bin"), dtype=np.uint64)
            assert a.size == int(count), name
            arrays[name] = a
    out = {"source": "kunpBFV kernels on B200 via oracle/ref_harness", "arrays": {}}
    for k in ("info", "qVec", "pVec", "tVec", "rVec", "pqtPsi", "qrPsi", "rng_key", "rng_nonce"):
        out[k] = [int(x) for x in arrays[k]]
    for name, a in arrays.items():
        out["arrays"][name] = {"count": int(a.size), "sha256": hashlib.sha256(a.tobytes()).hexdigest(),
                               "head": [int(x) for x in a[:8]]}
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(out['arrays'])} arrays")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
