"""Seeded inputs of the reference-kernel harness (oracle/ref_harness/ref_harness.cu),
regenerated bit-for-bit: limb l of input `seed` is N draws of splitmix64
starting from state (seed << 20) + l, each reduced mod the limb's prime."""
import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
C1 = np.uint64(0xBF58476D1CE4E5B9)
C2 = np.uint64(0x94D049BB133111EB)


def splitmix_stream(state: int, count: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(state) + k * GAMMA
        z = (z ^ (z >> np.uint64(30))) * C1
        z = (z ^ (z >> np.uint64(27))) * C2
        return z ^ (z >> np.uint64(31))


def gen(seed: int, mods, n: int) -> np.ndarray:
    out = np.empty((len(mods), n), dtype=np.uint64)
    for l, q in enumerate(mods):
        out[l] = splitmix_stream(((seed << 20) + l) & 0xFFFFFFFFFFFFFFFF, n) % np.uint64(q)
    return out


def digest(a) -> int:
    """sum_i mix(x_i ^ (i * gamma)) mod 2^64, mix = splitmix64's finaliser (same as the harness)."""
    x = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1)
    with np.errstate(over="ignore"):
        i = np.arange(x.size, dtype=np.uint64)
        z = x ^ (i * GAMMA)
        z = (z ^ (z >> np.uint64(30))) * C1
        z = (z ^ (z >> np.uint64(27))) * C2
        z = z ^ (z >> np.uint64(31))
        return int(np.sum(z, dtype=np.uint64))
