"""Shared helpers for the tests: seeded inputs and conversions."""
import numpy as np


def random_q(rng, bits):
    """Odd q with exactly `bits` bits."""
    q = int(rng.integers(0, 2**63)) | 1
    for _ in range((bits + 62) // 63):
        q = (q << 63) | int(rng.integers(0, 2**63))
    q &= (1 << bits) - 1
    return q | (1 << (bits - 1)) | 1


def uniform_below(rng, q, n, limbs=None):
    """n values uniform in [0, q) as (n, limbs) uint64 (rejection sampling of bits(q)-bit draws)."""
    bits = q.bit_length()
    limbs = limbs or (bits + 63) // 64
    out = np.zeros((n, limbs), dtype=np.uint64)
    filled = 0
    top_bits = bits - 64 * ((bits - 1) // 64)
    q_top_limbs = np.frombuffer(q.to_bytes(8 * limbs, "little"), dtype=np.uint64)
    while filled < n:
        k = max(16, 2 * (n - filled))
        cand = rng.integers(0, 2**64, size=(k, limbs), dtype=np.uint64, endpoint=False)
        cand[:, (bits - 1) // 64 + 1:] = 0
        cand[:, (bits - 1) // 64] &= np.uint64((1 << top_bits) - 1)
        # keep candidates below q: compare limb-wise from the top
        less = np.zeros(k, dtype=bool)
        equal = np.ones(k, dtype=bool)
        for j in range(limbs - 1, -1, -1):
            less |= equal & (cand[:, j] < q_top_limbs[j])
            equal &= cand[:, j] == q_top_limbs[j]
        keep = cand[less][: n - filled]
        out[filled: filled + len(keep)] = keep
        filled += len(keep)
    return out


def to_ints(x):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    raw = x.tobytes()
    w = 8 * x.shape[1]
    return [int.from_bytes(raw[i * w:(i + 1) * w], "little") for i in range(x.shape[0])]


def from_ints(vals, limbs):
    return np.frombuffer(b"".join(int(v).to_bytes(8 * limbs, "little") for v in vals),
                         dtype=np.uint64).reshape(len(vals), limbs).copy()
