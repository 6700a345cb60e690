"""Philox4x32-10 in NumPy, as used by the reference's generated kernels (oracle; test infrastructure only).

Triton's `tl.randint4x(seed, off)` (triton/language/random.py) runs Philox-4x32 with key
(seed & 0xFFFFFFFF, seed >> 32 of the int64-extended seed) and counter (off_lo, off_hi, 0, 0); the round
function multiplies c0 by 0xD2511F53 and c2 by 0xCD9E8D57 and the key steps by (0x9E3779B9, 0xBB67AE85).
`tl.rand4x` maps each 32-bit output x (as int32) to float32(x < 0 ? -x - 1 : x) * 4.6566127342e-10f.
The per-sweep key of every kernel is (base_seed * 1000003 + sweep * 7919 + 12345) mod 2147483629
(Spin_Colour_Kernel/generator.py:205, bitwise.py:145-147).
"""

from __future__ import annotations

import numpy as np

_M32 = np.uint64(0xFFFFFFFF)
ROUND_A, ROUND_B = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
KEY_A, KEY_B = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
#: float32 of Triton's scale 4.6566127342e-10 (bit pattern 0x2FFFFFFF, just below 2^-31)
UNIFORM_SCALE = np.float32(4.6566127342e-10)


def sweep_seed(base_seed: int, sweep: int) -> int:
    """Per-sweep Philox key (int32 range) of every class launch of sweep `sweep`."""
    v = int(base_seed) * 1000003 + int(sweep) * 7919 + 12345
    r = abs(v) % 2147483629          # C remainder: the sign follows the dividend
    return r if v >= 0 else -r


def raw4(seed: int, c0, c1=0, rounds: int = 10) -> np.ndarray:
    """Four uint32 Philox outputs per counter (c0, c1, 0, 0) under key `seed`: shape (4, N)."""
    x0 = (np.asarray(c0, np.int64).reshape(-1).astype(np.uint64)) & _M32
    x1 = (np.broadcast_to(np.asarray(c1, np.int64).reshape(-1), x0.shape).astype(np.uint64)) & _M32
    x2 = np.zeros_like(x0)
    x3 = np.zeros_like(x0)
    s = int(seed)
    k0 = np.uint64(s & 0xFFFFFFFF)
    k1 = np.uint64((s >> 32) & 0xFFFFFFFF)          # int64 seed: sign bits for negative int32 keys
    for _ in range(rounds):
        pb = ROUND_B * x2
        pa = ROUND_A * x0
        x0, x1, x2, x3 = (pb >> np.uint64(32)) ^ x1 ^ k0, pb & _M32, (pa >> np.uint64(32)) ^ x3 ^ k1, pa & _M32
        k0 = (k0 + KEY_A) & _M32
        k1 = (k1 + KEY_B) & _M32
    return np.stack([x0, x1, x2, x3]).astype(np.uint32)


def to_uniform(bits: np.ndarray) -> np.ndarray:
    """uint32 -> float32 in [0, 1), Triton's uint_to_uniform_float."""
    x = np.asarray(bits, np.uint32).view(np.int32)
    x = np.where(x < 0, ~x, x)                        # -x - 1 == ~x in two's complement
    return x.astype(np.float32) * UNIFORM_SCALE


def uniform4(seed: int, counters) -> np.ndarray:
    """Triton's tl.rand4x(seed, counters) for int32 counters: (4, N) float32."""
    return to_uniform(raw4(seed, counters))


def int32_counter(v) -> np.ndarray:
    """The kernels' `.to(tl.int32)` of an int64 counter: wrap to 32 bits (two's complement)."""
    return (np.asarray(v, np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
