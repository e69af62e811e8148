"""Host-side integer arithmetic the kernels rely on, checked exhaustively on
edge cases and on random operands (no GPU needed)."""
import random


def _div32(v, d):
    """The tile decoding of the partition kernels (Div32 in hg_device.cuh):
    q = mulhi64(M, v), M = floor((2^64 - 1) / d) + 1, for 32-bit v and d > 1."""
    if d == 1:
        return v
    m = (2**64 - 1) // d + 1
    return (m * v) >> 64


def test_div32_exact():
    rng = random.Random(5)
    edge_d = [1, 2, 3, 5, 7, 255, 256, 257, 4095, 4096, 4097, 65535, 65536, 65537,
              2**31 - 1, 2**31, 2**31 + 1, 2**32 - 2, 2**32 - 1]
    edge_v = [0, 1, 2, 3, 2**16 - 1, 2**16, 2**31 - 1, 2**31, 2**32 - 2, 2**32 - 1]
    for d in edge_d + [rng.randrange(1, 2**32) for _ in range(2000)]:
        for v in edge_v + [rng.randrange(0, 2**32) for _ in range(50)] + [d - 1, d, d + 1, 2 * d - 1, 2 * d]:
            if 0 <= v < 2**32:
                assert _div32(v, d) == v // d, (v, d)
