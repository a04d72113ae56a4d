"""Shared-memory layouts of the 256 x 256 cluster FFT (csrc/fft256_cluster.cuh),
restated here: each is injective, fits the exchange buffer, and every warp access
of every exchange (local writes / reads, cluster stores, cluster reads) touches
each of the 16 float2 bank pairs at most twice (two 128-byte wavefronts)."""
from collections import Counter

import pytest

LP, BP, AP, SM_FLOAT2 = 264, 260, 274, 17536


def lx(ln, k1, t):
    return ln * LP + 33 * (k1 >> 2) + 8 * (k1 & 3) + t


def bx(kcl, r):
    return kcl * BP + 2 * (kcl >> 2) + r


def ax(rl, kc):
    return rl * AP + kc + (kc >> 4)


def _worst(addrs):
    return max(Counter(a % 16 for a in addrs).values())


def _warps():
    for w in range(16):
        yield [32 * w + l for l in range(32)]


@pytest.mark.parametrize("fn,dims", [(lambda a, b: lx(a, b >> 3, b & 7), (64, 256)), (bx, (64, 256)), (ax, (64, 256))])
def test_layout_injective_and_in_buffer(fn, dims):
    idx = {fn(i, j) for i in range(dims[0]) for j in range(dims[1])}
    assert len(idx) == dims[0] * dims[1]
    assert min(idx) >= 0 and max(idx) < SM_FLOAT2


def test_local_exchange_conflict_free():
    for w in _warps():
        for k1 in range(32):  # stage-1 threads (line, tl) write k1
            assert _worst([lx(t >> 3, k1, t & 7) for t in w]) <= 2
        for a in range(4):  # stage-2 threads (line, g) read (4g + a, t)
            for tt in range(8):
                assert _worst([lx(t >> 3, 4 * (t & 7) + a, tt) for t in w]) <= 2


def test_cluster_exchanges_conflict_free():
    for q in range(4):
        for w in _warps():
            for kB in range(8):
                for a in range(4):  # A -> B stores into the owner of kB // 2
                    assert _worst([bx(4 * (t & 7) + a + 32 * (kB & 1), 64 * q + (t >> 3)) for t in w]) <= 2
            for e in range(32):  # B reads
                assert _worst([bx(t >> 3, (t & 7) + 8 * e) for t in w]) <= 2
            for e in range(32):  # B -> A stores
                assert _worst([ax((t & 7) + 8 * (e & 7), 64 * q + (t >> 3)) for t in w]) <= 2
            for a in range(4):  # A reads
                for kB in range(8):
                    assert _worst([ax(t >> 3, 4 * (t & 7) + a + 32 * kB) for t in w]) <= 2
