"""Index arithmetic of the ACA panel rings, checked on the CPU.

The top-level ACA (dense_hodlr_b200/csrc/aca.cu, residual_pass_wring and
wring_issue / wring_issue_tile) splits a CTA's slice [lo, hi) of a block's
rows among 16 warps and streams each warp's rows in chunks of 128 through a
2- or 3-stage shared-memory ring.  A tile copy must start on a 16-byte
boundary (an even arena row for FP64) and a tensor copy must land on a
128-byte boundary of shared memory; an unaligned copy is an invalid
instruction on the device.  This file restates that arithmetic line for line
and checks, over many slice shapes and block offsets, that

  * every copy starts on an even arena row (gbase + jb),
  * the per-column copies move an even row count of at most 128 rows,
  * the rows the lanes keep (ok[e]) cover [lo, hi) exactly once,
  * every stage of every warp starts on a 128-byte (indeed 4 KB) boundary,
  * the rings of all warps fit the shared memory the launch asks for.
"""
import numpy as np
import pytest

NT, E = 512, 4          # WR_NT, WR_E
NW = NT // 32           # WR_NW
ROWS = 32 * E           # WR_ROWS
BC, SMAX = 4, 3         # WR_BC, WR_SMAX


def warp_rows(lo, hi, gbase, w):
    """[wlo, whi) of warp w and its chunk starts (residual_pass_wring)."""
    x0 = lo - ((gbase + lo) & 1)
    rw = (hi - x0 + NW - 1) // NW
    rw = (rw + 1) & ~1
    wlo = x0 + w * rw
    whi = min(hi, wlo + rw)
    return wlo, whi, list(range(wlo, whi, ROWS)) if wlo < whi else []


def slices(m, G):
    """The row slices [lo, hi) of a block of m rows among G CTAs (aca_kernel)."""
    sm = (m + G - 1) // G
    out = []
    for g in range(G):
        lo = min(m, g * sm)
        out.append((lo, min(m, lo + sm)))
    return out


def wring_bytes(stages):
    return 8 * NW * stages * BC * ROWS


def ring_stages(kcap_max):
    """aca_ring_stages: 3, 2 or 0 stages beside kcap_max row coefficients."""
    for st in range(SMAX, 1, -1):
        if wring_bytes(st) + 8 * kcap_max <= 224 * 1024:
            return st
    return 0


def check_slice(lo, hi, gbase):
    covered = np.zeros(max(hi - lo, 0), dtype=np.int64)
    for w in range(NW):
        wlo, whi, chunks = warp_rows(lo, hi, gbase, w)
        for jb in chunks:
            assert (gbase + jb) % 2 == 0, (lo, hi, gbase, w, jb)
            assert gbase + jb >= 0
            count = (min(ROWS, whi - jb) + 1) & ~1
            assert 0 < count <= ROWS and count % 2 == 0
            for lane in range(32):
                for e in range(E):
                    j = jb + lane + 32 * e
                    if lo <= j < whi:
                        # a kept row lies inside the copied rows of both forms
                        assert j - jb < count
                        covered[j - lo] += 1
    assert np.all(covered == 1), (lo, hi, gbase)


@pytest.mark.parametrize("m,G", [(65536, 74), (131072, 74), (65536, 37), (32768, 18),
                                 (20000, 36), (4097, 2), (3001, 3), (256, 2), (129, 2)])
def test_ring_partition_of_group_slices(m, G):
    rng = np.random.default_rng(m + G)
    for gbase in [0, 1, int(rng.integers(0, 1 << 20)), int(rng.integers(0, 1 << 20)) | 1]:
        for lo, hi in slices(m, G):
            if lo < hi:
                check_slice(lo, hi, gbase)


def test_ring_partition_random_slices():
    rng = np.random.default_rng(7)
    for _ in range(300):
        lo = int(rng.integers(0, 5000))
        hi = lo + int(rng.integers(1, 4000))
        gbase = int(rng.integers(0, 1 << 22))
        check_slice(lo, hi, gbase)


@pytest.mark.parametrize("stages", [2, 3])
def test_ring_stages_are_128_byte_aligned(stages):
    # the ring heads dynamic shared memory, itself 128-byte aligned
    for w in range(NW):
        for slot in range(stages):
            off = 8 * ((w * stages + slot) * BC) * ROWS
            assert off % 128 == 0
            assert off + 8 * BC * ROWS <= wring_bytes(stages)


def test_ring_stage_count_fits_shared_memory():
    for kcap in [1, 64, 470, 1024, 4096, 4117, 8000, 12000]:
        st = ring_stages(kcap)
        if st:
            assert wring_bytes(st) + 8 * kcap <= 224 * 1024
        else:
            assert wring_bytes(2) + 8 * kcap > 224 * 1024
