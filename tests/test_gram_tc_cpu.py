"""CPU emulation of the tensor-core singlet Gram (csrc/gram_tc.cuh).

* Operand tiles: the K-major no-swizzle layout maps every (row, column) of a
  128 x 32 TF32 tile to its own 4-byte slot inside the 16 KiB tile; the
  16-byte stores of four columns are aligned; the shared-memory and
  instruction descriptors carry the fields the layout needs.
* Tensor copies: each chunk's two 2-D copies (32 rows of every basis slot,
  one per singlet-carrying electron block) start at a 16-byte aligned x
  coordinate inside the vector's slot, for the benchmark's and the
  uneven-size workload's state dimensions, and land 128-byte aligned inside
  the raw stage; the transform zeroes every row outside the block's range.
* The mbarrier protocol of the four roles (loader, transform, MMA, epilogue)
  completes under random interleavings, with every wait on the phase parity
  the kernel computes: no role waits on a phase that never completes.
"""

import random

import pytest

GC, RAW_STAGES, TILE_STAGES = 32, 3, 2
TMEM_COLS = 512
MAX_BASIS = 64
RAW_BYTES = MAX_BASIS * 2 * GC * 8
TILE_BYTES = 128 * GC * 4
SBO, LBO = (GC // 4) * 128, 128
SMEM = RAW_STAGES * RAW_BYTES + TILE_STAGES * 2 * TILE_BYTES + 1024
COMB_LD = 65
SMEM_LIMIT = 227 * 1024


def tile_offset(r, kk):
    return (r >> 3) * SBO + (kk >> 2) * LBO + (r & 7) * 16 + (kk & 3) * 4


def smem_desc(addr):
    return ((addr & 0x3FFFF) >> 4) | ((LBO >> 4) << 16) | ((SBO >> 4) << 32) | (1 << 46)


def test_tile_layout_and_descriptors():
    seen = set()
    for r in range(128):
        for kk in range(GC):
            off = tile_offset(r, kk)
            assert 0 <= off < TILE_BYTES and off % 4 == 0 and off not in seen
            seen.add(off)
            if kk % 4 == 0:
                assert off % 16 == 0
    assert len(seen) == 128 * GC
    # K step ks of an MMA: two 16-byte core matrices along K at ks * 2 * LBO
    for ks in range(GC // 8):
        for half in range(2):
            for r in range(128):
                for j in range(4):
                    assert tile_offset(r, 8 * ks + 4 * half + j) == ks * 2 * LBO + half * LBO + tile_offset(r, j)
    d = smem_desc(0x12345 & ~15)
    assert d & 0x3FFF == (0x12345 & ~15) >> 4
    assert (d >> 16) & 0x3FFF == LBO >> 4 and (d >> 32) & 0x3FFF == SBO >> 4
    assert (d >> 46) & 0x3 == 1 and d >> 61 == 0
    idesc = (1 << 4) | (2 << 7) | (2 << 10) | ((128 >> 3) << 17) | ((128 >> 4) << 24)
    assert (idesc >> 4) & 3 == 1 and (idesc >> 7) & 7 == 2 and (idesc >> 10) & 7 == 2
    assert (idesc >> 17) & 0x3F == 16 and (idesc >> 24) & 0x1F == 8 and (idesc >> 15) & 3 == 0


def test_tensor_memory_columns():
    # buffer a of chunk c: the large term at a * 256, the small terms 128 further;
    # epilogue warps read 64 columns from column 0 (C_rr) or 64 (C_ii, C_ri)
    cols = set()
    for a in range(2):
        for part in range(2):
            for col0 in (0, 64):
                for g in range(4):
                    for i in range(16):
                        cols.add(a * 256 + part * 128 + col0 + 16 * g + i)
    assert min(cols) == 0 and max(cols) == TMEM_COLS - 1 and len(cols) == TMEM_COLS


def test_shared_memory_budget():
    assert SMEM + 256 <= SMEM_LIMIT
    assert 3 * MAX_BASIS * COMB_LD * 8 <= RAW_STAGES * RAW_BYTES + TILE_STAGES * 2 * TILE_BYTES
    for nslot in (9, 17, 33, 41, 64):
        for h in range(2):
            assert (h * nslot * GC * 8) % 128 == 0
            for k in range(nslot):
                for g in range(8):
                    off = (h * nslot + k) * GC * 8 + g * 32
                    assert off % 16 == 0 and off + 32 <= RAW_BYTES


def gblk_for(ld):
    return max(1, min(32, (ld // 4 + 63) // 64))


@pytest.mark.parametrize("dims", [(221184,), (96,), (864,), (13824,), (864, 13824, 221184), (16,), (64,)])
def test_tensor_copies_stay_in_the_vector_slot(dims):
    ld = (max(dims) + 63) // 64 * 64
    gblk = gblk_for(ld)
    for n in dims:
        assert n % 8 == 0  # the host's condition for the tensor-core kernel
        q4 = n // 4
        rows_per = ((q4 + gblk - 1) // gblk + GC - 1) // GC * GC
        covered = 0
        for blk in range(gblk):
            r_begin = blk * rows_per
            r_end = min(q4, r_begin + rows_per)
            if r_begin >= r_end:
                continue
            covered += r_end - r_begin
            nchunks = (r_end - r_begin + GC - 1) // GC
            for c in range(nchunks):
                r0 = r_begin + c * GC
                for h in range(2):
                    x = (1 + h) * q4 + r0  # element coordinate inside the vector's slot
                    assert (x * 8) % 16 == 0 and x + GC <= ld
        assert covered == q4


class Bar:
    def __init__(self, count):
        self.count, self.arrived, self.phase = count, 0, 0

    def arrive(self):
        self.arrived += 1
        if self.arrived == self.count:
            self.arrived = 0
            self.phase += 1

    def done(self, parity):
        # phase with this parity completed: the current phase's parity differs
        return (self.phase & 1) != parity


def roles(nchunks, bars, log):
    raw_full, raw_empty, tile_full, tile_empty, acc_full, acc_empty = bars

    def loader():
        for c in range(nchunks):
            rs = c % RAW_STAGES
            if c >= RAW_STAGES:
                yield raw_empty[rs], ((c - RAW_STAGES) // RAW_STAGES) & 1
            log.append(("load", c))
            raw_full[rs].arrive()  # expect_tx + the copies' bytes

    def transform(w):
        for c in range(nchunks):
            rs, ts = c % RAW_STAGES, c % TILE_STAGES
            yield raw_full[rs], (c // RAW_STAGES) & 1
            if c >= TILE_STAGES:
                yield tile_empty[ts], ((c - TILE_STAGES) // TILE_STAGES) & 1
            assert ("load", c) in log
            raw_empty[rs].arrive()
            tile_full[ts].arrive()

    def mma():
        for c in range(nchunks):
            ts, a = c % TILE_STAGES, c & 1
            if c >= 2:
                yield acc_empty[a], ((c - 2) >> 1) & 1
            yield tile_full[ts], (c // TILE_STAGES) & 1
            log.append(("mma", c))
            tile_empty[ts].arrive()
            acc_full[a].arrive()

    def epilogue(w):
        for c in range(nchunks):
            a = c & 1
            yield acc_full[a], (c >> 1) & 1
            assert ("mma", c) in log
            log.append(("drain", c, w))
            acc_empty[a].arrive()

    return [loader()] + [transform(w) for w in range(4)] + [mma()] + [epilogue(w) for w in range(6)]


@pytest.mark.parametrize("nchunks", [1, 2, 3, 4, 5, 9, 54, 57])
def test_pipeline_protocol_completes(nchunks):
    for seed in range(20):
        rng = random.Random(seed)
        bars = ([Bar(1) for _ in range(RAW_STAGES)], [Bar(4) for _ in range(RAW_STAGES)],
                [Bar(4) for _ in range(TILE_STAGES)], [Bar(1) for _ in range(TILE_STAGES)],
                [Bar(1), Bar(1)], [Bar(6), Bar(6)])
        log = []
        live = roles(nchunks, bars, log)
        waiting = {i: None for i in range(len(live))}
        steps = 0
        while live and any(g is not None for g in live):
            ready = [i for i, g in enumerate(live) if g is not None and
                     (waiting[i] is None or waiting[i][0].done(waiting[i][1]))]
            assert ready, f"deadlock with {nchunks} chunks"
            i = rng.choice(ready)
            try:
                waiting[i] = next(live[i])
            except StopIteration:
                live[i] = None
            steps += 1
            assert steps < 100000
        assert sum(1 for e in log if e[0] == "drain") == 6 * nchunks
