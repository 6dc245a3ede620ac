"""CPU emulation of the persistent Lanczos kernel's schedule and addressing
(csrc/lanczos_persistent.cu).

* The item order visits every (phase, iteration, vector, tile) once, and each
  item's dependencies (all tiles of the phase before it for the same vector)
  come earlier in the order -- so a producer that waits for them only ever
  waits on items already taken by running CTAs, and every wait ends.
* Shared-memory stages fit, every bulk / tensor copy lands inside its stage,
  starts 16-byte aligned (128 for tensor copies) and reads inside the vector;
  tensor-copy coordinates stay inside the tensor map's dimensions; the
  combine and partial-sum indices stay inside their buffers.
"""

import pytest

ORREC = 24  # sizeof(ORec<float2>)
SMEM_LIMIT = 227 * 1024


def align128(b):
    return (b + 127) & ~127


def ntab(n1, nh):
    return 4 + n1 * (4 * 3 + 4 * 9) + nh * (4 * 2 + 4 * 4)


class PShape:
    """Mirror of PShape<N1L, NHL, N1R, NHR> (complex64)."""

    def __init__(self, n1l, nhl, n1r, nhr):
        self.HL = 3 ** n1l * 2 ** nhl
        self.HR = 3 ** n1r * 2 ** nhr
        self.TR = 16
        self.RS = 2 * self.HR + 2
        self.RT = (2 * self.HL + self.TR - 1) // self.TR
        self.LT = self.HR // 8
        self.PT = self.RT + self.LT
        self.LSPLIT = (self.HL + 255) // 256
        self.BL = self.HL // self.LSPLIT
        assert self.HL % self.LSPLIT == 0 and self.HR % 8 == 0
        self.NTAB_R, self.NTAB_L = ntab(n1r, nhr), ntab(n1l, nhl)
        self.TAB_BYTES = align128(max(self.NTAB_R, self.NTAB_L) * 8)
        self.OREC_R = (self.HR // 4 * ORREC + 15) // 16 * 16
        self.OREC_L = (self.HL // 8 * ORREC + 15) // 16 * 16 + 128  # + the pair operator
        self.OREC_BYTES = align128(max(self.OREC_R, self.OREC_L))
        self.R_TILE = self.TR * self.RS * 8
        self.L_TILE = 2 * self.HL * 16 * 8
        self.PBUF = 2048  # one pass-R partial buffer per consumer warp, after the L tile
        self.MAX_CW = 10
        self.TILE_BYTES = align128(max(2 * self.R_TILE, self.L_TILE + self.MAX_CW * self.PBUF))
        self.STAGE = self.TAB_BYTES + self.OREC_BYTES + self.TILE_BYTES
        self.SMEM = 2 * self.STAGE + 1024
        self.Q = self.HL * self.HR
        self.N = 4 * self.Q


def decode(ps, idx, mseg, nb, gv):
    full_groups = nb // gv
    per_group = mseg * gv * ps.PT
    if idx < full_groups * per_group:
        vg, r, g = idx // per_group, idx % per_group, gv
    else:
        vg, r, g = full_groups, idx - full_groups * per_group, nb - full_groups * gv
    j = r // (g * ps.PT)
    q = r - j * g * ps.PT
    if q < g * ps.RT:
        return 0, j, vg * gv + q // ps.RT, q % ps.RT
    q -= g * ps.RT
    return 1, j, vg * gv + q // ps.LT, q % ps.LT


SHAPES = {"full_221184": (2, 5, 1, 6), "prefix_13824": (2, 3, 1, 4)}


@pytest.mark.parametrize("shape", sorted(SHAPES))
@pytest.mark.parametrize("m,nb,gv", [(40, 48, 12), (16, 7, 3), (5, 13, 12), (3, 4, 12)])
def test_schedule_covers_items_once_and_dependencies_come_first(shape, m, nb, gv):
    ps = PShape(*SHAPES[shape])
    total = m * nb * ps.PT
    seen = {}
    for idx in range(total):
        key = decode(ps, idx, m, nb, gv)
        kind, j, b, tile = key
        assert 0 <= j < m and 0 <= b < nb
        assert 0 <= tile < (ps.RT if kind == 0 else ps.LT)
        assert key not in seen
        seen[key] = idx
    assert len(seen) == total
    last, first = {}, {}
    for (kind, j, b, _), idx in seen.items():
        ph = (2 * j + kind, b)
        last[ph] = max(last.get(ph, -1), idx)
        first[ph] = min(first.get(ph, total), idx)
    for (phase, b), idx0 in first.items():
        if phase > 0:
            assert last[(phase - 1, b)] < idx0


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_stage_layout_and_copy_addresses(shape):
    ps = PShape(*SHAPES[shape])
    assert ps.SMEM + 272 <= SMEM_LIMIT
    assert ps.STAGE % 128 == 0 and (ps.TAB_BYTES + ps.OREC_BYTES) % 128 == 0
    for nt in (ps.NTAB_R, ps.NTAB_L):
        assert nt * 8 % 16 == 0 and nt * 8 <= ps.TAB_BYTES
    assert max(ps.HR // 4, ps.HL // 8) * ORREC <= ps.OREC_BYTES
    # outer-index records (pass L: + the 128-byte pair operator): one bulk copy
    # each, a multiple of 16 bytes, inside the slot
    for size in (ps.OREC_R, ps.OREC_L):
        assert size % 16 == 0 and size <= ps.OREC_BYTES
    ld = (ps.N + 63) // 64 * 64
    m = 40
    vstride = (m + 1) * ld
    assert ld * 8 % 16 == 0 and vstride * 8 % 16 == 0
    for tile in range(ps.RT):
        row0 = tile * ps.TR
        rows = min(ps.TR, 2 * ps.HL - row0)
        for rr in range(rows):
            rho = row0 + rr
            ea = 1 if rho >= ps.HL else 0
            g = 2 * ea * ps.Q + (rho - ea * ps.HL) * ps.HR
            for which in (0, 1):
                for e in (0, 1):
                    src = g + e * ps.Q
                    assert 0 <= src and src + ps.HR <= ps.N and src * 8 % 16 == 0
                    dst = (which * ps.TR * ps.RS + rr * ps.RS + e * ps.HR) * 8
                    assert dst % 16 == 0 and dst + ps.HR * 8 <= ps.TILE_BYTES
        ch = ps.HR // 2
        for u in range(rows * 2 * ch):
            rr, rem = divmod(u, 2 * ch)
            e, c = divmod(rem, ch)
            rho = row0 + rr
            ea = 1 if rho >= ps.HL else 0
            slot = rr * ps.RS + e * ps.HR + 2 * c
            gg = (2 * ea + e) * ps.Q + (rho - ea * ps.HL) * ps.HR + 2 * c
            assert slot + 2 <= ps.TR * ps.RS and gg + 2 <= ps.N
    dims = (ps.HR, 2, ps.HL, 2, 48 * (m + 1))
    strides = (ps.Q * 8, ps.HR * 8, 2 * ps.Q * 8, ld * 8)
    assert all(s % 16 == 0 and s < 2 ** 40 for s in strides)
    box = (8, 2, ps.BL, 1, 1)
    assert all(1 <= b <= 256 for b in box) and box[0] * 8 % 16 == 0
    for tile in range(ps.LT):
        for ea in (0, 1):
            for part in range(ps.LSPLIT):
                coord = (tile * 8, 0, part * ps.BL, ea, 47 * (m + 1) + m - 1)
                assert coord[0] * 8 % 16 == 0
                assert all(0 <= c and c + b <= d for c, b, d in zip(coord, box, dims))
                dst = (ea * ps.HL + part * ps.BL) * 16 * 8
                assert dst % 128 == 0 and dst + ps.BL * 16 * 8 <= ps.L_TILE <= ps.TILE_BYTES
    part_stride = 3 * ps.LT
    assert (47 * part_stride + (ps.LT - 1) * 3 + 2) < 48 * part_stride


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_pass_l_partial_staging_matches_direct_loads(shape):
    """The per-warp cp.async staging of the pass-R partial (l_tile_math with a
    buffer): every 16-byte copy reads inside the vector from a 16-byte aligned
    address and lands inside the warp's 2 KiB buffer, the copies cover the
    buffer exactly once, and every lane reads back exactly the element the
    direct loads would have read."""
    ps = PShape(*SHAPES[shape])
    no = ps.HL // 8
    for cw in (8, 9, 10):
        assert ps.L_TILE + cw * ps.PBUF <= ps.TILE_BYTES
    for tile in range(ps.LT):
        c0 = tile * 8
        for o in range(no):
            buf = {}
            for lane in range(32):
                for k in range(4):
                    cidx = lane + 32 * k
                    seg, piece = divmod(cidx, 4)
                    se, si, sh, sg = seg >> 4, (seg >> 2) & 3, (seg >> 1) & 1, seg & 1
                    src = (2 * se + sh) * ps.Q + (o * 8 + sg * 4 + si) * ps.HR + c0 + 2 * piece
                    dst = seg * 8 + 2 * piece
                    assert src % 2 == 0 and 0 <= src and src + 2 <= ps.N
                    assert 0 <= dst and dst + 2 <= ps.PBUF // 8
                    for u in range(2):
                        assert dst + u not in buf
                        buf[dst + u] = src + u
            assert len(buf) == ps.PBUF // 8
            for lane in range(32):
                j, h, lg = lane & 7, (lane >> 3) & 1, lane >> 4
                lo = o * 8 + lg * 4
                for e in (0, 1):
                    for i in range(4):
                        direct = h * ps.Q + c0 + j + 2 * e * ps.Q + (lo + i) * ps.HR
                        assert buf[((e * 4 + i) * 4 + h * 2 + lg) * 8 + j] == direct
