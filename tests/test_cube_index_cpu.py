"""Index emulation of the general cube H psi kernels (csrc/hpsi.cu) on the CPU.

Replays the address arithmetic of ``cube_pass_l<T, NI, TR>`` and
``cube_pass_r<T, NI, TL>`` for every block and thread task of a launch --
shared-memory carve-up and tile slots, partner-cube offsets, coefficient
table offsets, global loads and stores -- and checks each against the size of
the buffer it addresses.  Launch parameters (grid, dynamic shared memory) are
derived from a plan the way ``cube_plan`` / ``try_cube_l`` / ``try_cube_r``
derive them.  Covered: one-shape plans of the 96-, 864- and 221,184-dimension
synthetic systems, and a plan mixing the 96- and 864-dimension shapes (the
launch kind that a batched run once formed; ``cube_plan`` now refuses it).
"""

import math

import numpy as np
import pytest

from rpm_b200 import synthetic

C64 = 8  # bytes of a complex64 element
OUTER_REC = {8: 24 + 8, 16: 48 + 8}  # sizeof(OuterRec<T>): 2 coefs + 2 reals + 2 uints


def a16(b):
    return (b + 15) & ~15


def side_of(dims, axes):
    """CubeSide of one radical group (build_cube_side): digit dims, strides,
    table offsets and the count of trailing spin-1/2 digits."""
    gd = [dims[a] for a in axes[1:]]
    K = len(gd)
    gs = [0] * K
    stride = 1
    for k in range(K - 1, -1, -1):
        gs[k] = stride
        stride *= gd[k]
    offD, offF, offX = [], [], []
    pos = 4
    for d in gd:
        offD.append(pos)
        offF.append(pos + 2 * d)
        offX.append(pos + 4 * d)
        pos += 4 * d + 4 * d * d
    inner = 0
    while inner < K and gd[K - 1 - inner] == 2:
        inner += 1
    return dict(K=K, dim=gd, gs=gs, half=stride, ntab=pos, offD=offD, offF=offF, offX=offX, inner=inner)


def offsets(dims, axes):
    strides = [math.prod(dims[a + 1:]) for a in range(len(dims))]
    gd = [dims[a] for a in axes]
    out = np.zeros(math.prod(gd), dtype=np.int64)
    for idx in range(out.size):
        rem, o = idx, 0
        for p in range(len(axes) - 1, -1, -1):
            o += (rem % gd[p]) * strides[axes[p]]
            rem //= gd[p]
        out[idx] = o
    return out


class View:
    def __init__(self, system):
        dims = tuple(system.dimensions)
        self.n = math.prod(dims)
        self.L = side_of(dims, system.left_axes)
        self.R = side_of(dims, system.right_axes)
        self.offl = offsets(dims, system.left_axes)
        self.offr = offsets(dims, system.right_axes)
        self.nl, self.nr = len(self.offl), len(self.offr)
        self.half_l, self.half_r = self.nl // 2, self.nr // 2


def plan_of(views):
    """cube_plan's maxima (without its one-shape check)."""
    def outer(side, ni):
        return math.prod(side["dim"][:max(0, side["K"] - ni)])
    p = dict(nl=max(v.nl for v in views), nr=max(v.nr for v in views), half_r=max(v.half_r for v in views),
             tab_cap=max(max(v.L["ntab"], v.R["ntab"]) for v in views),
             ni_l=min([2] + [v.L["inner"] for v in views]), ni_r=min([2] + [v.R["inner"] for v in views]))
    for side, key in (("L", "l"), ("R", "r")):
        for ni in (1, 2):
            p[f"n_outer_{key}{ni}"] = max(outer(getattr(v, side), ni) for v in views)
    p["tab_cap"] = (p["tab_cap"] + 1) & ~1
    return p


def check_table_reads(side, ni, no):
    """InnerConst and cube_apply table offsets stay inside the table."""
    K, ntab = side["K"], side["ntab"]
    for e in (0, 1):
        for i in range(1 << ni):
            for q in range(ni):
                k = K - ni + q
                bit = (i >> (ni - 1 - q)) & 1
                assert side["offD"][k] + e * 2 + bit < ntab
                assert side["offF"][k] + e * 2 + bit < ntab
                assert side["offX"][k] + (e * 2 + bit) * 4 + 2 + (1 - bit) < ntab
    for k in range(K - ni):
        d = side["dim"][k]
        for m in range(d):
            base = side["offX"][k] + m * 2 * d
            assert base + (1 * d) * 2 * d + 1 * d + (d - 1) < ntab
    assert no == side["half"] >> ni


def outer_digits(side, ni, o):
    """Digits of outer index o (digit k slowest) and their strides in outer units."""
    nout = side["K"] - ni
    digits, rem = [0] * nout, o
    for k in range(nout - 1, -1, -1):
        digits[k] = rem % side["dim"][k]
        rem //= side["dim"][k]
    return digits, [side["gs"][k] >> ni for k in range(nout)]


def emulate_pass_l(v, p, ni, tr):
    C, W = 1 << ni, 2 * tr
    n_outer_cap = p[f"n_outer_l{ni}"]
    host_smem = (a16(p["tab_cap"] * C64) + a16(n_outer_cap * OUTER_REC[C64]) + a16(p["nl"] * 4) + a16(W * 4)
                 + p["nl"] * W * C64)
    prefix = a16(p["tab_cap"] * C64) + a16(n_outer_cap * OUTER_REC[C64]) + a16(v.nl * 4) + a16(W * 4)
    tile_elems = v.nl * W
    assert prefix + tile_elems * C64 <= host_smem
    no = v.half_l >> ni
    assert no <= n_outer_cap
    check_table_reads(v.L, ni, no)
    plane = no * W
    for bx in range((p["half_r"] + tr - 1) // tr):
        r0 = bx * tr
        offB = []
        for c in range(W):
            j = r0 + c % tr
            if j < v.half_r:
                idx = (c // tr) * v.half_r + j
                assert 0 <= idx < v.nr
                offB.append(int(v.offr[idx]))
            else:
                offB.append(-1)
        for l in range(v.nl):
            e = 1 if l >= v.half_l else 0
            rem = l - e * v.half_l
            for c in range(W):
                dst = ((e * C + (rem & (C - 1))) * no + (rem >> ni)) * W + c
                assert 0 <= dst < tile_elems
                if offB[c] >= 0:
                    assert 0 <= v.offl[l] + offB[c] < v.n
        eoff = int(v.offl[v.half_l] - v.offl[0])
        for task in range(W * no):
            c, o = task % W, task // W
            if offB[c] < 0:
                continue
            h = c // tr
            digits, ostr = outer_digits(v.L, ni, o)
            for e in (0, 1):
                for i in range(C):
                    assert 0 <= (e * C + i) * plane + task < tile_elems
                    for k, m in enumerate(digits):
                        for mp in range(v.L["dim"][k]):
                            if mp != m:
                                assert 0 <= (e * C + i) * plane + task + (mp - m) * ostr[k] * W < tile_elems
                    partner = (e * C + i) * plane + task + (-tr if h else tr)
                    assert 0 <= partner < tile_elems
                    out = int(v.offl[o << ni]) + offB[c] + e * eoff + int(v.offl[i] - v.offl[0])
                    assert 0 <= out < v.n


def emulate_pass_r(v, p, ni, tl):
    C = 1 << ni
    n_outer_cap = p[f"n_outer_r{ni}"]
    host_smem = (a16(p["tab_cap"] * C64) + a16(n_outer_cap * OUTER_REC[C64]) + a16(tl * 4) + a16(p["nr"] * 4)
                 + 2 * tl * p["nr"] * C64)
    prefix = a16(p["tab_cap"] * C64) + a16(n_outer_cap * OUTER_REC[C64]) + a16(tl * 4) + a16(v.nr * 4)
    tile_elems = tl * v.nr  # each of the two tiles
    assert prefix + 2 * tile_elems * C64 <= host_smem
    no = v.half_r >> ni
    assert no <= n_outer_cap
    check_table_reads(v.R, ni, no)
    eoff = int(v.offr[v.half_r] - v.offr[0])
    for bx in range((p["nl"] + tl - 1) // tl):
        l0 = bx * tl
        rows = min(tl, v.nl - l0)
        for lt in range(max(rows, 0)):
            rowoff = int(v.offl[l0 + lt])
            for r in range(v.nr):
                e = 1 if r >= v.half_r else 0
                rem = r - e * v.half_r
                pos = lt * v.nr + (e * C + (rem & (C - 1))) * no + (rem >> ni)
                assert 0 <= pos < tile_elems
                assert 0 <= rowoff + v.offr[r] < v.n
        for task in range(max(rows, 0) * no):
            o, lt = task % no, task // no
            digits, ostr = outer_digits(v.R, ni, o)
            base = lt * v.nr + o
            for e in (0, 1):
                for i in range(C):
                    assert 0 <= base + (e * C + i) * no < tile_elems
                    for k, m in enumerate(digits):
                        for mp in range(v.R["dim"][k]):
                            if mp != m:
                                assert 0 <= base + (e * C + i) * no + (mp - m) * ostr[k] < tile_elems
                    out = int(v.offl[l0 + lt]) + int(v.offr[o << ni]) + e * eoff + int(v.offr[i] - v.offr[0])
                    assert 0 <= out < v.n


SYSTEMS = {
    "small96": lambda: synthetic.small_system(),
    "prefix864": lambda: synthetic.prefix_system(synthetic.full_system(), 3),
}


@pytest.mark.parametrize("names", [("small96",), ("prefix864",), ("small96", "prefix864")])
@pytest.mark.parametrize("tr,tl", [(1, 1), (8, 16), (4, 2)])
def test_cube_kernel_indices_in_bounds(names, tr, tl):
    views = [View(SYSTEMS[k]()) for k in names]
    p = plan_of(views)
    assert p["ni_l"] >= 1 and p["ni_r"] >= 1
    for v in views:
        emulate_pass_l(v, p, p["ni_l"], tr)
        emulate_pass_r(v, p, p["ni_r"], tl)


def test_cube_kernel_indices_full_system_pass_r_rows():
    """The full system's plan (one shape): pass R over the first rows' blocks."""
    v = View(synthetic.full_system())
    p = plan_of([v])
    assert p["ni_l"] >= 1 and p["ni_r"] >= 1
    check_table_reads(v.L, p["ni_l"], v.half_l >> p["ni_l"])
    check_table_reads(v.R, p["ni_r"], v.half_r >> p["ni_r"])
