"""Index maps of the shape-specialised passes' shared-memory staging, emulated on the CPU.

For every compiled digit pattern and both element types (complex64: two
elements per 16-byte copy, complex128: one) the pass-R unit map (rows x both
electron-B halves) and the pass-L unit map (all l x 16 columns) must cover
each staged element exactly once, inside the tile and inside the state.
The maps restate hpsi_fast.cu (PassR / PassL staging loops).
"""

import pytest

L_PATTERNS = [(2, 5), (2, 3), (2, 4), (2, 6), (1, 5), (1, 6), (0, 6), (1, 3)]
R_PATTERNS = [(1, 6), (1, 4), (1, 5), (1, 3), (1, 2), (2, 5), (0, 6), (0, 3)]


def half(n1, nh):
    return 3 ** n1 * 2 ** nh


@pytest.mark.parametrize("epu", [2, 1])
@pytest.mark.parametrize("pattern", R_PATTERNS)
def test_pass_r_staging_covers_each_row_element_once(epu, pattern):
    hr = half(*pattern)
    half_l = 48  # any left half; rows of one CTA
    tr = 16
    rs = 2 * hr + 2 if epu == 2 else 2 * hr + 1
    # an element is 16 / epu bytes: the row stride is an odd number of 16-byte units
    assert rs % epu == 0 and (rs // epu) % 2 == 1
    quarter = half_l * hr
    n = 4 * quarter
    ch = hr // epu
    for row0 in (0, 2 * half_l - tr):
        rows = min(tr, 2 * half_l - row0)
        slots, elems = set(), set()
        for idx in range(rows * 2 * ch):
            rr, rem = divmod(idx, 2 * ch)
            e, c = divmod(rem, ch)
            rho = row0 + rr
            ea = 1 if rho >= half_l else 0
            llo = rho - ea * half_l
            slot = rr * rs + e * hr + epu * c
            g = (2 * ea + e) * quarter + llo * hr + epu * c
            for k in range(epu):
                assert 0 <= slot + k < tr * rs and (slot + k) % rs < 2 * hr
                assert 0 <= g + k < n
                slots.add(slot + k)
                elems.add(g + k)
        assert len(slots) == len(elems) == rows * 2 * hr


@pytest.mark.parametrize("epu", [2, 1])
@pytest.mark.parametrize("pattern", L_PATTERNS)
def test_pass_l_staging_covers_each_column_element_once(epu, pattern):
    hl = half(*pattern)
    half_r = 64
    nl = 2 * hl
    quarter = hl * half_r
    n = 4 * quarter
    uh = 8 // epu
    for c0 in (0, half_r - 8):
        slots, elems = set(), set()
        for idx in range(nl * 2 * uh):
            l, h, q = idx // (2 * uh), (idx // uh) & 1, idx % uh
            ea = 1 if l >= hl else 0
            llo = l - ea * hl
            slot = l * 16 + h * 8 + epu * q
            g = (2 * ea + h) * quarter + llo * half_r + c0 + epu * q
            for k in range(epu):
                assert 0 <= slot + k < nl * 16
                assert 0 <= g + k < n
                slots.add(slot + k)
                elems.add(g + k)
        assert len(slots) == len(elems) == nl * 16


def test_complex128_tiles_fit_shared_memory_for_the_full_system():
    # pass L tile for the left pattern (2, 5), pass R tile for the right pattern (1, 6) at 16 bytes per element
    limit = 227 * 1024
    hl, hr = half(2, 5), half(1, 6)
    assert 2 * hl * 16 * 16 < limit
    assert 16 * (2 * hr + 1) * 16 < limit

