"""The proposal network's tensor-core operands, checked on the CPU.

mcscram_b200/csrc/mlp.cu stores its BF16 tiles as 8 x 8 blocks of 128
contiguous bytes and hands them to tcgen05.mma through shared-memory
descriptors without swizzling.  The hardware reads such a descriptor as a
"canonical layout" of 8-row x 16-byte core matrices:

  K-major : element (mn, k) at start + (mn % 8) * 16 + (mn // 8) * SBO + (k // 8) * LBO + (k % 8) * 2
  MN-major: element (mn, k) at start + (mn // 8) * SBO + (mn % 8) * 2 + (k % 8) * 16 + (k // 8) * LBO

(k < 16 within one kind::f16 instruction).  This file restates the kernel's
tile stores and the start offsets / strides of every MMA it issues, and
checks that each (m, k) of A and (n, k) of B lands on the element the
product needs: a layout mistake would otherwise only show as a wrong
gradient on the GPU.  The constants follow mlp.cu (tile widths 32 / 80 / 192
units, weights W1 as [hidden][feature] and W2 as [out][in] blocks).
"""
import itertools

TILE = 128
UNITS_X, UNITS_E, UNITS_C = 32, 80, 192
HID, IN = 64, 16


def row_block(units):
    return units // 8 * 128


def tile_offset(row, unit, units):
    """Byte offset of (row, unit) in a tile of `units` BF16 per row (chunk<> in mlp.cu)."""
    return ((row // 8) * (units // 8) + unit // 8) * 128 + (row % 8) * 16 + (unit % 8) * 2


def tile_decode(off, units):
    block, within = divmod(off, 128)
    rb, ub = divmod(block, units // 8)
    return rb * 8 + within // 16, ub * 8 + (within % 16) // 2


def w1_offset(h, f):  # B of layer 1: N = hidden, K = feature
    return ((h // 8) * (IN // 8) + f // 8) * 128 + (h % 8) * 16 + (f % 8) * 2


def w2_offset(o, i):  # [out][in] blocks
    return ((o // 8) * (HID // 8) + i // 8) * 128 + (o % 8) * 16 + (i % 8) * 2


def decode_w(off, n_inner):
    block, within = divmod(off, 128)
    ob, ib = divmod(block, n_inner // 8)
    return ob * 8 + within // 16, ib * 8 + (within % 16) // 2


def kmajor(start, lbo, sbo, mn, k):
    return start + (mn % 8) * 16 + (mn // 8) * sbo + (k // 8) * lbo + (k % 8) * 2


def mnmajor(start, lbo, sbo, mn, k):
    return start + (mn // 8) * sbo + (mn % 8) * 2 + (k % 8) * 16 + (k // 8) * lbo


def test_tile_layout_round_trips():
    for units in (UNITS_X, UNITS_E, UNITS_C):
        seen = set()
        for r, u in itertools.product(range(TILE), range(units)):
            off = tile_offset(r, u, units)
            assert off % 2 == 0 and off < TILE * units * 2
            assert tile_decode(off, units) == (r, u)
            seen.add(off)
        assert len(seen) == TILE * units


def test_layer1_operands():
    """D1 = X W1: A = the X tile (K-major, M = rows, K = features), B = W1
    (K-major, N = hidden, K = features); one K = 16 step."""
    for m, k in itertools.product(range(TILE), range(16)):
        assert tile_decode(kmajor(0, 128, row_block(UNITS_X), m, k), UNITS_X) == (m, k)
    for n, k in itertools.product(range(HID), range(16)):
        assert kmajor(0, 128, 2 * 128, n, k) == w1_offset(n, k)


def test_layer2_operands():
    """D2 = H1 W2 in four K = 16 steps: A = the E tile's units 0..63
    (K-major), B = W2's [out][in] blocks (K-major, N = out, K = in)."""
    for step in range(HID // 16):
        for m, k in itertools.product(range(TILE), range(16)):
            assert tile_decode(kmajor(256 * step, 128, row_block(UNITS_E), m, k), UNITS_E) == (m, 16 * step + k)
        for n, k in itertools.product(range(HID), range(16)):
            assert decode_w(kmajor(256 * step, 128, 8 * 128, n, k), HID) == (n, 16 * step + k)


def test_hidden_gradient_operands():
    """dH2 W2^T into D1 in four K = 16 steps over the out units: A = the C
    tile's units 64..127 (dH2, K-major), B = the same W2 blocks read MN-major
    as N = in, K = out (B[k = out][n = in] = W2t[out][in])."""
    for step in range(HID // 16):
        for m, k in itertools.product(range(TILE), range(16)):
            off = kmajor(8 * 128 + 256 * step, 128, row_block(UNITS_C), m, k)
            assert tile_decode(off, UNITS_C) == (m, 64 + 16 * step + k)
        for n, k in itertools.product(range(HID), range(16)):
            off = mnmajor(2 * (HID // 8) * 128 * step, (HID // 8) * 128, 128, n, k)
            assert decode_w(off, HID) == (16 * step + k, n)  # (out, in)


def test_weight_gradient_operands():
    """G1 += [dH2 | H2]^T [H1 | 1 | dz] and G2 += [dH1 | dH2]^T [X | 1], K =
    rows in eight steps; both operands MN-major (units as M or N)."""
    for step in range(TILE // 16):
        for m, k in itertools.product(range(128), range(16)):
            a1 = mnmajor(8 * 128 + 2 * row_block(UNITS_C) * step, row_block(UNITS_C), 128, m, k)
            assert tile_decode(a1, UNITS_C) == (16 * step + k, 64 + m)
            a2 = mnmajor(2 * row_block(UNITS_C) * step, row_block(UNITS_C), 128, m, k)
            assert tile_decode(a2, UNITS_C) == (16 * step + k, m)
        for n, k in itertools.product(range(80), range(16)):
            b1 = mnmajor(2 * row_block(UNITS_E) * step, row_block(UNITS_E), 128, n, k)
            assert tile_decode(b1, UNITS_E) == (16 * step + k, n)
        for n, k in itertools.product(range(32), range(16)):
            b2 = mnmajor(2 * row_block(UNITS_X) * step, row_block(UNITS_X), 128, n, k)
            assert tile_decode(b2, UNITS_X) == (16 * step + k, n)


def test_instruction_descriptor_fields():
    """kind::f16 instruction descriptor as mlp.cu's idesc() builds it: FP32
    accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), majors at
    bits 15 / 16, N >> 3 at bits 17-22, M >> 4 at bits 24-28."""
    def idesc(n, a_mn, b_mn, m=128):
        return (1 << 4) | (1 << 7) | (1 << 10) | (int(a_mn) << 15) | (int(b_mn) << 16) | ((n >> 3) << 17) | \
            ((m >> 4) << 24)
    for n, a_mn, b_mn in ((64, False, False), (64, False, True), (80, True, True), (32, True, True)):
        d = idesc(n, a_mn, b_mn)
        assert (d >> 4) & 3 == 1 and (d >> 7) & 7 == 1 and (d >> 10) & 7 == 1
        assert (d >> 15) & 1 == a_mn and (d >> 16) & 1 == b_mn
        assert ((d >> 17) & 0x3F) << 3 == n and ((d >> 24) & 0x1F) << 4 == 128
        assert n % 16 == 0 and 16 <= n <= 256  # valid N for M = 128
