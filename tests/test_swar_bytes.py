"""The byte-parallel (four bytes per 32-bit word) tests of the scan kernels, restated on the CPU.

The per-pair state passes read four state bytes per integer operation: the fine round-1 scan
(nibble equality, rkr_qsrp.cu qsrp_fine1_scan_kernel), the round-2 pass (round-1 class flags and
the codes below the exact-count cap, qsrp_round2_kernel) and the compaction's need mask
(QsrpCompactPolicy::need_bits).  Each identity relies on every byte's sum staying below 0x100 so that
no carry crosses into the next byte; these tests compare each word-wise form with the byte-by-byte
rule it replaces, exhaustively over the byte values and parameters that can occur.
"""
import numpy as np
import pytest

M32 = 0xFFFFFFFF


def compress(bits7):
    """Bit 7 of each byte -> four bits (byte i -> bit i): the multiply-and-shift of the kernels."""
    return ((bits7 * 0x00204081) & M32) >> 28


def words(rng, values, n):
    b = rng.choice(values, size=(n, 4))
    return b, (b[:, 0] | (b[:, 1] << 8) | (b[:, 2] << 16) | (b[:, 3] << 24)).astype(np.uint64)


def test_compress_maps_bit7_of_each_byte_to_one_bit():
    for m in range(16):
        x = sum(0x80 << (8 * i) for i in range(4) if m >> i & 1)
        assert compress(x) == m


@pytest.mark.parametrize("wl", list(range(-1, 16)))
def test_fine_scan_nibble_match(wl):
    rng = np.random.default_rng(wl + 5)
    bytes_, w = words(rng, np.arange(256), 4000)
    for wu in range(-1, 16):
        ml = ((wl if wl >= 0 else 16) * 0x01010101) & M32
        mu = ((wu if wu >= 0 else 16) * 0x01010101) & M32
        for k in range(0, 4000, 37):
            x = int(w[k])
            tl = (x & 0x0F0F0F0F) ^ ml
            tu = ((x >> 4) & 0x0F0F0F0F) ^ mu
            diff = (((tl + 0x7F7F7F7F) & M32) & ((tu + 0x7F7F7F7F) & M32)) & 0x80808080
            got = compress(diff ^ 0x80808080)
            want = sum(1 << e for e, v in enumerate(bytes_[k]) if (v & 15) == wl or (v >> 4) == wu)
            assert got == want


def class1_coarse(v, c_res, c_pr):
    """The byte rule the round-2 pass applies (non-mode-1 queries): 0 survives, 1 not."""
    cl, cu = v & 15, v >> 4
    if cl == 0:
        return 1  # a pair the fine pass resolved: its class is taken byte by byte
    return 1 if (cl <= c_res or cu >= c_pr) else 0


@pytest.mark.parametrize("c_res", list(range(-1, 16)))
def test_round2_class_flags(c_res):
    for c_pr in range(0, 17):
        kres = ((0x7F - c_res) * 0x01010101) & M32
        kpr = ((0x80 - c_pr) * 0x01010101) & M32
        for v0 in range(0, 256, 3):
            bs = [v0, (v0 * 7 + 1) & 255, (v0 * 13 + 5) & 255, (v0 * 31 + 11) & 255]
            x = sum(b << (8 * i) for i, b in enumerate(bs))
            lo, hi = x & 0x0F0F0F0F, (x >> 4) & 0x0F0F0F0F
            le_res = (((lo + kres) & M32) & 0x80808080) ^ 0x80808080
            ge_pr = ((hi + kpr) & M32) & 0x80808080
            zero = (((lo + 0x7F7F7F7F) & M32) & 0x80808080) ^ 0x80808080
            got = compress(le_res | ge_pr | zero)
            want = sum(1 << e for e, b in enumerate(bs) if class1_coarse(b, c_res, c_pr))
            assert got == want


@pytest.mark.parametrize("nb", [4, 12, 20, 32])
def test_round2_low_codes(nb):
    for cap in range(1, nb + 2):
        kcap = ((0x80 - cap) * 0x01010101) & M32
        for c0 in range(nb + 1):
            bs = [c0, (c0 + 3) % (nb + 1), (c0 * 5 + 1) % (nb + 1), nb - c0]
            x = sum(b << (8 * i) for i, b in enumerate(bs))
            got = compress((((x + kcap) & M32) & 0x80808080) ^ 0x80808080)
            assert got == sum(1 << e for e, b in enumerate(bs) if b < cap)


@pytest.mark.parametrize("nb", [16, 31, 32])
def test_compaction_need_mask(nb):
    codes = list(range(nb + 1)) + [0xFE, 0xFF]
    rng = np.random.default_rng(nb)
    for gmax in range(-1, nb + 1):
        gneed = (1 << (gmax + 1)) - 1
        g1 = (bin(gneed).count("1") * 0x01010101) & M32
        for state_any in (False, True):
            bytes_, w = words(rng, codes, 300)
            for k in range(300):
                x = int(w[k])
                le = ((((x | 0x80808080) - g1) & M32) & 0x80808080) ^ 0x80808080
                t = x ^ 0xFEFEFEFE
                fe = (~((((t & 0x7F7F7F7F) + 0x7F7F7F7F) & M32) | t) & M32) & 0x80808080
                got = compress(le | fe | ((x & 0x80808080) if state_any else 0))
                want = sum(1 << e for e, c in enumerate(bytes_[k])
                           if ((gneed >> c) & 1 if c <= nb else (c == 0xFE or state_any)))
                assert got == want
