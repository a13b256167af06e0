"""The oracle restatement of the Qref run-length coding of haplotype vectors
(utils.h:133-191 encode, utils.h:194- decode; qref_spec.md section I),
pinned against the worked example of qref_spec.md:144-172 and against the
reference's own coder compiled from its sources (oracle/_ref), byte for byte
and bit for bit, on vectors from all-zero to dense."""
import numpy as np
import pytest

from eimp_b200.bits import W

SPEC_BYTES = np.array([0x0a, 0x03, 0xaa, 0x02, 0xff, 0xff, 0x00, 0x20], np.uint8)
SPEC_RUNS = [10, 3, 298, 32767, 0, 32]   # alternating, starting with zeros


def runs_to_bits(runs, nbits):
    bits = np.zeros(nbits, np.uint8)
    pos, bit = 0, 0
    for r in runs:
        if bit:
            bits[pos:min(pos + r, nbits)] = 1
        pos += r
        bit ^= 1
    return bits


def words(bits):
    return np.packbits(bits, bitorder="little").view(np.uint64)


def test_spec_worked_example_decode():
    from oracle import restate as R
    nbits = sum(SPEC_RUNS)   # 33110
    full = nbits // 64        # 517 words: the runs run past the row, the excess is dropped
    out, rc = R.rle_decode(SPEC_BYTES, full)
    assert rc == 0
    np.testing.assert_array_equal(out, words(runs_to_bits(SPEC_RUNS, full * 64)))
    _, rc = R.rle_decode(SPEC_BYTES, full + 1)   # ends inside word 517: truncated
    assert rc == -1
    _, rc = R.rle_decode(SPEC_BYTES[:3], full)   # a two-byte run length cut after its first byte
    assert rc == -1


def test_spec_worked_example_encode():
    from oracle import restate as R
    runs = [10, 3, 298, 32799, 64 * 600 - 33110]
    bits = runs_to_bits(runs, 64 * 600)
    enc = R.rle_encode(words(bits))
    np.testing.assert_array_equal(enc[:8], SPEC_BYTES)
    out, rc = R.rle_decode(enc, 600)
    assert rc == 0
    np.testing.assert_array_equal(out, words(bits))


@pytest.mark.parametrize("density", [0.0, 1e-4, 0.003, 0.05, 0.5, 1.0])
def test_oracle_vs_reference_coder(density):
    from oracle import refcore, restate as R
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    rng = np.random.default_rng(int(density * 1e4) + 3)
    for nhaps in (2 * 1000, 2 * 5000 + 2, 2 * 20000):
        nw = W(nhaps)
        for _ in range(6):
            bits = np.zeros(nw * 64, np.uint8)
            bits[:nhaps] = rng.random(nhaps) < density
            if density and rng.random() < 0.5:   # a long run of ones across the 32767 limit
                a = int(rng.integers(0, max(1, nhaps - 40000)))
                bits[a:a + 40000] = 1
                bits[nhaps:] = 0
            w = words(bits)
            enc, renc = R.rle_encode(w), refcore.rle_encode(w)
            assert (enc is None) == (renc is None)
            if enc is None:
                continue
            np.testing.assert_array_equal(enc, renc)
            out, rc = R.rle_decode(enc, nw)
            assert rc == 0
            np.testing.assert_array_equal(out, w)
            np.testing.assert_array_equal(refcore.rle_decode(enc, nw), w)


def test_section_round_trip():
    """A Qref haplotype section of 300 variants of 3000 haplotypes (raw rows
    where the run-length code is not shorter) decodes back to the panel;
    a section cut short is reported."""
    from oracle import restate as R
    rng = np.random.default_rng(11)
    nh, M = 3000, 300
    nw = W(nh)
    af = rng.beta(0.1, 0.6, M)
    bits = np.zeros((M, nw * 64), np.uint8)
    bits[:, :nh] = rng.random((M, nh)) < af[:, None]
    rows = np.packbits(bits, axis=1, bitorder="little").view(np.uint64)
    sec = R.qref_section(rows)
    out, rc = R.qref_decode(sec, M, nw)
    assert rc == 0
    np.testing.assert_array_equal(out, rows)
    assert R.qref_decode(sec[:-5], M, nw)[1] == -2


def test_synthetic_qref_writer_matches_oracle():
    """The package's Qref writer for synthetic panels (eimp_b200.synth) gives
    the oracle's section byte for byte."""
    from eimp_b200 import synth
    from oracle import restate as R
    rng = np.random.default_rng(21)
    nh = 4000
    nw = W(nh)
    bits = np.zeros((120, nw * 64), np.uint8)
    bits[:, :nh] = rng.random((120, nh)) < rng.beta(0.08, 0.5, 120)[:, None]
    bits[7, 100:40000] = 1
    bits[8, :] = 1
    rows = np.packbits(bits, axis=1, bitorder="little").view(np.uint64)
    np.testing.assert_array_equal(synth.qref_section(rows), R.qref_section(rows))
