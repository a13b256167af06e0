"""Masked reference samples in the Qref decode (--excludeRefSamples): the
oracle restatement (oracle/restate.py qref_mask_row) against the reference's
own runlengthDecode with masked samples (utils.h:194-, compiled in
oracle/_ref) on run-length coded vectors -- random masks of diploid and
haploid samples, haploid samples stored as well-formed homozygous pairs and
as malformed 01/10 pairs, masks at word edges and at the last samples -- bit
for bit and in the masked-allele count; and the raw-vector rule equal to the
run-length rule wherever haploid pairs are well-formed."""
import numpy as np
import pytest

from eimp_b200.bits import W


def _vec(rng, nsamples, density, hap_flags, malformed=False):
    nw = W(2 * nsamples)
    bits = np.zeros(nw * 64, np.uint8)
    bits[:2 * nsamples] = rng.random(2 * nsamples) < density
    hs = np.flatnonzero(hap_flags)
    bits[2 * hs + 1] = bits[2 * hs]                     # haploid: homozygous pair
    if malformed and hs.size:
        bad = hs[rng.random(hs.size) < 0.3]
        bits[2 * bad] = 1
        bits[2 * bad + 1] = 0
    return np.packbits(bits, bitorder="little").view(np.uint64)


@pytest.mark.parametrize("density", [0.002, 0.05, 0.3])
@pytest.mark.parametrize("malformed", [False, True])
def test_mask_rle_vs_reference(density, malformed):
    from oracle import refcore, restate as R
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    rng = np.random.default_rng(int(density * 1000) + 7 * malformed)
    for nsamples in (1000, 4096, 4100, 20000 + 37):
        hap = rng.random(nsamples) < 0.2
        for case in range(4):
            if case == 0:
                masked = np.sort(rng.choice(nsamples, 5, replace=False))
            elif case == 1:
                masked = np.array(sorted({31, 32, 63, 64, 95} & set(range(nsamples))))   # word edges
            elif case == 2:
                masked = np.arange(nsamples - 40, nsamples)                              # the last samples
            else:
                masked = np.sort(rng.choice(nsamples, nsamples // 7, replace=False))
            w = _vec(rng, nsamples, density, hap, malformed)
            enc = refcore.rle_encode(w)
            if enc is None:
                continue
            nout = W(2 * (nsamples - masked.size))
            ref_row, ref_cnt = refcore.rle_decode_masked(enc, nout, masked, hap[masked])
            row, cnt = R.qref_mask_row(w, False, masked, hap[masked], nsamples, nout)
            np.testing.assert_array_equal(row, ref_row)
            assert cnt == ref_cnt
            # the raw-vector rule agrees where the haploid pairs are well-formed
            rrow, rcnt = R.qref_mask_row(w, True, masked, hap[masked], nsamples, nout)
            np.testing.assert_array_equal(rrow, row)
            if not malformed:
                assert rcnt == cnt


def test_mask_af_formula():
    from oracle import restate as R
    # float(an) * af - masked, over float(new an), in float arithmetic
    af = np.float32(0.3)
    got = R.qref_mask_af(af, 2 * 5000 - 10, 2 * 4990 - 9, 7)
    f = np.float32
    assert got == (f(f(9990) * af) - f(7)) / f(9971)
    assert got.dtype == np.float32
