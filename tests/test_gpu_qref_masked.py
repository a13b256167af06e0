"""GPU parity: the Qref haplotype section decoded with masked reference
samples (--excludeRefSamples, eimp_qref_decode_masked) against the oracle
restatement (oracle/restate.py qref_mask_row, pinned to the reference's own
masked runlengthDecode in tests/test_qref_mask_oracle.py): a panel with
haploid samples, raw and run-length coded variants, masks of diploid and
haploid samples at word edges and at the last samples; the kept rows bit
for bit and the corrected allele frequencies to the last bit."""
import numpy as np
import pytest

from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def _panel(rng, nsamples, nvar, hap):
    nw = W(2 * nsamples)
    rows = np.zeros((nvar, nw), np.uint64)
    for v in range(nvar):
        dens = [0.0005, 0.01, 0.2, 0.5][v % 4]
        bits = np.zeros(nw * 64, np.uint8)
        bits[:2 * nsamples] = rng.random(2 * nsamples) < dens
        hs = np.flatnonzero(hap)
        bits[2 * hs + 1] = bits[2 * hs]
        if v % 9 == 4 and hs.size:          # a few malformed haploid pairs
            bad = hs[: max(1, hs.size // 5)]
            bits[2 * bad] = 1
            bits[2 * bad + 1] = 0
        rows[v] = np.packbits(bits, bitorder="little").view(np.uint64)
    return rows


@pytest.mark.parametrize("masks", ["few", "edges", "last", "many"])
def test_qref_masked_vs_oracle(ctx, masks):
    from eimp_b200._lib import ptr
    from oracle import restate as R
    from test_qref_warp_emulated import host_index
    rng = np.random.default_rng({"few": 1, "edges": 2, "last": 3, "many": 4}[masks])
    nsamples, nvar = 2300, 300
    hap = rng.random(nsamples) < 0.25
    rows = _panel(rng, nsamples, nvar, hap)
    sec = R.qref_section(rows)
    rc, offs = host_index(sec, nvar, 2 * nsamples)
    assert rc == 0
    raw = np.array([int(sec[o:o + 8].view(np.uint64)[0]) == 0 for o in offs])
    assert raw.any() and not raw.all()
    masked = {"few": np.sort(rng.choice(nsamples, 6, replace=False)),
              "edges": np.array([0, 31, 32, 63, 64, 1023, 1024]),
              "last": np.arange(nsamples - 45, nsamples),
              "many": np.sort(rng.choice(nsamples, nsamples // 3, replace=False))}[masks].astype(np.int64)
    mh = hap[masked].astype(np.uint8)
    af = (rng.random(nvar) * 0.9 + 0.05).astype(np.float32)
    af_dev = af.copy()
    nout = nsamples - masked.size
    nwo = W(2 * nout)
    out = np.zeros((nvar, nwo), np.uint64)
    ctx.check(ctx.L.eimp_qref_decode_masked(ctx.h, ptr(sec), sec.size, nvar, nsamples, masked.size, ptr(masked),
                                            ptr(mh), int(hap.sum()), ptr(af_dev), None, 0, ptr(out)))
    an_b = 2 * nsamples - int(hap.sum())
    an_a = 2 * nout - (int(hap.sum()) - int(mh.sum()))
    for v in range(nvar):
        want, cnt = R.qref_mask_row(rows[v], bool(raw[v]), masked, mh, nsamples, nwo)
        np.testing.assert_array_equal(out[v], want)
        assert af_dev[v] == R.qref_mask_af(af[v], an_b, an_a, cnt), v
