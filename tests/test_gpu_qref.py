"""GPU parity: the Qref haplotype section (qref_spec.md section I) decoded on
the device against the panel it was encoded from, the oracle restatement and
the reference's own runlengthDecode (oracle/_ref); a malformed section is
reported as the reference reports it and leaves the context usable."""
import numpy as np
import pytest

from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def test_qref_cfg1_panel(ctx):
    """cfg1 panel: 20000 variants of 5000 haplotypes (2500 samples), rare
    variants run-length coded, common ones raw."""
    from eimp_b200 import synth
    from eimp_b200.engine import decode_qref_haplotypes
    from oracle import refcore, restate as R
    panel, _ = synth.generate("cfg1")
    rows = panel.sitemajor
    nw = W(panel.nhaps)
    sec = R.qref_section(rows)
    from test_qref_warp_emulated import host_index
    rc, offs = host_index(sec, rows.shape[0], panel.nhaps)
    assert rc == 0
    coded = np.array([int(sec[o:o + 8].view(np.uint64)[0]) > 0 for o in offs])
    assert coded.any() and not coded.all()   # both forms present
    got = decode_qref_haplotypes(ctx, sec, rows.shape[0], panel.nhaps // 2)
    np.testing.assert_array_equal(got, rows)
    if refcore.available():
        ref, rc = refcore.qref_decode(sec, rows.shape[0], nw)
        assert rc == 0
        np.testing.assert_array_equal(got, ref)


def test_qref_into_device_rows_with_stride(ctx):
    import torch
    from eimp_b200._lib import ptr
    from oracle import restate as R
    from test_qref_warp_emulated import host_index, mixed_section
    sec, Mref, nw = mixed_section()
    rc, offs = host_index(sec, Mref, 2 * 1500)
    good = Mref - 5   # the section's last five variants are malformed
    sec = sec[:offs[good]]
    ldw = nw + 3
    d = torch.full((good * ldw,), -1, dtype=torch.int64, device="cuda:0")
    torch.cuda.synchronize()
    host = np.zeros((good, nw), np.uint64)
    ctx.check(ctx.L.eimp_qref_decode(ctx.h, ptr(sec), sec.size, good, 1500, ptr(d), ldw, ptr(host)))
    want, st = R.qref_decode(sec, good, nw)
    assert st == 0
    np.testing.assert_array_equal(host, want)
    dd = d.cpu().numpy().view(np.uint64).reshape(good, ldw)
    np.testing.assert_array_equal(dd[:, :nw], want)
    assert (dd[:, nw:] == np.uint64(0xffffffffffffffff)).all()   # the stride padding is not written


def test_qref_truncated_reported(ctx):
    from eimp_b200._lib import EimpError
    from eimp_b200.engine import decode_qref_haplotypes
    from test_qref_warp_emulated import mixed_section
    sec, Mref, nw = mixed_section()
    with pytest.raises(EimpError, match="Truncated runlength sequence"):
        decode_qref_haplotypes(ctx, sec, Mref, 1500)
    with pytest.raises(EimpError, match="Failed reading haplotypes"):
        decode_qref_haplotypes(ctx, sec[:-1], Mref, 1500)
    # the context still decodes a good section afterwards
    from oracle import restate as R
    rows = np.arange(4 * nw, dtype=np.uint64).reshape(4, nw)
    got = decode_qref_haplotypes(ctx, R.qref_section(rows), 4, 1500)
    np.testing.assert_array_equal(got, rows)
