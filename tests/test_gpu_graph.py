"""GPU: capacity mode and the CUDA-graph form of a batch step.

With the batch buffers reserved (eimp_phase_reserve), phasing computes the
condensed-reference row offsets on the device; the results must equal the
default mode's.  A whole phase + impute step captured on the context's stream
(eimp_capture_begin/_end) and replayed twice (eimp_graph_launch) must give the
eager step's phased haplotypes, imputed bits and dosages bit-exactly.  A
reservation that is too small makes the kernels skip the batch and report
EIMP_E_CAPACITY (no access past the buffers)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_step_equals_eager(ctx, smalltest):
    import torch
    from eimp_b200.bits import W
    from eimp_b200.engine import PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    panel, groups = smalltest
    tg = groups[0]
    hm, sm, cm = typed_views(panel, tg.typed)
    Phaser(ctx, hm, sm, cm)
    L, h = ctx.L, ctx.h
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    nt, M, Mref, nh = tg.gt.shape[0], len(tg.typed), panel.nsites, panel.nhaps
    wM, ldb = W(M), (Mref + 63) // 64
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64) if a.dtype == np.uint64  # noqa: E731
                                   else np.ascontiguousarray(a)).to(dev)
    d_full, d_af, d_typed, d_st = t(panel.sitemajor), t(panel.af.astype(np.float32)), t(tg.typed), t(sm)
    d_gt = t(tg.gt.astype(np.uint8))
    out = dict(mats=torch.empty((nt, wM), dtype=torch.int64, device=dev),
               pats=torch.empty((nt, wM), dtype=torch.int64, device=dev),
               dm=torch.empty((nt, M), dtype=torch.float32, device=dev),
               dp=torch.empty((nt, M), dtype=torch.float32, device=dev),
               tc=torch.empty(nt, dtype=torch.float32, device=dev),
               nc=torch.empty(nt, dtype=torch.int32, device=dev),
               ph=torch.empty((nt, 2, wM), dtype=torch.int64, device=dev),
               dos=torch.empty((2 * nt, Mref), dtype=torch.float32, device=dev),
               bits=torch.empty((2 * nt, ldb), dtype=torch.int64, device=dev))
    p = PhaseParams(K=200, beamwidth=32).c()

    def step():
        ctx.check(L.eimp_imp_set_reference_dev(h, Mref, nh, d_full.data_ptr(), d_af.data_ptr(), M,
                                               d_typed.data_ptr(), d_st.data_ptr()))
        ctx.check(L.eimp_phase_targets_dev(h, C.byref(p), nt, d_gt.data_ptr(), out["mats"].data_ptr(),
                                           out["pats"].data_ptr(), out["dm"].data_ptr(), out["dp"].data_ptr(),
                                           out["tc"].data_ptr(), out["nc"].data_ptr()))
        with torch.cuda.stream(stream):
            out["ph"][:, 0].copy_(out["mats"])
            out["ph"][:, 1].copy_(out["pats"])
        ctx.check(L.eimp_imp_prepare_dev(h, nt, out["ph"].data_ptr(), d_gt.data_ptr(), 0, 0, 0))
        ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, out["bits"].data_ptr(), ldb, out["dos"].data_ptr(), Mref))

    def snapshot():
        ctx.synchronize()
        torch.cuda.synchronize()
        return {k: v.clone() for k, v in out.items()}

    step()
    ref = snapshot()
    rows = C.c_size_t(0)
    ctx.check(L.eimp_phase_cref_pbwt(h, C.byref(p), nt, tg.gt.ctypes.data, C.byref(rows), None, None, None, None))
    # capacity mode, eager
    ctx.check(L.eimp_phase_reserve(h, C.byref(p), nt, rows.value))
    for v in out.values():
        v.zero_()
    step()
    cap = snapshot()
    for k in ref:
        assert torch.equal(ref[k], cap[k]), k
    # captured and replayed twice
    ctx.check(L.eimp_capture_begin(h))
    step()
    ctx.check(L.eimp_capture_end(h))
    for _ in range(2):
        for v in out.values():
            v.zero_()
        torch.cuda.synchronize()
        ctx.check(L.eimp_graph_launch(h))
        got = snapshot()
        for k in ref:
            assert torch.equal(ref[k], got[k]), k
    # eager calls after the capture that rely on the captured reference build
    ctx.check(L.eimp_imp_prepare_dev(h, nt, out["ph"].data_ptr(), d_gt.data_ptr(), 0, 0, 0))
    ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, out["bits"].data_ptr(), ldb, out["dos"].data_ptr(), Mref))
    assert torch.equal(snapshot()["dos"], ref["dos"])
    # too few rows reserved: the batch is skipped and reported
    ctx.check(L.eimp_phase_reserve(h, C.byref(p), nt, rows.value - 1))
    ctx.check(L.eimp_phase_targets_dev(h, C.byref(p), nt, d_gt.data_ptr(), out["mats"].data_ptr(),
                                       out["pats"].data_ptr(), out["dm"].data_ptr(), out["dp"].data_ptr(),
                                       out["tc"].data_ptr(), out["nc"].data_ptr()))
    assert L.eimp_synchronize(h) == 3   # EIMP_E_CAPACITY
    ctx.check(L.eimp_phase_reserve(h, C.byref(p), nt, 0))
    step()
    assert torch.equal(snapshot()["dos"], ref["dos"])
