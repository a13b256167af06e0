"""The allocation-free best-haplotype entry point, called through the C ABI.

eimp_besthaps_noalloc serves callers that cannot let the library allocate
device memory (a framework that owns the device budget through its own pool, a
serving loop that forbids allocation after start-up): its scratch is a fixed
device array inside the library.  It must give the same best haplotypes and
flags as the regular entry point eimp_phase_prep, call after call -- the shared
array keeps the previous call's contents, so three calls in a row are checked,
the last one filling the whole array.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def _noalloc(L, stream, gt_d, hm_d, ntgt, M, nhaps, K, bh_d, fl_d):
    f = L.eimp_besthaps_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                  C.c_void_p, C.c_void_p]
    return f(stream, ntgt, M, gt_d.data_ptr(), hm_d.data_ptr(), nhaps, K, bh_d.data_ptr(), fl_d.data_ptr())


def test_besthaps_noalloc_matches_regular_entry_point():
    import torch
    from eimp_b200 import _lib, synth
    from eimp_b200.engine import Context, PhaseParams, Phaser

    L = _lib.load()
    g = np.load(golden_path("golden_tiny.npz"))
    panel, groups = synth.generate("small-test")
    cases = [(g["gt"], g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], 50)]
    hm2, sm2, cm2 = synth.typed_views(panel, groups[0].typed)
    cases.append((groups[0].gt, hm2, sm2, cm2, 200))
    # third call at the array's capacity: 8192 targets x 512 haplotypes fill
    # all EIMP_BESTHAPS_NOALLOC_MAX entries (largest offsets into the array)
    rng = np.random.default_rng(4096)
    Mx, nhx, ntx = 700, 512, 8192
    assert ntx * nhx == 4 << 20
    dense = (rng.random((nhx, Mx)) < 0.3).astype(np.uint8)
    from eimp_b200.bits import pack_rows, transpose_bits
    hm3 = pack_rows(dense, W(Mx))
    sm3 = transpose_bits(hm3, nhx, Mx)
    gt3 = (dense[rng.integers(0, nhx, ntx)] + dense[rng.integers(0, nhx, ntx)]).astype(np.uint8)
    gt3[rng.random(gt3.shape) < 0.01] = 3
    cases.append((gt3, hm3, sm3, np.linspace(0.0, 3.0, Mx, dtype=np.float32), 64))
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    # three calls in a row (different panels, targets and K): each must match
    # the regular entry point, whatever the previous call left in the array
    for gt, hm, sm, cm, K in cases:
        gt = np.ascontiguousarray(gt, dtype=np.uint8)
        ntgt, M = gt.shape
        nhaps = hm.shape[0]
        ref = Phaser(ctx, hm, sm, cm).prep(PhaseParams(K=K), gt)
        gt_d = torch.from_numpy(gt).to(dev)
        hm_d = torch.from_numpy(np.ascontiguousarray(hm).view(np.int64)).to(dev)
        bh_d = torch.full((ntgt, min(K, nhaps)), -1, dtype=torch.int32, device=dev)
        fl_d = torch.full((ntgt, W(nhaps)), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(L, None, gt_d, hm_d, ntgt, M, nhaps, K, bh_d, fl_d)
        assert rc == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(bh_d.cpu().numpy(), ref["besthaps"])
        np.testing.assert_array_equal(fl_d.cpu().numpy().view(np.uint64), ref["flags"])
    ctx.close()

