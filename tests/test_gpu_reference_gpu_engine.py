"""The reference's own GPU engine (GPUEngine.cu / GPUKernels.cu: crefTKernel and
pbwtPartedKernel, compiled unmodified for sm_100a; oracle/refgpu.py) and this
project's drop-in (eimp_gpu_run_cref_pbwt, GPUEngine's interface) on the same
inputs give the same forward and backward compressed PBWTs of the condensed
references and the same zero counts: the golden case, and a cfg2 block of
128 targets at the benchmarked K = 4,096.  The comparison covers each row's
[data, cumulative zeros] words; the reference leaves the padding words of a
row (its 4*Kwords stride) as its device allocation had them."""
import numpy as np
import pytest

from eimp_b200.bits import W, pack_genotypes

pytestmark = pytest.mark.gpu


def _inputs(pre, gt, nh, M):
    ns = pre["nsplits"]
    tgt, spl, bhf = [], [], []
    for t in range(gt.shape[0]):
        tgt.append(pack_genotypes(gt[t]))
        sw = np.zeros(W(M), np.uint64)
        s = pre["splits"][t][:ns[t]].astype(np.int64)
        np.bitwise_or.at(sw, s >> 6, np.uint64(1) << (s & 63).astype(np.uint64))
        spl.append(sw)
        bhf.append(np.ascontiguousarray(pre["flags"][t][:W(nh)]))
    off = np.concatenate([[0], np.cumsum(2 * ns.astype(np.int64) + 1)]).astype(np.uint32)
    return tgt, spl, bhf, off, ns


def _run(engine, K, M, nh, refT, tgt, spl, bhf, off, ns):
    Kwords = W(K)
    engine.initialize(K, Kwords, M, nh, nh, W(nh) * 8, refT)
    outs = [np.zeros(2 * (2 * int(n) + 1) * 4 * Kwords, np.uint32) for n in ns]
    c0s = [np.zeros(2 * int(n) + 1, np.int32) for n in ns]
    engine.runCrefPBWTKernel(tgt, spl, bhf, off, outs, c0s)
    return outs, c0s


def _compare(K, M, nh, refT, gt, pre):
    from eimp_b200.engine import GPUEngine
    from oracle.refgpu import RefGPUEngine
    args = _inputs(pre, gt, nh, M)
    ours = GPUEngine(0)
    o1, c1 = _run(ours, K, M, nh, refT, *args)
    ref = RefGPUEngine(0)
    o2, c2 = _run(ref, K, M, nh, refT, *args)
    ref.free()
    ours.free()
    kw = 2 * ((K + 31) // 32)
    for t in range(gt.shape[0]):
        a = o1[t].reshape(-1, 4 * W(K))
        b = o2[t].reshape(-1, 4 * W(K))
        np.testing.assert_array_equal(a[:, :kw], b[:, :kw])
        np.testing.assert_array_equal(c1[t], c2[t])


@pytest.fixture(scope="module")
def refgpu():
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("the reference's GPU engine is not built (oracle/Makefile target refgpu)")
    return refgpu


def test_reference_gpu_engine_golden(refgpu):
    from conftest import golden_path
    from eimp_b200.engine import Context, PhaseParams, Phaser
    g = np.load(golden_path("golden_tiny.npz"))
    nh, M = int(g["nhaps"]), int(g["M"])
    ctx = Context(0)
    pre = Phaser(ctx, g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"]).prep(PhaseParams(K=64), g["gt"])
    ctx.close()
    _compare(64, M, nh, g["sitemajor_typed"], g["gt"], pre)


def test_reference_gpu_engine_cfg2_block(refgpu):
    from eimp_b200 import synth
    from eimp_b200.engine import Context, PhaseParams, Phaser
    panel, groups = synth.generate("cfg2")
    tg = groups[0]
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    gt = tg.gt[:128]
    ctx = Context(0)
    pre = Phaser(ctx, hm, sm, cm).prep(PhaseParams(K=4096, beamwidth=128), gt)
    ctx.close()
    _compare(4096, len(tg.typed), panel.nhaps, sm, gt, pre)
