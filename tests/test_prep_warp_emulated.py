"""The phasing preparation kernels (eimp_b200/csrc/phase_prep.cu:
hamming_kernel, besthaps_kernel, monos_calls_kernel; Target::prepPhase,
Target.cpp:779-950) run on the CPU under the host warp emulator with the
address and undefined-behaviour sanitizers, in the library's launch order:
the Hamming counts of every (target, reference haplotype) pair, the K best
haplotypes, the monomorphic sites, the split and call sites and the cM
differences must equal the oracle restatement.  The genetic map has jumps
larger than cMmaxsplit, so homozygous sites split by distance (several in one
32-site chunk of the warp's scan); cases cover a partial last block of
targets, typed sites not a multiple of 64, panels of one and two CTA columns
and every targets-per-CTA variant (8, 4, 2, 1)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W, pack_rows

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")
CMMAX = 0.125


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("prep_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "phase_prep.cu")).read()
    a = src[src.index("__device__ __forceinline__ int block_sum_int"):src.index("cudaError_t launch_besthaps(")]
    b = src[src.index("__global__ void __launch_bounds__(256) monos_calls_kernel("):
            src.index("cudaError_t launch_monos_calls(")]
    for old, new in (("extern __shared__ uint64_t shm[];", "uint64_t *shm = reinterpret_cast<uint64_t *>(emu_smem_ptr);"),
                     ("extern __shared__ unsigned long long smo[];",
                      "unsigned long long *smo = reinterpret_cast<unsigned long long *>(emu_smem_ptr);")):
        assert (old in a) != (old in b)
        a, b = a.replace(old, new), b.replace(old, new)
    (d / "prep_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                    "namespace eimp {\n" + a + b + "}  // namespace eimp\n")
    exe = d / "prep_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "prep_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


@pytest.mark.parametrize("ntgt,M,nhaps,K,tb", [(11, 300, 700, 64, 8), (5, 1000, 200, 50, 4),
                                               (3, 64, 97, 40, 2), (3, 130, 97, 33, 1)])
def test_prep_emulated(emu_exe, tmp_path, ntgt, M, nhaps, K, tb):
    from oracle import restate as R
    rng = np.random.default_rng(M + 31 * nhaps + tb)
    dense = (rng.random((nhaps, M)) < rng.uniform(0.02, 0.5, M)[None, :]).astype(np.uint8)
    dense[:, rng.random(M) < 0.1] = 0   # some sites monomorphic in the panel
    hm = pack_rows(dense, W(M))
    gt = (dense[rng.integers(0, nhaps, ntgt)] + dense[rng.integers(0, nhaps, ntgt)]).astype(np.uint8)
    flip = rng.random(gt.shape) < 0.05
    gt[flip] = rng.integers(0, 3, int(flip.sum()))
    gt[rng.random(gt.shape) < 0.03] = 3
    inc = np.where(rng.random(M) < 0.04, rng.uniform(0.13, 0.4, M), rng.uniform(0.0, 0.004, M))
    cm = np.cumsum(inc).astype(np.float32)
    np.array([ntgt, M, nhaps, K, tb], np.int32).tofile(tmp_path / "params_i.bin")
    np.array([CMMAX], np.float32).tofile(tmp_path / "params_f.bin")
    gt.tofile(tmp_path / "gt.bin")
    hm.tofile(tmp_path / "hapmajor.bin")
    cm.tofile(tmp_path / "cm.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    rd = lambda n, dt: np.fromfile(tmp_path / n, dt)  # noqa: E731
    nerr = rd("o_nerr.bin", np.uint32).reshape(ntgt, nhaps)
    bh = rd("o_besthaps.bin", np.int32).reshape(ntgt, K)
    mo = rd("o_monos.bin", np.uint64).reshape(ntgt, W(M))
    sp = rd("o_splits.bin", np.int32).reshape(ntgt, M)
    ca = rd("o_calls.bin", np.int32).reshape(ntgt, M)
    cd = rd("o_cmdiffs.bin", np.float32).reshape(ntgt, M + 1)
    ns, nc = rd("o_nsplits.bin", np.int32), rd("o_ncalls.bin", np.int32)
    homsplits = 0
    for t in range(ntgt):
        obh, onerr = R.besthaps(gt[t], hm, K)
        np.testing.assert_array_equal(nerr[t], onerr, err_msg=f"target {t}: Hamming counts")
        np.testing.assert_array_equal(bh[t], obh, err_msg=f"target {t}: best haplotypes")
        omo = R.monos(hm, M, obh)
        np.testing.assert_array_equal(mo[t], omo, err_msg=f"target {t}: monomorphic sites")
        osp, oca, ocd = R.calllocs(gt[t], omo, cm, CMMAX)
        assert ns[t] == len(osp), f"target {t}: {ns[t]} splits, oracle {len(osp)}"
        if len(osp):
            np.testing.assert_array_equal(sp[t, :ns[t]], osp)
            assert nc[t] == len(oca)
            np.testing.assert_array_equal(ca[t, :nc[t]], oca)
            np.testing.assert_array_equal(cd[t, :ns[t] + 1], ocd)
            homsplits += int((gt[t, osp] != 1).sum())
    assert homsplits > 0   # the distance rule was exercised


@pytest.mark.parametrize("K,self0,haploid,tb", [(40, 3, True, 8), (0, -1, True, 4), (0, 3, False, 8),
                                                (33, 5, False, 2)])
def test_prep_exclusions_emulated(emu_exe, tmp_path, K, self0, haploid, tb):
    """Haplotypes a target may not select (Target.cpp:791-838): in phasing
    iterations after the first, the target's own two (its sample is self0 + t
    in the panel); with haploid reference samples, each one's placeholder
    second column.  Their Hamming counts must read 0xffffffff, the rest the
    oracle's; the selection is the K smallest (errors, index) among the
    others, in index order, or all of them when K covers them (K = 0 here:
    K is their count, as the reference clamps K to the haplotypes a target
    may select before it selects)."""
    from oracle import restate as R
    rng = np.random.default_rng([K, self0 + 1, tb])
    ntgt, M, nhaps = 9, 400, 160
    dense = (rng.random((nhaps, M)) < rng.uniform(0.02, 0.5, M)[None, :]).astype(np.uint8)
    hapl = (rng.random(nhaps // 2) < 0.25).astype(np.uint8) if haploid else np.zeros(nhaps // 2, np.uint8)
    if haploid:
        dense[1::2][hapl == 1] = dense[0::2][hapl == 1]   # a haploid sample as a homozygous pair
    hm = pack_rows(dense, W(M))
    gt = (dense[rng.integers(0, nhaps, ntgt)] + dense[rng.integers(0, nhaps, ntgt)]).astype(np.uint8)
    gt[rng.random(gt.shape) < 0.03] = 3
    cm = np.cumsum(rng.uniform(0.0, 0.01, M)).astype(np.float32)
    if K == 0:   # every selectable haplotype (the same count for every target here)
        K = nhaps - int(hapl.sum()) - (2 if self0 >= 0 else 0)
    np.array([ntgt, M, nhaps, K, tb, self0, int(haploid)], np.int32).tofile(tmp_path / "params_i.bin")
    np.array([CMMAX], np.float32).tofile(tmp_path / "params_f.bin")
    gt.tofile(tmp_path / "gt.bin")
    hm.tofile(tmp_path / "hapmajor.bin")
    cm.tofile(tmp_path / "cm.bin")
    hapl.tofile(tmp_path / "haploid.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    nerr = np.fromfile(tmp_path / "o_nerr.bin", np.uint32).reshape(ntgt, nhaps)
    bh = np.fromfile(tmp_path / "o_besthaps.bin", np.int32).reshape(ntgt, K)
    fl = np.fromfile(tmp_path / "o_flags.bin", np.uint64).reshape(ntgt, W(nhaps))
    h = np.arange(nhaps)
    for t in range(ntgt):
        excl = ((h & 1) == 1) & (hapl[h >> 1] == 1) if haploid else np.zeros(nhaps, bool)
        if self0 >= 0:
            excl |= (h >> 1) == self0 + t
        _, onerr = R.besthaps(gt[t], hm, nhaps)
        if haploid or K < nhaps - (2 if self0 >= 0 else 0):   # the counts are computed (launch_besthaps)
            np.testing.assert_array_equal(nerr[t, excl], np.uint32(0xffffffff))
            np.testing.assert_array_equal(nerr[t, ~excl], onerr[~excl], err_msg=f"target {t}: Hamming counts")
        allowed = h[~excl]
        if K >= len(allowed):
            want = allowed
        else:
            order = np.lexsort((allowed, onerr[allowed]))
            want = np.sort(allowed[order[:K]])
        np.testing.assert_array_equal(bh[t], want, err_msg=f"target {t}: best haplotypes")
        sel = np.zeros(W(nhaps) * 64, np.uint8)
        sel[want] = 1
        np.testing.assert_array_equal(fl[t], pack_rows(sel[None, :], W(nhaps))[0], err_msg=f"target {t}: flags")


@pytest.mark.parametrize("K", [64, 50, 200])
def test_prep_emulated_golden(emu_exe, tmp_path, K):
    """The reference's own preparation of the golden targets (Target::prepPhase:
    best haplotypes, monomorphic sites, split and call sites, cM differences;
    K = 200 takes every reference haplotype)."""
    g = np.load(golden_path("golden_tiny.npz"))
    pre = f"K{K}_"
    gt = np.ascontiguousarray(g["gt"], np.uint8)
    ntgt, M = gt.shape
    nhaps = int(g["nhaps"])
    np.array([ntgt, M, nhaps, K, 8], np.int32).tofile(tmp_path / "params_i.bin")
    np.array([CMMAX], np.float32).tofile(tmp_path / "params_f.bin")
    gt.tofile(tmp_path / "gt.bin")
    np.ascontiguousarray(g["hapmajor_typed"]).tofile(tmp_path / "hapmajor.bin")
    np.ascontiguousarray(g["cm_typed"], np.float32).tofile(tmp_path / "cm.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    rd = lambda n, dt: np.fromfile(tmp_path / n, dt)  # noqa: E731
    Kc = min(K, nhaps)
    np.testing.assert_array_equal(rd("o_besthaps.bin", np.int32).reshape(ntgt, K)[:, :Kc], g[pre + "besthaps"])
    np.testing.assert_array_equal(rd("o_monos.bin", np.uint64).reshape(ntgt, W(M)), g[pre + "monos"])
    ns, nc = rd("o_nsplits.bin", np.int32), rd("o_ncalls.bin", np.int32)
    np.testing.assert_array_equal(ns, g[pre + "nsplits"])
    np.testing.assert_array_equal(nc[ns > 0], g[pre + "ncalls"][ns > 0])
    sp = rd("o_splits.bin", np.int32).reshape(ntgt, M)
    ca = rd("o_calls.bin", np.int32).reshape(ntgt, M)
    cd = rd("o_cmdiffs.bin", np.float32).reshape(ntgt, M + 1)
    o_s = np.concatenate([[0], np.cumsum(g[pre + "nsplits"])])
    o_c = np.concatenate([[0], np.cumsum(g[pre + "ncalls"])])
    o_d = np.concatenate([[0], np.cumsum([s + 1 if s else 0 for s in g[pre + "nsplits"]])])
    for t in range(ntgt):
        np.testing.assert_array_equal(sp[t, :ns[t]], g[pre + "splits"][o_s[t]:o_s[t + 1]])
        if ns[t]:
            np.testing.assert_array_equal(ca[t, :nc[t]], g[pre + "calls"][o_c[t]:o_c[t + 1]])
            np.testing.assert_array_equal(cd[t, :ns[t] + 1], g[pre + "cmdiffs"][o_d[t]:o_d[t + 1]])


@pytest.mark.parametrize("K", [64, 175])
def test_prep_emulated_golden_haploid(emu_exe, tmp_path, K):
    """The reference's own best haplotypes of the diploid golden targets on a
    panel with haploid samples (their placeholder second columns are never
    chosen, Target.cpp:798-838); K = 175 is every existing haplotype (the
    reference clamps K to them, PBWTPhaser.cpp:159, 210)."""
    g = np.load(golden_path("golden_haploid.npz"))
    dip = g["tgt_haploid"] == 0
    gt = np.ascontiguousarray(g["gt"][dip], np.uint8)
    ntgt, M = gt.shape
    nhaps = int(g["nhaps"])
    hapl = np.ascontiguousarray(g["ref_haploid"], np.uint8)
    assert nhaps - int(hapl.sum()) == 175
    np.array([ntgt, M, nhaps, K, 8, -1, 1], np.int32).tofile(tmp_path / "params_i.bin")
    np.array([CMMAX], np.float32).tofile(tmp_path / "params_f.bin")
    gt.tofile(tmp_path / "gt.bin")
    np.ascontiguousarray(g["hapmajor_typed"]).tofile(tmp_path / "hapmajor.bin")
    np.ascontiguousarray(g["cm_typed"], np.float32).tofile(tmp_path / "cm.bin")
    hapl.tofile(tmp_path / "haploid.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    bh = np.fromfile(tmp_path / "o_besthaps.bin", np.int32).reshape(ntgt, K)
    np.testing.assert_array_equal(bh, g[f"K{64 if K == 64 else 200}_besthaps"])


def test_prep_emulated_bench_setting(emu_exe, tmp_path):
    """K = 4096 of the 5,000 cfg1 reference haplotypes (the threshold search
    picks most of the panel, with ties at the threshold taken in index order)
    at 2,000 typed sites: best haplotypes, monomorphic sites, split and call
    sites and cM differences against the oracle."""
    from eimp_b200 import synth
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    hm, _sm, cm = synth.typed_views(panel, tg.typed)
    gt = np.ascontiguousarray(tg.gt[:3], np.uint8)
    ntgt, M = gt.shape
    K = 4096
    np.array([ntgt, M, panel.nhaps, K, 8], np.int32).tofile(tmp_path / "params_i.bin")
    np.array([CMMAX], np.float32).tofile(tmp_path / "params_f.bin")
    gt.tofile(tmp_path / "gt.bin")
    np.ascontiguousarray(hm).tofile(tmp_path / "hapmajor.bin")
    np.ascontiguousarray(cm, np.float32).tofile(tmp_path / "cm.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    rd = lambda n, dt: np.fromfile(tmp_path / n, dt)  # noqa: E731
    nerr = rd("o_nerr.bin", np.uint32).reshape(ntgt, panel.nhaps)
    bh = rd("o_besthaps.bin", np.int32).reshape(ntgt, K)
    mo = rd("o_monos.bin", np.uint64).reshape(ntgt, W(M))
    ns, nc = rd("o_nsplits.bin", np.int32), rd("o_ncalls.bin", np.int32)
    sp = rd("o_splits.bin", np.int32).reshape(ntgt, M)
    ca = rd("o_calls.bin", np.int32).reshape(ntgt, M)
    cd = rd("o_cmdiffs.bin", np.float32).reshape(ntgt, M + 1)
    for t in range(ntgt):
        obh, onerr = R.besthaps(gt[t], hm, K)
        np.testing.assert_array_equal(nerr[t], onerr)
        np.testing.assert_array_equal(bh[t], obh)
        omo = R.monos(hm, M, obh)
        np.testing.assert_array_equal(mo[t], omo)
        osp, oca, ocd = R.calllocs(gt[t], omo, cm, CMMAX)
        assert ns[t] == len(osp) > 100
        np.testing.assert_array_equal(sp[t, :ns[t]], osp)
        np.testing.assert_array_equal(ca[t, :nc[t]], oca)
        np.testing.assert_array_equal(cd[t, :ns[t] + 1], ocd)
