"""The condensed-reference kernel (eimp_b200/csrc/phase_prep.cu cref_kernel;
Target::condensedReferenceT, Target.cpp:953-1059) run on the CPU under the
host warp emulator with the address and undefined-behaviour sanitizers: every
condensed row (inconsistency rows of the segments between split sites, allele
rows of the split sites, the padding columns past K) must equal the oracle
restatement, with split sites on word edges (bits 0, 31, 32 and 63), runs of
consecutive splits, splits at the first and the last site, homozygous split
sites, a target without splits, K a multiple of 32 and not, K == nhaps (the
identity selection) and K = 4096."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W, pack_rows, transpose_bits

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("cref_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "phase_prep.cu")).read()
    i = src.index("constexpr int CREF_WARPS = 8;")
    j = src.index("cudaError_t launch_cref(")
    body = src[i:j]
    a = "extern __shared__ uint64_t sm[];"
    assert a in body
    body = body.replace(a, "uint64_t *sm = reinterpret_cast<uint64_t *>(emu_smem_ptr);")
    (d / "cref_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                    "namespace eimp {\n" + body + "}  // namespace eimp\n")
    exe = d / "cref_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "cref_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def _splits(rng, M, kind):
    if kind == "none":
        return np.zeros(0, np.int64)
    if kind == "edges":
        s = {0, M - 1}
        for w in range(0, M, 64):
            for b in (0, 31, 32, 63):
                if w + b < M and rng.random() < 0.7:
                    s.add(w + b)
        start = int(rng.integers(0, M - 12))
        s.update(range(start, start + 10))   # consecutive splits
        return np.array(sorted(s), np.int64)
    dens = {"sparse": 0.02, "dense": 0.12, "busy": 0.5}[kind]
    return np.flatnonzero(rng.random(M) < dens).astype(np.int64)


@pytest.mark.parametrize("M,nhaps,K,kinds", [(700, 200, 64, ["edges", "none", "dense"]),
                                             (257, 150, 50, ["busy", "edges"]),
                                             (130, 96, 96, ["sparse", "edges"]),
                                             (300, 5000, 4096, ["dense"])])
def test_cref_emulated(emu_exe, tmp_path, M, nhaps, K, kinds):
    from oracle import restate as R
    rng = np.random.default_rng(M * 7 + K)
    ntgt = len(kinds)
    dense = (rng.random((nhaps, M)) < rng.uniform(0.05, 0.5, M)[None, :]).astype(np.uint8)
    hm = pack_rows(dense, W(M))
    sm = transpose_bits(hm, nhaps, M)
    gt = (dense[rng.integers(0, nhaps, ntgt)] + dense[rng.integers(0, nhaps, ntgt)]).astype(np.uint8)
    gt[rng.random(gt.shape) < 0.03] = 3
    bh = np.stack([np.arange(K) if K == nhaps else rng.choice(nhaps, K, replace=False) for _ in range(ntgt)])
    sp = [_splits(rng, M, k) for k in kinds]
    nsp = np.array([len(s) for s in sp], np.int32)
    rowoff = np.concatenate([[0], np.cumsum(2 * nsp + 1)]).astype(np.int64)
    splits = np.zeros((ntgt, M), np.int32)
    for t, s in enumerate(sp):
        splits[t, :len(s)] = s
    np.array([ntgt, M, nhaps, K], np.int32).tofile(tmp_path / "params_i.bin")
    gt.tofile(tmp_path / "gt.bin")
    hm.tofile(tmp_path / "hapmajor.bin")
    bh.astype(np.int32).tofile(tmp_path / "besthaps.bin")
    splits.tofile(tmp_path / "splits.bin")
    nsp.tofile(tmp_path / "nsplits.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_cref.bin", np.uint64).reshape(-1, W(K))
    for t in range(ntgt):
        ocr, _ = R.cref(gt[t], sm, nhaps, bh[t], sp[t])
        np.testing.assert_array_equal(out[rowoff[t]:rowoff[t + 1]], ocr, err_msg=f"target {t} ({kinds[t]})")


@pytest.mark.parametrize("K", [64, 50, 200])
def test_cref_emulated_golden(emu_exe, tmp_path, K):
    """The reference's own condensed references of the golden panel (made by
    its Target::condensedReferenceT from its own best haplotypes and split
    sites): K = 50 is not a multiple of 32, K = 200 takes every reference
    haplotype (the identity selection)."""
    g = np.load(golden_path("golden_tiny.npz"))
    pre = f"K{K}_"
    gt = np.ascontiguousarray(g["gt"], np.uint8)
    ntgt, M = gt.shape
    nhaps = int(g["nhaps"])
    ns = g[pre + "nsplits"].astype(np.int32)
    rowoff = np.concatenate([[0], np.cumsum(g[pre + "rows"])]).astype(np.int64)
    assert np.array_equal(np.diff(rowoff), 2 * ns + 1)
    splits = np.zeros((ntgt, M), np.int32)
    off = np.concatenate([[0], np.cumsum(ns)])
    for t in range(ntgt):
        splits[t, :ns[t]] = g[pre + "splits"][off[t]:off[t + 1]]
    np.array([ntgt, M, nhaps, K], np.int32).tofile(tmp_path / "params_i.bin")
    gt.tofile(tmp_path / "gt.bin")
    np.ascontiguousarray(g["hapmajor_typed"]).tofile(tmp_path / "hapmajor.bin")
    g[pre + "besthaps"].astype(np.int32).tofile(tmp_path / "besthaps.bin")
    splits.tofile(tmp_path / "splits.bin")
    ns.tofile(tmp_path / "nsplits.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_cref.bin", np.uint64).reshape(-1, W(K))
    np.testing.assert_array_equal(out, g[pre + "cref"])


def test_cref_emulated_bench_setting(emu_exe, tmp_path):
    """K = 4096 of the 5,000 cfg1 reference haplotypes with the oracle's own
    best haplotypes and split sites of cfg1 targets (16 CTAs per target)."""
    from eimp_b200 import synth
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    gt = np.ascontiguousarray(tg.gt[:2], np.uint8)
    ntgt, M = gt.shape
    K = 4096
    bh, sp = [], []
    for t in range(ntgt):
        b, _ = R.besthaps(gt[t], hm, K)
        bh.append(b)
        sp.append(R.calllocs(gt[t], R.monos(hm, M, b), cm)[0])
    nsp = np.array([len(s) for s in sp], np.int32)
    rowoff = np.concatenate([[0], np.cumsum(2 * nsp + 1)]).astype(np.int64)
    splits = np.zeros((ntgt, M), np.int32)
    for t, s in enumerate(sp):
        splits[t, :len(s)] = s
    np.array([ntgt, M, panel.nhaps, K], np.int32).tofile(tmp_path / "params_i.bin")
    gt.tofile(tmp_path / "gt.bin")
    np.ascontiguousarray(hm).tofile(tmp_path / "hapmajor.bin")
    np.stack(bh).astype(np.int32).tofile(tmp_path / "besthaps.bin")
    splits.tofile(tmp_path / "splits.bin")
    nsp.tofile(tmp_path / "nsplits.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_cref.bin", np.uint64).reshape(-1, W(K))
    for t in range(ntgt):
        ocr, _ = R.cref(gt[t], sm, panel.nhaps, bh[t], sp[t])
        np.testing.assert_array_equal(out[rowoff[t]:rowoff[t + 1]], ocr)
