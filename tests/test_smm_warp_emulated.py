"""The set-maximal match kernels (eimp_b200/csrc/imp_kernels.cu: smm_kernel
and the compact-tree smm_compact_kernel) run on the CPU under the host warp
emulator (tests/warp_emu): every warp collective must be reached by all 32
lanes from the same call site, no access may leave its buffers (address and
undefined-behaviour sanitizers), and the matches must equal the golden
fixtures made by the reference (TargetImp::calcSMMatches) and the oracle
restatement, with and without set-maximal errors (the haplotypes whose
trees outgrow the first launch's node pool are redone by the retry launch),
and both kernels must report a full pool or match buffer the same way."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W, pack_rows

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")
ERR_MATCH_OVERFLOW = 1 << 0
ERR_NODE_OVERFLOW = 1 << 1


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("smm_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    kh = open(os.path.join(CSRC, "kernels.h")).read()
    assert "#define SMM_WARPS 4" in kh and "#define SMMC_WARPS 2" in kh
    # one warp per block: each warp's shared memory is its own allocation
    kh = kh.replace("#define SMM_WARPS 4", "#define SMM_WARPS 1").replace("#define SMMC_WARPS 2", "#define SMMC_WARPS 1")
    (d / "kernels.h").write_text(kh)
    src = open(os.path.join(CSRC, "imp_kernels.cu")).read()
    # the match section only: the other kernels use block-wide barriers
    i = src.index("struct SNode {")
    j = src.index("// dosages (TargetImp::imputeBunch")
    j = src.rindex("// ----", 0, j)
    body = src[i:j]
    decl = "extern __shared__ uint8_t smem_raw[];"
    assert body.count(decl) == 2
    body = body.replace(decl, "uint8_t *smem_raw = emu_smem_ptr;")
    (d / "smm_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                   "namespace eimp {\n" + body + "}  // namespace eimp\n")
    exe = d / "smm_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "smm_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def run_kernel(exe, d, which, compr, count0, phased, gt, K, setmaxerrors=0, cap=None, pool=0):
    nh = phased.shape[0]
    M = gt.shape[1]
    cap = cap or M // 4 + 64
    os.makedirs(d, exist_ok=True)
    for name, a in [("params_i", np.array([nh, M, K, setmaxerrors, cap], np.int32)),
                    ("compr", compr.astype(np.uint32)), ("count0", count0.astype(np.int32)),
                    ("phased", phased.astype(np.uint64)), ("gt", gt.astype(np.uint8))]:
        np.ascontiguousarray(a).tofile(os.path.join(d, name + ".bin"))
    r = subprocess.run([exe, str(d), str(which), str(pool)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    m = np.fromfile(os.path.join(d, "o_matches.bin"), np.int32).reshape(nh, cap, 4)
    n = np.fromfile(os.path.join(d, "o_nmatch.bin"), np.int32)
    st = int(np.fromfile(os.path.join(d, "o_status.bin"), np.uint32)[0])
    retried, moved = (int(x) for x in np.fromfile(os.path.join(d, "o_retried.bin"), np.int32))
    run_kernel.moved = moved
    return [m[h, :n[h]].astype(np.int64) if n[h] >= 0 else None for h in range(nh)], n, st, retried


@pytest.mark.parametrize("which", [0, 1, 2], ids=["wide", "compact", "compact16"])
def test_matches_golden(emu_exe, tmp_path, which):
    from oracle import restate as R
    g = np.load(golden_path("golden_tiny.npz"))
    K = int(g["nhaps"])
    compr, c0, _ = R.pbwt(g["sitemajor_typed"], K)
    np.testing.assert_array_equal(compr, g["imp_compr"])
    got, n, st, _ = run_kernel(emu_exe, tmp_path / "k", which, compr, c0, g["imp_phased"], g["gt"], K)
    assert st == 0
    counts = g["imp_nmatches"]
    off = np.concatenate([[0], np.cumsum(counts)])
    for h in range(len(counts)):
        np.testing.assert_array_equal(got[h], g["imp_matches"][off[h]:off[h + 1]])


@pytest.mark.parametrize("which,pool", [(0, 0), (1, 0), (2, 0), (1, 4), (2, 4), (2, 1)],
                         ids=["wide", "compact", "compact16", "compact-pool", "compact16-pool", "compact16-pool1"])
@pytest.mark.parametrize("setmaxerrors", [0, 1])
def test_matches_vs_oracle_cfg1(emu_exe, tmp_path, which, pool, setmaxerrors):
    """cfg1 panel (5000 haplotypes, 2000 typed sites), 12 target haplotypes
    from the true haplotypes with their missing genotypes, one target with
    more than half of its sites missing (no matches).  With one set-maximal
    error the trees outgrow the first launch's node pool (up to 718 nodes):
    without global pools those haplotypes come from the retry pass; with
    them, the first pass moves their trees to a global pool and goes on, and
    with fewer pools than such haplotypes the rest are retried."""
    from eimp_b200 import synth
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 6
    _, sm, _ = typed_views(panel, tg.typed)
    M = len(tg.typed)
    gt = tg.gt[:nt].copy()
    gt[nt - 1, np.random.default_rng(5).permutation(M)[:M // 2 + 1]] = 3
    phased = pack_rows(tg.truth[:2 * nt], W(M))
    compr, c0, _ = R.pbwt(sm, panel.nhaps)
    got, n, st, retried = run_kernel(emu_exe, tmp_path / "k", which, compr, c0, phased, gt, panel.nhaps,
                                     setmaxerrors, cap=M + 64, pool=pool)
    moved = run_kernel.moved
    assert st == 0
    if pool == 0:
        assert (retried > 0) == (setmaxerrors > 0) and moved == 0
    elif setmaxerrors:
        assert moved > 0
        assert (retried > 0) == (moved > pool)
    assert n[2 * nt - 2] == 0 and n[2 * nt - 1] == 0
    for h in range(2 * nt):
        miss = np.where(gt[h // 2] == 3)[0].astype(np.int64)
        om = R.smmatches(compr, c0, M, panel.nhaps, phased[h], miss, setmaxerrors)
        np.testing.assert_array_equal(got[h], om)


def test_errors_reported(emu_exe, tmp_path):
    """A tree that outgrows the retry pool too (6 set-maximal errors), and a
    match list longer than its buffer: every kernel gives the haplotype match
    count -1 and the same status bits, and they agree on the other haplotypes."""
    from eimp_b200 import synth
    from eimp_b200.synth import typed_views
    from oracle import restate as R  # noqa: F401  (the PBWT restatement below)
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 2
    _, sm, _ = typed_views(panel, tg.typed)
    M = len(tg.typed)
    gt = tg.gt[:nt]
    phased = pack_rows(tg.truth[:2 * nt], W(M))
    compr, c0, _ = R.pbwt(sm, panel.nhaps)
    for sme, cap, bit in [(6, M + 64, ERR_NODE_OVERFLOW), (0, 4, ERR_MATCH_OVERFLOW)]:
        res = [run_kernel(emu_exe, tmp_path / f"k{w}_{sme}", w, compr, c0, phased, gt, panel.nhaps, sme, cap)
               for w in (0, 1, 2)]
        g0, n0, s0, _ = res[0]
        assert s0 == bit
        assert (n0 == -1).any()
        for g1, n1, s1, _ in res[1:]:
            np.testing.assert_array_equal(n0, n1)
            assert s1 == bit
            for a, b in zip(g0, g1):
                if a is not None:
                    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("which", [0, 1, 2], ids=["wide", "compact", "compact16"])
def test_matches_haploid_golden(emu_exe, tmp_path, which):
    """The reference's own matches of the haploid golden case: the 13 existing
    target haplotypes (a row map, PBWTImputer.cpp:130, 202) against its
    reduced imputation PBWT of the 175 existing panel haplotypes."""
    g = np.load(golden_path("golden_haploid.npz"))
    gt = np.ascontiguousarray(g["gt"], np.uint8)
    nt, M = gt.shape
    K = int(g["imp_K"])
    compr = np.ascontiguousarray(g["imp_compr"], np.uint32)
    count0 = compr[:, -1].astype(np.int32)   # the last pair's zeros (the tail is padded with ones)
    hapmap = np.array([h for t in range(nt) for h in ([2 * t] if g["tgt_haploid"][t] else [2 * t, 2 * t + 1])],
                      np.int32)
    cap = M // 4 + 64
    d = tmp_path / "k"
    os.makedirs(d, exist_ok=True)
    for name, a in [("params_i", np.array([len(hapmap), M, K, 0, cap, 2 * nt, 1], np.int32)), ("compr", compr),
                    ("count0", count0), ("phased", g["imp_phased"].astype(np.uint64)), ("gt", gt),
                    ("hapmap", hapmap)]:
        np.ascontiguousarray(a).tofile(d / (name + ".bin"))
    r = subprocess.run([emu_exe, str(d), str(which), "0"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    m = np.fromfile(d / "o_matches.bin", np.int32).reshape(2 * nt, cap, 4)
    n = np.fromfile(d / "o_nmatch.bin", np.int32)
    assert int(np.fromfile(d / "o_status.bin", np.uint32)[0]) == 0
    counts = g["imp_nmatches"]
    off = np.concatenate([[0], np.cumsum(counts)])
    for j, h in enumerate(hapmap):
        assert n[h] == counts[j]
        np.testing.assert_array_equal(m[h, :n[h]].astype(np.int64), g["imp_matches"][off[j]:off[j + 1]])
