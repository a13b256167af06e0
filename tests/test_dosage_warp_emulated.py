"""The dosage kernel (eimp_b200/csrc/imp_kernels.cu: dosage_kernel,
TargetImp::imputeBunch) runs on the CPU under the host warp emulator
(tests/warp_emu): every warp collective must be reached by all 32 lanes from
the same call site, no access may leave its buffers (address and
undefined-behaviour sanitizers), and the dosages and alleles must equal the
oracle restatement -- over the whole panel and over windows that start off a
64-site boundary, and on a panel built so that the low-frequency shortcut
(TargetImp.cpp:522-531) and more than 32 slots per tile occur."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W, pack_rows, transpose_bits, unpack_rows

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("dos_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "imp_kernels.cu")).read()
    i = src.index("// dosages (TargetImp::imputeBunch")
    i = src.rindex("// ----", 0, i)
    j = src.index("// launchers")
    j = src.rindex("// ----", 0, j)
    (d / "dosage_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                      "namespace eimp {\n" + src[i:j] + "}  // namespace eimp\n")
    exe = d / "dosage_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "dosage_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def segmap(typed, Mref):
    cnt = np.searchsorted(typed, np.arange(Mref), side="right")
    segm = np.maximum(cnt - 1, 0).astype(np.int32)
    common = np.zeros(Mref, np.uint8)
    common[typed] = 1
    return segm, common


def run_kernel(exe, d, matches, absperm, sitemajor_full, typed, af, phased, gt, b0, n, imputeCalls=False):
    nh = phased.shape[0]
    Mref, K = sitemajor_full.shape[0], absperm.shape[1]
    M = len(typed)
    cap = max(1, max(len(m) for m in matches))
    mt = np.zeros((nh, cap, 4), np.int32)
    nm = np.zeros(nh, np.int32)
    for h, m in enumerate(matches):
        mt[h, :len(m)] = m
        nm[h] = len(m)
    hapfull = transpose_bits(sitemajor_full, Mref, K)
    os.makedirs(d, exist_ok=True)
    params = np.array([nh, cap, K, hapfull.shape[1], M, phased.shape[1], K, b0, n, int(imputeCalls), Mref], np.int32)
    for name, a in [("params_i", params), ("matches", mt), ("nmatch", nm), ("absperm", absperm.astype(np.int32)),
                    ("hapfull", hapfull), ("typed", np.asarray(typed, np.int64)), ("af", af.astype(np.float32)),
                    ("phased", phased.astype(np.uint64)), ("gt", gt.astype(np.uint8))]:
        np.ascontiguousarray(a).tofile(os.path.join(d, name + ".bin"))
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    dos = np.fromfile(os.path.join(d, "o_dos.bin"), np.float32).reshape(nh, n)
    bits = np.fromfile(os.path.join(d, "o_bits.bin"), np.uint64).reshape(nh, (n + 63) // 64)
    # the segment map and the per-site pairs of the segment-map kernel
    segm, common = segmap(typed, Mref)
    np.testing.assert_array_equal(np.fromfile(os.path.join(d, "o_segm.bin"), np.int32), segm)
    si = np.fromfile(os.path.join(d, "o_sinfo.bin"), np.int32).reshape(Mref, 2)
    np.testing.assert_array_equal(si[:, 0] & 0x7fffffff, segm)
    np.testing.assert_array_equal(si[:, 0] < 0, common.astype(bool))
    np.testing.assert_array_equal(si[:, 1] < 0, af > 0.5)
    # the shortcut height: the smallest h with (double)(float maf * float K) < 0.01 * h
    maf = np.where(af > 0.5, np.float32(1) - af, af).astype(np.float32)
    x = (maf * np.float32(K)).astype(np.float32).astype(np.float64)
    h = si[:, 1] & 0x7fffffff
    assert np.all(x < 0.01 * h.astype(np.float64))
    assert np.all((h == 1) | ~(x < 0.01 * (h - 1).astype(np.float64)))
    return dos, bits


def oracle_full(matches, absperm, sitemajor_full, typed, af, nrefhaps, phased, gt):
    from oracle import restate as R
    out_d, out_b = [], []
    for h in range(phased.shape[0]):
        miss = np.where(gt[h // 2] == 3)[0].astype(np.int64)
        b, dd, _ = R.impute(matches[h], absperm, sitemajor_full, typed, af, nrefhaps, miss, phased[h])
        out_d.append(dd)
        out_b.append(b)
    return np.array(out_d), np.array(out_b)


def test_dosages_golden_windows(emu_exe, tmp_path):
    g = np.load(golden_path("golden_tiny.npz"))
    counts = g["imp_nmatches"]
    off = np.concatenate([[0], np.cumsum(counts)])
    matches = [g["imp_matches"][off[h]:off[h + 1]] for h in range(len(counts))]
    Mref = int(g["Mref"])
    args = (g["imp_absperm"], g["sitemajor_full"], g["typed"], g["af_full"])
    od, ob = oracle_full(matches, *args, int(g["nhaps"]), g["imp_phased"], g["gt"])
    full = unpack_rows(ob, Mref)
    for k, (b0, n) in enumerate(((0, Mref), (37, 500), (1000, 1999), (Mref - 10, 10))):
        dos, bits = run_kernel(emu_exe, tmp_path / f"w{k}", matches, *args, g["imp_phased"], g["gt"], b0, n)
        np.testing.assert_array_equal(dos, od[:, b0:b0 + n])
        np.testing.assert_array_equal(unpack_rows(bits, n), full[:, b0:b0 + n])


def test_dosages_shortcut_and_wide_tiles(emu_exe, tmp_path):
    """300 reference haplotypes, 200 of them one haplotype copied with rare
    differences at untyped sites only: the targets copying it have matches of
    height ~200 (more than 32 slots per tile, several pages of slots), and
    sites with one minor allele take the low-frequency shortcut, alt-major
    ones included."""
    from oracle import restate as R
    rng = np.random.default_rng(77)
    Mref, nh = 1500, 300
    typed = np.sort(rng.choice(Mref, 150, replace=False)).astype(np.int64)
    base = (rng.random(Mref) < 0.5).astype(np.uint8)
    ref = (rng.random((nh, Mref)) < 0.5).astype(np.uint8)
    ref[:200] = base
    untyped = np.setdiff1d(np.arange(Mref), typed)
    rare = rng.choice(untyped, 300, replace=False)
    for s in rare:                      # one haplotype differs from all others
        v = rng.integers(0, 2)
        ref[:, s] = v
        ref[rng.integers(0, nh), s] = 1 - v
    af = ref.mean(axis=0).astype(np.float32)
    sm_full = pack_rows(ref.T.copy(), W(nh))
    sm_typed = np.ascontiguousarray(sm_full[typed])
    nt = 3
    tgt = np.concatenate([np.repeat(base[None], 4, axis=0), ref[200:202]])[:2 * nt].copy()
    th = tgt[:, typed]
    gt = (th[0::2] + th[1::2]).astype(np.uint8)
    gt[1, :5] = 3
    phased = pack_rows(th, W(len(typed)))
    compr, c0, ap = R.pbwt(sm_typed, nh, absperm=True)
    matches = [R.smmatches(compr, c0, len(typed), nh, phased[h], np.where(gt[h // 2] == 3)[0].astype(np.int64))
               for h in range(2 * nt)]
    assert max(int((m[:, 3] - m[:, 2]).max()) + 1 for m in matches if len(m)) > 64
    od, ob = oracle_full(matches, ap, sm_full, typed, af, nh, phased, gt)
    dos, bits = run_kernel(emu_exe, tmp_path / "s", matches, ap, sm_full, typed, af, phased, gt, 0, Mref)
    np.testing.assert_array_equal(dos, od)
    np.testing.assert_array_equal(unpack_rows(bits, Mref), unpack_rows(ob, Mref))
    # the shortcut was taken: an imputed site covered by a match whose height
    # passes the test of TargetImp.cpp:526, for both allele orientations
    maf = np.where(af > 0.5, np.float32(1) - af, af).astype(np.float32)
    segm, common = segmap(typed, Mref)
    taken = set()
    for h, m in enumerate(matches):
        for st, en, rs, re in m:
            sites = np.flatnonzero((segm >= st) & (segm < en) & (common == 0))
            hit = sites[maf[sites].astype(np.float64) * nh < 0.01 * (re - rs + 1)]
            taken |= {bool(af[x] > 0.5) for x in hit}
    assert taken == {False, True}


def test_dosages_long_match_lists(emu_exe, tmp_path):
    """Targets unrelated to a random panel: short set-maximal matches, hundreds
    per haplotype, so every span's window start is found by the search over
    the sorted match list (more than 32 matches before most spans); windows
    starting at the panel's first site and deep inside it."""
    from oracle import restate as R
    rng = np.random.default_rng(4242)
    Mref, nh, M = 6000, 64, 3000
    typed = np.sort(rng.choice(Mref, M, replace=False)).astype(np.int64)
    ref = (rng.random((nh, Mref)) < 0.5).astype(np.uint8)
    af = ref.mean(axis=0).astype(np.float32)
    sm_full = pack_rows(ref.T.copy(), W(nh))
    sm_typed = np.ascontiguousarray(sm_full[typed])
    nt = 2
    th = (rng.random((2 * nt, M)) < 0.5).astype(np.uint8)
    gt = (th[0::2] + th[1::2]).astype(np.uint8)
    gt[0, rng.random(M) < 0.02] = 3
    phased = pack_rows(th, W(M))
    compr, c0, ap = R.pbwt(sm_typed, nh, absperm=True)
    matches = [R.smmatches(compr, c0, M, nh, phased[h], np.where(gt[h // 2] == 3)[0].astype(np.int64))
               for h in range(2 * nt)]
    assert min(len(m) for m in matches) > 300
    od, ob = oracle_full(matches, ap, sm_full, typed, af, nh, phased, gt)
    full = unpack_rows(ob, Mref)
    for k, (b0, n) in enumerate(((0, Mref), (3001, 2000), (Mref - 700, 700))):
        dos, bits = run_kernel(emu_exe, tmp_path / f"l{k}", matches, ap, sm_full, typed, af, phased, gt, b0, n)
        np.testing.assert_array_equal(dos, od[:, b0:b0 + n])
        np.testing.assert_array_equal(unpack_rows(bits, n), full[:, b0:b0 + n])


def test_dosage_division_helpers(tmp_path):
    """The dosage kernel's integer-only conversions (uint64 -> double below
    2^52, double -> float rounded to nearest even) give exactly the C casts
    of TargetImp.cpp:548, (float)((double)score / (double)sum), on 20 million
    random (score, sum) pairs of every magnitude and on random doubles in
    [2^-60, 1], ties included."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    src = open(os.path.join(CSRC, "imp_kernels.cu")).read()
    i = src.index("// uint64 -> double without the conversion unit")
    j = src.index("// one covered site's share of a match")
    prog = tmp_path / "conv.cpp"
    prog.write_text('#include "emu.h"\n' + src[i:j] + r'''
#include <random>
int main() {
    std::mt19937_64 r(12345);
    long bad = 0;
    for (long t = 0; t < 20000000; t++) {
        const int bitsz = 1 + (int)(r() % 52);
        const uint64_t sum = 1 + (r() >> (64 - bitsz)) % ((1ull << bitsz) - 1);
        const uint64_t score = (t & 7) == 0 ? sum : r() % (sum + 1);
        if (score == 0) continue;
        const float want = (float)((double)score / (double)sum);
        const float got = dos_f64_to_f32(dos_u64_to_f64(score) / dos_u64_to_f64(sum));
        if (want != got || dos_u64_to_f64(sum) != (double)sum) bad++;
    }
    for (long t = 0; t < 5000000; t++) {
        double q = std::ldexp(1.0 + (double)(r() >> 12) / 4503599627370496.0, -(int)(r() % 60) - 1);
        if (t % 3 == 0) {   // exact halfway cases between two floats
            const float f = (float)q;
            q = (double)f + std::ldexp(1.0, std::ilogb((double)f) - 24);
        }
        if (q > 1.0) q = 1.0;
        if ((float)q != dos_f64_to_f32(q)) bad++;
    }
    if (dos_f64_to_f32(1.0) != 1.0f) bad++;
    std::printf("%ld\n", bad);
    return bad != 0;
}
''')
    exe = tmp_path / "conv"
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", "-I", EMU, str(prog), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout + r.stderr


def test_dosages_haploid_golden(emu_exe, tmp_path):
    """The reference's own imputation of the haploid golden case: a reduced
    reference of the 175 existing panel haplotypes read through their panel
    columns (haploidsRefMap, TargetImp.cpp:536) and the 13 existing target
    haplotypes through a row map (PBWTImputer.cpp:130, 202); every site the
    reference writes (untyped, and missing typed ones) must equal its dosage
    and allele."""
    g = np.load(golden_path("golden_haploid.npz"))
    gt = np.ascontiguousarray(g["gt"], np.uint8)
    nt, M = gt.shape
    Mref, nh_panel, K = int(g["Mref"]), int(g["nhaps"]), int(g["imp_K"])
    hapl = g["ref_haploid"]
    refmap = np.array([c for s in range(nh_panel // 2) for c in ([2 * s] if hapl[s] else [2 * s, 2 * s + 1])],
                      np.int32)
    assert len(refmap) == K
    hapmap = np.array([h for t in range(nt) for h in ([2 * t] if g["tgt_haploid"][t] else [2 * t, 2 * t + 1])],
                      np.int32)
    counts = g["imp_nmatches"]
    assert len(counts) == len(hapmap)
    off = np.concatenate([[0], np.cumsum(counts)])
    cap = max(1, int(counts.max()))
    mt = np.zeros((2 * nt, cap, 4), np.int32)
    nm = np.zeros(2 * nt, np.int32)
    for j, h in enumerate(hapmap):
        mt[h, :counts[j]] = g["imp_matches"][off[j]:off[j + 1]]
        nm[h] = counts[j]
    hapfull = transpose_bits(g["sitemajor_full"], Mref, nh_panel)
    phased = g["imp_phased"]
    params = np.array([len(hapmap), cap, K, hapfull.shape[1], M, phased.shape[1], nh_panel, 0, Mref, 0, Mref,
                       2 * nt, 1], np.int32)
    for name, a in [("params_i", params), ("matches", mt), ("nmatch", nm),
                    ("absperm", g["imp_absperm"].astype(np.int32)), ("hapfull", hapfull),
                    ("typed", np.asarray(g["typed"], np.int64)), ("af", g["af_full"].astype(np.float32)),
                    ("phased", phased.astype(np.uint64)), ("gt", gt), ("hapmap", hapmap), ("refmap", refmap)]:
        np.ascontiguousarray(a).tofile(tmp_path / (name + ".bin"))
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    dos = np.fromfile(tmp_path / "o_dos.bin", np.float32).reshape(2 * nt, Mref)
    bits = np.fromfile(tmp_path / "o_bits.bin", np.uint64).reshape(2 * nt, (Mref + 63) // 64)
    sel = np.ones((nt, Mref), bool)
    sel[:, g["typed"]] = gt == 3
    for h in hapmap:
        s = sel[h // 2]
        np.testing.assert_array_equal(dos[h][s], g["imp_dos"][h][s])
        got, want = unpack_rows(bits[h:h + 1], Mref)[0], unpack_rows(g["imp_bits"][h:h + 1], Mref)[0]
        np.testing.assert_array_equal(got[s], want[s])
