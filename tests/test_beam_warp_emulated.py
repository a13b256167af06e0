"""The beam phasing kernel (eimp_b200/csrc/beam.cu) run on the CPU under the
host warp emulator (tests/warp_emu): every warp collective must be reached by
all 32 lanes from the same call site, no access may leave its buffers
(address and undefined-behaviour sanitizers), and the phased haplotypes,
dosages and confidences must equal the golden fixtures made by the reference
(beam 16 at K = 64, 50 and 200) and the oracle restatement (beams 128, 64 and
4 with pre-phasing; K = 4096 and beam 128 on cfg1 targets, the bench's
setting)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


def split_rows(flat, counts):
    out, o = [], 0
    for c in counts:
        out.append(flat[o:o + int(c)])
        o += int(c)
    return out


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("beam_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    kh = open(os.path.join(CSRC, "kernels.h")).read()
    assert "#define BEAM_WARPS 4" in kh
    # one warp per block: each warp's shared memory is its own allocation
    (d / "kernels.h").write_text(kh.replace("#define BEAM_WARPS 4", "#define BEAM_WARPS 1"))
    src = open(os.path.join(CSRC, "beam.cu")).read()
    # the launcher (triple-chevron launch, runtime attributes) is device-only
    i, j = src.index("static size_t beam_smem("), src.rindex("}  // namespace eimp")
    src = src[:i] + src[j:]
    decl = "extern __shared__ __align__(16) uint8_t smem_raw[];"
    assert decl in src
    src = src.replace(decl, "uint8_t *smem_raw = emu_smem_ptr;")
    (d / "beam_emu.cpp").write_text('#include "emu.h"\n' + src)
    exe = d / "beam_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-ffp-contract=off", "-fno-fast-math",
           "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-I", EMU, "-I", str(d),
           os.path.join(EMU, "beam_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def write_inputs(d, gt, monos, splits, calls, cmd, pbwt, count0, rows, K, P, prephase):
    nt, M = gt.shape
    ns = np.array([len(s) for s in splits], np.int32)
    nc = np.array([len(c) for c in calls], np.int32)
    sp = np.zeros((nt, M), np.int32)
    ca = np.zeros((nt, M), np.int32)
    cm = np.zeros((nt, M + 1), np.float32)
    for t in range(nt):
        sp[t, :ns[t]] = splits[t]
        ca[t, :nc[t]] = calls[t]
        cm[t, :len(cmd[t])] = cmd[t]
    rowoff = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    # history sizes of the reference defaults: HistorySize 100, HistorySizeFast 30, hist 1.0
    pi = np.array([nt, M, K, 100, P, 24, 30, 64, 10, int(prephase), 1], np.int32)
    pf = np.array([2.0, 0.003, 0.003, 0.5, 0.9, 0.99, 1.0], np.float32)
    for name, a in [("params_i", pi), ("params_f", pf), ("gt", gt.astype(np.uint8)), ("monos", monos),
                    ("splits", sp), ("nsplits", ns), ("calls", ca), ("ncalls", nc), ("cmd", cm),
                    ("pbwt", pbwt.astype(np.uint32)), ("count0", count0.astype(np.int32)), ("rowoff", rowoff)]:
        np.ascontiguousarray(a).tofile(os.path.join(d, name + ".bin"))


def run_emu(exe, d, nt, M, queue=False):
    r = subprocess.run([exe, str(d)] + (["queue"] if queue else []), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    wM = ((M + 511) // 512) * 8
    rd = lambda n, dt, shape: np.fromfile(os.path.join(d, n), dt).reshape(shape)
    return (rd("o_mats.bin", np.uint64, (nt, wM)), rd("o_pats.bin", np.uint64, (nt, wM)),
            rd("o_dm.bin", np.float32, (nt, M)), rd("o_dp.bin", np.float32, (nt, M)),
            rd("o_tc.bin", np.float32, (nt,)), rd("o_nc.bin", np.int32, (nt,)), rd("o_st.bin", np.uint32, (nt,)))


def golden_inputs(g, K):
    pre = f"K{K}_"
    ns = g[pre + "nsplits"]
    return dict(gt=g["gt"], monos=g[pre + "monos"], splits=split_rows(g[pre + "splits"], ns),
                calls=split_rows(g[pre + "calls"], g[pre + "ncalls"]),
                cmd=split_rows(g[pre + "cmdiffs"], [s + 1 if s else 0 for s in ns]),
                pbwt=g[pre + "pbwt"], count0=g[pre + "count0"], rows=g[pre + "rows"])


@pytest.mark.parametrize("K", [64, 50, 200])
def test_beam_emulated_matches_reference_golden(emu_exe, tmp_path, K):
    """The reference's own phasing of the golden panel (beam 16): K = 50 is
    not a multiple of 32 (padded PBWT rows), K = 200 takes every reference
    haplotype."""
    g = np.load(golden_path("golden_tiny.npz"))
    pre = f"K{K}_"
    write_inputs(tmp_path, K=K, P=16, prephase=False, **golden_inputs(g, K))
    nt, M = g["gt"].shape
    mats, pats, dm, dp, tc, nc, st = run_emu(emu_exe, tmp_path, nt, M)
    assert not st.any()
    np.testing.assert_array_equal(mats, g[pre + "mat"])
    np.testing.assert_array_equal(pats, g[pre + "pat"])
    np.testing.assert_array_equal(dm, g[pre + "dos_mat"])
    np.testing.assert_array_equal(dp, g[pre + "dos_pat"])
    np.testing.assert_array_equal(tc, g[pre + "totalconf"])
    np.testing.assert_array_equal(nc, g[pre + "ncallsites"])


def test_beam_emulated_persistent_queue(emu_exe, tmp_path):
    """The persistent form: one warp takes all eight targets from the queue in
    longest-first order and reuses one arena (filled with a pattern first);
    every target's outputs must equal the reference's."""
    g = np.load(golden_path("golden_tiny.npz"))
    K = 64
    write_inputs(tmp_path, K=K, P=16, prephase=False, **golden_inputs(g, K))
    nt, M = g["gt"].shape
    mats, pats, dm, dp, tc, nc, st = run_emu(emu_exe, tmp_path, nt, M, queue=True)
    assert not st.any()
    np.testing.assert_array_equal(mats, g["K64_mat"])
    np.testing.assert_array_equal(pats, g["K64_pat"])
    np.testing.assert_array_equal(dm, g["K64_dos_mat"])
    np.testing.assert_array_equal(dp, g["K64_dos_pat"])
    np.testing.assert_array_equal(tc, g["K64_totalconf"])
    np.testing.assert_array_equal(nc, g["K64_ncallsites"])


@pytest.mark.parametrize("P", [128, 64, 4])
def test_beam_emulated_prephasing_matches_oracle(emu_exe, tmp_path, P):
    """Beam 128 is the reference's default, the bench's setting and the
    kernel's limit (the merge table, heap and list arrays are sized for it);
    beam 64 runs the beam-path loops over more than one warp-width of paths;
    beam 4 makes most prunes select the P best of more candidates."""
    from oracle import restate as R
    if not R.available():
        pytest.skip("oracle library not built")
    g = np.load(golden_path("golden_tiny.npz"))
    K = 64
    write_inputs(tmp_path, K=K, P=P, prephase=True, **golden_inputs(g, K))
    nt, M = g["gt"].shape
    mats, pats, dm, dp, tc, nc, st = run_emu(emu_exe, tmp_path, nt, M)
    assert not st.any()
    om, op, odm, odp = R.phase_many(g["gt"], g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"],
                                    R.params_c(K=K, beamwidth=P, doPrePhasing=True), 4)
    np.testing.assert_array_equal(mats, om)
    np.testing.assert_array_equal(pats, op)
    np.testing.assert_array_equal(dm, odm)
    np.testing.assert_array_equal(dp, odp)


@pytest.mark.parametrize("prephase", [False, True])
def test_beam_emulated_start_phases_match_reference(emu_exe, tmp_path, prephase):
    """Start phases carried over from a previous chunk (VCFData::getStartPhase)
    against the reference's own Target::phase with the same chunkStartPhase."""
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    g = np.load(golden_path("golden_tiny.npz"))
    K = 64
    nt, M = g["gt"].shape
    phases = (np.arange(nt) % 3 != 0).astype(np.uint8)
    write_inputs(tmp_path, K=K, P=16, prephase=prephase, **golden_inputs(g, K))
    phases.tofile(os.path.join(tmp_path, "startph.bin"))
    mats, pats, dm, dp, tc, nc, st = run_emu(emu_exe, tmp_path, nt, M)
    assert not st.any()
    rc = refcore.RefCore.typed_only(g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], g["gt"],
                                    g["af_full"][g["typed"]])
    rc.set_start_phases(phases)
    rc.set_params(refcore.PhaseParams(K=K, beamwidth=16, doPrePhasing=prephase))
    for t in range(nt):
        m, p, a, b, c, n = rc.phase(t)
        np.testing.assert_array_equal(mats[t], m)
        np.testing.assert_array_equal(pats[t], p)
        np.testing.assert_array_equal(dm[t], a)
        np.testing.assert_array_equal(dp[t], b)
        assert tc[t] == np.float32(c) and nc[t] == n
    rc.close()



def test_beam_emulated_bench_setting(emu_exe, tmp_path):
    """K = 4096 conditioning haplotypes (PBWT rows of 128 words staged per
    warp) and beam 128 with the reference's history sizes, as the bench runs
    them: two cfg1 targets (5,000 reference haplotypes, 2,000 typed sites).
    The inputs come from the oracle's preparation, condensed reference and
    PBWTs (pinned to the reference's golden fixtures); the phased haplotypes
    and dosages must equal the oracle's beam."""
    from eimp_b200 import synth
    from oracle import restate as R
    if not R.available():
        pytest.skip("oracle library not built")
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    K, P = 4096, 128
    gt = np.ascontiguousarray(tg.gt[:2], np.uint8)
    nt, M = gt.shape
    monos, splits, calls, cmds, pb, c0s, rows = [], [], [], [], [], [], []
    for t in range(nt):
        bh, _ = R.besthaps(gt[t], hm, K)
        mo = R.monos(hm, M, bh)
        sp, ca, cd = R.calllocs(gt[t], mo, cm)
        cr, c0 = R.cref(gt[t], sm, panel.nhaps, bh, sp)
        pb.append(np.concatenate([R.pbwt(cr, K)[0], R.pbwt(cr, K, reverse=True)[0]]))
        monos.append(mo)
        splits.append(sp)
        calls.append(ca)
        cmds.append(cd)
        c0s.append(c0)
        rows.append(len(cr))
    assert min(len(s) for s in splits) > 100
    write_inputs(tmp_path, gt=gt, monos=np.stack(monos), splits=splits, calls=calls, cmd=cmds,
                 pbwt=np.concatenate(pb), count0=np.concatenate(c0s), rows=np.array(rows), K=K, P=P,
                 prephase=False)
    mats, pats, dm, dp, tc, nc, st = run_emu(emu_exe, tmp_path, nt, M)
    assert not st.any()
    om, op, odm, odp = R.phase_many(gt, hm, sm, cm, R.params_c(K=K, beamwidth=P), 2)
    np.testing.assert_array_equal(mats, om)
    np.testing.assert_array_equal(pats, op)
    np.testing.assert_array_equal(dm, odm)
    np.testing.assert_array_equal(dp, odp)
