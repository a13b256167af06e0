"""The condensed-reference PBWT kernel (eimp_b200/csrc/phase_prep.cu
pbwt_kernel; PBWT::buildComprPBWT, PBWT.cpp:207-285, forward and backward) run
on the CPU under the host warp emulator with the address and
undefined-behaviour sanitizers: every compressed row ([data, zeros through the
word] pairs, the tail padded with ones), the row padding and the forward zero
counts must equal the oracle restatement, for K a multiple of 32 and not, K
below one word, several warps, two words per thread, an empty target and rows
of all zeros and all ones."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")

CP_ASYNC_HOST = """
// host stand-ins of the asynchronous copies: a plain 16-byte copy
inline void cp_async16(void *smem, const void *gmem) { std::memcpy(smem, gmem, 16); }
inline void cp_async_commit() {}
inline void cp_async_wait_all() {}
"""


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("pbwt_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "phase_prep.cu")).read()
    i = src.index("// position p of the prefix order -> its slot in the swizzled array")
    j = src.index("template <int WPT>\nstatic cudaError_t launch_pbwt_w(")
    body = src[i:j]
    a = "extern __shared__ __align__(16) uint8_t smem[];"
    assert a in body
    body = body.replace(a, "uint8_t *smem = emu_smem_ptr;")
    (d / "pbwt_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                    "namespace eimp {\n" + CP_ASYNC_HOST + body + "}  // namespace eimp\n")
    exe = d / "pbwt_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "pbwt_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def _rows(rng, n, K):
    wK = W(K)
    dens = rng.choice([0.0, 0.02, 0.3, 0.5, 1.0], size=n, p=[0.1, 0.3, 0.25, 0.25, 0.1])
    bits = (rng.random((n, wK * 64)) < dens[:, None]).astype(np.uint8)
    bits[:, K:] = rng.integers(0, 2, (n, wK * 64 - K))   # past K: never read
    return np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wK)


@pytest.mark.parametrize("K,wpt,nrows", [(4096, 1, [9, 0, 5]), (1000, 1, [7, 3]), (20, 1, [6]),
                                         (2200, 2, [4, 5]), (64, 1, [1, 2])])
def test_pbwt_emulated(emu_exe, tmp_path, K, wpt, nrows):
    from oracle import restate as R
    rng = np.random.default_rng(K * 31 + len(nrows))
    rowoff = np.concatenate([[0], np.cumsum(nrows)]).astype(np.int64)
    cref = _rows(rng, int(rowoff[-1]), K)
    kw = 2 * ((K + 31) // 32)
    rowstride = kw + 6
    np.array([len(nrows), K, rowstride, 1, wpt], np.int32).tofile(tmp_path / "params_i.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    cref.tofile(tmp_path / "cref.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_pbwt.bin", np.uint32).reshape(-1, rowstride)
    c0 = np.fromfile(tmp_path / "o_count0.bin", np.int32)
    for t, n in enumerate(nrows):
        if n == 0:
            continue
        r0 = int(rowoff[t])
        rows = cref[r0:r0 + n]
        fwd, fc0 = R.pbwt(np.ascontiguousarray(rows), K)[:2]
        bck = R.pbwt(np.ascontiguousarray(rows[::-1]), K)[0]
        got = out[2 * r0:2 * r0 + 2 * n]
        np.testing.assert_array_equal(got[:n, :kw], fwd)
        np.testing.assert_array_equal(got[n:, :kw], bck)
        assert (got[:, kw:] == 0).all()   # row padding
        np.testing.assert_array_equal(c0[r0:r0 + n], fc0)


@pytest.mark.parametrize("K", [64, 50, 200])
def test_pbwt_emulated_golden(emu_exe, tmp_path, K):
    """The reference's own forward and backward PBWTs (PBWT::buildComprPBWT)
    of the golden panel's condensed references, and the forward zero counts."""
    g = np.load(golden_path("golden_tiny.npz"))
    pre = f"K{K}_"
    Kc = min(K, int(g["nhaps"]))
    rows = g[pre + "rows"].astype(np.int64)
    rowoff = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    kw = 2 * ((Kc + 31) // 32)
    np.array([len(rows), Kc, kw, 1, 1], np.int32).tofile(tmp_path / "params_i.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    np.ascontiguousarray(g[pre + "cref"]).tofile(tmp_path / "cref.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_pbwt.bin", np.uint32).reshape(-1, kw)
    np.testing.assert_array_equal(out, g[pre + "pbwt"])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "o_count0.bin", np.int32), g[pre + "count0"])


def test_pbwt_emulated_bench_setting(emu_exe, tmp_path):
    """K = 4096: the oracle's condensed references of two cfg1 targets (the
    rows the bench's PBWT sweep sees), forward and backward, against the
    oracle's PBWTs."""
    from eimp_b200 import synth
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    K = 4096
    crefs = []
    for t in range(2):
        b, _ = R.besthaps(tg.gt[t], hm, K)
        sp = R.calllocs(tg.gt[t], R.monos(hm, len(tg.typed), b), cm)[0]
        crefs.append(R.cref(tg.gt[t], sm, panel.nhaps, b, sp)[0])
    nrows = [len(c) for c in crefs]
    rowoff = np.concatenate([[0], np.cumsum(nrows)]).astype(np.int64)
    kw = 2 * ((K + 31) // 32)
    np.array([len(nrows), K, kw, 1, 1], np.int32).tofile(tmp_path / "params_i.bin")
    rowoff.tofile(tmp_path / "rowoff.bin")
    np.ascontiguousarray(np.concatenate(crefs)).tofile(tmp_path / "cref.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    out = np.fromfile(tmp_path / "o_pbwt.bin", np.uint32).reshape(-1, kw)
    c0 = np.fromfile(tmp_path / "o_count0.bin", np.int32)
    for t, cr in enumerate(crefs):
        r0, n = int(rowoff[t]), nrows[t]
        fwd, fc0 = R.pbwt(cr, K)[:2]
        np.testing.assert_array_equal(out[2 * r0:2 * r0 + n], fwd)
        np.testing.assert_array_equal(out[2 * r0 + n:2 * r0 + 2 * n], R.pbwt(cr, K, reverse=True)[0])
        np.testing.assert_array_equal(c0[r0:r0 + n], fc0)
