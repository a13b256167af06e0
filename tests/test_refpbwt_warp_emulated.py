"""The reference PBWT kernels (eimp_b200/csrc/imp_kernels.cu:
refpbwt_ckpt_kernel, refpbwt_fill_kernel; PBWT::buildComprPBWT with
refPBWT=true, PBWT.cpp:207-285, 136-142) run on the CPU under the host warp
emulator with the address and undefined-behaviour sanitizers: the compressed
rows, every prefix array and the zero counts must equal the oracle
restatement, with the orders in shared memory and in global scratch, the
site rows staged and read in place, and site counts that end on, before and
past a checkpoint interval and off a multiple of the checkpoint step."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from eimp_b200.bits import W

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("refpbwt_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "imp_kernels.cu")).read()
    i = src.index("// block-wide exclusive scan")
    i = src.rindex("// ----", 0, i)
    j = src.index("// bit-matrix transpose")
    j = src.rindex("// ----", 0, j)
    body = src[i:j]
    for a, b in [("extern __shared__ uint64_t rp_smem[];",
                  "uint64_t *rp_smem = reinterpret_cast<uint64_t *>(emu_smem_ptr);"),
                 ("extern __shared__ uint8_t smem[];", "uint8_t *smem = emu_smem_ptr;")]:
        assert a in body
        body = body.replace(a, b)
    (d / "refpbwt_emu.cpp").write_text('#include "emu.h"\n#include "common.cuh"\n#include "kernels.h"\n'
                                       "namespace eimp {\n" + body + "}  // namespace eimp\n")
    exe = d / "refpbwt_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "refpbwt_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


@pytest.mark.parametrize("M,K,in_smem,stage", [(150, 300, 1, 1), (128, 1100, 0, 1), (67, 700, 0, 0),
                                               (1, 64, 1, 0), (4, 33, 1, 1)])
def test_refpbwt_emulated(emu_exe, tmp_path, M, K, in_smem, stage):
    from oracle import restate as R
    rng = np.random.default_rng(M * 7919 + K)
    wN = W(K)
    dens = rng.choice([0.0, 0.01, 0.2, 0.5, 1.0], size=M, p=[0.05, 0.3, 0.3, 0.3, 0.05])
    bits = (rng.random((M, wN * 64)) < dens[:, None]).astype(np.uint8)
    bits[:, K:] = rng.integers(0, 2, (M, wN * 64 - K))   # padding past K is never read
    sm = np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(M, wN)
    np.array([M, K, wN, in_smem, stage], np.int32).tofile(tmp_path / "params_i.bin")
    sm.tofile(tmp_path / "sitemajor.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    kw = 2 * ((K + 31) // 32)
    compr = np.fromfile(tmp_path / "o_compr.bin", np.uint32).reshape(M, kw)
    ap = np.fromfile(tmp_path / "o_absperm.bin", np.int32).reshape(M + 1, K)
    c0 = np.fromfile(tmp_path / "o_count0.bin", np.int32)
    rc, rc0, rap = R.pbwt(np.ascontiguousarray(sm), K, absperm=True)
    np.testing.assert_array_equal(ap, rap)
    np.testing.assert_array_equal(compr, rc)
    np.testing.assert_array_equal(c0, rc0)


@pytest.mark.parametrize("in_smem,stage", [(1, 1), (0, 0)])
def test_refpbwt_emulated_golden(emu_exe, tmp_path, in_smem, stage):
    """The reference's own imputation PBWT of the golden panel's typed sites
    (PBWTImputer's compressed rows and prefix arrays)."""
    g = np.load(golden_path("golden_tiny.npz"))
    sm = np.ascontiguousarray(g["sitemajor_typed"])
    M, wN = sm.shape
    K = int(g["nhaps"])
    np.array([M, K, wN, in_smem, stage], np.int32).tofile(tmp_path / "params_i.bin")
    sm.tofile(tmp_path / "sitemajor.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    kw = 2 * ((K + 31) // 32)
    compr = np.fromfile(tmp_path / "o_compr.bin", np.uint32).reshape(M, kw)
    ap = np.fromfile(tmp_path / "o_absperm.bin", np.int32).reshape(M + 1, K)
    np.testing.assert_array_equal(compr, g["imp_compr"].reshape(M, kw))
    np.testing.assert_array_equal(ap, g["imp_absperm"].reshape(M + 1, K))
