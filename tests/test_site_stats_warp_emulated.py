"""The output-statistics kernel (eimp_b200/csrc/site_stats.cu) run on the CPU
under the host warp emulator (tests/warp_emu), with the address and
undefined-behaviour sanitizers: every value it writes must equal the oracle
restatement of VCFData::writeVCFImputedBunch (VCFData.cpp:3068-3446) on
random bunches with conflicts, missing typed calls, a ragged last warp,
haploid targets and the --overwriteCalls / --improveCalls / filter options
(with the --improveCalls run statistics)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from eimp_b200.bits import W, unpack_rows
from test_site_stats_oracle import random_case

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("stats_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "site_stats.cu")).read()
    # the launcher (triple-chevron launch) is device-only
    i, j = src.index("template <bool HAP>\nvoid launch_site_stats_t("), src.rindex("}  // namespace eimp")
    (d / "stats_emu.cpp").write_text('#include "emu.h"\n' + src[:i] + src[j:])
    exe = d / "stats_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-ffp-contract=off", "-fno-fast-math", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-I", EMU, "-I", str(d), os.path.join(EMU, "stats_main.cpp"), "-o",
           str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


@pytest.mark.parametrize("haploid", [False, True])
@pytest.mark.parametrize("overwrite,improve", [(False, False), (True, False), (False, True)])
def test_stats_kernel_emulated(emu_exe, tmp_path, overwrite, improve, haploid):
    from oracle import restate as R
    mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full = random_case(
        7, N=11, M=60, Mref=400, nsites=300, mref_begin=50)
    N, M = gt.shape
    hap = (np.arange(N) % 3 == 1).astype(np.uint8) if haploid else np.zeros(0, np.uint8)
    nsites = dos.shape[1]
    cnt = np.searchsorted(typed, np.arange(Mref), side="right")
    segm = np.maximum(cnt - 1, 0).astype(np.int32)
    common = np.zeros(Mref, np.uint8)
    common[typed] = 1
    params = np.array([N, mref_begin, nsites, bits.shape[1], nsites, phased.shape[1], M, M, Mref, int(overwrite),
                       int(improve)], np.int32)
    for name, a in [("params_i", params), ("params_f", np.array([0.3, 0.1], np.float32)), ("bits", bits),
                    ("dos", dos), ("phased", phased), ("pdm", pdm), ("pdp", pdp), ("gt", gt), ("segm", segm),
                    ("common", common), ("af", af_full), ("haptgt", hap)]:
        np.ascontiguousarray(a).tofile(tmp_path / f"{name}.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    rd = lambda n, dt: np.fromfile(tmp_path / n, dt)  # noqa: E731
    ref = R.site_stats(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full, overwrite, improve, 0.3,
                       0.1, want_ds=True, want_gp=True, haploid=hap if haploid else None)
    u32 = lambda a: np.ascontiguousarray(a, np.float32).view(np.uint32)  # noqa: E731
    np.testing.assert_array_equal(u32(rd("o_ads.bin", np.float32).reshape(2 * N, nsites)), u32(ref["ads"]))
    np.testing.assert_array_equal(unpack_rows(rd("o_gtbits.bin", np.uint64).reshape(2 * N, W(nsites)), nsites),
                                  unpack_rows(ref["gtbits"], nsites))
    np.testing.assert_array_equal(u32(rd("o_ds.bin", np.float32).reshape(N, nsites)), u32(ref["ds"]))
    np.testing.assert_array_equal(u32(rd("o_gp.bin", np.float32).reshape(3 * N, nsites)), u32(ref["gp"]))
    sf = rd("o_site_f.bin", np.float32).reshape(3, nsites)
    si = rd("o_site_i.bin", np.int32).reshape(2, nsites)
    for k, v in zip(("r2", "af", "maf"), sf):
        np.testing.assert_array_equal(v, ref[k], err_msg=k)
    np.testing.assert_array_equal(si[0], ref["ac"])
    np.testing.assert_array_equal(si[1], ref["an"])
    np.testing.assert_array_equal(rd("o_pass.bin", np.uint8), ref["passed"])
    assert int(rd("o_conf.bin", np.uint64)[0]) == ref["conflicts"]
    np.testing.assert_array_equal(rd("o_icnt.bin", np.uint64).astype(np.int64), ref["improve_counts"])
    np.testing.assert_allclose(rd("o_itot.bin", np.float64), ref["improve_totals"], rtol=1e-12, atol=0)
    if improve:
        assert ref["improve_counts"].sum() > 0
