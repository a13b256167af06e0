"""The Qref decode kernel (eimp_b200/csrc/qref_decode.cu) run on the CPU under
the host warp emulator with the address and undefined-behaviour sanitizers,
and the host index of a section (eimp_qref_index): every decoded row and
every truncation flag must equal the oracle restatement of
VCFData::qRefLoadNextVariant / runlengthDecode (VCFData.cpp:2378-2535,
utils.h:194-) on a section that mixes raw vectors at every byte alignment,
run-length codes with runs past the 32767 limit, the worked example of
qref_spec.md:144-172 and malformed codes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from eimp_b200.bits import W
from test_qref_oracle import SPEC_BYTES

CSRC = os.path.join(ROOT, "eimp_b200", "csrc")
EMU = os.path.join(ROOT, "tests", "warp_emu")


def variant(enc=None, raw=None):
    if raw is not None:
        return np.concatenate([np.zeros(8, np.uint8), raw.view(np.uint8)])
    return np.concatenate([np.array([len(enc)], np.uint64).view(np.uint8), np.asarray(enc, np.uint8)])


def mixed_section(nhaps=2 * 1500, seed=5):
    """Variants: random densities (raw where run-length coding is not
    shorter), odd-length codes shifting the next raw vector to every byte
    alignment, long runs of ones, the spec example padded out, and malformed
    codes: a two-byte run length cut after its first byte, runs that stop
    inside a word, runs that run past the row, a trailing short run after
    word-aligned runs."""
    from oracle import restate as R
    rng = np.random.default_rng(seed)
    nw = W(nhaps)
    vs = []
    for k in range(40):
        bits = np.zeros(nw * 64, np.uint8)
        dens = [0.0, 0.0005, 0.01, 0.2, 0.5][k % 5]
        bits[:nhaps] = rng.random(nhaps) < dens
        if k % 7 == 3:
            a = int(rng.integers(0, nhaps // 2))
            bits[a:nhaps] = 1
        row = np.packbits(bits, bitorder="little").view(np.uint64)
        enc = R.rle_encode(row)
        vs.append(variant(raw=row) if enc is None else variant(enc=enc))
        if k % 2 == 1:   # one run of ones: a 3- to 6-byte code shifts the next vector's byte alignment
            one = np.zeros(nw * 64, np.uint8)
            a = int(rng.integers(0, 300))
            one[a:a + int(rng.integers(1, 300))] = 1
            vs.append(variant(enc=R.rle_encode(np.packbits(one, bitorder="little").view(np.uint64))))
    vs.append(variant(enc=SPEC_BYTES))                      # runs past the row end, ending inside a word
    vs.append(variant(enc=[0x85]))                          # cut two-byte run length
    vs.append(variant(enc=[0x0a, 0x03]))                    # stops inside the first word
    vs.append(variant(enc=[0x80, 0x02] * 40))               # 256-bit runs, far past the row
    vs.append(variant(enc=[0xc0, 0x00] * (nw // 2) + [0x00, 0x05]))   # word-aligned runs, then a trailing short run
    return np.concatenate(vs), len(vs), nw


def oracle_rows(section, Mref, nw, offsets):
    from oracle import restate as R
    rows = np.zeros((Mref, nw), np.uint64)
    bad = np.zeros(Mref, bool)
    for v in range(Mref):
        o = int(offsets[v])
        es = int(section[o:o + 8].view(np.uint64)[0])
        if es == 0:
            rows[v] = section[o + 8:o + 8 + nw * 8].view(np.uint64)
        else:
            rows[v], rc = R.rle_decode(section[o + 8:o + 8 + es], nw)
            bad[v] = rc != 0
    return rows, bad


def host_index(section, Mref, nhaps):
    from eimp_b200 import _lib
    L = _lib.load()
    offs = np.zeros(Mref, np.int64)
    s = np.ascontiguousarray(section)
    rc = L.eimp_qref_index(s.ctypes.data, s.size, Mref, nhaps // 2, offs.ctypes.data)
    return rc, offs


@pytest.fixture(scope="module")
def emu_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("qref_emu")
    shutil.copy(os.path.join(CSRC, "common.cuh"), d / "common.cuh")
    shutil.copy(os.path.join(CSRC, "kernels.h"), d / "kernels.h")
    src = open(os.path.join(CSRC, "qref_decode.cu")).read()
    # the kernels only: everything from the first host launcher to the namespace's end is cut
    i, j = src.index("cudaError_t launch_qref_"), src.rindex("}  // namespace eimp")
    (d / "qref_emu.cpp").write_text('#include "emu.h"\n' + src[:i] + src[j:])
    exe = d / "qref_emu"
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", EMU, "-I", str(d), os.path.join(EMU, "qref_main.cpp"), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return str(exe)


def test_host_index():
    from oracle import restate as R
    sec, Mref, nw = mixed_section()
    rc, offs = host_index(sec, Mref, 2 * 1500)
    assert rc == 0
    o = 0
    for v in range(Mref):
        assert offs[v] == o
        es = int(sec[o:o + 8].view(np.uint64)[0])
        o += 8 + (es if es else nw * 8)
    assert o == sec.size
    assert host_index(sec[:-1], Mref, 2 * 1500)[0] != 0   # the last variant cut short
    head = sec[:offs[10]]   # the first 10 variants, all well-formed
    assert R.qref_decode(head, 10, nw)[1] == 0
    assert R.qref_decode(head[:-1], 10, nw)[1] == -2


def test_qref_kernel_emulated(emu_exe, tmp_path):
    sec, Mref, nw = mixed_section()
    rc, offs = host_index(sec, Mref, 2 * 1500)
    assert rc == 0
    np.array([Mref, nw], np.int64).tofile(tmp_path / "params.bin")
    sec.tofile(tmp_path / "section.bin")
    offs.tofile(tmp_path / "offsets.bin")
    r = subprocess.run([emu_exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"rc {r.returncode}: {r.stderr[-4000:]}"
    rows = np.fromfile(tmp_path / "o_rows.bin", np.uint64).reshape(Mref, nw)
    st = np.fromfile(tmp_path / "o_status.bin", np.uint32)
    want, bad = oracle_rows(sec, Mref, nw, offs)
    assert bad.sum() >= 3 and (~bad).sum() >= 40
    np.testing.assert_array_equal(st != 0, bad)
    np.testing.assert_array_equal(rows[~bad], want[~bad])
    aligns = {int(o + 8) % 4 for o, v in zip(offs, range(Mref)) if int(sec[o:o + 8].view(np.uint64)[0]) == 0}
    assert aligns == {0, 1, 2, 3}   # raw vectors at every byte alignment
