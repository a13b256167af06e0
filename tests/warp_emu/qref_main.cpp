// Runs qref_decode_kernel (generated host copy of eimp_b200/csrc/qref_decode.cu)
// under the warp emulator, one variant (warp) at a time.
//
//   qref_emu <dir>
//
// <dir> holds params.bin (Mref, nwords as int64), section.bin (the haplotype
// section, exactly its bytes), offsets.bin (int64 per variant).  Outputs:
// o_rows.bin (Mref x nwords words), o_status.bin (the status word after each
// variant).  Every variant reads the section from its own copy of exactly
// the bytes up to the next multiple of 4 past the section end, and writes its
// own row allocation, so the address sanitizer sees an access past either.
// Exit status 3: a divergent warp collective.
#include "qref_emu.cpp"

#include <string>
#include <thread>
#include <vector>

thread_local dim3 threadIdx, blockIdx, blockDim;
thread_local EmuWarp *emu_warp;
thread_local EmuBarrier *emu_block;
thread_local uint8_t *emu_smem_ptr;
std::atomic<int> emu_divergence{0};

template <class T> static std::vector<T> rd(const std::string &d, const char *name) {
    const std::string p = d + "/" + name;
    FILE *f = fopen(p.c_str(), "rb");
    if (!f) { perror(p.c_str()); exit(1); }
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<T> v(n / sizeof(T));
    if (n && fread(v.data(), 1, n, f) != (size_t)n) exit(2);
    fclose(f);
    return v;
}
template <class T> static void wr(const std::string &d, const char *name, const std::vector<T> &v) {
    const std::string p = d + "/" + name;
    FILE *f = fopen(p.c_str(), "wb");
    if (!f) { perror(p.c_str()); exit(1); }
    fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s <dir>\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const auto par = rd<int64_t>(d, "params.bin");
    const int Mref = (int)par[0], nw = (int)par[1];
    const auto sec = rd<uint8_t>(d, "section.bin");
    const auto offs = rd<int64_t>(d, "offsets.bin");
    // the section padded to a multiple of 4 bytes: the decoder reads aligned 32-bit words
    const size_t padded = (sec.size() + 3) / 4 * 4 + 4;
    std::vector<uint64_t> rows((size_t)Mref * nw);
    std::vector<uint32_t> st(Mref);
    for (int v = 0; v < Mref; v++) {
        uint8_t *s = (uint8_t *)aligned_alloc(16, (padded + 15) / 16 * 16);
        memset(s, 0xA5, padded);
        memcpy(s, sec.data(), sec.size());
        uint64_t *row = (uint64_t *)malloc((size_t)nw * 8);
        memset(row, 0x5A, (size_t)nw * 8);   // the decoder must write every word
        uint32_t status = 0;
        EmuWarp warp;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; l++)
            lanes.emplace_back([&, l] {
                threadIdx.x = (v & 3) * 32 + l;
                blockIdx.x = v >> 2;
                blockDim.x = 128;
                emu_warp = &warp;
                // the row pointer as the kernel computes it for variant v: out + v*ldw
                eimp::qref_decode_kernel(s, offs.data(), Mref, nw, row - (size_t)v * nw, (size_t)nw, &status);
            });
        for (auto &x : lanes) x.join();
        memcpy(rows.data() + (size_t)v * nw, row, (size_t)nw * 8);
        st[v] = status;
        free(row);
        free(s);
    }
    wr(d, "o_rows.bin", rows);
    wr(d, "o_status.bin", st);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
