// Definitions behind the htslib stand-in headers for the writer harness of
// the test oracle (oracle/_ref/libeimp_refwriter.so).  Test infrastructure
// written for this project.  The record calls that
// VCFData::writeVCFImputedBunch makes (bcf_init1, bcf_update_*, bcf_destroy)
// store what they are given in the bcf1_t stand-in; every other htslib call
// of VCFData.cpp belongs to file reading and writing, which the harness never
// runs, so it aborts with its name.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>

#include "htslib/synced_bcf_reader.h"
#include "htslib/vcf.h"
#include "hybridsys/ThreadUtils.h"
#include "version.h"

const char *const prog_timestamp = "harness";
const char *const prog_version = "harness";
const char *const prog_bugaddress = "harness";

void ThreadUtils::setThreadName(const std::string &) {}
const unsigned long ThreadUtils::MAX_THREAD_NAME_LEN = 15;

namespace {
[[noreturn]] void unused(const char *name) {
    std::fprintf(stderr, "writer harness: %s is not available (file I/O is not part of the harness)\n", name);
    std::abort();
}
}  // namespace

bcf1_t *bcf_init1(void) { return new bcf1_t(); }
void bcf_destroy(bcf1_t *v) { delete v; }
int bcf_update_id(const bcf_hdr_t *, bcf1_t *line, const char *id) { line->rec_id = id ? id : ""; return 0; }
int bcf_update_alleles_str(const bcf_hdr_t *, bcf1_t *line, const char *s) { line->rec_alleles = s ? s : ""; return 0; }
int bcf_update_info_float(const bcf_hdr_t *, bcf1_t *line, const char *key, const float *v, int n) {
    line->info_f[key].assign(v, v + n);
    return 0;
}
int bcf_update_info_int32(const bcf_hdr_t *, bcf1_t *line, const char *key, const int32_t *v, int n) {
    line->info_i[key].assign(v, v + n);
    return 0;
}
int bcf_update_info_flag(const bcf_hdr_t *, bcf1_t *line, const char *key, const char *, int n) {
    line->info_flag[key] = n;
    return 0;
}
int bcf_update_format_float(const bcf_hdr_t *, bcf1_t *line, const char *key, const float *v, int n) {
    line->fmt_f[key].assign(v, v + n);
    return 0;
}
int bcf_update_genotypes(const bcf_hdr_t *, bcf1_t *line, const void *gts, int n) {
    const int32_t *g = static_cast<const int32_t *>(gts);
    line->fmt_i["GT"].assign(g, g + n);
    return 0;
}

bcf1_t *bcf_dup(bcf1_t *) { unused("bcf_dup"); }
int bcf_unpack(bcf1_t *, int) { unused("bcf_unpack"); }
int bcf_update_alleles(const bcf_hdr_t *, bcf1_t *, const char **, int) { unused("bcf_update_alleles"); }
int bcf_get_genotypes(const bcf_hdr_t *, bcf1_t *, void *, int *) { unused("bcf_get_genotypes"); }
int bcf_get_info_float(const bcf_hdr_t *, bcf1_t *, const char *, void *, int *) { unused("bcf_get_info_float"); }
int bcf_add_filter(const bcf_hdr_t *, bcf1_t *, int) { unused("bcf_add_filter"); }
bcf_hdr_t *bcf_hdr_init(const char *) { unused("bcf_hdr_init"); }
bcf_hdr_t *bcf_hdr_dup(const bcf_hdr_t *) { unused("bcf_hdr_dup"); }
void bcf_hdr_destroy(bcf_hdr_t *) { unused("bcf_hdr_destroy"); }
bcf_hdr_t *bcf_hdr_read(htsFile *) { unused("bcf_hdr_read"); }
int bcf_hdr_write(htsFile *, bcf_hdr_t *) { unused("bcf_hdr_write"); }
int bcf_hdr_append(bcf_hdr_t *, const char *) { unused("bcf_hdr_append"); }
int bcf_hdr_add_sample(bcf_hdr_t *, const char *) { unused("bcf_hdr_add_sample"); }
int bcf_hdr_sync(bcf_hdr_t *) { unused("bcf_hdr_sync"); }
int bcf_hdr_id2int(const bcf_hdr_t *, int, const char *) { unused("bcf_hdr_id2int"); }
const char *bcf_hdr_id2name(const bcf_hdr_t *, int) { unused("bcf_hdr_id2name"); }
int bcf_write(htsFile *, bcf_hdr_t *, bcf1_t *) { unused("bcf_write"); }
hts_idx_t *bcf_index_load(const char *) { unused("bcf_index_load"); }
const char **bcf_index_seqnames(const hts_idx_t *, const bcf_hdr_t *, int *) { unused("bcf_index_seqnames"); }
htsFile *hts_open(const char *, const char *) { unused("hts_open"); }
int hts_close(htsFile *) { unused("hts_close"); }
int hts_set_threads(htsFile *, int) { unused("hts_set_threads"); }
const htsFormat *hts_get_format(htsFile *) { unused("hts_get_format"); }
const char *hts_version(void) { unused("hts_version"); }
void hts_idx_destroy(hts_idx_t *) { unused("hts_idx_destroy"); }
int hts_idx_get_stat(const hts_idx_t *, int, uint64_t *, uint64_t *) { unused("hts_idx_get_stat"); }
bcf_srs_t *bcf_sr_init(void) { unused("bcf_sr_init"); }
void bcf_sr_destroy(bcf_srs_t *) { unused("bcf_sr_destroy"); }
int bcf_sr_set_opt(bcf_srs_t *, bcf_sr_opt_t, ...) { unused("bcf_sr_set_opt"); }
int bcf_sr_set_threads(bcf_srs_t *, int) { unused("bcf_sr_set_threads"); }
int bcf_sr_set_regions(bcf_srs_t *, const char *, int) { unused("bcf_sr_set_regions"); }
int bcf_sr_add_reader(bcf_srs_t *, const char *) { unused("bcf_sr_add_reader"); }
const char *bcf_sr_strerror(int) { unused("bcf_sr_strerror"); }
bcf_hdr_t *bcf_sr_get_header(bcf_srs_t *, int) { unused("bcf_sr_get_header"); }
bcf1_t *bcf_sr_get_line(bcf_srs_t *, int) { unused("bcf_sr_get_line"); }
int bcf_sr_next_line(bcf_srs_t *) { unused("bcf_sr_next_line"); }
tbx_t *tbx_index_load(const char *) { unused("tbx_index_load"); }
const char **tbx_seqnames(tbx_t *, int *) { unused("tbx_seqnames"); }
void tbx_destroy(tbx_t *) { unused("tbx_destroy"); }
