/*
 * Stand-in for htslib's vcf.h, used ONLY to compile the reference's
 * VCFData.cpp into the writer harness of the test oracle
 * (oracle/_ref/libeimp_refwriter.so).  Test infrastructure written for this
 * project: it declares the names VCFData.cpp uses with the argument meaning
 * of htslib's public API, and keeps the values a record receives (FORMAT and
 * INFO fields, position, alleles) in plain containers inside bcf1_t, so that
 * the harness can read back what the reference's writer would have written.
 * Only the record calls of VCFData::writeVCFImputedBunch do work; every other
 * function is defined in writer_stubs.cpp and aborts if it is ever called.
 * The constants are htslib's published encodings (GT values, the float
 * missing/vector-end bit patterns).
 */
#ifndef EIMP_WRITER_STUB_VCF_H
#define EIMP_WRITER_STUB_VCF_H

#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

typedef struct kstring_t { size_t l, m; char *s; } kstring_t;

typedef struct hts_idx_t hts_idx_t;
enum htsExactFormat { unknown_format, vcf, bcf };
typedef struct htsFormat { int category; enum htsExactFormat format; } htsFormat;
typedef struct htsFile { int dummy; } htsFile;

typedef struct bcf_hdr_t {
    int nsamples_ori;
    char **samples;
} bcf_hdr_t;

typedef struct bcf_dec_t {
    char *id;
    char **allele;
} bcf_dec_t;

/* one record; the harness reads the recorded fields */
typedef struct bcf1_t {
    int64_t pos;
    int32_t rid;
    float qual;
    int n_allele;
    bcf_dec_t d;
    std::string rec_id, rec_alleles;
    std::map<std::string, std::vector<float>> info_f, fmt_f;
    std::map<std::string, std::vector<int32_t>> info_i, fmt_i;
    std::map<std::string, int> info_flag;
} bcf1_t;

typedef struct bcf_info_t { int key; } bcf_info_t;

#define BCF_DT_ID 0
#define BCF_DT_CTG 1
#define BCF_DT_SAMPLE 2
#define BCF_UN_STR 1
#define BCF_UN_FLT 2
#define BCF_UN_INFO 4
#define BCF_UN_SHR (BCF_UN_STR | BCF_UN_FLT | BCF_UN_INFO)
#define BCF_UN_FMT 8
#define BCF_UN_ALL (BCF_UN_SHR | BCF_UN_FMT)
#define BCF_HT_FLAG 0
#define BCF_HT_INT 1
#define BCF_HT_REAL 2
#define BCF_HT_STR 3

#define bcf_gt_phased(idx) ((((idx) + 1) << 1) | 1)
#define bcf_gt_unphased(idx) (((idx) + 1) << 1)
#define bcf_gt_missing 0
#define bcf_gt_is_missing(val) ((val) >> 1 ? 0 : 1)
#define bcf_gt_is_phased(idx) ((idx) & 1)
#define bcf_gt_allele(val) (((val) >> 1) - 1)
#define bcf_int32_vector_end (INT32_MIN + 1)
#define bcf_int32_missing INT32_MIN
#define bcf_float_missing 0x7F800001
#define bcf_float_vector_end 0x7F800002
static inline void bcf_float_set(float *ptr, uint32_t value) { std::memcpy(ptr, &value, 4); }
#define bcf_float_set_missing(x) bcf_float_set(&(x), bcf_float_missing)
#define bcf_float_set_vector_end(x) bcf_float_set(&(x), bcf_float_vector_end)
#define bcf_hdr_nsamples(hdr) ((hdr)->nsamples_ori)

bcf1_t *bcf_init1(void);
void bcf_destroy(bcf1_t *v);
bcf1_t *bcf_dup(bcf1_t *src);
int bcf_unpack(bcf1_t *b, int which);
int bcf_update_id(const bcf_hdr_t *hdr, bcf1_t *line, const char *id);
int bcf_update_alleles_str(const bcf_hdr_t *hdr, bcf1_t *line, const char *alleles_string);
int bcf_update_alleles(const bcf_hdr_t *hdr, bcf1_t *line, const char **alleles, int nals);
int bcf_update_info_float(const bcf_hdr_t *hdr, bcf1_t *line, const char *key, const float *values, int n);
int bcf_update_info_int32(const bcf_hdr_t *hdr, bcf1_t *line, const char *key, const int32_t *values, int n);
int bcf_update_info_flag(const bcf_hdr_t *hdr, bcf1_t *line, const char *key, const char *string, int n);
int bcf_update_format_float(const bcf_hdr_t *hdr, bcf1_t *line, const char *key, const float *values, int n);
int bcf_update_genotypes(const bcf_hdr_t *hdr, bcf1_t *line, const void *gts, int n);
int bcf_get_genotypes(const bcf_hdr_t *hdr, bcf1_t *line, void *dst, int *ndst);
int bcf_get_info_float(const bcf_hdr_t *hdr, bcf1_t *line, const char *tag, void *dst, int *ndst);
int bcf_add_filter(const bcf_hdr_t *hdr, bcf1_t *line, int flt_id);

bcf_hdr_t *bcf_hdr_init(const char *mode);
bcf_hdr_t *bcf_hdr_dup(const bcf_hdr_t *hdr);
void bcf_hdr_destroy(bcf_hdr_t *h);
bcf_hdr_t *bcf_hdr_read(htsFile *fp);
int bcf_hdr_write(htsFile *fp, bcf_hdr_t *h);
int bcf_hdr_append(bcf_hdr_t *h, const char *line);
int bcf_hdr_add_sample(bcf_hdr_t *hdr, const char *sample);
int bcf_hdr_sync(bcf_hdr_t *h);
int bcf_hdr_id2int(const bcf_hdr_t *hdr, int type, const char *id);
const char *bcf_hdr_id2name(const bcf_hdr_t *hdr, int rid);
int bcf_write(htsFile *fp, bcf_hdr_t *h, bcf1_t *v);
hts_idx_t *bcf_index_load(const char *fn);
const char **bcf_index_seqnames(const hts_idx_t *idx, const bcf_hdr_t *hdr, int *n);

htsFile *hts_open(const char *fn, const char *mode);
int hts_close(htsFile *fp);
int hts_set_threads(htsFile *fp, int n);
const htsFormat *hts_get_format(htsFile *fp);
const char *hts_version(void);
void hts_idx_destroy(hts_idx_t *idx);
int hts_idx_get_stat(const hts_idx_t *idx, int tid, uint64_t *mapped, uint64_t *unmapped);

#endif
