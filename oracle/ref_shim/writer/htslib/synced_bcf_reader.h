/*
 * Stand-in for htslib's synced_bcf_reader.h (and the tabix index calls that
 * header brings in), used ONLY to compile the reference's VCFData.cpp into
 * the writer harness of the test oracle.  Declarations only; the functions
 * are defined in writer_stubs.cpp and abort if called: the harness never
 * reads a file.
 */
#ifndef EIMP_WRITER_STUB_SYNCED_H
#define EIMP_WRITER_STUB_SYNCED_H

#include "vcf.h"

typedef struct bcf_srs_t { int errnum; } bcf_srs_t;
typedef struct tbx_t { hts_idx_t *idx; } tbx_t;

enum bcf_sr_opt_t { BCF_SR_REQUIRE_IDX, BCF_SR_PAIR_LOGIC };
#define BCF_SR_PAIR_SNPS 1
#define BCF_SR_PAIR_INDELS 2
#define BCF_SR_PAIR_ANY 4
#define BCF_SR_PAIR_SOME 8
#define BCF_SR_PAIR_SNP_REF 16
#define BCF_SR_PAIR_INDEL_REF 32
#define BCF_SR_PAIR_EXACT 64
#define BCF_SR_PAIR_BOTH (BCF_SR_PAIR_SNPS | BCF_SR_PAIR_INDELS)
#define BCF_SR_PAIR_BOTH_REF (BCF_SR_PAIR_SNPS | BCF_SR_PAIR_INDELS | BCF_SR_PAIR_SNP_REF | BCF_SR_PAIR_INDEL_REF)

bcf_srs_t *bcf_sr_init(void);
void bcf_sr_destroy(bcf_srs_t *readers);
int bcf_sr_set_opt(bcf_srs_t *readers, bcf_sr_opt_t opt, ...);
int bcf_sr_set_threads(bcf_srs_t *files, int n_threads);
int bcf_sr_set_regions(bcf_srs_t *readers, const char *regions, int is_file);
int bcf_sr_add_reader(bcf_srs_t *readers, const char *fname);
const char *bcf_sr_strerror(int errnum);
bcf_hdr_t *bcf_sr_get_header(bcf_srs_t *readers, int i);
bcf1_t *bcf_sr_get_line(bcf_srs_t *readers, int i);
int bcf_sr_next_line(bcf_srs_t *readers);

tbx_t *tbx_index_load(const char *fn);
const char **tbx_seqnames(tbx_t *tbx, int *n);
void tbx_destroy(tbx_t *tbx);

#endif
