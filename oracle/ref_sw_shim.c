/*
 * Test-infrastructure shim over the reference's own Smith-Waterman aligner (compiled from the
 * reference sources by oracle/build_ref_sw.sh): one call aligns a read to a haplotype the way
 * AlignmentUtils::create_read_aligned_to_ref does (genotyping/alignment_utils.cpp:574-579: seq1 =
 * haplotype, seq2 = read, the context sw_avx_init(false) sets up, its avx_function), and returns
 * what the caller reads back: score, alignment offset, CIGAR.  Only the checker uses it.
 */
#include <stdint.h>
#include <string.h>

#include "ro_sw.h"
#include "smithwaterman_common.h"

/* variant: 0 = the context's own function (ro_sw_avx512_run on AVX-512 hosts), 1 = int32 kernel,
 * 2 = int16 kernel, 3 = the older sw_avx512_run.  params may be NULL (genotyping parameters), else
 * {match, mismatch, gap_open, gap_extend}.  Returns the CIGAR op count written (<= cigar_cap). */
int ref_sw_align(const uint8_t* hap, int hap_len, const uint8_t* read, int read_len, const int32_t* params, int variant,
                 int32_t* score, int32_t* offset, int32_t* max_i, int32_t* max_j, uint32_t* cigar, int cigar_cap)
{
    static __thread p_lib_sw_avx ctx = 0;
    if (!ctx) ctx = sw_avx_init(0);
    if (!ctx) return -1;
    memcpy(ctx->seq1, hap, (size_t)hap_len);
    memcpy(ctx->seq2, read, (size_t)read_len);
    ctx->len1 = (int16_t)hap_len;
    ctx->len2 = (int16_t)read_len;
    if (params) {
        ctx->para.match = params[0];
        ctx->para.mismatch = params[1];
        ctx->para.gap_open = params[2];
        ctx->para.gap_extend = params[3];
    } else {
        ctx->para.match = 10;
        ctx->para.mismatch = -15;
        ctx->para.gap_open = -30;
        ctx->para.gap_extend = -5;
    }
    /* a cleared first run entry, as test_ro_sw.c:114-117 clears the context before each case: with an
     * empty read the trace-back pushes no run and would otherwise emit the previous call's first run */
    ctx->mm_aloc.cigar_buf[0] = 0;
    ctx->mm_aloc.cigar_buf[1] = 0;
    ctx->cigar_count = 0;
    ctx->score = 0;
    ctx->max_i = 0;
    ctx->max_j = 0;
    ctx->alignment_offset = 0;
    switch (variant) {
    case 1: ro_sw_avx512_run_int32(ctx); break;
    case 2: ro_sw_avx512_run_int16(ctx); break;
    case 3: sw_avx512_run(ctx); break;
    default: ctx->avx_function(ctx); break;
    }
    *score = ctx->score;
    *offset = ctx->alignment_offset;
    *max_i = ctx->max_i;
    *max_j = ctx->max_j;
    int n = (int)ctx->cigar_count;
    if (n > cigar_cap) n = cigar_cap;
    for (int k = 0; k < n; ++k) cigar[k] = ctx->cigar[k];
    return n;
}

/* ro_sw_should_use_int32_avx512: which kernel the context's function picks. */
int ref_sw_uses_int32(int hap_len, int read_len, int match)
{
    lib_sw_avx p;
    memset(&p, 0, sizeof(p));
    p.len1 = (int16_t)hap_len;
    p.len2 = (int16_t)read_len;
    p.para.match = match;
    return ro_sw_should_use_int32_avx512(&p);
}
