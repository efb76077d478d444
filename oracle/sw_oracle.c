/*
 * Smith-Waterman oracle: a scalar C restatement of the reference's read-to-haplotype aligner, test
 * infrastructure only (tests/, smoke() and the bench's CPU-baseline leg use it as the checker).
 *
 * It follows src/haplotypecaller/common/base/lib/ro_sw in the reference:
 *   ro_sw.c:26-40       which kernel runs: int32 when the read has fewer than 16 bases, match <= 0, or
 *                       min(lengths) x match > INT16_MAX; int16 otherwise
 *   sw_internal.h:19-22 low init (INT32_MIN/2, INT16_MIN/2) and cutoff (-1e8, INT16_MIN/4)
 *   sw_core_template.h:153-348
 *                       E = max(H(i,j-1)+open, E(i,j-1)+ext), F = max(F(i-1,j)+ext, H(i-1,j)+open),
 *                       H = max(cutoff, H(i-1,j-1)+(equal ? match : mismatch)); E wins over H only when
 *                       strictly greater (state insertion), then F likewise (state deletion); the
 *                       extension flags (4, 8) are set when the open score is not greater than the
 *                       extension score.  In the int16 kernel every add wraps in 16 bits.  H(0,j) =
 *                       H(i,0) = 0, E(i,0) = F(0,j) = low.  The best end cell is scanned over the last
 *                       row and last column in anti-diagonal order with the two tie rules below
 *   sw_core_template.h:354-365   inputs of 2048 bases or more: alignment_offset = 1, nothing else
 *   sw_cigar.c:22-171   trace-back with soft clips and extension states, run merge, reversal into BAM
 *                       CIGAR ops, at most cigar_max_len - 1 = 2047 ops
 * The reference walks anti-diagonals with vectors; this restatement fills the matrix row by row, which
 * gives the same cell values because every cell depends only on its left, upper and diagonal neighbours.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SW_MAX_SEQ 2048
#define ST_INS 1
#define ST_DEL 2
#define ST_INS_EXT 4
#define ST_DEL_EXT 8
#define ST_CLIP 9
#define OP_M 0
#define OP_I 1
#define OP_D 2
#define OP_S 4

/* ro_sw_should_use_int32_avx512 (ro_sw.c:26-40) */
int sw_oracle_uses_int32(int hap_len, int read_len, int match)
{
    if (read_len < 16 || match <= 0) return 1;
    int m = hap_len < read_len ? hap_len : read_len;
    return (long long)m * match > 32767;
}

static inline int32_t add16(int32_t a, int32_t b) { return (int16_t)(uint16_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t add32(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

/* variant: 0 = as the reference picks, 1 = int32, 2 = int16.  params = {match, mismatch, open, extend}.
 * Returns the number of CIGAR ops (BAM: length << 4 | op), of which the first min(n, cap) are written. */
int sw_oracle_align(const uint8_t* hap, int nrow, const uint8_t* read, int ncol, const int32_t* params, int variant,
                    int32_t* score_out, int32_t* offset_out, int32_t* max_i_out, int32_t* max_j_out, uint32_t* cigar,
                    int cap)
{
    *score_out = 0;
    *offset_out = 0;
    *max_i_out = 0;
    *max_j_out = 0;
    if ((nrow > ncol ? nrow : ncol) >= SW_MAX_SEQ) {
        *offset_out = 1;
        return 0;
    }
    int w16 = variant == 2 || (variant == 0 && !sw_oracle_uses_int32(nrow, ncol, params[0]));
    int32_t (*add)(int32_t, int32_t) = w16 ? add16 : add32;
    int32_t match = w16 ? (int16_t)params[0] : params[0];
    int32_t mismatch = w16 ? (int16_t)params[1] : params[1];
    int32_t open = w16 ? (int16_t)params[2] : params[2];
    int32_t ext = w16 ? (int16_t)params[3] : params[3];
    int32_t low = w16 ? -16384 : (INT32_MIN / 2);
    int32_t cutoff = w16 ? -8192 : -100000000;

    size_t w = (size_t)ncol + 1;
    int32_t* H = (int32_t*)malloc(sizeof(int32_t) * w * (size_t)(nrow + 1));
    int32_t* F = (int32_t*)malloc(sizeof(int32_t) * w);
    uint8_t* bt = (uint8_t*)calloc(w * (size_t)(nrow + 1), 1);
    int32_t* runs = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)(nrow + ncol + 4));
    if (!H || !F || !bt || !runs) {
        free(H); free(F); free(bt); free(runs);
        return -1;
    }
    for (int j = 0; j <= ncol; ++j) {
        H[j] = 0;
        F[j] = low;
    }
    for (int i = 1; i <= nrow; ++i) {
        int32_t* Hi = H + (size_t)i * w;
        const int32_t* Hu = Hi - w;
        Hi[0] = 0;
        int32_t E = low;
        for (int j = 1; j <= ncol; ++j) {
            int32_t eo = add(Hi[j - 1], open), ee = add(E, ext);
            E = eo > ee ? eo : ee;
            int code = eo > ee ? 0 : ST_INS_EXT;
            int32_t fe = add(F[j], ext), fo = add(Hu[j], open);
            F[j] = fe > fo ? fe : fo;
            code |= fo > fe ? 0 : ST_DEL_EXT;
            int32_t h = add(Hu[j - 1], hap[i - 1] == read[j - 1] ? match : mismatch);
            if (h < cutoff) h = cutoff;
            int st = 0;
            if (E > h) { st = ST_INS; h = E; }
            if (F[j] > h) { st = ST_DEL; h = F[j]; }
            Hi[j] = h;
            bt[(size_t)i * w + j] = (uint8_t)(st | code);
        }
    }

    /* best end cell: anti-diagonal a = 1 .. nrow + ncol; the last-row cell (nrow, a - nrow) first, then
     * the last-column cell (a - ncol, ncol) (sw_core_template.h:332-347) */
    int32_t best = w16 ? INT16_MIN : INT32_MIN;
    int mi = 0, mj = 0;
    for (int a = 1; a <= nrow + ncol; ++a) {
        if (a >= nrow + 1) {
            int i = nrow, j = a - nrow;
            int32_t s = H[(size_t)i * w + j];
            if (best < s || (best == s && abs(i - j) < abs(mi - mj))) { best = s; mi = i; mj = j; }
        }
        if (a >= ncol + 1) {
            int i = a - ncol, j = ncol;
            int32_t s = H[(size_t)i * w + j];
            if (best < s || (best == s && (mj == ncol || abs(i - j) <= abs(mi - mj)))) { best = s; mi = i; mj = j; }
        }
    }
    *score_out = best;
    *max_i_out = mi;
    *max_j_out = mj;

    /* trace-back (sw_cigar.c:36-146): runs of (state, length) in trace order, merged as they come */
    int nr = 0, i = mi, j = mj;
#define PUSH(stv, len) do { if (nr > 0 && runs[2 * nr - 2] == (stv)) runs[2 * nr - 1] += (len); \
                            else { runs[2 * nr] = (stv); runs[2 * nr + 1] = (len); ++nr; } } while (0)
    if (j < ncol) PUSH(ST_CLIP, ncol - j);
    int state = 0;
    while (i > 0 && j > 0) {
        int b = bt[(size_t)i * w + j];
        if (state == ST_INS_EXT) {
            --j;
            runs[2 * nr - 1] += 1;
            state = b & ST_INS_EXT;
        } else if (state == ST_DEL_EXT) {
            --i;
            runs[2 * nr - 1] += 1;
            state = b & ST_DEL_EXT;
        } else if ((b & 3) == 0) {
            --i; --j;
            PUSH(0, 1);
            state = 0;
        } else if ((b & 3) == ST_INS) {
            --j;
            PUSH(ST_INS, 1);
            state = b & ST_INS_EXT;
        } else {
            --i;
            PUSH(ST_DEL, 1);
            state = b & ST_DEL_EXT;
        }
    }
    if (j > 0) PUSH(ST_CLIP, j);
#undef PUSH
    *offset_out = i;

    /* read order, lengths > 0, at most SW_MAX_SEQ - 1 ops (sw_cigar.c:162-170) */
    int n = 0;
    for (int r = nr - 1; r >= 0; --r) {
        if (runs[2 * r + 1] <= 0 || n + 1 >= SW_MAX_SEQ) continue;
        int st = runs[2 * r];
        int op = st == 0 ? OP_M : st == ST_INS ? OP_I : st == ST_DEL ? OP_D : OP_S;
        if (n < cap) cigar[n] = ((uint32_t)runs[2 * r + 1] << 4) | (uint32_t)op;
        ++n;
    }
    free(H); free(F); free(bt); free(runs);
    return n;
}
