/*
 * PairHMM oracle: a scalar CPU restatement of the reference's PairHMM arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it (as oracle/_build/libphmm_oracle.so) to check the CUDA engine; the product never links it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares every function here with the
 * reference's own kernels built from source by oracle/build_ref.sh (bit-exact raw sums) and with
 * the reference's 104 golden vectors (src/haplotypecaller/pairhmm/resource/pairhmm-testdata.txt,
 * frozen into tests/golden/).
 *
 * What it restates (paths inside the reference project):
 *   probability tables        src/haplotypecaller/pairhmm/roDV_common/context.h:33-189
 *   base-class table           src/haplotypecaller/pairhmm/roDV_common/common.h:42-55
 *   inter per-row tables       src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:59-101
 *   inter cell update          src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:165-195,277-319
 *   inter boundary and sum     src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:230-273
 *   intra tables / prior       src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:88-112,149-156
 *   intra N handling           src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:13-44
 *   intra cell update          src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:235-280
 *   FP32 -> FP64 switch        src/haplotypecaller/pairhmm/roDV_intra/pairhmm_api.cpp:14-23,
 *                              src/haplotypecaller/pairhmm/roDV_schedule.cpp:35,269-279
 *   vector-API scheduler       src/haplotypecaller/pairhmm/roDV_schedule.cpp:87-152,154-361
 *
 * The recurrence (row i = read position 1..R, column j = haplotype position 1..H):
 *   M[i][j] = prior(i,j) * (mm_i*M[i-1][j-1] + gapm_i*I[i-1][j-1] + gapm_i*D[i-1][j-1])
 *   I[i][j] = mx_i*M[i-1][j] + xx_i*I[i-1][j]
 *   D[i][j] = my_i*M[i][j-1] + yy_i*D[i][j-1]
 *   M[0][*] = I[0][*] = 0, D[0][j] = C/H (j = 0..H), M = I = D = 0 at column 0 for i >= 1
 *   result  = log10(sum_j M[R][j] + sum_j I[R][j]) - log10(C)
 * with C = 2^120 in FP32 and 2^1020 in FP64.
 *
 * Arithmetic order matters for bit-exactness: the reference's AVX-512 objects are compiled with
 * GCC, whose -mavx512f makes FMA available and whose AVX-512 intrinsics are plain vector
 * arithmetic, so GCC contracts some multiply-adds into FMAs; its AVX2 objects (no -mfma) contract
 * none.  ORACLE_FUSED selects the AVX-512 contraction, ORACLE_UNFUSED plain multiply/add.  The
 * contraction found in the AVX-512 objects (matched bit for bit against oracle/_ref):
 *   inter  s = fma(Ddiag, gapm, fma(Mdiag, mm, Idiag*gapm))
 *   intra  s = fma(Ddiag, gapm, fma(Idiag, gapm, Mdiag*mm))
 *   both   I = fma(Iup, xx, Mup*mx)      D = fma(Dleft, yy, Mleft*my)      M = s * prior
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAX_QUAL 254
#define JAC_TOL 8.0
#define JAC_STEP 0.0001
#define JAC_SIZE 80001 /* (int)(JAC_TOL / JAC_STEP) + 1, context.h:15 */
#define MM_SIZE (((MAX_QUAL + 1) * (MAX_QUAL + 2)) >> 1)

enum { ORACLE_UNFUSED = 0, ORACLE_FUSED = 1 };
enum { ORACLE_INTER = 0, ORACLE_INTRA = 1 };

static float ph2pr_f[128];
static double ph2pr_d[128];
static float jac_f[JAC_SIZE];
static double jac_d[JAC_SIZE];
static float mm_f[MM_SIZE];
static double mm_d[MM_SIZE];
static int tables_ready = 0;

/* context.h:61-82 in float */
static int fast_round_f(float d) { return (d > 0.0f) ? (int)(d + 0.5f) : (int)(d - 0.5f); }
static int fast_round_d(double d) { return (d > 0.0) ? (int)(d + 0.5) : (int)(d - 0.5); }

static float approx_log10_sum_f(float small, float big)
{
    if (small > big) {
        float t = big;
        big = small;
        small = t;
    }
    if (isinf(small) || isinf(big)) return big;
    float diff = big - small;
    if (diff >= (float)JAC_TOL) return big;
    int ind = fast_round_f((float)(diff * (float)(1.0 / JAC_STEP)));
    return big + jac_f[ind];
}

static double approx_log10_sum_d(double small, double big)
{
    if (small > big) {
        double t = big;
        big = small;
        small = t;
    }
    if (isinf(small) || isinf(big)) return big;
    double diff = big - small;
    if (diff >= JAC_TOL) return big;
    int ind = fast_round_d(diff * (1.0 / JAC_STEP));
    return big + jac_d[ind];
}

void oracle_init(void)
{
    if (tables_ready) return;
    for (int k = 0; k < JAC_SIZE; k++) {
        double v = log10(1.0 + pow(10.0, -((double)k) * JAC_STEP));
        jac_f[k] = (float)v;
        jac_d[k] = v;
    }
    const double inv_ln10 = 1.0 / log(10);
    for (int i = 0, off = 0; i <= MAX_QUAL; off += ++i) {
        for (int j = 0; j <= i; j++) {
            /* context.h:50-60: the log10-sum runs in the context's own type */
            float sf = approx_log10_sum_f((float)(-0.1 * i), (float)(-0.1 * j));
            double lf = log1p(-fmin(1.0, pow(10.0, (double)sf))) * inv_ln10;
            mm_f[off + j] = (float)pow(10.0, lf);
            double sd = approx_log10_sum_d(-0.1 * i, -0.1 * j);
            double ld = log1p(-fmin(1.0, pow(10.0, sd))) * inv_ln10;
            mm_d[off + j] = pow(10.0, ld);
        }
    }
    for (int x = 0; x < 128; x++) {
        ph2pr_f[x] = powf(10.f, -((float)x) / 10.f);
        ph2pr_d[x] = pow(10.0, -((double)x) / 10.0);
    }
    tables_ready = 1;
}

static int mm_index(int iq, int dq)
{
    int mn = dq, mx = iq;
    if (iq <= dq) {
        mn = iq;
        mx = dq;
    }
    return ((mx * (mx + 1)) >> 1) + mn;
}

/* Table accessors so the Python side can compare the CUDA engine's tables too. */
float oracle_ph2pr_f32(int q) { oracle_init(); return ph2pr_f[q & 127]; }
double oracle_ph2pr_f64(int q) { oracle_init(); return ph2pr_d[q & 127]; }
float oracle_mm_f32(int iq, int dq) { oracle_init(); return mm_f[mm_index(iq & 127, dq & 127)]; }
double oracle_mm_f64(int iq, int dq) { oracle_init(); return mm_d[mm_index(iq & 127, dq & 127)]; }

/* common.h:42-55: A=0 C=1 T=2 G=3 N=4; other letters in 'A'..'T' are 0 (zero-initialised
 * table).  Bytes outside 'A'..'T' index out of the reference's table; they are class 0 here. */
static int base_class(uint8_t b)
{
    switch (b) {
    case 'A': return 0;
    case 'C': return 1;
    case 'T': return 2;
    case 'G': return 3;
    case 'N': return 4;
    default: return 0;
    }
}

static int is_match(int kernel, uint8_t r, uint8_t h)
{
    if (kernel == ORACLE_INTER) return r == h; /* pairhmm_inter.cpp:166-168: raw byte compare */
    int cr = base_class(r), ch = base_class(h);
    return cr == ch || cr == 4 || ch == 4; /* pairhmm_impl.cpp:26-42: N matches everything */
}

/* ---------------------------------------------------------------------------------------------
 * FP32: raw scaled sum, in the reference's arithmetic order.
 * ------------------------------------------------------------------------------------------- */
#define MUL_F(a, b) ((float)((float)(a) * (float)(b)))
#define ADD_F(a, b) ((float)((float)(a) + (float)(b)))

/* flush-to-zero of results, as the reference runs with MXCSR.FTZ set (common.h:58-62) */
static inline float ftz_f(float x) { return (fabsf(x) < 1.17549435e-38f) ? 0.0f * x : x; }
static inline double ftz_d(double x) { return (fabs(x) < 2.2250738585072014e-308) ? 0.0 * x : x; }

float oracle_raw_f32(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                     const uint8_t* iq, const uint8_t* dq, const uint8_t* cq, int kernel, int fused)
{
    oracle_init();
    if (hl == 0 || rl == 0) return 0.0f;
    const float one_third = 1.0f / 3.0f;
    float* Mr = (float*)calloc(hl + 1, sizeof(float));
    float* Ir = (float*)calloc(hl + 1, sizeof(float));
    float* Dr = (float*)calloc(hl + 1, sizeof(float));
    const float init_d = ldexpf(1.f, 120) / (float)hl;
    for (uint32_t j = 0; j <= hl; j++) Dr[j] = init_d;
    /* Mr/Ir/Dr[j] hold row i-1 at column j+1 (0-based j), like pairhmm_inter.cpp:151,187-194 */
    for (uint32_t i = 0; i < rl; i++) {
        const int qi = q[i] & 127, ii = iq[i] & 127, di = dq[i] & 127, ci = cq[i] & 127;
        const float dist = ph2pr_f[qi];
        const float pmis = (kernel == ORACLE_INTER) ? MUL_F(dist, one_third) : dist / 3.0f;
        const float pmat = 1.0f - dist;
        const float gapm = 1.0f - ph2pr_f[ci];
        const float mm = mm_f[mm_index(ii, di)];
        const float mx = ph2pr_f[ii], xx = ph2pr_f[ci], my = ph2pr_f[di], yy = ph2pr_f[ci];
        float Mdiag = 0.f, Idiag = 0.f, Ddiag = (i == 0) ? init_d : 0.f; /* column 0 */
        float Mleft = 0.f, Dleft = 0.f;
        for (uint32_t j = 0; j < hl; j++) {
            const float Mup = Mr[j], Iup = Ir[j], Dup = Dr[j];
            const float prior = is_match(kernel, rd[i], hap[j]) ? pmat : pmis;
            float s, M, I, D;
            if (fused) {
                if (kernel == ORACLE_INTER)
                    s = ftz_f(fmaf(Mdiag, mm, ftz_f(MUL_F(Idiag, gapm))));
                else
                    s = ftz_f(fmaf(Idiag, gapm, ftz_f(MUL_F(Mdiag, mm))));
                s = ftz_f(fmaf(Ddiag, gapm, s));
                I = ftz_f(fmaf(Iup, xx, ftz_f(MUL_F(Mup, mx))));
                D = ftz_f(fmaf(Dleft, yy, ftz_f(MUL_F(Mleft, my))));
            } else {
                s = ftz_f(ADD_F(ftz_f(ADD_F(ftz_f(MUL_F(Mdiag, mm)), ftz_f(MUL_F(Idiag, gapm)))), ftz_f(MUL_F(Ddiag, gapm))));
                I = ftz_f(ADD_F(ftz_f(MUL_F(Mup, mx)), ftz_f(MUL_F(Iup, xx))));
                D = ftz_f(ADD_F(ftz_f(MUL_F(Mleft, my)), ftz_f(MUL_F(Dleft, yy))));
            }
            M = ftz_f(MUL_F(s, prior));
            Mdiag = Mup;
            Idiag = Iup;
            Ddiag = Dup;
            Mleft = M;
            Dleft = D;
            Mr[j] = M;
            Ir[j] = I;
            Dr[j] = D;
        }
    }
    float sm = 0.f, si = 0.f;
    for (uint32_t j = 0; j < hl; j++) {
        sm = ftz_f(ADD_F(sm, Mr[j]));
        si = ftz_f(ADD_F(si, Ir[j]));
    }
    free(Mr);
    free(Ir);
    free(Dr);
    return ftz_f(ADD_F(sm, si));
}

/* ---------------------------------------------------------------------------------------------
 * FP64: same recurrence in double with C = 2^1020.  With fused = ORACLE_UNFUSED and the inter prior
 * this is the plain all-FP64 oracle; ORACLE_FUSED reproduces the AVX-512 build's FP64 bits.
 * ------------------------------------------------------------------------------------------- */
double oracle_raw_f64(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                      const uint8_t* iq, const uint8_t* dq, const uint8_t* cq, int kernel, int fused)
{
    oracle_init();
    if (hl == 0 || rl == 0) return 0.0;
    const double one_third = 1.0 / 3.0;
    double* Mr = (double*)calloc(hl + 1, sizeof(double));
    double* Ir = (double*)calloc(hl + 1, sizeof(double));
    double* Dr = (double*)calloc(hl + 1, sizeof(double));
    const double init_d = ldexp(1.0, 1020) / (double)hl;
    for (uint32_t j = 0; j <= hl; j++) Dr[j] = init_d;
    for (uint32_t i = 0; i < rl; i++) {
        const int qi = q[i] & 127, ii = iq[i] & 127, di = dq[i] & 127, ci = cq[i] & 127;
        const double dist = ph2pr_d[qi];
        const double pmis = (kernel == ORACLE_INTER) ? dist * one_third : dist / 3.0;
        const double pmat = 1.0 - dist;
        const double gapm = 1.0 - ph2pr_d[ci];
        const double mm = mm_d[mm_index(ii, di)];
        const double mx = ph2pr_d[ii], xx = ph2pr_d[ci], my = ph2pr_d[di], yy = ph2pr_d[ci];
        double Mdiag = 0., Idiag = 0., Ddiag = (i == 0) ? init_d : 0.;
        double Mleft = 0., Dleft = 0.;
        for (uint32_t j = 0; j < hl; j++) {
            const double Mup = Mr[j], Iup = Ir[j], Dup = Dr[j];
            const double prior = is_match(kernel, rd[i], hap[j]) ? pmat : pmis;
            double s, I, D;
            if (fused) {
                if (kernel == ORACLE_INTER)
                    s = ftz_d(fma(Mdiag, mm, ftz_d(Idiag * gapm)));
                else
                    s = ftz_d(fma(Idiag, gapm, ftz_d(Mdiag * mm)));
                s = ftz_d(fma(Ddiag, gapm, s));
                I = ftz_d(fma(Iup, xx, ftz_d(Mup * mx)));
                D = ftz_d(fma(Dleft, yy, ftz_d(Mleft * my)));
            } else {
                s = ftz_d(ftz_d(ftz_d(Mdiag * mm) + ftz_d(Idiag * gapm)) + ftz_d(Ddiag * gapm));
                I = ftz_d(ftz_d(Mup * mx) + ftz_d(Iup * xx));
                D = ftz_d(ftz_d(Mleft * my) + ftz_d(Dleft * yy));
            }
            const double M = ftz_d(s * prior);
            Mdiag = Mup;
            Idiag = Iup;
            Ddiag = Dup;
            Mleft = M;
            Dleft = D;
            Mr[j] = M;
            Ir[j] = I;
            Dr[j] = D;
        }
    }
    double sm = 0., si = 0.;
    for (uint32_t j = 0; j < hl; j++) {
        sm = ftz_d(sm + Mr[j]);
        si = ftz_d(si + Ir[j]);
    }
    free(Mr);
    free(Ir);
    free(Dr);
    return ftz_d(sm + si);
}

static const float LOG10_C_F = 36.1236000061f;               /* adapter.h:25 */
static const double LOG10_C_D = 307.050595577260822;        /* adapter.h:26 */
static const float MIN_ACCEPTED = 1e-28f;                   /* roDV_schedule.cpp:35 */

/* log10 of an FP32 raw sum as the inter path reports it (pairhmm_inter_api.h:10-12). */
double oracle_log10_from_f32(float raw) { return log10((double)raw) - (double)LOG10_C_F; }
double oracle_log10_from_f64(double raw) { return log10(raw) - LOG10_C_D; }

static int any_n(const uint8_t* p, uint32_t n)
{
    for (uint32_t i = 0; i < n; i++)
        if (p[i] == 'N') return 1;
    return 0;
}

/* All-FP64 oracle: log10 likelihood computed in double end to end with plain multiply/add.  A pair
 * with an 'N' in its read or haplotype uses the model the reference applies to it (N matches
 * every base, intra prior); other pairs the inter prior. */
double oracle_log10_f64(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                        const uint8_t* iq, const uint8_t* dq, const uint8_t* cq)
{
    const int kernel = (any_n(hap, hl) || any_n(rd, rl)) ? ORACLE_INTRA : ORACLE_INTER;
    return oracle_log10_from_f64(oracle_raw_f64(hap, hl, rd, rl, q, iq, dq, cq, kernel, ORACLE_UNFUSED));
}

/* One pair with the reference's FP32 -> FP64 switch; *used_f64 reports which precision won. */
double oracle_log10_switch(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                           const uint8_t* iq, const uint8_t* dq, const uint8_t* cq, int kernel, int fused,
                           int* used_f64)
{
    float r = oracle_raw_f32(hap, hl, rd, rl, q, iq, dq, cq, kernel, fused);
    if (r < MIN_ACCEPTED) {
        if (used_f64) *used_f64 = 1;
        return oracle_log10_from_f64(oracle_raw_f64(hap, hl, rd, rl, q, iq, dq, cq, kernel, fused));
    }
    if (used_f64) *used_f64 = 0;
    return oracle_log10_from_f32(r);
}

/* ---------------------------------------------------------------------------------------------
 * Whole batch in the packed layout of phmm_batch, with the reference's routing of a pair to a
 * kernel variant: pairs whose read or haplotype holds an 'N' go to the intra kernel, the others
 * to the inter kernel (roDV_schedule.cpp:96,105,417-441).  out / used_f64 are region blocks of
 * [hap][read].  Empty pairs get NaN.  Returns the number of pairs recomputed in FP64.
 * With fp64_only the FP32 pass is skipped and every pair is the all-FP64 oracle value.
 * ------------------------------------------------------------------------------------------- */
static int has_n(const uint8_t* p, uint64_t n)
{
    for (uint64_t i = 0; i < n; i++)
        if (p[i] == 'N') return 1;
    return 0;
}

uint64_t oracle_batch(uint32_t n_regions, const uint32_t* n_haps, const uint32_t* n_reads, const uint8_t* hap_bases,
                      const uint64_t* hap_off, const uint8_t* rb, const uint8_t* q, const uint8_t* iq, const uint8_t* dq,
                      const uint8_t* cq, const uint64_t* read_off, int fused, int fp64_only, double* out,
                      uint8_t* used_f64)
{
    oracle_init();
    uint64_t h0 = 0, r0 = 0, o = 0, n64 = 0;
    for (uint32_t g = 0; g < n_regions; g++) {
        for (uint32_t h = 0; h < n_haps[g]; h++) {
            const uint64_t ha = hap_off[h0 + h], hl = hap_off[h0 + h + 1] - ha;
            const int hn = has_n(hap_bases + ha, hl);
            for (uint32_t r = 0; r < n_reads[g]; r++, o++) {
                const uint64_t ra = read_off[r0 + r], rl = read_off[r0 + r + 1] - ra;
                int u = 0;
                if (hl == 0 || rl == 0) {
                    out[o] = NAN;
                } else if (fp64_only) {
                    out[o] = oracle_log10_f64(hap_bases + ha, (uint32_t)hl, rb + ra, (uint32_t)rl, q + ra, iq + ra,
                                              dq + ra, cq + ra);
                } else {
                    const int kernel = (hn || has_n(rb + ra, rl)) ? ORACLE_INTRA : ORACLE_INTER;
                    out[o] = oracle_log10_switch(hap_bases + ha, (uint32_t)hl, rb + ra, (uint32_t)rl, q + ra, iq + ra,
                                                 dq + ra, cq + ra, kernel, fused, &u);
                }
                if (used_f64) used_f64[o] = (uint8_t)u;
                n64 += (uint64_t)u;
            }
        }
        h0 += n_haps[g];
        r0 += n_reads[g];
    }
    return n64;
}
