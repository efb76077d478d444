// FP32 wavefront with packed FP32 arithmetic (sm_100a __ffma2_rn / __fmul2_rn / __fadd2_rn).
//
// Arithmetic per cell is exactly the reference's (see phmm_device.cuh for the operation order and
// the reference lines); a packed instruction applies it to two cells with the same per-component
// rounding as the scalar intrinsics, so results stay bit-identical.
//
// Mapping.  A warp sweeps two reads of one region, X in the .x components and Y in the .y
// components, through the same run of haplotype columns.  Lane l holds rows l*KH .. l*KH+KH-1 of
// both reads' stripes and works on stream column p = t - l at step t, so the two components of every
// float2 meet the same haplotype base: one packed instruction updates row a of X and row a of Y.
// Two values formed from a lane's bottom rows go to lane l+1 by shuffle (three, M, I and D, in
// PM_ALL); lane 31 holds both reads' last rows and sums them per haplotype.  Rows are padded at the
// top, each read by its own count, and pad rows reproduce the boundary row exactly (prior 0 keeps
// M = 0, I stays 0 because the rows above have M = I = 0, and xx = 1 keeps D = C/H).  Reads longer
// than one stripe run as stripes linked through a per-warp scratch row of float2 values.
//
// Lane state between steps.  A lane does not keep its rows' M, I and D at its last column: it keeps,
// per row, the values the next column starts from -- the diagonal sum s that M[i][j+1] = s * prior
// multiplies (formed from row i-1 at column j as soon as that row is known, for the lane's first
// row from the row above it, which arrives by shuffle) and D[i][j+1] (formed from row i at column
// j) -- plus the bottom row's M, I and D for the next lane.  That is 2 * KH + 3 values per read
// instead of 3 * KH + 3 (the row above's diagonal included), the same operations on the same
// operands, and a step's M and D of every row only wait for values of the previous step; the I
// chain down the lane's rows alone waits for this step's shuffle.
//
// Match prior.  A cell's prior depends only on its read row and the class of its haplotype base, and
// a lane's rows are fixed for a stripe, so each lane tabulates its rows' priors for the five base
// classes (kTabClasses; the class rides in the haplotype code word) in shared memory once per
// stripe.  A step then loads the priors of two row pairs with one 128-bit shared-memory load at its
// column's class, where a compare and a select per cell would otherwise take the integer pipe.
// Inter reads with bytes outside A/C/G/T can equal a haplotype byte of class 4; a warp holding such
// a row runs every step on the checked path, which corrects the class-4 priors by comparing bytes.
//
// Gap parameters: PM_EQ when a read's insertion, deletion and gap-continuation qualities are each
// constant along it and its insertion and deletion qualities are equal (the region API without a
// PCR model, and the benchmark data), PM_ROW otherwise.  In PM_EQ, mm, gapm and mx (= my) are held
// once per lane instead of once per row (xx stays per row: pad rows need xx = 1), which leaves
// registers for more rows per lane, and a cell takes 7 operations instead of 8 (M * mx serves both
// I of the row below and D of the next column).  In both modes the lane above forms the first row's
// I and diagonal sum (cells2_eq, cells2_row), so a step shuffles two values instead of three.
#pragma once

#include <cstdint>

#include "phmm_device.cuh"

namespace phmm {

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 rmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 rfma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 radd2(float2 a, float2 b) { return __fadd2_rn(a, b); }

__device__ __forceinline__ float2 shfl_up2(float2 v)
{
    return f2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}

// Prior table of one warp: [class][quad][lane] float4, a quad holding the (X, Y) priors of two row
// pairs.  A class plane spans tab_quads 512-byte quads; the code word's class field (class <<
// kTabShift, a multiple of 2 KB) becomes the plane offset by a right shift of tab_shift.
template <int KH>
__host__ __device__ constexpr int tab_quads()
{
    return KH > 4 ? 4 : KH > 2 ? 2 : 1;
}
template <int KH>
__host__ __device__ constexpr int tab_shift()
{
    return KH > 4 ? 0 : KH > 2 ? 1 : 2;
}
template <int KH>
__host__ __device__ constexpr int tab_floats4()
{
    return kTabClasses * tab_quads<KH>() * kWarp;
}

template <int KH, int PM>
struct LaneRows2 {
    static constexpr int NR = PM == PM_ROW ? KH : 1;
    float2 S[KH];                   // (X, Y) diagonal sum of row a for the lane's next column
    float2 Dn[KH];                  // (X, Y) D of row a at the lane's next column
    float2 Mb, Ib, Db;              // bottom row at the lane's last column (shuffled to lane + 1;
                                    // hand-off: Mb and Ib only feed lane 31's sums)
    float2 In, Sn;                  // hand-off: I of the row below the lane and that row's diagonal sum
                                    // for its next column, formed from the bottom row (shuffled to
                                    // lane + 1 in place of Mb, Ib and Db)
    float2 xxn;                     // PM_EQ, PM_ROW: xx of the row below the lane (1 for a pad row)
    float2 mmn, gmn, mxn;           // PM_ROW: that row's mm, gapm and mx
    float2 xx[KH];
    float2 mm[NR], gm[NR], mx[NR], my[NR];  // my: unused in PM_EQ (mx == my)
    uint32_t padX, padY;            // bit a: row a of the read is a pad row
};

// The two reads of a work item (Y may be absent: R = 0, every row a pad row).
struct ReadPair {
    uint64_t roff[2];
    int R[2];
    int pad[2];                     // pad rows above each read (all stripes together)
};

struct RowParams {
    float pa, pb, mm, gm, mx, xx, my;
    uint32_t rc;
    bool pad;
};

template <int V>
__device__ __forceinline__ RowParams row_params(const BatchView& b, const ProbTables<float>& tb, uint64_t roff, int R,
                                                int i)
{
    RowParams r;
    if (i >= 0 && i < R) {
        const uint64_t o = roff + (uint64_t)i;
        const int q = b.read_q[o] & 127, iq = b.read_i[o] & 127, dq = b.read_d[o] & 127, c = b.read_c[o] & 127;
        r.pa = tb.pmat[q];
        r.pb = (V == kInter) ? tb.pmis_inter[q] : tb.pmis_intra[q];
        r.mm = tb.mm[iq * 128 + dq];
        r.gm = tb.gapm[c];
        r.mx = tb.ph2pr[iq];
        r.xx = tb.ph2pr[c];
        r.my = tb.ph2pr[dq];
        r.rc = match_code(b.read_bases[o], V);
        r.pad = false;
    } else {
        r.pa = r.pb = r.mm = r.gm = r.mx = r.my = 0.f;
        r.xx = 1.f;
        r.rc = 0u;
        r.pad = true;
    }
    return r;
}

template <int V>
__device__ __forceinline__ float class_prior(const RowParams& r, uint32_t cls)
{
    return class_matches(cls, r.rc, V) ? r.pa : r.pb;  // pad rows: pa = pb = 0
}

// Loads this lane's rows of the stripe starting at padded row `first` and writes their prior table.
// Returns true when one of the lane's rows is an inter row with a byte outside A/C/G/T.
template <int KH, int V, int PM>
__device__ __forceinline__ bool load_rows2(LaneRows2<KH, PM>& L, float4* tab, const BatchView& b,
                                           const ProbTables<float>& tb, const ReadPair& rp, int first, int lane)
{
    constexpr int QJ = tab_quads<KH>();
    L.padX = 0;
    L.padY = 0;
    // columns before the lane's first haplotype compute from these and are discarded
#pragma unroll
    for (int a = 0; a < KH; ++a) L.S[a] = L.Dn[a] = f2(0.f, 0.f);
    L.Mb = L.Ib = L.Db = L.In = L.Sn = f2(0.f, 0.f);
    if (PM != PM_ALL) {
        // the row below the lane (for lane 31 the next stripe's first row), whose first-row inputs
        // this lane forms
        const int below = first + lane * KH + KH;
        const RowParams xn = row_params<V>(b, tb, rp.roff[0], rp.R[0], below - rp.pad[0]);
        const RowParams yn = row_params<V>(b, tb, rp.roff[1], rp.R[1], below - rp.pad[1]);
        L.xxn = f2(xn.xx, yn.xx);
        if (PM == PM_ROW) {
            L.mmn = f2(xn.mm, yn.mm);
            L.gmn = f2(xn.gm, yn.gm);
            L.mxn = f2(xn.mx, yn.mx);
        }
    }
    if (PM != PM_ROW) {
        // constant along the read: any real row gives them (pad rows ignore them)
        const RowParams x0 = row_params<V>(b, tb, rp.roff[0], rp.R[0], rp.R[0] > 0 ? 0 : -1);
        const RowParams y0 = row_params<V>(b, tb, rp.roff[1], rp.R[1], rp.R[1] > 0 ? 0 : -1);
        L.mm[0] = f2(x0.mm, y0.mm);
        L.gm[0] = f2(x0.gm, y0.gm);
        L.mx[0] = f2(x0.mx, y0.mx);
        L.my[0] = f2(x0.my, y0.my);
    }
    bool exotic = false;
    float2* t2 = reinterpret_cast<float2*>(tab);
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const int row = first + lane * KH + a;
        const RowParams X = row_params<V>(b, tb, rp.roff[0], rp.R[0], row - rp.pad[0]);
        const RowParams Y = row_params<V>(b, tb, rp.roff[1], rp.R[1], row - rp.pad[1]);
        L.xx[a] = f2(X.xx, Y.xx);
        if (PM == PM_ROW) {
            L.mm[a] = f2(X.mm, Y.mm);
            L.gm[a] = f2(X.gm, Y.gm);
            L.mx[a] = f2(X.mx, Y.mx);
            L.my[a] = f2(X.my, Y.my);
        }
        L.padX |= (X.pad ? 1u : 0u) << a;
        L.padY |= (Y.pad ? 1u : 0u) << a;
        if (V == kInter)
            exotic |= (!X.pad && base_class((uint8_t)X.rc) == 4u) || (!Y.pad && base_class((uint8_t)Y.rc) == 4u);
#pragma unroll
        for (int c = 0; c < kTabClasses; ++c)
            t2[((c * QJ + a / 2) * kWarp + lane) * 2 + (a & 1)] =
                f2(class_prior<V>(X, (uint32_t)c), class_prior<V>(Y, (uint32_t)c));
    }
    if (KH & 1) {
#pragma unroll
        for (int c = 0; c < kTabClasses; ++c) t2[((c * QJ + KH / 2) * kWarp + lane) * 2 + 1] = f2(0.f, 0.f);
    }
    return exotic;
}

// Haplotype code words staged in shared memory (build-time setting): each warp keeps a ring of
// kCodeRing words, the columns its lanes read in the current chunk of steps and the next
// kRingAhead chunks', copying the words of the chunk after those from global memory with cp.async
// while the current chunk computes, so a step reads its code word from shared memory instead of
// through L1.  A chunk reads columns [t0-31, t0+kChunk] and the copies in flight write
// [t0+(A)kChunk, t0+(A+1)kChunk) (A = kRingAhead): 31 + (A+1) kChunk <= kCodeRing slots, so no copy
// overwrites a word a lane still reads.  Columns stay within the stream's guard words
// (t0 + (A+1) kChunk <= Tcols + 32 + (A+1) kChunk <= Tcols + kCodePad).  Measured on B200 over the
// 2,000-region benchmark batch: 1.3% faster than loading the words through L1.
#ifndef PHMM_CODES_STAGED
#define PHMM_CODES_STAGED 1
#endif
#ifndef PHMM_CODE_RING
#define PHMM_CODE_RING 64
#endif
constexpr int kCodeRing = PHMM_CODE_RING;  // a power of two
// float4 slots the ring adds to a warp's shared prior table
constexpr int kRingFloat4 = PHMM_CODES_STAGED ? kCodeRing / 4 : 0;

// (compiled for the host, as the CPU warp emulator does, a copy completes at once)
#if PHMM_CODES_STAGED
__device__ __forceinline__ void copy_word_async(uint32_t* dst_shared, const uint32_t* src)
{
#ifdef __CUDA_ARCH__
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_shared);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
#else
    *dst_shared = *src;
#endif
}
__device__ __forceinline__ void copies_commit()
{
#ifdef __CUDA_ARCH__
    asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void copies_wait_all()
{
#ifdef __CUDA_ARCH__
    asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}
#endif

// Load the next step's priors during the current step (build-time setting): shortens the step of a
// warp that runs alone on its scheduler at the cost of KH register pairs.  Measured on B200 with 12
// warps per SM for KH >= 4: one region per call 140 instead of 124 GCUPS on the device, the
// 2,000-region batch 2279 instead of 2361 GCUPS.  Loading only the first two row pairs' priors ahead
// (the first rows of a step need them first) ran the batch 1.4% slower than none.  0 by default.
#ifndef PHMM_PRIOR_PREFETCH
#define PHMM_PRIOR_PREFETCH 0
#endif
// Chunks of code words the ring holds ahead of the chunk being computed: a prefetching step reads
// the word of the column after its own, which at a chunk's last step is the next chunk's first.
constexpr int kRingAhead = PHMM_PRIOR_PREFETCH ? 2 : 1;
static_assert(31 + (kRingAhead + 1) * kChunk <= kCodeRing && 32 + (kRingAhead + 1) * kChunk <= kCodePad,
              "code ring too small for the chunks it holds ahead");

template <int V>
__device__ __forceinline__ float2 diag_sum_p(float2 mm, float2 gm, float2 dgM, float2 dgI, float2 dgD)
{
    if (V == kInter) return rfma2(dgD, gm, rfma2(dgM, mm, rmul2(dgI, gm)));
    return rfma2(dgD, gm, rfma2(dgI, gm, rmul2(dgM, mm)));
}

template <int V, int PM, int KH>
__device__ __forceinline__ float2 diag_sum(const LaneRows2<KH, PM>& L, int r, float2 dgM, float2 dgI, float2 dgD)
{
    return diag_sum_p<V>(L.mm[r], L.gm[r], dgM, dgI, dgD);
}

// All KH row pairs of the lane for one step at column j (PM_ALL and PM_ROW).  (upM, upI, upD): the
// row above the lane's first row at column j; pr: the rows' priors at column j.  Per row i (the
// reference's operations):
//   M[i][j] = S * prior                                  S = s formed at the previous step
//   I[i][j] = fma(I[i-1][j], xx, M[i-1][j] * mx)
//   D[i][j] = Dn                                         Dn formed at the previous step
//   Dn      = D[i][j+1]  = fma(D[i][j], yy, M[i][j] * my)        (yy = xx, the same ph2pr[gcp])
//   S'      = s[i+1][j+1] from M, I, D[i][j]                     (diag_sum)
// and the row above's values give the first row's S' for the next column.  A row's pending S is
// read before the row above overwrites it.
template <int KH, int V, int PM>
__device__ __forceinline__ void cells2(LaneRows2<KH, PM>& L, const float2 (&pr)[KH], float2 upM, float2 upI,
                                       float2 upD)
{
    static_assert(PM != PM_EQ, "PM_EQ steps through cells2_eq");
    float2 Mab = upM, Iab = upI;    // the row above, this column
    float2 nM = rmul2(L.S[0], pr[0]);
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const int r = PM == PM_ROW ? a : 0;
        const float2 M = nM;
        if (a + 1 < KH) nM = rmul2(L.S[a + 1], pr[a + 1]);  // before S[a + 1] is overwritten below
        const float2 I = rfma2(Iab, L.xx[a], rmul2(Mab, L.mx[r]));
        const float2 D = L.Dn[a];
        L.Dn[a] = rfma2(D, L.xx[a], rmul2(M, L.my[r]));
        if (a + 1 < KH) {
            L.S[a + 1] = diag_sum<V, PM>(L, PM == PM_ROW ? a + 1 : 0, M, I, D);
        } else {
            L.Mb = M;
            L.Ib = I;
            L.Db = D;
        }
        Mab = M;
        Iab = I;
    }
    L.S[0] = diag_sum<V, PM>(L, 0, upM, upI, upD);
}

// The same step in PM_EQ, where mm, gapm and mx (= my) are one value per read, so the lane above
// can form the first row's inputs itself: upI = I[i0][j] of the lane's first row i0 and upS =
// s[i0][j+1], both formed by the lane above from its bottom row at column j with the same operations
// and operands (I from its M * mx and its copy of this lane's first xx, the sum from M, I, D).  That
// shuffles two values instead of three and leaves 7 operations per cell: M * mx serves I of the row
// below and D of the next column, and the bottom row's goes to the lane below as part of its I.
template <int KH, int V, int PM>
__device__ __forceinline__ void cells2_eq(LaneRows2<KH, PM>& L, const float2 (&pr)[KH], float2 upI, float2 upS)
{
    static_assert(PM == PM_EQ, "cells2_eq is the PM_EQ step");
    float2 Iab = upI, Pab = f2(0.f, 0.f);  // I and M * mx of the row above, this column
    float2 nM = rmul2(L.S[0], pr[0]);
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const float2 M = nM;
        if (a + 1 < KH) nM = rmul2(L.S[a + 1], pr[a + 1]);  // before S[a + 1] is overwritten below
        const float2 I = a == 0 ? upI : rfma2(Iab, L.xx[a], Pab);
        const float2 D = L.Dn[a];
        Pab = rmul2(M, L.mx[0]);
        L.Dn[a] = rfma2(D, L.xx[a], Pab);
        const float2 s = diag_sum<V, PM>(L, 0, M, I, D);
        if (a + 1 < KH) {
            L.S[a + 1] = s;
        } else {
            L.Mb = M;
            L.Ib = I;
            L.Sn = s;
            L.In = rfma2(I, L.xxn, Pab);
        }
        Iab = I;
    }
    L.S[0] = upS;
}

// The same hand-off with per-row gap parameters (PM_ROW): the lane above forms the first row's I
// with that row's mx and xx and its diagonal sum with that row's mm and gapm (mxn, xxn, mmn, gmn),
// the operations and operands the lane itself would use.  Two shuffled values instead of three; the
// 8 operations per cell stay (M * mx of the row below and M * my of the row differ).
template <int KH, int V, int PM>
__device__ __forceinline__ void cells2_row(LaneRows2<KH, PM>& L, const float2 (&pr)[KH], float2 upI, float2 upS)
{
    static_assert(PM == PM_ROW, "cells2_row is the PM_ROW step");
    float2 Mab = f2(0.f, 0.f), Iab = upI;  // the row above, this column
    float2 nM = rmul2(L.S[0], pr[0]);
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const float2 M = nM;
        if (a + 1 < KH) nM = rmul2(L.S[a + 1], pr[a + 1]);  // before S[a + 1] is overwritten below
        const float2 I = a == 0 ? upI : rfma2(Iab, L.xx[a], rmul2(Mab, L.mx[a]));
        const float2 D = L.Dn[a];
        L.Dn[a] = rfma2(D, L.xx[a], rmul2(M, L.my[a]));
        if (a + 1 < KH) {
            L.S[a + 1] = diag_sum<V, PM>(L, a + 1, M, I, D);
        } else {
            L.Mb = M;
            L.Ib = I;
            L.Sn = diag_sum_p<V>(L.mmn, L.gmn, M, I, D);
            L.In = rfma2(I, L.xxn, rmul2(M, L.mxn));
        }
        Mab = M;
        Iab = I;
    }
    L.S[0] = upS;
}

// Output side of a sweep: the two reads' likelihood columns and FP64 rerun lists.
struct SweepOut2 {
    double* out;
    uint8_t* pair_flags;
    uint64_t out_base[2];           // output index of the stream's first haplotype, per read
    uint32_t out_stride;            // output index step between consecutive haplotypes
    uint32_t read[2];               // global read indices (kNoRead: none)
    ClassDesc* cd64[2];             // FP64 class of each read (its rerun segment)
};

// Sweep one stripe of both reads over the column stream of haplotypes [g_lo, g_hi).
//   FROM_SCR: the row above lane 0 comes from the warp's scratch row (stripe > 0).
//   TO_SCR:   lane 31's bottom rows go to the scratch row (not the last stripe).
// first: the stripe's first padded row.  aboveX / aboveY: the row above the lane's first row is
// row 0 or a pad row, per read.  exotic: the warp holds an inter row with a byte outside A/C/G/T
// (every step runs the checked path).
template <int KH, int V, int PM, bool FROM_SCR, bool TO_SCR>
__device__ void sweep2(LaneRows2<KH, PM>& L, float4* tab, const BatchView& b, const ProbTables<float>& tb,
                       const PassControl& pc, const SweepOut2& so, const ReadPair& rp, int first, uint32_t g_lo,
                       uint32_t g_hi, float2* scr, int lane, bool aboveX, bool aboveY, bool exotic)
{
    constexpr int QJ = tab_quads<KH>();
    const uint64_t s0 = b.hap_off[g_lo];
    const int Tcols = (int)(b.hap_off[g_hi] - s0);
    const uint32_t* codes = (V == kInter ? b.codes_inter : b.codes_intra) + kCodePad + s0;
    const char* tab_lane = reinterpret_cast<const char*>(tab) + lane * (int)sizeof(float4);
    // the warp's code ring follows its prior table (PHMM_CODES_STAGED)
    uint32_t* ring = reinterpret_cast<uint32_t*>(tab + tab_floats4<KH>());
    const float C = Scale<float>::initial();
    const bool writer = lane == kWarp - 1;

    // Per-lane stream cursor: cur = haplotype being processed, nb = stream column of the next
    // boundary (first column of the next haplotype, or the end of the stream).
    uint32_t cur = g_lo;
    int nb = 0;
    bool started = false;
    float D0 = 0.f;
    // PM_EQ: lane 0's first-row sum below the boundary row (M = I = 0, D = C/H) for the next column
    // the lane above forms the first row's inputs (PM_EQ, PM_ROW)
    constexpr bool HANDOFF = PM != PM_ALL;
    float2 Stop = f2(0.f, 0.f);
    float2 sumM = f2(0.f, 0.f), sumI = f2(0.f, 0.f);

    const int steps = Tcols + kWarp;  // lane 31 reaches column Tcols (the end) at step Tcols + 31

    // Writer lane: per read, the open run of consecutive underflowed haplotypes (first haplotype,
    // its output index).
    uint32_t run_lo[2] = {0xffffffffu, 0xffffffffu};
    uint64_t run_oi[2] = {0, 0};
    auto close_run = [&](int k, uint32_t end) {
        if (run_lo[k] == 0xffffffffu) return;
        ClassDesc* cd = so.cd64[k];
        const unsigned int slot = atomicAdd(&cd->rerun_count, 1u);
        if (slot < cd->rerun_cap) {
            RerunEntry e;
            e.out_idx = run_oi[k];
            e.read = so.read[k];
            e.hap = run_lo[k];
            e.n_haps = end - run_lo[k];
            e.out_stride = so.out_stride;
            pc.rerun[cd->rerun_off + slot] = e;
            atomicAdd(&cd->rerun_pairs, end - run_lo[k]);
        } else {
            atomicOr(pc.status, kStatusRerunOverflow);
        }
        run_lo[k] = 0xffffffffu;
    };
    auto emit = [&](int k, float tot) {
        if (so.read[k] == kNoRead) return;
        const uint64_t oi = so.out_base[k] + (uint64_t)(cur - g_lo) * so.out_stride;
        so.out[oi] = log10((double)tot) - Scale<float>::log10_initial();
        const bool under = (double)tot < (double)1e-28f;
        if (under) {
            if (run_lo[k] == 0xffffffffu) {
                run_lo[k] = cur;
                run_oi[k] = oi;
            }
        } else {
            close_run(k, cur);
        }
        if (cur + 1 == g_hi) close_run(k, g_hi);
        if (so.pair_flags) so.pair_flags[oi] = under ? 1 : 0;
    };

    // Run by a lane whose column p has reached nb, after the step's shuffles.
    auto boundary = [&]() {
        if (started) {
            if (!TO_SCR && writer) {
                // sums of flushed non-negative values are 0 or normal: no flush needed
                emit(0, __fadd_rn(sumM.x, sumI.x));
                emit(1, __fadd_rn(sumM.y, sumI.y));
            }
            ++cur;
        }
        started = true;
        if (cur < g_hi) {
            const int H = (int)(b.hap_off[cur + 1] - b.hap_off[cur]);
            nb += H;
            D0 = C / (float)H;
            // Left edge of the new haplotype, column 0: M = I = 0 in every row, D = 0 in real rows
            // and C/H in pad rows, which stand for the boundary row 0 (as does the row above the
            // lane's first row when `above`).  The first column starts from the diagonal sums of
            // column 0 and from D[i][1] = fma(D[i][0], xx, 0 * my): C/H in pad rows (xx = 1), else 0.
            const float2 z = f2(0.f, 0.f);
            if (HANDOFF) Stop = diag_sum<V, PM>(L, 0, z, z, f2(D0, D0));
            float2 Dab = f2(aboveX ? D0 : 0.f, aboveY ? D0 : 0.f);
#pragma unroll
            for (int a = 0; a < KH; ++a) {
                const float2 Dc = f2(((L.padX >> a) & 1u) ? D0 : 0.f, ((L.padY >> a) & 1u) ? D0 : 0.f);
                L.S[a] = diag_sum<V, PM>(L, PM == PM_ROW ? a : 0, z, z, Dab);
                L.Dn[a] = Dc;
                Dab = Dc;
            }
            sumM = z;
            sumI = z;
        } else {
            nb = 0x7fffffff;
        }
    };

    // The priors of a column: its code word's class selects the plane of the lane's table.
    auto load_priors = [&](int p, float2(&dst)[KH]) -> uint32_t {
        // p lies in [-31, Tcols + 32]: the guard words around the stream cover it
#if PHMM_CODES_STAGED
        const uint32_t w = ring[p & (kCodeRing - 1)];
#else
        const uint32_t w = codes[p];
#endif
        const char* tp = tab_lane + ((w & kTabMask) >> tab_shift<KH>());
#pragma unroll
        for (int j = 0; j < QJ; ++j) {
            if (2 * j < KH) {
                const float4 q = *reinterpret_cast<const float4*>(tp + j * kWarp * (int)sizeof(float4));
                dst[2 * j] = f2(q.x, q.y);
                if (2 * j + 1 < KH) dst[2 * j + 1] = f2(q.z, q.w);
            }
        }
        return w;
    };
#if PHMM_CODES_STAGED
    // columns [-32, kRingAhead * kChunk) before the first chunk
    for (int q = lane - kWarp; q < kRingAhead * kChunk; q += kWarp) ring[q & (kCodeRing - 1)] = codes[q];
    __syncwarp();
#endif
#if PHMM_PRIOR_PREFETCH
    float2 prn[KH];
    uint32_t wn = load_priors(-lane, prn);
#endif

    auto step = [&](int t, bool check) {
        const int p = t - lane;
        // the row above the lane's first row: its M, I and D, or (hand-off) the first row's I and sum
        float2 uM, uI, uD;
        if (HANDOFF) {
            uI = shfl_up2(L.In);
            uD = shfl_up2(L.Sn);
        } else {
            uM = shfl_up2(L.Mb);
            uI = shfl_up2(L.Ib);
            uD = shfl_up2(L.Db);
        }
        if (check && p == nb) boundary();
        if (lane == 0) {
            if (FROM_SCR) {
                const bool ok = p >= 0 && p < Tcols;
                if (HANDOFF) {
                    uI = ok ? scr[2 * p + 0] : f2(0.f, 0.f);
                    uD = ok ? scr[2 * p + 1] : f2(0.f, 0.f);
                } else {
                    uM = ok ? scr[3 * p + 0] : f2(0.f, 0.f);
                    uI = ok ? scr[3 * p + 1] : f2(0.f, 0.f);
                    uD = ok ? scr[3 * p + 2] : f2(0.f, 0.f);
                }
            } else if (HANDOFF) {
                // below the boundary row (M = I = 0, D = C/H): I = fma(0, xx, 0 * mx) = 0
                uI = f2(0.f, 0.f);
                uD = Stop;
            } else {
                uM = f2(0.f, 0.f);
                uI = f2(0.f, 0.f);
                uD = f2(D0, D0);
            }
        }
        float2 pr[KH];
#if PHMM_PRIOR_PREFETCH
        const uint32_t w = wn;
#pragma unroll
        for (int a = 0; a < KH; ++a) pr[a] = prn[a];
        wn = load_priors(p + 1, prn);
#else
        const uint32_t w = load_priors(p, pr);
#endif
        if (V == kInter && check && exotic && (w & kTabMask) == (4u << kTabShift)) {
            // class 4 holds the mismatch prior for every row; a row whose byte equals this
            // haplotype byte takes the match prior (the raw byte compare of the inter variant)
            const uint32_t hb = w & kCodeMatchMask;
#pragma unroll
            for (int a = 0; a < KH; ++a) {
                const int row = first + lane * KH + a;
                const int iX = row - rp.pad[0], iY = row - rp.pad[1];
                if (iX >= 0 && iX < rp.R[0] && b.read_bases[rp.roff[0] + iX] == hb)
                    pr[a].x = tb.pmat[b.read_q[rp.roff[0] + iX] & 127];
                if (iY >= 0 && iY < rp.R[1] && b.read_bases[rp.roff[1] + iY] == hb)
                    pr[a].y = tb.pmat[b.read_q[rp.roff[1] + iY] & 127];
            }
        }
        if constexpr (PM == PM_EQ)
            cells2_eq<KH, V, PM>(L, pr, uI, uD);
        else if constexpr (PM == PM_ROW)
            cells2_row<KH, V, PM>(L, pr, uI, uD);
        else
            cells2<KH, V, PM>(L, pr, uM, uI, uD);
        if (TO_SCR) {
            if (writer && p >= 0 && p < Tcols) {
                if (HANDOFF) {
                    scr[2 * p + 0] = L.In;
                    scr[2 * p + 1] = L.Sn;
                } else {
                    scr[3 * p + 0] = L.Mb;
                    scr[3 * p + 1] = L.Ib;
                    scr[3 * p + 2] = L.Db;
                }
            }
        } else {
            sumM = radd2(sumM, L.Mb);
            sumI = radd2(sumI, L.Ib);
        }
    };

    for (int t0 = 0; t0 < steps; t0 += kChunk) {
#if PHMM_CODES_STAGED
        // the columns up to kRingAhead chunks ahead are in the ring; start copying the chunk after
        copies_wait_all();
        __syncwarp();
        if (lane < kChunk) {
            const int q = t0 + kRingAhead * kChunk + lane;
            copy_word_async(&ring[q & (kCodeRing - 1)], codes + q);
        }
        copies_commit();
#endif
        // Lanes cover stream columns [t0-31, t0+kChunk-1] in this chunk.  Lane 31 trails, so its
        // next boundary is the first boundary at or after t0-31: past the chunk means no lane meets
        // a boundary and the chunk needs no per-step check.
        const int nb31 = __shfl_sync(0xffffffffu, nb, kWarp - 1);
        if (!exotic && nb31 >= t0 + kChunk && t0 + kChunk <= steps) {
#pragma unroll
            for (int u = 0; u < kChunk; ++u) step(t0 + u, false);
        } else {
            for (int u = 0; u < kChunk; ++u)
                if (t0 + u < steps) step(t0 + u, true);
        }
    }
#if PHMM_CODES_STAGED
    copies_wait_all();
    __syncwarp();
#endif
}

}  // namespace phmm
