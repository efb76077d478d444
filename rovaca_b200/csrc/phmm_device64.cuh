// FP64 recompute (the pass that reruns the pairs whose FP32 sum underflowed): the lane state and step
// of the FP32 kernels (phmm_device2.cuh) in scalar double, one read per warp, with the reference's
// flush-to-zero.  LaneRowsEq for constant gap qualities with equal insertion and deletion quality
// (the FP64 classes of mode 0, PM_EQ), LaneRowsRow for per-row gap parameters (modes 1 and 2); the
// all-FP64 check kernels keep phmm_device.cuh's sweep.
//
// Lane state between steps: per row the pending diagonal sum s (M[i][j+1] = s * prior) and
// D[i][j+1]; the lane above forms the lane's first-row I and diagonal sum from its bottom row (mm,
// gapm and mx are one value per read), so a step shuffles two doubles.  Per cell the reference's
// operations on the same operands as phmm_device.cuh `cells` (M * mx, formed once, is also M * my
// since mx == my), each result flushed below 2^-1022 unless the warp's vote has shown that no result
// of the step can fall there: the same results bit for bit, with 2 K + 3 doubles of lane state
// instead of 4 K + 3, two shuffles instead of three, and (PM_EQ) 7 operations per cell instead of 8.
#pragma once

#include "phmm_device.cuh"

namespace phmm {

template <int K>
struct LaneRowsEq {
    double S[K];                    // diagonal sum of row k for the lane's next column
    double Dn[K];                   // D of row k at the lane's next column
    double In, Sn;                  // I of the row below the lane and its diagonal sum (to lane + 1)
    double Mb, Ib;                  // bottom row's M and I (lane 31's sums)
    double xx[K];
    double xxn;                     // xx of the row below the lane (1 for a pad row)
    double mm, gm, mx;              // one value per read (mx == my)
    uint32_t padmask;               // bit k: slot k is a pad row
};

// Loads this lane's rows of the stripe starting at padded row first_padded_row (pad rows above the
// read) and writes their priors to the warp's table.  Returns true when one of the lane's rows is an
// inter row with a byte outside A/C/G/T (see load_rows).
template <int K, int V>
__device__ __forceinline__ bool load_rows_eq(LaneRowsEq<K>& L, double* tab, const BatchView& b,
                                             const ProbTables<double>& tb, uint64_t roff, int R, int first_padded_row,
                                             int pad, int lane)
{
    bool exotic = false;
    L.padmask = 0;
    {
        // constant along the read: its first row gives them (pad rows ignore them)
        const int iq = R > 0 ? b.read_i[roff] & 127 : 0, dq = R > 0 ? b.read_d[roff] & 127 : 0;
        const int c = R > 0 ? b.read_c[roff] & 127 : 0;
        L.mm = tb.mm[iq * 128 + dq];
        L.gm = tb.gapm[c];
        L.mx = tb.ph2pr[iq];
    }
    // for lane 31 the row below is the next stripe's first row
    const int below = first_padded_row + lane * K + K - pad;
    L.xxn = below >= 0 && below < R ? tb.ph2pr[b.read_c[roff + (uint64_t)below] & 127] : 1.0;
    L.In = L.Sn = L.Mb = L.Ib = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        L.S[k] = L.Dn[k] = 0.0;
        const int i = first_padded_row + lane * K + k - pad;  // 0-based read position
        double pa = 0.0, pb = 0.0;  // pad rows: prior 0 for every class
        uint32_t rc = 0u;
        if (i >= 0 && i < R) {
            const uint64_t o = roff + (uint64_t)i;
            const int q = b.read_q[o] & 127;
            pa = tb.pmat[q];
            pb = (V == kInter) ? tb.pmis_inter[q] : tb.pmis_intra[q];
            L.xx[k] = tb.ph2pr[b.read_c[o] & 127];
            const uint8_t base = b.read_bases[o];
            rc = match_code(base, V);
            if (V == kInter) exotic |= base_class(base) == 4u;
        } else {
            L.xx[k] = 1.0;
            L.padmask |= 1u << k;
        }
#pragma unroll
        for (int c = 0; c < kTabClasses; ++c)
            tab[prior_slot<K>((uint32_t)c, k, lane)] = class_matches((uint32_t)c, rc, V) ? pa : pb;
    }
    return exotic;
}

// The same lane state with per-row gap parameters (PM_ROW: the FP64 classes of modes 1 and 2): each
// row's mm, gapm, mx and my, and those of the row below the lane (whose first-row I and diagonal sum
// this lane forms).
template <int K>
struct LaneRowsRow {
    double S[K];
    double Dn[K];
    double In, Sn;
    double Mb, Ib;
    double xx[K], mm[K], gm[K], mx[K], my[K];
    double xxn, mmn, gmn, mxn;      // the row below the lane (xx 1 and the rest 0 for a pad row)
    uint32_t padmask;
};

template <int K, int V>
__device__ __forceinline__ bool load_rows_row(LaneRowsRow<K>& L, double* tab, const BatchView& b,
                                              const ProbTables<double>& tb, uint64_t roff, int R, int first_padded_row,
                                              int pad, int lane)
{
    bool exotic = false;
    L.padmask = 0;
    L.In = L.Sn = L.Mb = L.Ib = 0.0;
    // gap parameters of read row i (a pad row: xx 1, the others 0)
    auto params = [&](int i, double& xx, double& mm, double& gm, double& mx, double& my) {
        if (i >= 0 && i < R) {
            const uint64_t o = roff + (uint64_t)i;
            const int iq = b.read_i[o] & 127, dq = b.read_d[o] & 127, c = b.read_c[o] & 127;
            xx = tb.ph2pr[c];
            mm = tb.mm[iq * 128 + dq];
            gm = tb.gapm[c];
            mx = tb.ph2pr[iq];
            my = tb.ph2pr[dq];
        } else {
            xx = 1.0;
            mm = gm = mx = my = 0.0;
        }
    };
    double myn;
    params(first_padded_row + lane * K + K - pad, L.xxn, L.mmn, L.gmn, L.mxn, myn);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        L.S[k] = L.Dn[k] = 0.0;
        const int i = first_padded_row + lane * K + k - pad;  // 0-based read position
        params(i, L.xx[k], L.mm[k], L.gm[k], L.mx[k], L.my[k]);
        double pa = 0.0, pb = 0.0;  // pad rows: prior 0 for every class
        uint32_t rc = 0u;
        if (i >= 0 && i < R) {
            const uint64_t o = roff + (uint64_t)i;
            const int q = b.read_q[o] & 127;
            pa = tb.pmat[q];
            pb = (V == kInter) ? tb.pmis_inter[q] : tb.pmis_intra[q];
            const uint8_t base = b.read_bases[o];
            rc = match_code(base, V);
            if (V == kInter) exotic |= base_class(base) == 4u;
        } else {
            L.padmask |= 1u << k;
        }
#pragma unroll
        for (int c = 0; c < kTabClasses; ++c)
            tab[prior_slot<K>((uint32_t)c, k, lane)] = class_matches((uint32_t)c, rc, V) ? pa : pb;
    }
    return exotic;
}

template <int V, bool FLUSH>
__device__ __forceinline__ double diag_eq(double gm, double mm, double dgM, double dgI, double dgD)
{
    auto fz = [](double x) { return FLUSH ? ftz(x) : x; };
    if (V == kInter) return fz(rfma(dgD, gm, fz(rfma(dgM, mm, fz(rmul(dgI, gm))))));
    return fz(rfma(dgD, gm, fz(rfma(dgI, gm, fz(rmul(dgM, mm))))));
}

// All K rows of the lane at one column.  upI, upS: the first row's I at this column and its diagonal
// sum for the next column, formed by the lane above; pr: the rows' priors at this column.
template <int K, int V, bool FLUSH>
__device__ __forceinline__ void cells_eq(LaneRowsEq<K>& L, const double (&pr)[K], double upI, double upS)
{
    auto fz = [](double x) { return FLUSH ? ftz(x) : x; };
    double Iab = upI, Pab = 0.0;  // I and M * mx of the row above, this column
    double nM = fz(rmul(L.S[0], pr[0]));
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double M = nM;
        if (k + 1 < K) nM = fz(rmul(L.S[k + 1], pr[k + 1]));  // before S[k + 1] is overwritten below
        const double I = k == 0 ? upI : fz(rfma(Iab, L.xx[k], Pab));
        const double D = L.Dn[k];
        Pab = fz(rmul(M, L.mx));
        L.Dn[k] = fz(rfma(D, L.xx[k], Pab));
        const double s = diag_eq<V, FLUSH>(L.gm, L.mm, M, I, D);
        if (k + 1 < K) {
            L.S[k + 1] = s;
        } else {
            L.Mb = M;
            L.Ib = I;
            L.Sn = s;
            L.In = fz(rfma(I, L.xxn, Pab));
        }
        Iab = I;
    }
    L.S[0] = upS;
}

// The same step with per-row gap parameters (8 operations per cell: M * mx of the row below and
// M * my of the row differ).
template <int K, int V, bool FLUSH>
__device__ __forceinline__ void cells_eq(LaneRowsRow<K>& L, const double (&pr)[K], double upI, double upS)
{
    auto fz = [](double x) { return FLUSH ? ftz(x) : x; };
    double Mab = 0.0, Iab = upI;  // the row above, this column
    double nM = fz(rmul(L.S[0], pr[0]));
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double M = nM;
        if (k + 1 < K) nM = fz(rmul(L.S[k + 1], pr[k + 1]));
        const double I = k == 0 ? upI : fz(rfma(Iab, L.xx[k], fz(rmul(Mab, L.mx[k]))));
        const double D = L.Dn[k];
        L.Dn[k] = fz(rfma(D, L.xx[k], fz(rmul(M, L.my[k]))));
        if (k + 1 < K) {
            L.S[k + 1] = diag_eq<V, FLUSH>(L.gm[k + 1], L.mm[k + 1], M, I, D);
        } else {
            L.Mb = M;
            L.Ib = I;
            L.Sn = diag_eq<V, FLUSH>(L.gmn, L.mmn, M, I, D);
            L.In = fz(rfma(I, L.xxn, fz(rmul(M, L.mxn))));
        }
        Mab = M;
        Iab = I;
    }
    L.S[0] = upS;
}

// A row's diagonal sum from (M, I, D) of the row above (flushed), with that row's gap parameters.
template <int V, int K>
__device__ __forceinline__ double row_diag(const LaneRowsEq<K>& L, int, double dgM, double dgI, double dgD)
{
    return diag_eq<V, true>(L.gm, L.mm, dgM, dgI, dgD);
}
template <int V, int K>
__device__ __forceinline__ double row_diag(const LaneRowsRow<K>& L, int k, double dgM, double dgI, double dgD)
{
    return diag_eq<V, true>(L.gm[k], L.mm[k], dgM, dgI, dgD);
}

// Whether every nonzero input of the lane's next PHMM_F64_VOTE_EVERY steps reaches
// flush_free_hi<K>(): its rows' pending sums and next-column D, and the two values it hands the lane
// below (that lane's first-row inputs).  The longest product chain of a step is still K + 1 factors
// (the insertion chain from the first row's M down to the value handed on), so the bound of
// rows_flush_free holds.
// The minimum is taken as a tree (depth log2(2 K + 2) instead of a chain of 2 K + 2 dependent
// operations): the next step's arithmetic waits on this vote.
template <int K, typename LR>
__device__ __forceinline__ bool rows_flush_free_eq(const LR& L)
{
    constexpr int N = 2 * K + 2;
    uint32_t v[N];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        v[2 * k] = (uint32_t)__double2hiint(L.S[k]) - 1u;
        v[2 * k + 1] = (uint32_t)__double2hiint(L.Dn[k]) - 1u;
    }
    v[2 * K] = (uint32_t)__double2hiint(L.In) - 1u;
    v[2 * K + 1] = (uint32_t)__double2hiint(L.Sn) - 1u;
#pragma unroll
    for (int w = 1; w < N; w *= 2) {
#pragma unroll
        for (int i = 0; i + w < N; i += 2 * w) v[i] = min(v[i], v[i + w]);
    }
    return v[0] >= flush_free_hi<K>() - 1u;
}

// Sweep one stripe over the column stream of haplotypes [g_lo, g_hi): as `sweep` (phmm_device.cuh),
// the scratch row holding the handed-on (I, sum) pair per column.  LR: LaneRowsEq or LaneRowsRow.
template <int K, int V, bool FROM_SCR, bool TO_SCR, typename LR>
__device__ void sweep_eq(LR& L, const double* tab, const BatchView& b, const ProbTables<double>& tb,
                         const SweepOut& so, uint32_t g_lo, uint32_t g_hi, double* scr, int lane, bool above_row0,
                         bool exotic, uint64_t roff, int R, int row0)
{
    const uint64_t s0 = b.hap_off[g_lo];
    const int Tcols = (int)(b.hap_off[g_hi] - s0);
    const uint32_t* codes = (V == kInter ? b.codes_inter : b.codes_intra) + kCodePad + s0;
    const double C = Scale<double>::initial();

    uint32_t cur = g_lo;
    int nb = 0;
    bool started = false;
    double D0 = 0.0;
    double Stop = 0.0;  // lane 0's first-row sum below the boundary row (M = I = 0, D = C/H)
    double sumM = 0.0, sumI = 0.0;
    bool flush_free = false;  // the current step's inputs are all 0 or above the bound

    const int steps = Tcols + kWarp;

    auto boundary = [&]() {
        if (started) {
            if (!TO_SCR && lane == kWarp - 1) {
                // sums of flushed non-negative values are 0 or normal: no flush needed
                const double tot = radd(sumM, sumI);
                const uint64_t oi = so.out_base + (uint64_t)(cur - g_lo) * so.out_stride;
                so.out[oi] = log10(tot) - Scale<double>::log10_initial();
            }
            ++cur;
        }
        started = true;
        if (cur < g_hi) {
            const int H = (int)(b.hap_off[cur + 1] - b.hap_off[cur]);
            nb += H;
            D0 = C / (double)H;
            // Left edge of the new haplotype: column 0 has M = I = 0 in every row, D = 0 in real rows
            // and C/H in pad rows (which stand for the boundary row, as does the row above the lane's
            // first row when above_row0).  The first column starts from the diagonal sums of column 0
            // and from D[i][1] = fma(D[i][0], xx, 0 * my): C/H in pad rows (xx = 1), else 0.
            Stop = row_diag<V, K>(L, 0, 0.0, 0.0, D0);
            double Dab = above_row0 ? D0 : 0.0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const double Dc = ((L.padmask >> k) & 1u) ? D0 : 0.0;
                L.S[k] = row_diag<V, K>(L, k, 0.0, 0.0, Dab);
                L.Dn[k] = Dc;
                Dab = Dc;
            }
            sumM = 0.0;
            sumI = 0.0;
        } else {
            nb = 0x7fffffff;
        }
    };

    auto step = [&](int t, bool check) {
        const int p = t - lane;
        double uI = shfl_up1(L.In);
        double uS = shfl_up1(L.Sn);
        if (check && p == nb) boundary();
        if (lane == 0) {
            if (FROM_SCR) {
                const bool ok = p >= 0 && p < Tcols;
                uI = ok ? scr[2 * p + 0] : 0.0;
                uS = ok ? scr[2 * p + 1] : 0.0;
            } else {
                // below the boundary row: I = fma(0, xx, 0 * mx) = 0
                uI = 0.0;
                uS = Stop;
            }
        }
        const uint32_t w = codes[p];
        const uint32_t cls = (w & kTabMask) >> kTabShift;
        double pr[K];
#pragma unroll
        for (int k = 0; k < K; ++k) pr[k] = tab[prior_slot<K>(cls, k, lane)];
        if (V == kInter && exotic && cls == 4u) {
            const uint32_t hb = w & kCodeMatchMask;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int i = row0 + lane * K + k;
                if (i >= 0 && i < R && b.read_bases[roff + i] == hb) pr[k] = tb.pmat[b.read_q[roff + i] & 127];
            }
        }
        constexpr bool kVote = PHMM_F64_VOTE && !FROM_SCR;
        if (kVote && flush_free)
            cells_eq<K, V, false>(L, pr, uI, uS);
        else
            cells_eq<K, V, true>(L, pr, uI, uS);
        if (TO_SCR) {
            if (lane == kWarp - 1 && p >= 0 && p < Tcols) {
                scr[2 * p + 0] = L.In;
                scr[2 * p + 1] = L.Sn;
            }
        } else {
            sumM = radd(sumM, L.Mb);
            sumI = radd(sumI, L.Ib);
        }
        if constexpr (kVote)
            if (PHMM_F64_VOTE_EVERY == 1 || t % PHMM_F64_VOTE_EVERY == PHMM_F64_VOTE_EVERY - 1)
                flush_free = __all_sync(0xffffffffu, rows_flush_free_eq<K>(L));
    };

    for (int t0 = 0; t0 < steps; t0 += kChunkScalar) {
        const int nb31 = __shfl_sync(0xffffffffu, nb, kWarp - 1);
        if (nb31 >= t0 + kChunkScalar && t0 + kChunkScalar <= steps) {
#pragma unroll
            for (int u = 0; u < kChunkScalar; ++u) step(t0 + u, false);
        } else {
            for (int u = 0; u < kChunkScalar; ++u)
                if (t0 + u < steps) step(t0 + u, true);
        }
    }
}

}  // namespace phmm
