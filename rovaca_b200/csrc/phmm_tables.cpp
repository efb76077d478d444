// Probability tables of the PairHMM, built on the host exactly as the reference builds them and
// uploaded once per engine.
//
// Reference: src/haplotypecaller/pairhmm/roDV_common/context.h
//   ph2pr[q] = 10^(-q/10) in the working type (powf for float, pow for double)      :98,138
//   Jacobian table log10(1 + 10^(-k*1e-4)), k = 0..80000, stored in the working type :44-48
//   approximateLog10SumLog10 in the working type, fastRound, tolerance 8             :61-82
//   matchToMatchProb[(max*(max+1))/2 + min] = 10^(log1p(-min(1, 10^sum))/ln 10)     :50-60,115-126
// and the per-row values of src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:63-79
// (1 - dist, dist * (1/3), 1 - ph2pr[gcp]) and roDV_intra/pairhmm_impl.cpp:151-156 (dist / 3).
// Qualities are masked with & 127 before any lookup (pairhmm_inter.cpp:66-69), so 128 entries per
// table suffice and the match-to-match table is stored as a full [ins][del] square.
#include "phmm_tables.h"

#include <algorithm>
#include <cmath>

namespace phmm {

namespace {

constexpr int kJacSize = 80001;  // (int)(8.0 / 0.0001) + 1
constexpr double kJacStep = 0.0001;
constexpr double kJacTolerance = 8.0;

template <typename T>
struct JacobianLog {
    std::vector<T> table;
    JacobianLog() : table(kJacSize)
    {
        for (int k = 0; k < kJacSize; ++k) table[k] = (T)(std::log10(1.0 + std::pow(10.0, -((double)k) * kJacStep)));
    }
    static int round_half_away(T d) { return (d > T(0)) ? (int)(d + T(0.5)) : (int)(d - T(0.5)); }
    T log10_sum(T small, T big) const
    {
        if (small > big) std::swap(small, big);
        if (std::isinf(small) || std::isinf(big)) return big;
        const T diff = big - small;
        if (diff >= (T)kJacTolerance) return big;
        const int ind = round_half_away((T)(diff * (T)(1.0 / kJacStep)));
        return big + table[ind];
    }
};

template <typename T>
T ph2pr_of(int q);
template <>
float ph2pr_of<float>(int q)
{
    return std::pow(10.f, -((float)q) / 10.f);
}
template <>
double ph2pr_of<double>(int q)
{
    return std::pow(10.0, -((double)q) / 10.0);
}

template <typename T>
void build(HostTables<T>& t)
{
    const JacobianLog<T> jac;
    const double inv_ln10 = 1.0 / std::log(10);
    // match-to-match over the quality range reachable after & 127
    std::vector<T> tri(128 * 129 / 2);
    for (int i = 0, off = 0; i < 128; off += ++i) {
        for (int j = 0; j <= i; ++j) {
            const T sum = jac.log10_sum((T)(-0.1 * i), (T)(-0.1 * j));
            const double lg = std::log1p(-std::min(1.0, std::pow(10.0, (double)sum))) * inv_ln10;
            tri[off + j] = (T)std::pow(10.0, lg);
        }
    }
    t.mm.resize(128 * 128);
    for (int a = 0; a < 128; ++a)
        for (int b = 0; b < 128; ++b) {
            const int mx = std::max(a, b), mn = std::min(a, b);
            t.mm[a * 128 + b] = tri[((mx * (mx + 1)) >> 1) + mn];
        }
    const T one_third = T(1.0) / T(3.0);
    t.ph2pr.resize(128);
    t.pmat.resize(128);
    t.pmis_inter.resize(128);
    t.pmis_intra.resize(128);
    t.gapm.resize(128);
    for (int q = 0; q < 128; ++q) {
        const T d = ph2pr_of<T>(q);
        t.ph2pr[q] = d;
        t.pmat[q] = T(1) - d;
        t.pmis_inter[q] = d * one_third;
        t.pmis_intra[q] = d / T(3);
        t.gapm[q] = T(1) - d;
    }
}

}  // namespace

const HostTables<float>& host_tables_f32()
{
    static const HostTables<float> t = [] {
        HostTables<float> x;
        build(x);
        return x;
    }();
    return t;
}

const HostTables<double>& host_tables_f64()
{
    static const HostTables<double> t = [] {
        HostTables<double> x;
        build(x);
        return x;
    }();
    return t;
}

const std::vector<double>& genotype_jacobian()
{
    static const std::vector<double> t = [] {
        std::vector<double> x(kJacSize);
        for (int k = 0; k < kJacSize; ++k) x[k] = std::log10(1.0 + std::pow(10.0, -kJacStep * (double)k));
        return x;
    }();
    return t;
}

double host_log10_two() { return std::log10(2.0); }

}  // namespace phmm
