// Host copies of the PairHMM probability tables (see phmm_tables.cpp for the reference lines).
#pragma once

#include <vector>

namespace phmm {

template <typename T>
struct HostTables {
    std::vector<T> ph2pr;       // [128]
    std::vector<T> pmat;        // [128] 1 - ph2pr[q]
    std::vector<T> pmis_inter;  // [128] ph2pr[q] * (1/3)
    std::vector<T> pmis_intra;  // [128] ph2pr[q] / 3
    std::vector<T> gapm;        // [128] 1 - ph2pr[c]
    std::vector<T> mm;          // [128*128] match-to-match, indexed [ins][del]
};

const HostTables<float>& host_tables_f32();
const HostTables<double>& host_tables_f64();

// The genotyping Jacobian table, log10(1 + 10^(-k * 1e-4)) for k = 0..80000 in double
// (common/utils/math_utils.h:209-242), and log10(2) from the host math library (Log10Cache).
const std::vector<double>& genotype_jacobian();
double host_log10_two();

}  // namespace phmm
