// Test-infrastructure shim: the reference's own genotyping arithmetic, compiled in place from its
// sources by oracle/build_ref_genotype.sh, behind one C function for the checker.
//
// For one sample at ploidy 2 it runs what HaplotypeCaller runs on the likelihood matrix that
// call_pairhmm returns:
//   AlleleLikelihoods::marginalize       haplotype -> allele maximum per read
//                                        (src/haplotypecaller/genotype/allele_likelihoods.hpp:189-221,
//                                         marginal_likelihoods_direct :702-730)
//   GenotypeLikelihoodCalculator         diploid genotype log10 likelihoods from the marginal matrix
//                                        (genotype_likelihood_calculator.h:44-142,
//                                         genotype_likelihood_calculator.cpp:59-170)
// Haplotypes and alleles are plain objects with the is_reference() the allele list asks for, reads
// are their indices: the templates only compare, hash and store them.
#include <cmath>
#include <cstdint>
#include <map>
#include <memory_resource>
#include <string>
#include <vector>

#include "allele_likelihoods.hpp"
#include "genotype_likelihood_calculator.h"
#include "genotype_likelihoods.h"
#include "indexed_allele_list.hpp"
#include "indexed_sample_list.hpp"

namespace {

struct ShimAllele {
    int32_t index;
    bool reference;
    bool is_reference() const { return reference; }
};
typedef const ShimAllele* pShimAllele;

}  // namespace

extern "C" {

// lk: [n_haps][n_reads] log10 likelihoods (the normalised matrix of kept reads; haplotype 0 is the
// reference haplotype).  hap_allele: per haplotype its allele in [0, n_alleles) or -1 (none).
// allele_lk: out [n_alleles][n_reads] marginal likelihoods.  gl: out [n_alleles (n_alleles + 1) / 2]
// diploid genotype log10 likelihoods in VCF order.  Returns 0, or -1 for arguments outside the
// reference's limits (1 <= n_alleles < 50).
int ref_genotype(int32_t n_haps, int32_t n_reads, const double* lk, int32_t n_alleles, const int8_t* hap_allele,
                 double* allele_lk, double* gl)
{
    using namespace rovaca;
    if (n_alleles < 1 || n_alleles >= 50 || n_haps < 0 || n_reads < 0) return -1;
    std::pmr::monotonic_buffer_resource arena;
    pMemoryPool pool = &arena;

    std::vector<ShimAllele> haps(n_haps), alleles(n_alleles);
    std::pmr::vector<pShimAllele> hap_list(pool), allele_list(pool);
    for (int32_t h = 0; h < n_haps; ++h) {
        haps[h] = ShimAllele{h, h == 0};
        hap_list.push_back(&haps[h]);
    }
    for (int32_t a = 0; a < n_alleles; ++a) {
        alleles[a] = ShimAllele{a, a == 0};
        allele_list.push_back(&alleles[a]);
    }
    typedef AlleleLikelihoods<int32_t, pShimAllele> HapLikelihoods;
    typename HapLikelihoods::TeVector2D evidence(pool), filtered(pool);
    std::pmr::vector<int32_t> reads(pool);
    for (int32_t r = 0; r < n_reads; ++r) reads.push_back(r);
    evidence.push_back(reads);
    filtered.push_back(std::pmr::vector<int32_t>(pool));
    DoubleVector3D values(pool);
    DoubleVector2D sample(pool);
    for (int32_t h = 0; h < n_haps; ++h) {
        DoubleVector row(pool);
        row.assign(lk + (size_t)h * n_reads, lk + (size_t)(h + 1) * n_reads);
        sample.push_back(std::move(row));
    }
    values.push_back(std::move(sample));

    InterfaceSampleList* samples = IndexedSampleList::create(std::vector<std::string>{"sample"});
    auto* hl = HapLikelihoods::create<int32_t, pShimAllele>(pool, samples, IndexedAlleleList<pShimAllele>::create(hap_list, pool),
                                                             std::move(evidence), std::move(filtered), std::move(values));
    std::pmr::map<pShimAllele, std::pmr::vector<pShimAllele>> allele_haps(pool);
    for (int32_t a = 0; a < n_alleles; ++a) allele_haps[allele_list[a]] = std::pmr::vector<pShimAllele>(pool);
    for (int32_t h = 0; h < n_haps; ++h)
        if (hap_allele[h] >= 0 && hap_allele[h] < n_alleles) allele_haps[allele_list[hap_allele[h]]].push_back(hap_list[h]);
    auto* al = hl->marginalize<pShimAllele>(allele_list, allele_haps);

    const DoubleVector2D& m = al->sample_likelihoods(0);
    for (int32_t a = 0; a < n_alleles; ++a)
        for (int32_t r = 0; r < n_reads; ++r) allele_lk[(size_t)a * n_reads + r] = m.at(a).at(r);

    pGenotypeLikelihoodCalculator calc = GenotypeLikelihoodCalculator::create(2, n_alleles, pool);
    pGenotypeLikelihoods g = calc->genotype_likelihoods(al->sample_matrix(0));
    for (size_t k = 0; k < g->_log10likelihoods.size(); ++k) gl[k] = g->_log10likelihoods[k];
    delete samples;
    return 0;
}

}  // extern "C"
