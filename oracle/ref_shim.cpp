// Test-infrastructure only: the exported C-ABI over the reference's own PairHMM kernels, built by
// oracle/build_ref.sh into oracle/_ref/libphmm_ref.so.  Tests use it to pin the oracle
// restatement (oracle/phmm_oracle.c); bench.py times ref_schedule as the CPU baseline.  Nothing in
// the product (rovaca_b200/) links or calls it.
//
// Compiled with the scheduler's flags (-mavx -mavx2, src/haplotypecaller/pairhmm/CMakeLists.txt:5)
// and dispatching like the reference: AVX-512 kernels when the CPU has them, else AVX2
// (roDV_common/cpu_features.h:53-90, roDV_schedule.cpp:224-231).
//   vector-API scheduler   src/haplotypecaller/pairhmm/roDV_schedule.cpp:154-361
//   process set-up         src/haplotypecaller/pairhmm/pairhmm_engine.cpp:34-36
#include <cstdint>
#include <vector>

#include "roDV_common/common.h"
#include "roDV_common/cpu_features.h"
#include "roDV_schedule.h"

extern "C" {
int ref_avx512_inter_width_f32(void);
int ref_avx512_inter_width_f64(void);
float ref_avx512_intra_raw_f32(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                               const uint8_t*, const uint8_t*);
double ref_avx512_intra_raw_f64(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                                const uint8_t*, const uint8_t*);
double ref_avx512_intra_log10(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                              const uint8_t*, const uint8_t*, int);
int ref_avx512_inter(int, uint32_t, const uint8_t* const*, const uint32_t*, const uint8_t* const*, const uint32_t*,
                     const uint8_t* const*, const uint8_t* const*, const uint8_t* const*, const uint8_t* const*, int,
                     double*);
int ref_avx2_inter_width_f32(void);
int ref_avx2_inter_width_f64(void);
float ref_avx2_intra_raw_f32(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                             const uint8_t*, const uint8_t*);
double ref_avx2_intra_raw_f64(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                              const uint8_t*, const uint8_t*);
double ref_avx2_intra_log10(const uint8_t*, uint32_t, const uint8_t*, uint32_t, const uint8_t*, const uint8_t*,
                            const uint8_t*, const uint8_t*, int);
int ref_avx2_inter(int, uint32_t, const uint8_t* const*, const uint32_t*, const uint8_t* const*, const uint32_t*,
                   const uint8_t* const*, const uint8_t* const*, const uint8_t* const*, const uint8_t* const*, int,
                   double*);
}

static bool use512() { return pairhmm::common::CpuFeatures::hasAVX512Support(); }

extern "C" {

// Base-to-index table and flush-to-zero on the calling thread, as init_pairhmm_ptr does.
void ref_init(void)
{
    pairhmm::common::ConvertChar::init();
    pairhmm::common::init_native();
}

// 512 when the AVX-512 kernels are the ones the reference would run here, 256 for AVX2, 0 if neither.
int ref_isa_bits(void)
{
    if (use512()) return 512;
    return pairhmm::common::CpuFeatures::hasAVX2Support() ? 256 : 0;
}

int ref_inter_width_f32(void) { return use512() ? ref_avx512_inter_width_f32() : ref_avx2_inter_width_f32(); }
int ref_inter_width_f64(void) { return use512() ? ref_avx512_inter_width_f64() : ref_avx2_inter_width_f64(); }

// Raw (2^120-scaled, not log) forward sum of the intra kernel in FP32.
float ref_intra_raw_f32(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                        const uint8_t* i, const uint8_t* d, const uint8_t* c)
{
    return use512() ? ref_avx512_intra_raw_f32(hap, hl, rs, rl, q, i, d, c)
                    : ref_avx2_intra_raw_f32(hap, hl, rs, rl, q, i, d, c);
}

// Raw (2^1020-scaled) forward sum of the intra kernel in FP64.
double ref_intra_raw_f64(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                         const uint8_t* i, const uint8_t* d, const uint8_t* c)
{
    return use512() ? ref_avx512_intra_raw_f64(hap, hl, rs, rl, q, i, d, c)
                    : ref_avx2_intra_raw_f64(hap, hl, rs, rl, q, i, d, c);
}

// log10 likelihood of one pair with the reference's FP32 -> FP64 switch at 1e-28.
double ref_intra_log10(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                       const uint8_t* i, const uint8_t* d, const uint8_t* c, int use_double)
{
    return use512() ? ref_avx512_intra_log10(hap, hl, rs, rl, q, i, d, c, use_double)
                    : ref_avx2_intra_log10(hap, hl, rs, rl, q, i, d, c, use_double);
}

// Inter kernel over exactly ref_inter_width_f32() (dbl=0) or ref_inter_width_f64() (dbl=1) pairs,
// given as parallel arrays.  raw=1 returns the scaled sums, raw=0 the log10 likelihoods.
int ref_inter(int dbl, uint32_t n, const uint8_t* const* hap, const uint32_t* hl, const uint8_t* const* rs,
              const uint32_t* rl, const uint8_t* const* q, const uint8_t* const* i, const uint8_t* const* d,
              const uint8_t* const* c, int raw, double* out)
{
    return use512() ? ref_avx512_inter(dbl, n, hap, hl, rs, rl, q, i, d, c, raw, out)
                    : ref_avx2_inter(dbl, n, hap, hl, rs, rl, q, i, d, c, raw, out);
}

// One region through the reference's vector-API scheduler (schedule_pairhmm).  Haplotypes and
// reads are concatenated with offset arrays of n+1 entries.  out is [n_reads][n_haps] log10.
int ref_schedule(uint32_t n_haps, const uint8_t* hap_bases, const uint64_t* hap_off, uint32_t n_reads,
                 const uint8_t* read_bases, const uint8_t* q, const uint8_t* i, const uint8_t* d, const uint8_t* c,
                 const uint64_t* read_off, double idle_f, double idle_d, double* out)
{
    std::vector<std::vector<uint8_t>> haps(n_haps), reads(n_reads), qq(n_reads), ii(n_reads), dd(n_reads), cc(n_reads);
    for (uint32_t h = 0; h < n_haps; ++h) haps[h].assign(hap_bases + hap_off[h], hap_bases + hap_off[h + 1]);
    for (uint32_t r = 0; r < n_reads; ++r) {
        const uint64_t a = read_off[r], b = read_off[r + 1];
        reads[r].assign(read_bases + a, read_bases + b);
        qq[r].assign(q + a, q + b);
        ii[r].assign(i + a, i + b);
        dd[r].assign(d + a, d + b);
        cc[r].assign(c + a, c + b);
    }
    std::vector<std::vector<double>> res;
    bool ok = pairhmm::schedule::schedule_pairhmm(haps, reads, res, qq, ii, dd, cc, false, idle_f, idle_d, false);
    if (!ok) return -1;
    for (uint32_t r = 0; r < n_reads; ++r)
        for (uint32_t h = 0; h < n_haps; ++h) out[(uint64_t)r * n_haps + h] = res[r][h];
    return 0;
}

}  // extern "C"
