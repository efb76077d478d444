// phmm_compute_regions_noalloc: the batch computation of phmm_compute_regions for callers that
// cannot allocate device memory.
//
// Who needs it: a caller whose process must not call cudaMalloc -- e.g. a host application whose
// GPU memory is owned by another framework's pool allocator (a second allocator would fragment or
// overcommit it), or a plugin that runs inside a host that forbids allocation on its worker
// threads.  Such callers cannot create a phmm_engine (its arena is cudaMalloc'ed).
//
// How: every device-side byte of the computation -- the probability tables, the batch plan, the
// staged reads and haplotypes, the haplotype match codes, the FP64 rerun list, the multi-stripe
// rows and the staged results -- lives in one file-scope __device__ array of kNoAllocBytes (64 MiB)
// that every GPU loading this library holds until the process exits.  The kernels are the engine's
// own FP32 and FP64 wavefront kernels, launched on the legacy default stream.
//
// Set-up: the first call on a device makes that device current, looks up the array's device
// address with cudaGetSymbolAddress and copies the probability tables into it (synchronously);
// make that first call before any stream capture on the device.  Calls are synchronous and are
// serialised per device by a host lock.  The array keeps the last call's contents; a call
// re-uploads everything it reads and resets what must start at zero (claim counters, rerun
// counts, status word, outputs), so it does not depend on earlier contents.  Work that another
// thread launches into the same array by some other route would race with a call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_kernels.h"
#include "phmm_plan.h"
#include "phmm_tables.h"

namespace phmm {
namespace {

constexpr size_t kNoAllocBytes = 64ull << 20;
constexpr int kNoAllocMultiWarps = 64;    // multi-stripe classes run on this many warps here
constexpr unsigned int kMultiCols = 4096; // = PlanLimits::max_stream_multi

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr size_t kDescBlock = sizeof(BatchDesc) + sizeof(ClassDesc) * kNumClasses + 4 * sizeof(unsigned int);
constexpr size_t kTables32 = (5 * 128 + 128 * 128) * sizeof(float);
constexpr size_t kTables64 = (5 * 128 + 128 * 128) * sizeof(double);

struct DeviceState {
    std::mutex mu;
    bool ready = false;
    char* base = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
    int occ[2][kClasses32] = {};
    ProbTables<float> tf{};
    ProbTables<double> td{};
};

constexpr int kMaxDevices = 64;
DeviceState g_devices[kMaxDevices];

// Offsets inside the array for one batch (tables first, then the batch's sections).
struct Layout {
    size_t desc, regions, read_off, hap_off, read_flags, hap_flags, items, rb, rq, ri, rd, rc, hb, ci, ca, out, pf,
        rerun, scratch, total;
};

Layout layout_for(const Plan& p)
{
    Layout L{};
    size_t o = up256(kTables32) + up256(kTables64);
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = up256(o + std::max<size_t>(bytes, 1));
        return at;
    };
    L.desc = take(kDescBlock);
    L.regions = take(p.regions.size() * sizeof(RegionDesc));
    L.read_off = take(p.read_off.size() * 8);
    L.hap_off = take(p.hap_off.size() * 8);
    L.read_flags = take(p.read_flags.size());
    L.hap_flags = take(p.hap_flags.size());
    L.items = take(p.items.size() * sizeof(WorkItem));
    L.rb = take(p.read_bases);
    L.rq = take(p.read_bases);
    L.ri = take(p.read_bases);
    L.rd = take(p.read_bases);
    L.rc = take(p.read_bases);
    L.hb = take(p.hap_bases);
    L.ci = take((p.hap_bases + 2 * kCodePad) * sizeof(uint32_t));
    L.ca = take((p.hap_bases + 2 * kCodePad) * sizeof(uint32_t));
    L.out = take(p.out_total * sizeof(double));
    L.pf = take(p.out_total);
    L.rerun = take(p.rerun_slots * sizeof(RerunEntry));
    L.scratch = take(p.max_multi_stream ? (size_t)kNoAllocMultiWarps * kMultiCols * 3 * sizeof(double) : 0);
    L.total = o;
    return L;
}

#define NA_CK(call)                                                                       \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);              \
            return PHMM_ERR_CUDA;                                                         \
        }                                                                                 \
    } while (0)

// Once per device, with the device current: the array's address and the probability tables.
phmm_status setup(DeviceState& d, int device, std::string& err)
{
    if (d.ready) return PHMM_OK;
    void* ptr = nullptr;
    NA_CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    cudaDeviceProp prop;
    NA_CK(cudaGetDeviceProperties(&prop, device));
    d.sms = prop.multiProcessorCount;
    for (int p = 0; p < 2; ++p)
        for (int c = 0; c < (p == 0 ? kClasses32 : kClasses64); ++c) {
            int b = 0;
            NA_CK(occupancy(p == 0 ? 32 : 64, c, &b));
            d.occ[p][c] = std::max(b, 1);
        }
    std::vector<char> host(up256(kTables32) + up256(kTables64));
    const HostTables<float>& hf = host_tables_f32();
    const HostTables<double>& hd = host_tables_f64();
    auto put = [](auto* dst, const auto& v) {
        std::copy(v.begin(), v.end(), dst);
        return dst + v.size();
    };
    float* f = (float*)host.data();
    for (const auto* v : {&hf.ph2pr, &hf.pmat, &hf.pmis_inter, &hf.pmis_intra, &hf.gapm, &hf.mm}) f = put(f, *v);
    double* g = (double*)(host.data() + up256(kTables32));
    for (const auto* v : {&hd.ph2pr, &hd.pmat, &hd.pmis_inter, &hd.pmis_intra, &hd.gapm, &hd.mm}) g = put(g, *v);
    NA_CK(cudaMemcpy(ptr, host.data(), host.size(), cudaMemcpyHostToDevice));
    const float* df = (const float*)ptr;
    const double* dd = (const double*)((const char*)ptr + up256(kTables32));
    d.tf = ProbTables<float>{df, df + 128, df + 256, df + 384, df + 512, df + 640};
    d.td = ProbTables<double>{dd, dd + 128, dd + 256, dd + 384, dd + 512, dd + 640};
    d.base = (char*)ptr;
    d.ready = true;
    return PHMM_OK;
}

phmm_status run(const phmm_batch& b, double* out, uint8_t* flags, int32_t device, std::string& err)
{
    Plan plan;
    phmm_status st = build_plan(b, PlanLimits(), plan, err);
    if (st != PHMM_OK) return st;
    if (plan.out_total && !out) {
        err = "out is null";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    const Layout L = layout_for(plan);
    if (L.total > kNoAllocBytes) {
        err = "batch needs " + std::to_string(L.total) + " bytes of device scratch; the no-allocation entry point has " +
              std::to_string(kNoAllocBytes) + " (split the batch)";
        return PHMM_ERR_LIMIT_EXCEEDED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        err = "no CUDA device available";
        return PHMM_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev || device >= kMaxDevices) {
        err = "device ordinal " + std::to_string(device) + " out of range";
        return PHMM_ERR_NO_DEVICE;
    }
    DeviceState& d = g_devices[device];
    std::lock_guard<std::mutex> lk(d.mu);
    // the calling thread's current device is put back on every return path
    int prev_device = -1;
    if (cudaGetDevice(&prev_device) != cudaSuccess) {
        cudaGetLastError();
        prev_device = -1;
    }
    struct RestoreDevice {
        int dev;
        ~RestoreDevice()
        {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev_device};
    NA_CK(cudaSetDevice(device));
    st = setup(d, device, err);
    if (st != PHMM_OK) return st;
    if (plan.out_total == 0) return PHMM_OK;
    char* base = d.base;

    // descriptor block: batch sizes, class descriptors with zeroed counters, zero status
    std::vector<char> desc(kDescBlock, 0);
    BatchDesc bd{};
    bd.hap_bases_total = plan.hap_bases;
    bd.out_total = plan.out_total;
    bd.n_regions = plan.n_regions;
    bd.n_reads = plan.n_reads;
    bd.n_haps = plan.n_haps;
    bd.n_items = (uint32_t)plan.items.size();
    std::memcpy(desc.data(), &bd, sizeof(bd));
    std::memcpy(desc.data() + sizeof(bd), plan.classes.data(), sizeof(ClassDesc) * kNumClasses);
    auto h2d = [&](size_t off, const void* src, size_t bytes) {
        return bytes ? cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    NA_CK(h2d(L.desc, desc.data(), desc.size()));
    NA_CK(h2d(L.regions, plan.regions.data(), plan.regions.size() * sizeof(RegionDesc)));
    NA_CK(h2d(L.read_off, plan.read_off.data(), plan.read_off.size() * 8));
    NA_CK(h2d(L.hap_off, plan.hap_off.data(), plan.hap_off.size() * 8));
    NA_CK(h2d(L.read_flags, plan.read_flags.data(), plan.read_flags.size()));
    NA_CK(h2d(L.hap_flags, plan.hap_flags.data(), plan.hap_flags.size()));
    NA_CK(h2d(L.items, plan.items.data(), plan.items.size() * sizeof(WorkItem)));
    if (plan.read_bases) {
        NA_CK(h2d(L.rb, b.read_bases + plan.read_base0, plan.read_bases));
        NA_CK(h2d(L.rq, b.read_qual + plan.read_base0, plan.read_bases));
        NA_CK(h2d(L.ri, b.read_ins + plan.read_base0, plan.read_bases));
        NA_CK(h2d(L.rd, b.read_del + plan.read_base0, plan.read_bases));
        NA_CK(h2d(L.rc, b.read_gcp + plan.read_base0, plan.read_bases));
    }
    NA_CK(h2d(L.hb, b.hap_bases + plan.hap_base0, plan.hap_bases));

    BatchView v{};
    v.read_bases = (const uint8_t*)(base + L.rb);
    v.read_q = (const uint8_t*)(base + L.rq);
    v.read_i = (const uint8_t*)(base + L.ri);
    v.read_d = (const uint8_t*)(base + L.rd);
    v.read_c = (const uint8_t*)(base + L.rc);
    v.read_off = (const uint64_t*)(base + L.read_off);
    v.read_flags = (const uint8_t*)(base + L.read_flags);
    v.hap_off = (const uint64_t*)(base + L.hap_off);
    v.codes_inter = (const uint32_t*)(base + L.ci);
    v.codes_intra = (const uint32_t*)(base + L.ca);
    v.hap_flags = (const uint8_t*)(base + L.hap_flags);
    v.regions = (const RegionDesc*)(base + L.regions);
    v.out = (double*)(base + L.out);
    v.pair_flags = (uint8_t*)(base + L.pf);
    ClassDesc* classes = (ClassDesc*)(base + L.desc + sizeof(BatchDesc));
    unsigned int* status = (unsigned int*)(base + L.desc + sizeof(BatchDesc) + sizeof(ClassDesc) * kNumClasses);
    NA_CK(launch_prep((const BatchDesc*)(base + L.desc), (const uint8_t*)(base + L.hb), (uint32_t*)(base + L.ci),
                      (uint32_t*)(base + L.ca), v.out, v.pair_flags, d.sms, 0));
    for (int pass = 0; pass < 2; ++pass) {
        const int n_cls = pass == 0 ? kClasses32 : kClasses64;
        const int slot0 = pass == 0 ? 0 : kClasses32;
        for (int c = 0; c < n_cls; ++c) {
            const uint32_t work = pass == 0 ? plan.classes[c].n_items : plan.classes[slot0 + c].rerun_cap;
            if (work == 0) continue;
            const bool multi = pass == 0 ? class32_multi(c) : (c % 9) == 8;
            const int wpb = kFwdBlock / kWarp;
            int grid = std::min<int>((int)((work + wpb - 1) / wpb), d.occ[pass][c] * d.sms);
            if (multi) grid = std::min(grid, kNoAllocMultiWarps / wpb);
            PassControl pc{};
            pc.cd = classes + slot0 + c;
            pc.cd64 = classes + kClasses32;
            pc.items = (const WorkItem*)(base + L.items);
            pc.rerun = (RerunEntry*)(base + L.rerun);
            pc.status = status;
            pc.scratch = plan.max_multi_stream ? (void*)(base + L.scratch) : nullptr;
            pc.scratch_cols = plan.max_multi_stream ? kMultiCols : 0u;
            NA_CK(launch_fwd(pass == 0 ? 32 : 64, c, v, d.tf, d.td, pc, std::max(grid, 1), 0));
        }
    }
    NA_CK(cudaMemcpy(out, v.out, plan.out_total * sizeof(double), cudaMemcpyDeviceToHost));
    if (flags) NA_CK(cudaMemcpy(flags, v.pair_flags, plan.out_total, cudaMemcpyDeviceToHost));
    unsigned int st_word = 0;
    NA_CK(cudaMemcpy(&st_word, status, sizeof(st_word), cudaMemcpyDeviceToHost));
    if (st_word != 0) {
        err = "kernel status word " + std::to_string(st_word);
        return PHMM_ERR_DEVICE_STATUS;
    }
    return PHMM_OK;
}

}  // namespace
}  // namespace phmm

extern "C" phmm_status phmm_compute_regions_noalloc(const phmm_batch* batch, double* out, uint8_t* pair_flags,
                                                    int32_t device)
{
    try {
        phmm::clear_error();
        if (!batch) return phmm::set_error(PHMM_ERR_INVALID_ARGUMENT, "batch is null");
        std::string err;
        const phmm_status st = phmm::run(*batch, out, pair_flags, device, err);
        return st == PHMM_OK ? PHMM_OK : phmm::set_error(st, err);
    } catch (const std::exception& ex) {
        return phmm::set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}
