// cmc_noalloc.cu -- cmc_launch_static: the Launch seam with no device allocation.
//
// Who needs it: a host that embeds this estimator but does not own device
// memory -- for example a process whose device memory is held by another
// framework's caching allocator, or a service loop that must not pay the
// device-wide synchronisation of cudaMalloc/cudaFree between launches.  Such a
// caller can pass device buffers for the batch key and the results, but cannot
// let the library call cudaMalloc for its own working memory.
//
// The engine's working memory (control words, the one-job descriptor and the
// failure bitmap) therefore lives in a file-scope __device__ array of fixed
// size, and the 1 KiB T0 table in another.  Every GPU that loads the library
// holds both until the process exits.  Limits: at most kStaticMaxTrials
// trials per call, and only parameter sets whose walk slots fit in shared
// memory (the global slot pool would need an allocation); both are checked and
// reported as CMC_EINVAL with a message.
//
// All calls on a device share the one array and it keeps the last call's
// contents; each call clears what must start at zero.  Calls that overlap on
// the GPU (different streams, or host threads without ordering) race on it, so
// a caller must order them, e.g. by issuing them on one stream.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cmc.h"
#include "cmc_capi_internal.hpp"
#include "cmc_engine.cuh"
#include "cmc_hostcore.hpp"

namespace cmc {

__global__ void cmc_compact_failures(const uint32_t* bits, uint64_t nbits, uint32_t value_base,
                                     uint32_t* out, uint32_t* count, uint64_t cap,
                                     const unsigned long long* nbits_dev);
void set_thread_error(const std::string& message);

namespace {

constexpr uint32_t kStaticMaxTrials = 1u << 20;  // per call
constexpr size_t kCtrlBytes = 256;
constexpr size_t kJobBytes = 512;
constexpr size_t kBitsBytes = kStaticMaxTrials / 8;  // 128 KiB failure bitmap
constexpr size_t kScratchBytes = kCtrlBytes + kJobBytes + kBitsBytes;
static_assert(sizeof(Ctrl) <= kCtrlBytes, "control block fits its region");
static_assert(sizeof(Job) <= kJobBytes, "job descriptor fits its region");

// The working memory of cmc_launch_static (about 129 KiB per GPU).
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];
static __device__ __align__(256) uint32_t g_static_t0[256];

// Writes the job (with the caller's device batch key) into the scratch and
// clears the control block and the bitmap words this call uses.
__global__ void static_prepare(Job job, const uint32_t* __restrict__ d_key,
                               unsigned char* __restrict__ scratch, uint32_t words) {
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(scratch);
    Job* j = reinterpret_cast<Job*>(scratch + kCtrlBytes);
    uint32_t* bits = reinterpret_cast<uint32_t*>(scratch + kCtrlBytes + kJobBytes);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        for (int i = 0; i < 44; ++i) job.batch_rk[i] = d_key[i];
        *j = job;
        *ctrl = Ctrl{};
    }
    for (uint32_t w = tid; w < words; w += gridDim.x * blockDim.x) bits[w] = 0;
}

// A bounded device wait that gave up is reported through the caller's count.
__global__ void static_finish(const unsigned char* __restrict__ scratch, uint32_t* d_nfailed) {
    const Ctrl* ctrl = reinterpret_cast<const Ctrl*>(scratch);
    if (ctrl->error) *d_nfailed = 0xffffffffu;
}

struct DeviceState {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_static_scratch
    uint32_t* t0 = nullptr;            // device address of g_static_t0
    Ctx* planner = nullptr;            // launch planner (no device memory of its own)
    std::vector<Job> jobs;             // the one-job table handed to the planner
};

constexpr int kMaxDevices = 64;
// Guards the per-device set-up and the planner, which calls share.
std::mutex g_setup_mutex;
DeviceState g_devices[kMaxDevices];
alignas(Ctx) unsigned char g_planner_storage[kMaxDevices][sizeof(Ctx)];

int fail(int code, const std::string& message) {
    set_thread_error(message);
    return code;
}

// Once per device, with that device current: the symbol addresses, the T0
// table, and a planner.  Returns 0 or a CMC_E* code.
// The caller holds g_setup_mutex.
int setup(int device, DeviceState*& out) {
    DeviceState& st = g_devices[device];
    if (st.ready) {
        out = &st;
        return CMC_OK;
    }
    void* scratch = nullptr;
    void* t0 = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&scratch, g_static_scratch);
    if (e != cudaSuccess)
        return fail(CMC_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress(&t0, g_static_t0);
    if (e != cudaSuccess)
        return fail(CMC_ECUDA, std::string("cudaGetSymbolAddress(T0): ") + cudaGetErrorString(e));
    uint32_t table[256];
    t0_table(table);
    e = cudaMemcpyToSymbol(g_static_t0, table, sizeof table);
    if (e != cudaSuccess)
        return fail(CMC_ECUDA, std::string("T0 upload: ") + cudaGetErrorString(e));
    int sms = 0, optin = 0, major = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess)
        return fail(CMC_ECUDA, "cudaDeviceGetAttribute failed");
    if (major < 10) return fail(CMC_EINVAL, "cmc_launch_static needs an sm_100 device");
    // the device maximum, the same value every caller sets (never lowered)
    if (engine_smem_cap(size_t(optin))) {
        cudaGetLastError();
        return fail(CMC_ECUDA, "cudaFuncSetAttribute on the engine kernels failed");
    }
    Ctx* planner = new (g_planner_storage[device]) Ctx();  // never destroyed: lives with the scratch
    planner->sms = sms;
    planner->smem_optin = size_t(optin);
    planner->may_allocate = false;  // global round caches and slots would need an allocation
    st.scratch = static_cast<unsigned char*>(scratch);
    st.t0 = static_cast<uint32_t*>(t0);
    st.planner = planner;
    st.jobs.resize(1);
    st.ready = true;
    out = &st;
    return CMC_OK;
}

}  // namespace

}  // namespace cmc

extern "C" int cmc_launch_static(const cmc_params* params, const uint32_t* d_batch_key,
                                 uint32_t first, uint32_t count, uint32_t* d_out_offsets,
                                 uint32_t* d_out_nfailed, void* stream) {
    using namespace cmc;
    if (!params || !d_batch_key || !d_out_offsets || !d_out_nfailed)
        return fail(CMC_EINVAL, "cmc_launch_static: null argument");
    if (count > kStaticMaxTrials)
        return fail(CMC_EINVAL, "cmc_launch_static: count must be at most " + std::to_string(kStaticMaxTrials) +
                                    " (the fixed working memory holds that many trials per call)");
    if (uint64_t(first) + count > 0x100000000ULL)
        return fail(CMC_EINVAL, "cmc_launch_static: offset range overflows");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return fail(CMC_ECUDA, "cmc_launch_static: no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceState* st = nullptr;
    int rc = setup(device, st);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (count == 0) {  // as cmc_launch_device: no trials, no failures
        const cudaError_t e = cudaMemsetAsync(d_out_nfailed, 0, sizeof(uint32_t), s);
        return e == cudaSuccess ? CMC_OK : fail(CMC_ECUDA, std::string("memset count: ") + cudaGetErrorString(e));
    }
    Ctx& pl_ctx = *st->planner;
    Job& job = st->jobs[0];
    if ((rc = pl_ctx.make_job(*params, first, count, 0, job))) return fail(rc, pl_ctx.err);
    Plan pl;
    if ((rc = pl_ctx.plan(st->jobs, pl))) return fail(rc, pl_ctx.err);
    if (!pl.slots_smem || pl.walker_ctas)
        return fail(CMC_EINVAL,
                    "cmc_launch_static: these parameters need walk slots in global memory, which "
                    "would be an allocation; use cmc_launch_device");
    const uint32_t words = (count + 31) / 32;
    // the launch checks below read cudaGetLastError: an earlier non-fatal
    // error of the caller's is not this call's
    cudaGetLastError();
    static_prepare<<<64, 256, 0, s>>>(job, d_batch_key, st->scratch, words);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CMC_ECUDA, std::string("prepare launch: ") + cudaGetErrorString(e));
    EngineArgs a{};
    a.jobs = reinterpret_cast<const Job*>(st->scratch + kCtrlBytes);
    a.njobs = 1;
    a.total = count;
    a.ctrl = reinterpret_cast<Ctrl*>(st->scratch);
    a.fail_bits = reinterpret_cast<uint32_t*>(st->scratch + kCtrlBytes + kJobBytes);
    a.gslots = nullptr;
    a.t0 = st->t0;
    a.slot_stride = pl.slot_stride;
    a.bins_bytes = pl.bins_bytes;
    a.ng = pl.ng;
    a.wg = pl.wg;
    a.ns = pl.ns;
    a.nw = pl.nw;
    a.isolate_walkers = pl.isolate;
    a.r256 = 256u;
    a.group_bytes = pl.group_bytes;
    a.group_off = pl.group_off;
    a.slots_off = pl.slots_off;
    a.spin_limit = pl_ctx.spin_limit;
    a.idle_polls = pl_ctx.spin_limit;
    a.pool_stage = pl.pool_stage;
    a.pool_fold = pl.pool_fold;
    // walk slots in shared memory (checked above)
    const void* fn = engine_kernel(pl.variant, true, pl.pool_stage != 0);
    // the engine's shared-memory limit was raised to the device maximum at set-up
    void* args[] = {&a};
    e = cudaLaunchKernel(fn, dim3(pl.ctas), dim3(pl.threads), args, pl.smem_bytes, s);
    if (e != cudaSuccess) return fail(CMC_ECUDA, std::string("engine launch: ") + cudaGetErrorString(e));
    cmc_compact_failures<<<1, 1024, 0, s>>>(a.fail_bits, count, first, d_out_offsets, d_out_nfailed,
                                            count, nullptr);
    static_finish<<<1, 1, 0, s>>>(st->scratch, d_out_nfailed);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CMC_ECUDA, std::string("compaction launch: ") + cudaGetErrorString(e));
    return CMC_OK;
}
