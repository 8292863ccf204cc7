// cmc_capi_internal.hpp -- the context behind the opaque cmc_ctx handle.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "cmc.h"
#include "cmc_engine.cuh"

namespace cmc {

constexpr uint32_t kMaxClasses = 16;  // plan classes per batched call
static_assert(kMaxClasses <= kMaxFusedClasses, "every class fits a fused launch");

struct Plan {
    uint32_t ng = 0, wg = 0, ns = 0, nw = 1;
    uint32_t walker_ctas = 0;  // > 0: split engine with this many walker CTAs
    uint32_t isolate = 0;      // walker warps alone on SM sub-partition 3
    bool slots_smem = true;
    uint32_t slot_stride = 0, bins_bytes = 0, group_bytes = 0;
    uint32_t group_off = 0, slots_off = 0, smem_bytes = 0, threads = 0, ctas = 0;
    int variant = 0;  // 0: u16 map/bins, 1: u32 map/bins, 2: u32 + 64-bit PRP domain
    uint64_t gslot_bytes = 0;     // global walk slots (0: slots in shared memory)
    uint32_t gcache_stride = 0;   // u16 entries per group's global round cache
    uint64_t gcache_bytes = 0;    // all groups' global round caches
    uint32_t pool_stage = 0;      // pooled direct passes: bytes per staging map (0: off)
    uint32_t pool_fold = 0;       // pooled direct passes: bytes per fold table (0: unfolded)
};

uint32_t choose_method(uint32_t h, uint64_t domain, double candidates, int force, bool may_allocate);
// Raises the engine kernels' dynamic shared-memory limit to the device's opt-in maximum.
int engine_smem_cap(size_t optin);
// The engine kernel for a plan's entry width (Plan::variant) and walk-slot
// placement, and the fused kernel of the same kind.
const void* engine_kernel(int variant, bool smem_slots, bool pooled = false);
const void* fused_engine_kernel(int variant, bool smem_slots);
// Estimated cost of one trial in AES-block equivalents (seeds, map, 0.1 t for the walk).
double job_cost(const Job& j);

// Planner options chosen by the autotuner for one mix of parameter sets.
struct TunedPlan {
    uint32_t wg = 0;
    int isolate = -1;
    int method = -1;
};

struct Ctx {
    int device = -1;
    int sms = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;       // the context's own stream
    cudaStream_t user_stream = nullptr;  // cmc_set_stream override
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    uint32_t* d_t0 = nullptr;  // T0 table, FIPS KAT schedule, self-test output
    Ctrl* d_ctrl = nullptr;      // one control block per plan class of a launch
    uint32_t ctrl_count = 1;     // control blocks the last run used
    Job* d_jobs = nullptr;
    size_t jobs_cap = 0;
    uint32_t* d_bits = nullptr;
    size_t bits_cap = 0;
    uint32_t* d_out = nullptr;
    size_t out_cap = 0;
    char* d_slots = nullptr;
    size_t slots_cap = 0;
    GSlotHeader* d_ghdr = nullptr;
    size_t ghdr_cap = 0;
    uint32_t* d_key = nullptr;
    unsigned long long* d_job_failed = nullptr;
    size_t job_failed_cap = 0;
    std::map<std::string, TunedPlan> tuned;  // autotuner results by job mix
    std::string tune_text;
    std::string err, plan_text;
    uint32_t kernels = 0;
    Plan last_plan;
    Ctrl last_ctrl{};
    // tuning overrides (0 = automatic)
    uint32_t force_wg = 0, force_ng = 0, force_global_slots = 0, force_walkers = 0;
    uint32_t max_slots_per_group = 8;
    int force_walker_ctas = -1;  // -1 auto, 0 in-SM walker, N split engine
    int force_isolate = -1;      // -1 auto, 0 contiguous warp roles, 1 isolated walkers
    // batched calls: captured CUDA graphs of the device side, by call shape
    struct GraphEntry {
        std::string key;
        cudaGraphExec_t exec = nullptr;
        uint32_t kernels = 0, ctrl_count = 1;
        std::string plan_text;
        Plan plan;
    };
    int use_graphs = 1;
    int use_fused = 1;  // batched calls: all plan classes in one persistent launch
    bool capturing = false;
    std::vector<GraphEntry> graphs;  // most recent last, at most 8
    std::vector<std::string> graph_seen;
    unsigned long long* h_failed = nullptr;  // pinned per-job counts of the last batched call
    size_t h_failed_cap = 0;
    uint32_t* h_nf = nullptr;                // pinned failure count of the last batched call
    std::string graph_state;                 // "eager", "captured" or "replayed"
    int force_method = -1;  // -1 auto, 0 direct, 1 cache (shared if h <= 12, else global), 2 global cache
    int force_pool = -1;    // pooled direct passes: -1 auto, 0 off, 1 on where they apply
    bool plan_no_dfold = false;  // plan() re-run without room for direct passes' fold tables
    bool may_allocate = true;  // false: no global round cache, global slots only if unavoidable
    uint32_t spin_limit = 1u << 26;
    uint32_t map_chains = 0;  // lookup chains per lane from a round cache (0: automatic)
    uint32_t fill_blocks = 0; // round-cache fill: independent blocks per thread and step (0: automatic)

    ~Ctx();
    int init(int dev);
    int fail(int code, const char* fmt, ...);
    int cuda(cudaError_t e, const char* what);
    template <typename T>
    int grow(T*& ptr, size_t& cap, size_t need, const char* what);
    int make_job(const cmc_params& p, uint32_t first, uint32_t count, uint64_t base, Job& j);
    int plan(const std::vector<Job>& jobs, Plan& pl);
    int upload_jobs(const std::vector<Job>& jobs, cudaStream_t st);
    int run(const std::vector<Job>& jobs, uint64_t total, cudaStream_t st, uint32_t value_base,
            uint32_t* d_out, uint32_t* d_count, uint64_t out_cap, unsigned long long* job_failed,
            unsigned long long* job_done, const std::vector<uint32_t>* class_bounds = nullptr);
    int check_ctrl();
    int launch_host(const cmc_params& p, const uint32_t key[44], uint32_t first, uint32_t count,
                    uint32_t* out, uint32_t* nfailed);
    int launch_device(const cmc_params& p, const uint32_t* d_key, uint32_t first, uint32_t count,
                      uint32_t* d_offsets, uint32_t* d_nfailed, cudaStream_t st);
    int prepare_jobs(const cmc_job* in, uint32_t n, uint32_t sample_div, std::vector<Job>& out,
                     std::vector<uint32_t>& order, uint64_t& total, std::vector<uint32_t>& bounds);
    std::string mix_key(const cmc_job* in, uint32_t n) const;
    std::string graph_key(const std::vector<Job>& jobs, const std::vector<uint32_t>& bounds,
                          uint64_t total, uint64_t dev_cap) const;
    int run_jobs(const cmc_job* in, uint32_t n, uint64_t* out_failed, uint32_t* out_offsets,
                 uint32_t* out_jobs, uint64_t cap, uint64_t* out_total);
    int autotune(const cmc_job* in, uint32_t n, uint32_t sample_div);
};

}  // namespace cmc
