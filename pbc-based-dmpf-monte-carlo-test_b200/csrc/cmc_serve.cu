// cmc_serve.cu -- serving loop: estimation jobs of different sizes admitted as
// they arrive and run together in the persistent engine (continuous batching).
//
// Admitted jobs keep their state on the device: per-job failure and trial
// counts (the engine's counters, indexed by server slot) and, per published
// grant, a job-table entry with the batch key, the first offset and the
// count -- the job's RNG position (trial identity is (seed, batch, offset)).
// The host grants trials: most of the work (95% by default) in arrival order,
// so no job starves and the tail stays that of plain per-job launches, the
// rest shortest remaining work first.  Two ways to run the grants:
//
//   resident (default): one engine launch stays on the device while jobs are
//   pending.  The host writes grants into a job ring and publishes them
//   through mapped host memory; the launch's producer groups pick them up as
//   they claim trials; the host polls per-entry walk counts by copy and reads
//   back finished entries' failure bits.  The launch exits once every active
//   job's trials are published and walked: one launch tail per busy period.
//
//   iterations: each cmc_server_step issues one engine launch over one size
//   class of jobs (shared or global walk slots), pipelined two deep on two
//   streams; a device scheduler kernel turns the grants into the table,
//   deriving batch keys with device AES and advancing device RNG counters.
//
// Finished batches are appended to the job's v3 journal (optional), and
// finished jobs free their slot.  A job's results are identical alone and in
// the mix: trial identity does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <thread>
#include <memory>
#include <string>
#include <vector>

#include "cmc.h"
#include "cmc_aes.cuh"
#include "cmc_capi_internal.hpp"
#include "cmc_engine.cuh"
#include "cmc_grants.hpp"
#include "cmc_hostcore.hpp"
#include "cmc_runner.hpp"

namespace cmc {

__global__ void cmc_compact_failures(const uint32_t* bits, uint64_t nbits, uint32_t value_base,
                                     uint32_t* out, uint32_t* count, uint64_t cap,
                                     const unsigned long long* nbits_dev);

namespace {

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Key schedule from 16 key bytes given as two little-endian u64
// (cuckoo_bench.cu:86-99): word j packs bytes 4j..4j+3 most significant first.
__device__ void dev_expand_u64(const Lanes& L, uint64_t lo, uint64_t hi, uint32_t* rk) {
    expand_key(L, bswap32((uint32_t)lo), bswap32((uint32_t)(lo >> 32)), bswap32((uint32_t)hi),
               bswap32((uint32_t)(hi >> 32)), rk);
}

// batch_key(seed, id) (cuckoo_bench.cu:393-404) on the device.
__device__ void dev_batch_key(const Lanes& L, uint64_t seed, uint64_t id, uint32_t* rk) {
    uint32_t master[44], x[4];
    dev_expand_u64(L, seed, seed ^ 0x9e3779b97f4a7c15ULL, master);
    encrypt_full(L, master, 0x42415443u, (uint32_t)(id >> 32), (uint32_t)id, 0x50524731u, x);
    const uint64_t lo = ((uint64_t)x[0] << 32) | x[1];
    const uint64_t hi = ((uint64_t)x[2] << 32) | x[3];
    dev_expand_u64(L, seed ^ lo, hi ^ (seed ^ 0x243f6a8885a308d3ULL), rk);
}

// One CTA: grants -> engine job table (see the file comment).
__global__ void __launch_bounds__(256) serve_schedule(ServeState* __restrict__ states,
                                                     const Grant* __restrict__ grants,
                                                     uint32_t ngrants, const uint32_t* __restrict__ t0,
                                                     Job* __restrict__ table,
                                                     GrantInfo* __restrict__ info,
                                                     unsigned long long* __restrict__ total) {
    char* smem = cmc_dyn_smem;
    uint32_t* tw = reinterpret_cast<uint32_t*>(smem);
    for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) {
        const uint32_t v = t0[i >> 6];
        tw[i] = (i & 32) ? __funnelshift_r(v, v, 16) : v;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const Lanes L{lane * 4, lane * 4 + 128, 256u};
    for (uint32_t g = threadIdx.x; g < ngrants; g += blockDim.x) {
        ServeState& st = states[grants[g].slot];
        const uint64_t per = 1ULL << st.bt;
        const uint64_t batch = st.next >> st.bt, off = st.next & (per - 1);
        unsigned long long n = grants[g].trials;
        n = min(n, (unsigned long long)(st.budget - st.next));
        n = min(n, (unsigned long long)(per - off));
        if (batch != st.key_batch) {
            dev_batch_key(L, st.seed, batch, st.job.batch_rk);
            st.key_batch = batch;
        }
        Job j = st.job;
        j.first = (uint32_t)off;
        j.count = (uint32_t)n;
        j.user = grants[g].slot;
        table[g] = j;
        info[g].batch = batch;
        info[g].slot = grants[g].slot;
        info[g].first = (uint32_t)off;
        info[g].count = (uint32_t)n;
        st.next += n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long base = 0;
        for (uint32_t g = 0; g < ngrants; ++g) {
            table[g].trial_base = base;
            info[g].base = base;
            base += table[g].count;
        }
        *total = base;
    }
}

struct HostJob {
    uint32_t id = 0;
    cmc_params params{};
    uint64_t seed = 0, budget = 0;
    uint64_t next = 0;       // trials granted (issued to the device)
    uint64_t processed = 0;  // trials whose results the host has read back
    int state = 0;  // 0 queued, 1 active, 2 done
    uint32_t slot = 0;
    double cost = 1;  // estimated AES blocks per trial
    uint64_t failed = 0;
    uint64_t admitted_at = 0;  // iteration number
    int global_slots = 0;      // 1: its table needs walk slots in global memory
    double latency_blocks = 0; // one trial's latency, in AES blocks of GPU throughput
    // failing offsets per uncommitted batch, and the journal
    std::vector<std::pair<uint64_t, std::vector<uint32_t>>> pending;
    std::unique_ptr<Journal> journal;
    Options jopt;
    uint32_t bt = 20;
};

}  // namespace

// One iteration in flight: its stream, device buffers, pinned read-back
// buffers and the grants it carries.  Two of them alternate, so the host
// plans and issues iteration i+1 while iteration i runs, and the next engine's
// CTAs start on the SMs the previous engine's tail frees.
struct StepBuf {
    cudaStream_t stream = nullptr;
    cudaEvent_t sched_done = nullptr;  // job states advanced by this iteration's scheduler
    cudaEvent_t done = nullptr;        // everything of this iteration finished
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // around the engine launch (timing)
    uint64_t trials = 0;               // trials this iteration carries
    Grant* d_grants = nullptr;
    Job* d_table = nullptr;
    GrantInfo* d_info = nullptr;
    unsigned long long* d_total = nullptr;
    Ctrl* d_ctrl = nullptr;
    uint32_t* d_bits = nullptr;
    uint32_t* d_list = nullptr;  // failures of the iteration (+ count)
    char* d_pool = nullptr;      // global walk slots and round caches
    uint64_t pool_bytes = 0;
    Grant* h_grants = nullptr;   // pinned
    GrantInfo* h_info = nullptr; // pinned
    uint32_t* h_count = nullptr; // pinned
    Ctrl* h_ctrl = nullptr;      // pinned
    bool busy = false;
    std::vector<uint32_t> grant_jobs;  // job id of each grant
};

struct Server {
    Ctx* ctx = nullptr;
    uint32_t max_jobs = 0, bt = 20;
    uint64_t mem_budget = 0, max_iter_trials = 0, iteration = 0;
    ServeState* d_states = nullptr;
    ServeState* h_stage = nullptr;  // pinned staging of admitted job states
    unsigned long long* d_failed = nullptr;
    unsigned long long* d_done = nullptr;
    StepBuf bufs[2];
    uint32_t cur = 0;       // buffer of the next iteration
    bool sched_seen = false;  // some iteration's scheduler has been issued
    cudaEvent_t origin = nullptr;  // time origin of the engine intervals
    cmc_server_stats stats{};
    double last_end_ms = -1;     // end of the previous engine interval (from origin)
    double first_start_ms = 0;
    std::vector<HostJob> jobs;
    std::deque<uint32_t> queue;
    std::vector<uint32_t> free_slots;
    uint64_t fixed_bytes = 0;
    double fifo_share = 0.95;  // part of each step's work granted in arrival order
    std::string err;
    unsigned long long* h_zero = nullptr;  // pinned zeros: counter resets by copy, never by kernel

    // ---- resident mode: one engine launch stays on the device while work is
    // published to it (see step_resident) ----
    static constexpr uint32_t kRing = 4096;               // job-table ring entries
    static constexpr uint64_t kRingBits = 1ULL << 24;     // failure-bitmap ring (trials in flight)
    struct REntry {
        uint32_t job, count, first;
        uint64_t base, batch;
        bool consumed;
    };
    bool resident = true;
    bool r_ready = false, r_running = false, r_stopping = false;
    std::deque<REntry> rlive;          // published entries not yet reclaimed; front = entry r_front
    uint64_t r_front = 0, r_entries = 0;
    uint64_t r_avail = 0;              // trials published (global index end)
    uint64_t r_begin = 0;              // first trial of the running (or next) launch
    Plan r_plan;
    ResidentQueue* h_rq = nullptr;     // mapped pinned host memory
    ResidentQueue* d_rq = nullptr;     // its device address
    Job* d_ring = nullptr;
    Job* h_ring = nullptr;             // pinned staging, one per ring entry
    uint32_t* d_rdone = nullptr;
    uint32_t* h_rdone = nullptr;       // pinned
    uint32_t* d_rbits = nullptr;
    uint32_t* h_rbits = nullptr;       // pinned mirror of the bitmap ring
    Ctrl* d_rctrl = nullptr;
    Ctrl* h_rctrl = nullptr;           // pinned
    unsigned long long* h_rnext = nullptr;  // pinned: the running launch's claim counter
    uint64_t r_claimed = 0;            // trials the running launch has claimed (at the last poll)
    char* d_rpool = nullptr;
    uint64_t rpool_bytes = 0;
    cudaStream_t r_kstream = nullptr, r_cstream = nullptr;
    cudaEvent_t r_e0 = nullptr, r_e1 = nullptr, r_kdone = nullptr;

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return CMC_OK;
        return fail(CMC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
    ~Server() {
        for (StepBuf& b : bufs) {
            if (b.stream) cudaStreamSynchronize(b.stream);
        }
        for (StepBuf& b : bufs) {
            cudaFree(b.d_grants);
            cudaFree(b.d_table);
            cudaFree(b.d_info);
            cudaFree(b.d_total);
            cudaFree(b.d_ctrl);
            cudaFree(b.d_bits);
            cudaFree(b.d_list);
            cudaFree(b.d_pool);
            cudaFreeHost(b.h_grants);
            cudaFreeHost(b.h_info);
            cudaFreeHost(b.h_count);
            cudaFreeHost(b.h_ctrl);
            if (b.sched_done) cudaEventDestroy(b.sched_done);
            if (b.done) cudaEventDestroy(b.done);
            if (b.e0) cudaEventDestroy(b.e0);
            if (b.e1) cudaEventDestroy(b.e1);
            if (b.stream) cudaStreamDestroy(b.stream);
        }
        if (r_kstream) cudaStreamSynchronize(r_kstream);
        if (r_cstream) cudaStreamSynchronize(r_cstream);
        cudaFree(d_ring);
        cudaFree(d_rdone);
        cudaFree(d_rbits);
        cudaFree(d_rctrl);
        cudaFree(d_rpool);
        cudaFreeHost(h_rq);
        cudaFreeHost(h_ring);
        cudaFreeHost(h_rdone);
        cudaFreeHost(h_rbits);
        cudaFreeHost(h_rctrl);
        cudaFreeHost(h_rnext);
        cudaFreeHost(h_zero);
        for (cudaEvent_t e : {r_e0, r_e1, r_kdone})
            if (e) cudaEventDestroy(e);
        if (r_kstream) cudaStreamDestroy(r_kstream);
        if (r_cstream) cudaStreamDestroy(r_cstream);
        if (origin) cudaEventDestroy(origin);
        cudaFree(d_states);
        cudaFreeHost(h_stage);
        cudaFree(d_failed);
        cudaFree(d_done);
    }

    int init(Ctx* c, uint32_t mj, uint64_t budget, uint32_t batch_bits, uint64_t iter_trials) {
        ctx = c;
        max_jobs = mj;
        mem_budget = budget;
        bt = batch_bits;
        max_iter_trials = iter_trials;
        int rc = cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        if (rc) return rc;
        auto alloc = [&](void** p, size_t bytes, const char* what) {
            if (cudaMalloc(p, bytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, std::string("cudaMalloc for ") + what);
            }
            return CMC_OK;
        };
        auto host = [&](void** p, size_t bytes, const char* what) {
            if (cudaHostAlloc(p, bytes, cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, std::string("cudaHostAlloc for ") + what);
            }
            return CMC_OK;
        };
        const size_t words = (max_iter_trials + 31) / 32;
        if ((rc = alloc((void**)&d_states, sizeof(ServeState) * mj, "job states"))) return rc;
        if ((rc = host((void**)&h_stage, sizeof(ServeState) * mj, "job state staging"))) return rc;
        if ((rc = host((void**)&h_zero, 64, "zeros"))) return rc;
        std::memset(h_zero, 0, 64);
        if ((rc = alloc((void**)&d_failed, 8 * mj, "failure counters"))) return rc;
        if ((rc = alloc((void**)&d_done, 8 * mj, "trial counters"))) return rc;
        for (StepBuf& b : bufs) {
            if ((rc = cuda(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking), "stream"))) return rc;
            if ((rc = cuda(cudaEventCreateWithFlags(&b.sched_done, cudaEventDisableTiming), "event"))) return rc;
            if ((rc = cuda(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming), "event"))) return rc;
            if ((rc = cuda(cudaEventCreate(&b.e0), "event"))) return rc;
            if ((rc = cuda(cudaEventCreate(&b.e1), "event"))) return rc;
            if ((rc = alloc((void**)&b.d_grants, sizeof(Grant) * mj, "grants"))) return rc;
            if ((rc = alloc((void**)&b.d_table, sizeof(Job) * mj, "job table"))) return rc;
            if ((rc = alloc((void**)&b.d_info, sizeof(GrantInfo) * mj, "grant info"))) return rc;
            if ((rc = alloc((void**)&b.d_total, 8, "total"))) return rc;
            if ((rc = alloc((void**)&b.d_ctrl, sizeof(Ctrl), "control block"))) return rc;
            if ((rc = alloc((void**)&b.d_bits, words * 4, "failure bitmap"))) return rc;
            if ((rc = alloc((void**)&b.d_list, (max_iter_trials + 1) * 4, "failure list"))) return rc;
            if ((rc = host((void**)&b.h_grants, sizeof(Grant) * mj, "grants"))) return rc;
            if ((rc = host((void**)&b.h_info, sizeof(GrantInfo) * mj, "grant info"))) return rc;
            if ((rc = host((void**)&b.h_count, 4, "count"))) return rc;
            if ((rc = host((void**)&b.h_ctrl, sizeof(Ctrl), "control block"))) return rc;
        }
        fixed_bytes = (sizeof(ServeState) + 16) * mj +
                      2 * ((sizeof(Grant) + sizeof(Job) + sizeof(GrantInfo)) * mj + words * 4 +
                           (max_iter_trials + 1) * 4 + 8 + sizeof(Ctrl));
        if (fixed_bytes > mem_budget) return fail(CMC_ENOMEM, "device-memory budget below the server's fixed state");
        for (uint32_t s = mj; s-- > 0;) free_slots.push_back(s);
        if ((rc = cuda(cudaMemsetAsync(d_failed, 0, 8 * mj, bufs[0].stream), "memset"))) return rc;
        if ((rc = cuda(cudaMemsetAsync(d_done, 0, 8 * mj, bufs[0].stream), "memset"))) return rc;
        if ((rc = cuda(cudaEventCreate(&origin), "event"))) return rc;
        if ((rc = cuda(cudaEventRecord(origin, bufs[0].stream), "event"))) return rc;
        if ((rc = cuda(cudaStreamSynchronize(bufs[0].stream), "init sync"))) return rc;
        if ((rc = cuda(cudaFuncSetAttribute((const void*)serve_schedule,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes),
                       "scheduler attribute")))
            return rc;
        return resident ? resident_setup() : CMC_OK;  // the first step then allocates nothing
    }

    // Plan for a set of active parameter sets; returns the global pool bytes
    // the plan needs: walk slots (0 for shared-memory slots), then round caches.
    int plan_for(const std::vector<uint32_t>& ids, Plan& pl, std::vector<Job>& shapes, uint64_t& pool,
                 const std::vector<uint32_t>* weights = nullptr) {
        shapes.clear();
        for (size_t i = 0; i < ids.size(); ++i) {
            Job j;
            int rc = ctx->make_job(jobs[ids[i]].params, 0, weights ? (*weights)[i] : 1, 0, j);
            if (rc) return fail(rc, ctx->err);
            shapes.push_back(j);
        }
        int rc = ctx->plan(shapes, pl);
        if (rc) return fail(rc, ctx->err);
        pool = cache_offset(pl) + pl.gcache_bytes;
        return CMC_OK;
    }

    static uint64_t cache_offset(const Plan& pl) { return (pl.gslot_bytes + 255) / 256 * 256; }

    // Admitted, unfinished jobs in admission order, and the number of jobs not
    // finished yet: kept up to date so that a long-lived server's steps do not
    // scan every job it has ever seen.
    std::vector<uint32_t> active_list;
    uint32_t unfinished = 0;

    std::vector<uint32_t> active_ids() const { return active_list; }

    void activate(HostJob& j) {
        j.state = 1;
        active_list.push_back(j.id);
    }

    void finish(HostJob& j) {
        if (j.state == 1) active_list.erase(std::find(active_list.begin(), active_list.end(), j.id));
        j.state = 2;
        --unfinished;
    }

    int submit(const cmc_params& p, uint64_t seed, uint64_t trials, const char* journal_dir,
               uint32_t* out_id) {
        if (trials == 0) return fail(CMC_EINVAL, "a job needs at least one trial");
        Job probe;
        int rc = ctx->make_job(p, 0, 1, 0, probe);
        if (rc) return fail(rc, ctx->err);
        HostJob j;
        j.id = uint32_t(jobs.size());
        j.params = p;
        j.seed = seed;
        j.budget = trials;
        // batches of 2^bt trials, the experiment sized to the next power of two
        // A budget runs as the first ceil(trials / 2^bt) batches of an experiment
        // of 2^et trials, et = ceil(log2 trials): a prefix of the reference's
        // own batches, so the budget is rounded up to whole batches.
        uint32_t et = 0;
        while ((1ULL << et) < trials) ++et;
        j.bt = std::min(bt, std::max(et, 1u));
        j.budget = ((trials + (1ULL << j.bt) - 1) >> j.bt) << j.bt;
        j.cost = job_cost(probe) + 0.2 * p.pnum;
        {
            // size class: do this table's walk slots fit in shared memory?
            std::vector<Job> one(1);
            one[0] = probe;
            Plan pl;
            if ((rc = ctx->plan(one, pl))) return fail(rc, ctx->err);
            j.global_slots = pl.slots_smem ? 0 : 1;
            // a trial's walk is ~2.4 t probes of ~300 (shared) or ~3000 (global)
            // cycles; expressed in blocks of GPU throughput (~4e10 blocks/s at 2 GHz)
            const double walk_cycles = 2.4 * p.pnum * (j.global_slots ? 3000.0 : 300.0);
            j.latency_blocks = walk_cycles / 2.0e9 * 4.0e10;
        }
        if (journal_dir && *journal_dir) {
            Options& o = j.jopt;
            o.mode = p.mode == CMC_MODE_BGH25 ? "bgh25" : "drrt18";
            o.input_mode = p.input_mode == CMC_INPUT_SEQUENTIAL ? "sequential" : "affine";
            o.pnum = p.pnum;
            o.ell_i = p.ell_i;
            o.k = p.k;
            o.buckets = p.buckets;
            o.max_kicks = p.kick;
            o.seed = seed;
            o.et = std::max(et, 1u);
            o.bt = j.bt;
            o.out = journal_dir;
            try {
                fs::create_directories(o.out);
                Counters c0;
                const std::vector<uint8_t> done = resume(o, p, c0);
                // resume from the first batch not yet committed (prefix runs)
                uint64_t b = 0;
                while (b < done.size() && done[b]) ++b;
                j.next = std::min<uint64_t>(j.budget, b << j.bt);
                j.processed = j.next;
                j.failed = c0.failed.load();  // committed failures of the prefix
                j.journal.reset(new Journal(o, p, 0));
            } catch (const std::exception& e) {
                return fail(CMC_EINVAL, std::string("journal: ") + e.what());
            }
        }
        jobs.push_back(std::move(j));
        queue.push_back(jobs.back().id);
        ++unfinished;
        if (out_id) *out_id = jobs.back().id;
        return CMC_OK;
    }

    // Admission on the stream of the next iteration: job state from pinned
    // staging (slot s's staging entry is rewritten only after the job in slot s
    // retired, i.e. after its upload was long consumed) and zeroed counters.
    int admit(cudaStream_t st) {
        while (!queue.empty() && !free_slots.empty()) {
            const uint32_t id = queue.front();
            HostJob& j = jobs[id];
            if (j.next >= j.budget) {  // fully journaled already
                queue.pop_front();
                finish(j);
                continue;
            }
            std::vector<uint32_t> ids = active_ids();
            ids.push_back(id);
            Plan pl;
            std::vector<Job> shapes;
            uint64_t pool = 0;
            int rc = plan_for(ids, pl, shapes, pool);
            if (rc) return rc;
            if (fixed_bytes + 2 * pool > mem_budget) {  // two iterations in flight
                if (ids.size() == 1)
                    return fail(CMC_ENOMEM, "job " + std::to_string(id) +
                                                " alone needs more device memory than the budget");
                break;  // wait for memory to free up
            }
            queue.pop_front();
            j.slot = free_slots.back();
            free_slots.pop_back();
            activate(j);
            j.admitted_at = iteration;
            ServeState state{};
            rc = ctx->make_job(j.params, 0, 1, 0, state.job);
            if (rc) return fail(rc, ctx->err);
            state.seed = j.seed;
            state.next = j.next;
            state.budget = j.budget;
            state.key_batch = ~0ULL;
            state.bt = j.bt;
            state.active = 1;
            h_stage[j.slot] = state;
            if ((rc = cuda(cudaMemcpyAsync(&d_states[j.slot], &h_stage[j.slot], sizeof state,
                                           cudaMemcpyHostToDevice, st), "upload job state")))
                return rc;
            if ((rc = cuda(cudaMemcpyAsync(&d_failed[j.slot], h_zero, 8, cudaMemcpyHostToDevice, st),
                           "reset counter")))
                return rc;
            if ((rc = cuda(cudaMemcpyAsync(&d_done[j.slot], h_zero, 8, cudaMemcpyHostToDevice, st),
                           "reset counter")))
                return rc;
        }
        return CMC_OK;
    }

    // One iteration: admit, plan and issue this iteration's grants, then read
    // back the previous iteration's results (which ran meanwhile) and commit
    // them.  Jobs finish in the call after their last trials were issued.
    int step(uint64_t work_blocks, uint32_t* finished, uint32_t cap, uint32_t* nfinished) {
        if (nfinished) *nfinished = 0;
        int rc = cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        if (rc) return rc;
        if (resident || r_running) return step_resident(work_blocks, finished, cap, nfinished);
        StepBuf& b = bufs[cur];
        StepBuf& prev = bufs[cur ^ 1];
        if (b.busy && (rc = process(b, finished, cap, nfinished))) return rc;  // not reached in order
        if ((rc = admit(b.stream))) return rc;
        std::vector<Grant> grants;
        std::vector<uint32_t> grant_jobs;
        if ((rc = plan_grants(work_blocks, grants, grant_jobs))) return rc;
        if (!grants.empty()) {
            if ((rc = issue(b, grants, grant_jobs))) return rc;
            cur ^= 1;
        }
        if (prev.busy) {
            uint32_t n = nfinished ? *nfinished : 0;
            if ((rc = process(prev, finished ? finished + std::min(n, cap) : nullptr, cap - std::min(n, cap),
                              &n)))
                return rc;
            if (nfinished) *nfinished += n;
        }
        return CMC_OK;
    }

    // Finishes every iteration in flight (used before the server goes away,
    // so journals hold every batch the device completed).
    int drain() {
        if (r_ready) {
            int rc = resident_close();
            if (rc) return rc;
        }
        for (int i = 0; i < 2; ++i) {
            StepBuf& b = bufs[(cur + i) & 1];  // oldest first
            if (b.busy) {
                int rc = process(b, nullptr, 0, nullptr);
                if (rc) return rc;
            }
        }
        return CMC_OK;
    }

    int plan_grants(uint64_t work_blocks, std::vector<Grant>& grants, std::vector<uint32_t>& grant_jobs,
                    bool one_class = true) {
        std::vector<uint32_t> all;  // active jobs with trials left to issue
        for (uint32_t id : active_ids())
            if (jobs[id].next < jobs[id].budget) all.push_back(id);
        if (all.empty()) return CMC_OK;
        // One size class per step, so the plan keeps shared-memory walk slots
        // whenever the granted tables allow: alternately the class of the
        // oldest job and the class of the job with the least remaining work.
        uint32_t oldest = all[0], smallest = all[0];
        auto remaining = [&](uint32_t id) { return double(jobs[id].budget - jobs[id].next) * jobs[id].cost; };
        for (uint32_t id : all) {
            if (jobs[id].admitted_at < jobs[oldest].admitted_at) oldest = id;
            if (remaining(id) < remaining(smallest)) smallest = id;
        }
        const int cls = (iteration % 2 == 1) ? jobs[oldest].global_slots : jobs[smallest].global_slots;
        std::vector<uint32_t> ids;
        for (uint32_t id : all)
            if (!one_class || jobs[id].global_slots == cls) ids.push_back(id);
        // the policy itself (cmc_grants.hpp): work size, arrival-order and
        // shortest-work shares, batch boundaries, heaviest-first order
        std::vector<GrantCandidate> cands;
        for (uint32_t id : ids) {
            const HostJob& j = jobs[id];
            cands.push_back(GrantCandidate{id, j.next, j.budget, j.bt, j.cost, j.latency_blocks, j.admitted_at});
        }
        for (const GrantShare& g : grant_shares(cands, work_blocks, fifo_share, max_iter_trials)) {
            HostJob& j = jobs[g.id];
            grants.push_back(Grant{j.slot, uint32_t(g.trials)});
            grant_jobs.push_back(g.id);
            j.next += g.trials;
        }
        return CMC_OK;
    }

    // Queue one iteration on b's stream: grants -> scheduler -> engine ->
    // compaction -> read-back into pinned memory.
    int issue(StepBuf& b, const std::vector<Grant>& grants, const std::vector<uint32_t>& grant_jobs) {
        int rc = CMC_OK;
        cudaStream_t st = b.stream;
        std::vector<uint32_t> weights;  // the plan weighs each shape by its granted trials
        for (const Grant& g : grants) weights.push_back(g.trials);
        Plan pl;
        std::vector<Job> shapes;
        uint64_t pool = 0;
        if ((rc = plan_for(grant_jobs, pl, shapes, pool, &weights))) return rc;
        if (pool > b.pool_bytes) {
            // grow with headroom (within the budget): each regrowth's cudaFree
            // waits for the device and drains the pipeline
            const uint64_t room = mem_budget > fixed_bytes ? (mem_budget - fixed_bytes) / 2 : pool;
            const uint64_t want = std::max(pool, std::min<uint64_t>(pool + pool / 2, room));
            cudaFree(b.d_pool);
            b.d_pool = nullptr;
            b.pool_bytes = 0;
            if (cudaMalloc((void**)&b.d_pool, want) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, "slot pool");
            }
            b.pool_bytes = want;
        }
        std::copy(grants.begin(), grants.end(), b.h_grants);
        if ((rc = cuda(cudaMemcpyAsync(b.d_grants, b.h_grants, grants.size() * sizeof(Grant),
                                       cudaMemcpyHostToDevice, st), "upload grants")))
            return rc;
        // schedulers run in issue order: each advances the RNG counters the
        // next one starts from
        cudaGetLastError();  // launch checks below read it: drop earlier non-fatal errors
        const StepBuf& other = bufs[(&b == &bufs[0]) ? 1 : 0];
        if (sched_seen && (rc = cuda(cudaStreamWaitEvent(st, other.sched_done, 0), "order schedulers")))
            return rc;
        serve_schedule<<<1, 256, kTableBytes, st>>>(d_states, b.d_grants, uint32_t(grants.size()), ctx->d_t0,
                                                    b.d_table, b.d_info, b.d_total);
        if ((rc = cuda(cudaGetLastError(), "scheduler launch"))) return rc;
        if ((rc = cuda(cudaEventRecord(b.sched_done, st), "event"))) return rc;
        sched_seen = true;
        if ((rc = cuda(cudaMemsetAsync(b.d_ctrl, 0, sizeof(Ctrl), st), "memset ctrl"))) return rc;
        if ((rc = cuda(cudaMemsetAsync(b.d_bits, 0, (max_iter_trials + 31) / 32 * 4, st), "memset bitmap")))
            return rc;
        EngineArgs a{};
        a.jobs = b.d_table;
        a.njobs = uint32_t(grants.size());
        a.total = 0;
        a.total_dev = b.d_total;
        a.count_by_user = 1;
        a.ctrl = b.d_ctrl;
        a.fail_bits = b.d_bits;
        a.job_failed = d_failed;
        a.job_done = d_done;
        a.gslots = pl.slots_smem ? nullptr : b.d_pool;
        a.gcache = pl.gcache_bytes ? reinterpret_cast<uint16_t*>(b.d_pool + cache_offset(pl)) : nullptr;
        a.gcache_stride = pl.gcache_stride;
        a.t0 = ctx->d_t0;
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
        a.spin_limit = ctx->spin_limit;
        a.idle_polls = ctx->spin_limit;
        a.map_chains = ctx->map_chains;
        a.fill_blocks = ctx->fill_blocks;
        a.pool_stage = pl.pool_stage;
        a.pool_fold = pl.pool_fold;
        const void* fn = engine_kernel(pl.variant, pl.slots_smem, pl.pool_stage != 0);
        // the context raised the engine's shared-memory limit to the device maximum
        void* args[] = {&a};
        if ((rc = cuda(cudaEventRecord(b.e0, st), "event"))) return rc;
        if ((rc = cuda(cudaLaunchKernel(fn, dim3(pl.ctas), dim3(pl.threads), args, pl.smem_bytes, st),
                       "engine launch")))
            return rc;
        if ((rc = cuda(cudaEventRecord(b.e1, st), "event"))) return rc;
        cmc_compact_failures<<<1, 1024, 0, st>>>(b.d_bits, 0, 0, b.d_list, b.d_list + max_iter_trials,
                                                 max_iter_trials, b.d_total);
        if ((rc = cuda(cudaGetLastError(), "compaction launch"))) return rc;
        if ((rc = cuda(cudaMemcpyAsync(b.h_info, b.d_info, grants.size() * sizeof(GrantInfo),
                                       cudaMemcpyDeviceToHost, st), "read grant info")))
            return rc;
        if ((rc = cuda(cudaMemcpyAsync(b.h_count, b.d_list + max_iter_trials, 4, cudaMemcpyDeviceToHost, st),
                       "read count")))
            return rc;
        if ((rc = cuda(cudaMemcpyAsync(b.h_ctrl, b.d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st),
                       "read ctrl")))
            return rc;
        if ((rc = cuda(cudaEventRecord(b.done, st), "event"))) return rc;
        b.grant_jobs = grant_jobs;
        b.trials = 0;
        for (const Grant& g : grants) b.trials += g.trials;
        b.busy = true;
        ++iteration;
        return CMC_OK;
    }

    // Wait for b's iteration, map its failures back to (job, batch, offset),
    // commit completed batches to journals and retire finished jobs.
    int process(StepBuf& b, uint32_t* finished, uint32_t cap, uint32_t* nfinished) {
        if (nfinished) *nfinished = 0;
        b.busy = false;
        int rc = cuda(cudaEventSynchronize(b.done), "iteration sync");
        if (rc) return rc;
        if (b.h_ctrl->error)
            return fail(-int(b.h_ctrl->error), std::string(ctrl_error_text(b.h_ctrl->error)) + " (site " +
                                                   std::to_string(b.h_ctrl->where) + "): results discarded");
        {
            float t0 = 0, t1 = 0;
            if ((rc = cuda(cudaEventElapsedTime(&t0, origin, b.e0), "engine timing"))) return rc;
            if ((rc = cuda(cudaEventElapsedTime(&t1, origin, b.e1), "engine timing"))) return rc;
            stats.iterations += 1;
            stats.trials += b.trials;
            stats.engine_ms += t1 - t0;
            // engines of consecutive iterations may overlap: count device time once
            stats.busy_ms += std::max(0.0, double(t1) - std::max(double(t0), last_end_ms));
            if (stats.iterations == 1) first_start_ms = t0;
            last_end_ms = std::max(last_end_ms, double(t1));
            stats.span_ms = last_end_ms - first_start_ms;
        }
        const uint32_t nf = *b.h_count;
        std::vector<uint32_t> fl(nf);
        if (nf) {
            if ((rc = cuda(cudaMemcpyAsync(fl.data(), b.d_list, nf * 4ULL, cudaMemcpyDeviceToHost, b.stream),
                           "read failures")))
                return rc;
            if ((rc = cuda(cudaStreamSynchronize(b.stream), "read failures"))) return rc;
        }
        // failures of this iteration into their job's pending batch lists
        size_t gi = 0;
        for (uint32_t g = 0; g < b.grant_jobs.size(); ++g) {
            const GrantInfo& info = b.h_info[g];
            HostJob& j = jobs[b.grant_jobs[g]];
            auto& pend = j.pending;
            if (pend.empty() || pend.back().first != info.batch) pend.push_back({info.batch, {}});
            while (gi < fl.size() && fl[gi] < info.base + info.count) {
                pend.back().second.push_back(info.first + uint32_t(fl[gi] - info.base));
                ++j.failed;
                ++gi;
            }
            j.processed += info.count;
        }
        // commit finished batches, retire finished jobs
        uint32_t nfin = 0;
        for (uint32_t id : b.grant_jobs) {
            HostJob& j = jobs[id];
            const uint64_t per = 1ULL << j.bt;
            while (!j.pending.empty()) {
                const uint64_t bb = j.pending.front().first;
                const uint64_t end = std::min<uint64_t>((bb + 1) << j.bt, j.budget);
                if (j.processed < end) break;  // batch not complete yet
                auto& offs = j.pending.front().second;
                std::sort(offs.begin(), offs.end());
                if (j.journal) {
                    try {
                        j.journal->append(bb, uint32_t(std::min<uint64_t>(per, batch_length(j.jopt, bb))), offs);
                    } catch (const std::exception& e) {
                        return fail(CMC_EINVAL, std::string("journal: ") + e.what());
                    }
                }
                j.pending.erase(j.pending.begin());
            }
            if (j.state == 1 && j.processed >= j.budget && j.pending.empty()) {
                finish(j);
                j.journal.reset();
                free_slots.push_back(j.slot);
                if (finished && nfin < cap) finished[nfin] = id;
                ++nfin;
            }
        }
        if (nfinished) *nfinished = nfin;
        return CMC_OK;
    }

    // ------------------------------------------------------------ resident --
    //
    // One engine launch stays on the device while jobs are served.  The host
    // writes job entries (one per grant, batch key derived on the host) into
    // a device ring by copy, waits for the copy, then raises `avail` in mapped
    // host memory; producer groups claim trial indices, wait (bounded) until
    // they are published, and find their entry by scanning the ring forward.
    // Walkers count finished walks per entry; the host polls those counts by
    // copy and reads the finished entries' failure bits.  When no active job
    // has trials left to publish, the host raises `stop`: the launch finishes
    // what was published and exits, so a busy period pays one launch tail (a
    // plain launch pays one per job).  Nothing is queued on the device that
    // needs an SM while the launch runs: counters and control words are reset
    // by copies.

    int resident_setup() {
        if (r_ready) return CMC_OK;
        auto alloc = [&](void** p, size_t bytes, const char* what) {
            if (cudaMalloc(p, bytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, std::string("cudaMalloc for ") + what);
            }
            return CMC_OK;
        };
        auto host = [&](void** p, size_t bytes, unsigned flags, const char* what) {
            if (cudaHostAlloc(p, bytes, flags) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, std::string("cudaHostAlloc for ") + what);
            }
            return CMC_OK;
        };
        int rc;
        if ((rc = host((void**)&h_rq, sizeof(ResidentQueue), cudaHostAllocMapped, "resident queue"))) return rc;
        std::memset(h_rq, 0, sizeof(ResidentQueue));
        if ((rc = cuda(cudaHostGetDevicePointer((void**)&d_rq, h_rq, 0), "map resident queue"))) return rc;
        if ((rc = alloc((void**)&d_ring, sizeof(Job) * kRing, "job ring"))) return rc;
        if ((rc = host((void**)&h_ring, sizeof(Job) * kRing, cudaHostAllocDefault, "job ring staging"))) return rc;
        if ((rc = alloc((void**)&d_rdone, 4 * kRing, "entry counts"))) return rc;
        if ((rc = host((void**)&h_rdone, 4 * kRing, cudaHostAllocDefault, "entry counts"))) return rc;
        if ((rc = alloc((void**)&d_rbits, kRingBits / 8, "bitmap ring"))) return rc;
        if ((rc = host((void**)&h_rbits, kRingBits / 8, cudaHostAllocDefault, "bitmap ring"))) return rc;
        if ((rc = alloc((void**)&d_rctrl, sizeof(Ctrl), "control block"))) return rc;
        if ((rc = host((void**)&h_rctrl, sizeof(Ctrl), cudaHostAllocDefault, "control block"))) return rc;
        if ((rc = host((void**)&h_rnext, 8, cudaHostAllocDefault, "claim counter"))) return rc;
        if ((rc = cuda(cudaStreamCreateWithFlags(&r_kstream, cudaStreamNonBlocking), "stream"))) return rc;
        if ((rc = cuda(cudaStreamCreateWithFlags(&r_cstream, cudaStreamNonBlocking), "stream"))) return rc;
        if ((rc = cuda(cudaEventCreate(&r_e0), "event"))) return rc;
        if ((rc = cuda(cudaEventCreate(&r_e1), "event"))) return rc;
        if ((rc = cuda(cudaEventCreateWithFlags(&r_kdone, cudaEventDisableTiming), "event"))) return rc;
        // no launch runs yet: plain memsets are fine here
        if ((rc = cuda(cudaMemsetAsync(d_rbits, 0, kRingBits / 8, r_cstream), "memset"))) return rc;
        if ((rc = cuda(cudaMemsetAsync(d_rdone, 0, 4 * kRing, r_cstream), "memset"))) return rc;
        if ((rc = cuda(cudaStreamSynchronize(r_cstream), "resident setup"))) return rc;
        r_ready = true;
        return CMC_OK;
    }

    // Plan of a resident launch: global walk slots with four isolated walker
    // warps (slot count does not depend on the table size), sized for every
    // active and queued job.
    int resident_plan(Plan& pl, uint64_t& pool) {
        std::vector<uint32_t> ids = active_ids();
        for (uint32_t id : queue) ids.push_back(id);
        const uint32_t gs = ctx->force_global_slots, wk = ctx->force_walkers;
        const int iso = ctx->force_isolate, wc = ctx->force_walker_ctas;
        ctx->force_global_slots = 1;
        ctx->force_isolate = 1;
        ctx->force_walkers = 4;
        ctx->force_walker_ctas = 0;
        std::vector<Job> shapes;
        const int rc = plan_for(ids, pl, shapes, pool);
        ctx->force_global_slots = gs;
        ctx->force_walkers = wk;
        ctx->force_isolate = iso;
        ctx->force_walker_ctas = wc;
        return rc;
    }

    // Can job `id` run under the running launch's plan (slot size, entry width)?
    bool fits(uint32_t id) {
        Plan one;
        uint64_t pool = 0;
        std::vector<Job> shapes;
        if (plan_for({id}, one, shapes, pool)) return false;
        const uint32_t entry = r_plan.variant ? 4 : 2;
        const Job& j = shapes[0];
        const uint64_t bins = (uint64_t(j.buckets) * entry + 15) / 16 * 16;
        const uint64_t map = (uint64_t(j.pnum) * j.k * entry + 15) / 16 * 16;
        // the map of every slot starts at the plan's bins_bytes
        return one.variant <= r_plan.variant && bins <= r_plan.bins_bytes &&
               r_plan.bins_bytes + map <= r_plan.slot_stride;
    }

    // Published trials no producer has claimed yet, in AES-block equivalents:
    // the work that keeps the running launch busy until the next publication.
    double resident_unclaimed() const {
        double w = 0;
        for (const REntry& e : rlive) {
            const uint64_t end = e.base + e.count;
            if (end > r_claimed) w += double(end - std::max(e.base, r_claimed)) * jobs[e.job].cost;
        }
        return w;
    }

    // Publishes one chunk of grants (returns the number of entries published).
    int resident_publish(uint64_t work_blocks, uint32_t& published) {
        published = 0;
        std::vector<Grant> grants;
        std::vector<uint32_t> grant_jobs;
        int rc = plan_grants(work_blocks, grants, grant_jobs, /*one_class=*/false);
        if (rc) return rc;
        size_t n = 0;
        for (; n < grants.size(); ++n) {
            const uint32_t id = grant_jobs[n];
            const uint64_t bits_front = rlive.empty() ? r_avail : rlive.front().base;
            const bool room = rlive.size() + 1 <= kRing && r_avail + grants[n].trials - bits_front <= kRingBits;
            if (!room || (r_running && !fits(id))) break;
            HostJob& j = jobs[id];
            const uint64_t first_trial = j.next - grants[n].trials;  // plan_grants advanced next
            const uint64_t per = 1ULL << j.bt;
            REntry e{id, grants[n].trials, uint32_t(first_trial & (per - 1)), r_avail, first_trial >> j.bt, false};
            Job& d = h_ring[r_entries % kRing];
            if ((rc = ctx->make_job(j.params, e.first, e.count, e.base, d))) return fail(rc, ctx->err);
            batch_key(j.seed, e.batch, d.batch_rk);
            d.user = j.slot;
            const uint32_t slot = uint32_t(r_entries % kRing);
            if ((rc = cuda(cudaMemcpyAsync(&d_ring[slot], &d, sizeof(Job), cudaMemcpyHostToDevice, r_cstream),
                           "publish entry")))
                return rc;
            if ((rc = cuda(cudaMemcpyAsync(&d_rdone[slot], h_zero, 4, cudaMemcpyHostToDevice, r_cstream),
                           "publish entry")))
                return rc;
            rlive.push_back(e);
            ++r_entries;
            r_avail += e.count;
            ++published;
        }
        // grants that did not fit go back to their jobs
        for (size_t i = n; i < grants.size(); ++i) jobs[grant_jobs[i]].next -= grants[i].trials;
        if (published) {
            // the entries are in device memory before `avail` admits them
            if ((rc = cuda(cudaStreamSynchronize(r_cstream), "publish"))) return rc;
            __atomic_store_n(&h_rq->avail, (unsigned long long)r_avail, __ATOMIC_RELEASE);
        }
        if (n < grants.size() && r_running && !fits(grant_jobs[n])) {
            // a larger table than the running plan holds: close this launch;
            // the next one is planned for it
            __atomic_store_n(&h_rq->stop, 1u, __ATOMIC_RELEASE);
            r_stopping = true;
        }
        return CMC_OK;
    }

    int resident_launch() {
        Plan pl;
        uint64_t pool = 0;
        int rc = resident_plan(pl, pool);
        if (rc) return rc;
        if (pool > rpool_bytes) {
            cudaFree(d_rpool);
            d_rpool = nullptr;
            rpool_bytes = 0;
            if (cudaMalloc((void**)&d_rpool, pool) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, "resident slot pool");
            }
            rpool_bytes = pool;
        }
        // the entry holding the launch's first trial
        uint64_t e_begin = r_front;
        for (const REntry& e : rlive) {
            if (r_begin >= e.base && r_begin - e.base < e.count) break;
            ++e_begin;
        }
        if (e_begin == r_front + rlive.size()) return fail(CMC_EINVAL, "resident launch without published work");
        __atomic_store_n(&h_rq->stop, 0u, __ATOMIC_RELEASE);
        cudaStream_t st = r_kstream;
        if ((rc = cuda(cudaMemcpyAsync(d_rctrl, h_zero, sizeof(Ctrl) <= 64 ? sizeof(Ctrl) : 64,
                                       cudaMemcpyHostToDevice, st), "reset ctrl")))
            return rc;
        static_assert(sizeof(Ctrl) <= 64, "control block reset copies 64 zero bytes");
        EngineArgs a{};
        a.jobs = d_ring;
        a.njobs = kRing;
        a.total = ~0ULL;
        a.gidx_begin = r_begin;
        a.ctrl = d_rctrl;
        a.fail_bits = d_rbits;
        a.bits_mask = kRingBits - 1;
        a.job_failed = d_failed;
        a.job_done = d_done;
        a.count_by_user = 1;
        a.rq = d_rq;
        a.ring_mask = kRing - 1;
        a.entry_begin = e_begin;
        a.entry_done = d_rdone;
        // walkers idle while producers wait on the host for new work: give
        // them a bound in polls well past the producers' bound in time
        a.idle_polls = uint32_t(std::min<uint64_t>(0xffffffffULL, 32ULL * ctx->spin_limit));
        a.gslots = pl.slots_smem ? nullptr : d_rpool;
        a.gcache = pl.gcache_bytes ? reinterpret_cast<uint16_t*>(d_rpool + cache_offset(pl)) : nullptr;
        a.gcache_stride = pl.gcache_stride;
        a.t0 = ctx->d_t0;
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
        a.spin_limit = ctx->spin_limit;
        a.map_chains = ctx->map_chains;
        a.fill_blocks = ctx->fill_blocks;
        // the resident launch claims trials from the host's ring: plain producers
        const void* fn = engine_kernel(pl.variant, pl.slots_smem);
        // the context raised the engine's shared-memory limit to the device maximum
        void* args[] = {&a};
        if ((rc = cuda(cudaEventRecord(r_e0, st), "event"))) return rc;
        if ((rc = cuda(cudaLaunchKernel(fn, dim3(pl.ctas), dim3(pl.threads), args, pl.smem_bytes, st),
                       "resident launch")))
            return rc;
        if ((rc = cuda(cudaEventRecord(r_e1, st), "event"))) return rc;
        if ((rc = cuda(cudaMemcpyAsync(h_rctrl, d_rctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st), "read ctrl")))
            return rc;
        if ((rc = cuda(cudaEventRecord(r_kdone, st), "event"))) return rc;
        r_plan = pl;
        r_running = true;
        r_stopping = false;
        return CMC_OK;
    }

    // The launch has exited: check it and account its device time.
    int resident_finished() {
        int rc = cuda(cudaEventSynchronize(r_kdone), "resident sync");
        if (rc) return rc;
        r_running = false;
        r_stopping = false;
        r_begin = r_avail;  // every published trial was claimed and walked
        if (h_rctrl->error)
            return fail(-int(h_rctrl->error), std::string(ctrl_error_text(h_rctrl->error)) + " (site " +
                                                  std::to_string(h_rctrl->where) + "): results discarded");
        float t0 = 0, t1 = 0;
        if ((rc = cuda(cudaEventElapsedTime(&t0, origin, r_e0), "engine timing"))) return rc;
        if ((rc = cuda(cudaEventElapsedTime(&t1, origin, r_e1), "engine timing"))) return rc;
        stats.iterations += 1;
        stats.engine_ms += t1 - t0;
        stats.busy_ms += std::max(0.0, double(t1) - std::max(double(t0), last_end_ms));
        if (stats.iterations == 1) first_start_ms = t0;
        last_end_ms = std::max(last_end_ms, double(t1));
        stats.span_ms = last_end_ms - first_start_ms;
        return CMC_OK;
    }

    // Reads finished entries back; returns how many entries it consumed.
    int resident_poll(uint32_t& consumed) {
        consumed = 0;
        int rc;
        if (r_running) {
            if ((rc = cuda(cudaMemcpyAsync(h_rnext, &d_rctrl->next, 8, cudaMemcpyDeviceToHost, r_cstream),
                           "poll")))
                return rc;
            if ((rc = cuda(cudaStreamSynchronize(r_cstream), "poll"))) return rc;
            r_claimed = std::min<uint64_t>(r_begin + *h_rnext, r_avail);
        } else {
            r_claimed = r_begin;
        }
        if (rlive.empty()) return CMC_OK;
        const uint32_t lo = uint32_t(r_front % kRing), n = uint32_t(rlive.size());
        const uint32_t n1 = std::min(n, kRing - lo);
        if ((rc = cuda(cudaMemcpyAsync(h_rdone + lo, d_rdone + lo, 4ULL * n1, cudaMemcpyDeviceToHost, r_cstream),
                       "poll")))
            return rc;
        if (n > n1 && (rc = cuda(cudaMemcpyAsync(h_rdone, d_rdone, 4ULL * (n - n1), cudaMemcpyDeviceToHost,
                                                 r_cstream), "poll")))
            return rc;
        if ((rc = cuda(cudaStreamSynchronize(r_cstream), "poll"))) return rc;
        std::vector<size_t> ready;
        for (size_t i = 0; i < rlive.size(); ++i) {
            const REntry& e = rlive[i];
            if (!e.consumed && h_rdone[(r_front + i) % kRing] >= e.count) ready.push_back(i);
        }
        if (ready.empty()) return CMC_OK;
        // failure bits of the finished entries (word ranges of the bit ring)
        const uint64_t words = kRingBits / 32;
        for (size_t i : ready) {
            const REntry& e = rlive[i];
            uint64_t w0 = (e.base & (kRingBits - 1)) / 32;
            uint64_t nw = (e.base % 32 + e.count + 31) / 32;
            while (nw) {
                const uint64_t take = std::min(nw, words - w0);
                if ((rc = cuda(cudaMemcpyAsync(h_rbits + w0, d_rbits + w0, 4 * take, cudaMemcpyDeviceToHost,
                                               r_cstream), "read failures")))
                    return rc;
                nw -= take;
                w0 = 0;
            }
        }
        if ((rc = cuda(cudaStreamSynchronize(r_cstream), "read failures"))) return rc;
        for (size_t i : ready) {
            REntry& e = rlive[i];
            HostJob& j = jobs[e.job];
            auto& pend = j.pending;
            if (pend.empty() || pend.back().first != e.batch) {
                // batches complete in order per job: insert keeping the list sorted
                auto it = pend.begin();
                while (it != pend.end() && it->first < e.batch) ++it;
                if (it == pend.end() || it->first != e.batch) it = pend.insert(it, {e.batch, {}});
                for (uint64_t g = e.base; g < e.base + e.count; ++g) {
                    const uint64_t b = g & (kRingBits - 1);
                    if (h_rbits[b >> 5] >> (b & 31) & 1u) {
                        it->second.push_back(e.first + uint32_t(g - e.base));
                        ++j.failed;
                    }
                }
            } else {
                for (uint64_t g = e.base; g < e.base + e.count; ++g) {
                    const uint64_t b = g & (kRingBits - 1);
                    if (h_rbits[b >> 5] >> (b & 31) & 1u) {
                        pend.back().second.push_back(e.first + uint32_t(g - e.base));
                        ++j.failed;
                    }
                }
            }
            j.processed += e.count;
            stats.trials += e.count;
            e.consumed = true;
            ++consumed;
        }
        while (!rlive.empty() && rlive.front().consumed) {
            rlive.pop_front();
            ++r_front;
        }
        return CMC_OK;
    }

    // Commits complete batches and retires finished jobs.  A job's entries
    // may finish out of order, so a batch is complete when every trial of it
    // was read back: the job's processed count covers it only once all its
    // earlier entries finished too, so completion is checked per batch from
    // the entries still in flight.
    int resident_commit(uint32_t* finished, uint32_t cap, uint32_t& nfin) {
        std::vector<uint64_t> inflight_min(jobs.size(), ~0ULL);  // lowest unfinished trial per job
        for (const REntry& e : rlive)
            if (!e.consumed) {
                const uint64_t t = (e.batch << jobs[e.job].bt) + e.first;
                inflight_min[e.job] = std::min(inflight_min[e.job], t);
            }
        for (uint32_t id : active_ids()) {
            HostJob& j = jobs[id];
            const uint64_t per = 1ULL << j.bt;
            const uint64_t done_upto = std::min(j.next, inflight_min[id]);  // every trial below is read back
            while (!j.pending.empty()) {
                const uint64_t bb = j.pending.front().first;
                const uint64_t end = std::min<uint64_t>((bb + 1) << j.bt, j.budget);
                if (done_upto < end) break;
                auto& offs = j.pending.front().second;
                std::sort(offs.begin(), offs.end());
                if (j.journal) {
                    try {
                        j.journal->append(bb, uint32_t(std::min<uint64_t>(per, batch_length(j.jopt, bb))), offs);
                    } catch (const std::exception& ex) {
                        return fail(CMC_EINVAL, std::string("journal: ") + ex.what());
                    }
                }
                j.pending.erase(j.pending.begin());
            }
            if (j.processed >= j.budget && j.pending.empty()) {
                finish(j);
                j.journal.reset();
                free_slots.push_back(j.slot);
                if (finished && nfin < cap) finished[nfin] = id;
                ++nfin;
            }
        }
        return CMC_OK;
    }

    int step_resident(uint64_t work_blocks, uint32_t* finished, uint32_t cap, uint32_t* nfinished) {
        int rc = resident_setup();
        if (rc) return rc;
        if (r_running) {
            const cudaError_t q = cudaEventQuery(r_kdone);
            if (q == cudaSuccess) {
                if ((rc = resident_finished())) return rc;
            } else if (q != cudaErrorNotReady) {
                return cuda(q, "resident launch");
            } else {
                cudaGetLastError();  // "not ready" is an answer, not an error to keep
            }
        }
        uint32_t consumed = 0;
        if ((rc = resident_poll(consumed))) return rc;
        uint32_t nfin = 0;
        if ((rc = resident_commit(finished, cap, nfin))) return rc;
        if (nfinished) *nfinished = nfin;
        if (!r_stopping && (rc = admit(r_cstream))) return rc;
        // keep about two chunks of unclaimed work published ahead of the device
        uint32_t published = 0;
        if (!r_stopping && resident_unclaimed() < 2.0 * double(work_blocks) &&
            (rc = resident_publish(work_blocks, published)))
            return rc;
        if (!r_running && r_avail > r_begin && (rc = resident_launch())) return rc;
        // nothing left to publish: close the launch once it has the last work
        bool more = !queue.empty();
        for (uint32_t id : active_ids()) more = more || jobs[id].next < jobs[id].budget;
        if (r_running && !r_stopping && !more) {
            __atomic_store_n(&h_rq->stop, 1u, __ATOMIC_RELEASE);
            r_stopping = true;
        }
        if (!published && !consumed && !nfin)
            std::this_thread::sleep_for(std::chrono::microseconds(50));  // nothing moved: poll gently
        return CMC_OK;
    }

    // Publishes nothing more, lets the launch finish, reads everything back.
    int resident_close() {
        if (r_running && !r_stopping) {
            __atomic_store_n(&h_rq->stop, 1u, __ATOMIC_RELEASE);
            r_stopping = true;
        }
        int rc;
        if (r_running && (rc = resident_finished())) return rc;
        uint32_t consumed = 0, nfin = 0;
        if ((rc = resident_poll(consumed))) return rc;
        return resident_commit(nullptr, 0, nfin);
    }

    int status(uint32_t id, uint64_t* done, uint64_t* failed, int* state) {
        if (id >= jobs.size()) return fail(CMC_EINVAL, "unknown job id");
        HostJob& j = jobs[id];
        if (done) *done = j.processed;
        if (failed) *failed = j.failed;
        if (state) *state = j.state;
        return CMC_OK;
    }
};

}  // namespace cmc

using cmc::Server;

extern "C" {

int cmc_server_create(cmc_ctx* ctx, uint32_t max_jobs, uint64_t mem_budget_bytes,
                      uint32_t batch_bits, uint64_t max_iteration_trials, cmc_server** out) {
    if (!ctx || !out || max_jobs == 0 || batch_bits == 0 || batch_bits > 30 || max_iteration_trials == 0 ||
        max_iteration_trials >= 0xffffffffULL)
        return CMC_EINVAL;
    *out = nullptr;
    Server* s = new (std::nothrow) Server();
    if (!s) return CMC_ENOMEM;
    const int rc = s->init(reinterpret_cast<cmc::Ctx*>(ctx), max_jobs, mem_budget_bytes, batch_bits,
                           max_iteration_trials);
    if (rc) {
        reinterpret_cast<cmc::Ctx*>(ctx)->err = s->err;
        delete s;
        return rc;
    }
    *out = reinterpret_cast<cmc_server*>(s);
    return CMC_OK;
}

int cmc_server_submit(cmc_server* server, const cmc_params* params, uint64_t seed, uint64_t trials,
                      const char* journal_dir, uint32_t* out_id) {
    if (!server || !params) return CMC_EINVAL;
    return reinterpret_cast<Server*>(server)->submit(*params, seed, trials, journal_dir, out_id);
}

int cmc_server_step(cmc_server* server, uint64_t work_blocks, uint32_t* out_finished, uint32_t cap,
                    uint32_t* out_nfinished) {
    if (!server) return CMC_EINVAL;
    return reinterpret_cast<Server*>(server)->step(work_blocks, out_finished, cap, out_nfinished);
}

int cmc_server_status(cmc_server* server, uint32_t job_id, uint64_t* out_trials_done,
                      uint64_t* out_failed, int* out_state) {
    if (!server) return CMC_EINVAL;
    return reinterpret_cast<Server*>(server)->status(job_id, out_trials_done, out_failed, out_state);
}

int cmc_server_policy(cmc_server* server, double fifo_share) {
    if (!server || !(fifo_share >= 0.0 && fifo_share <= 1.0)) return CMC_EINVAL;
    reinterpret_cast<Server*>(server)->fifo_share = fifo_share;
    return CMC_OK;
}

int cmc_server_set_option(cmc_server* server, const char* name, double value) {
    if (!server || !name) return CMC_EINVAL;
    Server* s = reinterpret_cast<Server*>(server);
    const std::string n(name);
    if (n == "fifo_share" && value >= 0.0 && value <= 1.0) {
        s->fifo_share = value;
    } else if (n == "resident" && (value == 0.0 || value == 1.0)) {
        s->resident = value != 0.0;
    } else {
        s->err = "unknown server option or value: " + n;
        return CMC_EINVAL;
    }
    return CMC_OK;
}

int cmc_server_get_stats(const cmc_server* server, cmc_server_stats* out) {
    if (!server || !out) return CMC_EINVAL;
    *out = reinterpret_cast<const Server*>(server)->stats;
    return CMC_OK;
}

uint32_t cmc_server_pending(const cmc_server* server) {
    if (!server) return 0;
    return reinterpret_cast<const Server*>(server)->unfinished;
}

const char* cmc_server_error(const cmc_server* server) {
    return server ? reinterpret_cast<const Server*>(server)->err.c_str() : "";
}

int cmc_server_destroy(cmc_server* server) {
    if (!server) return CMC_OK;
    Server* s = reinterpret_cast<Server*>(server);
    const int rc = s->drain();  // commit what the device finished
    if (rc) s->ctx->err = s->err;
    delete s;
    return rc;
}

}  // extern "C"
