// cmc_serve.cu -- serving loop: estimation jobs of different sizes admitted as
// they arrive and run together in the persistent engine (continuous batching).
//
// Each admitted job has a device-resident ServeState: its parameters, its RNG
// counter (`next`, the index of its next trial), its budget and the cached key
// of its current batch; its failure and trial counts accumulate on the device
// (the engine's per-job counters, indexed by server slot).  One iteration
// (`cmc_server_step`):
//   1. admits queued jobs while their slot memory fits the device-memory budget;
//   2. picks one size class (jobs whose walk slots fit in shared memory, or
//      not) and grants its jobs trials: half of the step's work in arrival
//      order, so no job starves, half shortest remaining work first;
//   3. the scheduler kernel turns the grants into the engine's job table on the
//      device -- clamping at batch ends, deriving a batch key with device AES
//      when a job enters a new batch, advancing the RNG counters, prefix-summing
//      the table -- and writes the iteration's trial total to device memory;
//   4. one engine launch runs every granted trial; the failure compaction
//      follows; the host maps failures back to (job, batch, offset);
//   5. finished batches are appended to the job's v3 journal (optional), and
//      finished jobs free their slot.
// A job's results are identical alone and in the mix: trial identity is
// (seed, batch, offset) and does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "cmc.h"
#include "cmc_aes.cuh"
#include "cmc_capi_internal.hpp"
#include "cmc_engine.cuh"
#include "cmc_hostcore.hpp"
#include "cmc_runner.hpp"

namespace cmc {

template <typename MapT, typename BinT, bool WIDE>
__global__ void cmc_engine(const EngineArgs a);
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
    uint64_t seed = 0, budget = 0, next = 0;
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

struct Server {
    Ctx* ctx = nullptr;
    uint32_t max_jobs = 0, bt = 20;
    uint64_t mem_budget = 0, max_iter_trials = 0, iteration = 0;
    ServeState* d_states = nullptr;
    Grant* d_grants = nullptr;
    Job* d_table = nullptr;
    GrantInfo* d_info = nullptr;
    unsigned long long* d_total = nullptr;
    unsigned long long* d_failed = nullptr;
    unsigned long long* d_done = nullptr;
    uint32_t* d_bits = nullptr;
    uint32_t* d_list = nullptr;  // failures of one iteration (+ count)
    char* d_slots = nullptr;
    size_t slots_bytes = 0;
    std::vector<HostJob> jobs;
    std::deque<uint32_t> queue;
    std::vector<uint32_t> free_slots;
    uint64_t fixed_bytes = 0;
    double fifo_share = 0.5;  // part of each step's work granted in arrival order
    std::string err;

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return CMC_OK;
        return fail(CMC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
    ~Server() {
        cudaFree(d_states);
        cudaFree(d_grants);
        cudaFree(d_table);
        cudaFree(d_info);
        cudaFree(d_total);
        cudaFree(d_failed);
        cudaFree(d_done);
        cudaFree(d_bits);
        cudaFree(d_list);
        cudaFree(d_slots);
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
        const size_t words = (max_iter_trials + 31) / 32;
        if ((rc = alloc((void**)&d_states, sizeof(ServeState) * mj, "job states"))) return rc;
        if ((rc = alloc((void**)&d_grants, sizeof(Grant) * mj, "grants"))) return rc;
        if ((rc = alloc((void**)&d_table, sizeof(Job) * mj, "job table"))) return rc;
        if ((rc = alloc((void**)&d_info, sizeof(GrantInfo) * mj, "grant info"))) return rc;
        if ((rc = alloc((void**)&d_total, 8, "total"))) return rc;
        if ((rc = alloc((void**)&d_failed, 8 * mj, "failure counters"))) return rc;
        if ((rc = alloc((void**)&d_done, 8 * mj, "trial counters"))) return rc;
        if ((rc = alloc((void**)&d_bits, words * 4, "failure bitmap"))) return rc;
        if ((rc = alloc((void**)&d_list, (max_iter_trials + 1) * 4, "failure list"))) return rc;
        fixed_bytes = (sizeof(ServeState) + sizeof(Grant) + sizeof(Job) + sizeof(GrantInfo) + 16) * mj +
                      words * 4 + (max_iter_trials + 1) * 4 + 8;
        if (fixed_bytes > mem_budget) return fail(CMC_ENOMEM, "device-memory budget below the server's fixed state");
        for (uint32_t s = mj; s-- > 0;) free_slots.push_back(s);
        if ((rc = cuda(cudaMemsetAsync(d_failed, 0, 8 * mj, ctx->stream), "memset"))) return rc;
        if ((rc = cuda(cudaMemsetAsync(d_done, 0, 8 * mj, ctx->stream), "memset"))) return rc;
        return cuda(cudaFuncSetAttribute((const void*)serve_schedule,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes),
                    "scheduler attribute");
    }

    // Plan for a set of active parameter sets; returns the global slot pool
    // bytes the plan needs (0 for shared-memory slots).
    int plan_for(const std::vector<uint32_t>& ids, Plan& pl, std::vector<Job>& shapes, uint64_t& pool) {
        shapes.clear();
        for (uint32_t id : ids) {
            Job j;
            int rc = ctx->make_job(jobs[id].params, 0, 1, 0, j);
            if (rc) return fail(rc, ctx->err);
            shapes.push_back(j);
        }
        int rc = ctx->plan(shapes, pl);
        if (rc) return fail(rc, ctx->err);
        pool = pl.slots_smem ? 0 : uint64_t(pl.ctas) * pl.ns * pl.slot_stride;
        return CMC_OK;
    }

    std::vector<uint32_t> active_ids() const {
        std::vector<uint32_t> v;
        for (const HostJob& j : jobs)
            if (j.state == 1) v.push_back(j.id);
        return v;
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
        const double c = std::ldexp(1.0, 2 * int(p.half_bits)) / double(p.domain);
        j.cost = 2.0 + std::min(8.0 * std::ldexp(1.0, int(p.half_bits)), 8.0 * p.k * p.pnum * c) +
                 0.3 * p.pnum;
        {
            // size class: do this table's walk slots fit in shared memory?
            std::vector<Job> one(1);
            one[0] = probe;
            Plan pl;
            if ((rc = ctx->plan(one, pl))) return fail(rc, ctx->err);
            j.global_slots = pl.slots_smem ? 0 : 1;
            // a trial's walk is ~2.4 t probes of ~300 (shared) or ~1300 (global)
            // cycles; expressed in blocks of GPU throughput (~4e10 blocks/s at 2 GHz)
            const double walk_cycles = 2.4 * p.pnum * (j.global_slots ? 1300.0 : 300.0);
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
                j.failed = c0.failed.load();  // committed failures of the prefix
                j.journal.reset(new Journal(o, p, 0));
            } catch (const std::exception& e) {
                return fail(CMC_EINVAL, std::string("journal: ") + e.what());
            }
        }
        jobs.push_back(std::move(j));
        queue.push_back(jobs.back().id);
        if (out_id) *out_id = jobs.back().id;
        return CMC_OK;
    }

    int admit() {
        while (!queue.empty() && !free_slots.empty()) {
            const uint32_t id = queue.front();
            HostJob& j = jobs[id];
            if (j.next >= j.budget) {  // fully journaled already
                queue.pop_front();
                j.state = 2;
                continue;
            }
            std::vector<uint32_t> ids = active_ids();
            ids.push_back(id);
            Plan pl;
            std::vector<Job> shapes;
            uint64_t pool = 0;
            int rc = plan_for(ids, pl, shapes, pool);
            if (rc) return rc;
            if (fixed_bytes + pool > mem_budget) {
                if (ids.size() == 1)
                    return fail(CMC_ENOMEM, "job " + std::to_string(id) +
                                                " alone needs more device memory than the budget");
                break;  // wait for memory to free up
            }
            queue.pop_front();
            j.slot = free_slots.back();
            free_slots.pop_back();
            j.state = 1;
            j.admitted_at = iteration;
            ServeState st{};
            rc = ctx->make_job(j.params, 0, 1, 0, st.job);
            if (rc) return fail(rc, ctx->err);
            st.seed = j.seed;
            st.next = j.next;
            st.budget = j.budget;
            st.key_batch = ~0ULL;
            st.bt = j.bt;
            st.active = 1;
            const uint64_t zero = 0;
            if ((rc = cuda(cudaMemcpyAsync(&d_states[j.slot], &st, sizeof st, cudaMemcpyHostToDevice,
                                           ctx->stream), "upload job state")))
                return rc;
            if ((rc = cuda(cudaMemcpyAsync(&d_failed[j.slot], &zero, 8, cudaMemcpyHostToDevice, ctx->stream),
                           "reset counter")))
                return rc;
            if ((rc = cuda(cudaMemcpyAsync(&d_done[j.slot], &zero, 8, cudaMemcpyHostToDevice, ctx->stream),
                           "reset counter")))
                return rc;
            if ((rc = cuda(cudaStreamSynchronize(ctx->stream), "admit sync"))) return rc;
        }
        return CMC_OK;
    }

    int step(uint64_t work_blocks, uint32_t* finished, uint32_t cap, uint32_t* nfinished) {
        if (nfinished) *nfinished = 0;
        int rc = cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        if (rc) return rc;
        if ((rc = admit())) return rc;
        std::vector<uint32_t> all = active_ids();
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
            if (jobs[id].global_slots == cls) ids.push_back(id);
        // grants: half of the work in arrival order (bounds the tail), the rest
        // shortest remaining work first (small jobs finish at once); the step
        // is at least 2.5x the latency of its slowest trial so that trial's
        // tail is covered
        std::vector<Grant> grants;
        std::vector<uint32_t> order = ids;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return remaining(a) < remaining(b); });
        double floor_blocks = 0;
        for (uint32_t id : ids) floor_blocks = std::max(floor_blocks, 2.5 * jobs[id].latency_blocks);
        work_blocks = std::max<uint64_t>(work_blocks, uint64_t(floor_blocks));
        // shares per job (trials), then one grant per job
        std::vector<uint64_t> share(ids.size(), 0);
        std::vector<uint32_t> pos(jobs.size(), 0);
        for (uint32_t i = 0; i < ids.size(); ++i) pos[ids[i]] = i;
        double left = double(work_blocks);
        uint64_t trials_left = max_iter_trials;
        auto room = [&](uint32_t id) {  // trials this job can still take in this step
            const HostJob& j = jobs[id];
            const uint64_t per = 1ULL << j.bt;
            const uint64_t next = j.next + share[pos[id]];
            uint64_t r = std::min<uint64_t>(j.budget - next, per - (next & (per - 1)));
            if (share[pos[id]] > 0 && (next & (per - 1)) == 0) r = 0;  // one batch per grant
            return std::min<uint64_t>(r, 0xffffffffULL - share[pos[id]]);
        };
        auto give = [&](uint32_t id, double blocks) {
            const HostJob& j = jobs[id];
            uint64_t n = uint64_t(std::max(1.0, blocks / j.cost));
            n = std::min<uint64_t>({n, room(id), trials_left});
            share[pos[id]] += n;
            trials_left -= n;
            left -= double(n) * j.cost;
        };
        std::vector<uint32_t> fifo = ids;
        std::sort(fifo.begin(), fifo.end(), [&](uint32_t a, uint32_t b) {
            return jobs[a].admitted_at != jobs[b].admitted_at ? jobs[a].admitted_at < jobs[b].admitted_at : a < b;
        });
        const double keep = double(work_blocks) * (1.0 - fifo_share);
        for (uint32_t id : fifo) {
            if (left <= keep || trials_left == 0) break;
            give(id, left - keep);
        }
        for (uint32_t id : order) {
            if (left <= 0 || trials_left == 0) break;
            give(id, left);
        }
        for (uint32_t i = 0; i < ids.size(); ++i) {
            if (share[i] == 0) continue;
            HostJob& j = jobs[ids[i]];
            grants.push_back(Grant{j.slot, uint32_t(share[i])});
            j.next += share[i];
        }
        if (grants.empty()) return CMC_OK;
        cudaStream_t st = ctx->stream;
        if ((rc = cuda(cudaMemcpyAsync(d_grants, grants.data(), grants.size() * sizeof(Grant),
                                       cudaMemcpyHostToDevice, st), "upload grants")))
            return rc;
        serve_schedule<<<1, 256, kTableBytes, st>>>(d_states, d_grants, uint32_t(grants.size()), ctx->d_t0,
                                                    d_table, d_info, d_total);
        if ((rc = cuda(cudaGetLastError(), "scheduler launch"))) return rc;
        // engine over the table the scheduler wrote
        Plan pl;
        std::vector<Job> shapes;
        uint64_t pool = 0;
        if ((rc = plan_for(ids, pl, shapes, pool))) return rc;
        if (pool > slots_bytes) {
            cudaFree(d_slots);
            d_slots = nullptr;
            slots_bytes = 0;
            if (cudaMalloc((void**)&d_slots, pool) != cudaSuccess) {
                cudaGetLastError();
                return fail(CMC_ENOMEM, "slot pool");
            }
            slots_bytes = pool;
        }
        if ((rc = cuda(cudaMemsetAsync(ctx->d_ctrl, 0, sizeof(Ctrl), st), "memset ctrl"))) return rc;
        if ((rc = cuda(cudaMemsetAsync(d_bits, 0, (max_iter_trials + 31) / 32 * 4, st), "memset bitmap")))
            return rc;
        EngineArgs a{};
        a.jobs = d_table;
        a.njobs = uint32_t(grants.size());
        a.total = 0;
        a.total_dev = d_total;
        a.count_by_user = 1;
        a.ctrl = ctx->d_ctrl;
        a.fail_bits = d_bits;
        a.job_failed = d_failed;
        a.job_done = d_done;
        a.gslots = pl.slots_smem ? nullptr : d_slots;
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
        const void* fn = pl.variant == 0 ? (const void*)cmc_engine<uint16_t, uint16_t, false>
                       : pl.variant == 1 ? (const void*)cmc_engine<uint32_t, uint32_t, false>
                                         : (const void*)cmc_engine<uint32_t, uint32_t, true>;
        if ((rc = cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(pl.smem_bytes)), "engine attribute")))
            return rc;
        void* args[] = {&a};
        if ((rc = cuda(cudaLaunchKernel(fn, dim3(pl.ctas), dim3(pl.threads), args, pl.smem_bytes, st),
                       "engine launch")))
            return rc;
        cmc_compact_failures<<<1, 1024, 0, st>>>(d_bits, 0, 0, d_list, d_list + max_iter_trials,
                                                 max_iter_trials, d_total);
        if ((rc = cuda(cudaGetLastError(), "compaction launch"))) return rc;
        std::vector<GrantInfo> info(grants.size());
        uint32_t nf = 0;
        if ((rc = cuda(cudaMemcpyAsync(info.data(), d_info, info.size() * sizeof(GrantInfo),
                                       cudaMemcpyDeviceToHost, st), "read grant info")))
            return rc;
        if ((rc = cuda(cudaMemcpyAsync(&nf, d_list + max_iter_trials, 4, cudaMemcpyDeviceToHost, st),
                       "read count")))
            return rc;
        if ((rc = cuda(cudaStreamSynchronize(st), "iteration sync"))) return rc;
        if ((rc = ctx->check_ctrl())) return fail(rc, ctx->err);
        ++iteration;
        std::vector<uint32_t> fl(nf);
        if (nf && (rc = cuda(cudaMemcpy(fl.data(), d_list, nf * 4ULL, cudaMemcpyDeviceToHost), "read failures")))
            return rc;
        // slot -> job
        std::vector<uint32_t> slot_job(max_jobs, ~0u);
        for (uint32_t id : ids) slot_job[jobs[id].slot] = id;
        // failures of this iteration into their job's pending batch lists
        size_t gi = 0;
        for (uint32_t g = 0; g < info.size(); ++g) {
            HostJob& j = jobs[slot_job[info[g].slot]];
            auto& pend = j.pending;
            if (pend.empty() || pend.back().first != info[g].batch) pend.push_back({info[g].batch, {}});
            while (gi < fl.size() && fl[gi] < info[g].base + info[g].count) {
                pend.back().second.push_back(info[g].first + uint32_t(fl[gi] - info[g].base));
                ++j.failed;
                ++gi;
            }
        }
        // commit finished batches, retire finished jobs
        uint32_t nfin = 0;
        for (uint32_t id : ids) {
            HostJob& j = jobs[id];
            const uint64_t per = 1ULL << j.bt;
            while (!j.pending.empty()) {
                const uint64_t b = j.pending.front().first;
                const uint64_t end = std::min<uint64_t>((b + 1) << j.bt, j.budget);
                if (j.next < end) break;  // batch not complete yet
                auto& offs = j.pending.front().second;
                std::sort(offs.begin(), offs.end());
                if (j.journal) {
                    try {
                        j.journal->append(b, uint32_t(std::min<uint64_t>(per, batch_length(j.jopt, b))), offs);
                    } catch (const std::exception& e) {
                        return fail(CMC_EINVAL, std::string("journal: ") + e.what());
                    }
                }
                j.pending.erase(j.pending.begin());
            }
            if (j.next >= j.budget && j.pending.empty()) {
                j.state = 2;
                j.journal.reset();
                free_slots.push_back(j.slot);
                if (finished && nfin < cap) finished[nfin] = id;
                ++nfin;
            }
        }
        if (nfinished) *nfinished = nfin;
        return CMC_OK;
    }

    int status(uint32_t id, uint64_t* done, uint64_t* failed, int* state) {
        if (id >= jobs.size()) return fail(CMC_EINVAL, "unknown job id");
        HostJob& j = jobs[id];
        if (done) *done = j.next;
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

uint32_t cmc_server_pending(const cmc_server* server) {
    if (!server) return 0;
    const Server* s = reinterpret_cast<const Server*>(server);
    uint32_t n = 0;
    for (const auto& j : s->jobs) n += j.state != 2;
    return n;
}

const char* cmc_server_error(const cmc_server* server) {
    return server ? reinterpret_cast<const Server*>(server)->err.c_str() : "";
}

int cmc_server_destroy(cmc_server* server) {
    delete reinterpret_cast<Server*>(server);
    return CMC_OK;
}

}  // extern "C"
