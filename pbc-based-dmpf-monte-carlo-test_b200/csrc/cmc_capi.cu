// cmc_capi.cu -- C ABI over the engine: per-device context, launch planning
// and the Launch seam (cuckoo_bench.cu:980-1031).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cmc.h"
#include "cmc_capi_internal.hpp"
#include "cmc_engine.cuh"
#include "cmc_hostcore.hpp"

namespace cmc {

template <typename MapT, typename BinT, bool WIDE, bool SMEMSLOTS>
__global__ void cmc_engine(const EngineArgs a);
template <typename MapT, typename BinT, bool WIDE>
__global__ void cmc_engine_split(const EngineArgs a);
template <typename MapT, typename BinT>
__global__ void cmc_engine_pooled(const EngineArgs a);
template <typename MapT, typename BinT, bool WIDE, bool SMEMSLOTS>
__global__ void cmc_engine_fused(const __grid_constant__ FusedArgs f);
__global__ void cmc_compact_failures(const uint32_t* bits, uint64_t nbits, uint32_t value_base,
                                     uint32_t* out, uint32_t* count, uint64_t cap,
                                     const unsigned long long* nbits_dev);
__global__ void cmc_selftest(const uint32_t* t0, const uint32_t* fips_rk, uint32_t* out,
                             uint32_t r256);

namespace {

thread_local std::string g_thread_error;


uint32_t round_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

}  // namespace

void set_thread_error(const std::string& message) { g_thread_error = message; }

int Ctx::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
}

int Ctx::cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CMC_OK;
    return fail(CMC_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <typename T>
int Ctx::grow(T*& ptr, size_t& cap, size_t need, const char* what) {
    if (need <= cap && ptr) return CMC_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t n = std::max<size_t>(need, 1);
    if (cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(CMC_ENOMEM, "cudaMalloc of %zu bytes for %s failed", n * sizeof(T), what);
    }
    cap = n;
    return CMC_OK;
}

// Map method of a parameter set.  Direct passes cost 8 AES blocks per Feistel
// evaluation, k*t*c evaluations per trial (c = 2^2h / D for cycle-walking).  A
// round cache costs 8 * 2^h blocks per trial and then 8 lookups per
// evaluation: from shared memory (h <= 12, a lookup ~1/64 block) or from an
// L2-resident global buffer (h <= 16; ~0.3 block: the 8 lookups of an
// evaluation are dependent L2 round trips, two chains in flight per lane).
uint32_t choose_method(uint32_t h, uint64_t domain, double candidates, int force, bool may_allocate) {
    const double c = std::ldexp(1.0, 2 * int(h)) / double(domain);
    const double direct = candidates * 8.0 * c;
    const double build = 8.0 * std::ldexp(1.0, int(h));
    const bool gcache_ok = may_allocate && domain <= 0xffffffffULL && h <= 16;
    if (force == 0) return kMethodDirect;
    if (force == 1) return h <= 12 ? kMethodCache : gcache_ok ? kMethodGCache : kMethodDirect;
    if (force == 2) return gcache_ok ? kMethodGCache : kMethodDirect;
    if (h <= 12 && build + direct / 64.0 < direct) return kMethodCache;
    if (gcache_ok && build + direct * 0.3 < direct) return kMethodGCache;
    return kMethodDirect;
}

// Fill a device job descriptor from derived parameters.
int Ctx::make_job(const cmc_params& p, uint32_t first, uint32_t count, uint64_t base, Job& j) {
    std::memset(&j, 0, sizeof j);
    if (p.mode != CMC_MODE_BGH25 && p.mode != CMC_MODE_DRRT18)
        return fail(CMC_EINVAL, "invalid mode %u", p.mode);
    if (p.k < 2 || p.k > 4) return fail(CMC_EINVAL, "k must be 2..4 (got %u)", p.k);
    if (p.pnum < 3 || p.pnum > 65534) return fail(CMC_EINVAL, "PNUM out of range");
    if (p.buckets < 1 || p.bucket_size < 1 || p.domain == 0)
        return fail(CMC_EINVAL, "invalid bucket parameters");
    if (p.domain > 0xffffffffULL) {
        if (p.half_bits > 32) return fail(CMC_EINVAL, "PRP half width above 32 bits");
    } else if (p.half_bits > 16) {
        return fail(CMC_EINVAL, "PRP half width inconsistent with domain");
    }
    if (uint64_t(p.pnum) * p.k > 0xffffffffULL) return fail(CMC_EINVAL, "too many candidates");
    j.pnum = p.pnum;
    j.k = p.k;
    j.buckets = p.buckets;
    j.kick = p.kick;
    j.mode = p.mode;
    j.input_mode = p.input_mode;
    j.half_bits = p.half_bits;
    j.domain = p.domain;
    j.mask = p.mask;
    j.range_mask = p.range_mask;
    j.width = p.bucket_size;
    j.width_magic = p.domain <= 0xffffffffULL ? uint32_t(0xffffffffULL / p.bucket_size) : 0;
    j.first = first;
    j.count = count;
    j.trial_base = base;
    j.method = choose_method(p.half_bits, p.domain, double(p.pnum) * p.k, force_method, may_allocate);
    return CMC_OK;
}

// Choose groups, warps per group and slot placement for a set of jobs.
int Ctx::plan(const std::vector<Job>& jobs, Plan& pl) {
    uint32_t max_b = 0, max_cand = 0, max_cache_h = 0, any_cache = 0, wide = 0, wide_domain = 0;
    uint32_t max_gcache_h = 0, any_gcache = 0, max_h = 0, dfold_h = 0, any_dfold = 0;
    double work = 0, cand_work = 0;
    for (const Job& j : jobs) {
        max_h = std::max(max_h, j.half_bits);
        if (!plan_no_dfold && j.method == kMethodDirect && j.domain <= 0xffffffffULL && j.half_bits <= 13) {
            any_dfold = 1;  // direct passes with a word-split round-2 fold table
            dfold_h = std::max(dfold_h, j.half_bits);
        }
        max_b = std::max(max_b, j.buckets);
        max_cand = std::max(max_cand, j.pnum * j.k);
        if (j.method == kMethodCache) {
            any_cache = 1;
            max_cache_h = std::max(max_cache_h, j.half_bits);
        }
        if (j.method == kMethodGCache) {
            any_gcache = 1;
            max_gcache_h = std::max(max_gcache_h, j.half_bits);
        }
        if (j.domain > 0xffffffffULL) wide_domain = 1;
        // 16-bit entries: 14-bit ordinal + 2-bit choice, never equal to 0xffff
        const bool narrow_ok = j.buckets <= 0xffff && j.pnum <= 16384 && !(j.k == 4 && j.pnum > 16383);
        if (!narrow_ok) wide = 1;
        work += double(j.count);
        cand_work += double(j.count) * j.pnum * j.k;
    }
    if (wide_domain) wide = 1;
    pl.variant = wide_domain ? 2 : (wide ? 1 : 0);
    const uint32_t entry = wide ? 4 : 2;
    pl.bins_bytes = round_up(max_b * entry, 16);
    const uint32_t map_bytes = round_up(max_cand * entry, 16);
    pl.slot_stride = round_up(pl.bins_bytes + map_bytes, 128);
    // a round-cache job keeps its fold table (and a shared-memory cache) in
    // its group's shared region
    const uint32_t cache_bytes = any_cache ? fold_table_bytes(max_cache_h) + (16u << max_cache_h) : 0;
    const uint32_t gfold_bytes = any_gcache ? fold_table_bytes(max_gcache_h) : 0;
    const uint32_t dfold_bytes = any_dfold ? fold_table_bytes(dfold_h) : 0;
    pl.group_bytes = kGroupHeaderBytes + std::max({cache_bytes, gfold_bytes, dfold_bytes});
    const double avg_cand = work > 0 ? cand_work / work : 0;
    // one-warp groups for direct passes up to 1,536 candidates per trial (with
    // pooled passes, measured: t=300 k=3 6.75 M trials/s against 5.14 M in
    // 4-warp groups; t=1000: 1.57 M against 1.61 M)
    pl.wg = (any_cache || any_gcache || avg_cand >= 1536.0) ? 4 : 1;
    if (force_wg) pl.wg = force_wg;
    pl.walker_ctas = force_walker_ctas > 0 ? uint32_t(force_walker_ctas) : 0;
    if (pl.walker_ctas >= uint32_t(sms)) return fail(CMC_EINVAL, "walker_ctas must be below the SM count");
    // Isolated walkers (sub-partition 3 only) pay off when walks are long
    // enough to hold producers back; short walks keep all 16 warps busy.
    double avg_probe_work = 0;
    for (const Job& j : jobs) avg_probe_work += double(j.count) * j.pnum;
    avg_probe_work = work > 0 ? avg_probe_work / work : 0;
    pl.isolate = pl.walker_ctas ? 0 : (force_isolate >= 0 ? uint32_t(force_isolate)
                                                          : (avg_probe_work >= 512 ? 1u : 0u));
    pl.nw = pl.walker_ctas ? 0 : (force_walkers ? force_walkers : 1);
    // measured best with isolated walkers: 2 groups of 6 producer warps on
    // sub-partitions 0..2 (2 x 7, adding two beside the walker, is within 3%)
    if (pl.isolate && !force_wg) pl.wg = (any_cache || any_gcache) ? 6 : 4;
    if (pl.isolate && pl.nw > 4) pl.nw = 4;
    // Pooled direct passes (producer_pooled): one-warp groups whose jobs all
    // use direct passes with 16-bit halves; each group then holds three trials'
    // headers and staged maps.  Dropped below if the walk slots go global.
    // Measured on B200 (same failure lists): t=64, B=96 24.4 -> 29.1 M
    // trials/s; t=27 42.3 -> 58.1 M; t=93 sequential 18.3 -> 20.7 M.
    // With h <= 10 the passes also take the round-2 fold (a trial's fold table
    // has at most 4 entries per round, so a warp's fold loads touch few
    // addresses): 111 table lookups per AES block instead of 124.
    pl.pool_stage = pl.pool_fold = 0;
    if (force_pool != 0 && !any_cache && !any_gcache && !wide_domain && pl.wg == 1 && !pl.walker_ctas) {
        pl.pool_stage = round_up(max_cand * entry, 16);
        pl.pool_fold = max_h <= 10 ? fold_table_bytes(max_h) : 0;
        pl.group_bytes = pool_group_bytes(pl.pool_stage, pl.pool_fold);  // its own fold, if any
    }
    const uint32_t budget = uint32_t(smem_optin) - kEngineTableBytes - kCtaSharedBytes;
    auto groups_for = [&](uint32_t nw) {
        uint32_t ng = std::min<uint32_t>(kMaxGroups, (16 - nw) / pl.wg);
        if (force_ng) ng = std::min(ng, force_ng);
        while (ng > 1 && ng * pl.group_bytes > budget) --ng;
        return ng;
    };
    const uint32_t ng = groups_for(pl.nw);
    if (ng * pl.group_bytes > budget)
        return fail(CMC_EINVAL, "round cache of %u bytes does not fit shared memory", cache_bytes);
    // Slots.  A CTA walks about slots / (probes per trial x probe latency)
    // trials per cycle: ~2.4 t probes per trial, ~300 cycles per probe in
    // shared memory (~800 when the walker shares its sub-partition with
    // producers), ~3000 in global memory (two dependent DRAM round trips
    // once the slots outgrow L2).  Its producers build AES blocks at a
    // measured ~0.157 per cycle (direct passes, shared-memory cache) or ~0.2
    // (global round cache), over the job's blocks per trial.  Shared-memory
    // slots (2..8 per group, giving up at most half of the groups) are kept
    // when their walks outpace the producers by 1.4x -- a small pool with
    // uneven walk lengths queues below that -- or beat global slots; global
    // slots take 32 per walker warp, with 4 walker warps on sub-partition 3
    // when walkers are isolated.  The split engine keeps one global slot per
    // walker-CTA thread.
    double avg_cost = 0;
    for (const Job& j : jobs) avg_cost += double(j.count) * job_cost(j);
    avg_cost = work > 0 ? avg_cost / work : 1;
    const double probes = std::max(1.0, 2.4 * avg_probe_work);
    const double produce = (any_gcache ? 0.2 : 0.157) / std::max(1.0, avg_cost);
    pl.slots_smem = false;
    for (uint32_t g = ng; !pl.walker_ctas && !force_global_slots &&
                          g >= std::max<uint32_t>(1, (ng + 1) / 2); --g) {
        const uint32_t left = budget - g * pl.group_bytes;
        const uint32_t s = std::min<uint32_t>({left / pl.slot_stride / g, 32 * pl.nw / g,
                                               max_slots_per_group});
        if (s >= 2) {
            pl.ng = g;
            pl.ns = g * s;
            pl.slots_smem = true;
            break;
        }
    }
    if (pl.walker_ctas) {
        pl.ng = ng;
        pl.ns = pl.walker_ctas * pl.ng * pl.wg * 32;
    } else {
        const uint32_t nw_g = (pl.isolate && !force_walkers) ? 4 : pl.nw;
        const uint32_t ng_g = groups_for(nw_g);
        const uint32_t ns_g = std::max<uint32_t>(1, std::min(kMaxSlots, 32 * nw_g) / ng_g) * ng_g;
        // a walker beside ALU-bound producers issues slower: ~800 cycles per
        // shared probe (measured at t=500, k=4), ~300 when isolated
        const double walk_smem = pl.slots_smem ? pl.ns / (probes * (pl.isolate ? 300.0 : 800.0)) : 0.0;
        const double walk_global = ns_g / (probes * 3000.0);
        const bool keep_smem = pl.slots_smem && (!may_allocate || walk_smem >= 1.4 * produce ||
                                                 walk_smem >= walk_global);
        if (!keep_smem) {
            pl.slots_smem = false;
            pl.nw = nw_g;
            pl.ng = ng_g;
            pl.ns = ns_g;
        }
    }
    if (!pl.slots_smem) pl.pool_stage = pl.pool_fold = 0;
    pl.group_off = kEngineTableBytes + kCtaSharedBytes;
    pl.slots_off = pl.group_off + pl.ng * pl.group_bytes;
    pl.smem_bytes = pl.slots_off + (pl.slots_smem ? pl.ns * pl.slot_stride : 0);
    if (pl.isolate) {
        pl.threads = 512;  // walker warps sit at ids 15, 11, ...; unused ids exit at once
    } else {
        pl.threads = (pl.ng * pl.wg + pl.nw) * 32;
    }
    pl.ctas = sms;
    pl.gslot_bytes = pl.walker_ctas  ? uint64_t(pl.ns) * pl.slot_stride
                     : pl.slots_smem ? 0
                                     : uint64_t(pl.ctas) * pl.ns * pl.slot_stride;
    pl.gcache_stride = any_gcache ? (8u << max_gcache_h) : 0;
    pl.gcache_bytes = uint64_t(pl.ctas) * pl.ng * pl.gcache_stride * 2;
    char buf[256];
    snprintf(buf, sizeof buf,
             "engine=%s variant=%s groups=%u warps_per_group=%u walkers=%u%s slots=%u slots_in=%s "
             "smem=%u threads=%u ctas=%u cache=%s%s",
             pl.walker_ctas ? "split" : "group", pl.variant == 0 ? "narrow" : pl.variant == 1 ? "wide" : "wide-domain", pl.ng, pl.wg,
             pl.walker_ctas ? pl.walker_ctas : pl.nw, pl.isolate ? "(isolated)" : "", pl.ns,
             pl.slots_smem ? "smem" : "global", pl.smem_bytes, pl.threads, pl.ctas,
             any_cache && any_gcache ? "smem+global" : any_cache ? "smem" : any_gcache ? "global" : "off",
             pl.pool_stage ? " pooled" : "");
    plan_text = buf;
    // The fold tables of direct passes (build_map_direct) come out of the walk
    // slots' shared memory; with fewer than 4 slots per group left, or none,
    // the walks lose more than the passes gain (measured at t=2000, h=13:
    // 9 -> 6 slots, 0.82 -> 0.72 M trials/s; t=1000: 18 -> 15 slots, 1.59 ->
    // 1.74 M), so plan again without them.
    if (any_dfold && !pl.pool_stage && (!pl.slots_smem || pl.ns < 4 * pl.ng)) {
        plan_no_dfold = true;
        const int rc2 = plan(jobs, pl);
        plan_no_dfold = false;
        return rc2;
    }
    return CMC_OK;
}

// Queue the engine launches over `jobs` (already on the device in d_jobs) --
// one per plan class, class c covering the job-table range
// [bounds[c], bounds[c + 1]) and so a contiguous range of global trial
// indices -- and the compaction of the shared failure bitmap.
int Ctx::run(const std::vector<Job>& jobs, uint64_t total, cudaStream_t st, uint32_t value_base,
             uint32_t* d_out, uint32_t* d_count, uint64_t out_cap_now,
             unsigned long long* job_failed, unsigned long long* job_done,
             const std::vector<uint32_t>* bounds_in) {
    // launch checks below read cudaGetLastError: start from a clean slate (an
    // earlier non-fatal error, e.g. of a timing query, is not this launch's)
    cudaGetLastError();
    std::vector<uint32_t> bounds = bounds_in ? *bounds_in : std::vector<uint32_t>{0, uint32_t(jobs.size())};
    const uint32_t nclass = uint32_t(bounds.size()) - 1;
    if (nclass < 1 || nclass > kMaxClasses) return fail(CMC_EINVAL, "bad plan classes");
    std::vector<Plan> plans(nclass);
    std::vector<double> class_work(nclass, 0.0), class_trials(nclass, 0.0);
    uint32_t heaviest = 0;
    uint64_t heaviest_trials = 0;
    bool any_split = false;
    std::string text;
    for (uint32_t c = 0; c < nclass; ++c) {
        std::vector<Job> part(jobs.begin() + bounds[c], jobs.begin() + bounds[c + 1]);
        int rc = plan(part, plans[c]);
        if (rc) return rc;
        any_split = any_split || plans[c].walker_ctas;
        uint64_t trials = 0;
        for (const Job& j : part) {
            trials += j.count;
            class_work[c] += job_cost(j) * j.count;
        }
        class_trials[c] = double(trials);
        if (trials > heaviest_trials) {
            heaviest_trials = trials;
            heaviest = c;
        }
        text += (c ? " | " : "") + plan_text;
    }
    // Several classes run as ONE persistent launch unless disabled or a class
    // uses the split engine; the classes then run side by side, so each gets
    // its own region of the global pool.  Launches one after another reuse one
    // region in stream order.
    const bool fuse = use_fused && nclass > 1 && nclass <= kMaxFusedClasses && !any_split;
    std::vector<uint64_t> region(nclass, 0);
    uint64_t pool = 0;
    for (uint32_t c = 0; c < nclass; ++c) {
        const uint64_t need = (plans[c].gslot_bytes + 255) / 256 * 256 + (plans[c].gcache_bytes + 255) / 256 * 256;
        if (fuse) {
            region[c] = pool;
            pool += need;
        } else {
            pool = std::max(pool, need);
        }
    }
    plan_text = fuse ? "fused(" + std::to_string(nclass) + ") " + text : text;
    const size_t words = (total + 31) / 32;
    int rc = grow(d_bits, bits_cap, words, "failure bitmap");
    if (rc) return rc;
    // walk slots, then the groups' round caches, per pool region
    if (pool && (rc = grow(d_slots, slots_cap, size_t(pool), "slot and cache pool"))) return rc;
    if ((rc = cuda(cudaMemsetAsync(d_ctrl, 0, nclass * sizeof(Ctrl), st), "memset ctrl"))) return rc;
    if ((rc = cuda(cudaMemsetAsync(d_bits, 0, words * 4, st), "memset bitmap"))) return rc;
    // timing events stay out of captured graphs: a replay records them
    // around the graph launch instead
    if (!capturing && (rc = cuda(cudaEventRecord(ev_start, st), "event"))) return rc;
    kernels = 0;
    auto class_args = [&](uint32_t c) {
        const Plan& pl = plans[c];
        char* base = d_slots + region[c];
        const size_t cache_off = size_t((pl.gslot_bytes + 255) / 256 * 256);
        EngineArgs a{};
        a.jobs = d_jobs;
        a.njobs = uint32_t(jobs.size());
        a.gidx_begin = jobs[bounds[c]].trial_base;
        a.total = bounds[c + 1] < jobs.size() ? jobs[bounds[c + 1]].trial_base : total;
        a.ctrl = d_ctrl + c;
        a.fail_bits = d_bits;
        a.job_failed = job_failed;
        a.job_done = job_done;
        a.gslots = pl.slots_smem ? nullptr : base;
        a.gcache = pl.gcache_bytes ? reinterpret_cast<uint16_t*>(base + cache_off) : nullptr;
        a.gcache_stride = pl.gcache_stride;
        a.ghdr = pl.walker_ctas ? d_ghdr : nullptr;
        a.split = pl.walker_ctas ? 1 : 0;
        a.producer_ctas = pl.ctas - pl.walker_ctas;
        a.total_groups = a.producer_ctas * pl.ng;
        a.t0 = d_t0;
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
        a.spin_limit = spin_limit;
        a.idle_polls = spin_limit;
        a.map_chains = map_chains;
        a.fill_blocks = fill_blocks;
        a.pool_stage = pl.pool_stage;
        a.pool_fold = pl.pool_fold;
        return a;
    };
    // Fused: one launch per entry width that two or more classes share (the
    // width is a template parameter of the engine), in the order of each
    // width's heaviest class; a class alone in its width runs by itself.
    std::vector<bool> launched(nclass, false);
    // Classes with pooled direct passes run their own kernel, unfused.
    for (uint32_t lead = 0; lead < nclass && fuse; ++lead) {
        if (launched[lead] || plans[lead].pool_stage) continue;
        std::vector<uint32_t> members;
        for (uint32_t c = lead; c < nclass; ++c)
            if (!launched[c] && !plans[c].pool_stage && plans[c].variant == plans[lead].variant &&
                plans[c].slots_smem == plans[lead].slots_smem)
                members.push_back(c);
        if (members.size() < 2) continue;
        FusedArgs fa{};
        fa.nclass = uint32_t(members.size());
        uint32_t smem = 0;
        double all = 0, cum = 0;
        for (uint32_t c : members) all += class_work[c];
        for (uint32_t i = 0; i < members.size(); ++i) {
            const uint32_t c = members[i];
            launched[c] = true;
            fa.cls[i] = class_args(c);
            fa.cost[i] = float(class_work[c] / std::max(1.0, class_trials[c]));
            fa.first_cta[i] = uint16_t(std::lround(double(sms) * cum / std::max(all, 1e-30)));
            cum += class_work[c];
            smem = std::max(smem, plans[c].smem_bytes);
        }
        fa.first_cta[members.size()] = uint16_t(sms);
        const void* fn = fused_engine_kernel(plans[lead].variant, plans[lead].slots_smem);
        void* args[] = {&fa};
        if ((rc = cuda(cudaLaunchKernel(fn, dim3(sms), dim3(512), args, smem, st), "fused engine launch")))
            return rc;
        ++kernels;
    }
    for (uint32_t c = 0; c < nclass; ++c) {
        if (launched[c]) continue;
        const Plan& pl = plans[c];
        if (pl.walker_ctas) {
            if ((rc = grow(d_ghdr, ghdr_cap, pl.ns, "slot headers"))) return rc;
            if ((rc = cuda(cudaMemsetAsync(d_ghdr, 0, size_t(pl.ns) * sizeof(GSlotHeader), st), "memset slots")))
                return rc;
        }
        EngineArgs a = class_args(c);
        const void* fn =
            pl.walker_ctas
                ? (pl.variant == 0   ? (const void*)cmc_engine_split<uint16_t, uint16_t, false>
                   : pl.variant == 1 ? (const void*)cmc_engine_split<uint32_t, uint32_t, false>
                                     : (const void*)cmc_engine_split<uint32_t, uint32_t, true>)
                : engine_kernel(pl.variant, pl.slots_smem, pl.pool_stage != 0);
        void* args[] = {&a};
        // The split engine's producer and walker CTAs hand trials to each other, so
        // they must all be resident at once: a cooperative launch guarantees it.
        if ((rc = cuda(pl.walker_ctas ? cudaLaunchCooperativeKernel(fn, dim3(pl.ctas), dim3(pl.threads),
                                                                     args, pl.smem_bytes, st)
                                      : cudaLaunchKernel(fn, dim3(pl.ctas), dim3(pl.threads), args,
                                                         pl.smem_bytes, st),
                       "engine launch")))
            return rc;
        ++kernels;
    }
    if (!capturing && (rc = cuda(cudaEventRecord(ev_stop, st), "event"))) return rc;
    if (d_out) {
        cmc_compact_failures<<<1, 1024, 0, st>>>(d_bits, total, value_base, d_out, d_count, out_cap_now,
                                                 nullptr);
        if ((rc = cuda(cudaGetLastError(), "compaction launch"))) return rc;
        ++kernels;
    }
    last_plan = plans[heaviest];
    ctrl_count = nclass;
    return CMC_OK;
}

int Ctx::check_ctrl() {
    Ctrl c[kMaxClasses]{};
    const uint32_t n = std::max<uint32_t>(1, ctrl_count);
    int rc = cuda(cudaMemcpy(c, d_ctrl, n * sizeof(Ctrl), cudaMemcpyDeviceToHost), "read ctrl");
    if (rc) return rc;
    Ctrl sum{};
    for (uint32_t i = 0; i < n; ++i) {
        if (c[i].error && !sum.error) {
            sum.error = c[i].error;
            sum.where = c[i].where;
        }
        sum.next += c[i].next;
        sum.walks += c[i].walks;
        sum.probes += c[i].probes;
        sum.slot_wait_cycles += c[i].slot_wait_cycles;
        sum.walker_idle_cycles += c[i].walker_idle_cycles;
        sum.walker_cycles += c[i].walker_cycles;
    }
    last_ctrl = sum;
    if (sum.error)
        return fail(-int(sum.error), "%s (site %u): results discarded", ctrl_error_text(sum.error),
                    sum.where);
    return CMC_OK;
}

const void* engine_kernel(int variant, bool smem_slots, bool pooled) {
    if (pooled && smem_slots && variant != 2)
        return variant == 0 ? (const void*)cmc_engine_pooled<uint16_t, uint16_t>
                            : (const void*)cmc_engine_pooled<uint32_t, uint32_t>;
    if (smem_slots)
        return variant == 0   ? (const void*)cmc_engine<uint16_t, uint16_t, false, true>
               : variant == 1 ? (const void*)cmc_engine<uint32_t, uint32_t, false, true>
                              : (const void*)cmc_engine<uint32_t, uint32_t, true, true>;
    return variant == 0   ? (const void*)cmc_engine<uint16_t, uint16_t, false, false>
           : variant == 1 ? (const void*)cmc_engine<uint32_t, uint32_t, false, false>
                          : (const void*)cmc_engine<uint32_t, uint32_t, true, false>;
}

const void* fused_engine_kernel(int variant, bool smem_slots) {
    if (smem_slots)
        return variant == 0   ? (const void*)cmc_engine_fused<uint16_t, uint16_t, false, true>
               : variant == 1 ? (const void*)cmc_engine_fused<uint32_t, uint32_t, false, true>
                              : (const void*)cmc_engine_fused<uint32_t, uint32_t, true, true>;
    return variant == 0   ? (const void*)cmc_engine_fused<uint16_t, uint16_t, false, false>
           : variant == 1 ? (const void*)cmc_engine_fused<uint32_t, uint32_t, false, false>
                          : (const void*)cmc_engine_fused<uint32_t, uint32_t, true, false>;
}

// Every engine kernel may use up to the device's opt-in shared memory.  Set
// once per device and never lowered, so launches of different plans -- and
// graphs captured from them -- are valid whatever ran in between.
int engine_smem_cap(size_t optin) {
    const void* fns[] = {engine_kernel(0, true), engine_kernel(1, true), engine_kernel(2, true),
                         engine_kernel(0, false), engine_kernel(1, false), engine_kernel(2, false),
                         (const void*)cmc_engine_split<uint16_t, uint16_t, false>,
                         (const void*)cmc_engine_split<uint32_t, uint32_t, false>,
                         (const void*)cmc_engine_split<uint32_t, uint32_t, true>,
                         fused_engine_kernel(0, true), fused_engine_kernel(1, true),
                         fused_engine_kernel(2, true), fused_engine_kernel(0, false),
                         fused_engine_kernel(1, false), fused_engine_kernel(2, false),
                         engine_kernel(0, true, true), engine_kernel(1, true, true)};
    for (const void* fn : fns)
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(optin)) != cudaSuccess)
            return CMC_ECUDA;
    return CMC_OK;
}

int Ctx::init(int dev) {
    device = dev;
    int rc = cuda(cudaSetDevice(dev), "cudaSetDevice");
    if (rc) return rc;
    cudaDeviceProp prop{};
    if ((rc = cuda(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties"))) return rc;
    if (prop.major < 10)
        return fail(CMC_EINVAL, "device %d (%s, sm_%d%d) is not an sm_100 GPU", dev, prop.name,
                    prop.major, prop.minor);
    sms = prop.multiProcessorCount;
    smem_optin = prop.sharedMemPerBlockOptin;
    if (engine_smem_cap(smem_optin)) {
        cudaGetLastError();
        return fail(CMC_ECUDA, "cudaFuncSetAttribute on the engine kernels failed");
    }
    if ((rc = cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream"))) return rc;
    if ((rc = cuda(cudaEventCreate(&ev_start), "event"))) return rc;
    if ((rc = cuda(cudaEventCreate(&ev_stop), "event"))) return rc;
    uint32_t t0[256];
    t0_table(t0);
    size_t cap = 0;
    if ((rc = grow(d_t0, cap, 256 + 44 + 32, "tables"))) return rc;
    uint32_t fips[44];
    expand_u64(0x0706050403020100ULL, 0x0f0e0d0c0b0a0908ULL, fips);
    if ((rc = cuda(cudaMemcpy(d_t0, t0, sizeof t0, cudaMemcpyHostToDevice), "upload T0"))) return rc;
    if ((rc = cuda(cudaMemcpy(d_t0 + 256, fips, sizeof fips, cudaMemcpyHostToDevice), "upload KAT key")))
        return rc;
    size_t c1 = 0;
    if ((rc = grow(d_ctrl, c1, kMaxClasses, "ctrl"))) return rc;
    const uint32_t kat_smem = kEngineTableBytes;
    if ((rc = cuda(cudaFuncSetAttribute((const void*)cmc_selftest,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, kat_smem),
                   "selftest attribute")))
        return rc;
    cmc_selftest<<<1, 32, kat_smem, stream>>>(d_t0, d_t0 + 256, d_t0 + 300, 256u);
    if ((rc = cuda(cudaGetLastError(), "selftest launch"))) return rc;
    uint32_t bad[32];
    if ((rc = cuda(cudaMemcpyAsync(bad, d_t0 + 300, sizeof bad, cudaMemcpyDeviceToHost, stream),
                   "selftest read")))
        return rc;
    if ((rc = cuda(cudaStreamSynchronize(stream), "selftest sync"))) return rc;
    for (int i = 0; i < 32; ++i)
        if (bad[i]) return fail(CMC_EKAT, "device AES known-answer test failed (lane %d, flags %u)", i, bad[i]);
    return CMC_OK;
}

Ctx::~Ctx() {
    if (device < 0) return;  // a planner that never touched a device holds nothing to free
    cudaSetDevice(device);
    cudaFree(d_t0);
    cudaFree(d_ctrl);
    cudaFree(d_jobs);
    cudaFree(d_bits);
    cudaFree(d_out);
    cudaFree(d_slots);
    cudaFree(d_ghdr);
    cudaFree(d_job_failed);
    cudaFree(d_key);
    for (GraphEntry& g : graphs) cudaGraphExecDestroy(g.exec);
    cudaFreeHost(h_failed);
    cudaFreeHost(h_nf);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (stream) cudaStreamDestroy(stream);
}

int Ctx::upload_jobs(const std::vector<Job>& jobs, cudaStream_t st) {
    int rc = grow(d_jobs, jobs_cap, jobs.size(), "job table");
    if (rc) return rc;
    return cuda(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(Job),
                                cudaMemcpyHostToDevice, st),
                "upload jobs");
}

int Ctx::launch_host(const cmc_params& p, const uint32_t key[44], uint32_t first, uint32_t count,
                     uint32_t* out, uint32_t* nfailed) {
    kernels = 0;
    if (!key || !out || !nfailed) return fail(CMC_EINVAL, "null argument");
    *nfailed = 0;
    if (count == 0) return CMC_OK;
    if (uint64_t(first) + count > 0x100000000ULL) return fail(CMC_EINVAL, "offset range overflows");
    int rc = cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    cudaStream_t st = user_stream ? user_stream : stream;
    std::vector<Job> jobs(1);
    if ((rc = make_job(p, first, count, 0, jobs[0]))) return rc;
    std::memcpy(jobs[0].batch_rk, key, 44 * 4);
    if ((rc = upload_jobs(jobs, st))) return rc;
    if ((rc = grow(d_out, out_cap, size_t(count) + 1, "failure list"))) return rc;
    if ((rc = run(jobs, count, st, first, d_out, d_out + count, count, nullptr, nullptr))) return rc;
    uint32_t nf = 0;
    if ((rc = cuda(cudaMemcpyAsync(&nf, d_out + count, 4, cudaMemcpyDeviceToHost, st), "read count")))
        return rc;
    if ((rc = cuda(cudaStreamSynchronize(st), "launch sync"))) return rc;
    if ((rc = check_ctrl())) return rc;
    if (nf > count) return fail(CMC_ERANGE, "GPU failure count out of range");
    if (nf && (rc = cuda(cudaMemcpyAsync(out, d_out, size_t(nf) * 4, cudaMemcpyDeviceToHost, st),
                         "read offsets")))
        return rc;
    if (nf && (rc = cuda(cudaStreamSynchronize(st), "offsets sync"))) return rc;
    *nfailed = nf;
    return CMC_OK;
}

int Ctx::launch_device(const cmc_params& p, const uint32_t* d_key_in, uint32_t first,
                       uint32_t count, uint32_t* d_offsets, uint32_t* d_nfailed, cudaStream_t st) {
    kernels = 0;
    if (!d_key_in || !d_offsets || !d_nfailed) return fail(CMC_EINVAL, "null argument");
    if (!st) st = stream;
    int rc = cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    if (count == 0) return cuda(cudaMemsetAsync(d_nfailed, 0, 4, st), "memset count");
    std::vector<Job> jobs(1);
    if ((rc = make_job(p, first, count, 0, jobs[0]))) return rc;
    if ((rc = upload_jobs(jobs, st))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_jobs[0].batch_rk, d_key_in, 44 * 4, cudaMemcpyDeviceToDevice, st),
                   "copy batch key")))
        return rc;
    return run(jobs, count, st, first, d_offsets, d_nfailed, count, nullptr, nullptr);
}

// Estimated AES-block cost of one trial of a job (map build + seeds), used to
// order a batch heaviest first.
double job_cost(const Job& j) {
    const double c = std::ldexp(1.0, 2 * int(j.half_bits)) / double(j.domain);
    const double direct = double(j.pnum) * j.k * 8.0 * c;
    const double build = 8.0 * std::ldexp(1.0, int(j.half_bits));
    const double map = j.method == kMethodCache    ? build + direct / 64.0
                       : j.method == kMethodGCache ? build + direct * 0.3
                                                   : direct;
    return 2.0 + map + 0.1 * j.pnum;
}

std::string Ctx::mix_key(const cmc_job* in, uint32_t n) const {
    std::vector<std::string> parts;
    for (uint32_t i = 0; i < n; ++i) {
        const cmc_params& p = in[i].params;
        char b[96];
        snprintf(b, sizeof b, "%u/%u/%u/%u/%u/%llu", p.mode, p.pnum, p.k, p.buckets, p.half_bits,
                 (unsigned long long)p.domain);
        parts.push_back(b);
    }
    std::sort(parts.begin(), parts.end());
    parts.erase(std::unique(parts.begin(), parts.end()), parts.end());
    std::string key;
    for (auto& x : parts) key += x + ";";
    return key;
}

// Everything a captured batched call bakes in: job shapes and counts in table
// order, plan classes, planner options and the device buffers it touches.
std::string Ctx::graph_key(const std::vector<Job>& jobs, const std::vector<uint32_t>& bounds,
                           uint64_t total, uint64_t dev_cap) const {
    std::string key;
    char b[160];
    for (const Job& j : jobs) {
        snprintf(b, sizeof b, "%u/%u/%u/%u/%u/%u/%u/%u/%llu/%u;", j.mode, j.input_mode, j.pnum, j.k,
                 j.buckets, j.kick, j.half_bits, j.method, (unsigned long long)j.domain, j.count);
        key += b;
    }
    for (uint32_t x : bounds) key += std::to_string(x) + ",";
    snprintf(b, sizeof b, "|%llu|%llu|%u/%u/%u/%u/%u/%d/%d/%d/%u/%u/%d|%p/%p/%p/%p/%p/%p/%p/%p",
             (unsigned long long)total, (unsigned long long)dev_cap, force_wg, force_ng,
             force_global_slots, force_walkers, max_slots_per_group, force_walker_ctas, force_isolate,
             force_method, spin_limit, map_chains * 16 + fill_blocks, use_fused, (void*)d_jobs, (void*)d_bits, (void*)d_out, (void*)d_slots,
             (void*)d_ctrl, (void*)d_job_failed, (void*)h_failed, (void*)h_nf);
    return key + b;
}

int Ctx::prepare_jobs(const cmc_job* in, uint32_t n, uint32_t sample_div, std::vector<Job>& out,
                      std::vector<uint32_t>& order, uint64_t& total, std::vector<uint32_t>& bounds) {
    if (!in || n == 0) return fail(CMC_EINVAL, "no jobs");
    std::vector<Job> tmp(n);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t count = in[i].count;
        if (sample_div > 1) count = std::max<uint32_t>(1, count / sample_div);
        if (count == 0) return fail(CMC_EINVAL, "job %u has no trials", i);
        if (uint64_t(in[i].first) + count > 0x100000000ULL)
            return fail(CMC_EINVAL, "job %u: offset range overflows", i);
        int rc = make_job(in[i].params, in[i].first, count, 0, tmp[i]);
        if (rc) return rc;
        batch_key(in[i].seed, in[i].batch, tmp[i].batch_rk);
        tmp[i].user = i;
    }
    // Plan classes: parameter sets whose own plans agree (slot placement,
    // warps per group, groups, walkers, entry width, cache kind) run under one
    // plan, so a small table never runs under
    // a plan made for a large one.  Classes run heaviest first; within a class, heaviest
    // trials first, so a launch ends on short ones.  Past kMaxClasses
    // signatures the lightest classes share the last launch.
    std::vector<uint32_t> cls(n, 0);
    if (force_walker_ctas <= 0) {
        std::map<std::string, uint32_t> ids;
        std::vector<double> weight;
        std::vector<uint32_t> sig(n);
        for (uint32_t i = 0; i < n; ++i) {
            Plan solo;
            int rc = plan(std::vector<Job>{tmp[i]}, solo);
            if (rc) return rc;
            const char cache = tmp[i].method == kMethodCache ? 's' : tmp[i].method == kMethodGCache ? 'g' : 'd';
            // (splitting classes further, by slot count, measured slower: 12
            // classes on the 64-set sweep gave 1.069 M trials/s against 1.090 M
            // with these 5 -- each class a CTA leaves costs it a walk drain)
            char key[96];
            snprintf(key, sizeof key, "%d/%u/%u/%u/%u/%d/%c", solo.slots_smem ? 1 : 0, solo.wg, solo.ng,
                     solo.nw, solo.isolate, solo.variant, cache);
            auto it = ids.emplace(key, uint32_t(ids.size())).first;
            sig[i] = it->second;
            if (weight.size() <= sig[i]) weight.resize(sig[i] + 1, 0.0);
            weight[sig[i]] += job_cost(tmp[i]) * tmp[i].count;
        }
        std::vector<uint32_t> rank(weight.size());
        for (uint32_t c = 0; c < rank.size(); ++c) rank[c] = c;
        std::stable_sort(rank.begin(), rank.end(), [&](uint32_t a, uint32_t b) { return weight[a] > weight[b]; });
        std::vector<uint32_t> pos(rank.size());
        for (uint32_t r = 0; r < rank.size(); ++r) pos[rank[r]] = std::min<uint32_t>(r, kMaxClasses - 1);
        for (uint32_t i = 0; i < n; ++i) cls[i] = pos[sig[i]];
    }
    order.resize(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return cls[a] != cls[b] ? cls[a] < cls[b] : job_cost(tmp[a]) > job_cost(tmp[b]);
    });
    bounds.assign(1, 0);
    for (uint32_t i = 1; i < n; ++i)
        if (cls[order[i]] != cls[order[i - 1]]) bounds.push_back(i);
    bounds.push_back(n);
    out.resize(n);
    total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        out[i] = tmp[order[i]];
        out[i].trial_base = total;
        total += out[i].count;
    }
    if (total >= 0xffffffffULL) return fail(CMC_EINVAL, "more than 2^32 - 1 trials in one batched call");
    return CMC_OK;
}

namespace {

// Apply a tuned plan for the duration of one call.
struct ScopedPlan {
    Ctx& c;
    uint32_t wg;
    int isolate, method;
    ScopedPlan(Ctx& ctx, const TunedPlan* t) : c(ctx), wg(ctx.force_wg), isolate(ctx.force_isolate),
                                               method(ctx.force_method) {
        if (t) {
            c.force_wg = t->wg;
            c.force_isolate = t->isolate;
            c.force_method = t->method;
        }
    }
    ~ScopedPlan() {
        c.force_wg = wg;
        c.force_isolate = isolate;
        c.force_method = method;
    }
};

}  // namespace

int Ctx::run_jobs(const cmc_job* in, uint32_t n, uint64_t* out_failed, uint32_t* out_offsets,
                  uint32_t* out_jobs, uint64_t cap, uint64_t* out_total) {
    kernels = 0;
    if (!out_failed) return fail(CMC_EINVAL, "null out_failed");
    int rc = cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    const auto it = tuned.find(mix_key(in, n));
    ScopedPlan scoped(*this, it == tuned.end() ? nullptr : &it->second);
    std::vector<Job> jobs;
    std::vector<uint32_t> order, bounds;
    uint64_t total = 0;
    if ((rc = prepare_jobs(in, n, 0, jobs, order, total, bounds))) return rc;
    cudaStream_t st = user_stream ? user_stream : stream;
    if ((rc = upload_jobs(jobs, st))) return rc;
    if ((rc = grow(d_job_failed, job_failed_cap, n, "job counters"))) return rc;
    const uint64_t dev_cap = out_offsets ? std::min<uint64_t>(cap, total) : 0;
    if ((rc = grow(d_out, out_cap, size_t(dev_cap) + 1, "failure list"))) return rc;
    if (h_failed_cap < n) {
        cudaFreeHost(h_failed);
        h_failed = nullptr;
        h_failed_cap = 0;
        if (cudaHostAlloc((void**)&h_failed, n * sizeof(unsigned long long), cudaHostAllocDefault) !=
            cudaSuccess) {
            cudaGetLastError();
            return fail(CMC_ENOMEM, "pinned job counters");
        }
        h_failed_cap = n;
    }
    if (!h_nf && cudaHostAlloc((void**)&h_nf, 4, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return fail(CMC_ENOMEM, "pinned count");
    }
    // The device side of the call: counters, the engine launches, the
    // compaction and the read-back into pinned memory.
    auto enqueue = [&]() -> int {
        int r = cuda(cudaMemsetAsync(d_job_failed, 0, n * sizeof(unsigned long long), st), "memset counters");
        if (r) return r;
        if ((r = run(jobs, total, st, 0, d_out, d_out + dev_cap, dev_cap, d_job_failed, nullptr, &bounds)))
            return r;
        if ((r = cuda(cudaMemcpyAsync(h_failed, d_job_failed, n * sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, st), "read counters")))
            return r;
        return cuda(cudaMemcpyAsync(h_nf, d_out + dev_cap, 4, cudaMemcpyDeviceToHost, st), "read count");
    };
    // A call shape seen before is captured into a CUDA graph on its second
    // call and replayed from the third: the job table is uploaded by copy
    // first, everything else is one graph launch.  The first call runs eagerly
    // so that buffers are sized and kernel attributes set before any capture.
    graph_state = "eager";
    if (use_graphs && force_walker_ctas <= 0) {
        const std::string key = graph_key(jobs, bounds, total, dev_cap);
        auto it = std::find_if(graphs.begin(), graphs.end(), [&](const GraphEntry& g) { return g.key == key; });
        if (it != graphs.end()) {
            if ((rc = cuda(cudaEventRecord(ev_start, st), "event"))) return rc;
            if ((rc = cuda(cudaGraphLaunch(it->exec, st), "graph launch"))) return rc;
            if ((rc = cuda(cudaEventRecord(ev_stop, st), "event"))) return rc;
            kernels = it->kernels;
            ctrl_count = it->ctrl_count;
            plan_text = it->plan_text;
            last_plan = it->plan;
            graph_state = "replayed";
        } else if (std::find(graph_seen.begin(), graph_seen.end(), key) != graph_seen.end()) {
            cudaGraph_t g = nullptr;
            capturing = true;
            rc = cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
            if (!rc) rc = enqueue();
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            capturing = false;
            cudaGraphExec_t ex = nullptr;
            const cudaError_t ie = (!rc && e == cudaSuccess && g) ? cudaGraphInstantiate(&ex, g, 0)
                                                                  : cudaErrorUnknown;
            if (ie == cudaSuccess) {
                if (graphs.size() >= 8) {
                    cudaGraphExecDestroy(graphs.front().exec);
                    graphs.erase(graphs.begin());
                }
                graphs.push_back(GraphEntry{key, ex, kernels, ctrl_count, plan_text, last_plan});
                if (g) cudaGraphDestroy(g);
                if ((rc = cuda(cudaEventRecord(ev_start, st), "event"))) return rc;
                if ((rc = cuda(cudaGraphLaunch(ex, st), "graph launch"))) return rc;
                if ((rc = cuda(cudaEventRecord(ev_stop, st), "event"))) return rc;
                graph_state = "captured";
            } else {
                // the shape could not be captured: run it eagerly
                const std::string why = rc ? err
                                      : std::string(cudaGetErrorName(e != cudaSuccess ? e : ie));
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                if ((rc = enqueue())) return rc;
                graph_state = "eager(capture failed: " + why + ")";
            }
        } else {
            if ((rc = enqueue())) return rc;
            // keyed by the buffers as this call left them (it may have grown some)
            graph_seen.push_back(graph_key(jobs, bounds, total, dev_cap));
            if (graph_seen.size() > 64) graph_seen.erase(graph_seen.begin());
        }
    } else if ((rc = enqueue())) {
        return rc;
    }
    if (use_graphs) plan_text += " graph=" + graph_state;
    if ((rc = cuda(cudaStreamSynchronize(st), "batched sync"))) return rc;
    if ((rc = check_ctrl())) return rc;
    std::vector<unsigned long long> failed(h_failed, h_failed + n);
    const uint32_t nf = *h_nf;
    uint64_t sum = 0;
    for (uint32_t i = 0; i < n; ++i) {
        out_failed[order[i]] = failed[i];
        sum += failed[i];
    }
    if (sum != nf) return fail(CMC_ERANGE, "per-job failure counts disagree with the bitmap");
    if (out_total) *out_total = nf;
    if (out_offsets && nf) {
        const uint64_t m = std::min<uint64_t>(nf, dev_cap);
        std::vector<uint32_t> g(m);
        if ((rc = cuda(cudaMemcpy(g.data(), d_out, m * 4, cudaMemcpyDeviceToHost), "read failures"))) return rc;
        // global index -> (original job, offset); global order is job-major in
        // the heavy-first order, so regroup by the caller's job order
        std::vector<std::pair<uint32_t, uint32_t>> pairs(m);
        for (uint64_t i = 0; i < m; ++i) {
            uint32_t lo = 0, hi = n;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (jobs[mid].trial_base <= g[i]) lo = mid; else hi = mid;
            }
            pairs[i] = {order[lo], jobs[lo].first + uint32_t(g[i] - jobs[lo].trial_base)};
        }
        std::sort(pairs.begin(), pairs.end());
        for (uint64_t i = 0; i < m; ++i) {
            out_offsets[i] = pairs[i].second;
            if (out_jobs) out_jobs[i] = pairs[i].first;
        }
    }
    return CMC_OK;
}

int Ctx::autotune(const cmc_job* in, uint32_t n, uint32_t sample_div) {
    int rc = cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    std::vector<Job> jobs;
    std::vector<uint32_t> order, bounds;
    uint64_t total = 0;
    if ((rc = prepare_jobs(in, n, sample_div ? sample_div : 64, jobs, order, total, bounds))) return rc;
    cudaStream_t st = user_stream ? user_stream : stream;
    bool any_cached = false;  // does the automatic choice use a round cache anywhere?
    for (const Job& j : jobs) any_cached = any_cached || j.method != kMethodDirect;
    std::vector<TunedPlan> cands{TunedPlan{0, -1, -1}};  // each class under its automatic plan
    for (int iso : {0, 1})
        for (uint32_t wg : {1u, 2u, 4u, 6u})
            for (int method : {-1, 0}) {
                if (method == 0 && !any_cached) continue;  // auto already picks direct
                cands.push_back(TunedPlan{wg, iso, method});
            }
    if ((rc = grow(d_job_failed, job_failed_cap, n, "job counters"))) return rc;
    double best_ms = 1e300;
    TunedPlan best{};
    std::string best_text;
    for (const TunedPlan& t : cands) {
        ScopedPlan scoped(*this, &t);
        // rebuild methods under the candidate's method choice
        std::vector<Job> js = jobs;
        for (uint32_t i = 0; i < n; ++i) {
            Job tmp;
            if ((rc = make_job(in[order[i]].params, js[i].first, js[i].count, js[i].trial_base, tmp))) return rc;
            js[i].method = tmp.method;
        }
        if ((rc = upload_jobs(js, st))) return rc;
        rc = run(js, total, st, 0, nullptr, nullptr, 0, d_job_failed, nullptr, &bounds);
        if (rc == CMC_EINVAL) continue;  // plan does not fit: skip the candidate
        if (rc) return rc;
        float ms = 0;
        if ((rc = cuda(cudaEventSynchronize(ev_stop), "tune sync"))) return rc;
        if ((rc = cuda(cudaEventElapsedTime(&ms, ev_start, ev_stop), "tune time"))) return rc;
        if ((rc = check_ctrl())) return rc;
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
            best_text = plan_text;
        }
    }
    if (best_ms == 1e300) return fail(CMC_EINVAL, "no candidate plan fits this mix");
    tuned[mix_key(in, n)] = best;
    char buf[512];
    snprintf(buf, sizeof buf, "%s | sample %.3f ms for %llu trials", best_text.c_str(), best_ms,
             (unsigned long long)total);
    tune_text = buf;
    return CMC_OK;
}

}  // namespace cmc

using cmc::Ctx;

extern "C" {

int cmc_init(int device, cmc_ctx** out) {
    if (!out) return CMC_EINVAL;
    *out = nullptr;
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) return CMC_ENOMEM;
    const int rc = c->init(device);
    if (rc) {
        cmc::g_thread_error = c->err;
        delete c;
        return rc;
    }
    *out = reinterpret_cast<cmc_ctx*>(c);
    return CMC_OK;
}

int cmc_destroy(cmc_ctx* ctx) {
    delete reinterpret_cast<Ctx*>(ctx);
    return CMC_OK;
}

const char* cmc_last_error(const cmc_ctx* ctx) {
    if (!ctx) return cmc::g_thread_error.c_str();
    return reinterpret_cast<const Ctx*>(ctx)->err.c_str();
}

int cmc_launch(cmc_ctx* ctx, const cmc_params* params, const uint32_t batch_key[44],
               uint32_t first, uint32_t count, uint32_t* out_offsets, uint32_t* out_nfailed) {
    if (!ctx || !params) return CMC_EINVAL;
    return reinterpret_cast<Ctx*>(ctx)->launch_host(*params, batch_key, first, count, out_offsets,
                                                     out_nfailed);
}

int cmc_launch_device(cmc_ctx* ctx, const cmc_params* params, const uint32_t* d_batch_key,
                      uint32_t first, uint32_t count, uint32_t* d_out_offsets,
                      uint32_t* d_out_nfailed, void* stream) {
    if (!ctx || !params) return CMC_EINVAL;
    return reinterpret_cast<Ctx*>(ctx)->launch_device(*params, d_batch_key, first, count,
                                                       d_out_offsets, d_out_nfailed,
                                                       static_cast<cudaStream_t>(stream));
}

int cmc_check(cmc_ctx* ctx) {
    if (!ctx) return CMC_EINVAL;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    int rc = c->cuda(cudaDeviceSynchronize(), "synchronize");
    if (rc) return rc;
    return c->check_ctrl();
}

int cmc_run_jobs(cmc_ctx* ctx, const cmc_job* jobs, uint32_t njobs, uint64_t* out_failed,
                 uint32_t* out_offsets, uint32_t* out_jobs, uint64_t cap, uint64_t* out_total) {
    if (!ctx) return CMC_EINVAL;
    return reinterpret_cast<Ctx*>(ctx)->run_jobs(jobs, njobs, out_failed, out_offsets, out_jobs, cap,
                                                  out_total);
}

int cmc_autotune(cmc_ctx* ctx, const cmc_job* jobs, uint32_t njobs, uint32_t sample_div,
                 const char** out_choice) {
    if (!ctx) return CMC_EINVAL;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    const int rc = c->autotune(jobs, njobs, sample_div);
    if (out_choice) *out_choice = c->tune_text.c_str();
    return rc;
}

int cmc_set_option(cmc_ctx* ctx, const char* name, int64_t value) {
    if (!ctx || !name) return CMC_EINVAL;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    const std::string n(name);
    if (n == "warps_per_group" && value >= 0 && value <= 15) c->force_wg = uint32_t(value);
    else if (n == "groups" && value >= 0 && value <= cmc::kMaxGroups) c->force_ng = uint32_t(value);
    else if (n == "global_slots" && (value == 0 || value == 1)) c->force_global_slots = uint32_t(value);
    else if (n == "method" && value >= -1 && value <= 2) c->force_method = int(value);
    else if (n == "pool" && value >= -1 && value <= 1) c->force_pool = int(value);
    else if (n == "graph" && (value == 0 || value == 1)) c->use_graphs = int(value);
    else if (n == "fused" && (value == 0 || value == 1)) c->use_fused = int(value);
    else if (n == "fill_blocks" && (value == 0 || (value >= 2 && value <= 4))) c->fill_blocks = uint32_t(value);
    else if (n == "map_chains" && (value == 0 || value == 1 || value == 2 || value == 4 || value == 8))
        c->map_chains = uint32_t(value);
    else if (n == "walkers" && value >= 0 && value <= 4) c->force_walkers = uint32_t(value);
    else if (n == "isolate_walkers" && value >= -1 && value <= 1) c->force_isolate = int(value);
    else if (n == "walker_ctas" && value >= -1 && value < c->sms) c->force_walker_ctas = int(value);
    else if (n == "slots_per_group" && value >= 0 && value <= 32)
        c->max_slots_per_group = value ? uint32_t(value) : 8u;
    else if (n == "spin_limit" && value >= 0 && value <= 0xffffffffLL)
        c->spin_limit = value ? uint32_t(value) : (1u << 26);
    else return c->fail(CMC_EINVAL, "unknown option or value out of range: %s=%lld", name, (long long)value);
    return CMC_OK;
}

int cmc_set_stream(cmc_ctx* ctx, void* stream) {
    if (!ctx) return CMC_EINVAL;
    reinterpret_cast<Ctx*>(ctx)->user_stream = static_cast<cudaStream_t>(stream);
    return CMC_OK;
}

double cmc_last_engine_ms(cmc_ctx* ctx) {
    if (!ctx) return -1.0;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (c->kernels == 0) return -1.0;
    float ms = 0.f;
    // a failure here must not stay pending for the next launch's error check
    if (cudaEventSynchronize(c->ev_stop) != cudaSuccess ||
        cudaEventElapsedTime(&ms, c->ev_start, c->ev_stop) != cudaSuccess) {
        cudaGetLastError();
        return -1.0;
    }
    return ms;
}

int cmc_last_stats(cmc_ctx* ctx, uint64_t out[6]) {
    if (!ctx || !out) return CMC_EINVAL;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    const cmc::Ctrl& s = c->last_ctrl;
    out[0] = s.walks;
    out[1] = s.probes;
    out[2] = s.slot_wait_cycles;
    out[3] = s.walker_idle_cycles;
    out[4] = s.walker_cycles;
    out[5] = s.error;
    return CMC_OK;
}

uint32_t cmc_last_kernel_count(const cmc_ctx* ctx) {
    return ctx ? reinterpret_cast<const Ctx*>(ctx)->kernels : 0;
}

int cmc_plan_describe(const cmc_params* params, uint32_t count, uint32_t sms, uint64_t smem_optin,
                      char* out, uint32_t cap) {
    if (!params || !out || cap == 0 || count == 0 || sms == 0 ||
        smem_optin < uint64_t(cmc::kEngineTableBytes) + cmc::kCtaSharedBytes + cmc::kGroupHeaderBytes) {
        cmc::set_thread_error("cmc_plan_describe: invalid argument");
        return CMC_EINVAL;
    }
    Ctx c;  // planner only: no device is selected and nothing is allocated
    c.sms = int(sms);
    c.smem_optin = size_t(smem_optin);
    std::vector<cmc::Job> jobs(1);
    int rc = c.make_job(*params, 0, count, 0, jobs[0]);
    cmc::Plan pl;
    if (!rc) rc = c.plan(jobs, pl);
    snprintf(out, cap, "%s", (rc ? c.err : c.plan_text).c_str());
    if (rc) cmc::set_thread_error(c.err);
    return rc;
}

const char* cmc_last_plan(const cmc_ctx* ctx) {
    return ctx ? reinterpret_cast<const Ctx*>(ctx)->plan_text.c_str() : "";
}

}  // extern "C"
