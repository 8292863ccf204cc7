// cmc_engine.cuh -- device data structures shared by the engine kernels and
// the host planner.
#pragma once
#include <cstdint>

namespace cmc {

constexpr uint32_t kMethodDirect = 0;  // candidates by 8-round AES Feistel passes
constexpr uint32_t kMethodCache = 1;   // 8*2^h round cache in shared memory, then lookups
constexpr uint32_t kMethodGCache = 2;  // the same round cache in global memory (L2), h <= 16

constexpr uint32_t kSlotFree = 0;
constexpr uint32_t kSlotReady = 1;
constexpr uint32_t kSlotFilling = 2;

constexpr uint32_t kMaxSlots = 128;  // one walker lane per slot, up to 4 walker warps
constexpr uint32_t kCtaSharedBytes = 4864;  // slot states and headers after the T-table
constexpr uint32_t kEngineTableBytes = 65536;  // replicated T-table at shared offset 0
constexpr uint32_t kMaxGroups = 14; // named barriers 1..14
constexpr uint32_t kGroupHeaderBytes = 1024;  // per-group shared header (the trial's job copy)

// Pooled direct passes (EngineArgs::pool_stage != 0): a one-warp group keeps
// kPoolContexts trials in flight, each with its own header (kPoolHeaderStride
// apart: 16 bytes more than a header, so the contexts' round constants fall in
// different banks), a staging map of pool_stage bytes after the headers, and,
// when pool_fold != 0, a round-2 fold table of pool_fold bytes after those.
constexpr uint32_t kPoolContexts = 3;  // measured: 2 and 3 within 0.3 % at t=64, 3 +5 % at t=27; 4 slower
constexpr uint32_t kPoolHeaderStride = kGroupHeaderBytes + 16;
__host__ __device__ constexpr uint32_t pool_group_bytes(uint32_t stage, uint32_t fold) {
    return kPoolContexts * (kPoolHeaderStride + stage + fold);
}

// A group's shared region: [header, kGroupHeaderBytes][round-2 fold table of a
// round-cache job][the round cache itself, when it is kept in shared memory].
// The fold table holds 8 rounds x 2^max(0, h - 8) entries of 16 bytes.
__host__ __device__ constexpr uint32_t fold_table_bytes(uint32_t h) {
    return 16u * (8u << (h > 8 ? h - 8 : 0));
}

// One experiment configuration applied to a contiguous run of trials of one
// batch.  The job table concatenates its jobs' trials: job j owns global
// indices [trial_base, trial_base + count); a launch runs a contiguous range.
struct Job {
    uint32_t batch_rk[44];  // batch key schedule (plain words)
    uint32_t pnum, k, buckets, kick;
    uint32_t mode, input_mode, half_bits, method;
    uint64_t domain, mask, range_mask, width;
    uint32_t width_magic;   // floor((2^32 - 1) / width) when domain < 2^32
    uint32_t first;         // first within-batch offset
    uint32_t count;         // trials of this job in the launch
    uint32_t user;          // caller tag (job id in batched/served mode)
    uint64_t trial_base;
};

struct Ctrl {
    unsigned long long next;   // work counter: next global trial index
    unsigned int error;        // 0, or a CMC_E* code (positive here)
    unsigned int where;        // which wait gave up (diagnostics)
    unsigned long long walks;  // walks completed (all jobs)
    unsigned long long probes; // probes spent (all jobs)
    unsigned long long slot_wait_cycles;   // producer leaders waiting for a free slot
    unsigned long long walker_idle_cycles; // walker warps with no slot to walk
    unsigned long long walker_cycles;      // walker warps' lifetime
    unsigned int slot_cursor;              // split engine: next slot to try
    unsigned int groups_done;              // split engine: producer groups finished
};

// What a nonzero Ctrl::error means, for the host's error message.
inline const char* ctrl_error_text(unsigned int error) {
    switch (error) {
    case 3: return "dynamic shared memory does not start where the T-table lookups address it";
    case 5: return "a device result was out of range";
    default: return "a bounded device wait gave up";
    }
}

// Resident launches: the host publishes work while the kernel runs.  Lives
// in mapped pinned host memory; the host writes `avail` before `stop`.
struct ResidentQueue {
    unsigned long long avail;  // trials with global index < avail are published
    unsigned int stop;         // 1: no more work in this launch
    unsigned int pad;
};

// Split engine: header of one global slot (one walker thread per slot).
struct __align__(64) GSlotHeader {
    unsigned long long gidx, walk, rnd;
    uint32_t job, offset;
    uint32_t state;  // kSlotFree / kSlotFilling / kSlotReady
};

struct EngineArgs {
    const Job* jobs;
    uint32_t njobs;
    uint64_t total;                     // the launch runs global trials [gidx_begin, total)
    uint64_t gidx_begin;
    Ctrl* ctrl;
    uint32_t* fail_bits;                // bit g = global trial g failed
    unsigned long long* job_failed;     // per job (optional)
    unsigned long long* job_done;       // per job (optional)
    char* gslots;                       // global slot pool (nullptr: slots in smem)
    const uint32_t* t0;                 // 256-word T0 table in global memory
    uint32_t slot_stride;               // bytes per slot
    uint32_t bins_bytes;                // map starts this far into a slot
    uint32_t ng, wg, ns;                // groups, warps per group, slots
    uint32_t nw;                        // walker warps (slot s -> walker s % nw)
    uint32_t isolate_walkers;           // walkers on warps 15, 11, 7, 3 (sub-partition 3)
    uint32_t r256;                      // the constant 256, kept opaque to the compiler
    // split engine: CTAs [0, producer_ctas) produce maps, the rest walk; slot s
    // is walked by thread s of the walker CTAs; headers in global memory
    GSlotHeader* ghdr;
    uint32_t split, producer_ctas, total_groups;
    // serving: the trial total is written by the scheduler kernel that runs
    // just before (nullptr: use `total`), and per-job counters are indexed by
    // Job::user (the server slot) rather than by table position
    const unsigned long long* total_dev;
    uint32_t count_by_user;
    uint32_t group_bytes;               // per-group smem (header + fold table + cache)
    uint32_t group_off;                 // smem offset of group 0
    uint32_t slots_off;                 // smem offset of slot 0 (smem slots)
    uint32_t spin_limit;                // producer waits: microseconds before one gives up
    uint32_t idle_polls;                // idle-walker polls before giving up (set by every launch)
    // global round caches (kMethodGCache jobs): group (cta, g) owns entries
    // [(cta * ng + g) * gcache_stride, +8 << h)
    uint16_t* gcache;
    uint32_t gcache_stride;
    // resident launch (rq != nullptr): `jobs` is a ring of ring_mask + 1
    // entries that the host fills ahead of `avail`; trial g belongs to the
    // first entry, scanning forward from entry_begin, whose range holds it;
    // the failure bitmap is a ring of bits_mask + 1 bits (bits_mask 0: no
    // ring); entry_done[e] counts the finished walks of ring entry e
    const ResidentQueue* rq;
    uint32_t ring_mask;
    uint32_t map_chains;                // lookup chains per lane from a round cache (0: automatic)
    uint32_t fill_blocks;               // round-cache fill: blocks per thread per step (0: automatic)
    uint32_t pool_stage;                // pooled direct passes: bytes per staging map (0: off)
    uint32_t pool_fold;                 // pooled direct passes: bytes per fold table (0: unfolded)
    unsigned long long entry_begin;
    unsigned long long bits_mask;
    unsigned int* entry_done;
};

// Batched calls: ONE persistent launch over the plan classes of a call (all
// classes of one entry width; see cmc_engine_fused).  Each
// class keeps its own engine arguments (plan, job range, control block and
// global pool region); CTAs [first_cta[c], first_cta[c + 1]) start on class c
// (in proportion to its estimated work), and a CTA whose class has no trials
// left to claim moves on to the class with the most estimated work left
// (unclaimed trials x cost per trial).
constexpr uint32_t kMaxFusedClasses = 16;
struct FusedArgs {
    EngineArgs cls[kMaxFusedClasses];
    float cost[kMaxFusedClasses];            // estimated AES blocks per trial
    uint16_t first_cta[kMaxFusedClasses + 1];
    uint32_t nclass;
};
static_assert(sizeof(FusedArgs) <= 4096, "fused launch arguments fit the classic parameter space");

// Serving: device-resident state of one admitted job.  `next` is the job's
// RNG counter -- the index of its next trial in the experiment, whose batch
// is next >> bt and offset next & (2^bt - 1); `job.batch_rk` caches the key of
// batch `key_batch`.
struct ServeState {
    Job job;
    unsigned long long seed;
    unsigned long long next;
    unsigned long long budget;
    unsigned long long key_batch;
    uint32_t bt, active;
};

// Serving: this iteration's share for one job.
struct Grant {
    uint32_t slot;
    uint32_t trials;
};

// Serving: where each table entry of an iteration came from.
struct GrantInfo {
    unsigned long long batch, base;
    uint32_t slot, first, count, pad;
};

}  // namespace cmc
