// cmc_engine.cu -- the per-trial Monte Carlo path on sm_100a.
//
// One persistent CTA per SM.  Its warps are split into
//   * NG producer groups of WG warps.  A group takes one trial at a time from
//     a global work counter, derives the trial's PRP key and walk seed
//     (cuckoo_bench.cu:226-238), and evaluates the bucket of every (item,
//     copy) pair -- the map -- either by direct 8-round AES Feistel passes or
//     from an 8*2^h round cache it builds first, in shared memory (h <= 12) or
//     in an L2-resident global buffer of its own (h <= 16)
//     (gpu_shared.cuh:70-91 is the reference's warp-per-trial version).  The
//     map and an empty table go into a slot.
//   * one walker warp.  Lane s owns slot s and runs the serial cuckoo
//     insertion walk (cuckoo_core.hpp:117-161) of the trial in it while the
//     producers already build later maps.  The reference runs that walk on
//     lane 0 of the producing warp with 31 lanes idle (gpu_shared.cuh:93).
// Failures are set in a bitmap indexed by the launch's global trial index and
// compacted in order by cmc_compact_failures (the reference appends offsets
// through an atomic counter and sorts on the host, cuckoo_bench.cu:313-316,738).
//
// All waits are bounded.  Producer waits (a free slot, new work in a resident
// launch) give up after spin_limit microseconds (%globaltimer); idle walkers
// count polls instead (a timer read in their loop measured 5x slower walks on
// global slots, as did one more value held across their loop) and give up
// after idle_polls polls, which the host always sets.  The
// kernel then records CMC_ETIMEOUT in Ctrl, with the waiting site in `where`,
// and returns.
#include <cstdint>

#include "cmc_aes.cuh"
#include "cmc_engine.cuh"

namespace cmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kErrBase = 3;     // == -CMC_EKAT: table_base_ok() failed
constexpr uint32_t kErrTimeout = 4;  // == -CMC_ETIMEOUT
constexpr uint32_t kErrRange = 5;    // == -CMC_ERANGE

struct GroupHeader {
    unsigned long long gidx;
    uint32_t job, offset;
    uint32_t rk[44];
    uint32_t r1[8][8];  // Round1 {c0, w3hi, c1, c2, c3} per Feistel round (padded)
    unsigned long long walk, rnd, shift, step;
    uint32_t slot, cand_next, abort, live;
    uint32_t done;             // pooled direct passes: candidates whose bucket is staged
    unsigned long long entry;  // resident launch: ring entry of the last trial
    unsigned long long avail;  // resident launch: the last published end this group read
    Job jd;                    // this trial's job descriptor, read at L2
};
static_assert(sizeof(GroupHeader) <= kGroupHeaderBytes, "the planner reserves kGroupHeaderBytes");

struct SlotHeader {
    unsigned long long gidx, walk, rnd;
    uint32_t job, offset;
};

struct CtaShared {
    uint32_t slot_state[kMaxSlots];
    SlotHeader slot_hdr[kMaxSlots];
    uint32_t groups_done;
    uint32_t next_class;  // fused launches: the class this CTA runs next
    EngineArgs args;      // fused launches: the current class's arguments
};
static_assert(sizeof(CtaShared) <= kCtaSharedBytes, "the planner reserves kCtaSharedBytes");

constexpr uint32_t kCtaSharedOff = kTableBytes;

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];"
                 : "=r"(v)
                 : "r"((uint32_t)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(p)),
                 "r"(v)
                 : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_acquire_sys(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 16-bit stores of the round cache fill, written as PTX.  As plain C++
// stores into the array that also holds the T-table, they cost one extra
// FMA-pipe instruction per table lookup of the loop (measured on B200 with a
// copy of the fill loop: 433 against 321 instructions per 32 blocks, 116
// against 4 on the FMA pipe; the producers' issue slots are the limit).  The
// memory clobber keeps them ordered with the other memory accesses.
__device__ __forceinline__ void st_shared_u16(uint16_t* p, uint32_t v) {
    asm volatile("st.shared.u16 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)),
                 "h"((unsigned short)v)
                 : "memory");
}

__device__ __forceinline__ void st_global_u16(uint16_t* p, uint32_t v) {
    asm volatile("st.global.u16 [%0], %1;" ::"l"(__cvta_generic_to_global(p)),
                 "h"((unsigned short)v)
                 : "memory");
}

// Map entries of the direct pass, written the same way (the slot holding the
// map sits in shared or global memory: a generic store).
__device__ __forceinline__ void st_map(uint16_t* p, uint32_t v) {
    asm volatile("st.u16 [%0], %1;" ::"l"(p), "h"((unsigned short)v) : "memory");
}

__device__ __forceinline__ void st_map(uint32_t* p, uint32_t v) {
    asm volatile("st.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void group_sync(uint32_t g, uint32_t nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(nthreads) : "memory");
}

__device__ __forceinline__ uint64_t splitmix(uint64_t& s) {
    s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// floor(y / width) for y < 2^32 with magic = floor((2^32 - 1) / width):
// the estimate is at most two below the quotient and never above it.
__device__ __forceinline__ uint32_t div_width(uint32_t y, uint32_t width, uint32_t magic) {
    uint32_t q = __umulhi(y, magic);
    uint32_t r = y - q * width;
    if (r >= width) { ++q; r -= width; }
    if (r >= width) { ++q; }
    return q;
}

// c / k for the copy counts k = 2, 3, 4: 0xAAAAAAAB = ceil(2^33 / 3) with a
// shift of 33 divides every 32-bit c by 3 exactly; 2 and 4 are shifts.
__device__ __forceinline__ uint32_t div_k(uint32_t c, uint32_t k) {
    return k == 3 ? __umulhi(c, 0xAAAAAAABu) >> 1 : c >> (k >> 1);
}

__device__ __forceinline__ uint32_t find_job(const Job* jobs, uint32_t njobs, uint64_t g) {
    uint32_t lo = 0, hi = njobs;  // last job with trial_base <= g
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (jobs[mid].trial_base <= g) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ Round1 load_round1(const GroupHeader* gh, uint32_t r) {
    const uint4 c4 = *reinterpret_cast<const uint4*>(&gh->r1[r][0]);
    return Round1{c4.x, c4.z, c4.w, gh->r1[r][4], c4.y};
}

// Warp-aggregated claim of candidate indices from a shared counter.
__device__ __forceinline__ uint32_t claim(uint32_t* counter, bool need, uint32_t lane) {
    const unsigned m = __ballot_sync(kFull, need);
    uint32_t base = 0;
    const int leader = __ffs(m) - 1;
    if (m && (int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(kFull, base, leader < 0 ? 0 : leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

// Per-trial PRP key schedule (cuckoo_bench.cu:226-232): the "KEY1" block of
// the trial's offset under the batch key, expanded into gh->rk.
__device__ __forceinline__ void trial_key(const Lanes& L, const Job& J, GroupHeader* gh) {
    uint32_t w[4];
    encrypt_full(L, J.batch_rk, 0x4b455931u, 0, gh->offset, 0x50525031u, w);
    expand_key(L, w[0], w[1], w[2], w[3], gh->rk);
}

// Per-trial walk seed and affine input map (cuckoo_bench.cu:233-238): the
// "WALK" block of the trial's offset under the batch key.
__device__ __forceinline__ void trial_walk_seed(const Lanes& L, const Job& J, GroupHeader* gh) {
    uint32_t w[4];
    encrypt_full(L, J.batch_rk, 0x57414c4bu, 0, gh->offset, 0x524e4731u, w);
    uint64_t walk = ((uint64_t)w[0] << 32) | w[1];
    const uint64_t shift = (((uint64_t)w[2] << 32) | w[3]) & J.range_mask;
    uint64_t input_state = shift ^ 0xd1b54a32d192ed03ULL;
    gh->step = (splitmix(input_state) | 1ULL) & J.range_mask;
    gh->shift = shift;
    gh->rnd = splitmix(walk);
    gh->walk = walk;
}

// Round-1 constants of Feistel round r (r < 8) into the trial's header.
__device__ __forceinline__ void store_round1(const Lanes& L, GroupHeader* gh, uint32_t r, uint32_t h) {
    const Round1 c = round1_consts(L, gh->rk, r, h);
    gh->r1[r][0] = c.c0; gh->r1[r][1] = c.w3hi; gh->r1[r][2] = c.c1;
    gh->r1[r][3] = c.c2; gh->r1[r][4] = c.c3;
}

// ---------------------------------------------------------------- producer --

// FOLD: rounds 1-2 of each pass from the trial's round-2 fold table, kept
// word-split (component c of entry v at fw[c * n + v], n = 8 << yb) so that a
// warp's loads of one component are conflict-free while a round has at most
// 32 entries (h <= 13): 111 table lookups and 4 fold loads per block instead
// of 124 lookups.
template <typename MapT, bool WIDE, bool FOLD = false>
__device__ __forceinline__ void build_map_direct(const Lanes& L, const Job& J, GroupHeader* gh,
                                                 const PrpKey& key, MapT* map, uint32_t lane,
                                                 const uint32_t* fw = nullptr) {
    const uint32_t k = J.k, ncand = J.pnum * k, h = J.half_bits;
    const uint64_t mask = J.mask, domain = J.domain;
    const bool sequential = J.input_mode == 0;
    const uint64_t shift = gh->shift, step = gh->step, range_mask = J.range_mask;
    uint32_t c = claim(&gh->cand_next, true, lane);
    bool has = c < ncand;
    uint64_t left = 0, right = 0;
    auto start = [&](uint32_t cand) {
        const uint32_t o = div_k(cand, k), j = cand - o * k;
        const uint64_t e = sequential ? (uint64_t)o : (shift + (uint64_t)o * step) & range_mask;
        const uint64_t y = e * k + j;
        left = y >> h;
        right = y & mask;
    };
    if (has) start(c);
    while (__any_sync(kFull, has)) {
        if constexpr (!WIDE) {
            uint32_t l = (uint32_t)left, r = (uint32_t)right;
            if constexpr (FOLD) {
                const uint32_t yb = h > 8 ? h - 8 : 0, n = 8u << yb;
#pragma unroll 1
                for (uint32_t rr = 0; rr < 8; ++rr) {
                    const uint2 k01 = *reinterpret_cast<const uint2*>(&gh->r1[rr][0]);
                    const uint32_t vi = (rr << yb) | (r >> 8);
                    const uint4 v = make_uint4(fw[vi], fw[n + vi], fw[2 * n + vi], fw[3 * n + vi]);
                    const uint32_t f = prp_f_folded(L, key, k01.x, k01.y, v, r) & (uint32_t)mask;
                    const uint32_t nr = (l ^ f) & (uint32_t)mask;
                    l = r;
                    r = nr;
                }
            } else {
#pragma unroll 1
                for (uint32_t rr = 0; rr < 8; ++rr) {
                    const Round1 rc = load_round1(gh, rr);
                    const uint32_t f = prp_f(L, key, rc, r) & (uint32_t)mask;
                    const uint32_t nr = (l ^ f) & (uint32_t)mask;
                    l = r;
                    r = nr;
                }
            }
            left = l;
            right = r;
        } else {
#pragma unroll 1
            for (uint32_t rr = 0; rr < 8; ++rr) {
                const uint32_t f = prp_f_wide(L, gh->rk, rr, h, (uint32_t)right);
                const uint64_t nr = (left ^ ((uint64_t)f & mask)) & mask;
                left = right;
                right = nr;
            }
        }
        const uint64_t y = (left << h) | right;
        const bool done = has && y < domain;
        if (done) {
            uint32_t b;
            if constexpr (!WIDE) b = div_width((uint32_t)y, (uint32_t)J.width, J.width_magic);
            else b = (uint32_t)(y / J.width);
            st_map(map + c, b);
        } else if (has) {
            left = y >> h;
            right = y & mask;
        }
        const uint32_t nc = claim(&gh->cand_next, done, lane);
        if (done) {
            c = nc;
            has = c < ncand;
            if (has) start(c);
        }
    }
}

// Candidates from a round cache (shared or global memory): 8 dependent
// lookups per Feistel evaluation.  CH independent candidates per lane keep CH
// lookup chains in flight, which hides the latency of an L2-resident cache.
template <typename MapT, int CH>
__device__ __forceinline__ void build_map_cache(const Job& J, GroupHeader* gh,
                                                const uint16_t* cache, MapT* map,
                                                uint32_t lane) {
    const uint32_t k = J.k, ncand = J.pnum * k, h = J.half_bits;
    const uint32_t mask = (uint32_t)J.mask;
    const uint32_t domain_m1 = (uint32_t)(J.domain - 1);
    const bool sequential = J.input_mode == 0;
    const uint64_t shift = gh->shift, step = gh->step, range_mask = J.range_mask;
    uint32_t c[CH], l[CH], r[CH];
    bool has[CH];
    auto start = [&](int i) {
        const uint32_t o = div_k(c[i], k), j = c[i] - o * k;
        const uint64_t e = sequential ? (uint64_t)o : (shift + (uint64_t)o * step) & range_mask;
        const uint32_t y = (uint32_t)(e * k + j);
        l[i] = y >> h;
        r[i] = y & mask;
    };
    bool any = false;
#pragma unroll
    for (int i = 0; i < CH; ++i) {
        c[i] = claim(&gh->cand_next, true, lane);
        has[i] = c[i] < ncand;
        l[i] = r[i] = 0;  // idle chains keep in-range indices
        if (has[i]) start(i);
        any |= has[i];
    }
    while (__any_sync(kFull, any)) {
#pragma unroll
        for (uint32_t rr = 0; rr < 8; ++rr) {
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                const uint32_t f = cache[(rr << h) | r[i]];
                const uint32_t nr = l[i] ^ f;
                l[i] = r[i];
                r[i] = nr;
            }
        }
        any = false;
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const uint32_t y = (l[i] << h) | r[i];
            const bool done = has[i] && y <= domain_m1;
            if (done) {
                map[c[i]] = (MapT)div_width(y, (uint32_t)J.width, J.width_magic);
            } else if (has[i]) {
                l[i] = y >> h;
                r[i] = y & mask;
            }
            const uint32_t nc = claim(&gh->cand_next, done, lane);
            if (done) {
                c[i] = nc;
                has[i] = c[i] < ncand;
                if (has[i]) start(i);
            }
            any |= has[i];
        }
    }
}

template <typename MapT>
__device__ __forceinline__ void map_from_cache(const Job& J, GroupHeader* gh, const uint16_t* cache,
                                               MapT* map, uint32_t lane, uint32_t chains) {
    if (chains >= 8) build_map_cache<MapT, 8>(J, gh, cache, map, lane);
    else if (chains >= 4) build_map_cache<MapT, 4>(J, gh, cache, map, lane);
    else if (chains == 2) build_map_cache<MapT, 2>(J, gh, cache, map, lane);
    else build_map_cache<MapT, 1>(J, gh, cache, map, lane);
}

// Round cache: entry (r, R) = F_r(R) & mask for the 8 rounds and every h-bit
// R, 8 * 2^h AES blocks.  N independent blocks per iteration: their unrolled
// round chains interleave, multiplying the ILP of each warp.  Rounds 1 and 2 come
// from the group's fold table (prp_f_folded): cache entry e = (r << h) | R
// uses fold entry (r << (h - 8)) | (R >> 8) = e >> 8 when h >= 8, and r =
// e >> h below.  A warp covers 32 consecutive R of one round (entries start
// 32-aligned), so its fold loads are one broadcast.
template <int N, bool SHARED>
__device__ __forceinline__ void fill_round_cache_n(const Lanes& L, const PrpKey& key,
                                                   const GroupHeader* gh, const uint4* fold,
                                                   uint16_t* cache, uint32_t h, uint32_t m,
                                                   uint32_t gt, uint32_t gthreads) {
    auto put = [&](uint32_t i, uint32_t v) {
        if constexpr (SHARED) st_shared_u16(cache + i, v);
        else st_global_u16(cache + i, v);
    };
    const uint32_t entries = 8u << h;
    const uint32_t vsh = h > 8 ? 8 : h;
    uint32_t e = gt;
    for (; e + (N - 1) * gthreads < entries; e += N * gthreads) {
        uint32_t f[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const uint32_t ei = e + i * gthreads;
            const uint2 k = *reinterpret_cast<const uint2*>(&gh->r1[ei >> h][0]);
            f[i] = prp_f_folded(L, key, k.x, k.y, fold[ei >> vsh], ei & m);
        }
#pragma unroll
        for (int i = 0; i < N; ++i) put(e + i * gthreads, f[i] & m);
    }
    for (; e < entries; e += gthreads) {
        const uint2 k = *reinterpret_cast<const uint2*>(&gh->r1[e >> h][0]);
        put(e, prp_f_folded(L, key, k.x, k.y, fold[e >> vsh], e & m) & m);
    }
}

// n independent blocks per thread per step.  Only the kernels with walk slots
// in shared memory carry the choice (default 3: t = 1024, B = 1536, N = 2^20
// measured 3.346 M trials/s with 2, 3.354 M with 3, 3.350 M with 4); the
// global-slot kernels keep a plain 2-block fill (cmc_engine below says why).
template <bool VAR, bool SHARED>
__device__ __forceinline__ void fill_round_cache(const Lanes& L, const PrpKey& key,
                                                 const GroupHeader* gh, const uint4* fold,
                                                 uint16_t* cache, uint32_t h, uint32_t m,
                                                 uint32_t gt, uint32_t gthreads, uint32_t n) {
    if (VAR && n == 4) fill_round_cache_n<4, SHARED>(L, key, gh, fold, cache, h, m, gt, gthreads);
    else if (VAR && n != 2) fill_round_cache_n<3, SHARED>(L, key, gh, fold, cache, h, m, gt, gthreads);
    else fill_round_cache_n<2, SHARED>(L, key, gh, fold, cache, h, m, gt, gthreads);
}

// The fold table of the group's current trial: entry v = (r, y) for Feistel
// round r and y = R >> 8 (fold_entry in cmc_aes.cuh).
__device__ __forceinline__ void build_fold_table(const Lanes& L, const PrpKey& key,
                                                 const GroupHeader* gh, uint4* fold, uint32_t h,
                                                 uint32_t gt, uint32_t gthreads) {
    const uint32_t yb = h > 8 ? h - 8 : 0;
    const uint32_t n = 8u << yb;
    for (uint32_t v = gt; v < n; v += gthreads) {
        const Round1 c = round1_consts(L, gh->rk, v >> yb, h);
        fold[v] = fold_entry(L, key, c, v & ((1u << yb) - 1u));
    }
}

// The same table word-split, for direct passes (build_map_direct<..., true>).
__device__ __forceinline__ void build_fold_table_split(const Lanes& L, const PrpKey& key,
                                                       const GroupHeader* gh, uint32_t* fw, uint32_t h,
                                                       uint32_t gt, uint32_t gthreads) {
    const uint32_t yb = h > 8 ? h - 8 : 0;
    const uint32_t n = 8u << yb;
    for (uint32_t v = gt; v < n; v += gthreads) {
        const Round1 c = round1_consts(L, gh->rk, v >> yb, h);
        const uint4 e = fold_entry(L, key, c, v & ((1u << yb) - 1u));
        fw[v] = e.x;
        fw[n + v] = e.y;
        fw[2 * n + v] = e.z;
        fw[3 * n + v] = e.w;
    }
}

template <typename MapT, typename BinT, bool WIDE, bool SPLIT, bool SMEMSLOTS>
__device__ __forceinline__ void producer(const EngineArgs& a, char* smem, CtaShared* cs, uint32_t g,
                                         uint32_t gt) {
    const uint32_t gthreads = a.wg * 32;
    const uint32_t lane = threadIdx.x & 31;
    const Lanes L{lane * 4, lane * 4 + 128, a.r256};
    char* gbase = smem + a.group_off + g * a.group_bytes;
    GroupHeader* gh = reinterpret_cast<GroupHeader*>(gbase);
    uint32_t cursor = 0;
    const unsigned long long total = a.total_dev ? *a.total_dev : a.total;

    if (gt == 0) {
        gh->entry = a.entry_begin;
        gh->avail = 0;
    }
    for (;;) {
        if (gt == 0) {
            const unsigned long long gi = a.gidx_begin + atomicAdd(&a.ctrl->next, 1ULL);
            gh->gidx = gi;
            gh->abort = 0;
            uint32_t live = gi < total;
            if (a.rq) {
                // Resident: wait until trial gi is published or the host
                // closes the launch.  Claims rise, so a group that leaves
                // holds an index past the final `avail`: every published
                // trial is taken by some group.
                // The wait backs off from 1 to 128 us between reads of host
                // memory (idle groups must not crowd the host's copies) and
                // gives up after spin_limit microseconds.
                live = gi < gh->avail;  // published as of this group's last read of host memory
                uint32_t nap = 1024;
                const unsigned long long t_start = globaltimer_ns();
                while (!live) {
                    const uint32_t stop = ld_acquire_sys(&a.rq->stop);
                    gh->avail = ld_acquire_sys(&a.rq->avail);
                    if (gi < gh->avail) {
                        live = 1;
                        break;
                    }
                    if (stop) break;
                    __nanosleep(nap);
                    nap = min(nap * 2, 131072u);
                    if (globaltimer_ns() - t_start > 1000ULL * a.spin_limit) {
                        atomicExch(&a.ctrl->error, kErrTimeout);
                        atomicExch(&a.ctrl->where, 6u);
                        break;
                    }
                }
                if (live) {
                    // the entry holding gi: entries are published in order
                    unsigned long long e = gh->entry;
                    uint32_t steps = 0;
                    for (;;) {
                        const Job* je = &a.jobs[e & a.ring_mask];
                        const unsigned long long base = __ldcg(&je->trial_base);
                        if (gi >= base && gi - base < __ldcg(&je->count)) {
                            gh->offset = __ldcg(&je->first) + (uint32_t)(gi - base);
                            break;
                        }
                        ++e;
                        if (++steps > a.ring_mask + 1) {  // inconsistent ring: never spin on it
                            atomicExch(&a.ctrl->error, kErrRange);
                            atomicExch(&a.ctrl->where, 5u);
                            live = 0;
                            break;
                        }
                    }
                    gh->entry = e;
                    gh->job = (uint32_t)(e & a.ring_mask);
                    // this trial's failure bit starts clear (the ring reuses bits)
                    if (live)
                        atomicAnd(&a.fail_bits[(gi & a.bits_mask) >> 5], ~(1u << (gi & 31)));
                }
            } else if (live) {
                const uint32_t j = find_job(a.jobs, a.njobs, gi);
                gh->job = j;
                gh->offset = a.jobs[j].first + (uint32_t)(gi - a.jobs[j].trial_base);
            }
            gh->live = live;
        }
        group_sync(g, gthreads);
        if (!gh->live) break;
        const unsigned long long gi = gh->gidx;
        {
            // this trial's job descriptor, read at L2: a resident ring entry
            // may have been rewritten since an earlier trial read it
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&a.jobs[gh->job]);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&gh->jd);
            for (uint32_t i = gt; i < sizeof(Job) / 4; i += gthreads) dst[i] = __ldcg(src + i);
        }
        group_sync(g, gthreads);
        const Job& J = gh->jd;

        // Per-trial PRP key and walk seed (cuckoo_bench.cu:226-238).
        if (gt == 0) {
            trial_key(L, J, gh);
            trial_walk_seed(L, J, gh);
            gh->cand_next = 0;
            // Claim a free slot (FREE -> FILLING).  In-CTA slots: any free
            // one, starting from this group's share of the pool.  Split
            // engine: the next slot of a global ring, waiting for its walk.
            uint32_t slot = 0xffffffffu;
            const long long wait0 = clock64();
            const unsigned long long wait_ns = globaltimer_ns();
            uint32_t ring = 0;
            if constexpr (SPLIT) ring = atomicAdd(&a.ctrl->slot_cursor, 1u) % a.ns;
            for (;;) {
                if constexpr (SPLIT) {
                    if (atomicCAS(&a.ghdr[ring].state, kSlotFree, kSlotFilling) == kSlotFree) slot = ring;
                } else {
                    for (uint32_t i = 0; i < a.ns; ++i) {
                        const uint32_t sidx = (g * (a.ns / a.ng) + cursor + i) % a.ns;
                        if (atomicCAS(&cs->slot_state[sidx], kSlotFree, kSlotFilling) == kSlotFree) {
                            slot = sidx;
                            break;
                        }
                    }
                }
                if (slot != 0xffffffffu) break;
                __nanosleep(128);
                if (globaltimer_ns() - wait_ns > 1000ULL * a.spin_limit) {
                    atomicExch(&a.ctrl->error, kErrTimeout);
                    atomicExch(&a.ctrl->where, 1u);
                    gh->abort = 1;
                    slot = 0;
                    break;
                }
            }
            gh->slot = slot;
            atomicAdd(&a.ctrl->slot_wait_cycles, (unsigned long long)(clock64() - wait0));
        }
        ++cursor;
        group_sync(g, gthreads);
        if (gh->abort) break;
        // the walker's last accesses to this slot happen-before ours
        if constexpr (SPLIT) __threadfence();
        else __threadfence_block();
        // A job uses a round cache only if this launch provides room for it
        // (a descriptor made under other options falls back to direct passes):
        // its fold table, and a shared-memory cache after it.
        const uint32_t cache_entries = 8u << J.half_bits;
        const uint32_t fold_end = kGroupHeaderBytes + fold_table_bytes(J.half_bits);
        const bool smem_cache = !WIDE && J.method == kMethodCache &&
                                fold_end + 2 * cache_entries <= a.group_bytes;
        const bool glob_cache = !WIDE && !smem_cache && J.method == kMethodGCache &&
                                a.gcache != nullptr && cache_entries <= a.gcache_stride &&
                                fold_end <= a.group_bytes;
        // direct passes take the fold too, in the shared-slot kernels (the
        // global-slot kernels are left as they are: their walks are sensitive
        // to the kernel's register allocation, cmc_engine below)
        const bool direct_fold = SMEMSLOTS && !WIDE && J.method == kMethodDirect && J.half_bits <= 13 &&
                                 fold_end <= a.group_bytes;
        uint4* fold = reinterpret_cast<uint4*>(gbase + kGroupHeaderBytes);
        PrpKey key;
        if constexpr (!WIDE) {
            prp_key_from_schedule(gh->rk, key);
            if (gt < 8) store_round1(L, gh, gt, J.half_bits);
            if (smem_cache || glob_cache) build_fold_table(L, key, gh, fold, J.half_bits, gt, gthreads);
            if constexpr (SMEMSLOTS) {
                if (direct_fold)
                    build_fold_table_split(L, key, gh, reinterpret_cast<uint32_t*>(fold), J.half_bits, gt,
                                           gthreads);
            }
        }
        group_sync(g, gthreads);

        const uint32_t slot = gh->slot;
        char* sbase = SPLIT    ? a.gslots + (size_t)slot * a.slot_stride
                      : a.gslots ? a.gslots + ((size_t)blockIdx.x * a.ns + slot) * a.slot_stride
                                 : smem + a.slots_off + (size_t)slot * a.slot_stride;
        BinT* bins = reinterpret_cast<BinT*>(sbase);
        MapT* map = reinterpret_cast<MapT*>(sbase + a.bins_bytes);
        {
            const uint32_t nvec = (J.buckets * (uint32_t)sizeof(BinT) + 15) / 16;
            uint4* b4 = reinterpret_cast<uint4*>(bins);
            for (uint32_t i = gt; i < nvec; i += gthreads) b4[i] = make_uint4(kFull, kFull, kFull, kFull);
        }
        if (smem_cache) {
            uint16_t* cache = reinterpret_cast<uint16_t*>(gbase + fold_end);
            fill_round_cache<SMEMSLOTS, true>(L, key, gh, fold, cache, J.half_bits, (uint32_t)J.mask,
                                              gt, gthreads, a.fill_blocks);
            group_sync(g, gthreads);
            map_from_cache<MapT>(J, gh, cache, map, lane, a.map_chains ? a.map_chains : 1);
        } else if (glob_cache) {
            uint16_t* gc = a.gcache + (size_t)(blockIdx.x * a.ng + g) * a.gcache_stride;
            fill_round_cache<SMEMSLOTS, false>(L, key, gh, fold, gc, J.half_bits, (uint32_t)J.mask,
                                               gt, gthreads, a.fill_blocks);
            group_sync(g, gthreads);  // orders the group's global writes before its reads
            // four chains hide L2/DRAM latency unless cycle-walking is heavy
            // (c = 2^2h / D > 2), where idle chains' gathers cost more than
            // the overlap gains (measured: t=1500, k=4, c~4: 4 chains 8% slower)
            const bool light_walk = (1ULL << (2 * J.half_bits)) <= 2 * J.domain;
            map_from_cache<MapT>(J, gh, gc, map, lane, a.map_chains ? a.map_chains : (light_walk ? 4 : 2));
        } else if (SMEMSLOTS && !WIDE && direct_fold) {
            build_map_direct<MapT, WIDE, SMEMSLOTS && !WIDE>(L, J, gh, key, map, lane,
                                                             reinterpret_cast<const uint32_t*>(fold));
        } else {
            build_map_direct<MapT, WIDE>(L, J, gh, key, map, lane);
        }
        if constexpr (SPLIT) __threadfence();
        else __threadfence_block();
        group_sync(g, gthreads);
        if (gt == 0) {
            if constexpr (SPLIT) {
                GSlotHeader& sh = a.ghdr[slot];
                sh.gidx = gi;
                sh.walk = gh->walk;
                sh.rnd = gh->rnd;
                sh.job = gh->job;
                sh.offset = gh->offset;
                __threadfence();
                st_release_gpu(&sh.state, kSlotReady);
            } else {
                SlotHeader& sh = cs->slot_hdr[slot];
                sh.gidx = gi;
                sh.walk = gh->walk;
                sh.rnd = gh->rnd;
                sh.job = gh->job;
                sh.offset = gh->offset;
                st_release(&cs->slot_state[slot], kSlotReady);
            }
        }
    }
    if (gt == 0) {
        if constexpr (SPLIT) {
            __threadfence();
            atomicAdd(&a.ctrl->groups_done, 1u);
        } else {
            __threadfence_block();
            atomicAdd(&cs->groups_done, 1u);
        }
    }
}

// Pooled direct passes for one-warp groups (the planner sets pool_stage only
// for launches whose jobs all use direct passes with 16-bit Feistel halves,
// walk slots in shared memory and no resident queue).  With one trial at a
// time, the last Feistel passes of each trial run with most lanes idle: the
// number of passes per candidate is geometric (cycle-walking), so a warp of
// 32 lanes on 192 candidates keeps ~78 % of its lanes busy.  Here the warp
// holds kPoolContexts trials: a lane whose context has no candidate left
// takes one from the next, loading that trial's key when it switches, and a
// finished trial is published (its staged map copied into a free slot) and
// replaced by the next one at the top of the loop, where the warp is
// converged.  A slot is held only while its map is copied.  With pool_fold
// set (h <= 10), rounds 1-2 of every pass come from the trial's round-2 fold
// table (fold_entry in cmc_aes.cuh), built when the trial starts.
template <typename MapT, typename BinT>
__device__ __forceinline__ void producer_pooled(const EngineArgs& a, char* smem, CtaShared* cs, uint32_t g,
                                                uint32_t lane) {
    const Lanes L{lane * 4, lane * 4 + 128, a.r256};
    char* gbase = smem + a.group_off + g * a.group_bytes;
    auto ctx = [&](uint32_t j) { return reinterpret_cast<GroupHeader*>(gbase + j * kPoolHeaderStride); };
    auto stage = [&](uint32_t j) {
        return reinterpret_cast<MapT*>(gbase + kPoolContexts * kPoolHeaderStride + j * a.pool_stage);
    };
    auto fold = [&](uint32_t j) {
        return reinterpret_cast<uint4*>(gbase + kPoolContexts * (kPoolHeaderStride + a.pool_stage) +
                                        j * a.pool_fold);
    };
    const unsigned long long total = a.total_dev ? *a.total_dev : a.total;
    if (lane < kPoolContexts) ctx(lane)->live = 0;
    __syncwarp();
    bool more = true, abort = false;
    uint32_t cursor = g;
    // this lane's trial parameters (those of context kj) and candidate
    int kj = -1, cj = -1;
    PrpKey key;
    uint32_t h = 0, mask = 0, kk = 0, width = 0, wmagic = 0, c = 0, l = 0, r = 0;
    uint64_t domain = 0, shift = 0, step = 0, rmask = 0;
    bool sequential = false;
    // take context j's key and parameters
    auto bind = [&](uint32_t j) {
        const GroupHeader* gh = ctx(j);
        const Job& J = gh->jd;
        prp_key_from_schedule(gh->rk, key);
        h = J.half_bits;
        mask = (uint32_t)J.mask;
        domain = J.domain;
        kk = J.k;
        width = (uint32_t)J.width;
        wmagic = J.width_magic;
        sequential = J.input_mode == 0;
        shift = gh->shift;
        step = gh->step;
        rmask = J.range_mask;
        kj = (int)j;
    };
    for (;;) {
        // converged: publish finished trials, start new ones
#pragma unroll 1
        for (uint32_t j = 0; j < kPoolContexts && !abort; ++j) {
            GroupHeader* gh = ctx(j);
            if (gh->live && gh->done == gh->jd.pnum * gh->jd.k) {
                const uint32_t ncand = gh->jd.pnum * gh->jd.k;
                uint32_t slot = 0;
                if (lane == 0) {
                    const long long wait0 = clock64();
                    const unsigned long long wait_ns = globaltimer_ns();
                    slot = 0xffffffffu;
                    for (;;) {
                        for (uint32_t i = 0; i < a.ns; ++i) {
                            const uint32_t sidx = (cursor + i) % a.ns;
                            if (atomicCAS(&cs->slot_state[sidx], kSlotFree, kSlotFilling) == kSlotFree) {
                                slot = sidx;
                                break;
                            }
                        }
                        if (slot != 0xffffffffu) break;
                        __nanosleep(128);
                        if (globaltimer_ns() - wait_ns > 1000ULL * a.spin_limit) {
                            atomicExch(&a.ctrl->error, kErrTimeout);
                            atomicExch(&a.ctrl->where, 1u);
                            break;
                        }
                    }
                    atomicAdd(&a.ctrl->slot_wait_cycles, (unsigned long long)(clock64() - wait0));
                }
                slot = __shfl_sync(kFull, slot, 0);
                if (slot == 0xffffffffu) {
                    abort = true;
                    break;
                }
                cursor = slot + 1;
                char* sbase = smem + a.slots_off + (size_t)slot * a.slot_stride;
                {
                    const uint32_t nvec = (gh->jd.buckets * (uint32_t)sizeof(BinT) + 15) / 16;
                    uint4* b4 = reinterpret_cast<uint4*>(sbase);
                    for (uint32_t i = lane; i < nvec; i += 32) b4[i] = make_uint4(kFull, kFull, kFull, kFull);
                    MapT* map = reinterpret_cast<MapT*>(sbase + a.bins_bytes);
                    const MapT* st = stage(j);
                    for (uint32_t i = lane; i < ncand; i += 32) map[i] = st[i];
                }
                __syncwarp();
                __threadfence_block();
                if (lane == 0) {
                    SlotHeader& sh = cs->slot_hdr[slot];
                    sh.gidx = gh->gidx;
                    sh.walk = gh->walk;
                    sh.rnd = gh->rnd;
                    sh.job = gh->job;
                    sh.offset = gh->offset;
                    st_release(&cs->slot_state[slot], kSlotReady);
                    gh->live = 0;
                }
                if (kj == (int)j) kj = -1;  // the context's next trial has another key
                __syncwarp();
            }
            if (!gh->live && more) {
                uint32_t claimed = 0;  // the claim holds a trial
                if (lane == 0) {
                    const unsigned long long gi = a.gidx_begin + atomicAdd(&a.ctrl->next, 1ULL);
                    gh->gidx = gi;
                    claimed = gi < total;
                    if (claimed) {
                        const uint32_t jb = find_job(a.jobs, a.njobs, gi);
                        gh->job = jb;
                        gh->offset = a.jobs[jb].first + (uint32_t)(gi - a.jobs[jb].trial_base);
                    }
                }
                claimed = __shfl_sync(kFull, claimed, 0);
                __syncwarp();
                if (!claimed) {
                    more = false;
                    continue;
                }
                {
                    const uint32_t* src = reinterpret_cast<const uint32_t*>(&a.jobs[gh->job]);
                    uint32_t* dst = reinterpret_cast<uint32_t*>(&gh->jd);
                    for (uint32_t i = lane; i < sizeof(Job) / 4; i += 32) dst[i] = __ldcg(src + i);
                }
                __syncwarp();
                const Job& J = gh->jd;
                // per-trial PRP key (lane 0) and walk seed (lane 1)
                if (lane == 0) {
                    trial_key(L, J, gh);
                } else if (lane == 1) {
                    trial_walk_seed(L, J, gh);
                    gh->cand_next = 0;
                    gh->done = 0;
                }
                __syncwarp();
                if (lane < 8) store_round1(L, gh, lane, J.half_bits);
                __syncwarp();
                if (a.pool_fold) {
                    // the trial's round-2 fold table (fold_entry in cmc_aes.cuh),
                    // built with its key; lanes take their own trial's key back
                    // before their next pass
                    prp_key_from_schedule(gh->rk, key);
                    kj = -1;
                    const uint32_t yb = J.half_bits > 8 ? J.half_bits - 8 : 0;
                    uint4* fd = fold(j);
                    for (uint32_t v = lane; v < (8u << yb); v += 32)
                        fd[v] = fold_entry(L, key, load_round1(gh, v >> yb), v & ((1u << yb) - 1u));
                    __syncwarp();
                }
                if (lane == 0) gh->live = 1;
                __syncwarp();
            }
        }
        if (abort) break;
        bool any_live = false;
        for (uint32_t j = 0; j < kPoolContexts; ++j) any_live |= ctx(j)->live != 0;
        if (!any_live) break;
        // lanes without a candidate take one, from the contexts in order
#pragma unroll 1
        for (uint32_t j = 0; j < kPoolContexts; ++j) {
            GroupHeader* gh = ctx(j);
            const bool need = cj < 0 && gh->live;
            const uint32_t nc = claim(&gh->cand_next, need, lane);
            if (need && nc < gh->jd.pnum * gh->jd.k) {
                cj = (int)j;
                c = nc;
                if (kj != (int)j) bind(j);
                const uint32_t o = div_k(c, kk), jc = c - o * kk;
                const uint64_t e = sequential ? (uint64_t)o : (shift + (uint64_t)o * step) & rmask;
                const uint32_t y = (uint32_t)(e * kk + jc);
                l = y >> h;
                r = y & mask;
            }
        }
        // one Feistel pass (8 rounds) per lane with a candidate
        if (cj >= 0) {
            if (kj != cj) bind((uint32_t)cj);
            const GroupHeader* gh = ctx((uint32_t)cj);
            if (a.pool_fold) {
                // rounds 1-2 from the fold table: entry (rr, R >> 8)
                const uint4* fd = fold((uint32_t)cj);
                const uint32_t yb = h > 8 ? h - 8 : 0;
#pragma unroll 1
                for (uint32_t rr = 0; rr < 8; ++rr) {
                    const uint2 k01 = *reinterpret_cast<const uint2*>(&gh->r1[rr][0]);
                    const uint32_t f = prp_f_folded(L, key, k01.x, k01.y, fd[(rr << yb) | (r >> 8)], r) & mask;
                    const uint32_t nr = (l ^ f) & mask;
                    l = r;
                    r = nr;
                }
            } else {
#pragma unroll 1
                for (uint32_t rr = 0; rr < 8; ++rr) {
                    const Round1 rc = load_round1(gh, rr);
                    const uint32_t f = prp_f(L, key, rc, r) & mask;
                    const uint32_t nr = (l ^ f) & mask;
                    l = r;
                    r = nr;
                }
            }
            const uint32_t y = (l << h) | r;
            if (y < domain) {
                stage((uint32_t)cj)[c] = (MapT)div_width(y, width, wmagic);
                atomicAdd(&ctx((uint32_t)cj)->done, 1u);
                cj = -1;
            } else {
                l = y >> h;
                r = y & mask;
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        __threadfence_block();
        atomicAdd(&cs->groups_done, 1u);
    }
}

// ------------------------------------------------------------------ walker --

// Slot storage seen by one walker lane: shared-memory offsets or global
// pointers.  Shared-memory accesses are written as PTX with the dynamic-shared
// base as the immediate, like the T-table lookups (lds in cmc_aes.cuh):
// measured +0.4 % at t=64 and t=300, equal elsewhere.
template <typename MapT, typename BinT, bool SMEM>
struct SlotMem;

template <typename MapT, typename BinT>
struct SlotMem<MapT, BinT, true> {
    uint32_t map_off, bin_off;
    __device__ __forceinline__ void bind(const EngineArgs& a, uint32_t slot) {
        bin_off = a.slots_off + slot * a.slot_stride;
        map_off = bin_off + a.bins_bytes;
    }
    __device__ __forceinline__ uint32_t map(uint32_t i) const {
        const uint32_t off = map_off + i * (uint32_t)sizeof(MapT);
        if constexpr (sizeof(MapT) == 2) {
            unsigned short v;
            asm volatile("ld.shared.u16 %0, [%1+" CMC_STR(CMC_DYN_SMEM_BASE) "];" : "=h"(v) : "r"(off));
            return v;
        } else {
            uint32_t v;
            asm volatile("ld.shared.u32 %0, [%1+" CMC_STR(CMC_DYN_SMEM_BASE) "];" : "=r"(v) : "r"(off));
            return v;
        }
    }
    __device__ __forceinline__ BinT bin(uint32_t i) const {
        const uint32_t off = bin_off + i * (uint32_t)sizeof(BinT);
        if constexpr (sizeof(BinT) == 2) {
            unsigned short v;
            asm volatile("ld.shared.u16 %0, [%1+" CMC_STR(CMC_DYN_SMEM_BASE) "];" : "=h"(v) : "r"(off));
            return (BinT)v;
        } else {
            uint32_t v;
            asm volatile("ld.shared.u32 %0, [%1+" CMC_STR(CMC_DYN_SMEM_BASE) "];" : "=r"(v) : "r"(off));
            return (BinT)v;
        }
    }
    __device__ __forceinline__ void set(uint32_t i, BinT v) const {
        const uint32_t off = bin_off + i * (uint32_t)sizeof(BinT);
        if constexpr (sizeof(BinT) == 2)
            asm volatile("st.shared.u16 [%0+" CMC_STR(CMC_DYN_SMEM_BASE) "], %1;" ::"r"(off),
                         "h"((unsigned short)v) : "memory");
        else
            asm volatile("st.shared.u32 [%0+" CMC_STR(CMC_DYN_SMEM_BASE) "], %1;" ::"r"(off), "r"((uint32_t)v)
                         : "memory");
    }
};

// Global slots are read and written at L2 (ld/st .cg): a slot is refilled by
// another thread, possibly on another SM, so no stale L1 line may serve it.
template <typename MapT, typename BinT>
struct SlotMem<MapT, BinT, false> {
    const MapT* mp;
    BinT* bp;
    __device__ __forceinline__ void bind(const EngineArgs& a, uint32_t slot) {
        char* base = a.gslots + (a.split ? (size_t)slot : ((size_t)blockIdx.x * a.ns + slot)) * a.slot_stride;
        bp = reinterpret_cast<BinT*>(base);
        mp = reinterpret_cast<const MapT*>(base + a.bins_bytes);
    }
    __device__ __forceinline__ uint32_t map(uint32_t i) const { return __ldcg(mp + i); }
    __device__ __forceinline__ BinT bin(uint32_t i) const { return __ldcg(bp + i); }
    __device__ __forceinline__ void set(uint32_t i, BinT v) const { __stcg(bp + i, v); }
};

// One lane's insertion walk over a filled slot (cuckoo_core.hpp:117-161).
// A map entry is a bucket index < B by construction (y < D = B * width);
// any other value is recorded as an error instead of being dereferenced.
template <typename MapT, typename BinT, bool SMEM>
struct Walk {
    static constexpr uint32_t kShift = sizeof(BinT) == 2 ? 14 : 16;
    static constexpr uint32_t kOrdMask = (1u << kShift) - 1u;
    static constexpr uint32_t kEmpty = sizeof(BinT) == 2 ? 0xffffu : 0xffffffffu;

    SlotMem<MapT, BinT, SMEM> mem;
    uint64_t walk, rnd, magic, digits, digits_next;
    uint32_t magic_shift, k, t, kick, nbins, ndigits, ndigits_next;
    uint32_t item, cur, count, phase, choice, target;
    bool bgh, active, failed, bad;

    __device__ __forceinline__ void begin(const EngineArgs& a, uint32_t slot, const Job& J,
                                          const SlotHeader& h) {
        mem.bind(a, slot);
        walk = h.walk;
        rnd = h.rnd;
        // at L2: a resident ring entry may have been rewritten since this SM
        // last read it
        k = __ldcg(&J.k);
        t = __ldcg(&J.pnum);
        kick = __ldcg(&J.kick);
        nbins = __ldcg(&J.buckets);
        bgh = __ldcg(&J.mode) == 1;
        // rnd / k == umulhi(rnd, magic) >> magic_shift for k in {2, 3, 4}
        magic = k == 3 ? 0xAAAAAAAAAAAAAAABULL : (k == 2 ? 0x8000000000000000ULL : 0x4000000000000000ULL);
        magic_shift = k == 3 ? 1 : 0;
        item = 0; cur = 0; count = 0; phase = 0; choice = 0; target = 0;
        digits = digits_next = 0;
        ndigits = ndigits_next = 0;
        active = true;
        failed = false;
        bad = false;
    }

    __device__ __forceinline__ BinT pack(uint32_t o, uint32_t j) const { return (BinT)(o | (j << kShift)); }

    __device__ __forceinline__ bool out_of_range(uint32_t b) {
        if (b < nbins) return false;
        bad = failed = true;
        active = false;
        return true;
    }

    // The next 32 base-k digits of the walk's randomness, exactly as the
    // reference consumes them one per probe ("if (r < k) r = splitmix(walk);
    // which = r % k; r /= k", cuckoo_core.hpp:126-127), packed 2 bits each.
    // The stream does not depend on the table, so it is decoded ahead of the
    // probes and stays off their load-to-load dependency chain.
    __device__ __forceinline__ uint64_t next_digits() {
        uint64_t d = 0;
#pragma unroll 4
        for (uint32_t i = 0; i < 32; ++i) {
            if (rnd < k) rnd = splitmix(walk);
            const uint64_t q = __umul64hi(rnd, magic) >> magic_shift;
            d |= (uint64_t)((uint32_t)rnd - (uint32_t)q * k) << (2 * i);
            rnd = q;
        }
        return d;
    }

    // Keeps at least 32 digits buffered (the current word and the next), for
    // walks over shared-memory slots.  The walker calls it before every
    // bgh_steps(32): the lanes of a warp decode their next words together,
    // once per 32 probes, instead of one lane at a time inside the probe loop
    // with the others waiting (measured at t = 1024, B = 1536: producers'
    // waits for a free slot 3.5e9 -> 0.8e9 cycles, 3.36 -> 3.47 M trials/s).
    __device__ __forceinline__ void top_up() {
        if (active && ndigits_next == 0) {
            digits_next = next_digits();
            ndigits_next = 32;
        }
    }

    // BGH25 random walk (cuckoo_core.hpp:123-133).  The table write happens
    // on every non-failing probe; on the failing probe the trial ends and its
    // table is never read again, so the write is harmless and unconditional.
    // Shared-memory slots take their digits from the buffer top_up fills;
    // global slots keep the digits decoded inside the loop: the walkers over
    // global slots ran ~3x slower with the buffer (the register-allocation
    // sensitivity described at cmc_engine below).  Loading the next item's
    // map entry beside each bin read (it is the next target whenever the bin
    // is empty) measured 1 % slower on shared slots and is not done.
    __device__ __forceinline__ void bgh_steps(int n, unsigned long long& probes) {
#pragma unroll 1
        for (int s = 0; s < n && active; ++s) {
            if (ndigits == 0) {
                if constexpr (SMEM) {
                    digits = digits_next;
                    ndigits = ndigits_next;
                    ndigits_next = 0;
                } else {
                    digits = next_digits();
                    ndigits = 32;
                }
            }
            const uint32_t which = (uint32_t)digits & 3u;
            digits >>= 2;
            --ndigits;
            probe(mem.map(cur * k + which), which, probes);
        }
    }

    // One probe: copy `which` of item cur goes to bin tgt.
    __device__ __forceinline__ void probe(uint32_t tgt, uint32_t which, unsigned long long& probes) {
        if (tgt >= nbins) {
            bad = true;
            tgt = 0;
        }
        const uint32_t old = mem.bin(tgt);
        mem.set(tgt, pack(cur, which));
        ++probes;
        const bool empty = old == kEmpty;
        item += empty;
        count = empty ? 0 : count + 1;
        cur = empty ? item : (old & kOrdMask);
        const bool fail = count > kick || bad;
        failed = fail;
        active = !fail && item != t;
    }

    // DRRT18: one probe per step.
    __device__ __forceinline__ void drrt_steps(int n, unsigned long long& probes) {
#pragma unroll 1
        for (int s = 0; s < n && active; ++s) drrt_step(probes);
    }

    // DRRT18 cycling eviction (cuckoo_core.hpp:134-158), one probe.
    __device__ __forceinline__ void drrt_step(unsigned long long& probes) {
        ++probes;
        if (phase == 0) {
            // a new item tries its copies in order
            const uint32_t b = mem.map(item * k + choice);
            if (out_of_range(b)) return;
            if (mem.bin(b) == kEmpty) {
                mem.set(b, pack(item, choice));
                ++item;
                choice = 0;
                active = item != t;
            } else if (++choice == k) {
                phase = 1;
                cur = item;
                choice = 0;
                target = mem.map(item * k);
                count = 0;
                out_of_range(target);
            }
            return;
        }
        const uint32_t displaced = mem.bin(target);
        if (displaced == kEmpty) {
            mem.set(target, pack(cur, choice));
            ++item;
            phase = 0;
            choice = 0;
            active = item != t;
            return;
        }
        if (count >= kick) {
            failed = true;
            active = false;
            return;
        }
        mem.set(target, pack(cur, choice));
        cur = displaced & kOrdMask;
        choice = (displaced >> kShift) & 3u;
        const uint32_t previous = target;
        bool found = false;
        for (uint32_t j = 0; j < k; ++j) {
            choice = choice + 1 == k ? 0 : choice + 1;
            const uint32_t next = mem.map(cur * k + choice);
            if (next != previous) {
                target = next;
                found = true;
                break;
            }
        }
        if (!found) {
            failed = true;
            active = false;
            return;
        }
        if (out_of_range(target)) return;
        ++count;
    }
};

template <typename MapT, typename BinT, bool SMEM>
__device__ __forceinline__ void walker(const EngineArgs& a, CtaShared* cs, uint32_t wi) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t my = lane * a.nw + wi;  // this lane's slot
    const bool owner = my < a.ns;
    Walk<MapT, BinT, SMEM> w;
    w.active = false;
    w.bgh = true;
    bool busy = false;  // holds a slot
    unsigned long long gidx = 0;
    uint32_t job = 0;
    unsigned long long probes = 0, walks = 0, idle_cycles = 0;
    uint32_t idle = 0;
    const long long born = clock64();
    for (;;) {
        if (!busy && owner && ld_acquire(&cs->slot_state[my]) == kSlotReady) {
            const SlotHeader h = cs->slot_hdr[my];
            job = h.job;
            gidx = h.gidx;
            w.begin(a, my, a.jobs[job], h);
            busy = true;
        }
        if (w.bgh) {
            if constexpr (SMEM) {
                w.top_up();
                w.bgh_steps(32, probes);
            } else {
                w.bgh_steps(64, probes);
            }
        }
        else w.drrt_steps(64, probes);
        if (busy && !w.active) {
            if (w.bad) {
                atomicExch(&a.ctrl->error, kErrRange);
                atomicExch(&a.ctrl->where, 3u);
            }
            const uint32_t cidx = a.count_by_user ? __ldcg(&a.jobs[job].user) : job;
            if (w.failed) {
                const unsigned long long bit = a.bits_mask ? (gidx & a.bits_mask) : gidx;
                atomicOr(&a.fail_bits[bit >> 5], 1u << (bit & 31));
                if (a.job_failed) atomicAdd(&a.job_failed[cidx], 1ULL);
            }
            if (a.job_done) atomicAdd(&a.job_done[cidx], 1ULL);
            if (a.entry_done) {
                __threadfence();  // the failure bit is visible before the count
                atomicAdd(&a.entry_done[job], 1u);
            }
            ++walks;
            busy = false;
            __threadfence_block();
            st_release(&cs->slot_state[my], kSlotFree);
        }
        if (!__any_sync(kFull, busy)) {
            // Every lane acquires groups_done itself; the warp leaves only when
            // all lanes saw every group finished and no slot is still READY.
            const bool done = __all_sync(kFull, ld_acquire(&cs->groups_done) == a.ng);
            const bool ready = owner && ld_acquire(&cs->slot_state[my]) == kSlotReady;
            if (!__any_sync(kFull, ready)) {
                if (done) break;
                const long long t0 = clock64();
                __nanosleep(128);
                idle_cycles += (unsigned long long)(clock64() - t0);
                if (++idle > a.idle_polls) {  // a kernel parameter: no register held in the loop
                    if (lane == 0) {
                        atomicExch(&a.ctrl->error, kErrTimeout);
                        atomicExch(&a.ctrl->where, 2u);
                    }
                    break;
                }
            }
        } else {
            idle = 0;
        }
    }
    // warp totals for diagnostics
    for (int o = 16; o; o >>= 1) {
        probes += __shfl_xor_sync(kFull, probes, o);
        walks += __shfl_xor_sync(kFull, walks, o);
    }
    if (lane == 0) {
        atomicAdd(&a.ctrl->probes, probes);
        atomicAdd(&a.ctrl->walks, walks);
        atomicAdd(&a.ctrl->walker_idle_cycles, idle_cycles);
        atomicAdd(&a.ctrl->walker_cycles, (unsigned long long)(clock64() - born));
    }
}

// Split engine walker: every thread of a walker CTA owns one global slot.
template <typename MapT, typename BinT>
__device__ __forceinline__ void walker_split(const EngineArgs& a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t my = (blockIdx.x - a.producer_ctas) * blockDim.x + threadIdx.x;
    const bool owner = my < a.ns;
    GSlotHeader* hdr = owner ? &a.ghdr[my] : a.ghdr;
    Walk<MapT, BinT, false> w;
    w.active = false;
    w.bgh = true;
    bool busy = false;
    unsigned long long gidx = 0;
    uint32_t job = 0;
    unsigned long long probes = 0, walks = 0, idle_cycles = 0;
    uint32_t idle = 0;
    const long long born = clock64();
    for (;;) {
        if (!busy && owner && ld_acquire_gpu(&hdr->state) == kSlotReady) {
            SlotHeader h;
            h.gidx = __ldcg(&hdr->gidx);
            h.walk = __ldcg(&hdr->walk);
            h.rnd = __ldcg(&hdr->rnd);
            h.job = __ldcg(&hdr->job);
            h.offset = __ldcg(&hdr->offset);
            job = h.job;
            gidx = h.gidx;
            w.begin(a, my, a.jobs[job], h);
            busy = true;
        }
        if (w.bgh) w.bgh_steps(64, probes);
        else w.drrt_steps(64, probes);
        if (busy && !w.active) {
            if (w.bad) {
                atomicExch(&a.ctrl->error, kErrRange);
                atomicExch(&a.ctrl->where, 3u);
            }
            const uint32_t cidx = a.count_by_user ? __ldcg(&a.jobs[job].user) : job;
            if (w.failed) {
                const unsigned long long bit = a.bits_mask ? (gidx & a.bits_mask) : gidx;
                atomicOr(&a.fail_bits[bit >> 5], 1u << (bit & 31));
                if (a.job_failed) atomicAdd(&a.job_failed[cidx], 1ULL);
            }
            if (a.job_done) atomicAdd(&a.job_done[cidx], 1ULL);
            if (a.entry_done) {
                __threadfence();  // the failure bit is visible before the count
                atomicAdd(&a.entry_done[job], 1u);
            }
            ++walks;
            busy = false;
            __threadfence();
            st_release_gpu(&hdr->state, kSlotFree);
        }
        if (!__any_sync(kFull, busy)) {
            const bool done = __all_sync(kFull, ld_acquire_gpu(&a.ctrl->groups_done) == a.total_groups);
            const bool ready = owner && ld_acquire_gpu(&hdr->state) == kSlotReady;
            if (!__any_sync(kFull, ready)) {
                if (done) break;
                const long long t0 = clock64();
                __nanosleep(256);
                idle_cycles += (unsigned long long)(clock64() - t0);
                if (++idle > a.idle_polls) {  // a kernel parameter: no register held in the loop
                    if (lane == 0) {
                        atomicExch(&a.ctrl->error, kErrTimeout);
                        atomicExch(&a.ctrl->where, 4u);
                    }
                    break;
                }
            }
        } else {
            idle = 0;
        }
    }
    for (int o = 16; o; o >>= 1) {
        probes += __shfl_xor_sync(kFull, probes, o);
        walks += __shfl_xor_sync(kFull, walks, o);
        idle_cycles += __shfl_xor_sync(kFull, idle_cycles, o);
    }
    if (lane == 0) {
        atomicAdd(&a.ctrl->probes, probes);
        atomicAdd(&a.ctrl->walks, walks);
        atomicAdd(&a.ctrl->walker_idle_cycles, idle_cycles / 32);
        atomicAdd(&a.ctrl->walker_cycles, (unsigned long long)(clock64() - born));
    }
}

// Bank-replicated table: row x = [T0[x] x 32][ror16(T0[x]) x 32].
__device__ __forceinline__ void build_table(const uint32_t* t0, char* smem) {
    uint32_t* tw = reinterpret_cast<uint32_t*>(smem);
    for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) {
        const uint32_t v = __ldg(&t0[i >> 6]);
        tw[i] = (i & 32) ? __funnelshift_r(v, v, 16) : v;
    }
}

// Warp roles of one engine run over `a` (the caller has built the table and
// cleared the CTA's slot states).  Warp w issues from SM sub-partition w % 4.
// With isolate_walkers the nw walker warps take ids 15, 11, 7, 3 (all on
// sub-partition 3) and producers take sub-partitions 0..2 first (12 warps),
// then the sub-partition-3 ids no walker uses.  The latency-bound walks then
// share their issue slots with few or no throughput-bound AES warps.  Warps
// with no role return at once.  SMEMSLOTS: the plan keeps its walk slots in
// shared memory (a.gslots null) or, if false, in global memory.
template <typename MapT, typename BinT, bool WIDE, bool SMEMSLOTS, bool POOL = false>
__device__ __forceinline__ void engine_roles(const EngineArgs& a, char* smem, CtaShared* cs) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t producer_idx = 0xffffffffu, walker_idx = 0xffffffffu;
    if (a.isolate_walkers) {
        if ((warp & 3) != 3) producer_idx = warp - (warp >> 2);
        else if ((15 - warp) / 4 < a.nw) walker_idx = (15 - warp) / 4;
        else producer_idx = 12 + (warp >> 2);
    } else if (warp < a.ng * a.wg) {
        producer_idx = warp;
    } else {
        walker_idx = warp - a.ng * a.wg;
    }
    if (producer_idx < a.ng * a.wg) {
        const uint32_t g = producer_idx / a.wg;
        if constexpr (POOL) producer_pooled<MapT, BinT>(a, smem, cs, g, lane);
        else producer<MapT, BinT, WIDE, false, SMEMSLOTS>(a, smem, cs, g, (producer_idx % a.wg) * 32 + lane);
    } else if (walker_idx < a.nw) {
        walker<MapT, BinT, SMEMSLOTS>(a, cs, walker_idx);
    }
}

__device__ __forceinline__ void reset_cta_slots(CtaShared* cs) {
    for (uint32_t i = threadIdx.x; i < kMaxSlots; i += blockDim.x) cs->slot_state[i] = kSlotFree;
    if (threadIdx.x == 0) cs->groups_done = 0;
}

}  // namespace

template <typename MapT, typename BinT, bool WIDE>
__global__ void __launch_bounds__(512, 1) cmc_engine_split(const EngineArgs a) {
    if (!table_base_ok()) {
        if (threadIdx.x == 0) atomicExch(&a.ctrl->error, kErrBase);
        return;
    }
    if (blockIdx.x >= a.producer_ctas) {
        walker_split<MapT, BinT>(a);
        return;
    }
    char* smem = cmc_dyn_smem;
    build_table(a.t0, smem);
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5;
    if (warp < a.ng * a.wg)
        producer<MapT, BinT, WIDE, true, false>(a, smem, nullptr, warp / a.wg,
                                         threadIdx.x - (warp / a.wg) * a.wg * 32);
}

// One instantiation per entry width and walk-slot placement.  The walkers'
// loop over global slots (two dependent L2/DRAM round trips per probe) turned
// ~4.4x slower when anything changed the register allocation of the kernel
// around it -- a 3- and 4-block variant of the round-cache fill, one more
// value held in the walker (measured, on B200; round trips per warp step
// 5.2k -> 23k cycles) -- so the global-slot kernels are compiled without those
// and the shared-slot kernels, whose walks are unaffected, keep the
// fill_blocks choice.
template <typename MapT, typename BinT, bool WIDE, bool SMEMSLOTS>
__global__ void __launch_bounds__(512, 1) cmc_engine(const EngineArgs a) {
    if (!table_base_ok()) {
        if (threadIdx.x == 0) atomicExch(&a.ctrl->error, kErrBase);
        return;
    }
    char* smem = cmc_dyn_smem;
    build_table(a.t0, smem);
    CtaShared* cs = reinterpret_cast<CtaShared*>(smem + kCtaSharedOff);
    reset_cta_slots(cs);
    __syncthreads();
    engine_roles<MapT, BinT, WIDE, SMEMSLOTS>(a, smem, cs);
}

// Pooled direct passes (producer_pooled): 16-bit Feistel halves, walk slots in
// shared memory.  A kernel of its own, so that the other kernels' register
// allocation is unchanged.
template <typename MapT, typename BinT>
__global__ void __launch_bounds__(512, 1) cmc_engine_pooled(const EngineArgs a) {
    if (!table_base_ok()) {
        if (threadIdx.x == 0) atomicExch(&a.ctrl->error, kErrBase);
        return;
    }
    char* smem = cmc_dyn_smem;
    build_table(a.t0, smem);
    CtaShared* cs = reinterpret_cast<CtaShared*>(smem + kCtaSharedOff);
    reset_cta_slots(cs);
    __syncthreads();
    engine_roles<MapT, BinT, false, true, true>(a, smem, cs);
}

// Plan classes of a batched call in one launch (FusedArgs in cmc_engine.cuh),
// all of one entry width and walk-slot placement.  A class's run ends for a
// CTA when its producers find no trial left to claim and its walker has walked
// every filled slot; the CTA then picks its next class.  The table is built
// once.
template <typename MapT, typename BinT, bool WIDE, bool SMEMSLOTS>
__global__ void __launch_bounds__(512, 1) cmc_engine_fused(const __grid_constant__ FusedArgs f) {
    if (!table_base_ok()) {
        if (threadIdx.x < f.nclass) atomicExch(&f.cls[threadIdx.x].ctrl->error, kErrBase);
        return;
    }
    char* smem = cmc_dyn_smem;
    build_table(f.cls[0].t0, smem);
    CtaShared* cs = reinterpret_cast<CtaShared*>(smem + kCtaSharedOff);
    uint32_t c = 0;
    while (c + 1 < f.nclass && blockIdx.x >= f.first_cta[c + 1]) ++c;
    for (;;) {
        // the class's arguments, copied to shared memory: the roles read them
        // at shared-memory latency rather than through generic loads of the
        // parameter block
        reset_cta_slots(cs);
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&f.cls[c]);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&cs->args);
            for (uint32_t i = threadIdx.x; i < sizeof(EngineArgs) / 4; i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        engine_roles<MapT, BinT, WIDE, SMEMSLOTS>(cs->args, smem, cs);
        __syncthreads();
        if (threadIdx.x == 0) {
            // the class with the most estimated work left; none: this CTA is done
            uint32_t best = 0xffffffffu;
            float best_left = 0.0f;
            for (uint32_t k = 0; k < f.nclass; ++k) {
                const EngineArgs& b = f.cls[k];
                const unsigned long long claimed = atomicAdd(&b.ctrl->next, 0ULL);
                const unsigned long long size = b.total - b.gidx_begin;
                if (atomicAdd(&b.ctrl->error, 0u) || claimed >= size) continue;
                const float left = float(size - claimed) * f.cost[k];
                if (left > best_left) {
                    best_left = left;
                    best = k;
                }
            }
            cs->next_class = best;
        }
        __syncthreads();
        c = cs->next_class;
        if (c >= f.nclass) break;
    }
}

// Ordered failure list from the bitmap: one CTA, block-wide exclusive scan.
// out[i] = value_base + (index of the i-th set bit) for i < cap; *count = the
// number of set bits.
__global__ void __launch_bounds__(1024) cmc_compact_failures(const uint32_t* __restrict__ bits,
                                                             uint64_t nbits, uint32_t value_base,
                                                             uint32_t* __restrict__ out,
                                                             uint32_t* __restrict__ count,
                                                             uint64_t cap,
                                                             const unsigned long long* nbits_dev) {
    __shared__ uint32_t warp_sums[32];
    if (nbits_dev) nbits = *nbits_dev;
    const uint64_t words = (nbits + 31) / 32;
    const uint64_t per = (words + blockDim.x - 1) / blockDim.x;
    const uint64_t w0 = per * threadIdx.x, w1 = min(words, w0 + per);
    uint32_t mine = 0;
    for (uint64_t w = w0; w < w1; ++w) mine += __popc(bits[w]);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = blockDim.x / 32;
        uint32_t v = lane < nw ? warp_sums[lane] : 0, s = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(kFull, s, o);
            if (lane >= (uint32_t)o) s += u;
        }
        if (lane < nw) warp_sums[lane] = s - v;  // exclusive
        if (lane == nw - 1) *count = s;
    }
    __syncthreads();
    uint32_t at = warp_sums[warp] + incl - mine;
    for (uint64_t w = w0; w < w1; ++w) {
        uint32_t b = bits[w];
        while (b) {
            const int i = __ffs(b) - 1;
            b &= b - 1;
            if (at < cap) out[at] = value_base + (uint32_t)(w * 32 + i);
            ++at;
        }
    }
}

// Device self-test: the FIPS-197 AES-128 vector on every lane through the
// shared-memory table, and the 124-lookup PRP round function and its folded
// form against the full encryption for pseudo-random keys, rounds and inputs.
__global__ void cmc_selftest(const uint32_t* t0, const uint32_t* fips_rk, uint32_t* out,
                             uint32_t r256) {
    char* smem = cmc_dyn_smem;
    uint32_t* tw = reinterpret_cast<uint32_t*>(smem);
    for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) {
        const uint32_t v = t0[i >> 6];
        tw[i] = (i & 32) ? __funnelshift_r(v, v, 16) : v;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const Lanes L{lane * 4, lane * 4 + 128, r256};
    uint32_t c[4];
    encrypt_full(L, fips_rk, 0x00112233u, 0x44556677u, 0x8899aabbu, 0xccddeeffu, c);
    uint32_t bad = table_base_ok() ? 0u : 16u;
    if (c[0] != 0x69c4e0d8u || c[1] != 0x6a7b0430u || c[2] != 0xd8cdb780u || c[3] != 0x70b4c55au)
        bad |= 1;
    // key expansion from words reproduces the FIPS schedule
    uint32_t rk[44];
    expand_key(L, fips_rk[0], fips_rk[1], fips_rk[2], fips_rk[3], rk);
    for (int i = 0; i < 44; ++i)
        if (rk[i] != fips_rk[i]) bad |= 2;
    uint64_t s = 0x1234567ULL + threadIdx.x;
    for (int it = 0; it < 8; ++it) {
        const uint32_t a = (uint32_t)splitmix(s), b = (uint32_t)splitmix(s);
        const uint32_t cc = (uint32_t)splitmix(s), d = (uint32_t)splitmix(s);
        expand_key(L, a, b, cc, d, rk);
        PrpKey key;
        prp_key_from_schedule(rk, key);
        const uint32_t h = 2 + (uint32_t)(splitmix(s) % 15);  // 2..16
        const uint32_t r = (uint32_t)(splitmix(s) & 7);
        const uint32_t R = (uint32_t)splitmix(s) & ((1u << h) - 1u);
        const Round1 rc = round1_consts(L, rk, r, h);
        uint32_t full[4];
        encrypt_full(L, rk, 0x43455350u, r, h, R, full);
        if ((prp_f(L, key, rc, R) & 0xffffu) != (full[3] & 0xffffu)) bad |= 4;
        // the round-2 fold of the round-cache fill gives the same value
        const uint4 v = fold_entry(L, key, rc, R >> 8);
        if ((prp_f_folded(L, key, rc.c0, rc.w3hi, v, R) & 0xffffu) != (full[3] & 0xffffu)) bad |= 8;

    }
    out[threadIdx.x] = bad;
}

// Explicit instantiations used by the launcher.
template __global__ void cmc_engine<uint16_t, uint16_t, false, true>(const EngineArgs);
template __global__ void cmc_engine<uint32_t, uint32_t, false, true>(const EngineArgs);
template __global__ void cmc_engine<uint32_t, uint32_t, true, true>(const EngineArgs);
template __global__ void cmc_engine<uint16_t, uint16_t, false, false>(const EngineArgs);
template __global__ void cmc_engine<uint32_t, uint32_t, false, false>(const EngineArgs);
template __global__ void cmc_engine<uint32_t, uint32_t, true, false>(const EngineArgs);
template __global__ void cmc_engine_pooled<uint16_t, uint16_t>(const EngineArgs);
template __global__ void cmc_engine_pooled<uint32_t, uint32_t>(const EngineArgs);
template __global__ void cmc_engine_split<uint16_t, uint16_t, false>(const EngineArgs);
template __global__ void cmc_engine_split<uint32_t, uint32_t, false>(const EngineArgs);
template __global__ void cmc_engine_split<uint32_t, uint32_t, true>(const EngineArgs);
template __global__ void cmc_engine_fused<uint16_t, uint16_t, false, true>(const __grid_constant__ FusedArgs);
template __global__ void cmc_engine_fused<uint32_t, uint32_t, false, true>(const __grid_constant__ FusedArgs);
template __global__ void cmc_engine_fused<uint32_t, uint32_t, true, true>(const __grid_constant__ FusedArgs);
template __global__ void cmc_engine_fused<uint16_t, uint16_t, false, false>(const __grid_constant__ FusedArgs);
template __global__ void cmc_engine_fused<uint32_t, uint32_t, false, false>(const __grid_constant__ FusedArgs);
template __global__ void cmc_engine_fused<uint32_t, uint32_t, true, false>(const __grid_constant__ FusedArgs);

}  // namespace cmc
