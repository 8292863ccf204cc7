/*
 * cmc.h -- C ABI of the B200 cuckoo-hashing Monte Carlo estimator (libcmc.so).
 *
 * The reference has no plugin layer; its replaceable seam is the Launch
 * callable that process_batch() invokes (cuckoo_bench.cu:724-736):
 *     launch(uint32_t n, uint32_t offset, const AesKey& batch_key,
 *            std::vector<uint32_t>& failures)
 * cmc_launch() is that seam as a C function: plain pointers and sizes, no
 * C++ or torch types.  Everything else here is the state the reference keeps
 * around that call (device set-up, parameters, batch keys) plus the batched
 * and served forms of the same computation.
 *
 * All functions return 0 on success or a negative CMC_E* code; they never
 * throw.  cmc_last_error() gives the message of the last failure on a
 * context (or on the calling thread when ctx is NULL).
 */
#ifndef CMC_H
#define CMC_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMC_OK 0
#define CMC_EINVAL (-1)       /* invalid argument or unsupported parameters   */
#define CMC_ECUDA (-2)        /* CUDA runtime error                           */
#define CMC_EKAT (-3)         /* device AES known-answer test failed          */
#define CMC_ETIMEOUT (-4)     /* a bounded device wait gave up                */
#define CMC_ERANGE (-5)       /* device result out of range (nf > n)          */
#define CMC_ENOMEM (-6)       /* allocation failed                            */

#define CMC_MODE_BGH25 1u     /* random-walk eviction (cuckoo_core.hpp:123-133) */
#define CMC_MODE_DRRT18 2u    /* cycling eviction     (cuckoo_core.hpp:134-158) */
#define CMC_INPUT_SEQUENTIAL 0u
#define CMC_INPUT_AFFINE 1u

/* Derived experiment parameters.  Mirrors Options+Params of the reference
 * (cuckoo_bench.cu:406-419, 499-526) with the copy count k generalised. */
typedef struct cmc_params {
    uint32_t mode;        /* CMC_MODE_*                                   */
    uint32_t input_mode;  /* CMC_INPUT_*                                  */
    uint32_t pnum;        /* t, items per trial, 3..65534                 */
    uint32_t ell_i;       /* key domain 2^ell_i, ell_i <= 61              */
    uint32_t k;           /* hash copies, 2..4 (reference: 3)             */
    uint32_t buckets;     /* B                                            */
    uint32_t kick;        /* eviction limit                               */
    uint32_t half_bits;   /* Feistel half width h                         */
    uint64_t bucket_size; /* ceil(k * 2^ell_i / B)                        */
    uint64_t domain;      /* D = B * bucket_size                          */
    uint64_t mask;        /* 2^h - 1                                      */
    uint64_t range_mask;  /* 2^ell_i - 1                                  */
} cmc_params;

/* parameters() (cuckoo_bench.cu:483-526), k-generalised; a zero override
 * keeps the reference derivation of B (resp. the eviction limit). */
int cmc_derive_params(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                      uint32_t buckets_override, uint32_t kick_override,
                      uint32_t input_mode, cmc_params* out);

/* batch_key(seed, batch_id) (cuckoo_bench.cu:393-404): the 44-word AES-128
 * key schedule of one batch. */
void cmc_batch_key(uint64_t seed, uint64_t batch_id, uint32_t out_w[44]);

/* Host AES-128 of one block under a 44-word schedule (cuckoo_bench.cu:360-392). */
void cmc_host_aes128(const uint32_t rk[44], const uint32_t in[4], uint32_t out[4]);

typedef struct cmc_ctx cmc_ctx;

/* Per-device set-up: table upload and the FIPS-197 known-answer test on the
 * device (cuckoo_bench.cu:1090-1095, 332-354).  One context per host thread. */
int cmc_init(int device, cmc_ctx** out);
int cmc_destroy(cmc_ctx* ctx);
const char* cmc_last_error(const cmc_ctx* ctx);

/* The Launch seam (cuckoo_bench.cu:980-1031): evaluate trials
 * [first, first+count) of the batch whose key schedule is batch_key (host
 * memory), append nothing and instead write the failing within-batch
 * offsets, ascending, to out_offsets (host memory, capacity count) and their
 * number to *out_nfailed.  Synchronous, like the reference. */
int cmc_launch(cmc_ctx* ctx, const cmc_params* params, const uint32_t batch_key[44],
               uint32_t first, uint32_t count, uint32_t* out_offsets, uint32_t* out_nfailed);

/* Device-resident form of cmc_launch: batch_key, out_offsets (capacity count)
 * and out_nfailed are device pointers; work is queued on `stream`
 * (cudaStream_t, NULL = the context's stream) and the call returns without
 * waiting.  cmc_check() afterwards reports bounded-wait timeouts. */
int cmc_launch_device(cmc_ctx* ctx, const cmc_params* params, const uint32_t* d_batch_key,
                      uint32_t first, uint32_t count, uint32_t* d_out_offsets,
                      uint32_t* d_out_nfailed, void* stream);
int cmc_check(cmc_ctx* ctx);

/* One entry of a batched launch: a parameter set and a run of trials of one
 * batch of its experiment (key = cmc_batch_key(seed, batch)). */
typedef struct cmc_job {
    cmc_params params;
    uint64_t seed;
    uint64_t batch;
    uint32_t first;  /* first within-batch offset */
    uint32_t count;  /* trials */
} cmc_job;

/* Batched form (no counterpart in the reference, which runs one parameter set
 * per process): all jobs in ONE persistent engine launch, heavy jobs first so
 * uneven table sizes balance across SMs.  Jobs whose best plans differ (walk
 * slots in shared or global memory, warps per group, entry width, cache kind)
 * form plan classes; each CTA runs one class at a time under that class's plan
 * and moves on to the class with the most work left when its own runs out.  out_failed[j] receives the number of
 * failing trials of job j.  If out_offsets is not NULL, the failing offsets are
 * written job by job in ascending order, out_jobs[i] (if not NULL) naming the
 * job of out_offsets[i]; cap is their capacity and *out_total the number of
 * failures (when it exceeds cap, only the counts are complete).  Total trials
 * per call must be below 2^32.  Synchronous. */
int cmc_run_jobs(cmc_ctx* ctx, const cmc_job* jobs, uint32_t njobs, uint64_t* out_failed,
                 uint32_t* out_offsets, uint32_t* out_jobs, uint64_t cap, uint64_t* out_total);

/* Autotuner: times candidate plans (warps per table, walker isolation, map
 * method) on a sample of every job (first count/sample_div trials, at least
 * one), keeps the fastest for this mix of parameter sets, and applies it to
 * later cmc_run_jobs calls with the same mix.  *out_choice (may be NULL)
 * receives a description of the chosen plan. */
int cmc_autotune(cmc_ctx* ctx, const cmc_job* jobs, uint32_t njobs, uint32_t sample_div,
                 const char** out_choice);

/* Serving (no counterpart in the reference): estimation jobs of different
 * sizes are submitted as they arrive and run together, continuously batched
 * into the persistent engine.  Job state (parameters, RNG counter = next trial,
 * budget, current batch key) and partial counts live on the device; each
 * cmc_server_step admits queued jobs while the device-memory budget allows,
 * grants trials to one size class of jobs (by default 95% of the step's work
 * in arrival order, the rest shortest remaining work first), runs one engine
 * launch over all grants and appends completed batches to each job's v3
 * journal (when a directory was given; an existing journal there is
 * resumed).  A budget runs as the first ceil(trials / 2^batch_bits) batches
 * of an experiment of 2^ceil(log2 trials) trials, so it is rounded up to
 * whole batches.  A job's failures are the same alone and in the mix. */
typedef struct cmc_server cmc_server;
int cmc_server_create(cmc_ctx* ctx, uint32_t max_jobs, uint64_t mem_budget_bytes,
                      uint32_t batch_bits, uint64_t max_iteration_trials, cmc_server** out);
int cmc_server_submit(cmc_server* server, const cmc_params* params, uint64_t seed,
                      uint64_t trials, const char* journal_dir, uint32_t* out_id);
/* One step.  Resident serving (the default): reads back finished work,
 * admits queued jobs, publishes grants worth about work_blocks AES blocks
 * whenever less than twice that is still unclaimed by the running launch,
 * and starts a launch if none runs; jobs are reported finished (up to cap ids
 * in out_finished) by the step that reads back their last trials.
 * Iterations ("resident" 0): work_blocks is the minimum AES-block budget of
 * the step's engine launch (it grows to an eighth of the outstanding work of
 * the granted size class, at most 20x, and to 2.5x the latency of the
 * slowest trial granted); launches are pipelined two deep, so a job is
 * reported by the call after the one that issued its last trials.
 * cmc_server_destroy commits the work still in flight before it frees the
 * server.  After a step returns an error (a device wait that gave up, a CUDA
 * error) the server's state is undefined: destroy it. */
int cmc_server_step(cmc_server* server, uint64_t work_blocks, uint32_t* out_finished,
                    uint32_t cap, uint32_t* out_nfinished);
/* out_state: 0 queued, 1 running, 2 done. */
int cmc_server_status(cmc_server* server, uint32_t job_id, uint64_t* out_trials_done,
                      uint64_t* out_failed, int* out_state);
/* Share (0..1, default 0.95) of each step's work granted in arrival order;
 * the rest goes shortest remaining work first.  1 is FIFO with backfill
 * (tail latency of plain per-job launches), lower shares favour short jobs:
 * measured on a 400-job stream, 0.95 keeps p99 at or below plain launches at
 * 60 and 200 jobs/s while halving p50; 0.5 cuts p50 by 5x but raises p99. */
int cmc_server_policy(cmc_server* server, double fifo_share);
/* Server options: "fifo_share" (as cmc_server_policy) and "resident" (0 or
 * 1, default 1).  Resident serving keeps one engine launch on the device
 * while jobs are pending: each step publishes grants into a job ring that
 * the running launch reads (completion is polled by copies; nothing waits
 * for a launch to end), and the launch exits once every active job's trials
 * are published and walked, so a busy period pays one launch tail.  While
 * jobs are pending, call cmc_server_step at least every few seconds: the
 * launch's wait for new work is bounded and reports CMC_ETIMEOUT past it. */
int cmc_server_set_option(cmc_server* server, const char* name, double value);
/* Device-time accounting of the iterations read back so far (CUDA events
 * around each engine launch): engine_ms sums the launches, busy_ms counts
 * time with at least one engine running once (pipelined iterations
 * overlap), span_ms runs from the first engine start to the last end. */
typedef struct cmc_server_stats {
    uint64_t iterations;
    uint64_t trials;
    double engine_ms;
    double busy_ms;
    double span_ms;
} cmc_server_stats;
int cmc_server_get_stats(const cmc_server* server, cmc_server_stats* out);
uint32_t cmc_server_pending(const cmc_server* server);
const char* cmc_server_error(const cmc_server* server);
int cmc_server_destroy(cmc_server* server);

/* Tuning knobs of the launch planner; value 0 (or -1 for "method") restores
 * the automatic choice.  Names: "warps_per_group" (1..15), "groups" (1..14),
 * "global_slots" (0/1: keep walk slots in global memory), "method"
 * (-1 auto, 0 direct AES passes, 1 round cache: in shared memory when the
 * PRP half width h <= 12, else in global memory, 2 round cache in global
 * memory, L2-resident, for any h <= 16), "walkers"
 * (1..4 walker warps), "isolate_walkers" (-1 auto, 0/1: walker warps alone
 * on SM sub-partition 3, producers on 0..2), "slots_per_group" (cap on
 * shared-memory slots per group, default 8), "walker_ctas" (-1 auto, 0 walks
 * inside each CTA, N > 0 dedicates N CTAs -- one per SM -- to walks over
 * global slots while the others only build maps), "spin_limit" (bound of a
 * device wait before it gives up with CMC_ETIMEOUT: microseconds for producer
 * waits, polls of a fraction of a microsecond for idle walkers -- 32x as many
 * in a resident server launch; default 2^26, about 67 s for producers),
 * "graph" (1, the default: cmc_run_jobs captures the device side of a call shape -- job shapes, counts and buffers -- into a CUDA
 * graph on its second call and replays it from the third; 0: always eager),
 * "map_chains" (0 automatic, or 1, 2, 4, 8: candidate lookup chains per lane
 * when a bucket map is built from a round cache), "fused" (1, the default:
 * the plan classes of a batched call run in one persistent launch whose CTAs
 * move to the class with the most work left; 0: one launch per class),
 * "fill_blocks" (0 automatic, or 2..4: AES blocks each thread keeps in flight
 * while filling a round cache, in plans whose walk slots are in shared
 * memory; automatic is 3 there and 2 elsewhere), "pool" (-1, the default:
 * one-warp groups whose jobs all take direct passes with 16-bit Feistel
 * halves and shared-memory walk slots keep three trials in flight and stage
 * their maps; 0: one trial at a time; 1 as -1 -- such plans run in a kernel
 * of their own, outside fused launches, and resident server launches never
 * pool).
 * Returns CMC_EINVAL for an unknown name or a value out of range. */
int cmc_set_option(cmc_ctx* ctx, const char* name, int64_t value);

/* No counterpart in the reference.  The Launch seam for callers that cannot
 * let this library allocate device memory -- e.g. a process whose device
 * memory is owned by another framework's caching allocator, or a service loop
 * that must not pay cudaMalloc/cudaFree's device-wide synchronisation.  Same
 * result as cmc_launch_device, on the current device, with no context and no
 * allocation: the working memory is a fixed file-scope device array (about
 * 129 KiB per GPU, held until the process exits).  Limits: count is 0..2^20
 * trials per call (0 writes *d_out_nfailed = 0, as cmc_launch_device does),
 * and parameter sets whose walk slots do not fit in shared memory are
 * rejected (CMC_EINVAL): among them every set that needs 32-bit table entries
 * (B > 65535 or t > 16384), whose bins and map exceed shared memory.  d_batch_key, d_out_offsets (capacity
 * count) and d_out_nfailed are device pointers; work is queued on `stream`.
 * The first call on a device sets up that device (symbol addresses, a 1 KiB
 * table upload), so it should come before any stream capture.  All calls on a
 * device share the working memory: calls that overlap on the GPU race, so order
 * them (e.g. one stream).  If a bounded device wait gives up or a device-side
 * check fails, *d_out_nfailed is set to 0xffffffff.  Errors:
 * cmc_last_error(NULL). */
int cmc_launch_static(const cmc_params* params, const uint32_t* d_batch_key, uint32_t first,
                      uint32_t count, uint32_t* d_out_offsets, uint32_t* d_out_nfailed,
                      void* stream);

/* Queue this context's host-buffer launches (cmc_launch) on `stream`
 * (cudaStream_t; NULL restores the context's own stream). */
int cmc_set_stream(cmc_ctx* ctx, void* stream);

/* Device time of the last engine kernel (CUDA events around that one
 * launch), in milliseconds; waits for it to finish.  -1 on error. */
double cmc_last_engine_ms(cmc_ctx* ctx);

/* Counters of the last checked launch (cmc_launch, or cmc_check after
 * cmc_launch_device): out[0] walks, out[1] probes, out[2] cycles producer
 * groups waited for a free slot, out[3] cycles walker warps had nothing to
 * walk, out[4] walker warps' total cycles, out[5] device error code. */
int cmc_last_stats(cmc_ctx* ctx, uint64_t out[6]);

/* Kernels launched by the last cmc_launch* call on this context. */
uint32_t cmc_last_kernel_count(const cmc_ctx* ctx);
/* Human-readable description of the last launch plan (engine, groups, ...). */
const char* cmc_last_plan(const cmc_ctx* ctx);
/* No counterpart in the reference.  Planner dry run, no device needed: writes
 * to out (cap bytes) the plan text cmc_launch would report for count trials
 * of params on a device with `sms` SMs and `smem_optin` bytes of opt-in
 * shared memory per block (148 and 232448 on B200), with default options.
 * Returns 0, or a CMC_E* code with the reason in out. */
int cmc_plan_describe(const cmc_params* params, uint32_t count, uint32_t sms, uint64_t smem_optin,
                      char* out, uint32_t cap);

#ifdef __cplusplus
}
#endif
#endif
