/*
 * cmc_oracle.h -- CPU restatement of the reference cuckoo Monte Carlo path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the GPU product is
 * compared against; nothing in the product links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
 * may use it.
 *
 * Parity pins (all checked by tests/test_oracle.py):
 *   - FIPS-197 AES-128 known answer        (cuckoo_bench.cu:332-344, cpu_trials.hpp:150-155)
 *   - batch-key AES vectors                (host_tests.cpp:37-46)
 *   - parameter derivations                (host_tests.cpp:158-159)
 *   - 32,768-trial golden failure lists    (cpu_golden.hpp:3-4, smoke_expected.json)
 *   - affine PNUM 3 known answers          (cpu_tests.cpp:30-39)
 *   - the reference's own CPU code (cpu_trials.hpp) compiled from its sources
 *     into oracle/_ref, at the benchmark shapes with B/kick overrides.
 */
#ifndef CMC_ORACLE_H
#define CMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    uint32_t mode;        /* 1 = bgh25 (random walk), 2 = drrt18 (cycling)      */
    uint32_t input_mode;  /* 0 = sequential, 1 = affine                         */
    uint32_t pnum;        /* t, items per trial                                 */
    uint32_t ell_i;       /* key domain is 2^ell_i                              */
    uint32_t k;           /* hash copies per item (reference: always 3)         */
    uint32_t buckets;     /* B                                                  */
    uint32_t kick;        /* eviction limit                                     */
    uint32_t half_bits;   /* Feistel half width h                               */
    uint64_t bucket_size; /* ceil(k * 2^ell_i / B)                              */
    uint64_t domain;      /* D = B * bucket_size                                */
    uint64_t mask;        /* 2^h - 1                                            */
    uint64_t range_mask;  /* 2^ell_i - 1                                        */
} orc_params;

typedef struct orc_stats {
    uint64_t probes;      /* table slots inspected                              */
    uint64_t evaluations; /* bucket() calls                                     */
    uint64_t distinct;    /* distinct (ordinal, copy) pairs evaluated           */
    uint64_t aes_blocks;  /* AES-128 blocks spent in the Feistel PRP            */
} orc_stats;

/* AES-128 on big-endian words (cuckoo_bench.cu:360-392). */
void orc_aes128(const uint32_t rk[44], uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                uint32_t out[4]);
/* Key schedule from 16 key bytes given as two little-endian u64 (cuckoo_bench.cu:86-99). */
void orc_expand_key(uint64_t lo, uint64_t hi, uint32_t rk[44]);
/* Key schedule from four big-endian key words (cuckoo_bench.cu:136-149). */
void orc_expand_key_words(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t rk[44]);
/* Per-batch AES key (cuckoo_bench.cu:393-404). */
void orc_batch_key(uint64_t seed, uint64_t batch_id, uint32_t rk[44]);
uint64_t orc_splitmix(uint64_t* state);

/* Reference parameters() (cuckoo_bench.cu:483-526), generalised to k copies.
 * buckets_override / kick_override of 0 keep the reference derivation.
 * Returns 0, or -1 when the derived domain would overflow. */
int orc_params_derive(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                      uint32_t buckets_override, uint32_t kick_override,
                      uint32_t input_mode, orc_params* out);
float orc_original_log2(uint64_t n);

/* Bucket of copy `which` of element `element` (cuckoo_bench.cu:161-184). */
uint32_t orc_bucket(const orc_params* p, const uint32_t prp_rk[44], uint64_t element,
                    uint32_t which);

/* Per-trial derived state (cuckoo_bench.cu:226-238). */
typedef struct orc_trial_seed {
    uint32_t prp_rk[44];
    uint64_t walk;        /* after the one splitmix advance */
    uint64_t randomness;
    uint64_t shift, step;
} orc_trial_seed;
void orc_trial_seed_derive(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
                           orc_trial_seed* out);

/* One trial (cpu_trials.hpp:69-127).  Returns 1 when the insertion failed.
 * `bins` (B entries, may be NULL) receives the final table, entry =
 * ordinal | choice << 16, 0xffffffff empty.  `stats` may be NULL. */
int orc_trial(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
              uint32_t* bins, orc_stats* stats);

/* Full bucket map of one trial: map[o*k + j] = bucket(o, j). */
void orc_trial_map(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
                   uint32_t* map);

/* Trials [first, first+count) of batch `batch_id`: writes the failing offsets
 * (sorted ascending) and returns their number.  `threads` <= 0 uses 1. */
uint32_t orc_batch(const orc_params* p, uint64_t seed, uint64_t batch_id, uint32_t first,
                   uint32_t count, int threads, uint32_t* out_offsets, orc_stats* stats);

#ifdef __cplusplus
}
#endif
#endif
