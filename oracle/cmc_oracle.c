/*
 * cmc_oracle.c -- CPU restatement of the reference cuckoo Monte Carlo path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see cmc_oracle.h.
 *
 * Every function names the reference lines it restates.  The S-box is
 * computed from its definition (inverse in GF(2^8) followed by the FIPS-197
 * affine map) rather than transcribed; round computations are the textbook
 * T-table formulation of FIPS-197 on big-endian words.
 */
#include "cmc_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ AES -- */

static uint8_t g_sbox[256];
static uint32_t g_te[4][256];
static pthread_once_t g_tables_once = PTHREAD_ONCE_INIT;

static uint8_t gf_mul(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    while (b) {
        if (b & 1) r ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
        b >>= 1;
    }
    return r;
}

static uint8_t rotl8(uint8_t x, int s) { return (uint8_t)((x << s) | (x >> (8 - s))); }

static void build_tables(void) {
    for (int x = 0; x < 256; ++x) {
        uint8_t inv = 0;
        if (x) {
            for (int y = 1; y < 256; ++y)
                if (gf_mul((uint8_t)x, (uint8_t)y) == 1) { inv = (uint8_t)y; break; }
        }
        g_sbox[x] = (uint8_t)(inv ^ rotl8(inv, 1) ^ rotl8(inv, 2) ^ rotl8(inv, 3) ^
                              rotl8(inv, 4) ^ 0x63);
    }
    for (int x = 0; x < 256; ++x) {
        const uint32_t s = g_sbox[x], s2 = gf_mul((uint8_t)s, 2), s3 = gf_mul((uint8_t)s, 3);
        /* column (2s, s, s, 3s) of MixColumns, most significant byte first */
        const uint32_t t = (s2 << 24) | (s << 16) | (s << 8) | s3;
        g_te[0][x] = t;
        g_te[1][x] = (t >> 8) | (t << 24);
        g_te[2][x] = (t >> 16) | (t << 16);
        g_te[3][x] = (t >> 24) | (t << 8);
    }
}

static void ensure_tables(void) { pthread_once(&g_tables_once, build_tables); }

static uint32_t sub_word(uint32_t v) {
    return ((uint32_t)g_sbox[v >> 24] << 24) | ((uint32_t)g_sbox[(v >> 16) & 255] << 16) |
           ((uint32_t)g_sbox[(v >> 8) & 255] << 8) | g_sbox[v & 255];
}

void orc_expand_key_words(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t rk[44]) {
    ensure_tables();
    rk[0] = a; rk[1] = b; rk[2] = c; rk[3] = d;
    uint32_t rcon = 1;
    for (int i = 4; i < 44; ++i) {
        uint32_t v = rk[i - 1];
        if ((i & 3) == 0) {
            v = sub_word((v << 8) | (v >> 24)) ^ (rcon << 24);
            rcon = (uint32_t)gf_mul((uint8_t)rcon, 2);
        }
        rk[i] = rk[i - 4] ^ v;
    }
}

void orc_expand_key(uint64_t lo, uint64_t hi, uint32_t rk[44]) {
    /* The 16 key bytes are lo's bytes (little-endian) then hi's; each schedule
     * word packs four consecutive bytes most-significant first. */
    uint8_t kb[16];
    for (int i = 0; i < 8; ++i) {
        kb[i] = (uint8_t)(lo >> (8 * i));
        kb[8 + i] = (uint8_t)(hi >> (8 * i));
    }
    uint32_t w[4];
    for (int j = 0; j < 4; ++j)
        w[j] = ((uint32_t)kb[4 * j] << 24) | ((uint32_t)kb[4 * j + 1] << 16) |
               ((uint32_t)kb[4 * j + 2] << 8) | kb[4 * j + 3];
    orc_expand_key_words(w[0], w[1], w[2], w[3], rk);
}

void orc_aes128(const uint32_t rk[44], uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                uint32_t out[4]) {
    ensure_tables();
    uint32_t s[4] = {a ^ rk[0], b ^ rk[1], c ^ rk[2], d ^ rk[3]};
    for (int r = 1; r < 10; ++r) {
        uint32_t t[4];
        for (int j = 0; j < 4; ++j)
            t[j] = g_te[0][s[j] >> 24] ^ g_te[1][(s[(j + 1) & 3] >> 16) & 255] ^
                   g_te[2][(s[(j + 2) & 3] >> 8) & 255] ^ g_te[3][s[(j + 3) & 3] & 255] ^
                   rk[4 * r + j];
        memcpy(s, t, sizeof t);
    }
    for (int j = 0; j < 4; ++j)
        out[j] = (((uint32_t)g_sbox[s[j] >> 24] << 24) |
                  ((uint32_t)g_sbox[(s[(j + 1) & 3] >> 16) & 255] << 16) |
                  ((uint32_t)g_sbox[(s[(j + 2) & 3] >> 8) & 255] << 8) |
                  g_sbox[s[(j + 3) & 3] & 255]) ^ rk[40 + j];
}

/* -------------------------------------------------------- seeds, splitmix -- */

uint64_t orc_splitmix(uint64_t* state) {
    /* splitmix64 (cuckoo_bench.cu:150-156, cuckoo_core.hpp:110-114) */
    *state += 0x9E3779B97F4A7C15ULL;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

void orc_batch_key(uint64_t seed, uint64_t batch_id, uint32_t rk[44]) {
    /* cuckoo_bench.cu:393-404: AES-PRG block of the batch id under the
     * seed-derived master key, folded back into a fresh key schedule. */
    uint32_t master[44], x[4];
    orc_expand_key(seed, seed ^ 0x9e3779b97f4a7c15ULL, master);
    orc_aes128(master, 0x42415443u, (uint32_t)(batch_id >> 32), (uint32_t)batch_id,
               0x50524731u, x);
    const uint64_t prg_lo = ((uint64_t)x[0] << 32) | x[1];
    const uint64_t prg_hi = ((uint64_t)x[2] << 32) | x[3];
    orc_expand_key(seed ^ prg_lo, prg_hi ^ (seed ^ 0x243f6a8885a308d3ULL), rk);
}

void orc_trial_seed_derive(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
                           orc_trial_seed* out) {
    /* cuckoo_bench.cu:226-238 / cpu_trials.hpp:71-80 */
    uint32_t w[4];
    orc_aes128(batch_rk, 0x4b455931u, 0, offset, 0x50525031u, w);
    orc_expand_key_words(w[0], w[1], w[2], w[3], out->prp_rk);
    orc_aes128(batch_rk, 0x57414c4bu, 0, offset, 0x524e4731u, w);
    uint64_t walk = ((uint64_t)w[0] << 32) | w[1];
    out->shift = (((uint64_t)w[2] << 32) | w[3]) & p->range_mask;
    uint64_t input_state = out->shift ^ 0xd1b54a32d192ed03ULL;
    out->step = (orc_splitmix(&input_state) | 1ULL) & p->range_mask;
    out->randomness = orc_splitmix(&walk);
    out->walk = walk;
}

/* ------------------------------------------------------------ parameters -- */

static unsigned bit_width_u64(uint64_t v) {
    unsigned n = 0;
    while (v) { ++n; v >>= 1; }
    return n;
}

float orc_original_log2(uint64_t n) {
    /* cuckoo_bench.cu:488-498.  The DRRT18 bucket count is defined through
     * this float-valued series, so the same operations must be evaluated in
     * the same order to reproduce it bit for bit. */
    if (n == 0) return -INFINITY;
    const unsigned e = bit_width_u64(n) - 1;
    const double x = (double)n / (double)(1ULL << e);
    if (x >= 2.0) return (float)(e + 1);
    const double z = (x - 1.0) / (x + 1.0), z2 = z * z;
    double term = z, sum = 0.0;
    for (int i = 1; i <= 23; i += 2) {
        sum += term / i;
        term *= z2;
    }
    return (float)((double)e + 2.0 * sum * 1.4426950408889634074);
}

int orc_params_derive(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                      uint32_t buckets_override, uint32_t kick_override,
                      uint32_t input_mode, orc_params* out) {
    memset(out, 0, sizeof *out);
    out->mode = mode;
    out->input_mode = input_mode;
    out->pnum = pnum;
    out->ell_i = ell_i;
    out->k = k;
    if (mode == 1) {
        const uint64_t overhead = pnum < 30 ? 100 : 50;
        out->buckets = (uint32_t)((uint64_t)pnum * (100 + overhead) / 100);
        out->kick = 3 * pnum;
    } else {
        const float lf = orc_original_log2(pnum);
        const float f = (float)((double)pnum * ((double)(170.0f + lf) / 123.5));
        out->buckets = (uint32_t)ceil((double)f);
        out->kick = 100;
    }
    if (buckets_override) out->buckets = buckets_override;
    if (kick_override) out->kick = kick_override;
    const uint64_t source = ((uint64_t)1 << ell_i) * k;
    out->bucket_size = source / out->buckets + (source % out->buckets != 0);
    if (out->buckets > UINT64_MAX / out->bucket_size) return -1;
    out->domain = out->buckets * out->bucket_size;
    uint32_t bits = bit_width_u64(out->domain - 1);
    if (bits < 2) bits = 2;
    if (bits & 1u) ++bits;
    out->half_bits = bits / 2;
    out->mask = (1ULL << out->half_bits) - 1ULL;
    out->range_mask = (ell_i >= 64) ? ~0ULL : ((1ULL << ell_i) - 1ULL);
    return 0;
}

/* ------------------------------------------------------------ PRP bucket -- */

static uint32_t bucket_counted(const orc_params* p, const uint32_t rk[44], uint64_t element,
                               uint32_t which, uint64_t* aes_blocks) {
    /* cuckoo_bench.cu:161-184: 8 Feistel rounds with the AES round function
     * AES_k("CESP", round, h, right).w3, cycle-walked into [0, D). */
    uint64_t y = element * p->k + which;
    do {
        uint64_t left = y >> p->half_bits, right = y & p->mask;
        for (uint32_t r = 0; r < 8; ++r) {
            uint32_t o[4];
            orc_aes128(rk, 0x43455350u, r, p->half_bits, (uint32_t)right, o);
            const uint64_t next = (left ^ ((uint64_t)o[3] & p->mask)) & p->mask;
            left = right;
            right = next;
        }
        if (aes_blocks) *aes_blocks += 8;
        y = (left << p->half_bits) | right;
    } while (y >= p->domain);
    return (uint32_t)(y / p->bucket_size);
}

uint32_t orc_bucket(const orc_params* p, const uint32_t prp_rk[44], uint64_t element,
                    uint32_t which) {
    return bucket_counted(p, prp_rk, element, which, NULL);
}

/* ----------------------------------------------------------------- trial -- */

#define ORC_EMPTY 0xffffffffu

typedef struct trial_ctx {
    const orc_params* p;
    const orc_trial_seed* seed;
    orc_stats* st;
    uint8_t* seen; /* k*t flags for the distinct-pair statistic, or NULL */
} trial_ctx;

static uint64_t element_of(const trial_ctx* c, uint32_t ordinal) {
    if (c->p->input_mode == 0) return ordinal;
    return (c->seed->shift + (uint64_t)ordinal * c->seed->step) & c->p->range_mask;
}

static uint32_t cand(trial_ctx* c, uint32_t ordinal, uint32_t which) {
    if (c->st) {
        c->st->evaluations++;
        if (c->seen && !c->seen[(size_t)ordinal * c->p->k + which]) {
            c->seen[(size_t)ordinal * c->p->k + which] = 1;
            c->st->distinct++;
        }
    }
    return bucket_counted(c->p, c->seed->prp_rk, element_of(c, ordinal), which,
                          c->st ? &c->st->aes_blocks : NULL);
}

int orc_trial(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
              uint32_t* bins_out, orc_stats* stats) {
    /* cpu_trials.hpp:69-127 (and cuckoo_core.hpp:117-161), generalised from
     * 3 to k copies: base-k digits for BGH25, cycling modulo k for DRRT18. */
    orc_trial_seed seed;
    orc_trial_seed_derive(p, batch_rk, offset, &seed);
    uint32_t* bins = bins_out ? bins_out : (uint32_t*)malloc(sizeof(uint32_t) * p->buckets);
    uint8_t* seen = stats ? (uint8_t*)calloc((size_t)p->pnum * p->k, 1) : NULL;
    trial_ctx c = {p, &seed, stats, seen};
    for (uint32_t i = 0; i < p->buckets; ++i) bins[i] = ORC_EMPTY;
    uint64_t walk = seed.walk, randomness = seed.randomness;
    const uint32_t k = p->k;
    int failed = 0;
    for (uint32_t item = 0; item < p->pnum && !failed; ++item) {
        if (p->mode == 1) {
            uint32_t cur = item, collisions = 0;
            for (;;) {
                if (randomness < k) randomness = orc_splitmix(&walk);
                const uint32_t which = (uint32_t)(randomness % k);
                randomness /= k;
                const uint32_t b = cand(&c, cur, which);
                const uint32_t old = bins[b];
                if (stats) stats->probes++;
                if (old == ORC_EMPTY) { bins[b] = cur | (which << 16); break; }
                if (++collisions > p->kick) { failed = 1; break; }
                bins[b] = cur | (which << 16);
                cur = old & 65535u;
            }
        } else {
            const uint32_t initial = cand(&c, item, 0);
            if (stats) stats->probes++;
            if (bins[initial] == ORC_EMPTY) { bins[initial] = item; continue; }
            int inserted = 0;
            for (uint32_t j = 1; j < k; ++j) {
                const uint32_t b = cand(&c, item, j);
                if (stats) stats->probes++;
                if (bins[b] == ORC_EMPTY) { bins[b] = item | (j << 16); inserted = 1; break; }
            }
            if (inserted) continue;
            uint32_t cur = item, choice = 0, target = initial, kicks = 0;
            for (;;) {
                const uint32_t displaced = bins[target];
                if (stats) stats->probes++;
                if (displaced == ORC_EMPTY) { bins[target] = cur | (choice << 16); break; }
                if (kicks >= p->kick) { failed = 1; break; }
                bins[target] = cur | (choice << 16);
                cur = displaced & 65535u;
                choice = (displaced >> 16) & 3u;
                const uint32_t previous = target;
                int found = 0;
                for (uint32_t s = 0; s < k; ++s) {
                    choice = (choice + 1) % k;
                    const uint32_t next = cand(&c, cur, choice);
                    if (next != previous) { target = next; found = 1; break; }
                }
                if (!found) { failed = 1; break; }
                ++kicks;
            }
        }
    }
    if (!bins_out) free(bins);
    free(seen);
    return failed;
}

void orc_trial_map(const orc_params* p, const uint32_t batch_rk[44], uint32_t offset,
                   uint32_t* map) {
    orc_trial_seed seed;
    orc_trial_seed_derive(p, batch_rk, offset, &seed);
    trial_ctx c = {p, &seed, NULL, NULL};
    for (uint32_t o = 0; o < p->pnum; ++o)
        for (uint32_t j = 0; j < p->k; ++j) map[(size_t)o * p->k + j] = cand(&c, o, j);
}

/* ----------------------------------------------------------------- batch -- */

typedef struct batch_job {
    const orc_params* p;
    uint32_t rk[44];
    uint32_t first, count;
    uint32_t next;              /* shared work counter (atomic) */
    uint8_t* failed;            /* count flags */
    orc_stats stats[64];
    int want_stats;
} batch_job;

typedef struct worker_arg { batch_job* job; int id; } worker_arg;

static void* batch_worker(void* arg) {
    worker_arg* w = (worker_arg*)arg;
    batch_job* j = w->job;
    for (;;) {
        const uint32_t at = __atomic_fetch_add(&j->next, 64u, __ATOMIC_RELAXED);
        if (at >= j->count) break;
        const uint32_t end = at + 64 < j->count ? at + 64 : j->count;
        for (uint32_t i = at; i < end; ++i)
            j->failed[i] = (uint8_t)orc_trial(j->p, j->rk, j->first + i, NULL,
                                              j->want_stats ? &j->stats[w->id] : NULL);
    }
    return NULL;
}

uint32_t orc_batch(const orc_params* p, uint64_t seed, uint64_t batch_id, uint32_t first,
                   uint32_t count, int threads, uint32_t* out_offsets, orc_stats* stats) {
    batch_job job;
    memset(&job, 0, sizeof job);
    job.p = p;
    orc_batch_key(seed, batch_id, job.rk);
    job.first = first;
    job.count = count;
    job.failed = (uint8_t*)calloc(count ? count : 1, 1);
    job.want_stats = stats != NULL;
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    pthread_t tids[64];
    worker_arg args[64];
    for (int t = 0; t < threads; ++t) {
        args[t].job = &job;
        args[t].id = t;
        if (t) pthread_create(&tids[t], NULL, batch_worker, &args[t]);
    }
    batch_worker(&args[0]);
    for (int t = 1; t < threads; ++t) pthread_join(tids[t], NULL);
    uint32_t n = 0;
    for (uint32_t i = 0; i < count; ++i)
        if (job.failed[i]) out_offsets[n++] = first + i;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        for (int t = 0; t < threads; ++t) {
            stats->probes += job.stats[t].probes;
            stats->evaluations += job.stats[t].evaluations;
            stats->distinct += job.stats[t].distinct;
            stats->aes_blocks += job.stats[t].aes_blocks;
        }
    }
    free(job.failed);
    return n;
}
