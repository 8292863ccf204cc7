// ref_harness.cpp -- C entry points over the reference's OWN CPU implementation.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the reference
// sources where they lie (-I <reference dir>); the compiled library goes to
// oracle/_ref/ and is never committed.  It pins the restatement in
// cmc_oracle.c and serves as the timed CPU baseline ("kind": "reference").
//
// The reference's cpu_trial / cpu_trial_cached / cpu_batch_launch
// (cpu_trials.hpp:69-198) take a Params struct (cuckoo_bench.cu:499); the
// benchmark shapes override its buckets and kick fields, and the derived
// fields are recomputed with the reference formula (cuckoo_bench.cu:513-525).
#define CUCKOO_HOST_TEST
#include "cuckoo_bench.cu"
#include "cpu_trials.hpp"

#include <thread>

namespace {

Options make_options(const char* mode, const char* input_mode, uint32_t pnum, uint32_t ell_i,
                     int workers) {
    Options o;
    o.mode = mode;
    o.input_mode = input_mode;
    o.pnum = pnum;
    o.ell_i = ell_i;
    o.workers = workers < 1 ? 1 : workers;
    o.out = "/nonexistent-cmc-ref-harness";  // pause_requested() probes <out>/PAUSE
    o.backend = "cpu-aesni";
    return o;
}

Params make_params(const Options& o, uint32_t buckets_override, uint32_t kick_override) {
    Params p = parameters(o);
    if (kick_override) p.kick = kick_override;
    if (buckets_override) {
        p.buckets = buckets_override;
        const uint64_t source = (uint64_t(1) << o.ell_i) * 3;
        p.bucket_size = source / p.buckets + (source % p.buckets != 0);
        p.ell_d = (uint32_t)std::ceil(original_log2_u64(p.bucket_size));
        p.domain = p.buckets * p.bucket_size;
        uint32_t bits = std::max<uint32_t>(bit_width_u64(p.domain - 1), 2u);
        if (bits & 1u) ++bits;
        p.half_bits = bits / 2;
        p.mask = (1ULL << p.half_bits) - 1ULL;
    }
    return p;
}

}  // namespace

extern "C" {

int ref_has_aesni() { return cpu_has_aesni() ? 1 : 0; }

int ref_self_test() {
    try {
        cpu_aes_self_test();
        return 0;
    } catch (...) {
        return -1;
    }
}

void ref_batch_key(uint64_t seed, uint64_t id, uint32_t out[44]) {
    const AesKey k = batch_key(seed, id);
    std::memcpy(out, k.w, sizeof(k.w));
}

void ref_host_aes(const uint32_t rk[44], const uint32_t in[4], uint32_t out[4]) {
    AesKey k;
    std::memcpy(k.w, rk, sizeof(k.w));
    host_aes128(k, in[0], in[1], in[2], in[3], out);
}

// out: buckets, kick, bucket_size, domain, mask, half_bits
int ref_params(const char* mode, uint32_t pnum, uint32_t ell_i, uint32_t buckets_override,
               uint32_t kick_override, uint64_t out[6]) {
    const Options o = make_options(mode, "sequential", pnum, ell_i, 1);
    const Params p = make_params(o, buckets_override, kick_override);
    out[0] = p.buckets; out[1] = p.kick; out[2] = p.bucket_size;
    out[3] = p.domain; out[4] = p.mask; out[5] = p.half_bits;
    return 0;
}

// Trials [first, first+count) of batch `batch`, reference cpu_trial (cached=0)
// or cpu_trial_cached (cached=1), on `workers` threads.  Returns the number of
// failures; out receives the sorted failing offsets.
uint32_t ref_batch(const char* mode, const char* input_mode, uint32_t pnum, uint32_t ell_i,
                   uint32_t buckets_override, uint32_t kick_override, uint64_t seed,
                   uint64_t batch, uint32_t first, uint32_t count, int workers, int cached,
                   uint32_t* out) {
    const Options o = make_options(mode, input_mode, pnum, ell_i, workers);
    const Params p = make_params(o, buckets_override, kick_override);
    const CpuAes aes(batch_key(seed, batch));
    std::vector<uint8_t> failed(count, 0);
    std::atomic<uint32_t> next{0};
    auto body = [&]() {
        std::vector<uint32_t> bins(p.buckets);
        std::vector<uint16_t> rounds(cached ? (size_t{8} << p.half_bits) : 0);
        for (;;) {
            const uint32_t at = next.fetch_add(16);
            if (at >= count) break;
            const uint32_t end = std::min(count, at + 16);
            for (uint32_t i = at; i < end; ++i)
                failed[i] = cached ? cpu_trial_cached(o, p, aes, first + i, bins, rounds)
                                   : cpu_trial(o, p, aes, first + i, bins);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < o.workers; ++w) pool.emplace_back(body);
    body();
    for (auto& t : pool) t.join();
    uint32_t n = 0;
    for (uint32_t i = 0; i < count; ++i)
        if (failed[i]) out[n++] = first + i;
    return n;
}

// The reference's own batch launcher (cpu_trials.hpp:161-198): trials
// [0, count) of the batch keyed by batch_key(seed, batch), helper threads
// claiming 256-trial grains.  This is the timed CPU baseline.
uint32_t ref_batch_launch(const char* mode, const char* input_mode, uint32_t pnum,
                          uint32_t ell_i, uint32_t buckets_override, uint32_t kick_override,
                          uint64_t seed, uint64_t batch, uint32_t count, int workers,
                          uint32_t* out, int* used_cache) {
    Options o = make_options(mode, input_mode, pnum, ell_i, workers);
    o.micro = 256;
    const Params p = make_params(o, buckets_override, kick_override);
    if (used_cache) *used_cache = round_cache_enabled(o, p) ? 1 : 0;
    Counters s;
    std::vector<uint32_t> failures;
    cpu_batch_launch(o, p, batch_key(seed, batch), count, s, failures);
    std::sort(failures.begin(), failures.end());
    std::copy(failures.begin(), failures.end(), out);
    return (uint32_t)failures.size();
}

}  // extern "C"
