// cmc_hostcore.cpp -- host-side pieces of the path that run once per batch or
// once per experiment: AES-128 on the host, batch keys, parameter derivation.
#include <cmath>
#include <cstring>
#include <limits>

#include "cmc.h"
#include "cmc_hostcore.hpp"

namespace cmc {

namespace {

uint8_t xtime(uint8_t x) { return static_cast<uint8_t>((x << 1) ^ ((x & 0x80) ? 0x1b : 0)); }

uint8_t gmul(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    for (; b; b >>= 1, a = xtime(a))
        if (b & 1) r ^= a;
    return r;
}

struct SboxTable {
    uint8_t s[256];
    SboxTable() {
        // S(x) = A(x^-1) ^ 0x63 over GF(2^8) / (x^8 + x^4 + x^3 + x + 1).
        for (int x = 0; x < 256; ++x) {
            uint8_t inv = 0;
            for (int y = 1; x && y < 256; ++y)
                if (gmul(static_cast<uint8_t>(x), static_cast<uint8_t>(y)) == 1) {
                    inv = static_cast<uint8_t>(y);
                    break;
                }
            uint8_t v = 0x63;
            for (int r = 0; r < 5; ++r)
                v ^= static_cast<uint8_t>((inv << r) | (inv >> ((8 - r) & 7)));
            s[x] = v;
        }
    }
};

const SboxTable& sbox_table() {
    static const SboxTable t;
    return t;
}

}  // namespace

const uint8_t* sbox() { return sbox_table().s; }

void t0_table(uint32_t out[256]) {
    const uint8_t* S = sbox();
    for (int x = 0; x < 256; ++x) {
        const uint32_t s = S[x], s2 = xtime(static_cast<uint8_t>(s)), s3 = s2 ^ s;
        out[x] = (s2 << 24) | (s << 16) | (s << 8) | s3;
    }
}

void expand_words(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t rk[44]) {
    const uint8_t* S = sbox();
    rk[0] = a; rk[1] = b; rk[2] = c; rk[3] = d;
    uint8_t rcon = 1;
    for (int i = 4; i < 44; ++i) {
        uint32_t v = rk[i - 1];
        if ((i & 3) == 0) {
            v = (v << 8) | (v >> 24);
            v = (uint32_t(S[v >> 24]) << 24) | (uint32_t(S[(v >> 16) & 255]) << 16) |
                (uint32_t(S[(v >> 8) & 255]) << 8) | S[v & 255];
            v ^= uint32_t(rcon) << 24;
            rcon = xtime(rcon);
        }
        rk[i] = rk[i - 4] ^ v;
    }
}

void expand_u64(uint64_t lo, uint64_t hi, uint32_t rk[44]) {
    // Key bytes: lo little-endian, then hi little-endian; words big-endian
    // over consecutive bytes (cuckoo_bench.cu:86-91).
    auto word = [](uint64_t x, int half) {
        uint32_t w = 0;
        for (int q = 0; q < 4; ++q) w = (w << 8) | uint32_t((x >> (8 * (4 * half + q))) & 255);
        return w;
    };
    expand_words(word(lo, 0), word(lo, 1), word(hi, 0), word(hi, 1), rk);
}

void host_aes128(const uint32_t rk[44], const uint32_t in[4], uint32_t out[4]) {
    const uint8_t* S = sbox();
    uint8_t st[16];
    for (int j = 0; j < 4; ++j)
        for (int q = 0; q < 4; ++q)
            st[4 * j + q] = static_cast<uint8_t>((in[j] ^ rk[j]) >> (24 - 8 * q));
    for (int round = 1; round <= 10; ++round) {
        uint8_t sh[16];
        // SubBytes + ShiftRows: row q of column j comes from column j+q.
        for (int j = 0; j < 4; ++j)
            for (int q = 0; q < 4; ++q) sh[4 * j + q] = S[st[4 * ((j + q) & 3) + q]];
        for (int j = 0; j < 4; ++j) {
            uint8_t* c = sh + 4 * j;
            if (round != 10) {
                const uint8_t a0 = c[0], a1 = c[1], a2 = c[2], a3 = c[3];
                c[0] = static_cast<uint8_t>(xtime(a0) ^ xtime(a1) ^ a1 ^ a2 ^ a3);
                c[1] = static_cast<uint8_t>(a0 ^ xtime(a1) ^ xtime(a2) ^ a2 ^ a3);
                c[2] = static_cast<uint8_t>(a0 ^ a1 ^ xtime(a2) ^ xtime(a3) ^ a3);
                c[3] = static_cast<uint8_t>(xtime(a0) ^ a0 ^ a1 ^ a2 ^ xtime(a3));
            }
            for (int q = 0; q < 4; ++q) c[q] ^= static_cast<uint8_t>(rk[4 * round + j] >> (24 - 8 * q));
        }
        std::memcpy(st, sh, 16);
    }
    for (int j = 0; j < 4; ++j)
        out[j] = (uint32_t(st[4 * j]) << 24) | (uint32_t(st[4 * j + 1]) << 16) |
                 (uint32_t(st[4 * j + 2]) << 8) | st[4 * j + 3];
}

void batch_key(uint64_t seed, uint64_t batch_id, uint32_t rk[44]) {
    uint32_t master[44];
    expand_u64(seed, seed ^ 0x9e3779b97f4a7c15ULL, master);
    const uint32_t in[4] = {0x42415443u, uint32_t(batch_id >> 32), uint32_t(batch_id), 0x50524731u};
    uint32_t x[4];
    host_aes128(master, in, x);
    const uint64_t lo = (uint64_t(x[0]) << 32) | x[1];
    const uint64_t hi = (uint64_t(x[2]) << 32) | x[3];
    expand_u64(seed ^ lo, hi ^ (seed ^ 0x243f6a8885a308d3ULL), rk);
}

unsigned bit_width(uint64_t v) {
    unsigned n = 0;
    for (; v; v >>= 1) ++n;
    return n;
}

float reference_log2(uint64_t n) {
    // The DRRT18 bucket count is defined through this float-valued atanh
    // series (cuckoo_bench.cu:488-498); evaluating the same operations in the
    // same order is what makes B identical.
    if (n == 0) return -std::numeric_limits<float>::infinity();
    const unsigned e = bit_width(n) - 1;
    const double x = double(n) / double(1ULL << e);
    if (x >= 2.0) return float(e + 1);
    const double z = (x - 1.0) / (x + 1.0), z2 = z * z;
    double term = z, sum = 0.0;
    for (int i = 1; i <= 23; i += 2) {
        sum += term / i;
        term *= z2;
    }
    return float(double(e) + 2.0 * sum * 1.4426950408889634074);
}

int derive_params(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                  uint32_t buckets_override, uint32_t kick_override, uint32_t input_mode,
                  cmc_params* out, const char** why) {
    auto fail = [&](const char* m) {
        if (why) *why = m;
        return CMC_EINVAL;
    };
    if (!out) return fail("null output");
    std::memset(out, 0, sizeof *out);
    if (mode != CMC_MODE_BGH25 && mode != CMC_MODE_DRRT18) return fail("mode must be bgh25 or drrt18");
    if (input_mode > 1) return fail("input mode must be sequential or affine");
    if (pnum < 3 || pnum > 65534) return fail("PNUM must be in 3..65534");
    if (ell_i > 61) return fail("ell-i must be <= 61");
    if (ell_i < 16 && (1ULL << ell_i) < pnum) return fail("2^ell-i must be >= PNUM");
    if (k < 2 || k > 4) return fail("k must be 2, 3 or 4");
    out->mode = mode;
    out->input_mode = input_mode;
    out->pnum = pnum;
    out->ell_i = ell_i;
    out->k = k;
    if (mode == CMC_MODE_BGH25) {
        const uint64_t overhead = pnum < 30 ? 100 : 50;
        out->buckets = uint32_t(uint64_t(pnum) * (100 + overhead) / 100);
        out->kick = 3 * pnum;
    } else {
        const float lf = reference_log2(pnum);
        const float f = float(double(pnum) * (double(170.0f + lf) / 123.5));
        out->buckets = uint32_t(std::ceil(double(f)));
        out->kick = 100;
    }
    if (buckets_override) out->buckets = buckets_override;
    if (kick_override) out->kick = kick_override;
    if (out->buckets < 1) return fail("buckets must be positive");
    const uint64_t source = (uint64_t(1) << ell_i) * k;  // ell_i <= 61, k <= 4: no overflow for k<=3
    if (ell_i == 61 && k == 4) return fail("k * 2^ell-i overflows 64 bits");
    out->bucket_size = source / out->buckets + (source % out->buckets != 0);
    if (out->buckets > std::numeric_limits<uint64_t>::max() / out->bucket_size)
        return fail("PRP domain overflow");
    out->domain = out->buckets * out->bucket_size;
    uint32_t bits = bit_width(out->domain - 1);
    if (bits < 2) bits = 2;
    if (bits & 1u) ++bits;
    out->half_bits = bits / 2;
    out->mask = (uint64_t(1) << out->half_bits) - 1;
    out->range_mask = (uint64_t(1) << ell_i) - 1;
    return CMC_OK;
}

}  // namespace cmc

extern "C" {

int cmc_derive_params(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                      uint32_t buckets_override, uint32_t kick_override, uint32_t input_mode,
                      cmc_params* out) {
    return cmc::derive_params(mode, pnum, ell_i, k, buckets_override, kick_override, input_mode,
                              out, nullptr);
}

void cmc_batch_key(uint64_t seed, uint64_t batch_id, uint32_t out_w[44]) {
    cmc::batch_key(seed, batch_id, out_w);
}

void cmc_host_aes128(const uint32_t rk[44], const uint32_t in[4], uint32_t out[4]) {
    cmc::host_aes128(rk, in, out);
}

}  // extern "C"
