// aes_bitslice.cuh -- a bitsliced AES-128, used only by aes_forms_bench.cu to
// measure the bitsliced form of the round function against the T-table form
// of cmc_aes.cuh on B200.  Not on the product path.
//
// Layout: W is a 32-bit word holding one bit of 32 independent blocks (slice
// j = block j).  A state is 128 words, s[8*n + i] = bit i (coefficient of x^i)
// of state byte n, n = row + 4*column as in FIPS-197 (input byte n goes to
// byte n).  All 32 blocks share one key, so a round-key bit is a whole word of
// zeros or ones.
//
// SubBytes is computed from its definition (FIPS-197 5.1.1): the inverse in
// GF(2^8) modulo x^8 + x^4 + x^3 + x + 1 as x^254 (4 multiplications, 7
// squarings), then the affine map.  That is ~700 gates per S-box, about six
// times the smallest published circuits (113 gates); the benchmark reports the
// measured instructions per gate so the smaller circuits can be costed too.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CMC_HD __host__ __device__ __forceinline__
#else
#define CMC_HD inline
#endif

namespace cmc {
namespace bitslice {

struct Byte8 {
    uint32_t b[8];
};

// Reduce a 15-coefficient product modulo x^8 + x^4 + x^3 + x + 1:
// x^k = x^(k-4) + x^(k-5) + x^(k-7) + x^(k-8) for k >= 8, highest first.
CMC_HD Byte8 reduce(uint32_t p[15]) {
#pragma unroll
    for (int k = 14; k >= 8; --k) {
        p[k - 4] ^= p[k];
        p[k - 5] ^= p[k];
        p[k - 7] ^= p[k];
        p[k - 8] ^= p[k];
    }
    Byte8 r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.b[i] = p[i];
    return r;
}

CMC_HD Byte8 gf_mul(const Byte8& a, const Byte8& b) {
    uint32_t p[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) p[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) p[i + j] ^= a.b[i] & b.b[j];
    return reduce(p);
}

// Squaring is linear: coefficient i moves to 2i.
CMC_HD Byte8 gf_sq(const Byte8& a) {
    uint32_t p[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) p[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) p[2 * i] = a.b[i];
    return reduce(p);
}

// x^254 = x^-1 (and 0 -> 0): 254 = 240 + 14, 240 = 15 * 16, 14 = 12 + 2.
CMC_HD Byte8 gf_inv(const Byte8& x) {
    const Byte8 x2 = gf_sq(x);
    const Byte8 x3 = gf_mul(x2, x);
    const Byte8 x12 = gf_sq(gf_sq(x3));
    const Byte8 x15 = gf_mul(x12, x3);
    const Byte8 x240 = gf_sq(gf_sq(gf_sq(gf_sq(x15))));
    const Byte8 x14 = gf_mul(x12, x2);
    return gf_mul(x240, x14);
}

// S(x) = A * x^-1 + 0x63: bit i of the result is
// b_i ^ b_(i+4) ^ b_(i+5) ^ b_(i+6) ^ b_(i+7) ^ c_i (indices mod 8).
CMC_HD Byte8 sbox(const Byte8& x) {
    const Byte8 v = gf_inv(x);
    Byte8 r;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t t = v.b[i] ^ v.b[(i + 4) & 7] ^ v.b[(i + 5) & 7] ^ v.b[(i + 6) & 7] ^
                           v.b[(i + 7) & 7];
        r.b[i] = ((0x63u >> i) & 1u) ? ~t : t;
    }
    return r;
}

// Multiplication by x (xtime): shift up, fold bit 7 into bits 0, 1, 3, 4.
CMC_HD Byte8 xtime(const Byte8& a) {
    Byte8 r;
    r.b[0] = a.b[7];
    r.b[1] = a.b[0] ^ a.b[7];
    r.b[2] = a.b[1];
    r.b[3] = a.b[2] ^ a.b[7];
    r.b[4] = a.b[3] ^ a.b[7];
    r.b[5] = a.b[4];
    r.b[6] = a.b[5];
    r.b[7] = a.b[6];
    return r;
}

CMC_HD Byte8 get(const uint32_t* s, int n) {
    Byte8 r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.b[i] = s[8 * n + i];
    return r;
}

CMC_HD void put(uint32_t* s, int n, const Byte8& v) {
#pragma unroll
    for (int i = 0; i < 8; ++i) s[8 * n + i] = v.b[i];
}

CMC_HD Byte8 bxor(const Byte8& a, const Byte8& b) {
    Byte8 r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.b[i] = a.b[i] ^ b.b[i];
    return r;
}

// ShiftRows: byte (row r, column c) takes the byte at (r, c + r mod 4).
CMC_HD void shift_rows(uint32_t* s) {
    uint32_t t[128];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int i = 0; i < 8; ++i) t[8 * (r + 4 * c) + i] = s[8 * (r + 4 * ((c + r) & 3)) + i];
#pragma unroll
    for (int k = 0; k < 128; ++k) s[k] = t[k];
}

// MixColumns with t = a0 ^ a1 ^ a2 ^ a3: b_r = a_r ^ t ^ xtime(a_r ^ a_(r+1)).
CMC_HD void mix_columns(uint32_t* s) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const Byte8 a0 = get(s, 4 * c), a1 = get(s, 4 * c + 1), a2 = get(s, 4 * c + 2),
                    a3 = get(s, 4 * c + 3);
        const Byte8 t = bxor(bxor(a0, a1), bxor(a2, a3));
        put(s, 4 * c + 0, bxor(bxor(a0, t), xtime(bxor(a0, a1))));
        put(s, 4 * c + 1, bxor(bxor(a1, t), xtime(bxor(a1, a2))));
        put(s, 4 * c + 2, bxor(bxor(a2, t), xtime(bxor(a2, a3))));
        put(s, 4 * c + 3, bxor(bxor(a3, t), xtime(bxor(a3, a0))));
    }
}

// Round key r as 128 masks: bit i of byte n of words rk[4r..4r+3] (byte n is
// byte 3 - n%4 of word n/4, most significant first).
inline void key_masks(const uint32_t rk[44], uint32_t masks[11][128]) {
    for (int r = 0; r < 11; ++r)
        for (int n = 0; n < 16; ++n) {
            const uint32_t byte = (rk[4 * r + n / 4] >> (24 - 8 * (n % 4))) & 0xffu;
            for (int i = 0; i < 8; ++i) masks[r][8 * n + i] = ((byte >> i) & 1u) ? 0xffffffffu : 0u;
        }
}

// 32 blocks (as 4 big-endian words each) <-> 128 slice words.
inline void to_slices(const uint32_t blocks[32][4], uint32_t s[128]) {
    for (int k = 0; k < 128; ++k) s[k] = 0;
    for (int j = 0; j < 32; ++j)
        for (int n = 0; n < 16; ++n) {
            const uint32_t byte = (blocks[j][n / 4] >> (24 - 8 * (n % 4))) & 0xffu;
            for (int i = 0; i < 8; ++i) s[8 * n + i] |= ((byte >> i) & 1u) << j;
        }
}

inline void from_slices(const uint32_t s[128], uint32_t blocks[32][4]) {
    for (int j = 0; j < 32; ++j)
        for (int w = 0; w < 4; ++w) blocks[j][w] = 0;
    for (int j = 0; j < 32; ++j)
        for (int n = 0; n < 16; ++n) {
            uint32_t byte = 0;
            for (int i = 0; i < 8; ++i) byte |= ((s[8 * n + i] >> j) & 1u) << i;
            blocks[j][n / 4] |= byte << (24 - 8 * (n % 4));
        }
}

}  // namespace bitslice
}  // namespace cmc
