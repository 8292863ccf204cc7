// cmc_aes.cuh -- AES-128 for the Feistel PRP, shared-memory T-table form for sm_100a.
//
// Table layout (64 KiB per CTA, built once per launch from a 1 KiB table):
//   256 rows of 256 bytes, row x = [T0[x] x 32 copies][T2[x] x 32 copies]
// where T0[x] is the MixColumns column (2s, s, s, 3s) of s = S[x] (most
// significant byte first) and T2 = ror16(T0).  Lane L reads copy L, which
// sits in bank L, so a warp-wide lookup with 32 arbitrary indices is one
// shared-memory wavefront.  The byte offset of lane L's T0[x] is
// (x << 8) | (L << 2) and of T2[x] is that plus 128: one PRMT builds it
// directly from the state word, with no shift/mask/add.
//
// One AES round column with T1 = ror8(T0) and T3 = ror8(T2):
//   t = T0[a] ^ T2[c] ^ ror8(T0[b] ^ T2[d] ^ rol8(k))
// so the round key is stored pre-rotated (rol8) and each column costs
// 4 PRMT + 4 LDS + 2 LOP3 + 1 rotate (a fifth PRMT).
//
// The PRP round function of the reference (cuckoo_bench.cu:161-184) is
//   F_r(R) = AES_k(0x43455350, r, h, R).w3 & (2^h - 1)
// and only its low h <= 16 bits are used, which permits three exact cuts:
//   round 1:  only the two low bytes of w3 = R ^ rk3 vary with R, so 14 of
//             16 lookups fold into four per-(trial, r) constants;
//   round 9:  only columns 1 and 2 feed the two output bytes that are kept;
//   round 10: only those two S-box bytes are computed.
// That is 2 + 7*16 + 8 + 2 = 124 lookups per block instead of 160.
#pragma once
#include <cstdint>

namespace cmc {

constexpr uint32_t kTableBytes = 65536;

// Measured on B200: the byte-permute form is about 10% faster than the
// FMA-pipe form below, so it is the default.
#ifndef CMC_FMA_OFFSETS
#define CMC_FMA_OFFSETS 0
#endif

// Rotations by one byte as byte permutes, and the column's two three-way XORs
// as explicit three-input logic operations (0x96 = a ^ b ^ c): measured on
// B200 at t = 1024, B = 1536, N = 2^20: 3.071 M trials/s against 3.034 M
// with funnel shifts and plain XORs.
__device__ __forceinline__ uint32_t ror8(uint32_t x) { return __byte_perm(x, x, 0x0321); }
__device__ __forceinline__ uint32_t rol8(uint32_t x) { return __byte_perm(x, x, 0x2103); }

__device__ __forceinline__ uint32_t xor3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// Byte offset of this lane's T0 (lb = lane*4) or T2 (lb = lane*4 + 128) entry
// for byte `B` of word w.
template <int B>
__device__ __forceinline__ uint32_t toff(uint32_t w, uint32_t lb) {
    return __byte_perm(w, lb, 0x5504 | (B << 4));
}

// The table sits at offset 0 of dynamic shared memory.
extern __shared__ __align__(1024) char cmc_dyn_smem[];

// Shared-window address at which dynamic shared memory starts in a kernel
// with no static shared variables: after the 1 KiB the hardware reserves per
// block on sm_90 and later (cudaDevAttrReservedSharedMemoryPerBlock).
#define CMC_DYN_SMEM_BASE 1024
#define CMC_STR_(x) #x
#define CMC_STR(x) CMC_STR_(x)
constexpr uint32_t kDynSmemBase = CMC_DYN_SMEM_BASE;

// Every kernel that calls lds() checks this once (cmc_selftest at context
// creation, the engine kernels at entry) and reports an error instead of
// reading the table at a wrong address.
__device__ __forceinline__ bool table_base_ok() {
    return (uint32_t)__cvta_generic_to_shared(cmc_dyn_smem) == kDynSmemBase;
}

// One table lookup: a shared load at [off + base] with the base as the
// instruction's immediate.  Written as a C++ load from cmc_dyn_smem + off, the
// compiler kept the base in a register in the engine kernels and spent one
// more (FMA-pipe) instruction per lookup on the add (measured on B200 at
// t = 1024, B = 1536, N = 2^20: 517 against 404 instructions per 32 blocks,
// 140 against 27 on the FMA pipe; 3.07 M against 3.35 M trials/s).  volatile keeps every lookup
// after the barrier that publishes the table.
__device__ __forceinline__ uint32_t lds(uint32_t off) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1+" CMC_STR(CMC_DYN_SMEM_BASE) "];" : "=r"(v) : "r"(off));
    return v;
}

struct Lanes {
    uint32_t lb0;  // lane*4
    uint32_t lb2;  // lane*4 + 128
    // 256 held in a register (from a kernel argument).  With CMC_FMA_OFFSETS
    // the offset of a top-byte lookup, (w >> 24) * 256 + lb0, is two
    // multiply-adds on the FMA pipe instead of one byte permute on the ALU
    // pipe, which the table lookups otherwise saturate.
    uint32_t r256;
};

__device__ __forceinline__ uint32_t top_byte_off(const Lanes& L, uint32_t w) {
#if CMC_FMA_OFFSETS
    return __umulhi(w, L.r256) * L.r256 + L.lb0;
#else
    return toff<3>(w, L.lb0);
#endif
}

// Column j of a full round: inputs s_j (byte 3), s_{j+1} (byte 2),
// s_{j+2} (byte 1), s_{j+3} (byte 0); kr = rol8(round key word).
__device__ __forceinline__ uint32_t column(const Lanes& L, uint32_t sa, uint32_t sb,
                                          uint32_t sc, uint32_t sd, uint32_t kr) {
    const uint32_t a = lds(top_byte_off(L, sa));
    const uint32_t b = lds(toff<2>(sb, L.lb0));
    const uint32_t c = lds(toff<1>(sc, L.lb2));
    const uint32_t d = lds(toff<0>(sd, L.lb2));
    return xor3(a, c, ror8(xor3(b, d, kr)));
}

__device__ __forceinline__ uint32_t sbox_byte(const Lanes& L, uint32_t x) {
    // S[x] is byte 1 of T0[x].
    return (lds(((x & 255u) << 8) | L.lb0) >> 8) & 255u;
}

__device__ __forceinline__ uint32_t sub_word(const Lanes& L, uint32_t v) {
    return (sbox_byte(L, v >> 24) << 24) | (sbox_byte(L, v >> 16) << 16) |
           (sbox_byte(L, v >> 8) << 8) | sbox_byte(L, v);
}

// FIPS-197 key schedule from four big-endian key words (cuckoo_bench.cu:136-149).
__device__ __forceinline__ void expand_key(const Lanes& L, uint32_t a, uint32_t b, uint32_t c,
                                           uint32_t d, uint32_t* rk) {
    rk[0] = a; rk[1] = b; rk[2] = c; rk[3] = d;
    uint32_t rcon = 1;
#pragma unroll 1
    for (int i = 4; i < 44; i += 4) {
        const uint32_t v = rk[i - 1];
        const uint32_t t = sub_word(L, (v << 8) | (v >> 24)) ^ (rcon << 24);
        rcon = (rcon << 1) ^ ((rcon & 0x80u) ? 0x1bu : 0u);
        rk[i] = rk[i - 4] ^ t;
        rk[i + 1] = rk[i - 3] ^ rk[i];
        rk[i + 2] = rk[i - 2] ^ rk[i + 1];
        rk[i + 3] = rk[i - 1] ^ rk[i + 2];
    }
}

// Full AES-128 block with all four output words; round keys read from a
// plain (non-rotated) 44-word schedule in any memory space.  Used for the
// per-trial seed blocks and the known-answer test, not for the PRP.
__device__ __forceinline__ void encrypt_full(const Lanes& L, const uint32_t* rk, uint32_t p0,
                                             uint32_t p1, uint32_t p2, uint32_t p3,
                                             uint32_t out[4]) {
    uint32_t s0 = p0 ^ rk[0], s1 = p1 ^ rk[1], s2 = p2 ^ rk[2], s3 = p3 ^ rk[3];
#pragma unroll 1
    for (int r = 1; r < 10; ++r) {
        const uint32_t t0 = column(L, s0, s1, s2, s3, rol8(rk[4 * r + 0]));
        const uint32_t t1 = column(L, s1, s2, s3, s0, rol8(rk[4 * r + 1]));
        const uint32_t t2 = column(L, s2, s3, s0, s1, rol8(rk[4 * r + 2]));
        const uint32_t t3 = column(L, s3, s0, s1, s2, rol8(rk[4 * r + 3]));
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
    const uint32_t st[4] = {s0, s1, s2, s3};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        out[j] = ((sbox_byte(L, st[j] >> 24) << 24) |
                  (sbox_byte(L, st[(j + 1) & 3] >> 16) << 16) |
                  (sbox_byte(L, st[(j + 2) & 3] >> 8) << 8) | sbox_byte(L, st[(j + 3) & 3])) ^
                 rk[40 + j];
    }
}

// Per-trial PRP key in the form the fast round function consumes.
struct PrpKey {
    uint32_t kr[32];  // rol8(rk[8..39])  (rounds 2..9; round 9 uses kr[29], kr[30])
    uint32_t k43lo;   // rk[43] & 0xffff
};

// Per-(trial, round r) constants of the first AES round (h <= 16).
struct Round1 {
    uint32_t c0, c1, c2, c3;  // see prp_f below
    uint32_t w3hi;            // rk[3] (only its two low bytes combine with R)
};

// Round-1 constants for Feistel round r (plaintext 0x43455350, r, h, R).
__device__ __forceinline__ Round1 round1_consts(const Lanes& L, const uint32_t* rk, uint32_t r,
                                                uint32_t h) {
    const uint32_t s0 = 0x43455350u ^ rk[0], s1 = r ^ rk[1], s2 = h ^ rk[2], s3 = rk[3];
    auto t0v = [&](uint32_t x, int byte) { return lds(((((x >> (8 * byte)) & 255u)) << 8) | L.lb0); };
    auto t2v = [&](uint32_t x, int byte) { return lds(((((x >> (8 * byte)) & 255u)) << 8) | L.lb2); };
    // Te0[a] ^ Te1[b] ^ Te2[c] ^ Te3[d] with Te1 = ror8(T0), Te3 = ror8(T2)
    Round1 c;
    c.c0 = t0v(s0, 3) ^ ror8(t0v(s1, 2)) ^ t2v(s2, 1) ^ rk[4];           // + Te3[s3 b0]
    c.c1 = t0v(s1, 3) ^ ror8(t0v(s2, 2)) ^ ror8(t2v(s0, 0)) ^ rk[5];     // + Te2[s3 b1]
    c.c2 = t0v(s2, 3) ^ ror8(t0v(s3, 2)) ^ t2v(s0, 1) ^ ror8(t2v(s1, 0)) ^ rk[6];
    c.c3 = t0v(s3, 3) ^ ror8(t0v(s0, 2)) ^ t2v(s1, 1) ^ ror8(t2v(s2, 0)) ^ rk[7];
    c.w3hi = rk[3];
    return c;
}

__device__ __forceinline__ void prp_key_from_schedule(const uint32_t* rk, PrpKey& k) {
#pragma unroll
    for (int i = 0; i < 32; ++i) k.kr[i] = rol8(rk[8 + i]);
    k.k43lo = rk[43] & 0xffffu;
}

// State after AES round 2 of AES_k(0x43455350, r, h, R) for R < 2^16.
__device__ __forceinline__ void round2_state(const Lanes& L, const PrpKey& k, const Round1& c,
                                             uint32_t R, uint32_t t[4]) {
    const uint32_t w3 = R ^ c.w3hi;
    // round 1: t0 = c0 ^ Te3[w3 b0], t1 = c1 ^ Te2[w3 b1], t2 = c2, t3 = c3
    const uint32_t s0 = c.c0 ^ ror8(lds(toff<0>(w3, L.lb2)));
    const uint32_t s1 = c.c1 ^ lds(toff<1>(w3, L.lb2));
    const uint32_t s2 = c.c2, s3 = c.c3;
    t[0] = column(L, s0, s1, s2, s3, k.kr[0]);
    t[1] = column(L, s1, s2, s3, s0, k.kr[1]);
    t[2] = column(L, s2, s3, s0, s1, k.kr[2]);
    t[3] = column(L, s3, s0, s1, s2, k.kr[3]);
}

// Rounds 3..10 from the state after round 2; low 16 bits of w3.
__device__ __forceinline__ uint32_t prp_tail(const Lanes& L, const PrpKey& k, uint32_t s0,
                                             uint32_t s1, uint32_t s2, uint32_t s3) {
    // rounds 3..8
#pragma unroll
    for (int r = 1; r < 7; ++r) {
        const uint32_t t0 = column(L, s0, s1, s2, s3, k.kr[4 * r + 0]);
        const uint32_t t1 = column(L, s1, s2, s3, s0, k.kr[4 * r + 1]);
        const uint32_t t2 = column(L, s2, s3, s0, s1, k.kr[4 * r + 2]);
        const uint32_t t3 = column(L, s3, s0, s1, s2, k.kr[4 * r + 3]);
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
    // round 9: columns 1 and 2 only
    const uint32_t u1 = column(L, s1, s2, s3, s0, k.kr[29]);
    const uint32_t u2 = column(L, s2, s3, s0, s1, k.kr[30]);
    // round 10: w3 bits 8..15 = S[u1 b1], bits 0..7 = S[u2 b0]
    const uint32_t hi = lds(toff<1>(u1, L.lb0));  // T0: S at bits 8..15
    const uint32_t lo = lds(toff<0>(u2, L.lb2));  // T2: S at bits 0..7
    return ((hi & 0xff00u) | (lo & 0x00ffu)) ^ k.k43lo;
}

// Low 16 bits of AES_k(0x43455350, r, h, R).w3 for R < 2^16.
__device__ __forceinline__ uint32_t prp_f(const Lanes& L, const PrpKey& k, const Round1& c,
                                          uint32_t R) {
    uint32_t t[4];
    round2_state(L, k, c, R, t);
    return prp_tail(L, k, t[0], t[1], t[2], t[3]);
}

// Round-2 fold.  For one trial key and Feistel round r, byte 0 of w3 = R ^ rk3
// enters round 1 only through state word 0 and byte 1 only through word 1
// (round2_state above), and round 2 is linear in its input columns' table
// outputs.  So the state after round 2 is U(w3 b0) ^ V(w3 b1) with
//   U(a) = (Te0[s0 b3], Te3[s0 b0], Te2[s0 b1], Te1[s0 b2]),  s0 = c0 ^ Te3[a]
// (the round-2 lookups that read word 0) and V holding the rest, round keys
// included.  V depends on R only through R >> 8 (R < 2^16): a table of
// 2^max(0, h-8) entries per round, built once per trial by fold_entry; the
// round cache fill then spends 5 lookups on rounds 1 and 2 instead of 18.
__device__ __forceinline__ void round2_u(const Lanes& L, uint32_t c0, uint32_t w3, uint32_t u[4]) {
    const uint32_t s0 = c0 ^ ror8(lds(toff<0>(w3, L.lb2)));
    u[0] = lds(top_byte_off(L, s0));
    u[1] = ror8(lds(toff<0>(s0, L.lb2)));
    u[2] = lds(toff<1>(s0, L.lb2));
    u[3] = ror8(lds(toff<2>(s0, L.lb0)));
}

// V entry for the R values with R >> 8 == y: the state after round 2 of
// R = y << 8 | (rk3 & 255) (so that w3 b0 = 0) with U(0) removed.
__device__ __forceinline__ uint4 fold_entry(const Lanes& L, const PrpKey& k, const Round1& c,
                                            uint32_t y) {
    uint32_t t[4], u[4];
    round2_state(L, k, c, (y << 8) | (c.w3hi & 255u), t);
    round2_u(L, c.c0, 0u, u);
    return make_uint4(t[0] ^ u[0], t[1] ^ u[1], t[2] ^ u[2], t[3] ^ u[3]);
}

// prp_f through the fold: v = the V entry of R >> 8 for this round.
__device__ __forceinline__ uint32_t prp_f_folded(const Lanes& L, const PrpKey& k, uint32_t c0,
                                                 uint32_t w3hi, const uint4& v, uint32_t R) {
    uint32_t u[4];
    round2_u(L, c0, R ^ w3hi, u);
    return prp_tail(L, k, u[0] ^ v.x, u[1] ^ v.y, u[2] ^ v.z, u[3] ^ v.w);
}

// Full 32-bit w3 of AES_k(0x43455350, r, h, R) for any 32-bit R (h > 16),
// from the plain schedule.  Slow path for PRP domains above 2^32.
__device__ __forceinline__ uint32_t prp_f_wide(const Lanes& L, const uint32_t* rk, uint32_t r,
                                               uint32_t h, uint32_t R) {
    uint32_t out[4];
    encrypt_full(L, rk, 0x43455350u, r, h, R, out);
    return out[3];
}

}  // namespace cmc
