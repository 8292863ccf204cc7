// aes_forms_bench.cu -- the two forms of the AES-128 round function on B200,
// for the choice between bank-replicated shared-memory T-tables (the engine's
// form, cmc_aes.cuh) and bitslicing (aes_bitslice.cuh).  Design evidence
// only: built by `make aes_forms_bench`, run by hand (and under ncu for the
// instruction counters); the library does not use it.
//
// Both kernels encrypt full AES-128 blocks (10 rounds, FIPS-197) under one key
// shared by all blocks, as the engine's round-cache fill does under one trial
// key, and fold the ciphertexts into a checksum so no work can be dropped.
//   tt_aes: 384 threads per CTA, 3 blocks in flight per thread, 160 table
//           lookups per block from the 64 KiB lane-replicated table.
//   bs_aes: 256 threads per CTA, 32 blocks per thread (one per bit of each of
//           128 state words); ShiftRows is kept implicit (byte positions are
//           re-indexed per round, so four rounds return to the identity) and
//           the S-box is one out-of-line function (code size).
// Before timing, both forms are checked on the device against the FIPS-197
// C.1 vector and the bitsliced circuit against the host AES on 32 random blocks.
//
// Output: blocks per clock per SM for each form at the measured clock, and the
// checks' results.  Run under ncu -k regex:'tt_aes|bs_aes' for the pipes.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "aes_bitslice.cuh"
#include "cmc_aes.cuh"
#include "cmc_hostcore.hpp"

namespace cmc {
namespace {

struct TtKeys {
    uint32_t rk[44];  // plain schedule (rounds 0 and 10)
    uint32_t kr[44];  // rol8 of each word (rounds 1..9, as column() takes them)
};

__constant__ uint32_t c_masks[11][128];

__device__ __forceinline__ void build_table(const uint32_t* t0) {
    uint32_t* tw = reinterpret_cast<uint32_t*>(cmc_dyn_smem);
    for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) {
        const uint32_t v = t0[i >> 6];
        tw[i] = (i & 32) ? __funnelshift_r(v, v, 16) : v;
    }
}

// One full block, T-table form: AddRoundKey, 9 table rounds, final S-box round.
__device__ __forceinline__ void tt_block(const Lanes& L, const TtKeys& k, uint32_t s[4]) {
    uint32_t s0 = s[0] ^ k.rk[0], s1 = s[1] ^ k.rk[1], s2 = s[2] ^ k.rk[2], s3 = s[3] ^ k.rk[3];
#pragma unroll
    for (int r = 1; r < 10; ++r) {
        const uint32_t t0 = column(L, s0, s1, s2, s3, k.kr[4 * r + 0]);
        const uint32_t t1 = column(L, s1, s2, s3, s0, k.kr[4 * r + 1]);
        const uint32_t t2 = column(L, s2, s3, s0, s1, k.kr[4 * r + 2]);
        const uint32_t t3 = column(L, s3, s0, s1, s2, k.kr[4 * r + 3]);
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
    const uint32_t st[4] = {s0, s1, s2, s3};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        // S[x] is byte 1 of T0[x]; gather the four bytes with byte permutes
        const uint32_t a = lds(toff<3>(st[j], L.lb0));
        const uint32_t b = lds(toff<2>(st[(j + 1) & 3], L.lb0));
        const uint32_t c = lds(toff<1>(st[(j + 2) & 3], L.lb0));
        const uint32_t d = lds(toff<0>(st[(j + 3) & 3], L.lb0));
        const uint32_t lo = __byte_perm(d, c, 0x0051), hi = __byte_perm(b, a, 0x0051);
        s[j] = __byte_perm(lo, hi, 0x5410) ^ k.rk[40 + j];
    }
}

template <int NB>
__global__ void __launch_bounds__(384, 1) tt_aes(const __grid_constant__ TtKeys k, const uint32_t* t0,
                                                 uint32_t* out, uint32_t iters) {
    build_table(t0);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const Lanes L{lane * 4, lane * 4 + 128, 256u};
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = table_base_ok() ? 0u : 0xdeadu;
#pragma unroll 1
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t s[NB][4];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            // every word is a different sum (carries reach every byte), so the
            // compiler can prove no two lookups equal: none is shared between
            // blocks or hoisted out of the loop
            const uint32_t base = tid * 0x85ebca6bu + it * 0xc2b2ae35u;
#pragma unroll
            for (int w = 0; w < 4; ++w) s[b][w] = base + uint32_t(4 * b + w + 1) * 0x9e3779b9u;
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) tt_block(L, k, s[b]);
#pragma unroll
        for (int b = 0; b < NB; ++b) acc ^= s[b][0] ^ s[b][1] ^ s[b][2] ^ s[b][3];
    }
    out[tid] = acc;
}

// FIPS-197 C.1 through the T-table form; out[0] = 1 when correct.
__global__ void tt_check(const __grid_constant__ TtKeys k, const uint32_t* t0, uint32_t* out) {
    build_table(t0);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const Lanes L{lane * 4, lane * 4 + 128, 256u};
    uint32_t s[4] = {0x00112233u, 0x44556677u, 0x8899aabbu, 0xccddeeffu};
    tt_block(L, k, s);
    const bool ok = table_base_ok() && s[0] == 0x69c4e0d8u && s[1] == 0x6a7b0430u &&
                    s[2] == 0xd8cdb780u && s[3] == 0x70b4c55au;
    if (threadIdx.x == 0) out[0] = ok ? 1u : 0u;
}

using bitslice::Byte8;

__device__ __noinline__ Byte8 bs_sbox(Byte8 x) { return bitslice::sbox(x); }

// Physical position of logical byte (r, c) after `sh` ShiftRows applied
// implicitly: (r, c + r*sh mod 4).
__host__ __device__ constexpr int phys(int r, int c, int sh) { return r + 4 * ((c + r * sh) & 3); }

// One round with SH = rounds so far mod 4 (ShiftRows of this round included).
template <int SH, bool MIX>
__device__ __forceinline__ void bs_round(uint32_t* s, int round) {
#pragma unroll
    for (int n = 0; n < 16; ++n) bitslice::put(s, n, bs_sbox(bitslice::get(s, n)));
    if (MIX) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const Byte8 a0 = bitslice::get(s, phys(0, c, SH)), a1 = bitslice::get(s, phys(1, c, SH)),
                        a2 = bitslice::get(s, phys(2, c, SH)), a3 = bitslice::get(s, phys(3, c, SH));
            const Byte8 t = bitslice::bxor(bitslice::bxor(a0, a1), bitslice::bxor(a2, a3));
            bitslice::put(s, phys(0, c, SH),
                          bitslice::bxor(bitslice::bxor(a0, t), bitslice::xtime(bitslice::bxor(a0, a1))));
            bitslice::put(s, phys(1, c, SH),
                          bitslice::bxor(bitslice::bxor(a1, t), bitslice::xtime(bitslice::bxor(a1, a2))));
            bitslice::put(s, phys(2, c, SH),
                          bitslice::bxor(bitslice::bxor(a2, t), bitslice::xtime(bitslice::bxor(a2, a3))));
            bitslice::put(s, phys(3, c, SH),
                          bitslice::bxor(bitslice::bxor(a3, t), bitslice::xtime(bitslice::bxor(a3, a0))));
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int i = 0; i < 8; ++i) s[8 * phys(r, c, SH) + i] ^= c_masks[round][8 * (r + 4 * c) + i];
}

// Ten rounds; on return logical byte (r, c) sits at phys(r, c, 2).
__device__ __forceinline__ void bs_block(uint32_t* s) {
#pragma unroll
    for (int k = 0; k < 128; ++k) s[k] ^= c_masks[0][k];
#pragma unroll 1
    for (int q = 0; q < 2; ++q) {
        bs_round<1, true>(s, 4 * q + 1);
        bs_round<2, true>(s, 4 * q + 2);
        bs_round<3, true>(s, 4 * q + 3);
        bs_round<0, true>(s, 4 * q + 4);
    }
    bs_round<1, true>(s, 9);
    bs_round<2, false>(s, 10);
}

__global__ void __launch_bounds__(256, 1) bs_aes(uint32_t* out, uint32_t iters) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
#pragma unroll 1
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t s[128];
#pragma unroll
        for (int k = 0; k < 128; ++k) s[k] = (tid * 0x9e3779b9u) ^ (it * 0x85ebca6bu) ^ (k * 0xc2b2ae35u);
        bs_block(s);
#pragma unroll
        for (int k = 0; k < 128; ++k) acc ^= s[k];
    }
    out[tid] = acc;
}

// 32 blocks given as slices in `in` through the bitsliced form; the result,
// re-indexed to logical byte order, goes to `out` (one thread).
__global__ void bs_check(const uint32_t* in, uint32_t* out) {
    uint32_t s[128];
#pragma unroll
    for (int k = 0; k < 128; ++k) s[k] = in[k];
    bs_block(s);
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int i = 0; i < 8; ++i) out[8 * (r + 4 * c) + i] = s[8 * phys(r, c, 2) + i];
}

int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
    return 0;
}

// The bitsliced circuit on the host against host_aes128 (32 random blocks).
bool host_check(const uint32_t rk[44], uint32_t masks[11][128]) {
    std::mt19937 g(7);
    uint32_t blocks[32][4], want[32][4], s[128];
    for (int j = 0; j < 32; ++j) {
        for (int w = 0; w < 4; ++w) blocks[j][w] = g();
        host_aes128(rk, blocks[j], want[j]);
    }
    bitslice::to_slices(blocks, s);
    for (int k = 0; k < 128; ++k) s[k] ^= masks[0][k];
    for (int r = 1; r <= 10; ++r) {
        for (int n = 0; n < 16; ++n) bitslice::put(s, n, bitslice::sbox(bitslice::get(s, n)));
        bitslice::shift_rows(s);
        if (r < 10) bitslice::mix_columns(s);
        for (int k = 0; k < 128; ++k) s[k] ^= masks[r][k];
    }
    uint32_t got[32][4];
    bitslice::from_slices(s, got);
    return std::memcmp(got, want, sizeof got) == 0;
}

}  // namespace
}  // namespace cmc

int main(int argc, char** argv) {
    using namespace cmc;
    const uint32_t tt_iters = argc > 1 ? uint32_t(std::atoi(argv[1])) : 2000;
    const uint32_t bs_iters = argc > 2 ? uint32_t(std::atoi(argv[2])) : 40;
    uint32_t rk[44], t0[256];
    expand_u64(0x0706050403020100ULL, 0x0f0e0d0c0b0a0908ULL, rk);  // FIPS-197 C.1 key
    t0_table(t0);
    static uint32_t masks[11][128];
    bitslice::key_masks(rk, masks);
    const bool host_ok = host_check(rk, masks);
    std::printf("host: bitsliced circuit vs host AES on 32 random blocks %s\n", host_ok ? "ok" : "FAIL");
    std::fflush(stdout);

    TtKeys k;
    for (int i = 0; i < 44; ++i) {
        k.rk[i] = rk[i];
        k.kr[i] = (rk[i] << 8) | (rk[i] >> 24);
    }
    int sms = 0, clk_khz = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0), "attr");
    check(cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, 0), "attr");
    check(cudaMemcpyToSymbol(c_masks, masks, sizeof masks), "masks");
    uint32_t *d_t0, *d_out, *d_in;
    check(cudaMalloc(&d_t0, sizeof t0), "malloc");
    check(cudaMalloc(&d_in, 128 * 4), "malloc");
    check(cudaMalloc(&d_out, size_t(sms) * 384 * 4), "malloc");
    check(cudaMemcpy(d_t0, t0, sizeof t0, cudaMemcpyHostToDevice), "t0");
    const int tt_smem = int(kTableBytes);
    check(cudaFuncSetAttribute(tt_aes<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, tt_smem), "attr");
    check(cudaFuncSetAttribute(tt_check, cudaFuncAttributeMaxDynamicSharedMemorySize, tt_smem), "attr");

    // device checks
    tt_check<<<1, 32, tt_smem>>>(k, d_t0, d_out);
    uint32_t tt_ok = 0;
    check(cudaMemcpy(&tt_ok, d_out, 4, cudaMemcpyDeviceToHost), "tt check");
    uint32_t fips[32][4], sl[128], res[128], outb[32][4];
    for (int j = 0; j < 32; ++j) {
        fips[j][0] = 0x00112233u; fips[j][1] = 0x44556677u; fips[j][2] = 0x8899aabbu; fips[j][3] = 0xccddeeffu;
    }
    bitslice::to_slices(fips, sl);
    check(cudaMemcpy(d_in, sl, sizeof sl, cudaMemcpyHostToDevice), "in");
    bs_check<<<1, 1>>>(d_in, d_out);
    check(cudaMemcpy(res, d_out, sizeof res, cudaMemcpyDeviceToHost), "bs check");
    bitslice::from_slices(res, outb);
    bool bs_ok = true;
    for (int j = 0; j < 32; ++j)
        bs_ok = bs_ok && outb[j][0] == 0x69c4e0d8u && outb[j][1] == 0x6a7b0430u &&
                outb[j][2] == 0xd8cdb780u && outb[j][3] == 0x70b4c55au;
    std::printf("checks: host bitsliced vs host AES %s, device T-table FIPS %s, device bitsliced FIPS %s\n",
                host_ok ? "ok" : "FAIL", tt_ok ? "ok" : "FAIL", bs_ok ? "ok" : "FAIL");
    if (!host_ok || !tt_ok || !bs_ok) return 1;

    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    const double hz = double(clk_khz) * 1e3;
    for (int rep = 0; rep < 3; ++rep) {
        float ms_tt = 0, ms_bs = 0;
        cudaEventRecord(e0);
        tt_aes<3><<<sms, 384, tt_smem>>>(k, d_t0, d_out, tt_iters);
        cudaEventRecord(e1);
        check(cudaEventSynchronize(e1), "tt run");
        cudaEventElapsedTime(&ms_tt, e0, e1);
        cudaEventRecord(e0);
        bs_aes<<<sms, 256>>>(d_out, bs_iters);
        cudaEventRecord(e1);
        check(cudaEventSynchronize(e1), "bs run");
        cudaEventElapsedTime(&ms_bs, e0, e1);
        const double tt_blocks = double(sms) * 384 * 3 * tt_iters, bs_blocks = double(sms) * 256 * 32 * bs_iters;
        std::printf("T-table: %.3f ms, %.4f blocks/clk/SM | bitsliced: %.3f ms, %.4f blocks/clk/SM "
                    "(at the %d MHz rated clock)\n",
                    ms_tt, tt_blocks / (ms_tt * 1e-3 * hz * sms), ms_bs,
                    bs_blocks / (ms_bs * 1e-3 * hz * sms), clk_khz / 1000);
    }
    return 0;
}
