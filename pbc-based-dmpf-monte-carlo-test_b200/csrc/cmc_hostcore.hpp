// cmc_hostcore.hpp -- host-side AES, batch keys and parameter derivation.
#pragma once
#include <cstdint>

#include "cmc.h"

namespace cmc {

const uint8_t* sbox();
void t0_table(uint32_t out[256]);
void expand_words(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t rk[44]);
void expand_u64(uint64_t lo, uint64_t hi, uint32_t rk[44]);
void host_aes128(const uint32_t rk[44], const uint32_t in[4], uint32_t out[4]);
void batch_key(uint64_t seed, uint64_t batch_id, uint32_t rk[44]);
unsigned bit_width(uint64_t v);
float reference_log2(uint64_t n);
int derive_params(uint32_t mode, uint32_t pnum, uint32_t ell_i, uint32_t k,
                  uint32_t buckets_override, uint32_t kick_override, uint32_t input_mode,
                  cmc_params* out, const char** why);

}  // namespace cmc
