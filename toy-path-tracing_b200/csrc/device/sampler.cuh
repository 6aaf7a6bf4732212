// Per-pixel sample streams on the device: Z-Sobol index permutation, Owen-
// scrambled Sobol (Laine-Karras) and the PCG hash, integer-exact restatement of
// crates/renderer/src/sampler/{pcg,zsobol,aux_rng,path_sampler}.rs.
#pragma once
#include <cstdint>

namespace tpt {

__device__ __forceinline__ uint32_t pcg_state_transition(uint32_t s) { return s * 747796405u + 2891336453u; }
__device__ __forceinline__ uint32_t pcg_output(uint32_t s) {
  s ^= s >> (4u + (s >> 28));
  s *= 277803737u;
  return s ^ (s >> 22);
}
__device__ __forceinline__ uint32_t pcg_hash(uint32_t k) { return pcg_output(pcg_state_transition(k)); }

__device__ __forceinline__ uint32_t lk_permutation(uint32_t v, uint32_t seed) {
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return v;
}

__device__ __forceinline__ float uint_to_float(uint32_t v) {
  const uint32_t mask = v >> 24;
  return __uint2float_rn(v & ~mask) * (1.0f / 4294967296.0f);
}

__device__ __forceinline__ uint64_t mix_bits(uint64_t v) {
  v ^= v >> 31;
  v *= 0x7fb5d329728ea185ull;
  v ^= v >> 27;
  v *= 0x81dadef4bc2dd44dull;
  v ^= v >> 33;
  return v;
}

__device__ __forceinline__ uint64_t left_shift_2(uint64_t v) {
  v &= 0xffffffffull;
  v = (v ^ (v << 16)) & 0x0000ffff0000ffffull;
  v = (v ^ (v << 8)) & 0x00ff00ff00ff00ffull;
  v = (v ^ (v << 4)) & 0x0f0f0f0f0f0f0f0full;
  v = (v ^ (v << 2)) & 0x3333333333333333ull;
  v = (v ^ (v << 1)) & 0x5555555555555555ull;
  return v;
}

// zsobol.rs:98-171 generator matrices, rows indexed by input bit.
__constant__ uint16_t c_sobol_dirs[3][16] = {
    {0xFFFF, 0x5555, 0x3333, 0x1111, 0x0F0F, 0x0505, 0x0303, 0x0101, 0x00FF, 0x0055, 0x0033, 0x0011, 0x000F,
     0x0005, 0x0003, 0x0001},
    {0xAA09, 0x7706, 0x3903, 0x1601, 0x09AA, 0x0677, 0x0339, 0x0116, 0x00A3, 0x0071, 0x003A, 0x0017, 0x0009,
     0x0006, 0x0003, 0x0001},
    {0xA0C3, 0x4041, 0x302D, 0x101E, 0x0B67, 0x079A, 0x02A4, 0x011B, 0x00C9, 0x0045, 0x002E, 0x001F, 0x000A,
     0x0004, 0x0003, 0x0001},
};
// zsobol.rs:238-263: the 24 permutations of a base-4 digit, one byte each
// (2 bits per digit: permutation p maps digit d to (byte_p >> 2d) & 3), packed
// into three 64-bit immediates so a per-lane index costs ALU work instead of a
// serialized constant-bank access.
__device__ __forceinline__ uint32_t perm_digit(uint32_t p, uint32_t digit) {
  uint64_t w;
  if (p < 8) w = 0xB1E19C6C78D8B4E4ull;        // p 0..7:  E4 B4 D8 78 6C 9C E1 B1
  else if (p < 16) w = 0x72D236C68D2D39C9ull;  // p 8..15: C9 39 2D 8D C6 36 D2 72
  else w = 0x93634B1B87271E4Eull;              // p 16..23: 4E 1E 27 87 1B 4B 63 93
  const uint32_t byte = (uint32_t)(w >> (8u * (p & 7u))) & 0xFFu;
  return (byte >> (2u * digit)) & 3u;
}

__device__ __forceinline__ uint32_t sobol_reversed(uint32_t index16, int dim) {
  if (dim == 0) return __brev(index16) >> 16;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i)
    if (index16 & (1u << i)) s ^= c_sobol_dirs[dim - 1][i];
  return s;
}

// IndexSampler (zsobol.rs:206-285) + PathSampler (path_sampler.rs:146-250)
struct PathSamplerDev {
  uint64_t morton;  // (encode_morton_2(px, py) << log2_spp) | sample
  uint32_t log2_spp;
  uint32_t n_base4_digits;
  uint32_t seed;  // the scramble seed: 0 is the reference's SCRAMBLE_SEED (path_sampler.rs:77)

  __device__ __forceinline__ void init(uint32_t px, uint32_t py, uint32_t sample, uint32_t log2spp, uint32_t ndig,
                                       uint32_t scramble = 0u) {
    log2_spp = log2spp;
    n_base4_digits = ndig;
    seed = scramble;
    morton = (((left_shift_2(py) << 1) | left_shift_2(px)) << log2spp) | (uint64_t)sample;
  }

  __device__ __forceinline__ uint64_t sample_index(uint32_t dimension) const {
    uint64_t out = 0;
    const bool pow2 = (log2_spp & 1u) != 0;
    const int last = pow2 ? 1 : 0;
    const uint64_t dim_hash = 0x55555555ull * (uint64_t)dimension;
    for (int i = (int)n_base4_digits - 1; i >= last; --i) {
      const uint32_t shift = 2u * (uint32_t)i - (pow2 ? 1u : 0u);
      const uint32_t digit = (uint32_t)((morton >> shift) & 3u);
      const uint64_t higher = morton >> (shift + 2);
      const uint32_t p = (uint32_t)((mix_bits(higher ^ dim_hash) >> 24) % 24u);
      out |= (uint64_t)perm_digit(p, digit) << shift;
    }
    if (pow2) out |= (morton & 1u) ^ (mix_bits((morton >> 1) ^ dim_hash) & 1u);
    return out;
  }

  __device__ __noinline__ void sobol(uint32_t dimension, int depth, float* out) const {
    const uint64_t si = sample_index(dimension);
    const uint32_t index = (uint32_t)si ^ (uint32_t)(si >> 32);
    const uint64_t sb = mix_bits(((uint64_t)this->seed << 32) | (uint64_t)dimension);  // seed_for_dimension
    const uint32_t seed = (uint32_t)sb ^ (uint32_t)(sb >> 32);
    const uint32_t idx = lk_permutation(__brev(index), seed);
    for (int d = 0; d < depth; ++d) {
      const uint32_t sob = sobol_reversed(idx >> 16, d);
      const uint32_t r = (8u * (uint32_t)d) & 31u;
      const uint32_t rot = r == 0 ? seed : ((seed >> r) | (seed << (32u - r)));
      out[d] = uint_to_float(__brev(lk_permutation(sob, rot)));
    }
  }
  __device__ __forceinline__ float sample_1d(uint32_t dim) const {
    float v[1];
    sobol(dim, 1, v);
    return v[0];
  }
  __device__ __forceinline__ void sample_2d(uint32_t dim, float& a, float& b) const {
    float v[2];
    sobol(dim, 2, v);
    a = v[0];
    b = v[1];
  }
  __device__ __forceinline__ uint32_t aux_rng_seed(uint32_t dim) const {
    const uint64_t si = sample_index(dim);
    const uint64_t bits = mix_bits(si ^ ((uint64_t)dim << 32) ^ (uint64_t)seed);
    return pcg_hash((uint32_t)bits ^ (uint32_t)(bits >> 32));
  }
};

// Dimension layout (path_sampler.rs:153-169): camera at 0, vertex `depth` at
// 2 + 16 * depth + offset.
constexpr uint32_t kDimCamera = 0;
__device__ __forceinline__ uint32_t vertex_dim(uint32_t depth, uint32_t offset) { return 2u + 16u * depth + offset; }
constexpr uint32_t kOffCategory = 0, kOffTree = 1, kOffLightAux = 2, kOffSurface = 3, kOffLobe = 5, kOffLayer = 6,
                   kOffDir = 7, kOffExtra0 = 9, kOffExtra1 = 10, kOffExtra2 = 11, kOffExtra3 = 12, kOffRr = 13,
                   kOffAuxSeed = 14;

}  // namespace tpt
