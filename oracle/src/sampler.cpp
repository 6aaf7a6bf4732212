// Oracle: sampler (crates/renderer/src/sampler/zsobol.rs:73-285, path_sampler.rs:172-250).
#include "sampler.h"

namespace orc {

namespace {
// zsobol.rs:98-171: Sobol generator matrices for the first four dimensions,
// one row per input bit (bit i of the 16-bit reversed index).
const uint16_t kSobolDirections[4][16] = {
    {0x8000, 0x4000, 0x2000, 0x1000, 0x0800, 0x0400, 0x0200, 0x0100, 0x0080, 0x0040, 0x0020, 0x0010,
     0x0008, 0x0004, 0x0002, 0x0001},
    {0xFFFF, 0x5555, 0x3333, 0x1111, 0x0F0F, 0x0505, 0x0303, 0x0101, 0x00FF, 0x0055, 0x0033, 0x0011,
     0x000F, 0x0005, 0x0003, 0x0001},
    {0xAA09, 0x7706, 0x3903, 0x1601, 0x09AA, 0x0677, 0x0339, 0x0116, 0x00A3, 0x0071, 0x003A, 0x0017,
     0x0009, 0x0006, 0x0003, 0x0001},
    {0xA0C3, 0x4041, 0x302D, 0x101E, 0x0B67, 0x079A, 0x02A4, 0x011B, 0x00C9, 0x0045, 0x002E, 0x001F,
     0x000A, 0x0004, 0x0003, 0x0001},
};

// zsobol.rs:238-263: the 24 permutations of four base-4 digits
const uint8_t kPerm[24][4] = {
    {0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 2, 1}, {0, 3, 1, 2},
    {1, 0, 2, 3}, {1, 0, 3, 2}, {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 2, 0}, {1, 3, 0, 2},
    {2, 1, 0, 3}, {2, 1, 3, 0}, {2, 0, 1, 3}, {2, 0, 3, 1}, {2, 3, 0, 1}, {2, 3, 1, 0},
    {3, 1, 2, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 2, 0, 1}, {3, 0, 2, 1}, {3, 0, 1, 2},
};

uint32_t log2_int(uint32_t v) { return 31u - (uint32_t)__builtin_clz(v); }
uint32_t round_up_pow2(uint32_t v) {
  if (v <= 1) return 1;
  return 1u << (32u - (uint32_t)__builtin_clz(v - 1));
}
uint32_t fold_u64(uint64_t v) { return (uint32_t)v ^ (uint32_t)(v >> 32); }
}  // namespace

uint16_t sobol_reversed_index(uint16_t index, int dimension) {
  if (dimension == 0) return reverse_bits16(index);
  uint16_t s = 0;
  for (int i = 0; i < 16; ++i)
    if (index & (1u << i)) s ^= kSobolDirections[dimension][i];
  return s;
}

void shuffled_scrambled_sobol(uint32_t index, uint32_t seed, int depth, uint32_t* out) {
  uint32_t idx = reverse_and_shuffle(index, seed);
  for (int d = 0; d < depth; ++d) {
    uint16_t sob = sobol_reversed_index((uint16_t)(idx >> 16), d);
    out[d] = scramble_and_reverse((uint32_t)sob, rotate_bytes(seed, (uint32_t)d));
  }
}

IndexSampler::IndexSampler(uint32_t spp, uint32_t rx, uint32_t ry) {
  log2_spp = log2_int(round_up_pow2(spp));
  uint32_t res = round_up_pow2(rx > ry ? rx : ry);
  uint32_t log4 = (log2_spp + 1) / 2;
  n_base4_digits = log2_int(res) + log4;
}

uint64_t IndexSampler::sample_index(uint32_t px, uint32_t py, uint32_t sample, uint32_t dimension) const {
  uint64_t morton = (encode_morton_2(px, py) << log2_spp) | (uint64_t)sample;
  return permuted_index(morton, dimension);
}

uint64_t IndexSampler::permuted_index(uint64_t morton, uint32_t dimension) const {
  uint64_t out = 0;
  bool pow2 = (log2_spp & 1u) != 0;
  uint32_t last = pow2 ? 1u : 0u;
  uint64_t dim_hash = 0x55555555ull * (uint64_t)dimension;
  for (int64_t i = (int64_t)n_base4_digits - 1; i >= (int64_t)last; --i) {
    uint32_t shift = 2u * (uint32_t)i - (pow2 ? 1u : 0u);
    uint32_t digit = (uint32_t)((morton >> shift) & 3u);
    uint64_t higher = morton >> (shift + 2);
    uint32_t p = (uint32_t)((mix_bits(higher ^ dim_hash) >> 24) % 24u);
    out |= (uint64_t)kPerm[p][digit] << shift;
  }
  if (pow2) {
    uint64_t digit = morton & 1u;
    out |= digit ^ (mix_bits((morton >> 1) ^ dim_hash) & 1u);
  }
  return out;
}

float PathSampler::sample_1d(uint32_t dim) const {
  uint32_t index = fold_u64(idx.sample_index(px, py, sample, dim));
  uint32_t seed = fold_u64(mix_bits(((uint64_t)this->seed << 32) | (uint64_t)dim));  // seed_for_dimension
  uint32_t v[1];
  shuffled_scrambled_sobol(index, seed, 1, v);
  return uint_to_float(v[0]);
}

Vec2 PathSampler::sample_2d(uint32_t dim) const {
  uint32_t index = fold_u64(idx.sample_index(px, py, sample, dim));
  uint32_t seed = fold_u64(mix_bits(((uint64_t)this->seed << 32) | (uint64_t)dim));  // seed_for_dimension
  uint32_t v[2];
  shuffled_scrambled_sobol(index, seed, 2, v);
  return Vec2(uint_to_float(v[0]), uint_to_float(v[1]));
}

uint32_t PathSampler::aux_rng_seed(uint32_t dim) const {
  uint64_t index = idx.sample_index(px, py, sample, dim);
  uint64_t bits = mix_bits(index ^ ((uint64_t)dim << 32) ^ (uint64_t)seed);
  return pcg_hash(fold_u64(bits));
}

// path_sampler.rs:189-210 (dimension base 2 + 16*depth)
VertexRandoms PathSampler::path_vertex_randoms(uint32_t depth) const {
  uint32_t base = 2u + depth * 16u;
  VertexRandoms r;
  r.light.u_category = sample_1d(base + 0);
  r.light.u_tree = sample_1d(base + 1);
  r.light.u_light_aux = sample_1d(base + 2);
  r.light.u_surface = sample_2d(base + 3);
  r.material.u_lobe = sample_1d(base + 5);
  r.material.u_layer = sample_1d(base + 6);
  r.material.u_dir = sample_2d(base + 7);
  r.material.u_extra0 = sample_1d(base + 9);
  r.material.u_extra1 = sample_1d(base + 10);
  r.material.u_extra2 = sample_1d(base + 11);
  r.material.u_extra3 = sample_1d(base + 12);
  r.u_rr = sample_1d(base + 13);
  r.aux_rng_seed = aux_rng_seed(base + 14);
  return r;
}

}  // namespace orc
