// Oracle: Z-Sobol index sampler + Owen-scrambled Sobol + PCG hash.
// Restates crates/renderer/src/sampler/{pcg,zsobol,aux_rng,path_sampler}.rs.
#pragma once
#include "common.h"

namespace orc {

// pcg.rs:1-13
inline uint32_t pcg_state_transition(uint32_t s) { return s * 747796405u + 2891336453u; }
inline uint32_t pcg_output(uint32_t s) {
  s ^= s >> (4u + (s >> 28));
  s *= 277803737u;
  return s ^ (s >> 22);
}
inline uint32_t pcg_hash(uint32_t k) { return pcg_output(pcg_state_transition(k)); }

// aux_rng.rs:15-29
struct AuxRng {
  uint32_t state;
  explicit AuxRng(uint32_t seed) : state(pcg_state_transition(seed)) {}
  uint32_t next_u32() { state = pcg_state_transition(state); return pcg_output(state); }
  float next_f32() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
};

inline uint32_t reverse_bits32(uint32_t v) {
  v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
  v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
  v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
  v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
  return (v >> 16) | (v << 16);
}
inline uint16_t reverse_bits16(uint16_t v) { return (uint16_t)(reverse_bits32(v) >> 16); }

// zsobol.rs:9-48
inline uint32_t laine_karras_permutation(uint32_t v, uint32_t seed) {
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return v;
}
inline uint32_t reverse_and_shuffle(uint32_t v, uint32_t seed) { return laine_karras_permutation(reverse_bits32(v), seed); }
inline uint32_t rotate_bytes(uint32_t v, uint32_t dist) {
  uint32_t r = (dist * 8u) & 31u;
  return r == 0 ? v : ((v >> r) | (v << (32u - r)));
}
inline uint32_t scramble_and_reverse(uint32_t v, uint32_t seed) { return reverse_bits32(laine_karras_permutation(v, seed)); }
inline float uint_to_float(uint32_t v) {
  uint32_t mask = v >> 24;
  uint32_t safe = v & ~mask;
  return (float)safe * (1.0f / 4294967296.0f);
}
inline uint64_t mix_bits(uint64_t v) {
  v ^= v >> 31;
  v *= 0x7fb5d329728ea185ull;
  v ^= v >> 27;
  v *= 0x81dadef4bc2dd44dull;
  v ^= v >> 33;
  return v;
}
inline uint64_t left_shift_2(uint64_t v) {
  v &= 0xffffffffull;
  v = (v ^ (v << 16)) & 0x0000ffff0000ffffull;
  v = (v ^ (v << 8)) & 0x00ff00ff00ff00ffull;
  v = (v ^ (v << 4)) & 0x0f0f0f0f0f0f0f0full;
  v = (v ^ (v << 2)) & 0x3333333333333333ull;
  v = (v ^ (v << 1)) & 0x5555555555555555ull;
  return v;
}
inline uint64_t encode_morton_2(uint32_t x, uint32_t y) { return (left_shift_2(y) << 1) | left_shift_2(x); }

uint16_t sobol_reversed_index(uint16_t index, int dimension);
void shuffled_scrambled_sobol(uint32_t index, uint32_t seed, int depth, uint32_t* out);

struct IndexSampler {
  uint32_t log2_spp = 0;
  uint32_t n_base4_digits = 0;
  IndexSampler() = default;
  IndexSampler(uint32_t spp, uint32_t res_x, uint32_t res_y);
  uint64_t sample_index(uint32_t px, uint32_t py, uint32_t sample, uint32_t dimension) const;
  uint64_t permuted_index(uint64_t morton, uint32_t dimension) const;
};

struct LightRandoms { float u_category, u_tree, u_light_aux; Vec2 u_surface; };
struct MaterialRandoms { float u_lobe, u_layer; Vec2 u_dir; float u_extra0, u_extra1, u_extra2, u_extra3; };
struct VertexRandoms { LightRandoms light; MaterialRandoms material; float u_rr; uint32_t aux_rng_seed; };

// path_sampler.rs:146-250
struct PathSampler {
  IndexSampler idx;
  uint32_t px, py, sample;
  // Scramble seed: 0 is the reference's SCRAMBLE_SEED (path_sampler.rs:77); other
  // values give independent streams (tpt_render_job.seed).
  uint32_t seed;
  PathSampler(uint32_t px_, uint32_t py_, uint32_t sample_, uint32_t spp, uint32_t rx, uint32_t ry,
              uint32_t seed_ = 0)
      : idx(spp, rx, ry), px(px_), py(py_), sample(sample_), seed(seed_) {}
  Vec2 camera_sample() const { return sample_2d(0); }
  uint32_t initial_aux_rng_seed() const { return aux_rng_seed(0x80000000u); }
  VertexRandoms path_vertex_randoms(uint32_t depth) const;
  float sample_1d(uint32_t dim) const;
  Vec2 sample_2d(uint32_t dim) const;
  uint32_t aux_rng_seed(uint32_t dim) const;
};

}  // namespace orc
