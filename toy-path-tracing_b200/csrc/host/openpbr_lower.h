// Host lowering of untextured OpenPBR materials into DevOpenPbr records, and
// the host halves of the tables' construction (sample tables whose
// trigonometry is evaluated once on the host, and the E_avg reductions).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/tpt.h"
#include "../device/render_types.h"

namespace tpt {

constexpr int kDaLen = 64 * 16 * 64 * 16;
constexpr int kCecLen = 64 * 64, kCecAvgLen = 64;
constexpr int kDecLen = 32 * 32 * 32, kDecAvgLen = 32 * 32;

// The eta of the specular albedo table (OpenPbrMaterial::requires_specular_eta)
// and of the coat table (requires_coat_eta), sanitized as the table cache does.
float openpbr_spec_table_eta(const tpt_openpbr_desc& m);
float openpbr_coat_table_eta(const tpt_openpbr_desc& m);

// make_bsdf's material part; `spec_da` / `coat_da` are the device tables for
// the two etas above, the E_avg arrays are host copies of the
// energy-compensation tables.
void lower_openpbr(const tpt_openpbr_desc& m, const float* spec_da, const float* coat_da, const float* cec_e_avg,
                   const float* dec_e_avg, DevOpenPbr* out);

// Inputs of the table-building kernels (directional_albedo.rs:134-167,
// 327-341, 700-725, 871-898): directions and sample points whose sines and
// cosines come from the host math library.
struct LutSampleTables {
  std::vector<float> da_dirs;     // 64 x 3: uniform-hemisphere directions
  std::vector<float> da_phi_cs;   // 16 x 2: cos, sin of the phi cell centres
  std::vector<float> cec_u;       // 256: stratified u
  std::vector<float> cec_cs;      // 256 x 2: cos, sin of 2 pi v
  std::vector<float> dec_uc;      // 4096: branch-selection u
  std::vector<float> dec_ux;      // 4096: u.x
  std::vector<float> dec_cs;      // 4096 x 2: cos, sin of 2 pi u.y
};
void lut_sample_tables(LutSampleTables* t);
// E_avg reductions over the E tables (same order as the reference's loops).
void conductor_e_avg(const float* e, float* e_avg);
void dielectric_e_avg(const float* e, float* e_avg);

}  // namespace tpt
