// Oracle (test infrastructure): path-replay adjoint of the MIS integrator
// with respect to OpenPBR material parameters.
//
// The reference renderer is not differentiable; this restates, on the CPU, the
// estimator the library's device adjoint computes, so that the device result
// can be checked sample by sample:
//
//  * Loss gradient per path: delta = dLoss/dimage[pixel] * exposure / spp
//    (the image is exposure times the running mean of spp samples, main.rs:
//    107-123).
//  * Detached sampling: sampled directions, lobe choices, Russian-roulette
//    probabilities and MIS weights are held fixed, so the sample weight
//    f cos / pdf of vertex i changes only through f, and every contribution
//    the path collects after vertex i scales with f_i.  With R_i the radiance
//    collected after vertex i, dL/dtheta = sum_i R_i * (df_i/dtheta) / f_i.
//  * Path replay: a first pass computes L (trace_mis); the second replays the
//    same path from its streams and subtracts what each vertex collects to get
//    R_i (replay_mis in render.cpp).
//  * df_i/dtheta: central difference of the closed-form BSDF at the fixed
//    (wo, wi) pair, between the material lowered at theta - h and theta + h
//    (clipped to the parameter's range; the divisor is the clipped span).  The
//    three base-colour channels are perturbed together: channel c of f depends
//    on base_color[c] only (diffuse albedo, metal F0 and F82 tint, coat
//    darkening base albedo are all per channel), so one pair of evaluations
//    gives all three partials.
//  * Accumulation in double per material: [base_color r, g, b,
//    specular_roughness, base_metalness, specular_ior, coat_weight].
#include <mutex>
#include <thread>
#include <atomic>

#include "render.h"

namespace orc {

constexpr int kGradParams = 7;
constexpr int kGroups = 5;  // base colour, roughness, metalness, ior, coat weight

namespace {

// Range of each parameter group (what the lowering accepts without clamping
// it away) and the index of its first gradient slot.
void group_range(int g, float* lo, float* hi) {
  *lo = 0.0f;
  *hi = 1.0f;
  if (g == 3) {  // specular_ior
    *lo = 1.0f;
    *hi = 10.0f;
  }
}
const int kGroupSlot[kGroups] = {0, 3, 4, 5, 6};

float* group_field(OpenPbrDesc& d, int g, int c) {
  switch (g) {
    case 0: return &d.base_color[c];
    case 1: return &d.specular_roughness;
    case 2: return &d.base_metalness;
    case 3: return &d.specular_ior;
    default: return &d.coat_weight;
  }
}

struct Perturbation {
  bool active = false;
  Material lo, hi;
  float span[3] = {0, 0, 0};
};

struct Tables {
  // per material, per group
  std::vector<Perturbation> pert;
  uint32_t mask = 0;
};

Tables build_tables(const RenderScene& s, uint32_t mask, float h, int nthreads) {
  Tables T;
  T.mask = mask;
  T.pert.resize(s.materials.size() * kGroups);
  for (size_t j = 0; j < s.materials.size(); ++j) {
    const Material& m = s.materials[j];
    if (m.kind != kOpenPbr) continue;
    for (int g = 0; g < kGroups; ++g) {
      if (!(mask & (1u << g))) continue;
      Perturbation& P = T.pert[j * kGroups + g];
      P.active = true;
      P.lo = m;
      P.hi = m;
      float rlo, rhi;
      group_range(g, &rlo, &rhi);
      const int nc = g == 0 ? 3 : 1;
      for (int c = 0; c < nc; ++c) {
        OpenPbrDesc base = m.openpbr;
        const float x = *group_field(base, g, c);
        const float a = std::fmax(x - h, rlo), b = std::fmin(x + h, rhi);
        *group_field(P.lo.openpbr, g, c) = a;
        *group_field(P.hi.openpbr, g, c) = b;
        P.span[c] = b - a;
      }
      P.lo.luts = openpbr_luts_for(P.lo.openpbr, nthreads);
      P.hi.luts = openpbr_luts_for(P.hi.openpbr, nthreads);
    }
  }
  return T;
}

Vec3 bsdf_f(const Material& m, bool front, Vec3 wo_l, Vec3 wi_l) {
  OpenPbrBsdf b{make_openpbr_params(m.openpbr, front, wo_l), m.luts};
  return b.eval(wo_l, wi_l, kRadiance);
}

struct GradSink : AdjointVertexSink {
  const RenderScene* s;
  const Tables* T;
  Vec3 delta;
  double* grad;  // this thread's accumulator, n_mat * kGradParams

  void vertex(uint32_t mi, const Vertex& v, Vec3 wi, Vec3 R) override {
    const Material& m = s->materials[mi];
    const Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    const Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
    const Vec3 f0 = bsdf_f(m, v.front_face, wo_l, wi_l);
    const float f0c[3] = {f0.x, f0.y, f0.z};
    const float w[3] = {delta.x * R.x, delta.y * R.y, delta.z * R.z};
    for (int g = 0; g < kGroups; ++g) {
      const Perturbation& P = T->pert[mi * kGroups + g];
      if (!P.active) continue;
      const Vec3 fp = bsdf_f(P.hi, v.front_face, wo_l, wi_l);
      const Vec3 fm = bsdf_f(P.lo, v.front_face, wo_l, wi_l);
      const float df[3] = {fp.x - fm.x, fp.y - fm.y, fp.z - fm.z};
      double* gm = grad + (size_t)mi * kGradParams + kGroupSlot[g];
      if (g == 0) {
        for (int c = 0; c < 3; ++c)
          if (f0c[c] > 0.0f && P.span[c] > 0.0f) gm[c] += (double)w[c] * ((double)df[c] / P.span[c]) / f0c[c];
      } else if (P.span[0] > 0.0f) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c)
          if (f0c[c] > 0.0f) acc += (double)w[c] * ((double)df[c] / P.span[0]) / f0c[c];
        gm[0] += acc;
      }
    }
  }
};

}  // namespace

// Gradient of a loss with respect to the OpenPBR parameters of every material,
// given dLoss/dimage (width * height * 3 floats); grad: n_mat * 7 doubles
// (overwritten).  Only MIS jobs.
void render_adjoint(const RenderScene& s, const RenderJob& job, const float* d_image, uint32_t mask, float h,
                    double* grad, int nthreads) {
  const Tables T = build_tables(s, mask, h, nthreads);
  const size_t nm = s.materials.size();
  std::fill(grad, grad + nm * kGradParams, 0.0);
  const uint32_t npix = job.width * job.height;
  std::mutex mu;
  std::atomic<uint32_t> next{0};
  auto worker = [&]() {
    std::vector<double> acc(nm * kGradParams, 0.0);
    GradSink sink;
    sink.s = &s;
    sink.T = &T;
    sink.grad = acc.data();
    for (;;) {
      const uint32_t pixel = next.fetch_add(1);
      if (pixel >= npix) break;
      const float scale = job.cam.exposure / (float)job.spp;
      sink.delta = Vec3(d_image[3 * pixel], d_image[3 * pixel + 1], d_image[3 * pixel + 2]) * scale;
      const uint32_t px = pixel % job.width, py = pixel / job.width;
      for (uint32_t i = 0; i < job.spp; ++i) {
        PathSampler ps(px, py, i, job.spp, job.width, job.height, job.seed);
        Vec2 us = ps.camera_sample();
        Ray r = job.cam.generate_ray_differential(job.width, job.height, px, py, us, job.spp);
        const Vec3 L = trace_mis(s, r, ps, job.max_depth);
        replay_mis(s, r, ps, job.max_depth, L, sink);
      }
    }
    std::lock_guard<std::mutex> lock(mu);
    for (size_t k = 0; k < acc.size(); ++k) grad[k] += acc[k];
  };
  const int nt = std::max(1, nthreads);
  std::vector<std::thread> ts;
  for (int t = 0; t < nt; ++t) ts.emplace_back(worker);
  for (auto& t : ts) t.join();
}

}  // namespace orc

extern "C" {

// cam11: eye(3) look_at(3) up(3) fov_y exposure.  mask bits: 1 base colour,
// 2 specular roughness, 4 metalness, 8 specular ior, 16 coat weight.
void orc_render_adjoint(void* h, const float* cam11, uint32_t w, uint32_t hgt, uint32_t spp, uint32_t depth,
                        const float* d_image, uint32_t mask, float step, double* grad, int nthreads,
                        uint32_t seed) {
  using namespace orc;
  RenderJob j;
  j.cam = Camera::make(Vec3(cam11[0], cam11[1], cam11[2]), Vec3(cam11[3], cam11[4], cam11[5]),
                       Vec3(cam11[6], cam11[7], cam11[8]), cam11[9], cam11[10]);
  j.width = w;
  j.height = hgt;
  j.spp = spp;
  j.max_depth = depth;
  j.integrator = 0;
  j.seed = seed;
  render_adjoint(*(const RenderScene*)h, j, d_image, mask, step, grad, nthreads);
}

}  // extern "C"
