// Scene upload, render half: vertex attributes, materials, per-instance
// shading records, the SG light tree and the emitter-triangle -> leaf map that
// replaces the reference's HashMap / linear searches (light_tree/mod.rs:101-108,
// scene/mod.rs:583-594).
#include <cmath>
#include <cstring>
#include <string>

#include "../host/env_build.h"
#include "../host/openpbr_lower.h"
#include "internal.h"

namespace tpt {

// The host-side view of a material: its kind, Lambert albedo and what it
// emits (the emissive material's colour and strength; an OpenPBR material's
// emission_color and emission_luminance).
HostMaterial host_material(const tpt_material_desc& m) {
  HostMaterial h{};
  h.kind = m.kind;
  std::memcpy(h.rho, m.rho, 12);
  if (m.kind == TPT_MATERIAL_OPENPBR && m.openpbr) {
    std::memcpy(h.color, m.openpbr->emission_color, 12);
    h.strength = m.openpbr->emission_luminance;
  } else {
    std::memcpy(h.color, m.color, 12);
    h.strength = m.strength;
  }
  return h;
}

tpt_status scene_alloc(tpt_scene* s, size_t bytes, void** out) {
  bytes = std::max<size_t>(bytes, 128);
  void* p = nullptr;
  tpt_status st = cuda_check(s->ctx, cudaMalloc(&p, bytes), "cudaMalloc(scene)");
  if (st) return st;
  s->allocations.push_back(p);
  s->device_bytes += bytes;
  *out = p;
  return TPT_OK;
}

namespace {
template <class T>
tpt_status put(tpt_scene* s, const std::vector<T>& v, const T** dst) {
  void* p = nullptr;
  tpt_status st = scene_alloc(s, v.size() * sizeof(T), &p);
  if (st) return st;
  if (!v.empty()) {
    st = cuda_check(s->ctx, cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy(scene)");
    if (st) return st;
  }
  *dst = (const T*)p;
  return TPT_OK;
}
}  // namespace

tpt_status lower_openpbr_material(tpt_context* ctx, const tpt_openpbr_desc& d, DevOpenPbr* out) {
  const float *spec_da = nullptr, *coat_da = nullptr;
  tpt_status st = ensure_ec_tables(ctx);
  if (!st) st = ensure_da_table(ctx, openpbr_spec_table_eta(d), &spec_da);
  if (!st && d.coat_weight > 0.0f) st = ensure_da_table(ctx, openpbr_coat_table_eta(d), &coat_da);
  if (st) return st;
  lower_openpbr(d, spec_da, coat_da, ctx->h_cec_e_avg.data(), ctx->h_dec_e_avg.data(), out);
  return TPT_OK;
}

tpt_status upload_render_data(tpt_scene* s, const tpt_scene_desc* desc) {
  tpt_context* ctx = s->ctx;
  // materials
  std::vector<HostMaterial> hmats(desc->num_materials);
  std::vector<DevMaterialRec> dmats(desc->num_materials);
  if (desc->num_materials && !desc->materials) return set_error(ctx, TPT_ERR_INVALID_ARG, "materials is NULL");
  std::vector<DevOpenPbr> opbr;
  s->material_kinds.assign(desc->num_materials, 0u);
  s->opbr_desc.clear();
  s->opbr_of_material.clear();
  for (uint32_t i = 0; i < desc->num_materials; ++i) {
    const tpt_material_desc& m = desc->materials[i];
    if (m.kind != TPT_MATERIAL_NORMALIZED_LAMBERT && m.kind != TPT_MATERIAL_EMISSIVE &&
        m.kind != TPT_MATERIAL_OPENPBR)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "material " + std::to_string(i) + ": unsupported kind");
    s->material_kinds[i] = m.kind;
    uint32_t opbr_index = 0;
    if (m.kind == TPT_MATERIAL_OPENPBR) {
      if (!m.openpbr) return set_error(ctx, TPT_ERR_INVALID_ARG, "material " + std::to_string(i) + ": openpbr is NULL");
      DevOpenPbr rec;
      tpt_status st = lower_openpbr_material(ctx, *m.openpbr, &rec);
      if (st) return st;
      opbr_index = (uint32_t)opbr.size();
      opbr.push_back(rec);
      s->opbr_desc.push_back(*m.openpbr);
    }
    s->opbr_of_material.push_back(m.kind == TPT_MATERIAL_OPENPBR ? opbr_index : kInvalidNode);
    HostMaterial h = host_material(m);
    hmats[i] = h;
    DevMaterialRec d{};
    d.kind = m.kind;
    std::memcpy(d.rho, m.rho, 12);
    std::memcpy(d.color, h.color, 12);
    d.strength = h.strength;
    d.openpbr = opbr_index;
    d.emits = m.kind == TPT_MATERIAL_OPENPBR && h.may_emit() ? 1u : 0u;
    dmats[i] = d;
  }
  for (uint32_t i = 0; i < desc->num_instances; ++i)
    if (desc->instances[i].material_index >= desc->num_materials && desc->num_materials)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "instance " + std::to_string(i) + ": material index out of range");
  // alpha tests (Material::has_alpha_test, untextured): per instance, the
  // clamped opacity its hits are tested against, 1 for none
  std::vector<float> ialpha;
  {
    std::vector<float> malpha(desc->num_materials, 1.0f);
    bool any = false;
    for (uint32_t i = 0; i < desc->num_materials; ++i) {
      const tpt_material_desc& m = desc->materials[i];
      const float o = m.kind == TPT_MATERIAL_OPENPBR ? m.openpbr->geometry_opacity : (m.has_opacity ? m.opacity : 1.0f);
      if (o < 1.0f) {
        malpha[i] = o < 0.0f ? 0.0f : o;
        any = true;
      }
    }
    if (any) {
      ialpha.resize(desc->num_instances, 1.0f);
      for (uint32_t i = 0; i < desc->num_instances; ++i)
        if (desc->num_materials) ialpha[i] = malpha[desc->instances[i].material_index];
    }
  }

  // vertex attributes, concatenated per mesh
  std::vector<float> pos, nrm, uv;
  std::vector<uint32_t> idx;
  std::vector<DevMeshInfo> minfo(desc->num_meshes);
  std::vector<HostMesh> hmesh(desc->num_meshes);
  for (uint32_t m = 0; m < desc->num_meshes; ++m) {
    const tpt_mesh_desc& md = desc->meshes[m];
    DevMeshInfo mi{};
    mi.vtx_base = (uint32_t)(pos.size() / 3);
    mi.idx_base = (uint32_t)idx.size();
    mi.num_tris = (uint32_t)(md.num_indices / 3);
    mi.flags = (md.normals ? 1u : 0u) | (md.uvs ? 2u : 0u);
    pos.insert(pos.end(), md.positions, md.positions + 3 * md.num_vertices);
    if (md.normals) nrm.resize(pos.size(), 0.0f), std::memcpy(&nrm[3 * mi.vtx_base], md.normals, 12 * md.num_vertices);
    else nrm.resize(pos.size(), 0.0f);
    uv.resize(2 * (pos.size() / 3), 0.0f);
    if (md.uvs) std::memcpy(&uv[2 * mi.vtx_base], md.uvs, 8 * md.num_vertices);
    idx.insert(idx.end(), md.indices, md.indices + md.num_indices);
    minfo[m] = mi;
    hmesh[m] = HostMesh{md.positions, md.normals, md.uvs, md.indices, (uint32_t)md.num_vertices, mi.num_tris};
  }

  // point, spot and directional lights (PointLight::new, SpotLight::new, DirectionalLight::new)
  if ((desc->num_point_lights && !desc->point_lights) || (desc->num_spot_lights && !desc->spot_lights) ||
      (desc->num_directional_lights && !desc->directional_lights))
    return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL light array");
  std::vector<HostPointLight> hpoints(desc->num_point_lights);
  std::vector<DevPointLight> dpoints(desc->num_point_lights);
  for (uint32_t i = 0; i < desc->num_point_lights; ++i) {
    const tpt_point_light_desc& d = desc->point_lights[i];
    HostPointLight h{};
    DevPointLight dp{};
    for (int k = 0; k < 3; ++k) {
      h.position[k] = dp.position[k] = d.position[k];
      h.color[k] = dp.color[k] = d.color[k];
    }
    h.intensity = dp.intensity = d.intensity;
    hpoints[i] = h;
    dpoints[i] = dp;
  }
  std::vector<HostSpotLight> hspots(desc->num_spot_lights);
  std::vector<DevSpotLight> dspots(desc->num_spot_lights);
  for (uint32_t i = 0; i < desc->num_spot_lights; ++i) {
    const tpt_spot_light_desc& d = desc->spot_lights[i];
    make_spot_light(d.position, d.direction, d.color, d.intensity, d.total_width, d.falloff_start, &hspots[i]);
    DevSpotLight ds{};
    std::memcpy(ds.position, hspots[i].position, 12);
    std::memcpy(ds.direction, hspots[i].direction, 12);
    std::memcpy(ds.color, hspots[i].color, 12);
    ds.intensity = hspots[i].intensity;
    ds.cos_total_width = hspots[i].cos_total_width;
    ds.cos_falloff_start = hspots[i].cos_falloff_start;
    dspots[i] = ds;
  }
  std::vector<DevDirLight> ddirs(desc->num_directional_lights);
  for (uint32_t i = 0; i < desc->num_directional_lights; ++i) {
    const tpt_directional_light_desc& d = desc->directional_lights[i];
    const float len = std::sqrt(d.direction[0] * d.direction[0] + d.direction[1] * d.direction[1] +
                                d.direction[2] * d.direction[2]);
    const float r = 1.0f / len;  // glam normalize: v * (1 / length)
    DevDirLight dd{};
    for (int k = 0; k < 3; ++k) {
      dd.direction[k] = d.direction[k] * r;
      dd.color[k] = d.color[k];
    }
    dd.intensity = d.intensity;
    ddirs[i] = dd;
  }
  s->num_point_lights = desc->num_point_lights;
  s->num_spot_lights = desc->num_spot_lights;
  s->num_directional_lights = desc->num_directional_lights;

  // light tree: the caller's, or built here (builder.rs)
  std::vector<HostInstance> hinst(desc->num_instances);
  for (uint32_t i = 0; i < desc->num_instances; ++i) {
    const tpt_instance_desc& id = desc->instances[i];
    hinst[i] = HostInstance{id.mesh_index, id.material_index, id.local_to_world, id.world_to_local, id.normal_to_world};
  }
  if (desc->light_tree.nodes) {
    s->light_tree.nodes.resize(desc->light_tree.num_nodes);
    std::memcpy(s->light_tree.nodes.data(), desc->light_tree.nodes, desc->light_tree.num_nodes * 64);
    s->light_tree.root = desc->light_tree.root;
    const uint64_t nn = desc->light_tree.num_nodes;
    if (nn && s->light_tree.root >= nn) return set_error(ctx, TPT_ERR_INVALID_ARG, "light tree root out of range");
    for (uint64_t i = 0; i < nn; ++i) {
      const LightNodeHost& n = s->light_tree.nodes[i];
      const bool leaf = n.leaf_instance != kInvalidNode;
      if (leaf && (n.leaf_instance == kLeafPoint || n.leaf_instance == kLeafSpot)) {
        if (n.leaf_triangle >= (n.leaf_instance == kLeafPoint ? desc->num_point_lights : desc->num_spot_lights))
          return set_error(ctx, TPT_ERR_INVALID_ARG, "light tree leaf names an unknown point or spot light");
      } else if (leaf) {
        if (n.leaf_instance >= desc->num_instances ||
            n.leaf_triangle >= minfo[desc->instances[n.leaf_instance].mesh_index].num_tris)
          return set_error(ctx, TPT_ERR_INVALID_ARG, "light tree leaf names an unknown triangle");
      } else if (n.left >= nn || n.right >= nn) {
        return set_error(ctx, TPT_ERR_INVALID_ARG, "light tree child index out of range");
      }
      if (n.parent != kInvalidNode && n.parent >= nn) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad light tree parent");
    }
  } else if (desc->num_materials) {
    HostSceneView view{hmesh.data(), desc->num_meshes, hinst.data(), desc->num_instances, hmats.data(),
                       desc->num_materials, hpoints.data(), desc->num_point_lights, hspots.data(),
                       desc->num_spot_lights};
    build_light_tree_host(view, &s->light_tree);
  }

  // emitter map: per emissive instance, one slot per triangle
  std::vector<DevShadeInstance> sinst(desc->num_instances);
  uint32_t map_size = 0;
  for (uint32_t i = 0; i < desc->num_instances; ++i) {
    const tpt_instance_desc& id = desc->instances[i];
    DevShadeInstance d{};
    const float* w = id.local_to_world;
    const float cols[12] = {w[0], w[1], w[2], w[4], w[5], w[6], w[8], w[9], w[10], w[12], w[13], w[14]};
    std::memcpy(d.l2w, cols, sizeof cols);
    std::memcpy(d.n2w, id.normal_to_world, 36);
    d.mesh = id.mesh_index;
    d.material = id.material_index;
    d.leaf_base = kInvalidNode;
    if (desc->num_materials && hmats[id.material_index].may_emit()) {
      d.leaf_base = map_size;
      map_size += minfo[id.mesh_index].num_tris;
    }
    sinst[i] = d;
  }
  std::vector<uint32_t> emap(map_size, kInvalidNode);
  for (uint32_t k = 0; k < s->light_tree.nodes.size(); ++k) {
    const LightNodeHost& n = s->light_tree.nodes[k];
    if (n.leaf_instance == kInvalidNode || n.leaf_instance == kLeafPoint || n.leaf_instance == kLeafSpot) continue;
    const uint32_t base = sinst[n.leaf_instance].leaf_base;
    if (base != kInvalidNode) emap[base + n.leaf_triangle] = k;
  }
  // area-light registry (BDPT light subpaths) and its emitter-map index
  std::vector<HostAreaLight> hal;
  float al_sum = 0.0f;
  {
    HostSceneView view{hmesh.data(), desc->num_meshes, hinst.data(), desc->num_instances, hmats.data(),
                       desc->num_materials};
    if (desc->num_materials) register_area_lights(view, &hal, &al_sum);
  }
  std::vector<DevAreaLight> dal(hal.size());
  std::vector<uint32_t> al_of(map_size, kInvalidNode);
  for (size_t k = 0; k < hal.size(); ++k) {
    dal[k] = DevAreaLight{hal[k].inst, hal[k].tri, hal[k].area, hal[k].weight, hal[k].prefix_weight, {0, 0, 0}};
    const uint32_t base = sinst[hal[k].inst].leaf_base;
    if (base != kInvalidNode) al_of[base + hal[k].tri] = (uint32_t)k;
  }
  std::vector<DevLightNodeRec> lnodes(s->light_tree.nodes.size());
  if (!lnodes.empty()) std::memcpy(lnodes.data(), s->light_tree.nodes.data(), lnodes.size() * 64);

  DevRenderData& R = s->render;
  tpt_status st = TPT_OK;
  if (!st) st = put(s, sinst, &R.inst);
  if (!st) st = put(s, minfo, &R.meshes);
  if (!st) st = put(s, pos, &R.pos);
  if (!st) st = put(s, nrm, &R.nrm);
  if (!st) st = put(s, uv, &R.uv);
  if (!st) st = put(s, idx, &R.idx);
  if (!st) st = put(s, dmats, &R.mats);
  if (!st) st = put(s, lnodes, &R.ltree);
  if (!st) st = put(s, emap, &R.emitter_leaf);
  if (!st) st = put(s, opbr, &R.openpbr);
  if (!st) st = put(s, dal, &R.area_lights);
  if (!st) st = put(s, al_of, &R.area_light_of);
  if (!st) st = put(s, dpoints, &R.points);
  if (!st) st = put(s, dspots, &R.spots);
  if (!st) st = put(s, ddirs, &R.dirs);
  const float* d_alpha = nullptr;
  if (!st && !ialpha.empty()) st = put(s, ialpha, &d_alpha);
  if (st) return st;
  s->geo.inst_alpha = d_alpha;
  R.num_area_lights = (uint32_t)dal.size();
  R.area_light_weight_sum = al_sum;
  R.cec_e = ctx->d_cec_e;
  R.dec_e = ctx->d_dec_e;
  R.ltree_root = s->light_tree.root;
  R.num_materials = desc->num_materials;
  // the environment (EnvironmentLight::from_pixels): map and distributions
  R.has_env = 0;
  R.env = DevEnvironment{};
  EnvHost env;
  const tpt_environment_desc* ed = desc->environment;
  if (ed) {
    if (!ed->pixels || ed->width == 0 || ed->height == 0)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "environment map must be non-empty");
    build_environment(ed->width, ed->height, ed->pixels, ed->scale, ed->rotate_y, &env);
    std::vector<float> px(ed->pixels, ed->pixels + (size_t)ed->width * ed->height * 3);
    st = put(s, px, &R.env.pixels);
    if (!st) st = put(s, env.dist.weights, &R.env.dist.weights);
    if (!st) st = put(s, env.dist.levels, &R.env.dist.levels);
    if (!st) st = put(s, env.mis.weights, &R.env.mis.weights);
    if (!st) st = put(s, env.mis.levels, &R.env.mis.levels);
    if (st) return st;
    R.env.width = env.width;
    R.env.height = env.height;
    R.env.scale = env.scale;
    std::memcpy(R.env.rot, env.rot, sizeof env.rot);
    std::memcpy(R.env.inv_rot, env.inv_rot, sizeof env.inv_rot);
    R.env.dist.num_levels = (uint32_t)(env.dist.levels.size() / 3);
    R.env.dist.total_weight = env.dist.total_weight;
    R.env.mis.num_levels = (uint32_t)(env.mis.levels.size() / 3);
    R.env.mis.total_weight = env.mis.total_weight;
    R.has_env = 1;
  }
  // LightSampler::build_from_scene (light/mod.rs:134-188): the Tree category,
  // the Environment (weighted by its total power), then one per directional
  // light with luminance(color) * intensity > 0
  const float tree_w = lnodes.empty() ? 0.0f : std::fmax(lnodes[R.ltree_root].flux, 0.0f);
  R.has_tree = tree_w > 0.0f ? 1u : 0u;
  std::vector<uint32_t> kinds;
  std::vector<float> weights;
  if (tree_w > 0.0f) {
    kinds.push_back(kCatTree);
    weights.push_back(tree_w);
  }
  const float env_w = R.has_env ? std::fmax(env.total_power, 0.0f) : 0.0f;
  if (env_w > 0.0f) {
    kinds.push_back(kCatEnv);
    weights.push_back(env_w);
  }
  for (uint32_t i = 0; i < desc->num_directional_lights; ++i) {
    const DevDirLight& d = ddirs[i];
    const float w = std::fmax((0.2126f * d.color[0] + 0.7152f * d.color[1] + 0.0722f * d.color[2]) * d.intensity,
                              0.0f);
    if (w > 0.0f) {
      kinds.push_back(1u + i);
      weights.push_back(w);
    }
  }
  std::vector<float> cdf(1, 0.0f), pmf(weights.size());
  float total = 0.0f;
  for (float w : weights) {
    total += w;
    cdf.push_back(total);
  }
  if (total > 0.0f) {
    const float inv = 1.0f / total;
    for (float& c : cdf) c *= inv;
  }
  for (size_t k = 0; k < weights.size(); ++k) pmf[k] = total > 0.0f ? weights[k] / total : 0.0f;
  R.tree_cat_pmf = R.has_tree && total > 0.0f ? tree_w / total : 0.0f;
  R.env.cat_pmf = env_w > 0.0f && total > 0.0f ? env_w / total : 0.0f;  // LightSampler::category_pmf
  R.num_cat = total > 0.0f ? (uint32_t)kinds.size() : 0u;
  R.num_extra_lights =
      desc->num_point_lights + desc->num_spot_lights + desc->num_directional_lights + (R.has_env ? 1u : 0u);
  if (!st) st = put(s, cdf, &R.cat_cdf);
  if (!st) st = put(s, pmf, &R.cat_pmf);
  if (!st) st = put(s, kinds, &R.cat_kind);
  return st;
}

}  // namespace tpt

struct tpt_light_tree {
  tpt::LightTreeHost t;
};

extern "C" {

tpt_status tpt_light_tree_build(const tpt_scene_desc* desc, tpt_light_tree** out) {
  return tpt_light_tree_build_threads(desc, 0, out);
}

tpt_status tpt_light_tree_build_threads(const tpt_scene_desc* desc, int threads, tpt_light_tree** out) {
  using namespace tpt;
  if (!desc || !out) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if ((desc->num_meshes && !desc->meshes) || (desc->num_instances && !desc->instances) ||
      (desc->num_materials && !desc->materials))
    return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL array in scene description");
  std::vector<HostMaterial> hm(desc->num_materials);
  for (uint32_t i = 0; i < desc->num_materials; ++i) {
    if (desc->materials[i].kind == TPT_MATERIAL_OPENPBR && !desc->materials[i].openpbr)
      return set_error(nullptr, TPT_ERR_INVALID_ARG, "material " + std::to_string(i) + ": openpbr is NULL");
    hm[i] = host_material(desc->materials[i]);
  }
  std::vector<HostMesh> meshes(desc->num_meshes);
  for (uint32_t i = 0; i < desc->num_meshes; ++i) {
    const tpt_mesh_desc& md = desc->meshes[i];
    if (!md.positions || !md.indices || md.num_indices % 3)
      return set_error(nullptr, TPT_ERR_INVALID_ARG, "bad mesh " + std::to_string(i));
    for (uint64_t k = 0; k < md.num_indices; ++k)
      if (md.indices[k] >= md.num_vertices) return set_error(nullptr, TPT_ERR_INVALID_ARG, "index out of range");
    meshes[i] = HostMesh{md.positions, md.normals, md.uvs, md.indices, (uint32_t)md.num_vertices,
                         (uint32_t)(md.num_indices / 3)};
  }
  std::vector<HostInstance> inst(desc->num_instances);
  for (uint32_t i = 0; i < desc->num_instances; ++i) {
    const tpt_instance_desc& id = desc->instances[i];
    if (id.mesh_index >= desc->num_meshes || id.material_index >= desc->num_materials)
      return set_error(nullptr, TPT_ERR_INVALID_ARG, "instance " + std::to_string(i) + " references out of range");
    inst[i] = HostInstance{id.mesh_index, id.material_index, id.local_to_world, id.world_to_local, id.normal_to_world};
  }
  if ((desc->num_point_lights && !desc->point_lights) || (desc->num_spot_lights && !desc->spot_lights))
    return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL light array");
  std::vector<HostPointLight> points(desc->num_point_lights);
  for (uint32_t i = 0; i < desc->num_point_lights; ++i) {
    const tpt_point_light_desc& d = desc->point_lights[i];
    for (int k = 0; k < 3; ++k) {
      points[i].position[k] = d.position[k];
      points[i].color[k] = d.color[k];
    }
    points[i].intensity = d.intensity;
  }
  std::vector<HostSpotLight> spots(desc->num_spot_lights);
  for (uint32_t i = 0; i < desc->num_spot_lights; ++i) {
    const tpt_spot_light_desc& d = desc->spot_lights[i];
    make_spot_light(d.position, d.direction, d.color, d.intensity, d.total_width, d.falloff_start, &spots[i]);
  }
  auto* t = new tpt_light_tree();
  HostSceneView v{meshes.data(), desc->num_meshes, inst.data(), desc->num_instances, hm.data(), desc->num_materials,
                  points.data(), desc->num_point_lights, spots.data(), desc->num_spot_lights};
  if (!build_light_tree_host(v, &t->t, threads)) {
    delete t;
    return set_error(nullptr, TPT_ERR_INVALID_ARG, "no emitter with positive flux: build_light_tree returns None");
  }
  *out = t;
  return TPT_OK;
}

tpt_status tpt_light_tree_view_of(const tpt_light_tree* tree, tpt_light_tree_view* view) {
  if (!tree || !view) return tpt::set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  view->nodes = reinterpret_cast<const tpt_light_node*>(tree->t.nodes.data());
  view->num_nodes = tree->t.nodes.size();
  view->root = tree->t.root;
  return TPT_OK;
}

tpt_status tpt_light_tree_free(tpt_light_tree* tree) {
  delete tree;
  return TPT_OK;
}

}  // extern "C"
