// SPDX-License-Identifier: Apache-2.0
// CudaOffscreenRenderer over the C ABI; see the header for the mapping.
#include "cuda_offscreen_renderer.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <variant>

namespace lotus_cuda_host {

namespace {

Lotus::FrameStatus to_status(int32_t s) {
  return s == LOTUS_PASS ? Lotus::FrameStatus::Pass
                         : (s == LOTUS_SKIP ? Lotus::FrameStatus::Skip : Lotus::FrameStatus::Fail);
}

// Column-major 4x4 product a * b.
Lotus::Matrix4 multiply(const Lotus::Matrix4& a, const Lotus::Matrix4& b) {
  Lotus::Matrix4 m{};
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) {
      float s = 0.0f;
      for (int k = 0; k < 4; ++k) s += a[k * 4 + r] * b[c * 4 + k];
      m[c * 4 + r] = s;
    }
  return m;
}

// The sRGB transfer function's inverse (IEC 61966-2-1).
float srgb_to_linear(float c) {
  return c <= 0.04045f ? c / 12.92f : std::pow((c + 0.055f) / 1.055f, 2.4f);
}

// A texture's texels as linear RGBA floats.
std::vector<float> texels_rgba32f(const Lotus::Texture& t) {
  const size_t n = (size_t)t.width * t.height;
  std::vector<float> out(4 * n, 0.0f);
  if (t.format == Lotus::TextureFormat::Rgba32Float) {
    std::memcpy(out.data(), t.texels.data(), std::min(t.texels.size(), out.size() * sizeof(float)));
    return out;
  }
  const bool srgb = t.format == Lotus::TextureFormat::Rgba8Srgb;
  for (size_t i = 0; i < n && 4 * i + 3 < t.texels.size(); ++i)
    for (int c = 0; c < 4; ++c) {
      const float v = t.texels[4 * i + c] / 255.0f;
      out[4 * i + c] = (srgb && c < 3) ? srgb_to_linear(v) : v;
    }
  return out;
}

}  // namespace

std::unique_ptr<Lotus::OffscreenRenderer> CudaOffscreenRenderer::Create(int device, Lotus::FrameStatus& status,
    std::string& error) {
  lotus_cuda_options options{};
  options.device = device;
  lotus_cuda_renderer* handle = nullptr;
  char detail[256] = {};
  const int32_t s = lotus_cuda_create(&options, &handle, detail, sizeof(detail));
  status = to_status(s);
  if (s != LOTUS_PASS) {
    error = detail;
    return nullptr;
  }
  error.clear();
  return std::unique_ptr<Lotus::OffscreenRenderer>(new CudaOffscreenRenderer(device, handle));
}

CudaOffscreenRenderer::~CudaOffscreenRenderer() {
  if (handle_) lotus_cuda_destroy(handle_);
}

Lotus::GpuFrameEvidence CudaOffscreenRenderer::Render(const Lotus::DrawSummary&, const Lotus::OffscreenTarget&,
    std::uint32_t) {
  Lotus::GpuFrameEvidence e;
  e.status = Lotus::FrameStatus::Skip;
  e.detail = "the bootstrap raster draw is not part of the CUDA integrator backend";
  return e;
}

Lotus::BackendCapability CudaOffscreenRenderer::RayQueryCapability() const {
  char detail[256] = {};
  Lotus::BackendCapability c;
  c.available = lotus_cuda_capability(device_, detail, sizeof(detail)) == LOTUS_PASS;
  c.detail = detail;
  return c;
}

Lotus::GpuSceneEvidence CudaOffscreenRenderer::UpdateScene(const Lotus::SceneUpdate& u) {
  Lotus::GpuSceneEvidence ev;
  auto fail = [&](const std::string& why) {
    ev.status = Lotus::FrameStatus::Fail;
    ev.detail = why;
    failed_ = true;
    failure_ = why;
    return ev;
  };
  if (failed_) return fail("the renderer has failed: " + failure_);
  // An empty plan records no GPU work (vulkan_backend.hpp:812-815).
  if (u.geometry_releases.empty() && u.geometry_uploads.empty() && u.texture_releases.empty() &&
      u.texture_uploads.empty() && !u.instances_changed && !u.materials_changed && !u.environment_changed &&
      !u.lights_changed) {
    ev.status = Lotus::FrameStatus::Pass;
    return ev;
  }
  if (UpdateIncrementally(u, ev)) return ev;
  // Releases, then uploads (extraction.hpp:95-106).
  auto drop = [](auto& list, const void* p) {
    list.erase(std::remove_if(list.begin(), list.end(), [&](const auto& s) { return s.get() == p; }), list.end());
  };
  for (const Lotus::MeshGeometry* g : u.geometry_releases) drop(geometries_, g);
  for (const Lotus::Texture* t : u.texture_releases) drop(textures_, t);
  for (const auto& g : u.geometry_uploads) geometries_.push_back(g);
  for (const auto& t : u.texture_uploads) textures_.push_back(t);
  if (u.instances_changed) instances_ = u.instances;
  if (u.materials_changed) materials_ = u.materials;
  if (u.environment_changed) {
    environment_ = u.environment;
    environment_map_ = u.environment_map;
  }
  if (u.lights_changed) lights_ = u.lights;

  // The scene description, rebuilt whole.
  std::vector<lotus_geometry> geos(geometries_.size());
  std::vector<std::vector<float>> positions(geometries_.size()), normals(geometries_.size()),
      texcoords(geometries_.size()), colors(geometries_.size());
  std::vector<std::vector<uint32_t>> triangles(geometries_.size()), color_counts(geometries_.size());
  for (size_t g = 0; g < geometries_.size(); ++g) {
    const Lotus::MeshGeometry& m = *geometries_[g];
    positions[g].reserve(3 * m.positions.size());
    for (const auto& p : m.positions) positions[g].insert(positions[g].end(), p.begin(), p.end());
    triangles[g].reserve(3 * m.triangles.size());
    for (const auto& t : m.triangles) triangles[g].insert(triangles[g].end(), t.begin(), t.end());
    if (!m.normals.empty()) {
      if (m.normals.size() != 3 * m.triangles.size()) return fail("shading normals must be one per triangle corner");
      for (const auto& n : m.normals) normals[g].insert(normals[g].end(), n.begin(), n.end());
    }
    geos[g].positions = positions[g].data();
    geos[g].triangles = triangles[g].data();
    geos[g].normals = normals[g].empty() ? nullptr : normals[g].data();
    geos[g].vertex_count = (uint32_t)m.positions.size();
    geos[g].triangle_count = (uint32_t)m.triangles.size();
    // Texture-coordinate sets in key order, one (s, t) per triangle corner.
    for (const auto& [name, set] : m.texcoords) {
      if (set.size() != 3 * m.triangles.size())
        return fail("texture coordinates must be one per triangle corner (set " + name + ")");
      for (const auto& st : set) texcoords[g].insert(texcoords[g].end(), st.begin(), st.end());
    }
    geos[g].texcoords = texcoords[g].empty() ? nullptr : texcoords[g].data();
    geos[g].texcoord_sets = texcoords[g].empty() ? 0u : (uint32_t)m.texcoords.size();
    // Colour sets in key order: one RGB per triangle corner, or one for the
    // mesh (MeshGeometry::colors, render_world.hpp:52-55).
    for (const auto& [name, set] : m.colors) {
      if (set.size() != 1 && set.size() != 3 * m.triangles.size())
        return fail("colours must be one per triangle corner or one per mesh (set " + name + ")");
      for (const auto& c : set) colors[g].insert(colors[g].end(), c.begin(), c.end());
      color_counts[g].push_back((uint32_t)set.size());
    }
    geos[g].color_sets = (uint32_t)color_counts[g].size();
    geos[g].colors = colors[g].empty() ? nullptr : colors[g].data();
    geos[g].color_counts = color_counts[g].empty() ? nullptr : color_counts[g].data();
  }
  // Every resident texture (TextureFormat, material.hpp:15-23), counted
  // from 1 by the lookups that name it.
  std::vector<lotus_texture> texs(textures_.size());
  std::unordered_map<const Lotus::Texture*, uint32_t> texture_ref;
  for (size_t i = 0; i < textures_.size(); ++i) {
    const Lotus::Texture& t = *textures_[i];
    if (t.texels.size() != (size_t)t.width * t.height * Lotus::TexelBytes(t.format))
      return fail("texture " + std::to_string(i) + " has the wrong number of texel bytes");
    texs[i].texels = t.texels.data();
    texs[i].width = t.width;
    texs[i].height = t.height;
    texs[i].format = t.format == Lotus::TextureFormat::Rgba8Srgb     ? LOTUS_TEXTURE_RGBA8_SRGB
                     : t.format == Lotus::TextureFormat::Rgba32Float ? LOTUS_TEXTURE_RGBA32_FLOAT
                                                                     : LOTUS_TEXTURE_RGBA8_UNORM;
    texture_ref[&t] = (uint32_t)i + 1;
  }
  std::vector<lotus_texture_input> inputs;
  std::vector<lotus_material> mats(std::max<size_t>(materials_.size(), 1));
  for (size_t i = 0; i < materials_.size(); ++i) {
    const Lotus::SceneMaterial& sm = materials_[i];
    const auto* preview = std::get_if<Lotus::PreviewSurface>(&sm.material.surface);
    const auto* gltf = std::get_if<Lotus::GltfPbr>(&sm.material.surface);
    if (!preview && !gltf)
      return fail("material " + std::to_string(i) + ": only UsdPreviewSurface and glTF PBR are built");
    lotus_material& m = mats[i];
    // Each texture-input slot (material.hpp:262-312) with its resolved
    // image (SceneMaterial::textures; none: the lookup's fallback).
    const std::optional<Lotus::TextureInput>* slots[LOTUS_TEXTURE_SLOTS] = {};
    slots[LOTUS_SLOT_OPACITY] = &sm.material.geometry.opacity_texture;
    slots[LOTUS_SLOT_NORMAL] = &sm.material.geometry.normal_texture;
    if (preview) {
      slots[LOTUS_SLOT_BASE_COLOR] = &preview->base_color_texture;
      slots[LOTUS_SLOT_ROUGHNESS] = &preview->roughness_texture;
      slots[LOTUS_SLOT_METALLIC] = &preview->metallic_texture;
      slots[LOTUS_SLOT_EMISSION] = &preview->emission_texture;
      slots[LOTUS_SLOT_SPECULAR_COLOR] = &preview->specular_color_texture;
    } else {
      slots[LOTUS_GLTF_SLOT_BASE_COLOR] = &gltf->base_color.texture;
      slots[LOTUS_GLTF_SLOT_METALLIC] = &gltf->metallic.texture;
      slots[LOTUS_GLTF_SLOT_ROUGHNESS] = &gltf->roughness.texture;
      slots[LOTUS_GLTF_SLOT_EMISSIVE] = &gltf->emissive.texture;
      slots[LOTUS_GLTF_SLOT_SPECULAR] = &gltf->specular.texture;
      slots[LOTUS_GLTF_SLOT_SPECULAR_COLOR] = &gltf->specular_color.texture;
      slots[LOTUS_GLTF_SLOT_TRANSMISSION] = &gltf->transmission.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT] = &gltf->clearcoat.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT_ROUGHNESS] = &gltf->clearcoat_roughness.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL] = &gltf->clearcoat_normal_texture;
      slots[LOTUS_GLTF_SLOT_SHEEN_COLOR] = &gltf->sheen_color.texture;
      slots[LOTUS_GLTF_SLOT_SHEEN_ROUGHNESS] = &gltf->sheen_roughness.texture;
    }
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k) {
      if (!slots[k] || !*slots[k]) continue;
      const Lotus::TextureInput& in = **slots[k];
      lotus_texture_input d{};
      const Lotus::Texture* image = k < sm.textures.size() ? sm.textures[k] : nullptr;
      const auto ref = image ? texture_ref.find(image) : texture_ref.end();
      d.texture = ref == texture_ref.end() ? LOTUS_NO_TEXTURE : ref->second;
      d.channel = in.channel;
      d.wrap_s = (uint32_t)in.wrap_s;
      d.wrap_t = (uint32_t)in.wrap_t;
      std::memcpy(d.scale, in.scale.data(), 16);
      std::memcpy(d.bias, in.bias.data(), 16);
      std::memcpy(d.fallback, in.fallback.data(), 16);
      std::memcpy(d.st_transform, in.st_transform.data(), 24);
      inputs.push_back(d);
      m.lookups[k] = (uint32_t)inputs.size();
    }
    std::memcpy(m.texcoord_fallback, sm.material.geometry.texcoord_fallback.data(), 8);
    std::memcpy(m.normal, sm.material.geometry.normal.data(), 12);
    m.opacity = sm.material.geometry.opacity;
    m.opacity_threshold = sm.material.geometry.opacity_threshold;
    if (gltf) {
      m.model = LOTUS_MODEL_GLTF_PBR;
      std::memcpy(m.base_color, gltf->base_color.value.data(), 12);
      m.metallic = gltf->metallic.value;
      m.roughness = gltf->roughness.value;
      std::memcpy(m.emission, gltf->emissive.value.data(), 12);
      m.emissive_strength = gltf->emissive_strength;
      m.ior = gltf->ior;
      m.specular = gltf->specular.value;
      std::memcpy(m.specular_color, gltf->specular_color.value.data(), 12);
      m.transmission = gltf->transmission.value;
      m.clearcoat = gltf->clearcoat.value;
      m.clearcoat_roughness = gltf->clearcoat_roughness.value;
      std::memcpy(m.sheen_color, gltf->sheen_color.value.data(), 12);
      m.sheen_roughness = gltf->sheen_roughness.value;
      continue;
    }
    const Lotus::PreviewSurface& p = *preview;
    std::memcpy(m.base_color, p.base_color.data(), 12);
    m.roughness = p.roughness;
    std::memcpy(m.emission, p.emission.data(), 12);
    m.metallic = p.metallic;
    std::memcpy(m.specular_color, p.specular_color.data(), 12);
    m.ior = p.ior;
    std::memcpy(m.transmission_color, p.transmission_color.data(), 12);
    m.transmission = p.transmission;
    m.flags = (p.use_specular_workflow ? LOTUS_MATERIAL_SPECULAR_WORKFLOW : 0u) |
              (p.thin_walled ? LOTUS_MATERIAL_THIN_WALLED : 0u);
  }
  if (materials_.empty()) {
    // A GPU scene starts with the default material alone (extraction.hpp).
    const Lotus::PreviewSurface p;
    std::memcpy(mats[0].base_color, p.base_color.data(), 12);
    mats[0].roughness = p.roughness;
    mats[0].ior = p.ior;
    mats[0].transmission_color[0] = mats[0].transmission_color[1] = mats[0].transmission_color[2] = 1.0f;
    mats[0].opacity = 1.0f;
  }
  std::vector<lotus_instance> insts;
  {
    std::string error;
    if (!InstanceArray(insts, error)) return fail(error);
  }
  lotus_environment env{};
  std::vector<float> env_texels;
  if (environment_map_ && environment_map_->texture) {
    const Lotus::Texture& t = *environment_map_->texture;
    env_texels = texels_rgba32f(t);
    env.texels = env_texels.data();
    env.width = t.width;
    env.height = t.height;
    std::memcpy(env.scale, environment_map_->scale.data(), 12);
    // Rows: the image frame's unit axes in world space, the columns of
    // world_from_environment's linear part.
    const Lotus::Matrix4& w = environment_map_->world_from_environment;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) env.environment_from_world[3 * r + c] = w[4 * r + c];
  }
  // The analytic lights (render_world.hpp:79-114), field for field.
  std::vector<lotus_light> lights(lights_.size());
  for (size_t i = 0; i < lights_.size(); ++i) {
    const Lotus::Light& l = lights_[i];
    lotus_light& d = lights[i];
    d.shape = l.shape == Lotus::LightShape::Sphere ? LOTUS_LIGHT_SPHERE
              : l.shape == Lotus::LightShape::Rect ? LOTUS_LIGHT_RECT
              : l.shape == Lotus::LightShape::Disk ? LOTUS_LIGHT_DISK
                                                   : LOTUS_LIGHT_DISTANT;
    d.normalize = l.normalize ? 1u : 0u;
    std::memcpy(d.world_from_light, l.world_from_light.data(), 64);
    std::memcpy(d.radiance, l.radiance.data(), 12);
    d.radius = l.radius;
    d.width = l.width;
    d.height = l.height;
    d.angle = l.angle;
  }
  lotus_scene_desc desc{};
  desc.lights = lights.empty() ? nullptr : lights.data();
  desc.light_count = (uint32_t)lights.size();
  desc.geometries = geos.data();
  desc.instances = insts.data();
  desc.materials = mats.data();
  desc.environment = env.texels ? &env : nullptr;
  desc.geometry_count = (uint32_t)geos.size();
  desc.instance_count = (uint32_t)insts.size();
  desc.material_count = (uint32_t)mats.size();
  desc.textures = texs.empty() ? nullptr : texs.data();
  desc.texture_count = (uint32_t)texs.size();
  desc.texture_inputs = inputs.empty() ? nullptr : inputs.data();
  desc.texture_input_count = (uint32_t)inputs.size();
  std::memcpy(desc.environment_constant, environment_.data(), 12);
  lotus_scene_result res{};
  const int32_t s = lotus_cuda_update_scene(handle_, &desc, &res);
  ev.status = to_status(s);
  ev.detail = res.detail;
  if (s != LOTUS_PASS) {
    failed_ = true;
    failure_ = ev.detail;
    return ev;
  }
  resident_ = true;
  device_bytes_ = res.device_bytes;
  material_slots_ = (uint32_t)mats.size();
  environment_map_bound_ = env.texels != nullptr;
  SceneStats(u, res, ev);
  return ev;
}

void CudaOffscreenRenderer::SceneStats(const Lotus::SceneUpdate& u, const lotus_scene_result& res,
    Lotus::GpuSceneEvidence& ev) const {
  ev.stats.source_revision = u.source_revision;
  ev.stats.resident_geometries = (uint32_t)geometries_.size();
  ev.stats.instance_count = res.instance_count;
  ev.stats.material_count = material_slots_;
  ev.stats.environment_map = environment_map_bound_;
  ev.stats.resident_textures = (uint32_t)textures_.size();
  ev.stats.acceleration_available = true;
  ev.stats.blas_count = (uint32_t)geometries_.size();
  ev.stats.tlas_instance_count = res.instance_count;
  ev.timings.available = true;
  ev.timings.blas_build_gpu_ms = res.build_gpu_ms;
}

// The resident instances in the C ABI's form: geometry slots are the
// positions in geometries_.
bool CudaOffscreenRenderer::InstanceArray(std::vector<lotus_instance>& insts, std::string& error) const {
  std::unordered_map<const Lotus::MeshGeometry*, uint32_t> slot;
  for (size_t g = 0; g < geometries_.size(); ++g) slot[geometries_[g].get()] = (uint32_t)g;
  insts.assign(instances_.size(), lotus_instance{});
  for (size_t i = 0; i < instances_.size(); ++i) {
    const Lotus::SceneInstance& si = instances_[i];
    const auto it = slot.find(si.geometry);
    if (it == slot.end()) {
      error = "instance " + std::to_string(i) + " names a geometry that is not resident";
      return false;
    }
    std::memcpy(insts[i].world_from_object, si.world_from_object.data(), 64);
    insts[i].geometry = it->second;
    insts[i].material = si.material;
    // The set its material's lookups read, counted from 1 (0: none).
    insts[i].texcoord_set = si.texcoords == Lotus::kNoTexcoords ? LOTUS_NO_TEXCOORDS : si.texcoords + 1;
    insts[i].color_set = si.colors == Lotus::kNoColors ? LOTUS_NO_COLORS : si.colors + 1;
  }
  return true;
}

bool CudaOffscreenRenderer::UpdateIncrementally(const Lotus::SceneUpdate& u, Lotus::GpuSceneEvidence& ev) {
  if (!resident_ || !u.texture_releases.empty() || !u.texture_uploads.empty() || u.materials_changed ||
      u.environment_changed || u.lights_changed)
    return false;
  // Every release and upload must be one side of a replacement whose
  // topology (vertex count, triangles, presence of corner normals) is kept.
  if (u.geometry_releases.size() != u.geometry_replacements.size() ||
      u.geometry_uploads.size() != u.geometry_replacements.size())
    return false;
  std::vector<std::pair<size_t, std::shared_ptr<const Lotus::MeshGeometry>>> edits;
  for (const Lotus::SceneGeometryReplacement& r : u.geometry_replacements) {
    size_t at = geometries_.size();
    for (size_t g = 0; g < geometries_.size(); ++g)
      if (geometries_[g].get() == r.previous) at = g;
    std::shared_ptr<const Lotus::MeshGeometry> next;
    for (const auto& up : u.geometry_uploads)
      if (up.get() == r.replacement) next = up;
    if (at == geometries_.size() || !next || !r.previous) return false;
    const Lotus::MeshGeometry& a = *r.previous;
    const Lotus::MeshGeometry& b = *next;
    if (a.positions.size() != b.positions.size() || a.triangles != b.triangles ||
        a.normals.empty() != b.normals.empty() || (!b.normals.empty() && b.normals.size() != 3 * b.triangles.size()) ||
        a.texcoords != b.texcoords || a.colors != b.colors)
      return false;
    edits.emplace_back(at, next);
  }
  if (edits.empty() && !u.instances_changed) return false;
  auto fail = [&](const lotus_scene_result& res, int32_t s) {
    ev.status = to_status(s);
    ev.detail = res.detail;
    failed_ = true;
    failure_ = ev.detail;
    return true;
  };
  lotus_scene_result res{};
  for (const auto& [at, next] : edits) {
    std::vector<float> positions, normals;
    positions.reserve(3 * next->positions.size());
    for (const auto& p : next->positions) positions.insert(positions.end(), p.begin(), p.end());
    for (const auto& n : next->normals) normals.insert(normals.end(), n.begin(), n.end());
    const int32_t s = lotus_cuda_update_geometry(handle_, (uint32_t)at, positions.data(),
        (uint32_t)next->positions.size(), normals.empty() ? nullptr : normals.data(), &res);
    if (s != LOTUS_PASS) return fail(res, s);
    geometries_[at] = next;
  }
  if (u.instances_changed) {
    instances_ = u.instances;
    std::vector<lotus_instance> insts;
    std::string error;
    if (!InstanceArray(insts, error)) {
      ev.status = Lotus::FrameStatus::Fail;
      ev.detail = error;
      failed_ = true;
      failure_ = error;
      return true;
    }
    const int32_t s = lotus_cuda_update_instances(handle_, insts.data(), (uint32_t)insts.size(), &res);
    if (s != LOTUS_PASS) return fail(res, s);
  }
  ev.status = Lotus::FrameStatus::Pass;
  device_bytes_ = res.device_bytes;
  SceneStats(u, res, ev);
  return true;
}

bool CudaOffscreenRenderer::FillFrame(const Lotus::Matrix4& world_to_clip, const Lotus::OffscreenTarget& t,
    std::uint32_t frame_count, const Lotus::PathTracingSettings& s, lotus_frame_desc& f, std::string& error) const {
  f = lotus_frame_desc{};
  switch (s.output) {
    case Lotus::SceneOutput::Radiance: f.settings.output = LOTUS_OUTPUT_RADIANCE; break;
    case Lotus::SceneOutput::Barycentrics: f.settings.output = LOTUS_OUTPUT_BARYCENTRICS; break;
    case Lotus::SceneOutput::ShadingNormal: f.settings.output = LOTUS_OUTPUT_SHADING_NORMAL; break;
    case Lotus::SceneOutput::Albedo: f.settings.output = LOTUS_OUTPUT_ALBEDO; break;
    case Lotus::SceneOutput::RoughnessMetallic: f.settings.output = LOTUS_OUTPUT_ROUGHNESS_METALLIC; break;
    default:
      error = "unknown scene output";
      return false;
  }
  std::memcpy(f.world_to_clip, world_to_clip.data(), 64);
  f.target.width = t.width;
  f.target.height = t.height;
  std::memcpy(f.target.display_window, t.display_window.data(), 16);
  std::memcpy(f.target.data_window, t.data_window.data(), 16);
  std::memcpy(f.target.clear_color, t.clear_color.data(), 16);
  f.target.read_back = t.read_back ? 1u : 0u;
  f.target.clear_depth = t.clear_depth;
  f.settings.integrator =
      s.integrator == Lotus::Integrator::Wavefront ? LOTUS_INTEGRATOR_WAVEFRONT : LOTUS_INTEGRATOR_REFERENCE;
  f.settings.light_sampling = s.light_sampling == Lotus::LightSampling::Bsdf ? LOTUS_LIGHT_SAMPLING_BSDF
                              : s.light_sampling == Lotus::LightSampling::Mis ? LOTUS_LIGHT_SAMPLING_MIS
                                                                              : LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL;
  f.settings.sample_index = s.sample_index;
  f.settings.max_bounces = s.max_bounces;
  f.settings.max_samples = s.max_samples;
  f.settings.restir_candidates = s.restir_candidates;
  f.settings.restir_temporal = s.restir_temporal ? 1u : 0u;
  f.settings.restir_max_history_candidates = s.restir_max_history_candidates;
  f.settings.restir_spatial = s.restir_spatial ? 1u : 0u;
  f.settings.restir_spatial_radius = s.restir_spatial_radius;
  f.settings.restir_proposal = (uint32_t)s.restir_proposal;
  f.settings.environment_background = s.environment_background ? 1u : 0u;
  f.frame_count = frame_count;
  // Every scene frame writes the camera pass's D32 depth, as the
  // reference's does (vulkan_backend.hpp:769-773).
  f.flags = LOTUS_FRAME_TIMINGS | LOTUS_FRAME_DEPTH | (t.clear_depth_enabled ? 0u : LOTUS_FRAME_DEPTH_KEEP);
  return true;
}

void CudaOffscreenRenderer::FillEvidence(const lotus_frame_desc& f, const lotus_frame_result& r,
    std::vector<float>& color, Lotus::GpuFrameEvidence& e) {
  e.status = to_status(r.status);
  e.detail = r.detail;
  e.completion = r.completion;
  e.frames_rendered = r.frames_rendered;
  e.samples_per_pixel = r.samples_per_pixel;
  e.primary_ray_timestamp_available = true;
  e.primary_ray_gpu_ms = r.gpu_ms;
  e.wavefront_rounds = r.wavefront_rounds;
  e.wavefront_path_counts.assign(r.wavefront_path_counts,
      r.wavefront_path_counts + std::min<uint32_t>(r.wavefront_path_count_size, LOTUS_MAX_REPORTED_BOUNCES));
  e.wavefront_timings.available = r.timings_available != 0;
  e.wavefront_timings.camera_gpu_ms = r.camera_gpu_ms;
  e.wavefront_timings.intersect_gpu_ms = r.extend_gpu_ms;
  e.wavefront_timings.shade_gpu_ms = r.shade_gpu_ms + r.shadow_gpu_ms;
  e.wavefront_timings.tail_gpu_ms = r.tail_gpu_ms;
  if (r.status == LOTUS_PASS && f.target.read_back) {
    // RGBA32F, top-left rows, linear (vulkan_backend.hpp:30-38).
    Lotus::ColorProduct& c = e.color;
    c.width = f.target.width;
    c.height = f.target.height;
    c.row_pitch = f.target.width * 16;
    c.pixel_format = "rgba32-sfloat";
    c.origin = "top-left";
    c.color_space = "linear";
    c.payload.resize(color.size() * sizeof(float));
    std::memcpy(c.payload.data(), color.data(), c.payload.size());
    // D32 window depth, top-left rows (vulkan_backend.hpp:40-47, 1318-1324).
    if (f.flags & LOTUS_FRAME_DEPTH) {
      Lotus::DepthProduct& d = e.depth;
      d.payload.resize((size_t)f.target.width * f.target.height);
      if (lotus_cuda_read_depth(handle_, d.payload.data(), d.payload.size()) == LOTUS_PASS) {
        d.width = f.target.width;
        d.height = f.target.height;
        d.row_pitch = f.target.width * sizeof(float);
        d.pixel_format = "d32-sfloat";
        d.origin = "top-left";
      } else {
        d.payload.clear();
      }
    }
  }
}

Lotus::GpuFrameEvidence CudaOffscreenRenderer::RenderScene(const Lotus::DrawSummary& draw,
    const Lotus::OffscreenTarget& target, std::uint32_t frame_count, const Lotus::PathTracingSettings& settings) {
  Lotus::GpuFrameEvidence e;
  lotus_frame_desc f;
  std::string error;
  if (!FillFrame(draw.world_to_clip, target, frame_count, settings, f, error)) {
    e.status = Lotus::FrameStatus::Fail;
    e.detail = error;
    return e;
  }
  std::vector<float> color(target.read_back ? (size_t)target.width * target.height * 4 : 0);
  lotus_frame_result r{};
  lotus_cuda_render(handle_, &f, &r, color.empty() ? nullptr : color.data());
  FillEvidence(f, r, color, e);
  return e;
}

Lotus::GpuFrameEvidence CudaOffscreenRenderer::RenderTemporalScene(const Lotus::FrameSnapshot& snapshot,
    const Lotus::OffscreenTarget& target, std::uint32_t frame_count, const Lotus::TemporalFrameSettings& temporal,
    const Lotus::PathTracingSettings& settings) {
  Lotus::GpuFrameEvidence e;
  lotus_temporal_desc d{};
  std::string error;
  const Lotus::Matrix4 world_to_clip = multiply(snapshot.camera.projection, snapshot.camera.view);
  if (!FillFrame(world_to_clip, target, frame_count, settings, d.frame, error)) {
    e.status = Lotus::FrameStatus::Fail;
    e.detail = error;
    return e;
  }
  // The stream's history: the preceding frame's camera unless this frame is
  // a cut.
  const bool history = have_previous_camera_ && !temporal.camera_cut;
  const Lotus::Camera& prev = history ? previous_camera_ : snapshot.camera;
  std::memcpy(d.current_view, snapshot.camera.view.data(), 64);
  std::memcpy(d.previous_view, prev.view.data(), 64);
  const Lotus::Matrix4 prev_clip = multiply(prev.projection, prev.view);
  std::memcpy(d.previous_world_to_clip, prev_clip.data(), 64);
  d.validation[0] = temporal.validation.absolute_depth_tolerance;
  d.validation[1] = temporal.validation.relative_depth_tolerance;
  d.validation[2] = temporal.validation.minimum_normal_cosine;
  d.validation[3] = temporal.validation.max_motion_pixels;
  d.history_available = history ? 1u : 0u;
  d.accumulate_radiance = temporal.accumulate_radiance ? 1u : 0u;
  d.max_history_samples = temporal.max_history_samples;
  d.filter_iterations = temporal.filter_iterations;
  d.history_rectification = (uint32_t)temporal.history_rectification;
  std::vector<float> color(target.read_back ? (size_t)target.width * target.height * 4 : 0);
  lotus_frame_result r{};
  lotus_cuda_render_temporal(handle_, &d, &r, color.empty() ? nullptr : color.data());
  FillEvidence(d.frame, r, color, e);
  if (r.status == LOTUS_PASS) {
    FillTemporalProducts(d, history, have_previous_camera_ && temporal.camera_cut, e);
    // Only success advances history (vulkan_backend.hpp:793-806).
    previous_camera_ = snapshot.camera;
    have_previous_camera_ = true;
  }
  return e;
}

namespace {

static_assert(sizeof(Lotus::TemporalPixel) == 64, "the surface product is 64 bytes per pixel");
static_assert(sizeof(Lotus::TemporalValidityPixel) == 16, "the validity product is 16 bytes per pixel");
static_assert(sizeof(Lotus::TemporalRadiancePixel) == 32, "the radiance product is 32 bytes per pixel");
static_assert(sizeof(Lotus::RestirPixel) == 48, "the initial reservoirs are 48 bytes per pixel");
static_assert(sizeof(Lotus::RestirReusePixel) == 64, "the reuse records are 64 bytes per pixel");

// One product into `out` (the C ABI's byte layout is the reference's type's);
// empty when the frame has no such product.
template <typename T>
void read_product(lotus_cuda_renderer* handle, uint32_t product, size_t pixels, std::vector<T>& out) {
  out.resize(pixels);
  const int64_t got = lotus_cuda_read_product(handle, product, out.data(), pixels * sizeof(T));
  out.resize(got > 0 ? (size_t)got / sizeof(T) : 0);
}

}  // namespace

void CudaOffscreenRenderer::FillTemporalProducts(const lotus_temporal_desc& d, bool history, bool camera_cut,
    Lotus::GpuFrameEvidence& e) {
  const uint32_t w = d.frame.target.width, h = d.frame.target.height;
  const size_t n = (size_t)w * h;
  Lotus::TemporalProducts& t = e.temporal;
  t.available = true;
  t.history_available = history;
  t.reset_reason = history ? Lotus::TemporalResetReason::None
                           : (camera_cut ? Lotus::TemporalResetReason::CameraCut
                                         : Lotus::TemporalResetReason::FirstFrame);
  t.width = w;
  t.height = h;
  t.row_pitch = w * (uint32_t)sizeof(Lotus::TemporalPixel);
  read_product(handle_, LOTUS_PRODUCT_SURFACE, n, t.current);
  if (history) read_product(handle_, LOTUS_PRODUCT_PREVIOUS_SURFACE, n, t.previous);
  read_product(handle_, LOTUS_PRODUCT_VALIDITY, n, t.validity);
  t.validity_row_pitch = w * (uint32_t)sizeof(Lotus::TemporalValidityPixel);
  if (d.accumulate_radiance) {
    t.radiance_available = true;
    read_product(handle_, LOTUS_PRODUCT_RADIANCE, n, t.radiance);
    if (history) read_product(handle_, LOTUS_PRODUCT_PREVIOUS_RADIANCE, n, t.previous_radiance);
    t.radiance_row_pitch = w * (uint32_t)sizeof(Lotus::TemporalRadiancePixel);
    read_product(handle_, LOTUS_PRODUCT_BATCH, n, t.batch);
    t.batch_sample_index = d.frame.settings.sample_index;
    t.batch_samples = d.frame.frame_count;
    t.filter_iterations = d.filter_iterations;
  }
  if (d.frame.settings.light_sampling != LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL) return;
  Lotus::RestirProducts& r = e.restir;
  r.available = true;
  r.width = w;
  r.height = h;
  r.row_pitch = w * (uint32_t)sizeof(Lotus::RestirPixel);
  read_product(handle_, LOTUS_PRODUCT_RESTIR_INITIAL, n, r.initial);
  if (d.frame.settings.restir_temporal) {
    r.temporal_row_pitch = w * (uint32_t)sizeof(Lotus::RestirReusePixel);
    read_product(handle_, LOTUS_PRODUCT_RESTIR_TEMPORAL, n, r.temporal);
    read_product(handle_, LOTUS_PRODUCT_RESTIR_PREVIOUS, n, r.previous);
    r.history_available = history && !r.previous.empty();
  }
  if (d.frame.settings.restir_spatial) {
    r.spatial_row_pitch = w * (uint32_t)sizeof(Lotus::RestirReusePixel);
    read_product(handle_, LOTUS_PRODUCT_RESTIR_SPATIAL, n, r.spatial);
    read_product(handle_, LOTUS_PRODUCT_RESTIR_SOURCES, n, r.spatial_sources);
  }
}

// ReadBackScene (vulkan_backend.hpp:819-821): the resident scene as the
// device holds it, through lotus_cuda_read_scene, decoded into the
// reference's contents. The CUDA backend keeps no texture-coordinate or
// colour sets and no textures, so those stay empty.
Lotus::GpuSceneContents CudaOffscreenRenderer::ReadBackScene() {
  Lotus::GpuSceneContents c;
  auto fail = [&](const std::string& d) {
    c = Lotus::GpuSceneContents{};
    c.status = Lotus::FrameStatus::Fail;
    c.detail = d;
    return c;
  };
  if (failed_) return fail("the renderer failed earlier: " + failure_);
  c.status = Lotus::FrameStatus::Pass;
  if (!resident_) return c;
  auto read = [&](uint32_t what, uint32_t index, std::vector<unsigned char>& out) {
    const int64_t n = lotus_cuda_read_scene(handle_, what, index, nullptr, 0);
    if (n < 0) return false;
    out.resize((size_t)n);
    return n == 0 || lotus_cuda_read_scene(handle_, what, index, out.data(), out.size()) == n;
  };
  std::vector<unsigned char> bytes;
  for (uint32_t g = 0; g < geometries_.size(); ++g) {
    Lotus::GpuGeometryContents geo;
    geo.slot = g;
    if (!read(LOTUS_SCENE_POSITIONS, g, bytes)) return fail("scene readback: positions");
    geo.positions.resize(bytes.size() / 12);
    std::memcpy(geo.positions.data(), bytes.data(), bytes.size());
    if (!read(LOTUS_SCENE_TRIANGLES, g, bytes)) return fail("scene readback: triangles");
    geo.triangles.resize(bytes.size() / 12);
    std::memcpy(geo.triangles.data(), bytes.data(), bytes.size());
    if (!read(LOTUS_SCENE_NORMALS, g, bytes)) return fail("scene readback: normals");
    geo.normals.resize(bytes.size() / 12);
    std::memcpy(geo.normals.data(), bytes.data(), bytes.size());
    c.geometries.push_back(std::move(geo));
  }
  if (!read(LOTUS_SCENE_INSTANCES, 0, bytes)) return fail("scene readback: instances");
  const size_t n_inst = bytes.size() / sizeof(lotus_instance);
  const auto* inst = reinterpret_cast<const lotus_instance*>(bytes.data());
  for (size_t i = 0; i < n_inst; ++i) {
    Lotus::GpuInstanceContents ic;
    std::memcpy(ic.world_from_object.data(), inst[i].world_from_object, 64);
    ic.geometry_slot = inst[i].geometry;
    ic.material_slot = inst[i].material;
    c.instances.push_back(ic);
    // The TLAS input: the transform's first three rows, row-major.
    Lotus::GpuTlasInstanceContents t;
    for (int row = 0; row < 3; ++row)
      for (int col = 0; col < 4; ++col) t.object_to_world[row * 4 + col] = inst[i].world_from_object[col * 4 + row];
    t.geometry_slot = inst[i].geometry;
    t.mask = 0xFFu;
    c.tlas_instances.push_back(t);
  }
  std::vector<unsigned char> mat_bytes;
  if (!read(LOTUS_SCENE_MATERIALS, 0, mat_bytes)) return fail("scene readback: materials");
  const auto* mats = reinterpret_cast<const lotus_material*>(mat_bytes.data());
  for (size_t i = 0; i < mat_bytes.size() / sizeof(lotus_material); ++i) {
    Lotus::GpuMaterialContents mc;
    mc.material.geometry.opacity = mats[i].opacity;
    mc.material.geometry.opacity_threshold = mats[i].opacity_threshold;
    if (mats[i].model == LOTUS_MODEL_GLTF_PBR) {
      Lotus::GltfPbr& g = mc.material.surface.emplace<Lotus::GltfPbr>();
      std::memcpy(g.base_color.value.data(), mats[i].base_color, 12);
      g.metallic.value = mats[i].metallic;
      g.roughness.value = mats[i].roughness;
      std::memcpy(g.emissive.value.data(), mats[i].emission, 12);
      g.emissive_strength = mats[i].emissive_strength;
      g.ior = mats[i].ior;
      g.specular.value = mats[i].specular;
      std::memcpy(g.specular_color.value.data(), mats[i].specular_color, 12);
      g.transmission.value = mats[i].transmission;
      g.clearcoat.value = mats[i].clearcoat;
      g.clearcoat_roughness.value = mats[i].clearcoat_roughness;
      std::memcpy(g.sheen_color.value.data(), mats[i].sheen_color, 12);
      g.sheen_roughness.value = mats[i].sheen_roughness;
      c.materials.push_back(mc);
      continue;
    }
    Lotus::PreviewSurface& p = Lotus::Preview(mc.material);
    std::memcpy(p.base_color.data(), mats[i].base_color, 12);
    p.roughness = mats[i].roughness;
    std::memcpy(p.emission.data(), mats[i].emission, 12);
    p.metallic = mats[i].metallic;
    std::memcpy(p.specular_color.data(), mats[i].specular_color, 12);
    p.ior = mats[i].ior;
    std::memcpy(p.transmission_color.data(), mats[i].transmission_color, 12);
    p.transmission = mats[i].transmission;
    p.use_specular_workflow = (mats[i].flags & LOTUS_MATERIAL_SPECULAR_WORKFLOW) != 0;
    p.thin_walled = (mats[i].flags & LOTUS_MATERIAL_THIN_WALLED) != 0;
    c.materials.push_back(mc);
  }
  if (!read(LOTUS_SCENE_ENVIRONMENT, 0, bytes) || bytes.size() != 12) return fail("scene readback: environment");
  std::memcpy(c.environment.data(), bytes.data(), 12);
  return c;
}

Lotus::PresentEvidence CudaOffscreenRenderer::Present(std::uint32_t, std::uint32_t, const Lotus::PresentView&) {
  Lotus::PresentEvidence p;
  p.status = Lotus::FrameStatus::Skip;
  p.detail = "presentation is a graphics-side part of the reference; the CUDA backend has none";
  return p;
}

Lotus::GpuResidency CudaOffscreenRenderer::Residency() const {
  Lotus::GpuResidency r;
  Lotus::GpuAllocationGroup g;
  g.owner = "scene";
  g.device_local = true;
  g.allocations = 1;
  g.bytes = device_bytes_;
  r.groups.push_back(g);
  r.device_local_bytes = device_bytes_;
  r.budget_available = false;
  r.budget_detail = "the CUDA backend reports the resident scene only";
  return r;
}

}  // namespace lotus_cuda_host
