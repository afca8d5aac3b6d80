// SPDX-License-Identifier: Apache-2.0
// Test driver of CudaOffscreenRenderer (hydra_lotus_b200/host): reads a
// scene and a frame from a small binary file, turns them into the
// reference's own types (MeshGeometry, SceneInstance, SceneMaterial with a
// PreviewSurface, SceneEnvironmentMap, SceneUpdate, DrawSummary,
// OffscreenTarget, PathTracingSettings), drives the adapter through
// Lotus::OffscreenRenderer's interface as a reference host would, and
// writes the colour product's floats to the output file. Prints one JSON
// line with the evidence. tests/test_gpu_adapter.py writes the input and
// compares the output with the C ABI's own render of the same frame.
//
// Input (little-endian): "LTSC", u32 version 1; u32 geometry, instance and
// material counts; f32 environment constant[3]; u32 has_environment (then
// u32 width, height; f32 scale[3], rows[9]; f32 texels[4 w h]); per
// geometry u32 vertices, triangles, has_normals, f32 positions[3 v], u32
// indices[3 t], f32 normals[9 t] when present; per instance f32 m[16], u32
// geometry, material; per material the lotus_material; the frame:
// f32 world_to_clip[16], u32 width, height, integrator, light_sampling,
// max_bounces, sample_index, frame_count.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "../hydra_lotus_b200/host/cuda_offscreen_renderer.hpp"

namespace {

struct Reader {
  std::vector<char> data;
  size_t at = 0;
  template <typename T>
  T get() {
    T v{};
    if (at + sizeof(T) <= data.size()) std::memcpy(&v, data.data() + at, sizeof(T));
    at += sizeof(T);
    return v;
  }
  template <typename T>
  void get(T* out, size_t n) {
    for (size_t i = 0; i < n; ++i) out[i] = get<T>();
  }
  bool ok() const { return at <= data.size(); }
};

const char* status_name(Lotus::FrameStatus s) {
  return s == Lotus::FrameStatus::Pass ? "pass" : (s == Lotus::FrameStatus::Skip ? "skip" : "fail");
}

}  // namespace

template <typename T>
void dump(const std::string& path, const std::vector<T>& v) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

// Two temporal frames through RenderTemporalScene with a still camera
// (view identity, projection the file's world_to_clip): ReSTIR DI with
// temporal reuse and a spatial pass of radius 2, radiance accumulation
// capped at 5 samples and 2 a-trous iterations. Writes each frame's colour
// and its temporal and ReSTIR products to <prefix><frame>_<name>.bin.
int temporal_frames(Lotus::OffscreenRenderer& renderer, const Lotus::DrawSummary& draw,
    const Lotus::OffscreenTarget& target, Lotus::PathTracingSettings settings, const std::string& prefix) {
  settings.light_sampling = Lotus::LightSampling::RestirInitial;
  settings.restir_temporal = true;
  settings.restir_spatial = true;
  settings.restir_spatial_radius = 2;
  Lotus::FrameSnapshot snapshot;
  snapshot.camera.projection = draw.world_to_clip;
  Lotus::TemporalFrameSettings temporal;
  temporal.width = target.width;
  temporal.height = target.height;
  temporal.accumulate_radiance = true;
  temporal.max_history_samples = 5;
  temporal.filter_iterations = 2;
  int code = 0;
  for (int k = 0; k < 2; ++k) {
    temporal.frame_index = (uint64_t)k;
    const Lotus::GpuFrameEvidence e = renderer.RenderTemporalScene(snapshot, target, 1, temporal, settings);
    const std::string base = prefix + std::to_string(k) + "_";
    dump(base + "color.bin", e.color.payload);
    dump(base + "surface.bin", e.temporal.current);
    dump(base + "validity.bin", e.temporal.validity);
    dump(base + "radiance.bin", e.temporal.radiance);
    dump(base + "batch.bin", e.temporal.batch);
    dump(base + "restir_initial.bin", e.restir.initial);
    dump(base + "restir_temporal.bin", e.restir.temporal);
    dump(base + "restir_spatial.bin", e.restir.spatial);
    dump(base + "restir_sources.bin", e.restir.spatial_sources);
    std::printf("{\"frame\": %d, \"render\": \"%s\", \"detail\": \"%s\", \"temporal\": %s, "
                "\"history\": %s, \"restir\": %s, \"restir_history\": %s, \"surface_pixels\": %zu, "
                "\"previous_pixels\": %zu, \"restir_previous_pixels\": %zu, \"filter_iterations\": %u}\n",
        k, status_name(e.status), e.detail.c_str(), e.temporal.available ? "true" : "false",
        e.temporal.history_available ? "true" : "false", e.restir.available ? "true" : "false",
        e.restir.history_available ? "true" : "false", e.temporal.current.size(), e.temporal.previous.size(),
        e.restir.previous.size(), e.temporal.filter_iterations);
    if (e.status != Lotus::FrameStatus::Pass) code = 1;
  }
  return code;
}

int main(int argc, char** argv) {
  const bool temporal_mode = argc == 5 && std::string(argv[3]) == "--temporal";
  if (argc != 3 && argc != 6 && !temporal_mode) {
    std::fprintf(stderr,
        "usage: adapter_harness <scene file> <output floats> "
        "[<dx> <after instance edit floats> <after point edit floats>]\n");
    return 2;
  }
  Reader in;
  {
    std::ifstream f(argv[1], std::ios::binary);
    in.data.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  char magic[4];
  in.get(magic, 4);
  if (std::memcmp(magic, "LTSC", 4) != 0 || in.get<uint32_t>() != 3) {
    std::fprintf(stderr, "not a scene file\n");
    return 2;
  }
  const uint32_t ng = in.get<uint32_t>(), ni = in.get<uint32_t>(), nm = in.get<uint32_t>();
  Lotus::SceneUpdate update;
  update.source_revision = 1;
  update.environment_changed = true;
  in.get(update.environment.data(), 3);
  std::shared_ptr<Lotus::Texture> env_texture;
  if (in.get<uint32_t>()) {
    env_texture = std::make_shared<Lotus::Texture>();
    env_texture->width = in.get<uint32_t>();
    env_texture->height = in.get<uint32_t>();
    env_texture->format = Lotus::TextureFormat::Rgba32Float;
    Lotus::SceneEnvironmentMap map;
    in.get(map.scale.data(), 3);
    float rows[9];
    in.get(rows, 9);
    // world_from_environment's columns are the image frame's axes.
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) map.world_from_environment[4 * r + c] = rows[3 * r + c];
    std::vector<float> texels(4 * (size_t)env_texture->width * env_texture->height);
    in.get(texels.data(), texels.size());
    env_texture->texels.resize(texels.size() * sizeof(float));
    std::memcpy(env_texture->texels.data(), texels.data(), env_texture->texels.size());
    map.texture = env_texture.get();
    update.texture_uploads.push_back(env_texture);
    update.environment_map = map;
  }
  std::vector<std::shared_ptr<Lotus::MeshGeometry>> meshes;
  for (uint32_t g = 0; g < ng; ++g) {
    auto m = std::make_shared<Lotus::MeshGeometry>();
    const uint32_t nv = in.get<uint32_t>(), nt = in.get<uint32_t>(), has_normals = in.get<uint32_t>();
    m->positions.resize(nv);
    for (auto& p : m->positions) in.get(p.data(), 3);
    m->triangles.resize(nt);
    for (auto& t : m->triangles) in.get(t.data(), 3);
    if (has_normals) {
      m->normals.resize(3 * (size_t)nt);
      for (auto& n : m->normals) in.get(n.data(), 3);
    }
    // Texture-coordinate sets, named so that key order is file order.
    const uint32_t sets = in.get<uint32_t>();
    for (uint32_t k = 0; k < sets; ++k) {
      auto& set = m->texcoords["st" + std::to_string(100 + k)];
      set.resize(3 * (size_t)nt);
      for (auto& st : set) in.get(st.data(), 2);
    }
    meshes.push_back(m);
    update.geometry_uploads.push_back(m);
  }
  update.instances_changed = true;
  for (uint32_t i = 0; i < ni; ++i) {
    Lotus::SceneInstance s;
    in.get(s.world_from_object.data(), 16);
    const uint32_t g = in.get<uint32_t>();
    s.material = in.get<uint32_t>();
    const uint32_t set = in.get<uint32_t>();
    s.texcoords = set == 0 ? Lotus::kNoTexcoords : set - 1;
    s.geometry = g < meshes.size() ? meshes[g].get() : nullptr;
    update.instances.push_back(s);
  }
  update.materials_changed = true;
  std::vector<lotus_material> materials(nm);
  for (uint32_t i = 0; i < nm; ++i) materials[i] = in.get<lotus_material>();
  // The images, then the texture inputs the materials' lookups name.
  std::vector<std::shared_ptr<Lotus::Texture>> textures(in.get<uint32_t>());
  for (auto& t : textures) {
    t = std::make_shared<Lotus::Texture>();
    t->width = in.get<uint32_t>();
    t->height = in.get<uint32_t>();
    const uint32_t format = in.get<uint32_t>();
    t->format = format == LOTUS_TEXTURE_RGBA8_SRGB     ? Lotus::TextureFormat::Rgba8Srgb
                : format == LOTUS_TEXTURE_RGBA32_FLOAT ? Lotus::TextureFormat::Rgba32Float
                                                       : Lotus::TextureFormat::Rgba8Unorm;
    t->texels.resize((size_t)t->width * t->height * Lotus::TexelBytes(t->format));
    in.get(t->texels.data(), t->texels.size());
    update.texture_uploads.push_back(t);
  }
  std::vector<lotus_texture_input> inputs(in.get<uint32_t>());
  for (auto& input : inputs) input = in.get<lotus_texture_input>();
  for (uint32_t i = 0; i < nm; ++i) {
    const lotus_material& lm = materials[i];
    Lotus::SceneMaterial sm;
    std::optional<Lotus::TextureInput>* slots[LOTUS_TEXTURE_SLOTS] = {};
    slots[LOTUS_SLOT_OPACITY] = &sm.material.geometry.opacity_texture;
    slots[LOTUS_SLOT_NORMAL] = &sm.material.geometry.normal_texture;
    if (lm.model == LOTUS_MODEL_GLTF_PBR) {
      // MaterialX's glTF PBR surface (material.hpp:180-217).
      Lotus::GltfPbr& g = sm.material.surface.emplace<Lotus::GltfPbr>();
      std::memcpy(g.base_color.value.data(), lm.base_color, 12);
      g.metallic.value = lm.metallic;
      g.roughness.value = lm.roughness;
      std::memcpy(g.emissive.value.data(), lm.emission, 12);
      g.emissive_strength = lm.emissive_strength;
      g.ior = lm.ior;
      g.specular.value = lm.specular;
      std::memcpy(g.specular_color.value.data(), lm.specular_color, 12);
      g.transmission.value = lm.transmission;
      g.clearcoat.value = lm.clearcoat;
      g.clearcoat_roughness.value = lm.clearcoat_roughness;
      std::memcpy(g.sheen_color.value.data(), lm.sheen_color, 12);
      g.sheen_roughness.value = lm.sheen_roughness;
      slots[LOTUS_GLTF_SLOT_BASE_COLOR] = &g.base_color.texture;
      slots[LOTUS_GLTF_SLOT_METALLIC] = &g.metallic.texture;
      slots[LOTUS_GLTF_SLOT_ROUGHNESS] = &g.roughness.texture;
      slots[LOTUS_GLTF_SLOT_EMISSIVE] = &g.emissive.texture;
      slots[LOTUS_GLTF_SLOT_SPECULAR] = &g.specular.texture;
      slots[LOTUS_GLTF_SLOT_SPECULAR_COLOR] = &g.specular_color.texture;
      slots[LOTUS_GLTF_SLOT_TRANSMISSION] = &g.transmission.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT] = &g.clearcoat.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT_ROUGHNESS] = &g.clearcoat_roughness.texture;
      slots[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL] = &g.clearcoat_normal_texture;
      slots[LOTUS_GLTF_SLOT_SHEEN_COLOR] = &g.sheen_color.texture;
      slots[LOTUS_GLTF_SLOT_SHEEN_ROUGHNESS] = &g.sheen_roughness.texture;
    } else {
      Lotus::PreviewSurface& p = sm.material.surface.emplace<Lotus::PreviewSurface>();
      std::memcpy(p.base_color.data(), lm.base_color, 12);
      p.roughness = lm.roughness;
      std::memcpy(p.emission.data(), lm.emission, 12);
      p.metallic = lm.metallic;
      std::memcpy(p.specular_color.data(), lm.specular_color, 12);
      p.ior = lm.ior;
      std::memcpy(p.transmission_color.data(), lm.transmission_color, 12);
      p.transmission = lm.transmission;
      p.use_specular_workflow = (lm.flags & LOTUS_MATERIAL_SPECULAR_WORKFLOW) != 0;
      p.thin_walled = (lm.flags & LOTUS_MATERIAL_THIN_WALLED) != 0;
      slots[LOTUS_SLOT_BASE_COLOR] = &p.base_color_texture;
      slots[LOTUS_SLOT_ROUGHNESS] = &p.roughness_texture;
      slots[LOTUS_SLOT_METALLIC] = &p.metallic_texture;
      slots[LOTUS_SLOT_EMISSION] = &p.emission_texture;
      slots[LOTUS_SLOT_SPECULAR_COLOR] = &p.specular_color_texture;
    }
    sm.material.geometry.opacity = lm.opacity;
    sm.material.geometry.opacity_threshold = lm.opacity_threshold;
    std::memcpy(sm.material.geometry.texcoord_fallback.data(), lm.texcoord_fallback, 8);
    if (lm.normal[0] != 0.0f || lm.normal[1] != 0.0f || lm.normal[2] != 0.0f)
      std::memcpy(sm.material.geometry.normal.data(), lm.normal, 12);
    // Each slot's lookup, its image resolved as the host's extraction
    // would (SceneMaterial::textures; none for a key without an image).
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k) {
      if (!slots[k] || lm.lookups[k] == LOTUS_NO_LOOKUP || lm.lookups[k] > inputs.size()) continue;
      const lotus_texture_input& d = inputs[lm.lookups[k] - 1];
      Lotus::TextureInput t;
      t.texture = d.texture == LOTUS_NO_TEXTURE ? std::string("missing") : "tex" + std::to_string(d.texture);
      t.channel = d.channel;
      t.wrap_s = (Lotus::TextureWrap)d.wrap_s;
      t.wrap_t = (Lotus::TextureWrap)d.wrap_t;
      std::memcpy(t.scale.data(), d.scale, 16);
      std::memcpy(t.bias.data(), d.bias, 16);
      std::memcpy(t.fallback.data(), d.fallback, 16);
      std::memcpy(t.st_transform.data(), d.st_transform, 24);
      *slots[k] = t;
      sm.textures[k] = d.texture != LOTUS_NO_TEXTURE && d.texture <= textures.size()
                           ? textures[d.texture - 1].get()
                           : nullptr;
    }
    update.materials.push_back(sm);
  }
  // The analytic lights, as the reference's Light (render_world.hpp:86-114).
  const uint32_t nl = in.get<uint32_t>();
  if (nl) update.lights_changed = true;
  for (uint32_t i = 0; i < nl; ++i) {
    const lotus_light ll = in.get<lotus_light>();
    Lotus::Light l;
    l.shape = ll.shape == LOTUS_LIGHT_SPHERE ? Lotus::LightShape::Sphere
              : ll.shape == LOTUS_LIGHT_RECT ? Lotus::LightShape::Rect
              : ll.shape == LOTUS_LIGHT_DISK ? Lotus::LightShape::Disk
                                             : Lotus::LightShape::Distant;
    l.normalize = ll.normalize != 0;
    std::memcpy(l.world_from_light.data(), ll.world_from_light, 64);
    std::memcpy(l.radiance.data(), ll.radiance, 12);
    l.radius = ll.radius;
    l.width = ll.width;
    l.height = ll.height;
    l.angle = ll.angle;
    update.lights.push_back(l);
  }
  Lotus::DrawSummary draw;
  in.get(draw.world_to_clip.data(), 16);
  Lotus::OffscreenTarget target;
  target.width = in.get<uint32_t>();
  target.height = in.get<uint32_t>();
  Lotus::PathTracingSettings settings;
  settings.integrator = in.get<uint32_t>() == LOTUS_INTEGRATOR_WAVEFRONT ? Lotus::Integrator::Wavefront
                                                                         : Lotus::Integrator::Reference;
  const uint32_t ls = in.get<uint32_t>();
  settings.light_sampling = ls == LOTUS_LIGHT_SAMPLING_BSDF ? Lotus::LightSampling::Bsdf : Lotus::LightSampling::Mis;
  settings.max_bounces = in.get<uint32_t>();
  settings.sample_index = in.get<uint32_t>();
  const uint32_t frame_count = in.get<uint32_t>();
  if (!in.ok()) {
    std::fprintf(stderr, "truncated scene file\n");
    return 2;
  }

  Lotus::FrameStatus status;
  std::string error;
  std::unique_ptr<Lotus::OffscreenRenderer> renderer =
      lotus_cuda_host::CudaOffscreenRenderer::Create(0, status, error);
  if (!renderer) {
    std::printf("{\"create\": \"%s\", \"detail\": \"%s\"}\n", status_name(status), error.c_str());
    return status == Lotus::FrameStatus::Skip ? 77 : 1;
  }
  const Lotus::BackendCapability cap = renderer->RayQueryCapability();
  const Lotus::GpuSceneEvidence scene = renderer->UpdateScene(update);
  if (temporal_mode) {
    if (scene.status != Lotus::FrameStatus::Pass) {
      std::printf("{\"update\": \"%s\", \"detail\": \"%s\"}\n", status_name(scene.status), scene.detail.c_str());
      return 1;
    }
    return temporal_frames(*renderer, draw, target, settings, argv[4]);
  }
  const Lotus::GpuFrameEvidence frame = renderer->RenderScene(draw, target, frame_count, settings);
  const Lotus::GpuFrameEvidence bootstrap = renderer->Render(draw, target, 1);
  const Lotus::PresentEvidence present = renderer->Present(target.width, target.height);
  std::printf(
      "{\"capability\": %s, \"update\": \"%s\", \"update_detail\": \"%s\", \"instances\": %u, "
      "\"render\": \"%s\", \"render_detail\": \"%s\", \"spp\": %u, \"rounds\": %u, \"paths\": %zu, "
      "\"pixel_format\": \"%s\", \"row_pitch\": %u, \"bytes\": %zu, \"bootstrap\": \"%s\", \"present\": \"%s\"}\n",
      cap.available ? "true" : "false", status_name(scene.status), scene.detail.c_str(), scene.stats.instance_count,
      status_name(frame.status), frame.detail.c_str(), frame.samples_per_pixel, frame.wavefront_rounds,
      frame.wavefront_path_counts.size(), frame.color.pixel_format.c_str(), frame.color.row_pitch,
      frame.color.payload.size(), status_name(bootstrap.status), status_name(present.status));
  {
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char*>(frame.color.payload.data()), (std::streamsize)frame.color.payload.size());
  }
  if (frame.status != Lotus::FrameStatus::Pass) return 1;
  if (argc == 3) return 0;
  // Edits, as a host's SceneExtraction plans them: an instance-only plan
  // (instance 0 moves by dx), then a geometry replacement with the same
  // topology (geometry 0's positions y += 0.01 x) whose instances name the
  // replacement.
  const float dx = std::strtof(argv[3], nullptr);
  Lotus::SceneUpdate moved;
  moved.source_revision = 2;
  moved.instances_changed = true;
  moved.instances = update.instances;
  moved.instances[0].world_from_object[12] += dx;
  const Lotus::GpuSceneEvidence s2 = renderer->UpdateScene(moved);
  const Lotus::GpuFrameEvidence f2 = renderer->RenderScene(draw, target, frame_count, settings);
  auto replacement = std::make_shared<Lotus::MeshGeometry>(*meshes[0]);
  for (auto& p : replacement->positions) p[1] += 0.01f * p[0];
  Lotus::SceneUpdate edited;
  edited.source_revision = 3;
  edited.geometry_releases.push_back(meshes[0].get());
  edited.geometry_uploads.push_back(replacement);
  edited.geometry_replacements.push_back({meshes[0].get(), replacement.get()});
  edited.instances_changed = true;
  edited.instances = moved.instances;
  for (auto& inst : edited.instances)
    if (inst.geometry == meshes[0].get()) inst.geometry = replacement.get();
  const Lotus::GpuSceneEvidence s3 = renderer->UpdateScene(edited);
  const Lotus::GpuFrameEvidence f3 = renderer->RenderScene(draw, target, frame_count, settings);
  // ReadBackScene after the edits: every instance as uploaded, and the
  // geometry each instance names holding that geometry's points.
  const Lotus::GpuSceneContents contents = renderer->ReadBackScene();
  bool readback = contents.status == Lotus::FrameStatus::Pass && contents.instances.size() == edited.instances.size() &&
                  contents.tlas_instances.size() == edited.instances.size();
  for (size_t i = 0; readback && i < edited.instances.size(); ++i) {
    const Lotus::GpuInstanceContents& got = contents.instances[i];
    readback = got.world_from_object == edited.instances[i].world_from_object &&
               got.material_slot == edited.instances[i].material && got.geometry_slot < contents.geometries.size() &&
               contents.geometries[got.geometry_slot].positions == edited.instances[i].geometry->positions &&
               contents.geometries[got.geometry_slot].triangles == edited.instances[i].geometry->triangles;
  }
  std::printf("{\"instance_edit\": \"%s\", \"instance_edit_render\": \"%s\", \"point_edit\": \"%s\", "
              "\"point_edit_render\": \"%s\", \"readback\": \"%s\", \"materials\": %zu, \"detail\": \"%s%s%s\"}\n",
      status_name(s2.status), status_name(f2.status), status_name(s3.status), status_name(f3.status),
      readback ? "pass" : "fail", contents.materials.size(), s2.detail.c_str(), s3.detail.c_str(),
      contents.detail.c_str());
  {
    std::ofstream out(argv[4], std::ios::binary);
    out.write(reinterpret_cast<const char*>(f2.color.payload.data()), (std::streamsize)f2.color.payload.size());
  }
  {
    std::ofstream out(argv[5], std::ios::binary);
    out.write(reinterpret_cast<const char*>(f3.color.payload.data()), (std::streamsize)f3.color.payload.size());
  }
  return s2.status == Lotus::FrameStatus::Pass && f2.status == Lotus::FrameStatus::Pass &&
                 s3.status == Lotus::FrameStatus::Pass && f3.status == Lotus::FrameStatus::Pass && readback
             ? 0
             : 1;
}
