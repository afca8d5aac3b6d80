// SPDX-License-Identifier: Apache-2.0
// CudaOffscreenRenderer: the reference's Lotus::OffscreenRenderer
// (include/lotus/vulkan_backend.hpp:753-842 in hydra-lotus) implemented over
// the CUDA backend's C ABI (include/lotus_cuda.h), so that a host written
// against the reference — lotus-headless, the Hydra delegate — renders
// through the B200 path by creating this renderer instead of the Vulkan
// one. It compiles against the reference's own headers and adds no
// dependency beyond them and liblotus_cuda.
//
// What maps where:
//   UpdateScene(SceneUpdate)  resident geometry, instances, UsdPreviewSurface
//                             and glTF PBR materials and the environment,
//                             rebuilt into one
//                             lotus_scene_desc -> lotus_cuda_update_scene
//   RenderScene(...)          lotus_cuda_render (Radiance output)
//   RenderTemporalScene(...)  lotus_cuda_render_temporal with the snapshot's
//                             camera; the scene is the one UpdateScene made
//                             resident (the host applies the snapshot's plan
//                             through UpdateScene first, as it does for
//                             RenderScene)
//   RayQueryCapability()      lotus_cuda_capability
//   ReadBackScene()           lotus_cuda_read_scene
//   Render, Present           Skip: the bootstrap raster and presentation are
//                             graphics-side parts of the reference that this
//                             backend does not build
//   Residency()               the resident scene's device bytes
// Analytic lights (Lotus::Light) map field for field to lotus_light; the
// resident textures to lotus_texture, each model's texture inputs in the
// reference's slot numbering (material.hpp:262-312) to lotus_texture_input,
// each geometry's texture-coordinate sets in key order and each instance's
// set, and each geometry's colour sets in key order and each instance's
// colour set. Scene content the backend does not build (the reserved
// Standard Surface and OpenPBR models) makes UpdateScene Fail with the
// reason, as the reference Fails on unsupported content.
#pragma once

#include <lotus/vulkan_backend.hpp>

#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/lotus_cuda.h"

namespace lotus_cuda_host {

class CudaOffscreenRenderer final : public Lotus::OffscreenRenderer {
 public:
  // The CreateOffscreenRenderer counterpart: Pass with a renderer, Skip
  // without an sm_100 device, Fail otherwise (status and error say which).
  static std::unique_ptr<Lotus::OffscreenRenderer> Create(int device, Lotus::FrameStatus& status,
      std::string& error);
  ~CudaOffscreenRenderer() override;

  Lotus::GpuFrameEvidence Render(const Lotus::DrawSummary& draw, const Lotus::OffscreenTarget& target,
      std::uint32_t frame_count) override;
  Lotus::BackendCapability RayQueryCapability() const override;
  Lotus::GpuFrameEvidence RenderScene(const Lotus::DrawSummary& draw, const Lotus::OffscreenTarget& target,
      std::uint32_t frame_count, const Lotus::PathTracingSettings& settings = {}) override;
  Lotus::GpuFrameEvidence RenderTemporalScene(const Lotus::FrameSnapshot& snapshot,
      const Lotus::OffscreenTarget& target, std::uint32_t frame_count,
      const Lotus::TemporalFrameSettings& temporal, const Lotus::PathTracingSettings& settings = {}) override;
  Lotus::GpuSceneEvidence UpdateScene(const Lotus::SceneUpdate& update) override;
  Lotus::GpuSceneContents ReadBackScene() override;
  Lotus::PresentEvidence Present(std::uint32_t width, std::uint32_t height,
      const Lotus::PresentView& view = {}) override;
  Lotus::GpuResidency Residency() const override;

 private:
  CudaOffscreenRenderer(int device, lotus_cuda_renderer* handle) : device_(device), handle_(handle) {}
  bool FillFrame(const Lotus::Matrix4& world_to_clip, const Lotus::OffscreenTarget& target,
      std::uint32_t frame_count, const Lotus::PathTracingSettings& settings, lotus_frame_desc& frame,
      std::string& error) const;
  void FillEvidence(const lotus_frame_desc& frame, const lotus_frame_result& result, std::vector<float>& color,
      Lotus::GpuFrameEvidence& evidence);
  // Plans that change instances only, or replace geometries with ones of
  // the same topology (SceneGeometryReplacement), go to the incremental
  // entry points; returns false when the plan needs a full update.
  bool UpdateIncrementally(const Lotus::SceneUpdate& update, Lotus::GpuSceneEvidence& evidence);
  // The temporal and ReSTIR products of the frame just rendered
  // (TemporalProducts, RestirProducts), read back through the C ABI.
  void FillTemporalProducts(const lotus_temporal_desc& desc, bool history, bool camera_cut,
      Lotus::GpuFrameEvidence& evidence);
  bool InstanceArray(std::vector<lotus_instance>& out, std::string& error) const;
  void SceneStats(const Lotus::SceneUpdate& update, const lotus_scene_result& result,
      Lotus::GpuSceneEvidence& evidence) const;

  int device_;
  lotus_cuda_renderer* handle_;
  bool failed_ = false;
  std::string failure_;
  // Resident scene, as the updates left it.
  std::vector<std::shared_ptr<const Lotus::MeshGeometry>> geometries_;
  std::vector<std::shared_ptr<const Lotus::Texture>> textures_;
  std::vector<Lotus::SceneInstance> instances_;
  std::vector<Lotus::SceneMaterial> materials_;
  std::array<float, 3> environment_{};
  std::optional<Lotus::SceneEnvironmentMap> environment_map_;
  std::vector<Lotus::Light> lights_;  // the analytic lights, in key order
  std::uint64_t device_bytes_ = 0;
  bool resident_ = false;  // a full update has made the scene resident
  std::uint32_t material_slots_ = 0;
  bool environment_map_bound_ = false;
  // The preceding temporal frame's camera.
  bool have_previous_camera_ = false;
  Lotus::Camera previous_camera_;
};

}  // namespace lotus_cuda_host
