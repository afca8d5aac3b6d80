// SPDX-License-Identifier: Apache-2.0
// Hit reconstruction, light sampling, the environment image and the camera
// on the device (backend/vulkan/shaders/common/scene.slang and
// common/transport.slang in hydra-lotus), over the SoA tables of scene.cuh.
#pragma once

#include "bsdf.cuh"
#include "gltf.cuh"
#include "scene.cuh"

namespace lotus {

struct SurfaceHit {
  F3 position;
  F3 normal;          // geometric, facing the incoming ray
  F3 shading_normal;
  float area;
  F3 base_color;
  float roughness;
  float metallic;
  Closure bsdf;       // UsdPreviewSurface's closure
  F3 emission;
  bool gltf;          // the closure is glTF PBR's: `composed`, built from `gltf_terms`
  GltfClosure composed;
  GltfTerms gltf_terms;
};

__device__ __forceinline__ F3 transform_point(const float4* m, F3 p) { return row_point(m, p); }

__device__ __forceinline__ float triangle_area(F3 p0, F3 p1, F3 p2) {
  return 0.5f * length(cross(p1 - p0, p2 - p0));
}

// ShadingNormal (scene.slang:467-488).
__device__ __forceinline__ F3 shading_normal(const float* n, float b1, float b2, const float4* m,
    F3 geometric, F3 direction) {
  const F3 n0 = V(n[0], n[1], n[2]), n1 = V(n[3], n[4], n[5]), n2 = V(n[6], n[7], n[8]);
  const F3 object = n0 + b1 * (n1 - n0) + b2 * (n2 - n0);
  const F3 c0 = V(m[0].x, m[1].x, m[2].x);
  const F3 c1 = V(m[0].y, m[1].y, m[2].y);
  const F3 c2 = V(m[0].z, m[1].z, m[2].z);
  const F3 world = cross(c1, c2) * object.x + cross(c2, c0) * object.y + cross(c0, c1) * object.z;
  const float length2 = dot(world, world);
  if (!(length2 > 0.0f) || isinf(length2)) return geometric;
  F3 s = world * rsqrt_rn(length2);
  if (dot(s, geometric) < 0.0f) s = -s;
  return dot(s, direction) < 0.0f ? s : geometric;
}

__device__ __forceinline__ float saturate1(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// TangentFrame (scene.slang:490-538): the texture coordinates'
// differentials in world space, orthonormalized about the interpolated
// shading normal, keeping the handedness of mirrored coordinates and
// transforms; a frame about the normal alone where the instance has no
// coordinates or they are degenerate or ill-conditioned. A normal-map
// lookup (L non-null) transforms the differentials as its coordinates.
__device__ __forceinline__ Frame tangent_frame(const SceneView& S, uint32_t instance, const TextureLookup* L,
    uint32_t primitive, F3 edge1, F3 edge2, F3 normal) {
  Frame basis = make_frame(normal);
  const uint32_t base = S.inst_texcoords[instance];
  if (base == kNoTexture) return basis;
  const float2* c = S.texcoords + base + 3 * (size_t)primitive;
  const float2 st0 = c[0], st1 = c[1], st2 = c[2];
  float u1 = st1.x - st0.x, v1 = st1.y - st0.y, u2 = st2.x - st0.x, v2 = st2.y - st0.y;
  if (L != nullptr) {
    const float a1 = L->st_s.x * u1 + L->st_s.y * v1, b1 = L->st_t.x * u1 + L->st_t.y * v1;
    const float a2 = L->st_s.x * u2 + L->st_s.y * v2, b2 = L->st_t.x * u2 + L->st_t.y * v2;
    u1 = a1;
    v1 = b1;
    u2 = a2;
    v2 = b2;
  }
  const float uv_scale = fmaxf(fmaxf(fabsf(u1), fabsf(v1)), fmaxf(fabsf(u2), fabsf(v2)));
  const float edge_scale = fmaxf(fmaxf(fmaxf(fabsf(edge1.x), fabsf(edge1.y)), fabsf(edge1.z)),
      fmaxf(fmaxf(fabsf(edge2.x), fabsf(edge2.y)), fabsf(edge2.z)));
  if (!(uv_scale > 0.0f) || isinf(uv_scale) || !(edge_scale > 0.0f) || isinf(edge_scale)) return basis;
  u1 = u1 / uv_scale;
  v1 = v1 / uv_scale;
  u2 = u2 / uv_scale;
  v2 = v2 / uv_scale;
  edge1 = V(edge1.x / edge_scale, edge1.y / edge_scale, edge1.z / edge_scale);
  edge2 = V(edge2.x / edge_scale, edge2.y / edge_scale, edge2.z / edge_scale);
  const float determinant = u1 * v2 - v1 * u2;
  if (!(fabsf(determinant) > 1e-8f)) return basis;
  const float orientation = determinant < 0.0f ? -1.0f : 1.0f;
  F3 tangent = orientation * (edge1 * v2 - edge2 * v1);
  const F3 bitangent = orientation * (edge2 * u1 - edge1 * u2);
  tangent = tangent - normal * dot(normal, tangent);
  const float length2 = dot(tangent, tangent);
  if (!(length2 > 1e-16f) || isinf(length2)) return basis;
  basis.t = tangent * rsqrt_rn(length2);
  basis.b = cross(normal, basis.t);
  if (dot(basis.b, bitangent) < 0.0f) basis.b = -basis.b;
  return basis;
}

// MappedNormal (scene.slang:541-556): the tangent-space normal through the
// frame, turned to the geometric side; the frame's normal where the input
// is zero or non-finite or the mapped normal faces away from the ray.
__device__ __forceinline__ F3 mapped_normal(F3 tangent_normal, const Frame& basis, F3 geometric, F3 direction) {
  const float magnitude = fmaxf(fmaxf(fabsf(tangent_normal.x), fabsf(tangent_normal.y)), fabsf(tangent_normal.z));
  if (!(magnitude > 0.0f) || !isfinite(tangent_normal.x) || !isfinite(tangent_normal.y) ||
      !isfinite(tangent_normal.z))
    return basis.n;
  F3 shading = normalize(basis.to_world(V(tangent_normal.x / magnitude, tangent_normal.y / magnitude,
      tangent_normal.z / magnitude)));
  if (dot(shading, geometric) < 0.0f) shading = -shading;
  return dot(shading, direction) < 0.0f ? shading : basis.n;
}

// PreviewEmission (scene.slang:570-577): the constant, or the lookup's RGB
// at (s, t), negative parts cut.
__device__ __forceinline__ F3 preview_emission(const SceneView& S, const MaterialRecord& mat,
    const MaterialLookups& ml, float s, float t) {
  const uint32_t k = ml.slot[LOTUS_SLOT_EMISSION];
  if (k == kNoTexture) return V(mat.emission_metallic);
  const float4 v = texture_lookup(S, S.lookups[k], s, t);
  return V(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f));
}

// GltfEmission (scene.slang:579-588): emissive, or its lookup's RGB with
// negative parts cut, times the strength.
__device__ __forceinline__ F3 gltf_emission(const SceneView& S, const MaterialRecord& mat,
    const MaterialLookups& ml, float s, float t) {
  const float strength = mat.gltf.w;
  const uint32_t k = ml.slot[LOTUS_GLTF_SLOT_EMISSIVE];
  if (k == kNoTexture) return V(mat.emission_metallic) * strength;
  const float4 v = texture_lookup(S, S.lookups[k], s, t);
  return V(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f)) * strength;
}

// Emission (scene.slang:590-600) by the material's model.
__device__ __forceinline__ F3 material_emission(const SceneView& S, const MaterialRecord& mat,
    const MaterialLookups& ml, float s, float t) {
  return (__float_as_uint(mat.coverage.z) & kMaterialGltf) ? gltf_emission(S, mat, ml, s, t)
                                                           : preview_emission(S, mat, ml, s, t);
}

// EvaluatePreview's textured inputs (scene.slang:1184-1230): each lookup
// replaces its input's constant, clamped into the input's range, and a
// tangent-space normal other than the identity maps the shading normal.
// Not inlined: shading of untextured materials keeps its registers.
struct TexturedInputs {
  F3 base_color;
  float roughness;
  float metallic;
  F3 emission;
  F3 specular;
  F3 shading_normal;
};

static __device__ __noinline__ TexturedInputs textured_inputs(const SceneView& S, uint32_t instance, uint32_t material,
    uint32_t primitive, float b1, float b2, F3 edge1, F3 edge2, F3 geometric, F3 shading, F3 direction,
    F3 base_color) {
  const MaterialRecord mat = S.materials[material];
  const MaterialLookups ml = S.mat_lookups[material];
  TexturedInputs out;
  out.base_color = base_color;
  out.roughness = mat.base_roughness.w;
  out.metallic = mat.emission_metallic.w;
  out.specular = V(mat.specular_ior);
  out.shading_normal = shading;
  float s, t;
  hit_texcoords(S, instance, ml, primitive, b1, b2, s, t);
  uint32_t k = ml.slot[LOTUS_SLOT_BASE_COLOR];
  if (k != kNoTexture) {
    const float4 v = texture_lookup(S, S.lookups[k], s, t);
    out.base_color = V(saturate1(v.x), saturate1(v.y), saturate1(v.z));
  }
  k = ml.slot[LOTUS_SLOT_ROUGHNESS];
  if (k != kNoTexture)
    out.roughness = saturate1(lookup_channel(texture_lookup(S, S.lookups[k], s, t), S.lookups[k].channel));
  k = ml.slot[LOTUS_SLOT_METALLIC];
  if (k != kNoTexture)
    out.metallic = saturate1(lookup_channel(texture_lookup(S, S.lookups[k], s, t), S.lookups[k].channel));
  out.emission = preview_emission(S, mat, ml, s, t);
  F3 tangent_normal = V(ml.normal[0], ml.normal[1], ml.normal[2]);
  const uint32_t normal_lookup = ml.slot[LOTUS_SLOT_NORMAL];
  if (normal_lookup != kNoTexture) {
    const float4 v = texture_lookup(S, S.lookups[normal_lookup], s, t);
    tangent_normal = V(fminf(fmaxf(v.x, -1.0f), 1.0f), fminf(fmaxf(v.y, -1.0f), 1.0f), fminf(fmaxf(v.z, -1.0f), 1.0f));
  }
  k = ml.slot[LOTUS_SLOT_SPECULAR_COLOR];
  if (k != kNoTexture) {
    const float4 v = texture_lookup(S, S.lookups[k], s, t);
    if (isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) out.specular = V(saturate1(v.x), saturate1(v.y), saturate1(v.z));
  }
  // The constant-material path is kept exactly when the input is the
  // identity.
  if (tangent_normal.x != 0.0f || tangent_normal.y != 0.0f || tangent_normal.z != 1.0f)
    out.shading_normal = mapped_normal(tangent_normal,
        tangent_frame(S, instance, normal_lookup != kNoTexture ? &S.lookups[normal_lookup] : nullptr, primitive,
            edge1, edge2, shading),
        geometric, direction);
  return out;
}

// What EvaluateGltfPbr gives the hit (scene.slang:1276-1406).
struct GltfHit {
  F3 base_color;
  float roughness;
  float metallic;
  F3 emission;
  F3 shading_normal;
  GltfTerms terms;
  GltfClosure closure;
};

__device__ __forceinline__ float gltf_scalar(const SceneView& S, const MaterialLookups& ml, uint32_t slot,
    float s, float t, float constant) {
  const uint32_t k = ml.slot[slot];
  if (k == kNoTexture) return constant;
  return saturate(lookup_channel(texture_lookup(S, S.lookups[k], s, t), S.lookups[k].channel));
}

__device__ __forceinline__ F3 clamp_unit_normal(float4 v) {
  return V(fminf(fmaxf(v.x, -1.0f), 1.0f), fminf(fmaxf(v.y, -1.0f), 1.0f), fminf(fmaxf(v.z, -1.0f), 1.0f));
}

// EvaluateGltfPbr (scene.slang:1276-1406): the model's inputs at the hit,
// each texture lookup replacing its constant, clamped into its range; the
// mapped shading normal; the coat's normal in the shading frame; the terms
// with their table values at wo; and the closure. Not inlined: the
// shading kernels keep none of its registers for other materials.
static __device__ __noinline__ GltfHit gltf_hit(const SceneView& S, uint32_t instance, uint32_t material,
    uint32_t primitive, float b1, float b2, F3 edge1, F3 edge2, F3 geometric, F3 shading, F3 direction) {
  const MaterialRecord mat = S.materials[material];
  const MaterialLookups ml = S.mat_lookups[material];
  GltfHit out;
  out.base_color = V(mat.base_roughness);
  out.roughness = mat.base_roughness.w;
  out.metallic = mat.emission_metallic.w;
  out.emission = V(mat.emission_metallic) * mat.gltf.w;
  F3 tangent_normal = V(ml.normal[0], ml.normal[1], ml.normal[2]);
  const float dielectric_f0 = mat.coverage.w;
  float specular = mat.gltf.x;
  float transmission = mat.transmission.w;
  F3 specular_color = V(mat.specular_ior);
  float clearcoat = mat.gltf.y;
  F3 sheen_color = V(mat.sheen);
  float sheen_roughness = mat.sheen.w;
  float clearcoat_roughness = mat.gltf.z;
  const F3 mesh_normal = shading;
  F3 coat_tangent_normal = V(0.0f, 0.0f, 1.0f);
  out.shading_normal = shading;
  if (__float_as_uint(mat.coverage.z) & kMaterialTextured) {
    float s, t;
    hit_texcoords(S, instance, ml, primitive, b1, b2, s, t);
    uint32_t k = ml.slot[LOTUS_GLTF_SLOT_BASE_COLOR];
    if (k != kNoTexture) {
      const float4 v = texture_lookup(S, S.lookups[k], s, t);
      out.base_color = V(saturate(v.x), saturate(v.y), saturate(v.z));
    }
    out.roughness = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_ROUGHNESS, s, t, out.roughness);
    out.metallic = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_METALLIC, s, t, out.metallic);
    out.emission = gltf_emission(S, mat, ml, s, t);
    k = ml.slot[LOTUS_SLOT_NORMAL];
    if (k != kNoTexture) tangent_normal = clamp_unit_normal(texture_lookup(S, S.lookups[k], s, t));
    specular = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_SPECULAR, s, t, specular);
    transmission = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_TRANSMISSION, s, t, transmission);
    clearcoat = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_CLEARCOAT, s, t, clearcoat);
    clearcoat_roughness = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_CLEARCOAT_ROUGHNESS, s, t, clearcoat_roughness);
    sheen_roughness = gltf_scalar(S, ml, LOTUS_GLTF_SLOT_SHEEN_ROUGHNESS, s, t, sheen_roughness);
    k = ml.slot[LOTUS_GLTF_SLOT_SPECULAR_COLOR];
    if (k != kNoTexture) {
      const float4 v = texture_lookup(S, S.lookups[k], s, t);
      specular_color = V(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f));
    }
    k = ml.slot[LOTUS_GLTF_SLOT_SHEEN_COLOR];
    if (k != kNoTexture) {
      const float4 v = texture_lookup(S, S.lookups[k], s, t);
      sheen_color = V(saturate(v.x), saturate(v.y), saturate(v.z));
    }
    k = ml.slot[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL];
    if (k != kNoTexture) coat_tangent_normal = clamp_unit_normal(texture_lookup(S, S.lookups[k], s, t));
  }
  if (tangent_normal.x != 0.0f || tangent_normal.y != 0.0f || tangent_normal.z != 1.0f) {
    const uint32_t k = ml.slot[LOTUS_SLOT_NORMAL];
    out.shading_normal = mapped_normal(tangent_normal,
        tangent_frame(S, instance, k != kNoTexture ? &S.lookups[k] : nullptr, primitive, edge1, edge2, shading),
        geometric, direction);
  }
  // The closure's outgoing direction in the shading frame: without a coat
  // only its cosine counts.
  const float cos_o = dot(out.shading_normal, -direction);
  F3 wo = V(sqrtf(fmaxf(1.0f - cos_o * cos_o, 0.0f)), 0.0f, cos_o);
  GltfInputs in;
  in.base_color = out.base_color;
  in.roughness = out.roughness;
  in.metallic = out.metallic;
  in.dielectric_f0 = dielectric_f0;
  in.specular = specular;
  in.specular_color = specular_color;
  in.transmission = transmission;
  in.clearcoat = clearcoat;
  in.clearcoat_roughness = clearcoat_roughness;
  in.clearcoat_normal = V(0.0f, 0.0f, 1.0f);
  in.sheen_color = sheen_color;
  in.sheen_roughness = sheen_roughness;
  if (clearcoat > 0.0f) {
    F3 coat_normal = mesh_normal;
    if (coat_tangent_normal.x != 0.0f || coat_tangent_normal.y != 0.0f || coat_tangent_normal.z != 1.0f) {
      const uint32_t k = ml.slot[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL];
      coat_normal = mapped_normal(coat_tangent_normal,
          tangent_frame(S, instance, k != kNoTexture ? &S.lookups[k] : nullptr, primitive, edge1, edge2,
              mesh_normal),
          geometric, direction);
    }
    const Frame basis = make_frame(out.shading_normal);
    const F3 local = basis.to_local(-direction);
    wo.x = local.x;
    wo.y = local.y;
    in.clearcoat_normal = normalize(basis.to_local(coat_normal));
  }
  out.terms = make_gltf_terms(in, wo, S.albedo_tables);
  out.closure = make_gltf_closure(out.terms, wo);
  return out;
}

// HitColor (scene.slang:376-386): the instance's colour set at the hit,
// one value for the whole mesh or the corners' interpolated.
__device__ __forceinline__ F3 hit_color(const SceneView& S, uint2 set, uint32_t primitive, float b1, float b2) {
  const float* c = S.colors + set.x;
  if (set.y) return V(c[0], c[1], c[2]);
  c += 9 * (size_t)primitive;
  const F3 c0 = V(c[0], c[1], c[2]), c1 = V(c[3], c[4], c[5]), c2 = V(c[6], c[7], c[8]);
  return c0 + b1 * (c1 - c0) + b2 * (c2 - c0);
}

// ReconstructHit and EvaluatePreview (scene.slang:1408-1449, 1184-1260).
// The corners come from the leaf-ordered triangle pool, which holds the
// geometry's own positions. A texture lookup replaces its input's constant,
// clamped into the input's range.
// kFullShading false: the scene has no texture lookups (SceneView::full_shading
// clear), and the hit compiles without them.
template <bool kFullShading = true>
__device__ __forceinline__ SurfaceHit reconstruct_hit(const SceneView& S, uint32_t instance,
    uint32_t tri, float b1, float b2, F3 direction, uint32_t* primitive_out = nullptr) {
  const InstanceShading rec = S.inst_shade[instance];
  const float4* tv = S.tris + kTriStride * (size_t)tri;
  const float4 a = tv[0], b = tv[1], c = tv[2];
  const uint32_t primitive = __float_as_uint(a.w);
  if (primitive_out) *primitive_out = primitive;
  const F3 p0 = transform_point(rec.m, V(a));
  const F3 p1 = transform_point(rec.m, V(b));
  const F3 p2 = transform_point(rec.m, V(c));
  SurfaceHit sh;
  sh.position = p0 + b1 * (p1 - p0) + b2 * (p2 - p0);
  const F3 normal = normalize(cross(p1 - p0, p2 - p0));
  sh.area = triangle_area(p0, p1, p2);
  sh.normal = dot(normal, direction) > 0.0f ? -normal : normal;
  sh.shading_normal = sh.normal;
  if (rec.normals != kNoLights)
    sh.shading_normal = shading_normal(S.normals + 9 * ((size_t)rec.normals + primitive), b1, b2,
        rec.m, sh.normal, direction);
  const MaterialRecord mat = S.materials[rec.material];
  sh.base_color = V(mat.base_roughness);
  sh.roughness = mat.base_roughness.w;
  sh.metallic = mat.emission_metallic.w;
  const uint32_t flags = __float_as_uint(mat.coverage.z);
  F3 emission = V(mat.emission_metallic);
  F3 specular = V(mat.specular_ior);
  sh.gltf = false;
  if (kFullShading && (flags & kMaterialGltf)) {
    const GltfHit g = gltf_hit(S, instance, rec.material, primitive, b1, b2, p1 - p0, p2 - p0, sh.normal,
        sh.shading_normal, direction);
    sh.base_color = g.base_color;
    sh.roughness = g.roughness;
    sh.metallic = g.metallic;
    sh.shading_normal = g.shading_normal;
    sh.emission = g.emission;
    sh.gltf = true;
    sh.composed = g.closure;
    sh.gltf_terms = g.terms;
    // MakeBsdfClosure(model, composed) (bsdf.slang:42-50): the preview
    // closure it carries beside the composed one.
    sh.bsdf = make_closure(V(0.0f), 1.0f, 0.0f, 1.5f, false, V(0.0f), 0.0f, V(1.0f), false, true);
    return sh;
  }
  if (kFullShading) {
    // EvaluatePreview's base colour: the instance's colour set, clamped,
    // where it reads one.
    const uint2 set = S.inst_colors[instance];
    if (set.x != kNoTexture) {
      const F3 c = hit_color(S, set, primitive, b1, b2);
      sh.base_color = V(saturate(c.x), saturate(c.y), saturate(c.z));
    }
  }
  if (kFullShading && (flags & kMaterialTextured)) {
    const TexturedInputs ti = textured_inputs(S, instance, rec.material, primitive, b1, b2, p1 - p0, p2 - p0,
        sh.normal, sh.shading_normal, direction, sh.base_color);
    sh.base_color = ti.base_color;
    sh.roughness = ti.roughness;
    sh.metallic = ti.metallic;
    emission = ti.emission;
    specular = ti.specular;
    sh.shading_normal = ti.shading_normal;
  }
  const float transmission = mat.transmission.w;
  bool entering = true;
  if (transmission > 0.0f) {
    const F3 outward = rec.mirror ? -normal : normal;
    entering = dot(outward, direction) < 0.0f;
  }
  sh.bsdf = make_closure(sh.base_color, sh.roughness, sh.metallic, mat.specular_ior.w,
      (flags & 1u) != 0, specular, transmission, V(mat.transmission),
      (flags & 2u) != 0, entering);
  sh.emission = emission;
  return sh;
}

// BsdfEvaluate, BsdfPdf and BsdfSample (bsdf.slang:52-90): the hit's
// closure by its model. kFullShading false: no glTF PBR material is in the
// scene, and only UsdPreviewSurface's closure is compiled.
template <bool kFullShading>
__device__ __forceinline__ F3 surface_evaluate(const SurfaceHit& sh, F3 wo, F3 wi) {
  if (kFullShading && sh.gltf) return gltf_evaluate(sh.composed, wo, wi);
  return bsdf_evaluate(sh.bsdf, wo, wi);
}

template <bool kFullShading>
__device__ __forceinline__ float surface_pdf(const SurfaceHit& sh, F3 wo, F3 wi) {
  if (kFullShading && sh.gltf) return gltf_pdf(sh.composed, wo, wi);
  return bsdf_pdf(sh.bsdf, wo, wi);
}

template <bool kFullShading>
__device__ __forceinline__ bool surface_sample(const SurfaceHit& sh, F3 wo, F3 u, BsdfSample& s) {
  if (kFullShading && sh.gltf) return gltf_sample(sh.composed, wo, u, s);
  return bsdf_sample(sh.bsdf, wo, u, s);
}

struct LightSample {
  F3 direction;
  float distance;
  F3 radiance;
  float pdf;
  bool delta;
};

__device__ __forceinline__ LightSample no_light() {
  LightSample s;
  s.direction = V(0.0f, 0.0f, 1.0f);
  s.distance = 0.0f;
  s.radiance = V(0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  return s;
}

// A textured emitter's radiance at barycentrics (b1, b2) of light-table
// entry `light`: Emission(material, HitTexcoords) * Coverage(hit)
// (scene.slang:655-657). Not inlined, as textured_inputs.
static __device__ __noinline__ F3 textured_light_radiance(const SceneView& S, uint32_t light, float b1, float b2) {
  const uint32_t instance = S.lights[light].instance;
  const InstanceShading& rec = S.inst_shade[instance];
  const uint32_t primitive = light - rec.light_offset;
  const MaterialRecord& mat = S.materials[rec.material];
  const MaterialLookups ml = S.mat_lookups[rec.material];
  float s, t;
  hit_texcoords(S, instance, ml, primitive, b1, b2, s, t);
  return material_emission(S, mat, ml, s, t) * material_coverage(S, mat, rec.material, instance, primitive, b1, b2);
}

// SampleTriangle (scene.slang:632-677), over the light table's
// world-space corners.
template <bool kFullShading = true>
__device__ __forceinline__ LightSample sample_triangle(const SceneView& S, uint32_t light,
    float pdf, float ux, float uy, F3 origin) {
  const float root = sqrtf(ux);
  const float b1 = root * (1.0f - uy), b2 = root * uy;
  const float4* lv = S.light_verts + 3 * (size_t)light;
  const F3 p0 = V(lv[0]), p1 = V(lv[1]), p2 = V(lv[2]);
  const F3 position = p0 + b1 * (p1 - p0) + b2 * (p2 - p0);
  const F3 normal = normalize(cross(p1 - p0, p2 - p0));
  const float area = triangle_area(p0, p1, p2);
  const float4 stored = S.light_radiance[light];
  F3 radiance = V(stored);
  if (kFullShading && stored.w != 0.0f) radiance = textured_light_radiance(S, light, b1, b2);
  const F3 toward = position - origin;
  const float distance2 = dot(toward, toward);
  if (!(area > 0.0f) || !(distance2 > 0.0f) || max_component(radiance) <= 0.0f) return no_light();
  LightSample s;
  s.direction = toward * rsqrt_rn(distance2);
  const float cosine = fabsf(dot(normal, s.direction));
  if (!(cosine > 0.0f)) return no_light();
  const F3 end = offset_ray_origin(position, dot(normal, s.direction) > 0.0f ? -normal : normal);
  s.distance = fmaxf(0.0f, dot(end - origin, s.direction));
  s.radiance = radiance;
  s.pdf = pdf / area * distance2 / cosine;
  s.delta = false;
  return s;
}

// FindInterval (scene.slang:775-789): the largest i in [0, count) with
// F[i] <= u. The binary search counts the entries <= u; a guide table
// (entry k: the entries <= k / K, K a power of two so k / K and u * K are
// exact) narrows it to [guide[k], guide[k + 1]] for the u of bucket k, the
// same answer as a search over all count + 1 entries.
__device__ __forceinline__ uint32_t find_interval(const float* __restrict__ F, uint64_t first,
    uint32_t count, float u, const uint32_t* __restrict__ guide, uint32_t buckets) {
  const uint32_t k = min((uint32_t)(u * float(buckets)), buckets - 1u);
  uint32_t low = guide[k], len = guide[k + 1] - guide[k];
  while (len > 0) {
    const uint32_t half = len >> 1;
    const uint32_t middle = low + half;
    if (F[first + middle] <= u) {
      low = middle + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return min(max(low, 1u), count) - 1;
}

// SampleCumulative (scene.slang:794-800).
__device__ __forceinline__ float sample_cumulative(const float* __restrict__ F, uint64_t first,
    uint32_t count, float u, uint32_t& cell, const uint32_t* __restrict__ guide, uint32_t buckets) {
  cell = find_interval(F, first, count, u, guide, buckets);
  const float low = F[first + cell];
  const float width = F[first + cell + 1] - low;
  const float offset = width > 0.0f ? (u - low) / width : 0.5f;
  return fminf((float(cell) + offset) / float(count), 0.99999994f);
}

__device__ __forceinline__ void environment_uv(F3 local, float& u, float& v) {
  const float uu = 0.5f - latan2(local.x, local.z) * (0.5f / kPi);
  v = lacos(fminf(fmaxf(local.y, -1.0f), 1.0f)) * (1.0f / kPi);
  u = uu - floorf(uu);
}

__device__ __forceinline__ F3 environment_direction(float u, float v) {
  const float theta = kPi * v;
  const float phi = kPi * (1.0f - 2.0f * u);
  float sin_theta, cos_theta, sin_phi, cos_phi;
  lsincos(theta, sin_theta, cos_theta);
  lsincos(phi, sin_phi, cos_phi);
  return V(sin_theta * sin_phi, cos_theta, sin_theta * cos_phi);
}

// EnvironmentLookup (scene.slang:819-824): FP32 bilinear filtering,
// repeating across longitude and clamped at the poles.
__device__ __forceinline__ F3 environment_lookup(const SceneView& S, float u, float v) {
  const float x = u * float(S.env_width) - 0.5f;
  const float y = v * float(S.env_height) - 0.5f;
  const float fx0 = floorf(x), fy0 = floorf(y);
  const float ax = x - fx0, ay = y - fy0;
  const int w = (int)S.env_width, h = (int)S.env_height;
  int x0 = (int)fx0 % w;
  if (x0 < 0) x0 += w;
  const int x1 = x0 + 1 == w ? 0 : x0 + 1;
  const int iy = (int)fy0;
  const int y0 = min(max(iy, 0), h - 1);
  const int y1 = min(max(iy + 1, 0), h - 1);
  const float4 t00 = S.env_texels[(size_t)y0 * w + x0];
  const float4 t10 = S.env_texels[(size_t)y0 * w + x1];
  const float4 t01 = S.env_texels[(size_t)y1 * w + x0];
  const float4 t11 = S.env_texels[(size_t)y1 * w + x1];
  const float rx = (t00.x * (1.0f - ax) + t10.x * ax) * (1.0f - ay) + (t01.x * (1.0f - ax) + t11.x * ax) * ay;
  const float ry = (t00.y * (1.0f - ax) + t10.y * ax) * (1.0f - ay) + (t01.y * (1.0f - ax) + t11.y * ax) * ay;
  const float rz = (t00.z * (1.0f - ax) + t10.z * ax) * (1.0f - ay) + (t01.z * (1.0f - ax) + t11.z * ax) * ay;
  return V(fmaxf(rx, 0.0f) * S.env_scale[0], fmaxf(ry, 0.0f) * S.env_scale[1],
      fmaxf(rz, 0.0f) * S.env_scale[2]);
}

__device__ __forceinline__ float environment_direction_pdf(const SceneView& S, float u, float v) {
  const uint32_t column = min((uint32_t)(u * float(S.env_columns)), S.env_columns - 1);
  const uint32_t row = min((uint32_t)(v * float(S.env_rows)), S.env_rows - 1);
  const float sin_theta = lsin(kPi * v);
  if (!(sin_theta > 0.0f)) return 0.0f;
  return S.env_floats[(uint64_t)row * S.env_columns + column] / (2.0f * kPi * kPi * sin_theta);
}

// SampleEnvironment (scene.slang:845-872).
__device__ __forceinline__ LightSample sample_environment(const SceneView& S, float selection,
    float ux, float uy) {
  const uint64_t cells = (uint64_t)S.env_columns * S.env_rows;
  uint32_t row, column;
  const float v = sample_cumulative(S.env_floats, cells, S.env_rows, ux, row, S.env_guide, kEnvGuideMarginal);
  const float u = sample_cumulative(S.env_floats,
      cells + S.env_rows + 1 + (uint64_t)row * (S.env_columns + 1), S.env_columns, uy, column,
      S.env_guide + (kEnvGuideMarginal + 1) + (size_t)row * (kEnvGuideConditional + 1), kEnvGuideConditional);
  const float sin_theta = lsin(kPi * v);
  const float density = S.env_floats[(uint64_t)row * S.env_columns + column];
  if (!(sin_theta > 0.0f) || !(density > 0.0f)) return no_light();
  const F3 local = environment_direction(u, v);
  const F3 r0 = V(S.env_frame[0], S.env_frame[1], S.env_frame[2]);
  const F3 r1 = V(S.env_frame[3], S.env_frame[4], S.env_frame[5]);
  const F3 r2 = V(S.env_frame[6], S.env_frame[7], S.env_frame[8]);
  LightSample s;
  s.direction = normalize(local.x * r0 + local.y * r1 + local.z * r2);
  s.distance = kFloatMax;
  s.radiance = environment_lookup(S, u, v);
  s.pdf = selection * density / (2.0f * kPi * kPi * sin_theta);
  s.delta = false;
  return s;
}

// EnvironmentRadiance (scene.slang:877-890).
__device__ __forceinline__ F3 environment_radiance(const SceneView& S, F3 direction, bool weigh,
    float pdf) {
  const F3 r0 = V(S.env_frame[0], S.env_frame[1], S.env_frame[2]);
  const F3 r1 = V(S.env_frame[3], S.env_frame[4], S.env_frame[5]);
  const F3 r2 = V(S.env_frame[6], S.env_frame[7], S.env_frame[8]);
  const F3 local = V(dot(r0, direction), dot(r1, direction), dot(r2, direction));
  float u, v;
  environment_uv(local, u, v);
  const F3 radiance = environment_lookup(S, u, v);
  if (!weigh || !(S.env_selection > 0.0f)) return radiance;
  return radiance * power_heuristic(pdf, S.env_selection * environment_direction_pdf(S, u, v));
}

// SampleConcentricDisk (sampling.slang:89-104): Shirley and Chiu's map of
// the square onto the unit disk.
__device__ __forceinline__ void sample_concentric_disk(float ux, float uy, float& a, float& b) {
  const float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
  if (ox == 0.0f && oy == 0.0f) {
    a = b = 0.0f;
    return;
  }
  float radius, theta;
  if (fabsf(ox) > fabsf(oy)) {
    radius = ox;
    theta = 0.25f * kPi * (oy / ox);
  } else {
    radius = oy;
    theta = 0.5f * kPi - 0.25f * kPi * (ox / oy);
  }
  float sn, cs;
  lsincos(theta, sn, cs);
  a = radius * cs;
  b = radius * sn;
}

// SampleUniformCone (sampling.slang:109-116), about +z.
__device__ __forceinline__ F3 sample_uniform_cone(float ux, float uy, float one_minus_cos_max) {
  const float one_minus_cos = ux * one_minus_cos_max;
  const float sin_theta = sqrtf(fmaxf(0.0f, one_minus_cos * (2.0f - one_minus_cos)));
  const float phi = 2.0f * kPi * uy;
  float sn, cs;
  lsincos(phi, sn, cs);
  return V(sin_theta * cs, sin_theta * sn, 1.0f - one_minus_cos);
}

// SphereConePdf (scene.slang:683-690): the solid-angle density of a
// sphere's cone, 1 - cos(theta_max) without cancellation for small spheres.
__device__ __forceinline__ float sphere_cone_pdf(float sin2_max) {
  const float one_minus_cos = sin2_max < 0.00068523f ? 0.5f * sin2_max
                                                     : 1.0f - sqrtf(fmaxf(0.0f, 1.0f - sin2_max));
  return 1.0f / (2.0f * kPi * one_minus_cos);
}

// SampleAnalytic (scene.slang:695-768): a sphere by solid angle over its
// cone (PBRT 4th ed. 6.2.4), a rect or disk by area, a distant light over
// its cone, a parallel light along its direction (a delta light).
__device__ __forceinline__ LightSample sample_analytic(const AnalyticLight& light, float selection,
    float ux, float uy, F3 origin) {
  LightSample s = no_light();
  s.radiance = V(light.radiance);
  if (light.shape == kSphereLight) {
    const F3 centre = V(light.position);
    const float radius = light.position.w;
    const F3 to_centre = centre - origin;
    const float distance2 = dot(to_centre, to_centre);
    if (!(distance2 > radius * radius)) return no_light();
    const float sin2_max = radius * radius / distance2;
    const float sin_max = sqrtf(sin2_max);
    const float cos_max = sqrtf(fmaxf(0.0f, 1.0f - sin2_max));
    float cos_theta = (cos_max - 1.0f) * ux + 1.0f;
    float sin2_theta = 1.0f - cos_theta * cos_theta;
    if (sin2_max < 0.00068523f) {
      sin2_theta = sin2_max * ux;
      cos_theta = sqrtf(1.0f - sin2_theta);
    }
    const float cos_alpha = sin2_theta / sin_max + cos_theta * sqrtf(fmaxf(0.0f, 1.0f - sin2_theta / sin2_max));
    const float sin_alpha = sqrtf(fmaxf(0.0f, 1.0f - cos_alpha * cos_alpha));
    const float phi = 2.0f * kPi * uy;
    float sn, cs;
    lsincos(phi, sn, cs);
    const Frame frame = make_frame(normalize(to_centre));
    const F3 outward = frame.to_world(-V(sin_alpha * cs, sin_alpha * sn, cos_alpha));
    const F3 toward = centre + radius * outward - origin;
    s.distance = length(toward);
    s.direction = toward / s.distance;
    s.pdf = selection * sphere_cone_pdf(sin2_max);
  } else if (light.shape == kRectLight || light.shape == kDiskLight) {
    float a, b;
    if (light.shape == kRectLight) {
      a = 2.0f * ux - 1.0f;
      b = 2.0f * uy - 1.0f;
    } else {
      sample_concentric_disk(ux, uy, a, b);
    }
    const F3 toward = V(light.position) + a * V(light.axis_u) + b * V(light.axis_v) - origin;
    const float distance2 = dot(toward, toward);
    if (!(distance2 > 0.0f)) return no_light();
    s.distance = sqrtf(distance2);
    s.direction = toward / s.distance;
    const float cosine = -dot(V(light.normal), s.direction);
    if (!(cosine > 0.0f)) return no_light();
    s.pdf = selection * distance2 / (cosine * light.normal.w);
  } else if (light.shape == kDistantLight) {
    const Frame frame = make_frame(V(light.axis_u));
    s.direction = normalize(frame.to_world(sample_uniform_cone(ux, uy, light.axis_u.w)));
    s.distance = kFloatMax;
    s.pdf = selection / (2.0f * kPi * light.axis_u.w);
  } else {
    s.direction = V(light.axis_u);
    s.distance = kFloatMax;
    s.pdf = selection;
    s.delta = true;
  }
  return s;
}

// ParallelLight (scene.slang:986-1000): a parallel light's direction and
// irradiance as a delta light of density 1; no light for other shapes.
__device__ __forceinline__ LightSample parallel_light(const SceneView& S, uint32_t index) {
  const AnalyticLight& light = S.analytic[index];
  if (light.shape != kParallelLight) return no_light();
  LightSample s;
  s.direction = V(light.axis_u);
  s.distance = kFloatMax;
  s.radiance = V(light.radiance);
  s.pdf = 1.0f;
  s.delta = true;
  return s;
}

// CrossedLight (scene.slang:1019-1091): the emission of analytic light
// `index` if the ray crosses it before `distance` (a sphere's near side
// from outside it, by the nearer root without cancellation; a rect's or
// disk's emitting side; a distant light's cone for an escaping ray),
// weighed against light sampling's density when `weigh`.
__device__ __forceinline__ F3 crossed_light(const SceneView& S, uint32_t index, F3 origin, F3 direction,
    float distance, bool escaped, bool weigh, float pdf) {
  const AnalyticLight& light = S.analytic[index];
  const uint32_t shape = light.shape;
  float light_pdf = 0.0f;
  if (shape == kSphereLight) {
    const float radius = light.position.w;
    const F3 offset = origin - V(light.position);
    const float c = dot(offset, offset) - radius * radius;
    const float b = -dot(offset, direction);
    const F3 perpendicular = offset + b * direction;
    const float discriminant = radius * radius - dot(perpendicular, perpendicular);
    if (!(c > 0.0f) || !(b > 0.0f) || discriminant < 0.0f) return V(0.0f);
    const float t = c / (b + sqrtf(discriminant));
    if (!(t < distance)) return V(0.0f);
    light_pdf = sphere_cone_pdf(radius * radius / dot(offset, offset));
  } else if (shape == kRectLight || shape == kDiskLight) {
    const F3 n = V(light.normal);
    const float facing = dot(direction, n);
    if (!(facing < 0.0f)) return V(0.0f);
    const float t = dot(V(light.position) - origin, n) / facing;
    if (!(t > 0.0f) || !(t < distance)) return V(0.0f);
    const F3 q = origin + t * direction - V(light.position);
    const F3 u = V(light.axis_u), v = V(light.axis_v);
    const float uu = dot(u, u), uv = dot(u, v), vv = dot(v, v);
    const float qu = dot(q, u), qv = dot(q, v);
    const float determinant = uu * vv - uv * uv;
    const float a = (qu * vv - qv * uv) / determinant;
    const float b = (qv * uu - qu * uv) / determinant;
    if (shape == kRectLight ? !(fabsf(a) <= 1.0f && fabsf(b) <= 1.0f) : !(a * a + b * b <= 1.0f)) return V(0.0f);
    light_pdf = t * t / (-facing * light.normal.w);
  } else if (shape == kDistantLight && escaped) {
    const F3 toward = V(light.axis_u);
    const float one_minus_cos = light.axis_u.w;
    const float cosine = dot(direction, toward);
    if (one_minus_cos <= 1.0f) {
      const F3 across = cross(direction, toward);
      if (!(cosine > 0.0f) || !(dot(across, across) <= one_minus_cos * (2.0f - one_minus_cos))) return V(0.0f);
    } else if (!(cosine >= 1.0f - one_minus_cos)) {
      return V(0.0f);
    }
    light_pdf = 1.0f / (2.0f * kPi * one_minus_cos);
  } else {
    return V(0.0f);
  }
  const float weight = weigh ? power_heuristic(pdf, light.radiance.w * light_pdf) : 1.0f;
  return V(light.radiance) * weight;
}

// OverlapsBox (scene.slang:1095-1103).
__device__ __forceinline__ bool overlaps_box(float4 low, float4 high, F3 origin, F3 inverse, float distance) {
  const float t0x = (low.x - origin.x) * inverse.x, t1x = (high.x - origin.x) * inverse.x;
  const float t0y = (low.y - origin.y) * inverse.y, t1y = (high.y - origin.y) * inverse.y;
  const float t0z = (low.z - origin.z) * inverse.z, t1z = (high.z - origin.z) * inverse.z;
  const float nx = fminf(t0x, t1x), ny = fminf(t0y, t1y), nz = fminf(t0z, t1z);
  const float fx = fmaxf(t0x, t1x), fy = fmaxf(t0y, t1y), fz = fmaxf(t0z, t1z);
  return fmaxf(fmaxf(nx, ny), fmaxf(nz, 0.0f)) <= fminf(fminf(fx, fy), fminf(fz, distance));
}

// CrossedLights (scene.slang:1110-1178): the analytic lights the ray
// crosses before `distance`, summed in the crossing hierarchy's traversal
// order (child 0 before child 1, the second of two interior children
// stacked), then, for an escaping ray, the distant lights. Lights neither
// block rays nor each other.
static __device__ __noinline__ F3 crossed_lights(const SceneView& S, F3 origin, F3 direction, float distance,
    bool escaped, bool weigh, float pdf) {
  F3 sum = V(0.0f);
  if (S.light_node_count != 0) {
    const F3 inverse = safe_inverse(direction);
    uint32_t stack[kLightStackSize];
    uint32_t depth = 0, node = 0;
    // A hierarchy of n nodes is walked in at most n steps.
    for (uint32_t step = 0; step < S.light_node_count; ++step) {
      const LightNode current = S.light_nodes[node];
      const uint32_t child0 = __float_as_uint(current.low0.w);
      const uint32_t child1 = __float_as_uint(current.low1.w);
      const bool enter0 = overlaps_box(current.low0, current.high0, origin, inverse, distance);
      const bool enter1 =
          child1 != kNoLightChild && overlaps_box(current.low1, current.high1, origin, inverse, distance);
      uint32_t next = 0xFFFFFFFFu;
      if (enter0) {
        if ((child0 & kLightLeaf) != 0)
          sum = sum + crossed_light(S, child0 & ~kLightLeaf, origin, direction, distance, escaped, weigh, pdf);
        else
          next = child0;
      }
      if (enter1) {
        if ((child1 & kLightLeaf) != 0)
          sum = sum + crossed_light(S, child1 & ~kLightLeaf, origin, direction, distance, escaped, weigh, pdf);
        else if (next == 0xFFFFFFFFu)
          next = child1;
        else if (depth < kLightStackSize)
          stack[depth++] = child1;
      }
      if (next == 0xFFFFFFFFu) {
        if (depth == 0) break;
        next = stack[--depth];
      }
      node = next;
    }
  }
  if (escaped)
    for (uint32_t i = 0; i < S.distant_count; ++i)
      sum = sum + crossed_light(S, S.distant[i], origin, direction, distance, escaped, weigh, pdf);
  return sum;
}

// SampleLight (scene.slang:894-909): Vose's alias table, then a point.
// kAnalytic = false leaves out the analytic lights' code, for scenes
// without them.
template <bool kAnalytic = true, bool kFullShading = true>
__device__ __forceinline__ LightSample sample_light(const SceneView& S, float u0, float u1,
    float u2, float u3, F3 origin) {
  const uint32_t count = S.light_count;
  const uint32_t column = min((uint32_t)(u0 * float(count)), count - 1);
  const LightRecord record = S.lights[column];
  const uint32_t light = u1 < record.threshold ? column : record.alias;
  const LightRecord chosen = S.lights[light];
  if (chosen.instance == kEnvironmentLight) return sample_environment(S, chosen.pdf, u2, u3);
  if (kAnalytic && (chosen.instance & kAnalyticLight) != 0)
    return sample_analytic(S.analytic[chosen.instance & ~kAnalyticLight], chosen.pdf, u2, u3, origin);
  return sample_triangle<kFullShading>(S, light, chosen.pdf, u2, u3, origin);
}

// EmitterPdf (scene.slang:1004-1010).
__device__ __forceinline__ float emitter_pdf(const SceneView& S, uint32_t instance,
    uint32_t primitive, float area) {
  const uint32_t first = S.inst_shade[instance].light_offset;
  if (first == kNoLights || !(area > 0.0f)) return 0.0f;
  return S.lights[first + primitive].pdf / area;
}

// A primary-hit record's instance for a camera ray that hit nothing.
constexpr uint32_t kNoPrimaryHit = 0xFFFFFFFFu;

// The frame's camera and target, set per RenderScene call; sample_index
// and accumulated advance on the device between samples.
struct FrameConst {
  float clip_to_world[16];
  float world_to_clip[16];  // Vulkan clip (the depth product's projection)
  float ndc[4];
  float background[4];
  uint32_t width, height;
  uint32_t rect[4];
  uint32_t max_bounces;
  uint32_t sample_lights;
  uint32_t sample_index;
  uint32_t accumulated;
  uint32_t add_sample;
  uint32_t environment_background;
  // RestirInitial: the depth-0 direct light is the final reservoir's
  // (restir_final: RestirPixel records `restir_stride` bytes apart).
  uint32_t restir_primary;
  uint32_t restir_stride;
  const unsigned char* restir_final;
  // The primary hits of sample `primary_sample`, when a pass before it
  // (ReSTIR's initial reservoirs) traced the same camera rays: per pixel
  // (instance, triangle, b1, b2), instance ~0 for a miss, and the path's
  // random state after the trace. Null otherwise.
  const uint4* primary_hit;
  const uint32_t* primary_rng;
  uint32_t primary_sample;
  // The wavefront's samples: `wave` consecutive samples from sample_index
  // (0 counts as 1), sample k's paths in the slots k * wave_stride + pixel.
  uint32_t wave;
  uint32_t wave_stride;
};

// CameraRay (scene.slang:273-283).
__device__ __forceinline__ void camera_ray(const FrameConst& f, float nx, float ny, F3& origin,
    F3& direction, float& tmax) {
  const float* c = f.clip_to_world;
  float n[4], a[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    n[r] = c[r] * nx + c[4 + r] * ny + c[8 + r] * 0.0f + c[12 + r] * 1.0f;
    a[r] = c[r] * nx + c[4 + r] * ny + c[8 + r] * 1.0f + c[12 + r] * 1.0f;
  }
  origin = V(n[0] / n[3], n[1] / n[3], n[2] / n[3]);
  direction = normalize(V(a[0], a[1], a[2]) * n[3] - V(n[0], n[1], n[2]) * a[3]);
  tmax = a[3] == 0.0f ? kFloatMax : length(V(a[0] / a[3], a[1] / a[3], a[2] / a[3]) - origin);
}

constexpr uint32_t kUnweightedLight = 1;
constexpr uint32_t kRouletteBounces = 3;
constexpr float kMaxSurvival = 0.95f;

// StartPath (transport.slang:53-69): the camera ray through a uniformly
// distributed point of the pixel, and the path's random state after it.
__device__ __forceinline__ void start_path(const FrameConst& f, uint32_t px, uint32_t py,
    uint32_t sample_index, F3& origin, F3& direction, float& tmax, uint32_t& rng) {
  const uint32_t pixel_index = py * f.width + px;
  rng = seed_random(pixel_index, sample_index);
  const float ux = next_random(rng);
  const float uy = next_random(rng);
  const float film_x = float(px) + 0.5f + (ux - 0.5f);
  const float film_y = float(py) + 0.5f + (uy - 0.5f);
  camera_ray(f, film_x * f.ndc[0] + f.ndc[2], film_y * f.ndc[1] + f.ndc[3], origin, direction, tmax);
}

}  // namespace lotus
