"""Scene descriptions and the seeded synthetic workloads.

A ``Scene`` holds numpy arrays in the layout of include/lotus_cuda.h and
turns them into a ``lotus_scene_desc`` that both the CUDA library and the
oracle read. The workloads are procedural and seeded; no dataset is used:

- ``cornell_reference``: the reference's own Cornell box fixture
  (adapters/common/reference.cpp:221-279 in hydra-lotus), which its golden
  images validation/reference/cornell-box-{mean,variance}.pfm were rendered
  from. Used to pin the oracle and the kernels against those images.
- ``box_room``: the small box room workload (36 triangles, 256x256).
- ``sphere_field``: the 1080p workload of 4096 instanced, Perlin-displaced
  icospheres over a 100x100 ground grid with 64 emissive triangles and an
  importance-sampled 2048x1024 sky.
"""

import ctypes as C
import math

import numpy as np

from . import abi

F32 = np.float32


# ---------------------------------------------------------------------------
# Matrices (column-major 4x4 floats, Lotus::Matrix4)

def identity():
    return np.eye(4, dtype=F32).reshape(-1, order="F")


def multiply(left, right):
    """Multiply (render_world.cpp:288-300): float sums in the same order."""
    left = np.asarray(left, dtype=F32)
    right = np.asarray(right, dtype=F32)
    out = np.zeros(16, dtype=F32)
    for column in range(4):
        for row in range(4):
            s = F32(0.0)
            for index in range(4):
                s = F32(s + F32(left[index * 4 + row] * right[column * 4 + index]))
            out[column * 4 + row] = s
    return out


def perspective(fovy_degrees, aspect, near, far):
    """OpenGL projection, column-major."""
    f = 1.0 / math.tan(math.radians(fovy_degrees) / 2.0)
    m = np.zeros(16, dtype=F32)
    m[0] = f / aspect
    m[5] = f
    m[10] = (far + near) / (near - far)
    m[11] = -1.0
    m[14] = 2.0 * far * near / (near - far)
    return m


def look_at(eye, target, up=(0.0, 1.0, 0.0)):
    """World to a right-handed view space looking down -Z, column-major."""
    eye = np.asarray(eye, dtype=np.float64)
    forward = np.asarray(target, dtype=np.float64) - eye
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(up, dtype=np.float64))
    right /= np.linalg.norm(right)
    true_up = np.cross(right, forward)
    rot = np.stack([right, true_up, -forward])  # rows
    m = np.eye(4)
    m[:3, :3] = rot
    m[:3, 3] = -rot @ eye
    return m.astype(F32).reshape(-1, order="F")


def affine(linear=None, translation=(0.0, 0.0, 0.0)):
    m = np.eye(4, dtype=np.float64)
    if linear is not None:
        m[:3, :3] = linear
    m[:3, 3] = translation
    return m.astype(F32).reshape(-1, order="F")


def rotation_y(radians):
    c, s = math.cos(radians), math.sin(radians)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], dtype=np.float64)


def rotation_xyz(rx, ry, rz):
    cx, sx = math.cos(rx), math.sin(rx)
    cy, sy = math.cos(ry), math.sin(ry)
    cz, sz = math.cos(rz), math.sin(rz)
    x = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    y = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    z = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return z @ y @ x


# ---------------------------------------------------------------------------
# Scene

def preview_material(base_color=(0.18, 0.18, 0.18), roughness=0.5, metallic=0.0,
                     ior=1.5, emission=(0.0, 0.0, 0.0), specular_color=(0.0, 0.0, 0.0),
                     transmission=0.0, transmission_color=(1.0, 1.0, 1.0),
                     opacity=1.0, opacity_threshold=0.0, flags=0):
    """UsdPreviewSurface with its defaults (material.hpp:137-173)."""
    m = abi.Material()
    m.base_color[:] = [float(v) for v in base_color]
    m.roughness = roughness
    m.metallic = metallic
    m.ior = ior
    m.emission[:] = [float(v) for v in emission]
    m.specular_color[:] = [float(v) for v in specular_color]
    m.transmission = transmission
    m.transmission_color[:] = [float(v) for v in transmission_color]
    m.opacity = opacity
    m.opacity_threshold = opacity_threshold
    m.flags = flags
    return m


def gltf_material(base_color=(1.0, 1.0, 1.0), metallic=1.0, roughness=1.0, emissive=(0.0, 0.0, 0.0),
                  emissive_strength=1.0, ior=1.5, specular=1.0, specular_color=(1.0, 1.0, 1.0),
                  transmission=0.0, clearcoat=0.0, clearcoat_roughness=0.0, sheen_color=(0.0, 0.0, 0.0),
                  sheen_roughness=0.0, opacity=1.0, opacity_threshold=0.0):
    """MaterialX's glTF PBR surface with the definition's defaults, a rough
    white metal (GltfPbr, material.hpp:180-217)."""
    m = abi.Material()
    m.model = abi.MODEL_GLTF_PBR
    m.base_color[:] = [float(v) for v in base_color]
    m.metallic = metallic
    m.roughness = roughness
    m.emission[:] = [float(v) for v in emissive]
    m.emissive_strength = emissive_strength
    m.ior = ior
    m.specular = specular
    m.specular_color[:] = [float(v) for v in specular_color]
    m.transmission = transmission
    m.clearcoat = clearcoat
    m.clearcoat_roughness = clearcoat_roughness
    m.sheen_color[:] = [float(v) for v in sheen_color]
    m.sheen_roughness = sheen_roughness
    m.opacity = opacity
    m.opacity_threshold = opacity_threshold
    return m


class Scene:
    """A scene in the C ABI's layout, plus its camera and target size."""

    def __init__(self, name="scene"):
        self.name = name
        self.geometries = []
        self.instances = []
        self.materials = [preview_material()]  # slot 0: the default material
        self.environment = None
        self.environment_constant = (0.0, 0.0, 0.0)
        self.lights = []  # analytic lights (abi.Light)
        self.world_to_clip = identity()
        self.view = None  # world to view space, when the temporal passes need it
        self.width = 0
        self.height = 0
        # Texture lookups: per geometry its texture-coordinate sets
        # (sets, triangles, 3 corners, 2); per instance the set its material
        # reads (k > 0: set k - 1; 0 or absent: the material's fallback); the
        # images (rows from the top) with their LOTUS_TEXTURE_* formats; the
        # texture inputs.
        self.texcoords = {}
        self.instance_texcoords = {}
        self.colors = {}            # geometry -> (flat RGB array, per-set value counts)
        self.instance_colors = {}
        self.textures = []
        self.texture_inputs = []
        self._desc = None

    def add_texture(self, texels, fmt):
        """An image (H, W, 4): uint8 for abi.TEXTURE_RGBA8_UNORM / _SRGB,
        float32 for abi.TEXTURE_RGBA32_FLOAT. Returns the reference a
        texture input names it by (its index + 1)."""
        dtype = F32 if fmt == abi.TEXTURE_RGBA32_FLOAT else np.uint8
        texels = np.ascontiguousarray(texels, dtype=dtype)
        assert texels.ndim == 3 and texels.shape[2] == 4
        self.textures.append((texels, fmt))
        self._desc = None
        return len(self.textures)

    def add_texture_input(self, texture=0, channel=0, wrap_s=abi.WRAP_BLACK, wrap_t=abi.WRAP_BLACK,
                          scale=(1.0, 1.0, 1.0, 1.0), bias=(0.0, 0.0, 0.0, 0.0), fallback=(0.0, 0.0, 0.0, 1.0),
                          st_transform=(1.0, 0.0, 0.0, 0.0, 1.0, 0.0)):
        """A texture input (TextureInput, material.hpp:52-74); `texture` is
        add_texture's reference (0: none, the lookup returns `fallback`).
        Returns the reference a material slot names it by (index + 1)."""
        t = abi.TextureInput()
        t.texture, t.channel, t.wrap_s, t.wrap_t = texture, channel, wrap_s, wrap_t
        t.scale[:] = [float(v) for v in scale]
        t.bias[:] = [float(v) for v in bias]
        t.fallback[:] = [float(v) for v in fallback]
        t.st_transform[:] = [float(v) for v in st_transform]
        self.texture_inputs.append(t)
        self._desc = None
        return len(self.texture_inputs)

    def set_colors(self, geometry, sets):
        """Geometry `geometry`'s colour sets (MeshGeometry::colors, in key
        order): each an array of RGB, one per triangle corner (triangle by
        triangle) or one for the whole mesh."""
        arrays = [np.ascontiguousarray(c, dtype=F32).reshape(-1, 3) for c in sets]
        counts = np.array([a.shape[0] for a in arrays], dtype=np.uint32)
        self.colors[geometry] = (np.ascontiguousarray(np.concatenate(arrays).reshape(-1)), counts)
        self._desc = None

    def set_texcoords(self, geometry, sets):
        """Geometry `geometry`'s texture-coordinate sets: (sets, triangles,
        3, 2) per-corner (s, t)."""
        sets = np.ascontiguousarray(sets, dtype=F32)
        assert sets.ndim == 4 and sets.shape[1:] == (self.geometries[geometry][1].shape[0], 3, 2)
        self.texcoords[geometry] = sets
        self._desc = None

    def add_geometry(self, positions, triangles, normals=None):
        positions = np.ascontiguousarray(positions, dtype=F32).reshape(-1, 3)
        triangles = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        if normals is not None:
            normals = np.ascontiguousarray(normals, dtype=F32).reshape(-1, 3, 3)
        self.geometries.append((positions, triangles, normals))
        self._desc = None
        return len(self.geometries) - 1

    def add_material(self, material):
        self.materials.append(material)
        self._desc = None
        return len(self.materials) - 1

    def add_instance(self, geometry, material, world_from_object=None, texcoord_set=0, color_set=0):
        m = identity() if world_from_object is None else np.asarray(world_from_object, dtype=F32)
        self.instances.append((m.copy(), geometry, material))
        if texcoord_set:
            self.instance_texcoords[len(self.instances) - 1] = texcoord_set
        if color_set:
            self.instance_colors[len(self.instances) - 1] = color_set
        self._desc = None
        return len(self.instances) - 1

    def set_instance(self, index, world_from_object=None, material=None):
        """Edits instance `index`: its transform and/or material slot."""
        m, g, mat = self.instances[index]
        if world_from_object is not None:
            m = np.asarray(world_from_object, dtype=F32).copy()
        self.instances[index] = (m, g, mat if material is None else material)
        self._desc = None

    def set_positions(self, geometry, positions, normals=None):
        """A point edit of `geometry`: new positions (same vertex count) and,
        when it has corner normals, new ones."""
        p, t, n = self.geometries[geometry]
        positions = np.ascontiguousarray(positions, dtype=F32).reshape(-1, 3)
        assert positions.shape == p.shape
        if normals is not None:
            normals = np.ascontiguousarray(normals, dtype=F32).reshape(-1, 3, 3)
        self.geometries[geometry] = (positions, t, normals if n is not None else None)
        self._desc = None

    def add_light(self, shape, world_from_light=None, radiance=(1.0, 1.0, 1.0), normalize=False,
                  radius=0.5, width=1.0, height=1.0, angle=0.53):
        """An analytic light (Lotus::Light): abi.LIGHT_SPHERE, _RECT, _DISK or
        _DISTANT, in the frame `world_from_light` (column-major)."""
        light = abi.Light()
        light.shape = shape
        light.normalize = 1 if normalize else 0
        m = identity() if world_from_light is None else np.asarray(world_from_light, dtype=F32)
        light.world_from_light[:] = [float(v) for v in m.reshape(-1)]
        light.radiance[:] = [float(v) for v in radiance]
        light.radius, light.width, light.height, light.angle = radius, width, height, angle
        self.lights.append(light)
        self._desc = None
        return len(self.lights) - 1

    def set_environment(self, texels, scale=(1.0, 1.0, 1.0), rows=None):
        texels = np.ascontiguousarray(texels, dtype=F32)
        assert texels.ndim == 3 and texels.shape[2] == 4
        rows = np.eye(3, dtype=F32) if rows is None else np.asarray(rows, dtype=F32)
        self.environment = (texels, tuple(scale), rows)
        self._desc = None

    @property
    def triangle_count(self):
        return sum(int(t.shape[0]) for _, t, _ in self.geometries)

    @property
    def traced_triangle_count(self):
        return sum(int(self.geometries[g][1].shape[0]) for _, g, _ in self.instances)

    def desc(self):
        """The lotus_scene_desc; the Scene keeps its arrays alive."""
        if self._desc is not None:
            return self._desc
        geos = (abi.Geometry * max(1, len(self.geometries)))()
        for i, (p, t, n) in enumerate(self.geometries):
            geos[i].positions = p.ctypes.data_as(C.POINTER(C.c_float))
            geos[i].triangles = t.ctypes.data_as(C.POINTER(C.c_uint32))
            geos[i].normals = (n.ctypes.data_as(C.POINTER(C.c_float)) if n is not None
                               else C.POINTER(C.c_float)())
            geos[i].vertex_count = p.shape[0]
            geos[i].triangle_count = t.shape[0]
            if i in self.texcoords:
                geos[i].texcoords = self.texcoords[i].ctypes.data_as(C.POINTER(C.c_float))
                geos[i].texcoord_sets = self.texcoords[i].shape[0]
            if i in self.colors:
                values, counts = self.colors[i]
                geos[i].colors = values.ctypes.data_as(C.POINTER(C.c_float))
                geos[i].color_counts = counts.ctypes.data_as(C.POINTER(C.c_uint32))
                geos[i].color_sets = counts.shape[0]
        insts = (abi.Instance * max(1, len(self.instances)))()
        for i, (m, g, mat) in enumerate(self.instances):
            insts[i].world_from_object[:] = [float(v) for v in m]
            insts[i].geometry = g
            insts[i].material = mat
            insts[i].texcoord_set = self.instance_texcoords.get(i, 0)
            insts[i].color_set = self.instance_colors.get(i, 0)
        mats = (abi.Material * len(self.materials))(*self.materials)
        d = abi.SceneDesc()
        d.geometries = geos
        d.instances = insts
        d.materials = mats
        d.geometry_count = len(self.geometries)
        d.instance_count = len(self.instances)
        d.material_count = len(self.materials)
        d.environment_constant[:] = [float(v) for v in self.environment_constant]
        env = None
        if self.environment is not None:
            texels, scale, rows = self.environment
            env = abi.Environment()
            env.texels = texels.ctypes.data_as(C.POINTER(C.c_float))
            env.height, env.width = texels.shape[0], texels.shape[1]
            env.scale[:] = [float(v) for v in scale]
            env.environment_from_world[:] = [float(v) for v in rows.reshape(-1)]
            d.environment = C.pointer(env)
        lights = None
        if self.lights:
            lights = (abi.Light * len(self.lights))(*self.lights)
            d.lights = lights
            d.light_count = len(self.lights)
        textures = inputs = None
        if self.textures:
            textures = (abi.Texture * len(self.textures))()
            for i, (texels, fmt) in enumerate(self.textures):
                textures[i].texels = texels.ctypes.data
                textures[i].height, textures[i].width = texels.shape[0], texels.shape[1]
                textures[i].format = fmt
            d.textures = textures
            d.texture_count = len(self.textures)
        if self.texture_inputs:
            inputs = (abi.TextureInput * len(self.texture_inputs))(*self.texture_inputs)
            d.texture_inputs = inputs
            d.texture_input_count = len(self.texture_inputs)
        self._keep = (geos, insts, mats, env, lights, textures, inputs)
        self._desc = d
        return d

    def frame(self, settings=None, frame_count=1, **kw):
        return abi.make_frame(self.world_to_clip, self.width, self.height, settings,
                              frame_count, **kw)


# ---------------------------------------------------------------------------
# Meshes

def quad(corners):
    """Quad (reference.cpp:24-31): four corners around it, two triangles."""
    return np.asarray(corners, dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)


def unit_cube():
    """UnitCube (reference.cpp:33-43)."""
    p = np.array([[-.5, -.5, -.5], [.5, -.5, -.5], [.5, .5, -.5], [-.5, .5, -.5],
                  [-.5, -.5, .5], [.5, -.5, .5], [.5, .5, .5], [-.5, .5, .5]], dtype=F32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 7, 6], [3, 6, 2], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]],
                 dtype=np.uint32)
    return p, t


def block(size, degrees, centre):
    """Block (reference.cpp:45-56): scale the unit cube, turn it about +Y,
    move it."""
    radians = degrees * 3.14159265358979323846 / 180.0
    c = F32(math.cos(radians))
    s = F32(math.sin(radians))
    sx, sy, sz = (F32(v) for v in size)
    return np.array([c * sx, 0, -s * sx, 0, 0, sy, 0, 0, s * sz, 0, c * sz, 0,
                     centre[0], centre[1], centre[2], 1], dtype=F32)


def icosphere(subdivisions):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9),
             (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2),
             (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
             (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, dtype=np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        edges.sort(axis=1)
        unique, inverse = np.unique(edges, axis=0, return_inverse=True)
        mids = v[unique[:, 0]] + v[unique[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mids])
        n = f.shape[0]
        inverse = inverse.reshape(-1)
        a = base + inverse[:n]
        b = base + inverse[n:2 * n]
        c = base + inverse[2 * n:]
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
                            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)])
    return v, f.astype(np.uint32)


def perlin3(points, seed):
    """Perlin's improved gradient noise (SIGGRAPH 2002) at (N, 3) points."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256)
    perm = np.concatenate([perm, perm])
    grads = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1],
                      [1, 0, -1], [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]],
                     dtype=np.float64)
    p = np.asarray(points, dtype=np.float64)
    cell = np.floor(p).astype(np.int64)
    frac = p - cell
    cell &= 255
    fade = frac * frac * frac * (frac * (frac * 6 - 15) + 10)
    result = np.zeros(p.shape[0])
    for corner in range(8):
        o = np.array([(corner >> 0) & 1, (corner >> 1) & 1, (corner >> 2) & 1])
        c = (cell + o) & 255
        h = perm[perm[perm[c[:, 0]] + c[:, 1]] + c[:, 2]] % 12
        d = frac - o
        dotp = np.sum(grads[h] * d, axis=1)
        w = np.prod(np.where(o == 1, fade, 1 - fade), axis=1)
        result += w * dotp
    return result


def corner_normals(positions, triangles):
    """Smooth (area-weighted) vertex normals, one per triangle corner."""
    p = positions.astype(np.float64)
    t = triangles.astype(np.int64)
    face = np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]])
    vn = np.zeros_like(p)
    for k in range(3):
        np.add.at(vn, t[:, k], face)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    return vn[t].astype(F32)


# ---------------------------------------------------------------------------
# Workloads

CORNELL_WHITE = (0.73, 0.73, 0.73)
CORNELL_RED = (0.63, 0.065, 0.05)
CORNELL_GREEN = (0.14, 0.45, 0.091)


def cornell_camera():
    """The bootstrap camera of SetCornellBox (reference.cpp:222-237)."""
    focal, near, far = F32(2.41421356), F32(1.0), F32(10.0)
    view = identity()
    view[14] = -3.0
    projection = np.array([focal, 0, 0, 0, 0, focal, 0, 0,
                           0, 0, (far + near) / (near - far), -1,
                           0, 0, F32(2.0) * far * near / (near - far), 0], dtype=F32)
    return multiply(projection, view)


def cornell_reference(red_scale=1.0, size=128):
    """The reference's Cornell box fixture (reference.cpp:221-279): coated
    diffuse walls (ior 1.5, roughness 0.5), a GGX metal block, a coated
    white block and an emitter under the ceiling; black environment.
    ``red_scale`` scales the red wall's albedo (SetCornellRedWall, the
    comparison's negative control)."""
    s = Scene("cornell-reference")
    white = s.add_material(preview_material(CORNELL_WHITE))
    red = s.add_material(preview_material(tuple(F32(c * red_scale) for c in CORNELL_RED)))
    green = s.add_material(preview_material(CORNELL_GREEN))
    for corners, mat in [
        ([[-1, -1, 1], [1, -1, 1], [1, -1, -1], [-1, -1, -1]], white),   # floor
        ([[-1, 1, 1], [-1, 1, -1], [1, 1, -1], [1, 1, 1]], white),       # ceiling
        ([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1]], white),   # back
        ([[-1, -1, 1], [-1, -1, -1], [-1, 1, -1], [-1, 1, 1]], red),     # left
        ([[1, -1, -1], [1, -1, 1], [1, 1, 1], [1, 1, -1]], green),       # right
    ]:
        s.add_instance(s.add_geometry(*quad(corners)), mat)
    light = s.add_material(preview_material((0.0, 0.0, 0.0), emission=(15.0, 13.0, 10.0)))
    s.add_instance(s.add_geometry(*quad([[-0.35, 0.98, 0.35], [-0.35, 0.98, -0.35],
                                         [0.35, 0.98, -0.35], [0.35, 0.98, 0.35]])), light)
    metal = s.add_material(preview_material((0.95, 0.85, 0.6), roughness=0.35, metallic=1.0))
    cube = s.add_geometry(*unit_cube())
    s.add_instance(cube, metal, block((0.6, 1.2, 0.6), 17.0, (-0.35, -0.399, -0.3)))
    cube2 = s.add_geometry(*unit_cube())
    s.add_instance(cube2, white, block((0.6, 0.6, 0.6), -18.0, (0.38, -0.699, 0.3)))
    s.world_to_clip = cornell_camera()
    s.width = s.height = size
    return s


def cornell_gltf(size=128):
    """The reference's cornell-gltf-v1 benchmark workload (MakeWorkload,
    adapters/common/workloads.cpp:104-122 in hydra-lotus): the Cornell box
    with every material MaterialX's glTF PBR of the same base colour,
    roughness, metallic and emission, the rest at the definition's
    defaults."""
    s = cornell_reference(size=size)
    s.name = "cornell-gltf"
    for k, m in enumerate(s.materials):
        s.materials[k] = gltf_material(tuple(m.base_color), metallic=m.metallic, roughness=m.roughness,
                                       emissive=tuple(m.emission))
    s._desc = None
    return s


def box_room(seed=0, size=256):
    """The seeded box room: 10 wall triangles (floor, ceiling, back, left,
    right; open front), two boxes of 12 triangles with a y-rotation in
    [0, pi) and sides in [0.2, 0.6], resting on the floor, and a 2-triangle
    ceiling light of radiance (17, 12, 4): 36 triangles. Lambert walls and
    boxes (ior 1: uncoated) with albedo in [0.1, 0.8] per channel; the
    Cornell camera."""
    rng = np.random.default_rng(seed)
    s = Scene(f"box-room-{seed}")

    def lambert():
        return s.add_material(preview_material(tuple(rng.uniform(0.1, 0.8, 3)), ior=1.0))

    for corners in ([[-1, -1, 1], [1, -1, 1], [1, -1, -1], [-1, -1, -1]],
                    [[-1, 1, 1], [-1, 1, -1], [1, 1, -1], [1, 1, 1]],
                    [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1]],
                    [[-1, -1, 1], [-1, -1, -1], [-1, 1, -1], [-1, 1, 1]],
                    [[1, -1, -1], [1, -1, 1], [1, 1, 1], [1, 1, -1]]):
        s.add_instance(s.add_geometry(*quad(corners)), lambert())
    light = s.add_material(preview_material((0.0, 0.0, 0.0), ior=1.0,
                                            emission=(17.0, 12.0, 4.0)))
    s.add_instance(s.add_geometry(*quad([[-0.35, 0.98, 0.35], [-0.35, 0.98, -0.35],
                                         [0.35, 0.98, -0.35], [0.35, 0.98, 0.35]])), light)
    cube = s.add_geometry(*unit_cube())
    for k in range(2):
        size_xyz = rng.uniform(0.2, 0.6, 3)
        angle = rng.uniform(0.0, math.pi)
        cx = (-0.4 if k == 0 else 0.4) + rng.uniform(-0.15, 0.15)
        cz = rng.uniform(-0.5, 0.3)
        centre = (cx, -1.0 + size_xyz[1] / 2 + 1e-3, cz)
        s.add_instance(cube, lambert(), block(size_xyz, math.degrees(angle), centre))
    s.world_to_clip = cornell_camera()
    s.width = s.height = size
    return s


def procedural_sky(width=2048, height=1024, seed=0, sun_elevation=0.6, sun_azimuth=0.8):
    """A lat-long sky: a log-normal field over a vertical gradient, plus one
    sun lobe. Rows run from +Y (top) to -Y, as the environment lookup
    expects."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = np.pi * v[:, None]
    phi = np.pi * (1.0 - 2.0 * u[None, :])
    d = np.stack([np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi),
                  np.sin(theta) * np.cos(phi)], axis=-1)
    coarse = rng.normal(0.0, 1.0, (16, 32))
    yi = np.clip((v * 16).astype(int), 0, 15)
    xi = np.clip((u * 32).astype(int), 0, 31)
    field = np.exp(0.35 * coarse[yi][:, xi])
    up = np.clip(d[..., 1], 0.0, 1.0)
    base = np.where(d[..., 1] >= 0.0, 0.6 + 0.8 * up, 0.15)
    sky = np.stack([0.55 * base, 0.7 * base, 1.0 * base], -1) * field[..., None]
    sun = np.array([math.cos(sun_elevation) * math.sin(sun_azimuth), math.sin(sun_elevation),
                    math.cos(sun_elevation) * math.cos(sun_azimuth)])
    cosine = np.clip(d @ sun, -1.0, 1.0)
    lobe = 4000.0 * np.exp((cosine - 1.0) * 4000.0)
    sky += np.stack([lobe, 0.9 * lobe, 0.75 * lobe], -1)
    texels = np.ones((height, width, 4), dtype=F32)
    texels[..., :3] = sky.astype(F32)
    return texels


def sphere_field(seed=0, width=1920, height=1080, prototypes=320, grid=100,
                 spacing=2.0, spheres=4096, emitters=64, sky_size=(2048, 1024)):
    """4096 instanced, Perlin-displaced icospheres (subdivision 3 or 4 by
    seed; ``prototypes`` unique meshes, about 1M unique triangles) with radii
    log-uniform in [0.05, 2] on a ``grid`` x ``grid`` ground; equal thirds
    Lambert, GGX conductor (roughness in [0.02, 0.8]) and smooth dielectric
    (ior 1.5); 64 emissive triangles with log-normal radiance (sigma 1); an
    importance-sampled procedural sky."""
    rng = np.random.default_rng(seed)
    s = Scene(f"sphere-field-{seed}")
    protos = []
    for k in range(prototypes):
        sub = 3 if rng.random() < 0.5 else 4
        v, f = icosphere(sub)
        freq = rng.uniform(1.5, 3.0)
        offset = rng.uniform(-100, 100, 3)
        r = 1.0 + 0.25 * perlin3(v * freq + offset, seed * 7919 + k)
        p = (v * r[:, None]).astype(F32)
        protos.append(s.add_geometry(p, f, corner_normals(p, f)))
    half = grid * spacing / 2.0
    ground = s.add_material(preview_material((0.45, 0.45, 0.42), roughness=0.8, ior=1.0))
    s.add_instance(s.add_geometry(*quad([[-half, 0, half], [half, 0, half],
                                         [half, 0, -half], [-half, 0, -half]])), ground)
    cells = rng.choice(grid * grid, spheres, replace=False)
    kinds = rng.permutation(np.arange(spheres) % 3)
    for n, cell in enumerate(cells):
        i, j = divmod(int(cell), grid)
        radius = math.exp(rng.uniform(math.log(0.05), math.log(2.0)))
        x = (i - (grid - 1) / 2.0) * spacing
        z = (j - (grid - 1) / 2.0) * spacing
        kind = kinds[n]
        if kind == 0:
            mat = preview_material(tuple(rng.uniform(0.1, 0.8, 3)), roughness=0.6, ior=1.0)
        elif kind == 1:
            mat = preview_material(tuple(rng.uniform(0.5, 1.0, 3)),
                                   roughness=rng.uniform(0.02, 0.8), metallic=1.0)
        else:
            mat = preview_material((1.0, 1.0, 1.0), roughness=0.0, ior=1.5, transmission=1.0)
        m = s.add_material(mat)
        lin = rotation_y(rng.uniform(0, 2 * math.pi)) * radius
        s.add_instance(protos[int(rng.integers(prototypes))], m,
                       affine(lin, (x, radius * 0.9, z)))
    tri = s.add_geometry(np.array([[-0.5, 0, -0.2887], [0.5, 0, -0.2887], [0, 0, 0.5774]],
                                  dtype=F32), np.array([[0, 1, 2]], dtype=np.uint32))
    for k in range(emitters):
        radiance = math.exp(rng.normal(0.0, 1.0)) * 20.0
        tint = rng.uniform(0.6, 1.0, 3)
        mat = s.add_material(preview_material((0.0, 0.0, 0.0), ior=1.0,
                                              emission=tuple(radiance * tint)))
        lin = rotation_xyz(rng.uniform(-0.5, 0.5) + math.pi, rng.uniform(0, 2 * math.pi),
                           rng.uniform(-0.5, 0.5)) * rng.uniform(2.0, 5.0)
        pos = (rng.uniform(-half * 0.6, half * 0.6), rng.uniform(6.0, 14.0),
               rng.uniform(-half * 0.6, half * 0.6))
        s.add_instance(tri, mat, affine(lin, pos))
    s.set_environment(procedural_sky(sky_size[0], sky_size[1], seed))
    extent = grid * spacing
    eye = (0.24 * extent, 0.11 * extent, 0.24 * extent)
    view = look_at(eye, (0.0, 0.0, 0.0))
    s.world_to_clip = multiply(perspective(50.0, width / height, 0.1, 1000.0), view)
    s.width, s.height = width, height
    return s


def restir_room(seed=0, size=96, emitters=10000, sigma=2.0, aspect=1.0):
    """The box room with ``emitters`` small emissive triangles on its floor,
    their power log-normal (sigma 2), and the ceiling light removed: a
    many-light scene for ReSTIR DI. Lambert walls and boxes."""
    rng = np.random.default_rng(seed + 1000)
    s = box_room(seed=seed, size=size)
    s.name = f"restir-room-{seed}-{emitters}"
    # Drop the ceiling light (instance 5): many small lights instead.
    s.instances = [inst for k, inst in enumerate(s.instances) if k != 5]
    tri = s.add_geometry(np.array([[-0.5, 0.0, -0.2887], [0.5, 0.0, -0.2887], [0.0, 0.0, 0.5774]],
                                  dtype=F32), np.array([[0, 2, 1]], dtype=np.uint32))
    for k in range(emitters):
        side = F32(rng.uniform(0.01, 0.04))
        power = math.exp(rng.normal(0.0, sigma))
        area = 0.4330127 * float(side) ** 2
        radiance = 0.02 * power / area / max(1.0, emitters / 100.0)
        tint = rng.uniform(0.5, 1.0, 3)
        mat = s.add_material(preview_material((0.0, 0.0, 0.0), ior=1.0,
                                              emission=tuple(radiance * tint)))
        lin = rotation_y(rng.uniform(0, 2 * math.pi)) * float(side)
        pos = (rng.uniform(-0.95, 0.95), -0.999, rng.uniform(-0.95, 0.95))
        s.add_instance(tri, mat, affine(lin, pos))
    s.width = int(size * aspect)
    s.height = size
    return s


def orbit_camera(frame, frames=120, radius=3.0, amplitude=0.35, aspect=1.0):
    """The view and world-to-clip of frame ``frame`` of a camera swinging
    about the box room's vertical axis, looking at its centre (45 degree
    vertical field of view, as the Cornell camera)."""
    theta = amplitude * math.sin(2.0 * math.pi * frame / frames)
    eye = (radius * math.sin(theta), 0.0, radius * math.cos(theta))
    view = look_at(eye, (0.0, 0.0, 0.0))
    projection = perspective(45.0, aspect, 1.0, 10.0)
    return view, multiply(projection, view)


def box_room_wide(seed=0, width=1920, height=1080, emitters=0):
    """The box room (config 1's scene) framed for a wide target: the orbit
    camera's first frame (the Cornell camera's eye and field of view) with
    the target's aspect, its view matrix kept for the temporal passes. With
    `emitters`, the many-light variant (restir_room: that many emissive
    floor triangles in place of the ceiling light)."""
    s = restir_room(seed=seed, size=width, emitters=emitters) if emitters else box_room(seed=seed, size=width)
    s.width, s.height = width, height
    s.view, s.world_to_clip = orbit_camera(0, aspect=width / height)
    return s


def batch_room(seed=0, triangles=100_000, size=256):
    """A config-1-style scene of about ``triangles`` traced triangles: the
    seeded box room (walls, two boxes, ceiling light) filled with small
    instanced, Perlin-displaced icospheres (four prototypes of subdivision
    4, 5120 triangles each) in equal thirds Lambert, GGX conductor and
    smooth dielectric; the Cornell camera on a size x size target."""
    rng = np.random.default_rng(seed + 7000)
    s = box_room(seed=seed, size=size)
    s.name = f"batch-room-{seed}-{triangles}"
    protos = []
    for k in range(4):
        v, f = icosphere(4)
        r = 1.0 + 0.25 * perlin3(v * rng.uniform(1.5, 3.0) + rng.uniform(-100, 100, 3), seed * 131 + k)
        p = (v * r[:, None]).astype(F32)
        protos.append(s.add_geometry(p, f, corner_normals(p, f)))
    count = max(1, int(round((triangles - 36) / 5120.0)))
    radius = min(0.15, 0.6 / max(1.0, count ** (1.0 / 3.0)))
    for n in range(count):
        kind = n % 3
        if kind == 0:
            mat = preview_material(tuple(rng.uniform(0.1, 0.8, 3)), roughness=0.6, ior=1.0)
        elif kind == 1:
            mat = preview_material(tuple(rng.uniform(0.5, 1.0, 3)), roughness=rng.uniform(0.02, 0.8),
                                   metallic=1.0)
        else:
            mat = preview_material((1.0, 1.0, 1.0), roughness=0.0, ior=1.5, transmission=1.0)
        rad = radius * rng.uniform(0.5, 1.0)
        pos = tuple(rng.uniform(-0.95 + rad, 0.95 - rad, 3))
        s.add_instance(protos[n % 4], s.add_material(mat),
                       affine(rotation_y(rng.uniform(0, 2 * math.pi)) * rad, pos))
    return s


def batch_workload(count=64, seed=0):
    """Config 4: ``count`` independent batch rooms, traced triangles
    log-uniform in [1e4, 2e6], resolutions uniform over 256^2, 512^2, 768^2
    and 1024^2 (seeded)."""
    rng = np.random.default_rng(seed + 4000)
    out = []
    for k in range(count):
        tris = int(math.exp(rng.uniform(math.log(1e4), math.log(2e6))))
        size = int(rng.choice([256, 512, 768, 1024]))
        out.append(batch_room(seed=seed * 1000 + k, triangles=tris, size=size))
    return out


def grid_mesh(quads=512, size=96):
    """One indexed grid of quads x quads quads in the xz-plane (512: 524,288
    triangles and 263,169 vertices, the shape of the reference's
    `geometry-v1` workload), gently displaced, under a constant sky, with
    the camera above it."""
    s = Scene(f"grid-{quads}")
    k = np.arange(quads + 1, dtype=np.float64) / quads * 2.0 - 1.0
    x, z = np.meshgrid(k, k, indexing="xy")
    y = 0.05 * np.sin(6.0 * x) * np.cos(5.0 * z)
    p = np.stack([x, y, z], axis=-1).reshape(-1, 3).astype(F32)
    i = np.arange(quads, dtype=np.uint32)
    a = (i[None, :] + (quads + 1) * i[:, None]).reshape(-1)
    b, c, d = a + 1, a + quads + 1, a + quads + 2
    f = np.stack([np.stack([a, c, b], -1), np.stack([b, c, d], -1)], axis=1).reshape(-1, 3)
    g = s.add_geometry(p, f)
    s.add_instance(g, s.add_material(preview_material((0.6, 0.6, 0.6), roughness=0.5, ior=1.0)))
    s.add_instance(s.add_geometry(*quad([[-0.3, 1.5, -0.3], [0.3, 1.5, -0.3], [0.3, 1.5, 0.3], [-0.3, 1.5, 0.3]])),
                   s.add_material(preview_material((0.0, 0.0, 0.0), ior=1.0, emission=(20.0, 20.0, 20.0))))
    s.environment_constant = (0.3, 0.35, 0.4)
    s.world_to_clip = multiply(perspective(50.0, 1.0, 0.1, 100.0), look_at((0.0, 2.2, 2.2), (0.0, 0.0, 0.0)))
    s.width = s.height = size
    return s


def big_mesh(seed=0, size=96, subdivisions=6):
    """One displaced icosphere of 20 * 4^subdivisions triangles (81,920 at
    6, above the per-CTA SAH builder's limit, so it builds as an LBVH) with
    a GGX and a Lambert instance of it under the procedural sky."""
    s = Scene(f"big-mesh-{seed}")
    v, f = icosphere(subdivisions)
    r = 1.0 + 0.2 * perlin3(v * 3.0, seed)
    p = (v * r[:, None]).astype(F32)
    g = s.add_geometry(p, f, corner_normals(p, f))
    metal = s.add_material(preview_material((0.9, 0.7, 0.5), roughness=0.3, metallic=1.0))
    clay = s.add_material(preview_material((0.6, 0.6, 0.6), roughness=0.7, ior=1.0))
    s.add_instance(g, metal, affine(np.eye(3), (-1.2, 0.0, 0.0)))
    s.add_instance(g, clay, affine(rotation_y(0.7) * 0.8, (1.2, 0.0, 0.0)))
    s.add_instance(s.add_geometry(*quad([[-6, -1.2, 6], [6, -1.2, 6], [6, -1.2, -6], [-6, -1.2, -6]])), clay)
    s.set_environment(procedural_sky(256, 128, seed))
    s.world_to_clip = multiply(perspective(45.0, 1.0, 0.1, 100.0), look_at((0.0, 1.5, 6.0), (0.0, 0.0, 0.0)))
    s.width = s.height = size
    return s


# ---------------------------------------------------------------------------
# Analytic lights (Lotus::Light, render_world.hpp:79-114)

# Frames whose -Z side faces down (-Y) and towards +X: a rect or disk in the
# light's XY plane emits from its -Z side.
FACING_DOWN = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, -1.0, 0.0]])
FACING_PLUS_X = np.array([[0.0, 0.0, -1.0], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0]])


def towards(direction):
    """A frame whose +Z axis is `direction`: a distant light shining from
    there along its -Z axis."""
    z = np.asarray(direction, dtype=np.float64)
    z = z / np.linalg.norm(z)
    helper = np.array([0.0, 1.0, 0.0]) if abs(z[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    x = np.cross(helper, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def lit_room(seed=0, size=128, parallel=True, environment=False):
    """The box room with one light of every analytic shape besides its
    ceiling emitter: two spheres (one small enough for the cone sampler's
    small-angle branch from most of the room), a rect under the ceiling
    facing down, a disk on the left wall facing +X, a distant light of 5
    degrees and, with `parallel`, a parallel light, both reaching in through
    the open front; optionally the procedural sky."""
    s = box_room(seed=seed, size=size)
    s.name = f"lit-room-{seed}"
    s.add_light(abi.LIGHT_SPHERE, affine(translation=(-0.45, 0.35, -0.35)), radiance=(6.0, 4.5, 2.0),
                radius=0.12)
    s.add_light(abi.LIGHT_SPHERE, affine(linear=np.eye(3) * 0.5, translation=(0.55, -0.2, -0.6)),
                radiance=(400.0, 300.0, 500.0), radius=0.02)
    s.add_light(abi.LIGHT_RECT, affine(linear=FACING_DOWN, translation=(0.3, 0.9, 0.2)),
                radiance=(2.0, 3.0, 4.0), width=0.5, height=0.3)
    s.add_light(abi.LIGHT_DISK, affine(linear=FACING_PLUS_X, translation=(-0.97, -0.3, 0.1)),
                radiance=(5.0, 1.0, 1.0), radius=0.2, normalize=True)
    s.add_light(abi.LIGHT_DISTANT, affine(linear=towards((0.3, 0.4, 1.0))), radiance=(3.0, 3.0, 2.5),
                angle=5.0)
    if parallel:
        s.add_light(abi.LIGHT_DISTANT, affine(linear=towards((-0.2, 0.3, 1.0))), radiance=(1.5, 1.2, 1.0),
                    angle=0.0)
    if environment:
        s.set_environment(procedural_sky(256, 128, seed=seed))
    return s


def many_lights(seed=0, size=128, count=48):
    """A ground plane with a few boxes under `count` seeded analytic lights
    (spheres, rects and disks in equal shares, log-normal radiance) hovering
    above it: the crossing hierarchy holds every one, and rays cross several
    on their way."""
    rng = np.random.default_rng(seed)
    s = Scene(f"many-lights-{seed}")
    ground = s.add_material(preview_material((0.5, 0.5, 0.5), roughness=0.6, ior=1.0))
    s.add_instance(s.add_geometry(*quad([[-4, 0, 4], [4, 0, 4], [4, 0, -4], [-4, 0, -4]])), ground)
    cube = s.add_geometry(*unit_cube())
    for k in range(6):
        extent = rng.uniform(0.3, 0.9, 3)
        centre = (rng.uniform(-2.5, 2.5), extent[1] / 2 + 1e-3, rng.uniform(-2.5, 2.5))
        mat = s.add_material(preview_material(tuple(rng.uniform(0.2, 0.8, 3)), roughness=rng.uniform(0.1, 0.9),
                                              metallic=float(k % 2), ior=1.5))
        s.add_instance(cube, mat, block(extent, rng.uniform(0.0, 180.0), centre))
    for k in range(count):
        centre = (rng.uniform(-3.5, 3.5), rng.uniform(0.6, 2.5), rng.uniform(-3.5, 3.5))
        radiance = tuple(float(v) for v in np.exp(rng.normal(0.5, 1.0, 3)))
        shape = (abi.LIGHT_SPHERE, abi.LIGHT_RECT, abi.LIGHT_DISK)[k % 3]
        if shape == abi.LIGHT_SPHERE:
            s.add_light(shape, affine(translation=centre), radiance=radiance, radius=rng.uniform(0.03, 0.25))
        elif shape == abi.LIGHT_RECT:
            s.add_light(shape, affine(linear=FACING_DOWN @ rotation_y(0.0), translation=centre), radiance=radiance,
                        width=rng.uniform(0.1, 0.6), height=rng.uniform(0.1, 0.6))
        else:
            s.add_light(shape, affine(linear=FACING_DOWN, translation=centre), radiance=radiance,
                        radius=rng.uniform(0.05, 0.3))
    s.world_to_clip = multiply(perspective(55.0, 1.0, 0.1, 100.0), look_at((0.0, 4.0, 6.5), (0.0, 0.6, 0.0)))
    s.width = s.height = size
    return s


def lit_plane(shape, size=33, height=1.0, radius=0.25, radiance=(2.0, 2.0, 2.0), albedo=0.5):
    """A Lambert plane (y = 0, albedo `albedo`, uncoated) under one analytic
    light centred `height` above the origin, seen from above: at the
    plane's centre the light's irradiance has a closed form (a sphere:
    pi L r^2 / h^2; a downward disk: pi L r^2 / (r^2 + h^2)), so the centre
    pixel's direct radiance is albedo * L * r^2 / h^2 or
    albedo * L * r^2 / (r^2 + h^2)."""
    s = Scene(f"lit-plane-{shape}")
    mat = s.add_material(preview_material((albedo, albedo, albedo), roughness=1.0, ior=1.0))
    s.add_instance(s.add_geometry(*quad([[-50, 0, 50], [50, 0, 50], [50, 0, -50], [-50, 0, -50]])), mat)
    if shape == abi.LIGHT_SPHERE:
        s.add_light(shape, affine(translation=(0.0, height, 0.0)), radiance=radiance, radius=radius)
    else:
        s.add_light(shape, affine(linear=FACING_DOWN, translation=(0.0, height, 0.0)), radiance=radiance,
                    radius=radius)
    s.world_to_clip = multiply(perspective(20.0, 1.0, 0.1, 100.0),
                               look_at((0.0, 3.0, 1e-3), (0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0)))
    s.width = s.height = size
    return s


def light_grid(side=16, size=512, seed=0):
    """The box room without its ceiling emitter, lit by a side x side grid
    of sphere lights (radius 0.025) 0.85 above its centre, spaced 0.12 x
    15 / (side - 1) over [-0.9, 0.9] in x and z, with radiance (12, 10, 8)
    scaled by 256 / side^2 so that the grid's power does not change with
    its side: the shape of the reference's many-lights-v1 light grid
    (SCENE.md's workloads), on the seeded box room."""
    s = box_room(seed=seed, size=size)
    s.name = f"light-grid-{side}x{side}"
    s.instances = [inst for k, inst in enumerate(s.instances) if k != 5]
    spacing = 0.0 if side == 1 else 0.12 * (15.0 / float(side - 1))
    first = 0.0 if side == 1 else -0.9
    scale = 256.0 / float(side * side)
    for y in range(side):
        for x in range(side):
            s.add_light(abi.LIGHT_SPHERE, affine(translation=(first + spacing * x, 0.85, first + spacing * y)),
                        radiance=(12.0 * scale, 10.0 * scale, 8.0 * scale), radius=0.025)
    return s


# ---------------------------------------------------------------------------
# The reference's material-basics-v1 fixture

def _fixed(value):
    """A coordinate rounded to a multiple of 1e-6 (halves away from zero), as
    the fixture's USD file spells it; -0 becomes +0."""
    scaled = value * 1e6
    rounded = math.floor(abs(scaled) + 0.5)
    return float(F32(math.copysign(rounded, scaled) / 1e6 + 0.0))


def uv_sphere(segments=32, rings=16):
    """The unit UV sphere of the material fixtures (material_fixtures.cpp:29-64
    in hydra-lotus): a pole vertex, rings-1 rings of `segments` vertices and
    the other pole; the caps are triangle fans, the bands quads split as
    fans from their first vertex. Its points double as its corner normals.
    Returns (positions, triangles, corner normals)."""
    points = [(0.0, 1.0, 0.0)]
    for i in range(1, rings):
        theta = math.pi * i / rings
        for j in range(segments):
            phi = 2.0 * math.pi * j / segments
            points.append((_fixed(math.sin(theta) * math.cos(phi)), _fixed(math.cos(theta)),
                           _fixed(-math.sin(theta) * math.sin(phi))))
    points.append((0.0, -1.0, 0.0))
    bottom = len(points) - 1

    def ring(i, j):
        return 1 + (i - 1) * segments + j % segments

    faces = [[0, ring(1, j), ring(1, j + 1)] for j in range(segments)]
    for i in range(1, rings - 1):
        for j in range(segments):
            faces.append([ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)])
    faces += [[ring(rings - 1, j), bottom, ring(rings - 1, j + 1)] for j in range(segments)]
    triangles = []
    for v in faces:
        for k in range(1, len(v) - 1):
            triangles.append((v[0], v[k], v[k + 1]))
    positions = np.asarray(points, dtype=F32)
    triangles = np.asarray(triangles, dtype=np.uint32)
    return positions, triangles, positions[triangles]


def _rotation_x_deg(degrees):
    c, s = math.cos(math.radians(degrees)), math.sin(math.radians(degrees))
    return np.array([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]], dtype=np.float64)


def _rotation_y_deg(degrees):
    c, s = math.cos(math.radians(degrees)), math.sin(math.radians(degrees))
    return np.array([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]], dtype=np.float64)


def material_studio(name, size):
    """The camera, lights and backdrop every material fixture shares
    (SetStudio, material_fixtures.cpp:119-157 in hydra-lotus): a camera at
    z = 6.5 looking down -Z (focal 3.125, clip 1..100), a constant dome of
    0.5, a 3x3 rect light of radiance 4 at (1.5, 2.5, 4) turned 20 degrees
    about Y and -30 about X, and a 6x6 backdrop quad at z = -1 with a 0.5
    grey coated-diffuse material."""
    s = Scene(name)
    focal, near, far = F32(3.125), F32(1.0), F32(100.0)
    view = identity()
    view[14] = -6.5
    projection = np.array([focal, 0, 0, 0, 0, focal, 0, 0,
                           0, 0, (far + near) / (near - far), -1,
                           0, 0, F32(2.0) * far * near / (near - far), 0], dtype=F32)
    s.world_to_clip = multiply(projection, view)
    s.width = s.height = size
    s.environment_constant = (0.5, 0.5, 0.5)
    key = np.eye(4)
    key[:3, 3] = (1.5, 2.5, 4.0)
    key = key @ _rotation_y_deg(20.0) @ _rotation_x_deg(-30.0)
    s.add_light(abi.LIGHT_RECT, key.astype(F32).reshape(-1, order="F"),
                radiance=(4.0, 4.0, 4.0), width=3.0, height=3.0)
    backdrop = s.add_geometry(*quad([[-3, -3, -1], [3, -3, -1], [3, 3, -1], [-3, 3, -1]]))
    s.add_instance(backdrop, s.add_material(preview_material((0.5, 0.5, 0.5))))
    return s


def material_basics(metal50_scale=1.0, size=128):
    """The reference's material-basics-v1 fixture (SetMaterialBasics,
    material_fixtures.cpp:161-211 in hydra-lotus), which its golden images
    validation/reference/material-basics-v1-{mean,variance}.pfm were
    rendered from: a 4x4 grid of UV spheres of radius 0.4, centres 0.9
    apart, in the material studio. Rows from the top: coated diffuse base
    colours (white, red, dark, clamped), coated diffuse roughness 0, 0.25,
    0.5, 1, a copper GGX conductor at roughness 0, 0.25, 0.5, 1, and gold
    at metallic 0.25 and 0.75, ior 2.5, and the specular workflow.
    ``metal50_scale`` scales the half-rough copper's base colour (the
    fixture's negative control, DarkerMetal, scales it by 0.9)."""
    s = material_studio("material-basics-v1", size)
    grey, copper, gold = (0.5, 0.5, 0.5), (0.95, 0.64, 0.54), (0.9, 0.6, 0.2)
    balls = [
        preview_material((0.8, 0.8, 0.8)),
        preview_material((0.8, 0.1, 0.05)),
        preview_material((0.04, 0.04, 0.04)),
        preview_material((1.0, 0.5, 0.0), roughness=1.0),
        preview_material(grey, roughness=0.0),
        preview_material(grey, roughness=0.25),
        preview_material(grey, roughness=0.5),
        preview_material(grey, roughness=1.0),
        preview_material(copper, roughness=0.0, metallic=1.0),
        preview_material(copper, roughness=0.25, metallic=1.0),
        preview_material(tuple(F32(c) * F32(metal50_scale) for c in copper), roughness=0.5,
                         metallic=1.0),
        preview_material(copper, roughness=1.0, metallic=1.0),
        preview_material(gold, roughness=0.3, metallic=0.25),
        preview_material(gold, roughness=0.3, metallic=0.75),
        preview_material((0.1, 0.2, 0.6), roughness=0.1, ior=2.5),
        preview_material((0.05, 0.05, 0.05), roughness=0.2, specular_color=(0.9, 0.6, 0.3),
                         flags=abi.MATERIAL_SPECULAR_WORKFLOW),
    ]
    ball = s.add_geometry(*uv_sphere())
    columns, rows = (-1.35, -0.45, 0.45, 1.35), (1.35, 0.45, -0.45, -1.35)
    for i, material in enumerate(balls):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.4
        placed[12], placed[13] = columns[i % 4], rows[i // 4]
        s.add_instance(ball, s.add_material(material), placed)
    return s


def _texture_image(size, texel):
    """An 8-bit image of size x size texels, rows from the top, texel(x, y)
    giving its RGBA codes."""
    return np.array([[texel(x, y) for x in range(size)] for y in range(size)], dtype=np.uint8)


def _transform2d_double(scale_s, scale_t, degrees, translate_s, translate_t, inner=(1, 0, 0, 0, 1, 0)):
    c, s = math.cos(degrees * (math.pi / 180.0)), math.sin(degrees * (math.pi / 180.0))
    local = (c * scale_s, -s * scale_t, translate_s, s * scale_s, c * scale_t, translate_t)
    i = inner
    return (local[0] * i[0] + local[1] * i[3], local[0] * i[1] + local[1] * i[4], local[0] * i[2] + local[1] * i[5] + local[2],
            local[3] * i[0] + local[4] * i[3], local[3] * i[1] + local[4] * i[4], local[3] * i[2] + local[4] * i[5] + local[5])


def _transform2d(scale_s, scale_t, degrees, translate_s, translate_t, inner=None):
    """A UsdTransform2d's st matrix as the reference's adapter composes it
    (in double, then rounded): scale, then a counter-clockwise rotation,
    then the translation, applied after `inner` (a double matrix from
    _transform2d_double); rows (m0 m1 m2), (m3 m4 m5)."""
    m = _transform2d_double(scale_s, scale_t, degrees, translate_s, translate_t,
                            inner if inner is not None else (1, 0, 0, 0, 1, 0))
    return tuple(float(F32(v)) for v in m)


def material_textures(shifted_repeat=False, size=160):
    """The reference's material-textures-v1 fixture (SetMaterialTextures,
    material_fixtures.cpp:390-500 in hydra-lotus), which its golden images
    validation/reference/material-textures-v1-{mean,variance}.pfm were
    rendered from: 25 unit cards (scale 0.7, a 5 x 5 grid 0.8 apart) in the
    material studio, each a UsdPreviewSurface whose base colour (and for
    some roughness and metallic) is a texture lookup: the 4x4 palette under
    each wrap mode over coordinates from -0.5 to 1.5, sRGB / raw / auto
    decoding, a grey ramp, grey-alpha and RGBA channels on roughness and
    metallic, scale and bias, missing images (fallbacks), a second
    coordinate set, indexed and turned coordinates, the material's
    coordinate fallback, an st transform, constants, and a 64x64 checker
    minified. ``shifted_repeat`` moves the Repeat card's s by 1/8 (the
    fixture's negative control, ShiftedRepeat: a texel-centre error)."""
    s = material_studio("material-textures-v1", size)

    def palette(x, y):
        return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)

    def ramp(x, y):
        v = 15 + 15 * (x + 4 * y)
        return (v, v, v, 255)

    def grey_alpha(x, y):
        v = 50 + 60 * x
        return (v, v, v, 230 - 60 * y)

    def rgba(x, y):
        return (220 - 60 * x, 40 + 60 * y, 40 + 60 * ((x + y) % 4), 30 + 65 * x)

    def checker(x, y):
        v = 255 if (x + y) % 2 == 0 else 0
        return (v, v, v, 255)

    srgb, unorm = abi.TEXTURE_RGBA8_SRGB, abi.TEXTURE_RGBA8_UNORM
    tex = {
        "palette|sRGB": s.add_texture(_texture_image(4, palette), srgb),
        "palette|raw": s.add_texture(_texture_image(4, palette), unorm),
        "palette|auto": s.add_texture(_texture_image(4, palette), srgb),
        "ramp|auto": s.add_texture(_texture_image(4, ramp), unorm),
        "grey-alpha|auto": s.add_texture(_texture_image(4, grey_alpha), unorm),
        "rgba|sRGB": s.add_texture(_texture_image(4, rgba), srgb),
        "rgba|raw": s.add_texture(_texture_image(4, rgba), unorm),
        "checker|raw": s.add_texture(_texture_image(64, checker), unorm),
    }
    clamp, black, rep, mirror = abi.WRAP_CLAMP, abi.WRAP_BLACK, abi.WRAP_REPEAT, abi.WRAP_MIRROR

    def lookup(key, wrap_s=clamp, wrap_t=clamp, **kw):
        return s.add_texture_input(tex.get(key, 0), wrap_s=wrap_s, wrap_t=wrap_t, **kw)

    def textured(base, texcoords="st", **kw):
        m = preview_material(**kw)
        m.lookups[abi.SLOT_BASE_COLOR] = base
        return m, texcoords

    def constant(**kw):
        return preview_material(**kw), "st"

    unit = [(0, 0), (1, 0), (1, 1), (0, 1)]
    wide = [(-0.5, -0.5), (1.5, -0.5), (1.5, 1.5), (-0.5, 1.5)]
    turned = [(1, 0), (1, 1), (0, 1), (0, 0)]
    one = {"st": unit}
    spread = {"st": wide}
    two = {"st": unit, "uv1": turned}

    grey_alpha_m, _ = textured(lookup("grey-alpha|auto"))
    grey_alpha_m.lookups[abi.SLOT_ROUGHNESS] = lookup("grey-alpha|auto", channel=3)
    alpha_m, _ = textured(lookup("rgba|sRGB"))
    alpha_m.lookups[abi.SLOT_ROUGHNESS] = lookup("rgba|sRGB", channel=3)
    orm = preview_material(base_color=(0.95, 0.64, 0.54))
    orm.lookups[abi.SLOT_METALLIC] = lookup("rgba|raw", channel=2)
    orm.lookups[abi.SLOT_ROUGHNESS] = lookup("rgba|raw", channel=1)
    missing = lookup("missing|sRGB", scale=(0.5, 0.5, 0.5, 1.0), fallback=(0.9, 0.2, 0.6, 1.0))
    no_file = lookup("|auto", fallback=(0.2, 0.6, 0.9, 1.0))
    constant_m, _ = textured(lookup("palette|sRGB"))
    constant_m.texcoord_fallback[:] = [0.6, 0.3]
    absent_m, _ = textured(lookup("palette|sRGB"))
    absent_m.texcoord_fallback[:] = [0.1, 0.9]
    cards = [
        ("UseMetadata", textured(lookup("palette|sRGB", black, black)), spread),
        ("Clamp", textured(lookup("palette|sRGB")), spread),
        ("Repeat", textured(lookup("palette|sRGB", rep, rep)), spread),
        ("Mirror", textured(lookup("palette|sRGB", mirror, mirror)), spread),
        ("Mixed", textured(lookup("palette|sRGB", rep, black)), spread),
        ("Srgb", textured(lookup("palette|sRGB")), one),
        ("Raw", textured(lookup("palette|raw")), one),
        ("Auto", textured(lookup("palette|auto")), one),
        ("Grey", textured(lookup("ramp|auto")), one),
        ("GreyAlpha", (grey_alpha_m, "st"), one),
        ("Alpha", (alpha_m, "st"), one),
        ("Orm", (orm, "st"), one),
        ("ScaleBias", textured(lookup("palette|raw", scale=(2.0, 2.0, 2.0, 1.0), bias=(-0.5, -0.5, -0.5, 0.0))),
         one),
        ("Missing", textured(missing), one),
        ("NoFile", textured(no_file), one),
        ("Vertex", textured(lookup("palette|sRGB")), one),
        ("Indexed", textured(lookup("palette|sRGB")), {"st": [(1, 0), (0, 0), (0, 1), (1, 1)]}),
        ("Named", textured(lookup("palette|sRGB"), "uv1"), two),
        ("Constant", (constant_m, ""), one),
        ("Absent", (absent_m, "absent"), one),
        ("Transform2d", textured(lookup("palette|sRGB", st_transform=_transform2d(2, 2, 30, 0.25, 0))), one),
        ("SecondSource", textured(lookup("palette|sRGB")), two),
        ("ColourOnScalar", constant(base_color=(0.3, 0.5, 0.7)), one),
        ("ScalarOnColour", constant(), one),
        ("Minified", textured(lookup("checker|raw", rep, rep)), one),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    positions = [(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)]
    for i, (name, (material, set_name), sets) in enumerate(cards):
        card = s.add_geometry(np.array(positions, dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
        names = sorted(sets)
        corners = []
        for key in names:
            f = [list(c) for c in sets[key]]
            if shifted_repeat and name == "Repeat" and key == "st":
                for c in f:
                    c[0] = float(F32(c[0]) + F32(0.125))
            # The fan (0, 1, 2), (0, 2, 3) of the face's four corners.
            corners.append([[f[0], f[1], f[2]], [f[0], f[2], f[3]]])
        s.set_texcoords(card, np.array(corners, dtype=F32))
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.7
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        texcoord_set = names.index(set_name) + 1 if set_name in names else 0
        s.add_instance(card, s.add_material(material), placed, texcoord_set=texcoord_set)
    return s


def texture_cutouts(size=96):
    """Texture lookups on coverage and emission, in the material studio:
    cards masked by an 8x8 cutout's alpha at threshold 0.5 and
    fractionally (threshold 0), a ramp's red as opacity at threshold 0.5,
    an inverted mask (scale -1, bias 1), a card that glows through a mask,
    a card whose emission is a texture (and so is each light sample's
    radiance), and a masked card in front of a half-covered one. For
    parity of every path with the oracle, not a reference golden."""
    s = material_studio("texture-cutouts", size)

    def cutout(x, y):
        dx, dy = 2 * x - 7, 2 * y - 7
        d = dx * dx + dy * dy
        return (60 + 20 * x, 200 - 15 * y, 60, 255 if d <= 26 else 96 if d <= 50 else 0)

    def ramp(x, y):
        v = 15 + 15 * (x + 4 * y)
        return (v, v, v, 255)

    def palette(x, y):
        return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)

    cut = s.add_texture(_texture_image(8, cutout), abi.TEXTURE_RGBA8_SRGB)
    rmp = s.add_texture(_texture_image(4, ramp), abi.TEXTURE_RGBA8_UNORM)
    pal = s.add_texture(_texture_image(4, palette), abi.TEXTURE_RGBA8_SRGB)
    clamp, rep = abi.WRAP_CLAMP, abi.WRAP_REPEAT

    def masked(threshold, wrap=clamp):
        m = preview_material(opacity_threshold=threshold)
        m.lookups[abi.SLOT_BASE_COLOR] = s.add_texture_input(cut, wrap_s=wrap, wrap_t=wrap)
        m.lookups[abi.SLOT_OPACITY] = s.add_texture_input(cut, channel=3, wrap_s=wrap, wrap_t=wrap)
        return m

    ramp_m = preview_material(base_color=(0.2, 0.6, 0.7), opacity_threshold=0.5)
    ramp_m.lookups[abi.SLOT_OPACITY] = s.add_texture_input(rmp, channel=0, wrap_s=clamp, wrap_t=clamp)
    inverted = preview_material(base_color=(0.2, 0.6, 0.7), opacity_threshold=0.5)
    inverted.lookups[abi.SLOT_OPACITY] = s.add_texture_input(
        cut, channel=3, wrap_s=clamp, wrap_t=clamp, scale=(1, 1, 1, -1), bias=(0, 0, 0, 1))
    glowing = masked(0.5)
    glowing.lookups[abi.SLOT_BASE_COLOR] = 0
    glowing.emission[:] = [1.0, 0.6, 0.2]
    lamp = preview_material(base_color=(0.1, 0.1, 0.1))
    lamp.lookups[abi.SLOT_EMISSION] = s.add_texture_input(pal, wrap_s=clamp, wrap_t=clamp, scale=(3, 3, 3, 1))
    half = preview_material(base_color=(0.7, 0.3, 0.2), opacity=0.5)
    looks = [masked(0.5), masked(0.0), ramp_m, inverted, glowing, lamp, masked(0.5, rep), half]
    positions = np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32)
    corners = np.array([[[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]]], dtype=F32)
    wide = np.array([[[[-0.5, -0.5], [1.5, -0.5], [1.5, 1.5]], [[-0.5, -0.5], [1.5, 1.5], [-0.5, 1.5]]]],
                    dtype=F32)
    columns, rows = (-1.2, 0.0, 1.2), (1.2, 0.0, -1.2)
    for i, material in enumerate(looks):
        card = s.add_geometry(positions, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
        s.set_texcoords(card, wide if i == 6 else corners)
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 1.0
        placed[12], placed[13] = columns[i % 3], rows[i // 3]
        if i == 7:
            placed[14] = -0.3  # behind the masked card at the same place
            placed[12], placed[13] = columns[0], rows[0]
        s.add_instance(card, s.add_material(material), placed, texcoord_set=1)
    return s


# The coarse polygon sphere of the reference's material fixtures
# (CoarseSphere, material_fixtures.cpp:594-628 in hydra-lotus): 16 segments,
# 8 rings, faces counter-clockwise seen from outside, points rounded to six
# decimals (Fixed) as its USD files store them.
_COARSE_SEGMENTS, _COARSE_RINGS = 16, 8


def _fixed(v):
    return float(F32(round(v * 1e6) / 1e6 + 0.0))


def coarse_sphere_polygons():
    """(points in double, faces as vertex lists)."""
    points = [(0.0, 1.0, 0.0)]
    for i in range(1, _COARSE_RINGS):
        theta = math.pi * i / _COARSE_RINGS
        for j in range(_COARSE_SEGMENTS):
            phi = 2 * math.pi * j / _COARSE_SEGMENTS
            points.append((math.sin(theta) * math.cos(phi), math.cos(theta), -math.sin(theta) * math.sin(phi)))
    points.append((0.0, -1.0, 0.0))
    bottom = len(points) - 1

    def ring(i, j):
        return 1 + (i - 1) * _COARSE_SEGMENTS + j % _COARSE_SEGMENTS

    faces = [[0, ring(1, j), ring(1, j + 1)] for j in range(_COARSE_SEGMENTS)]
    for i in range(1, _COARSE_RINGS - 1):
        for j in range(_COARSE_SEGMENTS):
            faces.append([ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)])
    faces += [[ring(_COARSE_RINGS - 1, j), bottom, ring(_COARSE_RINGS - 1, j + 1)] for j in range(_COARSE_SEGMENTS)]
    return points, faces


def coarse_sphere_corners(faces):
    """Each triangle corner as the adapter's fan triangulation makes them
    (right-handed faces): (vertex, face, face-vertex index)."""
    corners, first = [], 0
    for f, vertices in enumerate(faces):
        for k in range(1, len(vertices) - 1):
            for i in (0, k, k + 1):
                corners.append((vertices[i], f, first + i))
        first += len(vertices)
    return corners


def coarse_sphere_latlong(scale=(4.0, 2.0)):
    """The coarse sphere's (s, t) per face vertex in face order, times
    `scale` (LatLong, material_fixtures.cpp:632-656)."""
    seg, rings = float(_COARSE_SEGMENTS), float(_COARSE_RINGS)
    out = []

    def st(s, t):
        out.append((float(F32(s * scale[0])), float(F32(t * scale[1]))))

    for j in range(_COARSE_SEGMENTS):
        st((j + 0.5) / seg, 1)
        st(j / seg, 1 - 1 / rings)
        st((j + 1) / seg, 1 - 1 / rings)
    for i in range(1, _COARSE_RINGS - 1):
        for j in range(_COARSE_SEGMENTS):
            top, bot = 1 - i / rings, 1 - (i + 1) / rings
            st(j / seg, top)
            st(j / seg, bot)
            st((j + 1) / seg, bot)
            st((j + 1) / seg, top)
    for j in range(_COARSE_SEGMENTS):
        st(j / seg, 1 / rings)
        st((j + 0.5) / seg, 0)
        st((j + 1) / seg, 1 / rings)
    return out


def material_alpha(srgb_alpha=False, size=160):
    """The reference's material-alpha-v1 fixture (SetMaterialAlpha,
    material_fixtures.cpp:1056-1200 in hydra-lotus), which its golden images
    validation/reference/material-alpha-v1-{mean,variance}.pfm were rendered
    from: 24 cards and a coarse sphere (scale 0.7 / 0.35, a 5 x 5 grid 0.8
    apart) in the material studio: constant coverage (half, quarter, zero,
    thresholds below, at and above), texture coverage from RGBA and
    grey-alpha images, a cutout (masked at 0.5 and fractional), a ramp's red,
    an inverted mask, a black border, a missing image's fallback, a minified
    checker, a masked card over a half-covered one, a masked sphere, and
    emitters through a mask and at half coverage. ``srgb_alpha`` decodes the
    sRGB images' alpha as colour (the fixture's negative control,
    SrgbAlpha)."""
    s = material_studio("material-alpha-v1", size)

    def rgba(x, y):
        return (220 - 60 * x, 40 + 60 * y, 40 + 60 * ((x + y) % 4), 30 + 65 * x)

    def cutout(x, y):
        dx, dy = 2 * x - 7, 2 * y - 7
        d = dx * dx + dy * dy
        return (60 + 20 * x, 200 - 15 * y, 60, 255 if d <= 26 else 96 if d <= 50 else 0)

    def grey_alpha(x, y):
        v = 50 + 60 * x
        return (v, v, v, 230 - 60 * y)

    def ramp(x, y):
        v = 15 + 15 * (x + 4 * y)
        return (v, v, v, 255)

    def palette(x, y):
        return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)

    def checker(x, y):
        v = 255 if (x + y) % 2 == 0 else 0
        return (v, v, v, 255)

    srgb, unorm = abi.TEXTURE_RGBA8_SRGB, abi.TEXTURE_RGBA8_UNORM

    def image(size_, texel, fmt):
        img = _texture_image(size_, texel)
        if srgb_alpha and fmt == srgb:
            a = img[..., 3].astype(np.float64) / 255.0
            lin = np.where(a <= 0.04045, a / 12.92, ((a + 0.055) / 1.055) ** 2.4)
            img[..., 3] = np.floor(lin * 255.0 + 0.5).astype(np.uint8)
        return s.add_texture(img, fmt)

    tex = {
        "rgba|sRGB": image(4, rgba, srgb),
        "cutout|sRGB": image(8, cutout, srgb),
        "grey-alpha|auto": image(4, grey_alpha, unorm),
        "ramp|raw": image(4, ramp, unorm),
        "palette|sRGB": image(4, palette, srgb),
        "checker|raw": image(64, checker, unorm),
    }
    clamp, rep, black = abi.WRAP_CLAMP, abi.WRAP_REPEAT, abi.WRAP_BLACK

    def lookup(key, wrap=clamp, **kw):
        return s.add_texture_input(tex.get(key, 0), wrap_s=wrap, wrap_t=wrap, **kw)

    def covered(opacity, threshold=0.0):
        return preview_material(base_color=(0.2, 0.6, 0.7), opacity=opacity, opacity_threshold=threshold)

    def masked(key, threshold=0.5, wrap=clamp, **kw):
        m = preview_material(opacity_threshold=threshold)
        m.lookups[abi.SLOT_BASE_COLOR] = lookup(key, wrap, **kw)
        m.lookups[abi.SLOT_OPACITY] = lookup(key, wrap, channel=3, **kw)
        return m

    ramp_m = covered(1.0, 0.5)
    ramp_m.lookups[abi.SLOT_OPACITY] = lookup("ramp|raw", channel=0)
    inverted = covered(1.0, 0.5)
    inverted.lookups[abi.SLOT_OPACITY] = lookup("cutout|sRGB", channel=3, scale=(1, 1, 1, -1), bias=(0, 0, 0, 1))
    minified = covered(1.0, 0.5)
    minified.lookups[abi.SLOT_OPACITY] = lookup("checker|raw", rep, channel=0)
    glowing_mask = masked("cutout|sRGB")
    glowing_mask.lookups[abi.SLOT_BASE_COLOR] = 0
    glowing_mask.emission[:] = [1.0, 0.6, 0.2]
    glowing_half = preview_material(emission=(1.0, 0.6, 0.2), opacity=0.5)
    looks = {
        "Half": covered(0.5), "Quarter": covered(0.25), "Zero": covered(0.0), "Presence": covered(0.5),
        "Clamped": covered(1.0, 1.0), "Below": covered(0.4, 0.5), "Equal": covered(0.5, 0.5),
        "Above": covered(0.6, 0.5), "NonFinite": covered(1.0), "ThresholdMap": covered(0.5),
        "Alpha": masked("rgba|sRGB"), "Cutout": masked("cutout|sRGB"), "GreyAlpha": masked("grey-alpha|auto"),
        "Ramp": ramp_m, "NoAlpha": masked("palette|sRGB"), "Fractional": masked("cutout|sRGB", 0.0),
        "Inverted": inverted, "BlackBorder": masked("palette|sRGB", wrap=black),
        "Missing": masked("missing|sRGB", 0.0, fallback=(0.9, 0.2, 0.6, 0.3)),
        "Minified": minified, "SphereCutout": masked("cutout|sRGB", wrap=rep),
        "GlowingMask": glowing_mask, "GlowingHalf": glowing_half,
    }
    slot = {name: s.add_material(m) for name, m in looks.items()}
    display = s.add_material(preview_material(base_color=(0.2, 0.6, 0.7), opacity=0.3))

    card_p = np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32)
    card_t = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    plain = s.add_geometry(card_p, card_t)
    mapped = s.add_geometry(card_p, card_t)
    s.set_texcoords(mapped, np.array([[[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]]], dtype=F32))
    wide = s.add_geometry(card_p, card_t)
    w = [(-0.5, -0.5), (1.5, -0.5), (1.5, 1.5), (-0.5, 1.5)]
    s.set_texcoords(wide, np.array([[[w[0], w[1], w[2]], [w[0], w[2], w[3]]]], dtype=F32))
    stacked = s.add_geometry(
        np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0),
                  (-0.15, -0.15, 0.4), (0.45, -0.15, 0.4), (0.45, 0.45, 0.4), (-0.15, 0.45, 0.4)], dtype=F32),
        np.array([[0, 1, 2], [0, 2, 3], [4, 5, 6], [4, 6, 7]], dtype=np.uint32))
    points, faces = coarse_sphere_polygons()
    corners = coarse_sphere_corners(faces)
    fixed = np.array([[_fixed(c) for c in p] for p in points], dtype=F32)
    tris = np.array([[corners[i][0], corners[i + 1][0], corners[i + 2][0]] for i in range(0, len(corners), 3)],
                    dtype=np.uint32)
    normals = np.array([fixed[v] for v, _, _ in corners], dtype=F32).reshape(-1, 3, 3)
    sphere = s.add_geometry(fixed, tris, normals)
    latlong = coarse_sphere_latlong()
    s.set_texcoords(sphere, np.array([latlong[fv] for _, _, fv in corners], dtype=F32).reshape(1, -1, 3, 2))
    objects = [
        ("Half", plain), ("Quarter", plain), ("Zero", plain), ("Presence", plain), ("Clamped", plain),
        ("Below", plain), ("Equal", plain), ("Above", plain), ("NonFinite", plain), ("ThresholdMap", mapped),
        ("Alpha", mapped), ("Cutout", mapped), ("GreyAlpha", mapped), ("Ramp", mapped), ("NoAlpha", mapped),
        ("Fractional", mapped), ("Inverted", mapped), ("BlackBorder", wide), ("Missing", mapped),
        ("Minified", mapped), ("Half", stacked), ("SphereCutout", sphere), ("GlowingMask", mapped),
        ("GlowingHalf", plain), (None, plain),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (name, geo) in enumerate(objects):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.35 if geo == sphere else 0.7
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        has_st = geo in s.texcoords
        s.add_instance(geo, display if name is None else slot[name], placed, texcoord_set=1 if has_st else 0)
    return s


def coarse_sphere_polygons_reversed():
    """The coarse sphere with each face's vertices reversed, as a
    left-handed mesh lists them (CoarseSphere(true))."""
    points, faces = coarse_sphere_polygons()
    return points, [list(reversed(f)) for f in faces]


def coarse_sphere_corners_left(faces):
    """Corners of a left-handed mesh as the adapter triangulates it: a
    quad as (v2, v1, v0), (v2, v0, v3), other faces as (v0, v[k + 1], v[k])
    (Polygons::Corners, material_fixtures.cpp:525-549)."""
    corners, first = [], 0
    for f, vertices in enumerate(faces):
        if len(vertices) == 4:
            tris = [(2, 1, 0), (2, 0, 3)]
        else:
            tris = [(0, k + 1, k) for k in range(1, len(vertices) - 1)]
        for tri in tris:
            for i in tri:
                corners.append((vertices[i], f, first + i))
        first += len(vertices)
    return corners


def coarse_smooth_normals(points, faces, left_handed=False):
    """Storm's smooth vertex normals in float (SmoothNormals,
    material_fixtures.cpp:565-589): per vertex the sum over its faces'
    corners of cross(next - vertex, previous - vertex) (the two swapped on
    a left-handed face), divided by the float length."""
    pos = [[F32(_fixed(c)) for c in p] for p in points]
    sums = [[F32(0.0)] * 3 for _ in points]
    for vertices in faces:
        n = len(vertices)
        for i in range(n):
            curr = pos[vertices[i]]
            prev = pos[vertices[(i + n - 1) % n]]
            nxt = pos[vertices[(i + 1) % n]]
            if left_handed:
                prev, nxt = nxt, prev
            a = [nxt[k] - curr[k] for k in range(3)]
            b = [prev[k] - curr[k] for k in range(3)]
            s = sums[vertices[i]]
            sums[vertices[i]] = [s[0] + (a[1] * b[2] - a[2] * b[1]), s[1] + (a[2] * b[0] - a[0] * b[2]),
                                 s[2] + (a[0] * b[1] - a[1] * b[0])]
    out = []
    for s in sums:
        length = np.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
        scale = 1.0 / float(max(length, F32(1e-10)))
        out.append([float(F32(float(c) * scale)) for c in s])
    return out


def material_normals(flipped_green=False, size=160):
    """The reference's material-normals-v1 fixture (SetMaterialNormals,
    material_fixtures.cpp:692-828 in hydra-lotus), which its golden images
    validation/reference/material-normals-v1-{mean,variance}.pfm were
    rendered from: coarse spheres (scale 0.35) with faceted, per-vertex,
    face-uniform, computed (Storm's smooth normals, right- and left-handed)
    and inward corner normals, and cards (scale 0.7) and spheres with
    tangent-space normal maps: raw, sRGB-decoded, unscaled and DirectX
    images, a constant normal in the normal-only frame, an absent
    coordinate set, mirrored and rotated coordinates, mirrored and
    stretched transforms, and a glossy copper sphere. ``flipped_green``
    reads the Mapped look's map with green negated (the fixture's negative
    control, FlippedGreen)."""
    s = material_studio("material-normals-v1", size)

    def tilts(x, y):
        return (32 + 64 * x, 224 - 64 * y, 200, 255)

    def tilts_dx(x, y):
        return (32 + 64 * x, 31 + 64 * y, 200, 255)

    raw = s.add_texture(_texture_image(4, tilts), abi.TEXTURE_RGBA8_UNORM)
    auto = s.add_texture(_texture_image(4, tilts), abi.TEXTURE_RGBA8_SRGB)
    dx = s.add_texture(_texture_image(4, tilts_dx), abi.TEXTURE_RGBA8_UNORM)
    clamp, rep = abi.WRAP_CLAMP, abi.WRAP_REPEAT

    def normal_map(texture, wrap=clamp, green=(2.0, -1.0)):
        return s.add_texture_input(texture, wrap_s=wrap, wrap_t=wrap, scale=(2.0, green[0], 2.0, 1.0),
                                   bias=(-1.0, green[1], -1.0, 0.0))

    def bumpy(lookup):
        m = preview_material(base_color=(0.7, 0.7, 0.7), roughness=0.4)
        if lookup:
            m.lookups[abi.SLOT_NORMAL] = lookup
        return m, "st" if lookup else ""

    constant_m, _ = bumpy(0)
    constant_m.normal[:] = [0.4, 0.3, 0.866]
    absent_m, _ = bumpy(normal_map(raw))
    absent_m.texcoord_fallback[:] = [0.25, 0.75]
    glossy = preview_material(base_color=(0.95, 0.64, 0.54), roughness=0.25, metallic=1.0)
    glossy.lookups[abi.SLOT_NORMAL] = normal_map(raw, rep)
    looks = {
        "Smooth": (preview_material(base_color=(0.6, 0.6, 0.6), roughness=0.3), ""),
        "Mapped": bumpy(normal_map(raw, green=(-2.0, 1.0) if flipped_green else (2.0, -1.0))),
        "Auto": bumpy(normal_map(auto)),
        "Unscaled": bumpy(s.add_texture_input(raw, wrap_s=clamp, wrap_t=clamp)),
        "DirectX": bumpy(normal_map(dx, green=(-2.0, 1.0))),
        "Constant": (constant_m, ""),
        "AbsentSet": (absent_m, "absent"),
        "SphereMapped": bumpy(normal_map(raw, rep)),
        "SphereGlossy": (glossy, "st"),
    }
    slot = {name: (s.add_material(m), set_name) for name, (m, set_name) in looks.items()}

    points, faces = coarse_sphere_polygons()
    corners = coarse_sphere_corners(faces)
    fixed = np.array([[_fixed(c) for c in p] for p in points], dtype=F32)
    tris = np.array([[corners[i][0], corners[i + 1][0], corners[i + 2][0]] for i in range(0, len(corners), 3)],
                    dtype=np.uint32)
    latlong = coarse_sphere_latlong()
    mapped_st = np.array([latlong[fv] for _, _, fv in corners], dtype=F32).reshape(1, -1, 3, 2)

    def per_vertex(values):
        return np.array([values[v] for v, _, _ in corners], dtype=F32).reshape(-1, 3, 3)

    point_normals = [[_fixed(c) for c in p] for p in points]
    inward = [[_fixed(-c) for c in p] for p in points]
    face_normals = []
    for f in faces:
        c = [sum(points[v][k] for v in f) for k in range(3)]
        length = math.sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2])
        face_normals.append([_fixed(c[k] / length) for k in range(3)])
    uniform = np.array([face_normals[f] for _, f, _ in corners], dtype=F32).reshape(-1, 3, 3)
    smooth = per_vertex(coarse_smooth_normals(points, faces))
    rpoints, rfaces = coarse_sphere_polygons_reversed()
    rcorners = coarse_sphere_corners_left(rfaces)
    rtris = np.array([[rcorners[i][0], rcorners[i + 1][0], rcorners[i + 2][0]] for i in range(0, len(rcorners), 3)],
                     dtype=np.uint32)
    rsmooth = coarse_smooth_normals(rpoints, rfaces, left_handed=True)
    left_normals = np.array([rsmooth[v] for v, _, _ in rcorners], dtype=F32).reshape(-1, 3, 3)

    def sphere_mesh(normals, mapped):
        g = s.add_geometry(fixed, tris, normals)
        if mapped:
            s.set_texcoords(g, mapped_st)
        return g

    def card(face):
        g = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)],
                                    dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
        s.set_texcoords(g, np.array([[[face[0], face[1], face[2]], [face[0], face[2], face[3]]]], dtype=F32))
        return g

    unit = [(0, 0), (1, 0), (1, 1), (0, 1)]
    turned = [(1, 0), (1, 1), (0, 1), (0, 0)]
    sphere, card_scale = (0.35, 0.35, 0.35), (0.7, 0.7, 0.7)
    objects = [
        ("Smooth", sphere_mesh(None, False), sphere),
        ("Smooth", sphere_mesh(per_vertex(point_normals), False), sphere),
        ("Smooth", sphere_mesh(per_vertex(point_normals), False), sphere),
        ("Smooth", sphere_mesh(uniform, False), sphere),
        ("Smooth", sphere_mesh(per_vertex(point_normals), False), sphere),
        ("Smooth", sphere_mesh(smooth, False), sphere),
        ("Smooth", s.add_geometry(fixed, rtris, left_normals), sphere),
        ("Smooth", sphere_mesh(smooth, False), sphere),
        ("Smooth", sphere_mesh(None, False), sphere),
        ("Smooth", sphere_mesh(per_vertex(inward), False), sphere),
        ("Mapped", card(unit), card_scale),
        ("Auto", card(unit), card_scale),
        ("Unscaled", card(unit), card_scale),
        ("DirectX", card(unit), card_scale),
        ("Constant", card(unit), card_scale),
        ("Mapped", card([(1, 0), (0, 0), (0, 1), (1, 1)]), card_scale),
        ("Mapped", card(turned), card_scale),
        ("Mapped", card(unit), (-0.7, 0.7, 0.7)),
        ("Mapped", card(unit), (0.7, 0.35, 0.7)),
        ("AbsentSet", card(unit), card_scale),
        ("SphereMapped", sphere_mesh(per_vertex(point_normals), True), sphere),
        ("SphereMapped", sphere_mesh(None, True), sphere),
        ("SphereMapped", sphere_mesh(smooth, True), sphere),
        ("SphereGlossy", sphere_mesh(per_vertex(point_normals), True), sphere),
        ("Constant", sphere_mesh(per_vertex(point_normals), True), sphere),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (look, geo, scale) in enumerate(objects):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0], placed[5], placed[10] = scale
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        material, set_name = slot[look]
        s.add_instance(geo, material, placed, texcoord_set=1 if set_name == "st" and geo in s.texcoords else 0)
    return s


def _coarse_smooth_sphere(s):
    """The coarse polygon sphere with its points (rounded) as corner
    normals, as a geometry of scene `s`; with the st set when `mapped`."""
    points, faces = coarse_sphere_polygons()
    corners = coarse_sphere_corners(faces)
    fixed = np.array([[_fixed(c) for c in p] for p in points], dtype=F32)
    tris = np.array([[corners[i][0], corners[i + 1][0], corners[i + 2][0]] for i in range(0, len(corners), 3)],
                    dtype=np.uint32)
    normals = np.array([fixed[v] for v, _, _ in corners], dtype=F32).reshape(-1, 3, 3)
    return s.add_geometry(fixed, tris, normals)


def material_transmission(untinted=False, size=160):
    """The reference's material-transmission-v1 fixture
    (SetMaterialTransmission, material_fixtures.cpp:1588-1671 in
    hydra-lotus): 15 objects on the middle three rows in the material
    studio: solid coarse spheres of smooth, rough, tinted, index-matched and
    partial transmission, thin-walled cards (smooth, rough, tinted,
    index-matched, ior 2.42), a mirrored sphere and the translator's no-ops.
    ``untinted`` drops the tinted sphere's transmission colour (the
    fixture's negative control, UntintedGlass)."""
    s = material_studio("material-transmission-v1", size)
    teal, amber = (0.2, 0.6, 0.7), (0.9, 0.45, 0.15)

    def glass(roughness, tint=(1.0, 1.0, 1.0), thin=False, ior=1.5):
        return preview_material(base_color=(0.8, 0.8, 0.8), roughness=roughness, transmission=1.0,
                                transmission_color=tint, ior=ior,
                                flags=abi.MATERIAL_THIN_WALLED if thin else 0)

    looks = {
        "Smooth": glass(0.0), "Rough": glass(0.35),
        "Tinted": glass(0.0, (1.0, 1.0, 1.0) if untinted else amber),
        "Matched": glass(0.4, (0.5, 0.8, 0.9), ior=1.0),
        "Partial": preview_material(base_color=teal, roughness=0.15, transmission=0.5, metallic=0.25),
        "ThinSmooth": glass(0.0, thin=True), "ThinRough": glass(0.4, thin=True),
        "ThinTinted": glass(0.1, (0.3, 0.7, 0.9), thin=True),
        "ThinMatched": glass(0.2, (0.9, 0.6, 0.3), thin=True, ior=1.0),
        "ThinDense": glass(0.0, thin=True, ior=2.42),
        "Depth": glass(0.0), "NoSpecular": glass(0.2), "Ignored": glass(0.1),
        "Graph": preview_material(base_color=teal, roughness=0.3),
    }
    slot = {name: s.add_material(m) for name, m in looks.items()}
    sphere = _coarse_smooth_sphere(s)
    card = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32),
                          np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    objects = [("Smooth", sphere, False), ("Rough", sphere, False), ("Tinted", sphere, False),
               ("Matched", sphere, False), ("Partial", sphere, False), ("ThinSmooth", card, False),
               ("ThinRough", card, False), ("ThinTinted", card, False), ("ThinMatched", card, False),
               ("ThinDense", card, False), ("Smooth", sphere, True), ("Depth", sphere, False),
               ("NoSpecular", sphere, False), ("Ignored", sphere, False), ("Graph", sphere, False)]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (0.8, 0.0, -0.8)
    for i, (look, geo, mirrored) in enumerate(objects):
        scale = 0.35 if geo == sphere else 0.7
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = -scale if mirrored else scale
        placed[5] = placed[10] = scale
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        s.add_instance(geo, slot[look], placed)
    return s


def material_transforms(reversed_rotation=False, size=160):
    """The reference's material-transforms-v1 fixture
    (SetMaterialTransforms, material_fixtures.cpp:1749-1825 in hydra-lotus):
    15 cards on the middle three rows in the material studio whose lookups
    carry UsdTransform2d st transforms: scale, rotation, translation, both,
    a flip, a normal map turned and tiled, a transform on one input only, a
    chain of two, on emission, on a constant's coordinates (no set), on an
    absent set's fallback, on coverage, the identity, and a connected
    rotation left untranslated. ``reversed_rotation`` reverses the rotated
    card's rotation (the fixture's negative control, ReversedRotation)."""
    s = material_studio("material-transforms-v1", size)

    def palette_img(x, y):
        return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)

    def tilts_img(x, y):
        return (32 + 64 * x, 224 - 64 * y, 200, 255)

    def ramp_img(x, y):
        v = 15 + 15 * (x + 4 * y)
        return (v, v, v, 255)

    def cutout_img(x, y):
        dx, dy = 2 * x - 7, 2 * y - 7
        d = dx * dx + dy * dy
        return (60 + 20 * x, 200 - 15 * y, 60, 255 if d <= 26 else 96 if d <= 50 else 0)

    pal = s.add_texture(_texture_image(4, palette_img), abi.TEXTURE_RGBA8_SRGB)
    tlt = s.add_texture(_texture_image(4, tilts_img), abi.TEXTURE_RGBA8_UNORM)
    rmp = s.add_texture(_texture_image(4, ramp_img), abi.TEXTURE_RGBA8_UNORM)
    cut = s.add_texture(_texture_image(8, cutout_img), abi.TEXTURE_RGBA8_SRGB)
    rep, clamp = abi.WRAP_REPEAT, abi.WRAP_CLAMP

    def placed(texture, transform, wrap=rep, **kw):
        return s.add_texture_input(texture, wrap_s=wrap, wrap_t=wrap, st_transform=transform, **kw)

    def palette(transform, wrap=rep, texcoords="st"):
        m = preview_material()
        m.lookups[abi.SLOT_BASE_COLOR] = placed(pal, transform, wrap)
        return m, texcoords

    def tilts(transform):
        m = preview_material(base_color=(0.7, 0.7, 0.7), roughness=0.4)
        m.lookups[abi.SLOT_NORMAL] = placed(tlt, transform, scale=(2, 2, 2, 1), bias=(-1, -1, -1, 0))
        return m, "st"

    t = _transform2d
    per_input, _ = palette(t(1, 1, 0, 0, 0))
    per_input.lookups[abi.SLOT_ROUGHNESS] = placed(rmp, t(4, 4, 0, 0, 0), channel=0)
    emission = preview_material(base_color=(0.0, 0.0, 0.0))
    emission.lookups[abi.SLOT_EMISSION] = placed(pal, t(1, 1, 60, 0, 0))
    constant, _ = palette(t(1, 1, 0, 0.125, 0.5), clamp)
    constant.texcoord_fallback[:] = [0.5, 0.25]
    absent, _ = palette(t(2, 2, 0, 0, 0), clamp)
    absent.texcoord_fallback[:] = [0.125, 0.25]
    coverage = preview_material(base_color=(0.2, 0.6, 0.7), opacity_threshold=0.5)
    coverage.lookups[abi.SLOT_OPACITY] = placed(cut, t(1, 1, 45, 0, 0), channel=3)
    cards = [
        ("Scale", palette(t(2, 2, 0, 0, 0))),
        ("Rotate", palette(t(1, 1, -30 if reversed_rotation else 30, 0, 0))),
        ("Translate", palette(t(1, 1, 0, 0.25, 0.5))),
        ("Combined", palette(t(2, 1, 30, 0.25, 0))),
        ("Flip", palette(t(-1, 1, 0, 0, 0))),
        ("NormalTurned", tilts(t(1, 1, 90, 0, 0))),
        ("NormalTiled", tilts(t(3, 3, 0, 0, 0))),
        ("PerInput", (per_input, "st")),
        ("Chain", palette(t(1, 1, 45, 0, 0, _transform2d_double(2, 2, 0, 0, 0)))),
        ("Emission", (emission, "st")),
        ("ConstantIn", (constant, "")),
        ("Absent", (absent, "absent")),
        ("Coverage", (coverage, "st")),
        ("Identity", palette(t(1, 1, 0, 0, 0))),
        ("Connected", (preview_material(), "st")),
    ]
    positions = np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32)
    corners = np.array([[[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]]], dtype=F32)
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (0.8, 0.0, -0.8)
    for i, (name, (material, set_name)) in enumerate(cards):
        card = s.add_geometry(positions, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
        has_st = name != "ConstantIn"
        if has_st:
            s.set_texcoords(card, corners)
        placed_m = np.eye(4, dtype=F32).reshape(-1)
        placed_m[0] = placed_m[5] = placed_m[10] = 0.7
        placed_m[12], placed_m[13] = columns[i % 5], rows[i // 5]
        s.add_instance(card, s.add_material(material), placed_m,
                       texcoord_set=1 if has_st and set_name == "st" else 0)
    return s


def _glow_image(srgb):
    """The 4x4 float image of the reference's material fixtures (Glow,
    material_fixtures.cpp:827-848): RGBE-decoded values, the colour
    channels decoded from sRGB in double where `srgb`."""
    out = np.zeros((4, 4, 4), dtype=F32)
    for y in range(4):
        for x in range(4):
            unit = float(F32(math.ldexp(1.0, 127 + y - 136)))
            v = [(240 - 50 * x) * unit, (80 + 50 * x) * unit, 160 * unit, 1.0]
            for c in range(4):
                if srgb and c < 3:
                    v[c] = v[c] / 12.92 if v[c] <= 0.04045 else ((v[c] + 0.055) / 1.055) ** 2.4
                out[y, x, c] = F32(v[c])
    return out


def material_emission(raw_emission=False, size=160):
    """The reference's material-emission-v1 fixture (SetMaterialEmission,
    material_fixtures.cpp:875-1009 in hydra-lotus): 25 objects in the
    material studio: constant emitters (warm, bright, dim, clamped, a
    metal), a back-facing, mirrored, stretched and tilted card, a faceted
    sphere, emission maps (sRGB, raw, auto, grey, scale and bias, a missing
    image's fallback, inverted, float images raw / auto / sRGB-decoded), a
    textured sphere, a map shared with the base colour, an unlit card and a
    card whose second quad is a subset bound to an emitter. ``raw_emission``
    reads the sRGB palette as raw (the fixture's negative control,
    RawEmission)."""
    s = material_studio("material-emission-v1", size)

    def palette(x, y):
        return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)

    def ramp(x, y):
        v = 15 + 15 * (x + 4 * y)
        return (v, v, v, 255)

    srgb, unorm, flt = abi.TEXTURE_RGBA8_SRGB, abi.TEXTURE_RGBA8_UNORM, abi.TEXTURE_RGBA32_FLOAT
    tex = {
        "palette|sRGB": s.add_texture(_texture_image(4, palette), unorm if raw_emission else srgb),
        "palette|raw": s.add_texture(_texture_image(4, palette), unorm),
        "palette|auto": s.add_texture(_texture_image(4, palette), srgb),
        "ramp|auto": s.add_texture(_texture_image(4, ramp), unorm),
        "glow|raw": s.add_texture(_glow_image(False), flt),
        "glow|auto": s.add_texture(_glow_image(False), flt),
        "glow|sRGB": s.add_texture(_glow_image(True), flt),
    }
    clamp, rep = abi.WRAP_CLAMP, abi.WRAP_REPEAT

    def lookup(key, wrap=clamp, **kw):
        return s.add_texture_input(tex.get(key, 0), wrap_s=wrap, wrap_t=wrap, **kw)

    def glowing(ref, **kw):
        m = preview_material(**kw)
        m.lookups[abi.SLOT_EMISSION] = ref
        return m

    shared = glowing(lookup("palette|sRGB"))
    shared.lookups[abi.SLOT_BASE_COLOR] = lookup("palette|sRGB")
    looks = {
        "Warm": preview_material(emission=(1.0, 0.6, 0.2)),
        "Bright": preview_material(emission=(6.0, 6.0, 6.0)),
        "Dim": preview_material(emission=(0.05, 0.1, 0.2)),
        "Clamped": preview_material(emission=(2.0, 0.0, 0.5)),
        "NonFinite": preview_material(),
        "Metal": preview_material(base_color=(0.95, 0.64, 0.54), roughness=0.25, metallic=1.0,
                                  emission=(0.6, 0.2, 0.1)),
        "Cool": preview_material(emission=(0.4, 0.8, 1.0)),
        "Srgb": glowing(lookup("palette|sRGB")),
        "Raw": glowing(lookup("palette|raw")),
        "Auto": glowing(lookup("palette|auto")),
        "Grey": glowing(lookup("ramp|auto")),
        "ScaleBias": glowing(lookup("palette|raw", scale=(3, 3, 3, 1), bias=(0.2, 0.1, 0.0, 0.0))),
        "Missing": glowing(lookup("missing|sRGB", fallback=(2.0, 1.0, 0.5, 1.0))),
        "Inverted": glowing(lookup("palette|raw", scale=(-1, -1, -1, 1), bias=(1, 1, 1, 0))),
        "Hdr": glowing(lookup("glow|raw")),
        "HdrAuto": glowing(lookup("glow|auto")),
        "HdrSrgb": glowing(lookup("glow|sRGB")),
        "SphereTextured": glowing(lookup("palette|sRGB", rep)),
        "Shared": shared,
        "Unlit": glowing(lookup("palette|sRGB"), base_color=(0.0, 0.0, 0.0), ior=1.0),
        "Base": preview_material(base_color=(0.6, 0.6, 0.6), roughness=0.3),
    }
    slot = {name: s.add_material(m) for name, m in looks.items()}

    points, faces = coarse_sphere_polygons()
    corners = coarse_sphere_corners(faces)
    fixed = np.array([[_fixed(c) for c in p] for p in points], dtype=F32)
    tris = np.array([[corners[i][0], corners[i + 1][0], corners[i + 2][0]] for i in range(0, len(corners), 3)],
                    dtype=np.uint32)
    faceted = s.add_geometry(fixed, tris)
    smooth = s.add_geometry(fixed, tris, np.array([fixed[v] for v, _, _ in corners], dtype=F32).reshape(-1, 3, 3))
    textured = s.add_geometry(fixed, tris)
    latlong = coarse_sphere_latlong()
    s.set_texcoords(textured, np.array([latlong[fv] for _, _, fv in corners], dtype=F32).reshape(1, -1, 3, 2))
    card_p = np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32)
    plain = s.add_geometry(card_p, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    mapped = s.add_geometry(card_p, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    s.set_texcoords(mapped, np.array([[[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]]], dtype=F32))
    back = s.add_geometry(card_p, np.array([[0, 3, 2], [0, 2, 1]], dtype=np.uint32))
    # TwoQuads' faces as the subset split leaves them (FacesOf): the left
    # quad's points 0, 1, 4, 5 and the right quad's 1, 2, 3, 4.
    left = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.0, -0.5, 0.0), (0.0, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32),
                          np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    right = s.add_geometry(np.array([(0.0, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (0.0, 0.5, 0.0)], dtype=F32),
                           np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    sph, crd = (0.35, 0.35, 0.35), (0.7, 0.7, 0.7)
    objects = [
        ("Warm", plain, crd, 0), ("Bright", plain, crd, 0), ("Dim", plain, crd, 0), ("Clamped", plain, crd, 0),
        ("NonFinite", plain, crd, 0), ("Metal", smooth, sph, 0), ("Warm", back, crd, 0),
        ("Warm", plain, (-0.7, 0.7, 0.7), 0), ("Warm", plain, (0.7, 0.35, 0.7), 0), ("Cool", faceted, sph, 0),
        ("Srgb", mapped, crd, 0), ("Raw", mapped, crd, 0), ("Auto", mapped, crd, 0), ("Grey", mapped, crd, 0),
        ("ScaleBias", mapped, crd, 0), ("Missing", mapped, crd, 0), ("Inverted", mapped, crd, 0),
        ("Hdr", mapped, crd, 0), ("HdrAuto", mapped, crd, 0), ("HdrSrgb", mapped, crd, 0),
        ("Warm", plain, crd, 60), ("SphereTextured", textured, sph, 0), ("Shared", mapped, crd, 0),
        ("Unlit", mapped, crd, 0), ("Base", None, crd, 0),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (look, geo, scale, rotate_x) in enumerate(objects):
        t = np.eye(4)
        t[0, 3], t[1, 3] = columns[i % 5], rows[i // 5]
        c, sn = math.cos(rotate_x * math.pi / 180), math.sin(rotate_x * math.pi / 180)
        rx = np.array([[1, 0, 0, 0], [0, c, -sn, 0], [0, sn, c, 0], [0, 0, 0, 1]], dtype=np.float64)
        sc = np.diag([scale[0], scale[1], scale[2], 1.0])
        m = (t @ rx @ sc).astype(F32).reshape(-1, order="F")
        if geo is None:
            s.add_instance(left, slot["Base"], m)
            s.add_instance(right, slot["Warm"], m)
        else:
            s.add_instance(geo, slot[look], m, texcoord_set=1 if geo in s.texcoords else 0)
    return s


def _place2d(pivot, scale, degrees, offset, order):
    """ND_place2d's st matrix in double (Place2d, material_fixtures.cpp:
    1394-1413 in hydra-lotus): it moves by the offset, rotates about the
    pivot and divides by the scale, in operation order `order`."""
    c, s = math.cos(degrees * (math.pi / 180.0)), math.sin(degrees * (math.pi / 180.0))
    m = [0.0] * 6
    if order == 0:
        m[0], m[1] = c / scale[0], s / scale[1]
        m[3], m[4] = -s / scale[0], c / scale[1]
        m[2] = -(m[0] * pivot[0] + m[1] * pivot[1]) - offset[0] + pivot[0]
        m[5] = -(m[3] * pivot[0] + m[4] * pivot[1]) - offset[1] + pivot[1]
    else:
        m[0], m[1] = c / scale[0], s / scale[0]
        m[3], m[4] = -s / scale[1], c / scale[1]
        x, y = -pivot[0] - offset[0], -pivot[1] - offset[1]
        m[2] = (c * x + s * y) / scale[0] + pivot[0]
        m[5] = (-s * x + c * y) / scale[1] + pivot[1]
    return m


def gltf_place(scale, degrees, offset):
    """ND_gltf_image's placement as the reference's translator composes it
    (GltfPlace, material_fixtures.cpp:1415-1421): ND_place2d about (0, 1)
    in order 0, the scale inverted, the rotation negated and the offset
    negated in s; rounded to float."""
    m = _place2d((0.0, 1.0), (1.0 / scale[0], 1.0 / scale[1]), -degrees, (-offset[0], offset[1]), 0)
    return tuple(float(F32(v)) for v in m)


def _palette(x, y):
    return (40 + 60 * x, 40 + 60 * y, 200 if (x + y) % 2 == 0 else 60, 255)


def _rgba(x, y):
    return (220 - 60 * x, 40 + 60 * y, 40 + 60 * ((x + y) % 4), 30 + 65 * x)


def _tilts(x, y):
    return (32 + 64 * x, 224 - 64 * y, 200, 255)


def _cutout(x, y):
    dx, dy = 2 * x - 7, 2 * y - 7
    d = dx * dx + dy * dy
    return (60 + 20 * x, 200 - 15 * y, 60, 255 if d <= 26 else (96 if d <= 50 else 0))


def _unit_card(s):
    """A unit card in the XY plane with the st set over the unit square
    (Card({{"st", Corners(kUnit)}}), material_fixtures.cpp:315-330)."""
    g = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)],
                                dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    s.set_texcoords(g, np.array([[[(0, 0), (1, 0), (1, 1)], [(0, 0), (1, 1), (0, 1)]]], dtype=F32))
    return g


def _wrapped_sphere(s):
    """The coarse sphere with its points as corner normals and the st set
    longitude by latitude times (4, 2)."""
    g = _coarse_smooth_sphere(s)
    points, faces = coarse_sphere_polygons()
    corners = coarse_sphere_corners(faces)
    latlong = coarse_sphere_latlong()
    s.set_texcoords(g, np.array([latlong[fv] for _, _, fv in corners], dtype=F32).reshape(1, -1, 3, 2))
    return g


def material_gltf(exchanged_channels=False, size=160):
    """The reference's material-gltf-v1 fixture (SetMaterialGltf,
    material_fixtures.cpp:2274-2371 in hydra-lotus), which its golden
    images validation/reference/material-gltf-v1-{mean,variance}.pfm were
    rendered from: MaterialX's glTF PBR surface on a 5x5 grid in the
    material studio, coarse spheres (scale 0.35) and st-mapped cards (scale
    0.7). Rows from the top: constants (the definition's defaults, a red
    dielectric, a glossy grey, copper, a half-metal); base-colour images
    (plain, a factor, the same as ND_gltf_colorimage, copper with metallic
    and roughness packed in one image, a placed image); normal maps and
    emission; alpha modes; unrepresented inputs, which render as the rest
    of the material. ``exchanged_channels`` reads Packed's metallic from
    green and roughness from blue (the fixture's negative control,
    ExchangedChannels)."""
    s = material_studio("material-gltf-v1", size)
    palette_tex = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_SRGB)
    rgba_tex = s.add_texture(_texture_image(4, _rgba), abi.TEXTURE_RGBA8_UNORM)
    tilts_tex = s.add_texture(_texture_image(4, _tilts), abi.TEXTURE_RGBA8_UNORM)
    cutout_tex = s.add_texture(_texture_image(8, _cutout), abi.TEXTURE_RGBA8_SRGB)
    rep = abi.WRAP_REPEAT
    copper, red, teal, grey = (0.95, 0.64, 0.54), (0.8, 0.2, 0.1), (0.2, 0.6, 0.7), (0.7, 0.7, 0.7)
    transparent = (0.0, 0.0, 0.0, 0.0)

    def periodic(texture, **kw):
        return s.add_texture_input(texture, wrap_s=rep, wrap_t=rep, **kw)

    palette = periodic(palette_tex, fallback=transparent)
    tinted = periodic(palette_tex, fallback=transparent, scale=(1.0, 0.5, 0.25, 1.0))
    rotated = periodic(palette_tex, fallback=transparent, st_transform=gltf_place((2.0, 1.0), 30.0,
                                                                                   (float(F32(0.1)), float(F32(0.2)))))

    def textured(lookup):
        m = gltf_material((1.0, 1.0, 1.0), 0.0, 0.6)
        m.lookups[abi.GLTF_SLOT_BASE_COLOR] = lookup
        return m, True

    packed = gltf_material(copper, 1.0, 1.0)
    packed.lookups[abi.GLTF_SLOT_METALLIC] = periodic(rgba_tex, fallback=transparent,
                                                      channel=1 if exchanged_channels else 2)
    packed.lookups[abi.GLTF_SLOT_ROUGHNESS] = periodic(rgba_tex, fallback=transparent,
                                                       channel=2 if exchanged_channels else 1)
    bumps = periodic(tilts_tex, scale=(2.0, 2.0, 2.0, 1.0), bias=(-1.0, -1.0, -1.0, 0.0),
                     fallback=(-1.0, -1.0, -1.0, 1.0))
    gltf_bumps = periodic(tilts_tex, scale=(2.0, 2.0, 2.0, 1.0), bias=(-1.0, -1.0, -1.0, 0.0),
                          fallback=(0.0, 0.0, 1.0, 1.0))

    def bumpy(m, lookup):
        m.lookups[abi.SLOT_NORMAL] = lookup
        return m, True

    emissive = gltf_material(grey, 0.0, 0.4, emissive=(1.0, 0.6, 0.2))
    emissive_map = gltf_material(grey, 0.0, 0.4, emissive_strength=2.0)
    emissive_map.lookups[abi.GLTF_SLOT_EMISSIVE] = periodic(palette_tex)
    cutout = periodic(cutout_tex, fallback=transparent)
    mask = gltf_material((1.0, 1.0, 1.0), 0.0, 0.6, opacity_threshold=0.5)
    mask.lookups[abi.GLTF_SLOT_BASE_COLOR] = cutout
    mask.lookups[abi.SLOT_OPACITY] = periodic(cutout_tex, fallback=transparent, channel=3)
    blend = gltf_material((1.0, 1.0, 1.0), 0.0, 0.6, opacity_threshold=0.0)
    blend.lookups[abi.GLTF_SLOT_BASE_COLOR] = cutout
    blend.lookups[abi.SLOT_OPACITY] = periodic(cutout_tex, fallback=transparent, channel=3)
    unlit = gltf_material((0.0, 0.0, 0.0), 0.0, 1.0, emissive=teal, specular=0.0)
    looks = [
        ("Defaults", (gltf_material((1.0, 1.0, 1.0), 1.0, 1.0), False)),
        ("Dielectric", (gltf_material(red, 0.0, 0.5), False)),
        ("Glossy", (gltf_material((0.5, 0.5, 0.5), 0.0, 0.1), False)),
        ("Metal", (gltf_material(copper, 1.0, 0.3), False)),
        ("Mixed", (gltf_material((0.9, 0.6, 0.2), 0.5, 0.3), False)),
        ("Image", textured(palette)),
        ("Factor", textured(tinted)),
        ("ColorImage", textured(tinted)),
        ("Packed", (packed, True)),
        ("Rotated", textured(rotated)),
        ("GltfNormal", bumpy(gltf_material(grey, 0.0, 0.4), gltf_bumps)),
        ("NormalMap", bumpy(gltf_material(grey, 0.0, 0.4), bumps)),
        ("NormalMetal", bumpy(gltf_material(copper, 1.0, 0.25), gltf_bumps)),
        ("Emissive", (emissive, False)),
        ("EmissiveMap", (emissive_map, True)),
        ("Opaque", (gltf_material(teal, 0.0, 0.5), False)),
        ("Mask", (mask, True)),
        ("MaskZero", (gltf_material(teal, 0.0, 0.5), False)),
        ("MaskAll", (gltf_material(teal, 0.0, 0.5, opacity=0.0), False)),
        ("Blend", (blend, True)),
        ("Iridescence", (gltf_material(red, 0.0, 0.5), False)),
        ("Thickness", (gltf_material(red, 0.0, 0.5), False)),
        ("Unlit", (unlit, False)),
        ("Anisotropy", (gltf_material(red, 0.0, 0.5), False)),
        ("VertexColor", (gltf_material((1.0, 1.0, 1.0), 0.0, 0.6), False)),
    ]
    smooth = _coarse_smooth_sphere(s)
    wrapped = _wrapped_sphere(s)
    card = _unit_card(s)
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (name, (m, uses_st)) in enumerate(looks):
        ball = i < 5 or name == "NormalMetal"
        geo = wrapped if name == "NormalMetal" else (smooth if ball else card)
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.35 if ball else 0.7
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        s.add_instance(geo, s.add_material(m), placed,
                       texcoord_set=1 if uses_st and geo in s.texcoords else 0)
    return s


def material_gltf_extensions(exchanged_coat=False, size=160):
    """The reference's material-gltf-extensions-v1 fixture
    (SetMaterialGltfExtensions, material_fixtures.cpp:2063-2272 in
    hydra-lotus), which its golden images validation/reference/
    material-gltf-extensions-v1-{mean,variance}.pfm were rendered from:
    glTF PBR's extensions on the 5x5 grid in the material studio. Rows from
    the top: the dielectric's reflection (ior 1 and 2.4, half specular, a
    tinted and a mapped specular); thin transmission on cards; clearcoat
    (over a rough red dielectric and copper, rough, over a normal-mapped
    base, with its own normal map); sheen over a dark rough dielectric;
    every extension together, mapped coat and specular colour, and inputs
    the model does not represent. Spheres are wrapped in (s, t) where a
    lookup reads. ``exchanged_coat`` swaps CoatRough's clearcoat weight and
    roughness (the fixture's negative control, ExchangedCoat)."""
    s = material_studio("material-gltf-extensions-v1", size)
    palette_tex = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_SRGB)
    rgba_tex = s.add_texture(_texture_image(4, _rgba), abi.TEXTURE_RGBA8_UNORM)
    tilts_tex = s.add_texture(_texture_image(4, _tilts), abi.TEXTURE_RGBA8_UNORM)
    rep = abi.WRAP_REPEAT
    transparent = (0.0, 0.0, 0.0, 0.0)
    copper, red, teal = (0.95, 0.64, 0.54), (0.8, 0.2, 0.1), (0.2, 0.6, 0.7)
    dark, white = (0.05, 0.05, 0.08), (1.0, 1.0, 1.0)

    def periodic(texture, **kw):
        return s.add_texture_input(texture, wrap_s=rep, wrap_t=rep, **kw)

    palette = periodic(palette_tex, fallback=transparent)

    def scalars(channel):
        return periodic(rgba_tex, fallback=transparent, channel=channel)

    bumps = periodic(tilts_tex, scale=(2.0, 2.0, 2.0, 1.0), bias=(-1.0, -1.0, -1.0, 0.0),
                     fallback=(0.0, 0.0, 1.0, 1.0))
    looks = []

    def add(name, base, metallic, roughness, textured=False, **kw):
        m = gltf_material(base, metallic, roughness, **kw)
        looks.append((name, m, textured))
        return m

    # The dielectric's reflection.
    add("IorOne", red, 0.0, 0.2, ior=1.0)
    add("IorHigh", red, 0.0, 0.2, ior=2.4)
    add("SpecularHalf", red, 0.0, 0.2, specular=0.5)
    add("SpecularTint", (0.6, 0.6, 0.6), 0.0, 0.2, ior=2.4, specular_color=(1.0, 0.3, 0.1))
    add("SpecularMap", red, 0.0, 0.2, True, ior=2.4).lookups[abi.GLTF_SLOT_SPECULAR] = scalars(0)
    # Transmission.
    add("Glass", white, 0.0, 0.0, transmission=1.0)
    add("GlassRough", white, 0.0, 0.4, transmission=1.0)
    add("GlassTinted", teal, 0.0, 0.0, transmission=1.0)
    add("GlassHalf", (0.9, 0.6, 0.2), 0.0, 0.3, transmission=0.5)
    add("GlassMap", white, 0.0, 0.1, True).lookups[abi.GLTF_SLOT_TRANSMISSION] = scalars(1)
    # Clearcoat.
    add("Coat", red, 0.0, 0.7, clearcoat=1.0)
    add("CoatMetal", copper, 1.0, 0.4, clearcoat=0.5)
    add("CoatRough", red, 0.0, 0.7, clearcoat=0.5 if exchanged_coat else 1.0,
        clearcoat_roughness=1.0 if exchanged_coat else 0.5)
    add("CoatOverBumps", red, 0.0, 0.7, True, clearcoat=1.0).lookups[abi.SLOT_NORMAL] = bumps
    add("CoatNormal", red, 0.0, 0.7, True, clearcoat=1.0).lookups[abi.GLTF_SLOT_CLEARCOAT_NORMAL] = bumps
    # Sheen.
    add("Sheen", dark, 0.0, 0.8, sheen_color=white, sheen_roughness=0.7)
    add("SheenColor", dark, 0.0, 0.8, sheen_color=(0.9, 0.4, 0.1), sheen_roughness=0.5)
    add("SheenRough", dark, 0.0, 0.8, sheen_color=(0.5, 0.5, 0.5), sheen_roughness=1.0)
    sheen_map = add("SheenMap", dark, 0.0, 0.8, True)
    sheen_map.lookups[abi.GLTF_SLOT_SHEEN_COLOR] = palette
    sheen_map.lookups[abi.GLTF_SLOT_SHEEN_ROUGHNESS] = scalars(1)
    add("SheenCoat", dark, 0.0, 0.8, sheen_color=(0.9, 0.4, 0.1), sheen_roughness=0.5, clearcoat=1.0)
    # Together, mapped weights, and unrepresented inputs.
    add("All", (0.9, 0.6, 0.2), 0.3, 0.4, ior=1.8, specular=0.8, specular_color=(1.0, 0.8, 0.6),
        transmission=0.4, clearcoat=0.7, clearcoat_roughness=0.2, sheen_color=(0.3, 0.5, 0.8),
        sheen_roughness=0.6)
    coat_map = add("CoatMap", red, 0.0, 0.7, True)
    coat_map.lookups[abi.GLTF_SLOT_CLEARCOAT] = scalars(0)
    coat_map.lookups[abi.GLTF_SLOT_CLEARCOAT_ROUGHNESS] = scalars(2)
    add("SpecularColorMap", (0.6, 0.6, 0.6), 0.0, 0.2, True, ior=2.4).lookups[
        abi.GLTF_SLOT_SPECULAR_COLOR] = palette
    add("Thickness", teal, 0.0, 0.0, transmission=1.0)
    add("Diagnosed", red, 0.0, 0.7, clearcoat=1.0)

    smooth = _coarse_smooth_sphere(s)
    wrapped = _wrapped_sphere(s)
    card = _unit_card(s)
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (name, m, textured) in enumerate(looks):
        is_card = name.startswith("Glass") or name == "Thickness"
        geo = card if is_card else (wrapped if textured else smooth)
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.7 if is_card else 0.35
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        s.add_instance(geo, s.add_material(m), placed, texcoord_set=1 if textured else 0)
    return s


# The reference's glTF furnace planes (GltfFurnaceFailure,
# adapters/headless/main.cpp:1632-1700 in hydra-lotus): white glTF PBR
# materials that return a white environment whatever their lobes.
GLTF_FURNACE_PLANES = {
    "dielectric": {"metallic": 0.0, "roughness": 0.2},
    "rough dielectric": {"metallic": 0.0, "roughness": 1.0},
    "metal": {"metallic": 1.0, "roughness": 0.2},
    "rough metal": {"metallic": 1.0, "roughness": 1.0},
    "clearcoat": {"metallic": 0.0, "roughness": 0.5, "clearcoat": 1.0},
    "rough clearcoat": {"metallic": 0.0, "roughness": 0.5, "clearcoat": 0.5, "clearcoat_roughness": 0.4},
    "sheen": {"metallic": 0.0, "roughness": 0.5, "sheen_color": (1.0, 1.0, 1.0), "sheen_roughness": 0.7},
    "transmission": {"metallic": 0.0, "roughness": 0.2, "transmission": 1.0},
    "half transmission": {"metallic": 0.0, "roughness": 0.5, "transmission": 0.5, "specular": 0.5},
    "every extension": {"metallic": 0.3, "roughness": 0.5, "ior": 1.8, "transmission": 0.4, "clearcoat": 0.7,
                        "clearcoat_roughness": 0.2, "sheen_color": (0.5, 0.5, 0.5), "sheen_roughness": 0.6},
}


def gltf_furnace(plane, cos_view, size=64):
    """A 32x32 white glTF PBR plane tilted about X to view cosine
    `cos_view` under a white constant environment, seen by the bootstrap
    camera with an orthographic projection (GltfFurnaceFailure,
    adapters/headless/main.cpp:1700-1720): no scattered ray meets the plane
    again, so each pixel's mean is the closure's directional albedo, 1 for
    an energy-conserving white closure."""
    s = Scene(f"gltf-furnace-{plane}-{cos_view}")
    view = identity()
    view[14] = -3.0
    projection = identity()
    projection[10] = F32(-2.0) / F32(9.0)
    projection[14] = F32(-11.0) / F32(9.0)
    s.world_to_clip = multiply(projection, view)
    s.width = s.height = size
    s.environment_constant = (1.0, 1.0, 1.0)
    g = s.add_geometry(np.array([(-16, -16, 0), (16, -16, 0), (16, 16, 0), (-16, 16, 0)], dtype=F32),
                       np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
    tilted = identity()
    sin_view = float(F32(math.sqrt(1.0 - float(F32(cos_view)) ** 2)))
    tilted[5], tilted[6], tilted[9], tilted[10] = cos_view, sin_view, -sin_view, cos_view
    s.add_instance(g, s.add_material(gltf_material(**GLTF_FURNACE_PLANES[plane])), tilted)
    return s


def material_primvars(swapped_colors=False, size=160):
    """The reference's material-primvars-v1 fixture (SetMaterialPrimvars,
    material_fixtures.cpp:1941-2031 in hydra-lotus), which its golden images
    validation/reference/material-primvars-v1-{mean,variance}.pfm were
    rendered from, in the form its translator hands the renderer: cards and
    two-quad meshes (scale 0.7, the middle three rows of the 5x5 grid) whose
    colour sets a UsdPreviewSurface material's base colour reads by name —
    per corner (vertex, varying, face-varying), per face, one value for the
    mesh, displayColor, an absent set (the material's own colour), an
    out-of-range colour the shader clamps, a set no material reads, unbound
    meshes' displayColor, and displayOpacity as constant coverage.
    ``swapped_colors`` swaps red and blue of the Vertex mesh's colours (the
    fixture's negative control, SwappedColors)."""
    s = material_studio("material-primvars-v1", size)
    corners = [(1, 0, 0), (1, 1, 0), (0, 1, 1), (0, 0, 1)]
    straight, reversed_ = (0, 1, 2, 3), (3, 2, 1, 0)

    def card():
        return s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)],
                                       dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))

    def colored(at, swap=False):
        g = card()
        values = [corners[at[c]] for c in (0, 1, 2, 0, 2, 3)]
        if swap:
            values = [(b, gg, r) for r, gg, b in values]
        s.set_colors(g, [values])
        return g

    def constant(color):
        g = card()
        s.set_colors(g, [[color]])
        return g

    def uniform():
        g = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.0, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0),
                                     (0.0, 0.5, 0.0), (-0.5, 0.5, 0.0)], dtype=F32),
                           np.array([[0, 1, 4], [0, 4, 5], [1, 2, 3], [1, 3, 4]], dtype=np.uint32))
        faces = (0, 0, 1, 1)
        s.set_colors(g, [[(1.0, 0.5, 0.0) if f == 0 else (0.0, 0.5, 1.0) for f in faces for _ in range(3)]])
        return g

    reader = lambda fallback=(0.0, 0.0, 0.0): preview_material(fallback, roughness=0.4)
    teal = (0.2, 0.6, 0.7)
    looks = {
        "Tint": reader(),
        "Display": reader(),
        "Absent": reader((1.0, 0.25, 0.0)),
        "Unnamed": reader((0.25, 0.5, 0.75)),
        "Glowing": preview_material((0.5, 0.5, 0.5)),
        "Varying": preview_material(),
        "OpacityColor": preview_material(teal, opacity=0.25),
        "OpacityOnly": preview_material(opacity=0.5),
        "Teal": preview_material(teal),
    }
    slot = {name: s.add_material(m) for name, m in looks.items()}
    # (geometry, material, whether the material reads the mesh's one set)
    objects = [
        (colored(straight, swapped_colors), "Tint", True),
        (colored(straight), "Tint", True),
        (colored(reversed_), "Tint", True),
        (uniform(), "Tint", True),
        (constant((0.25, 0.75, 0.5)), "Tint", True),
        (constant((0.2, 0.6, 0.7)), "Display", True),
        (card(), "Absent", False),
        (constant((1.5, -0.5, 0.5)), "Unnamed", True),
        (colored(straight), "Glowing", False),
        (colored(straight), "Varying", True),
        (uniform(), "Varying", True),
        (colored(reversed_), "Varying", True),
        (card(), "OpacityColor", False),
        (card(), "OpacityOnly", False),
        (card(), "Teal", False),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (0.8, 0.0, -0.8)
    for i, (geo, look, reads) in enumerate(objects):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.7
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        s.add_instance(geo, slot[look], placed, color_set=1 if reads else 0)
    return s


def _faces_of(points, triangles, faces_of_triangle, faces, normals=None, texcoords=None, colors=None):
    """The part of a mesh a GeomSubset binds, as extraction hands it over
    (FacesOf, material_fixtures.cpp:342-375 in hydra-lotus): the triangles
    whose source face is in `faces`, in order, the points they use in
    point order, and their corners' normals, texture-coordinate sets and
    colour sets (a whole-mesh colour kept whole). `texcoords` and `colors`
    are lists of per-corner arrays in key order."""
    kept = [t for t in range(len(triangles)) if faces_of_triangle[t] in faces]
    used = sorted({int(v) for t in kept for v in triangles[t]})
    index = {v: i for i, v in enumerate(used)}
    part_points = np.array([points[v] for v in used], dtype=F32)
    part_tris = np.array([[index[int(v)] for v in triangles[t]] for t in kept], dtype=np.uint32)
    part_normals = None if normals is None else np.array([normals[t] for t in kept], dtype=F32)
    part_st = [np.array([s[3 * t:3 * t + 3] for t in kept], dtype=F32).reshape(-1, 3, 2) for s in texcoords or []]
    part_colors = [c if len(c) == 1 else [c[3 * t + k] for t in kept for k in range(3)] for c in colors or []]
    return part_points, part_tris, part_normals, part_st, part_colors


def material_subsets(ignored_subset=False, size=160):
    """The reference's material-subsets-v1 fixture (SetMaterialSubsets,
    material_fixtures.cpp:1840-1939 in hydra-lotus), which its golden images
    validation/reference/material-subsets-v1-{mean,variance}.pfm were
    rendered from, in the form extraction hands the renderer: each bound
    GeomSubset a mesh of its own faces (and the rest of the mesh another),
    each with its material — partial and full splits, an unbound rest lit by
    displayColor, a subset without a binding, another family, coordinate
    sets per part, an emitting part, a half-covered part, overlapping and
    out-of-range subsets, a sphere's top, a hole, a material shared by two
    parts, a colour set per part and a mirrored card. ``ignored_subset``
    binds Partial's subset to the mesh's grey (the fixture's negative
    control, IgnoredSubset)."""
    s = material_studio("material-subsets-v1", size)
    palette_tex = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_SRGB)
    clamp = abi.WRAP_CLAMP
    red, blue, grey = (0.8, 0.1, 0.05), (0.1, 0.2, 0.8), (0.6, 0.6, 0.6)
    teal = (0.2, 0.6, 0.7)

    def textured():
        m = preview_material()
        m.lookups[abi.SLOT_BASE_COLOR] = s.add_texture_input(palette_tex, wrap_s=clamp, wrap_t=clamp)
        return m

    looks = {
        "Grey": (preview_material(grey, roughness=0.3), None, None),
        "Red": (preview_material(red, roughness=0.3), None, None),
        "Blue": (preview_material(blue, roughness=0.3), None, None),
        "Glow": (preview_material(emission=(2.0, 1.0, 0.5)), None, None),
        "Half": (preview_material(red, opacity=0.5), None, None),
        "Palette": (textured(), "st", None),
        "Turned": (textured(), "uv1", None),
        "Tint": (preview_material((0.0, 0.0, 0.0), roughness=0.4), None, "tint"),
        "": (preview_material(teal), None, None),  # an unbound part's displayColor material
    }
    slot = {name: s.add_material(m) for name, (m, _, _) in looks.items()}
    # TwoQuads: the left and right quads, faces 0 and 1.
    quad_points = [(-0.5, -0.5, 0.0), (0.0, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (0.0, 0.5, 0.0),
                   (-0.5, 0.5, 0.0)]
    quad_tris = [(0, 1, 4), (0, 4, 5), (1, 2, 3), (1, 3, 4)]
    quad_faces = (0, 0, 1, 1)

    def corners(face):
        return [face[0], face[1], face[2], face[0], face[2], face[3]]

    left = [(0, 0), (0.5, 0), (0.5, 1), (0, 1)]
    right = [(0.5, 0), (1, 0), (1, 1), (0.5, 1)]
    swap = lambda face: [(t_, s_) for s_, t_ in face]
    sets_st = {"st": corners(left) + corners(right), "uv1": corners(swap(left)) + corners(swap(right))}
    tints = [(1, 0, 0), (1, 0.5, 0), (1, 1, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)]
    tinted = {"tint": [tints[v] for tri in quad_tris for v in tri]}
    teal_colors = {"displayColor": [teal]}

    def quads(faces, st=None, colors=None):
        st_names = sorted(st) if st else []
        color_names = sorted(colors) if colors else []
        p, t, _, part_st, part_colors = _faces_of(
            quad_points, quad_tris, quad_faces, faces, texcoords=[st[n] for n in st_names],
            colors=[colors[n] for n in color_names])
        return (p, t, None, dict(zip(st_names, part_st)), dict(zip(color_names, part_colors)))

    points, polys = coarse_sphere_polygons()
    sphere_corners = coarse_sphere_corners(polys)
    fixed = [[_fixed(c) for c in p] for p in points]
    sphere_tris = [(sphere_corners[i][0], sphere_corners[i + 1][0], sphere_corners[i + 2][0])
                   for i in range(0, len(sphere_corners), 3)]
    sphere_faces = [sphere_corners[i][1] for i in range(0, len(sphere_corners), 3)]
    sphere_normals = np.array([fixed[v] for v, _, _ in sphere_corners], dtype=F32).reshape(-1, 3, 3)

    def ball(faces):
        p, t, n, _, _ = _faces_of(fixed, sphere_tris, sphere_faces, faces, normals=sphere_normals)
        return (p, t, n, {}, {})

    top, bottom = set(range(32)), set(range(32, len(polys)))
    whole = quads({0, 1})

    def partial(mesh_look, subset_look):
        return [(quads({0}), mesh_look), (quads({1}), subset_look)]

    objects = [
        (partial("Grey", "Grey" if ignored_subset else "Red"), 0.7, 0.7),
        ([(quads({0}), "Red"), (quads({1}), "Blue")], 0.7, 0.7),
        ([(quads({0}, colors=teal_colors), ""), (quads({1}, colors=teal_colors), "Red")], 0.7, 0.7),
        ([(whole, "Blue")], 0.7, 0.7),
        (partial("Blue", "Red"), 0.7, 0.7),
        ([(quads({0}, st=sets_st), "Turned"), (quads({1}, st=sets_st), "Palette")], 0.7, 0.7),
        (partial("Grey", "Glow"), 0.7, 0.7),
        (partial("Grey", "Half"), 0.7, 0.7),
        ([(whole, "Red")], 0.7, 0.7),
        (partial("Grey", "Red"), 0.7, 0.7),
        ([(ball(bottom), "Grey"), (ball(top), "Red")], 0.35, 0.35),
        ([(quads({1}), "Red")], 0.7, 0.7),
        ([(quads({0}), "Red"), (quads({1}), "Red")], 0.7, 0.7),
        ([(quads({0}, colors=tinted), "Grey"), (quads({1}, colors=tinted), "Tint")], 0.7, 0.7),
        (partial("Grey", "Red"), -0.7, 0.7),
    ]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (0.8, 0.0, -0.8)
    for i, (parts, scale_x, scale) in enumerate(objects):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0], placed[5], placed[10] = scale_x, scale, scale
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        for (p, t, n, st, colors), look in parts:
            g = s.add_geometry(p, t, n)
            st_names, color_names = sorted(st), sorted(colors)
            if st_names:
                s.set_texcoords(g, np.stack([st[k] for k in st_names]))
            if color_names:
                s.set_colors(g, [colors[k] for k in color_names])
            _, wants_st, wants_color = looks[look]
            tex_set = st_names.index(wants_st) + 1 if wants_st in st_names else 0
            color_set = color_names.index(wants_color) + 1 if wants_color in color_names else 0
            s.add_instance(g, slot[look], placed, texcoord_set=tex_set, color_set=color_set)
    return s


def _ramp(x, y):
    v = 15 + 15 * (x + 4 * y)
    return (v, v, v, 255)


def material_mtlx(unweighted_image=False, size=160):
    """The reference's material-mtlx-v1 fixture (SetMaterialMtlx,
    material_fixtures.cpp:1247-1382 in hydra-lotus), which its golden
    images validation/reference/material-mtlx-v1-{mean,variance}.pfm were
    rendered from, in the form its MaterialX translator hands the renderer:
    Standard Surface networks as UsdPreviewSurface materials (weighted base
    colours, metal, ior 2.5 and 1, emission times its colour, opacity,
    clamped inputs, unrepresented lobes, precedence over a preview
    surface), image lookups (sRGB and raw, a weighted image, metalness and
    roughness channels, an emission map, periodic / clamp / mirror /
    constant addressing, a named coordinate set, normal maps at two scales,
    tiling) and defaults of what is not translated, on coarse spheres
    (scale 0.35) and cards (0.7) of the 5x5 grid. ``unweighted_image``
    drops the weighted image's 0.5 base weight (the fixture's negative
    control, UnweightedImage)."""
    s = material_studio("material-mtlx-v1", size)
    srgb = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_SRGB)
    raw = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_UNORM)
    rgba = s.add_texture(_texture_image(4, _rgba), abi.TEXTURE_RGBA8_UNORM)
    ramp = s.add_texture(_texture_image(4, _ramp), abi.TEXTURE_RGBA8_UNORM)
    tilts = s.add_texture(_texture_image(4, _tilts), abi.TEXTURE_RGBA8_UNORM)
    rep, clamp, mirror, black = abi.WRAP_REPEAT, abi.WRAP_CLAMP, abi.WRAP_MIRROR, abi.WRAP_BLACK

    def standard(base=(0.8, 0.8, 0.8), roughness=0.2, **kw):
        return preview_material(base, roughness=roughness, **kw)

    def textured(texture, wrap=rep, uv="st", **kw):
        m = standard()
        m.lookups[abi.SLOT_BASE_COLOR] = s.add_texture_input(texture, wrap_s=wrap, wrap_t=wrap, **kw)
        return m, uv

    def bumpy(scale):
        m = standard((0.7, 0.7, 0.7), 0.4)
        m.lookups[abi.SLOT_NORMAL] = s.add_texture_input(
            tilts, wrap_s=rep, wrap_t=rep, scale=(2.0 * scale, 2.0 * scale, 2.0, 1.0),
            bias=(-scale, -scale, -1.0, 0.0), fallback=(-scale, -scale, -1.0, 1.0))
        return m, "st"

    copper, teal, black_ = (0.95, 0.64, 0.54), (0.2, 0.6, 0.7), (0.0, 0.0, 0.0)
    channels = standard(copper)
    channels.lookups[abi.SLOT_METALLIC] = s.add_texture_input(rgba, channel=2, wrap_s=rep, wrap_t=rep)
    channels.lookups[abi.SLOT_ROUGHNESS] = s.add_texture_input(ramp, wrap_s=rep, wrap_t=rep)
    emission_map = standard(black_)
    emission_map.lookups[abi.SLOT_EMISSION] = s.add_texture_input(raw, wrap_s=rep, wrap_t=rep)
    weight = 1.0 if unweighted_image else 0.5
    looks = {
        "Defaults": (standard(), None),
        "Weighted": (standard((float(F32(0.5) * F32(0.9)), float(F32(0.5) * F32(0.3)),
                               float(F32(0.5) * F32(0.1)))), None),
        "Metal": (standard(copper, 0.3, metallic=1.0), None),
        "Ior": (standard((0.1, 0.2, 0.6), 0.1, ior=2.5), None),
        "NoSpecular": (standard((0.6, 0.6, 0.6), 0.1, ior=1.0), None),
        "Emissive": (standard(black_, emission=(2.0, float(F32(2.0) * F32(0.6)), float(F32(2.0) * F32(0.2)))),
                     None),
        "Opacity": (standard(teal, opacity=0.5), None),
        "Clamped": (standard((1.0, float(F32(1.5) * F32(0.5)), 0.0), 1.0), None),
        "Lobes": (standard(teal), None),
        "Precedence": (standard((0.1, 0.2, 0.8)), None),
        "Srgb": textured(srgb),
        "Raw": textured(raw),
        "WeightedImage": textured(srgb, scale=(weight, weight, weight, 1.0), fallback=(0.0, 0.0, 0.0, 1.0)),
        "Channels": (channels, "st"),
        "EmissionMap": (emission_map, "st"),
        "Clamp": textured(srgb, wrap=clamp),
        "Mirror": textured(srgb, wrap=mirror),
        "Constant": textured(srgb, wrap=black),
        "Named": textured(srgb, uv="uv1"),
        "NormalMap": bumpy(1.0),
        "NormalScale": bumpy(0.5),
        "Tiled": textured(srgb),
        "Fileless": (standard((0.2, 0.6, 0.9)), None),
        "Untranslated": (standard(), None),
    }
    slot = {name: (s.add_material(m), uv) for name, (m, uv) in looks.items()}
    smooth = _coarse_smooth_sphere(s)
    bumpy_sphere = _wrapped_sphere(s)

    def card(sets):
        g = s.add_geometry(np.array([(-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0)],
                                    dtype=F32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))
        if sets:
            s.set_texcoords(g, np.array([[[f[0], f[1], f[2]], [f[0], f[2], f[3]]] for f in sets], dtype=F32))
        return g, ["st", "uv1"][:len(sets)]

    unit = [(0, 0), (1, 0), (1, 1), (0, 1)]
    wide_face = [(-0.5, -0.5), (1.5, -0.5), (1.5, 1.5), (-0.5, 1.5)]
    turned = [(1, 0), (1, 1), (0, 1), (0, 0)]
    plain, mapped, wide, named = card([]), card([unit]), card([wide_face]), card([unit, turned])
    sphere = (smooth, [])
    bumpy_geo = (bumpy_sphere, ["st"])
    objects = [("Defaults", sphere), ("Weighted", sphere), ("Metal", sphere), ("Ior", sphere),
               ("NoSpecular", sphere), ("Emissive", plain), ("Opacity", plain), ("Clamped", plain),
               ("Lobes", plain), ("Precedence", plain), ("Srgb", mapped), ("Raw", mapped),
               ("WeightedImage", mapped), ("Channels", mapped), ("EmissionMap", mapped), ("Srgb", wide),
               ("Clamp", wide), ("Mirror", wide), ("Constant", wide), ("Named", named),
               ("NormalMap", bumpy_geo), ("NormalScale", mapped), ("Tiled", mapped), ("Fileless", plain),
               ("Untranslated", mapped)]
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, (look, (geo, sets)) in enumerate(objects):
        material, uv = slot[look]
        scale = 0.35 if geo in (smooth, bumpy_sphere) else 0.7
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = scale
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        s.add_instance(geo, material, placed, texcoord_set=sets.index(uv) + 1 if uv in sets else 0)
    return s


def _srgb_to_linear(value):
    """The sRGB transfer function's decode, in double (IEC 61966-2-1)."""
    return value / 12.92 if value <= 0.04045 else ((value + 0.055) / 1.055) ** 2.4


def material_graphs(reversed_gltf_rotation=False, size=160):
    """The reference's material-graphs-v1 fixture (SetMaterialGraphs,
    material_fixtures.cpp:1440-1564 in hydra-lotus), which its golden
    images validation/reference/material-graphs-v1-{mean,variance}.pfm were
    rendered from, in the form its MaterialX graph translator hands the
    renderer: 25 st-mapped cards (scale 0.7) whose Standard Surface base
    colours come from node graphs folded into constants or texture inputs —
    sRGB and linear constants, sRGB and raw images, separated channels, a
    colour image times its colour, multiply / mix / weight / add as scale
    and bias, tiling, place2d in both operation orders, a glTF image's
    placement, coordinate arithmetic, glTF and ND normal maps, invert,
    combine, clamp, a mix's default, a file-less image's default, a folded
    power, an image's alpha as roughness, and an untranslated graph's
    default. ``reversed_gltf_rotation`` turns the glTF image's rotation the
    other way (the fixture's negative control, ReversedGltfRotation)."""
    s = material_studio("material-graphs-v1", size)
    srgb = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_SRGB)
    raw = s.add_texture(_texture_image(4, _palette), abi.TEXTURE_RGBA8_UNORM)
    rgba_tex = s.add_texture(_texture_image(4, _rgba), abi.TEXTURE_RGBA8_UNORM)
    tilts = s.add_texture(_texture_image(4, _tilts), abi.TEXTURE_RGBA8_UNORM)
    rep = abi.WRAP_REPEAT

    def standard(base=(0.8, 0.8, 0.8), roughness=0.2):
        return preview_material(base, roughness=roughness)

    def lookup(texture=None, **kw):
        return s.add_texture_input(srgb if texture is None else texture, wrap_s=rep, wrap_t=rep, **kw)

    def textured(**kw):
        m = standard()
        m.lookups[abi.SLOT_BASE_COLOR] = lookup(**kw)
        return m

    def bumpy(fallback):
        m = standard((0.7, 0.7, 0.7), 0.4)
        m.lookups[abi.SLOT_NORMAL] = lookup(tilts, scale=(2.0, 2.0, 2.0, 1.0), bias=(-1.0, -1.0, -1.0, 0.0),
                                            fallback=fallback)
        return m

    decoded = tuple(float(F32(_srgb_to_linear(float(F32(c))))) for c in (0.8, 0.4, 0.2))
    separate = standard((0.95, 0.64, 0.54))
    separate.lookups[abi.SLOT_ROUGHNESS] = lookup(rgba_tex, channel=1)
    separate.lookups[abi.SLOT_METALLIC] = lookup(rgba_tex, channel=2)
    placed_scale, placed_offset, degrees = (2.0, 1.0), (float(F32(0.1)), float(F32(0.2))), 30.0
    half = dict(scale=(0.5, 0.5, 0.5, 1.0), fallback=(0.0, 0.0, 0.0, 1.0))
    folded = tuple(float(F32((float(F32(c)) + float(F32(0.1))) ** 2.0)) for c in (0.2, 0.3, 0.4))
    alpha = standard()
    alpha.lookups[abi.SLOT_BASE_COLOR] = lookup(rgba_tex, fallback=(0.0, 0.0, 0.0, 0.0))
    alpha.lookups[abi.SLOT_ROUGHNESS] = lookup(rgba_tex, fallback=(0.0, 0.0, 0.0, 0.0), channel=3)
    rotation = -degrees if reversed_gltf_rotation else degrees
    looks = [
        standard(decoded), standard(decoded),
        textured(), textured(texture=raw), separate,
        textured(scale=(1.0, 0.5, 0.25, 1.0), fallback=(0.0, 0.0, 0.0, 0.0)),
        textured(**half), textured(**half), textured(**half),
        textured(scale=(0.5, 0.5, 0.5, 1.0), bias=(0.1, 0.1, 0.1, 0.0), fallback=(0.1, 0.1, 0.1, 1.0)),
        textured(st_transform=(2.0, 0.0, -0.25, 0.0, 3.0, -0.5)),
        textured(st_transform=tuple(float(F32(v)) for v in _place2d((0.5, 0.5), placed_scale, degrees,
                                                                      placed_offset, 0))),
        textured(st_transform=tuple(float(F32(v)) for v in _place2d((0.5, 0.5), placed_scale, degrees,
                                                                      placed_offset, 1))),
        textured(st_transform=gltf_place(placed_scale, rotation, placed_offset)),
        textured(st_transform=(2.0, 0.0, 0.25, 0.0, 2.0, 0.0)),
        bumpy((0.0, 0.0, 1.0, 1.0)), bumpy((-1.0, -1.0, -1.0, 1.0)),
        textured(scale=(-1.0, -1.0, -1.0, 1.0), bias=(1.0, 1.0, 1.0, 0.0), fallback=(1.0, 1.0, 1.0, 1.0)),
        textured(scale=(0.5, 1.0, 1.0, 1.0)),
        textured(),
        textured(scale=(0.0, 0.0, 0.0, 1.0), bias=(0.2, 0.6, 0.9, 0.0), fallback=(0.2, 0.6, 0.9, 1.0)),
        standard((float(F32(0.5) * F32(0.4)), 0.5, float(F32(0.5) * F32(1.6)))),
        standard(folded),
        alpha,
        standard(),
    ]
    card = _unit_card(s)
    columns, rows = (-1.6, -0.8, 0.0, 0.8, 1.6), (1.6, 0.8, 0.0, -0.8, -1.6)
    for i, m in enumerate(looks):
        placed = np.eye(4, dtype=F32).reshape(-1)
        placed[0] = placed[5] = placed[10] = 0.7
        placed[12], placed[13] = columns[i % 5], rows[i // 5]
        uses_st = any(k != 0 for k in m.lookups)
        s.add_instance(card, s.add_material(m), placed, texcoord_set=1 if uses_st else 0)
    return s
