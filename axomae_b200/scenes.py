"""Seeded synthetic scenes in the shape of the Nova workloads, mapped onto the reference's scene
API semantics (one principled material per mesh, u8 albedo/metallic/normal textures, a FLOATX4
environment map, a camera given by perspective + look-at matrices):

  spheres_scene      64 UV spheres (32x16 segments, 1024 triangles each incl. the pole fans) on a
                     20x20 ground quad, Lambertian albedo U[0.2, 0.8]^3, constant environment 1.0.
  heightfield_scene  an N x N quad grid (2 N^2 triangles) displaced by seeded 6-octave fBm of
                     amplitude 0.3; per-quad material drawn 50/50 from Lambert (albedo U[0.1, 0.9])
                     and GGX conductor (roughness U[0.05, 0.8], F0 U[0.5, 1.0]) through an atlas
                     with a 2x2 texel block per quad; log-normal(0, 1.5) environment map.
  mixed_scene        random spheres + boxes with Lambert / GGX conductor / GGX dielectric (IOR 1.5).
  instanced_scene    K seeded meshes placed many times with random rigid transforms.

Material mapping onto the reference's PrincipledMaterial (NovaMaterials.h:116-121):
  Lambert        metal = 0, roughness = 1 (metallic texture .g = 255, .b = 0)
  GGX conductor  metal = 1 (.b = 255), .g = roughness, albedo = F0
  GGX dielectric eta = (1.5, 1.5, 1.5), k = 0 -> transmission = 1
  Burley diffuse metal = 0, roughness from .g

The scene is a plain dictionary of numpy arrays:
  meshes     [{vertices (n,3) f32, normals, tangents, bitangents, uv (n,2), indices (m,3) u32}]
  instances  [{mesh, material, m, inv (4x4, column-major 16 floats), n (3x3 column-major 9 floats)}]
  materials  [{albedo, metallic, normalmap, emissive (texture index or -1), eta, k, anisotropy}]
  textures   [{format "u8"|"f32", pixels, width, height, channels, is_rgba, invert_u, invert_v}]
  envmap     texture index,  inv_P / inv_V  column-major 16 floats.
"""
import math

import numpy as np

IDENTITY16 = np.eye(4, dtype=np.float32).flatten(order="F")
IDENTITY9 = np.eye(3, dtype=np.float32).flatten(order="F")


def col_major(m: np.ndarray) -> np.ndarray:
    return np.asarray(m, np.float64).flatten(order="F").astype(np.float32)


def perspective(fovy_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    """glm::perspective (right-handed, depth -1..1)."""
    f = 1.0 / math.tan(math.radians(fovy_deg) / 2.0)
    P = np.zeros((4, 4))
    P[0, 0] = f / aspect
    P[1, 1] = f
    P[2, 2] = -(far + near) / (far - near)
    P[2, 3] = -2.0 * far * near / (far - near)
    P[3, 2] = -1.0
    return P


def look_at(eye, center, up) -> np.ndarray:
    """glm::lookAt (right-handed)."""
    eye, center, up = (np.asarray(v, np.float64) for v in (eye, center, up))
    f = center - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, u, -f
    V[0, 3], V[1, 3], V[2, 3] = -s @ eye, -u @ eye, f @ eye
    return V


def camera(eye, center, width, height, fovy=60.0, up=(0.0, 1.0, 0.0)):
    P = perspective(fovy, width / height, 0.1, 1000.0)
    V = look_at(eye, center, up)
    return col_major(np.linalg.inv(P)), col_major(np.linalg.inv(V)), col_major(P), col_major(V)


def transform_record(M: np.ndarray):
    """transform4x4_t {m, inv, n} for a 4x4 model matrix (n = transpose(inverse(mat3(m))))."""
    M = np.asarray(M, np.float64)
    inv = np.linalg.inv(M)
    n = np.linalg.inv(M[:3, :3]).T
    return col_major(M), col_major(inv), col_major(n)


def pack_rgba8(rgba: np.ndarray) -> np.ndarray:
    """(..., 4) uint8 -> uint32 words with r in the lowest byte (reference RGBA byte order)."""
    rgba = np.asarray(rgba, np.uint32)
    return (rgba[..., 0] | (rgba[..., 1] << 8) | (rgba[..., 2] << 16) | (rgba[..., 3] << 24)).astype(np.uint32)


def u8_texture(rgba: np.ndarray) -> dict:
    rgba = np.asarray(rgba)
    h, w = rgba.shape[:2]
    return {"format": "u8", "pixels": pack_rgba8(rgba).reshape(-1), "width": w, "height": h, "channels": 4,
            "is_rgba": 1, "invert_u": 0, "invert_v": 0}


def solid_u8(color) -> dict:
    c = np.clip(np.round(np.asarray(color, np.float64) * 255.0), 0, 255).astype(np.uint8)
    if c.size == 3:
        c = np.concatenate([c, [255]])
    return u8_texture(np.tile(c, (2, 2, 1)))


def f32_texture(rgba: np.ndarray, invert_u=0) -> dict:
    rgba = np.ascontiguousarray(rgba, np.float32)
    h, w = rgba.shape[:2]
    return {"format": "f32", "pixels": rgba.reshape(-1), "width": w, "height": h, "channels": 4, "is_rgba": 1,
            "invert_u": invert_u, "invert_v": 0}


def uv_sphere(center, radius, seg_u=32, seg_v=16):
    """UV sphere with (seg_v+1) x (seg_u+1) vertices and 2*seg_u*seg_v triangles (pole fans included,
    their pole-row triangles are geometrically degenerate like a standard UV sphere's)."""
    cu = np.arange(seg_u + 1) / seg_u
    cv = np.arange(seg_v + 1) / seg_v
    phi = cu * 2 * np.pi
    theta = cv * np.pi
    T, P = np.meshgrid(theta, phi, indexing="ij")
    n = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1)
    tan = np.stack([-np.sin(P), np.zeros_like(P), np.cos(P)], -1)
    bit = np.cross(n, tan)
    pos = np.asarray(center) + radius * n
    U, Vv = np.meshgrid(cv, cu, indexing="ij")
    uv = np.stack([Vv, U], -1)
    idx = []
    W = seg_u + 1
    for j in range(seg_v):
        for i in range(seg_u):
            a, b, c, d = j * W + i, j * W + i + 1, (j + 1) * W + i, (j + 1) * W + i + 1
            idx.append((a, b, c))  # counter-clockwise seen from outside: outward geometric normal
            idx.append((b, d, c))
    return {"vertices": pos.reshape(-1, 3).astype(np.float32), "normals": n.reshape(-1, 3).astype(np.float32),
            "tangents": tan.reshape(-1, 3).astype(np.float32), "bitangents": bit.reshape(-1, 3).astype(np.float32),
            "uv": uv.reshape(-1, 2).astype(np.float32), "indices": np.asarray(idx, np.uint32)}


def quad(size, y=0.0):
    h = size / 2.0
    v = np.array([[-h, y, -h], [h, y, -h], [h, y, h], [-h, y, h]], np.float32)
    n = np.tile([0, 1, 0], (4, 1)).astype(np.float32)
    t = np.tile([1, 0, 0], (4, 1)).astype(np.float32)
    b = np.cross(n, t).astype(np.float32)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    return {"vertices": v, "normals": n, "tangents": t, "bitangents": b, "uv": uv,
            "indices": np.array([[0, 2, 1], [0, 3, 2]], np.uint32)}


def grid_quad(size, n, y=0.0):
    """A size x size ground plane at height y tessellated into n x n quads (2 n^2 triangles, facing +y)."""
    h = size / 2.0
    c = np.arange(n + 1) / n
    X, Z = np.meshgrid(-h + size * c, -h + size * c, indexing="xy")
    v = np.stack([X, np.full_like(X, y), Z], -1).reshape(-1, 3).astype(np.float32)
    k = v.shape[0]
    nrm = np.tile([0, 1, 0], (k, 1)).astype(np.float32)
    t = np.tile([1, 0, 0], (k, 1)).astype(np.float32)
    b = np.cross(nrm, t).astype(np.float32)
    U, V = np.meshgrid(c, c, indexing="xy")
    uv = np.stack([U, V], -1).reshape(-1, 2).astype(np.float32)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a = (j * (n + 1) + i).reshape(-1)
    bb, cc, dd = a + 1, a + n + 1, a + n + 2
    idx = np.stack([np.stack([a, cc, dd], -1), np.stack([a, dd, bb], -1)], 1).reshape(-1, 3)
    return {"vertices": v, "normals": nrm, "tangents": t, "bitangents": b, "uv": uv,
            "indices": idx.astype(np.uint32)}


def box(center, half, rot):
    """Axis box of half extents `half` rotated by `rot` (3x3), 24 vertices, 12 triangles."""
    faces = []
    for axis in range(3):
        for sgn in (-1, 1):
            n = np.zeros(3)
            n[axis] = sgn
            a1, a2 = [(axis + 1) % 3, (axis + 2) % 3]
            t = np.zeros(3)
            t[a1] = 1
            bvec = np.cross(n, t)
            c = n * half[axis]
            corners = []
            for su, sv in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = c + t * su * half[a1] + bvec * sv * half[a2]
                corners.append(p)
            faces.append((np.array(corners), n, t, bvec))
    V, N, Tn, B, UV, I = [], [], [], [], [], []
    for k, (corners, n, t, bvec) in enumerate(faces):
        base = 4 * k
        for j, p in enumerate(corners):
            V.append(rot @ p + center)
            N.append(rot @ n)
            Tn.append(rot @ t)
            B.append(rot @ bvec)
            UV.append([[0, 0], [1, 0], [1, 1], [0, 1]][j])
        if np.dot(np.cross(corners[1] - corners[0], corners[2] - corners[0]), n) > 0:
            I += [(base, base + 1, base + 2), (base, base + 2, base + 3)]
        else:
            I += [(base, base + 2, base + 1), (base, base + 3, base + 2)]
    return {"vertices": np.asarray(V, np.float32), "normals": np.asarray(N, np.float32),
            "tangents": np.asarray(Tn, np.float32), "bitangents": np.asarray(B, np.float32),
            "uv": np.asarray(UV, np.float32), "indices": np.asarray(I, np.uint32)}


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


FLAT_NORMAL = (128, 128, 255, 255)


class _Builder:
    def __init__(self):
        self.meshes, self.instances, self.materials, self.textures = [], [], [], []
        self._cache = {}

    def tex(self, t: dict, key=None) -> int:
        if key is not None and key in self._cache:
            return self._cache[key]
        self.textures.append(t)
        i = len(self.textures) - 1
        if key is not None:
            self._cache[key] = i
        return i

    def flat_normal(self) -> int:
        return self.tex(u8_texture(np.tile(np.array(FLAT_NORMAL, np.uint8), (2, 2, 1))), key="flatnormal")

    def material(self, albedo_tex, metallic_tex, eta=(0, 0, 0), k=(0, 0, 0), normalmap=None) -> int:
        self.materials.append({"albedo": albedo_tex, "metallic": metallic_tex,
                               "normalmap": self.flat_normal() if normalmap is None else normalmap,
                               "emissive": -1, "eta": tuple(eta), "k": tuple(k), "anisotropy": 0.0})
        return len(self.materials) - 1

    def lambert(self, albedo) -> int:
        met = self.tex(u8_texture(np.tile(np.array([0, 255, 0, 255], np.uint8), (2, 2, 1))), key="lambert_met")
        return self.material(self.tex(solid_u8(albedo)), met)

    def conductor(self, f0, roughness) -> int:
        g = int(np.clip(round(roughness * 255), 0, 255))
        met = self.tex(u8_texture(np.tile(np.array([0, g, 255, 255], np.uint8), (2, 2, 1))))
        return self.material(self.tex(solid_u8(f0)), met)

    def dielectric(self, roughness, ior=1.5, tint=(1.0, 1.0, 1.0)) -> int:
        g = int(np.clip(round(roughness * 255), 0, 255))
        met = self.tex(u8_texture(np.tile(np.array([0, g, 0, 255], np.uint8), (2, 2, 1))))
        return self.material(self.tex(solid_u8(tint)), met, eta=(ior, ior, ior))

    def burley(self, albedo, roughness) -> int:
        g = int(np.clip(round(roughness * 255), 0, 255))
        met = self.tex(u8_texture(np.tile(np.array([0, g, 0, 255], np.uint8), (2, 2, 1))))
        return self.material(self.tex(solid_u8(albedo)), met)

    def add(self, mesh: dict, material: int, M=None) -> int:
        self.meshes.append(mesh)
        mi = len(self.meshes) - 1
        self.place(mi, material, M)
        return mi

    def place(self, mesh_index: int, material: int, M=None):
        if M is None:
            m, inv, n = IDENTITY16, IDENTITY16, IDENTITY9
        else:
            m, inv, n = transform_record(M)
        self.instances.append({"mesh": mesh_index, "material": material, "m": m, "inv": inv, "n": n})

    def finish(self, env: int, cam) -> dict:
        inv_P, inv_V, P, V = cam
        return {"meshes": self.meshes, "instances": self.instances, "materials": self.materials,
                "textures": self.textures, "envmap": env, "inv_P": inv_P, "inv_V": inv_V, "P": P, "V": V}


def spheres_scene(width=512, height=512, n_spheres=64, seed=0, seg_u=32, seg_v=16) -> dict:
    rng = np.random.default_rng(seed)
    b = _Builder()
    b.add(quad(20.0), b.lambert((0.5, 0.5, 0.5)))
    for _ in range(n_spheres):
        r = rng.uniform(0.5, 1.0)
        c = (rng.uniform(-9, 9), r, rng.uniform(-9, 9))
        b.add(uv_sphere(c, r, seg_u, seg_v), b.lambert(rng.uniform(0.2, 0.8, 3)))
    env = b.tex(f32_texture(np.ones((2, 2, 4), np.float32)))
    return b.finish(env, camera((0.0, 9.0, 20.0), (0.0, 0.0, 0.0), width, height))


def fbm(x, z, rng, octaves=6):
    """Seeded value-noise fBm in [-1, 1] (bilinear lattice noise, lacunarity 2, gain 0.5)."""
    total = np.zeros_like(x)
    amp, freq, norm = 1.0, 1.0, 0.0
    for _ in range(octaves):
        g = rng.uniform(-1, 1, (int(8 * freq) + 2, int(8 * freq) + 2))
        gx, gz = x * 8 * freq, z * 8 * freq
        ix, iz = np.floor(gx).astype(int), np.floor(gz).astype(int)
        fx, fz = gx - ix, gz - iz
        fx, fz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
        v = (g[ix, iz] * (1 - fx) * (1 - fz) + g[ix + 1, iz] * fx * (1 - fz) + g[ix, iz + 1] * (1 - fx) * fz +
             g[ix + 1, iz + 1] * fx * fz)
        total += amp * v
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def heightfield_scene(n=1024, width=1920, height=1080, env_w=2048, env_h=1024, seed=0, size=20.0,
                      amplitude=0.3) -> dict:
    """n x n quads; unshared vertices per quad so each quad's uv lands on its own atlas texel."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    Hh = amplitude * fbm(X, Z, rng)
    P = np.stack([(X - 0.5) * size, Hh, (Z - 0.5) * size], -1)
    # smooth normals from central differences
    dx = np.gradient(Hh, size / n, axis=0)
    dz = np.gradient(Hh, size / n, axis=1)
    N = np.stack([-dx, np.ones_like(dx), -dz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    Tg = np.stack([np.ones_like(dx), dx, np.zeros_like(dx)], -1)
    Tg /= np.linalg.norm(Tg, axis=-1, keepdims=True)
    Bt = np.cross(N, Tg)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.reshape(-1), j.reshape(-1)
    corners = [(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)]

    def gather(A):
        return np.stack([A[a, c] for a, c in corners], 1).reshape(-1, A.shape[-1]).astype(np.float32)

    verts, norms, tans, bits = gather(P), gather(N), gather(Tg), gather(Bt)
    # Atlas with a 2x2 block of identical texels per quad: the quad's corners map to texel
    # coordinates (2i, 2j) .. (2i+1, 2j+1) of a 2n x 2n texture (uv = texel / (2n - 1), the
    # bilinear convention of TextureContext.h:139-140), so every bilinear tap stays inside the
    # quad's block and the triangle's uv determinant is non-zero.  (Identical uvs on a triangle
    # would send the reference's hit record down its degenerate-uv branch, which flips the
    # geometric normal, embree.cpp:319-323.)
    k = 2 * n - 1
    cu = np.stack([2 * i, 2 * i + 1, 2 * i + 1, 2 * i], 1) / k
    cv = np.stack([2 * j, 2 * j, 2 * j + 1, 2 * j + 1], 1) / k
    uv = np.stack([cu, cv], -1).reshape(-1, 2).astype(np.float32)
    base = (np.arange(n * n) * 4).astype(np.uint32)
    idx = np.stack([np.stack([base, base + 2, base + 1], -1), np.stack([base, base + 3, base + 2], -1)], 1)
    idx = idx.reshape(-1, 3).astype(np.uint32)
    # per-quad materials
    is_metal = rng.uniform(size=n * n) < 0.5
    lam_alb = rng.uniform(0.1, 0.9, (n * n, 3))
    rough = rng.uniform(0.05, 0.8, n * n)
    f0 = rng.uniform(0.5, 1.0, (n * n, 3))
    albedo = np.where(is_metal[:, None], f0, lam_alb)
    alb_rgba = np.concatenate([np.round(albedo * 255), np.full((n * n, 1), 255)], 1).astype(np.uint8)
    met_rgba = np.zeros((n * n, 4), np.uint8)
    met_rgba[:, 1] = np.where(is_metal, np.round(rough * 255), 255).astype(np.uint8)
    met_rgba[:, 2] = np.where(is_metal, 255, 0).astype(np.uint8)
    met_rgba[:, 3] = 255
    # atlas row = v index (j), column = u index (i); each quad owns a 2x2 texel block
    alb_img = np.repeat(np.repeat(alb_rgba.reshape(n, n, 4).transpose(1, 0, 2), 2, 0), 2, 1)
    met_img = np.repeat(np.repeat(met_rgba.reshape(n, n, 4).transpose(1, 0, 2), 2, 0), 2, 1)
    b = _Builder()
    mat = b.material(b.tex(u8_texture(alb_img)), b.tex(u8_texture(met_img)))
    b.add({"vertices": verts, "normals": norms, "tangents": tans, "bitangents": bits, "uv": uv, "indices": idx}, mat)
    env = rng.lognormal(0.0, 1.5, (env_h, env_w, 3)).astype(np.float32)
    env = np.concatenate([env, np.ones((env_h, env_w, 1), np.float32)], -1)
    e = b.tex(f32_texture(env))
    return b.finish(e, camera((0.0, 7.0, 13.0), (0.0, 0.0, -1.0), width, height))


def mixed_scene(target_tris=50000, width=256, height=256, seed=0, env_w=256, env_h=128) -> dict:
    """Random spheres and boxes on a tessellated 40 x 40 ground until `target_tris` triangles;
    materials 1/3 Lambert, 1/3 GGX conductor, 1/3 GGX dielectric IOR 1.5.  The ground is cut into
    32 x 32 quads: two ground triangles spanning the whole scene would sit in almost every node of a
    BVH built with node-box split candidates (aggregate/native/BvhBuilder.cpp:151-184) and leave
    leaves of thousands of triangles there."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    g = grid_quad(40.0, 32)
    b.add(g, b.lambert((0.6, 0.6, 0.6)))
    tris = len(g["indices"])
    while tris < target_tris:
        kind = rng.integers(3)
        if kind == 0:
            mat = b.lambert(rng.uniform(0.1, 0.9, 3))
        elif kind == 1:
            mat = b.conductor(rng.uniform(0.5, 1.0, 3), rng.uniform(0.05, 0.8))
        else:
            mat = b.dielectric(rng.uniform(0.05, 0.5))
        c = np.array([rng.uniform(-15, 15), rng.uniform(0.5, 3.0), rng.uniform(-15, 15)])
        if rng.uniform() < 0.7:
            su = int(rng.choice([16, 32, 64, 128]))
            mesh = uv_sphere(c, rng.uniform(0.3, 1.5), su, su // 2)
        else:
            mesh = box(c, rng.uniform(0.2, 1.2, 3), random_rotation(rng))
        b.add(mesh, mat)
        tris += len(mesh["indices"])
    env = rng.lognormal(0.0, 1.0, (env_h, env_w, 3)).astype(np.float32)
    env = np.concatenate([env, np.ones((env_h, env_w, 1), np.float32)], -1)
    e = b.tex(f32_texture(env))
    return b.finish(e, camera((0.0, 12.0, 30.0), (0.0, 0.0, 0.0), width, height))


def blob_mesh(n_tris, rng):
    """A seeded closed 'blob' (perturbed UV sphere) with about n_tris triangles, unit radius."""
    su = max(8, int(round(math.sqrt(n_tris))))
    sv = max(4, n_tris // (2 * su))
    m = uv_sphere((0.0, 0.0, 0.0), 1.0, su, sv)
    k = rng.uniform(0.1, 0.3, 3)
    ph = rng.uniform(0, 2 * np.pi, 3)
    p = m["vertices"].astype(np.float64)
    r = 1.0 + k[0] * np.sin(3 * p[:, 0] + ph[0]) * np.sin(2 * p[:, 1] + ph[1]) + k[1] * np.cos(4 * p[:, 2] + ph[2])
    m["vertices"] = (p * r[:, None]).astype(np.float32)
    return m


def instanced_scene(n_meshes=10, n_instances=1000, tris_per_mesh=10000, width=3840, height=2160, seed=0,
                    box_size=100.0, env_w=4096, env_h=2048) -> dict:
    rng = np.random.default_rng(seed)
    b = _Builder()
    protos = [blob_mesh(tris_per_mesh, rng) for _ in range(n_meshes)]
    for p in protos:
        b.meshes.append(p)
    mats = []
    for k in range(8):
        kind = k % 4
        if kind == 0:
            mats.append(b.lambert(rng.uniform(0.1, 0.9, 3)))
        elif kind == 1:
            mats.append(b.conductor(rng.uniform(0.5, 1.0, 3), rng.uniform(0.05, 0.8)))
        elif kind == 2:
            mats.append(b.dielectric(rng.uniform(0.05, 0.5)))
        else:
            mats.append(b.burley(rng.uniform(0.1, 0.9, 3), rng.uniform(0.2, 1.0)))
    for _ in range(n_instances):
        M = np.eye(4)
        M[:3, :3] = random_rotation(rng) * rng.uniform(0.5, 3.0)
        M[:3, 3] = rng.uniform(-box_size / 2, box_size / 2, 3)
        b.place(int(rng.integers(n_meshes)), int(rng.choice(mats)), M)
    env = rng.lognormal(0.0, 1.0, (env_h, env_w, 3)).astype(np.float32)
    env = np.concatenate([env, np.ones((env_h, env_w, 1), np.float32)], -1)
    e = b.tex(f32_texture(env))
    return b.finish(e, camera((0.0, 0.0, box_size * 1.2), (0.0, 0.0, 0.0), width, height))


def batch_jobs(n_jobs=32, seed=0, tris=(50000, 500000), res=(256, 2048), spp_choices=(1, 4, 16, 64),
               depth_choices=(3, 6, 12)):
    """The batched workload: `n_jobs` seeded jobs, each a mixed spheres + boxes scene of
    U[tris] triangles (1/3 Lambert, 1/3 GGX conductor, 1/3 GGX dielectric IOR 1.5), a square
    frame whose pixel count is log-uniform in [res[0]^2, res[1]^2], spp drawn from `spp_choices`
    and max depth from `depth_choices`.  Returns a list of dicts
    {scene, width, height, spp, depth, seed}."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        n_tris = int(rng.integers(tris[0], tris[1] + 1))
        side = int(round(math.exp(rng.uniform(math.log(res[0]), math.log(res[1])))))
        spp = int(rng.choice(spp_choices))
        depth = int(rng.choice(depth_choices))
        scene = mixed_scene(n_tris, side, side, seed=seed * 1000 + j + 1)
        jobs.append({"scene": scene, "width": side, "height": side, "spp": spp, "depth": depth, "seed": j})
    return jobs


def scene_stats(scene: dict) -> dict:
    tris = sum(len(scene["meshes"][x["mesh"]]["indices"]) for x in scene["instances"])
    return {"instances": len(scene["instances"]), "meshes": len(scene["meshes"]), "triangles": tris}
