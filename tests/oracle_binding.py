"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure: the oracle is the parity checker for the CUDA path and the timed CPU
baseline.  Only tests/, the smoke check and bench.py's CPU-baseline leg load it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


class OrcMesh(C.Structure):
    _fields_ = [("vertices", f32p), ("normals", f32p), ("tangents", f32p), ("bitangents", f32p), ("uv", f32p),
                ("indices", u32p), ("n_verts", C.c_uint32), ("n_tris", C.c_uint32)]


class OrcInstance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("material", C.c_uint32), ("m", C.c_float * 16), ("inv", C.c_float * 16),
                ("n", C.c_float * 9)]


class OrcMaterial(C.Structure):
    _fields_ = [("albedo", C.c_int32), ("metallic", C.c_int32), ("normalmap", C.c_int32), ("emissive", C.c_int32),
                ("eta", C.c_float * 3), ("k", C.c_float * 3), ("anisotropy", C.c_float)]


class OrcTexture(C.Structure):
    _fields_ = [("u8_pixels", u32p), ("f32_pixels", f32p), ("width", C.c_int32), ("height", C.c_int32),
                ("channels", C.c_int32), ("is_rgba", C.c_int32), ("invert_u", C.c_int32), ("invert_v", C.c_int32)]


class OrcScene(C.Structure):
    _fields_ = [("meshes", C.POINTER(OrcMesh)), ("n_meshes", C.c_uint32),
                ("instances", C.POINTER(OrcInstance)), ("n_instances", C.c_uint32),
                ("materials", C.POINTER(OrcMaterial)), ("n_materials", C.c_uint32),
                ("textures", C.POINTER(OrcTexture)), ("n_textures", C.c_uint32),
                ("envmap", C.c_int32), ("inv_P", C.c_float * 16), ("inv_V", C.c_float * 16)]


class OrcOptions(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("seed", C.c_uint32), ("index_mode", C.c_int32), ("rr_start", C.c_int32), ("threads", C.c_int32),
                ("tile", C.c_int32), ("vertical_invert", C.c_int32)]


class OrcStats(C.Structure):
    _fields_ = [("segments", C.c_uint64), ("traced", C.c_uint64), ("node_visits", C.c_uint64),
                ("tri_tests", C.c_uint64), ("seconds", C.c_double)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_sobol_table.argtypes = [u32p]
        L.orc_sobol_samples.argtypes = [u32p, u32p, C.c_uint64, C.c_uint32, f32p]
        L.orc_acos_lut.argtypes = [f32p, C.c_int32]
        L.orc_build.argtypes = [C.POINTER(OrcScene)]
        L.orc_build.restype = C.c_void_p
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_bvh_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_sample_path.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_int32, C.c_int32, C.c_int32, f32p,
                                      C.c_int32, f32p]
        L.orc_sample_path.restype = C.c_int32
        L.orc_render_aov.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_int32, C.c_float, C.c_float, f32p]
        L.orc_render_aov.restype = C.c_int32
        L.orc_set_diff_params.argtypes = [C.c_void_p, f32p, f32p]
        L.orc_set_diff_params.restype = C.c_int32
        L.orc_set_perturbation.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_int32, C.c_float]
        L.orc_set_perturbation.restype = C.c_int32
        L.orc_backward.argtypes = [C.c_void_p, C.POINTER(OrcOptions), f32p, f32p, f32p, C.c_int32]
        L.orc_backward.restype = C.c_int32
        L.orc_backward_range.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_int32, C.c_int32, f32p, f32p, f32p,
                                         C.c_int32]
        L.orc_backward_range.restype = C.c_int32
        L.orc_scatter.argtypes = [C.c_void_p, C.c_uint64, f32p, f32p, i32p, f32p, f32p, f32p, u32p, i32p, C.c_uint32,
                                  f32p, f32p, f32p, f32p, i32p]
        L.orc_trace.argtypes = [C.c_void_p, C.c_uint64, f32p, f32p, i32p, f32p, f32p, f32p, C.POINTER(OrcStats)]
        L.orc_camera_rays.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_uint64, i32p, i32p, i32p, f32p, f32p]
        L.orc_render.argtypes = [C.c_void_p, C.POINTER(OrcOptions), f32p, i32p, C.c_int64, C.POINTER(OrcStats)]
        L.orc_render.restype = C.c_int32
        L.orc_sample_radiance.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_uint64, i32p, i32p, i32p, f32p]
        L.orc_bake_irradiance.argtypes = [f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, f32p]
        L.orc_bake_irradiance.restype = C.c_int32
        L.orc_env_sample.argtypes = [f32p, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, f32p, f32p]
        L.orc_fresnel_real.argtypes = [C.c_float, C.c_float, f32p]
        L.orc_fresnel_real.restype = C.c_float
        L.orc_vndf_sample.argtypes = [C.c_float, C.c_float, f32p, f32p, f32p]
        L.orc_vndf_g1.argtypes = [C.c_float, C.c_float, f32p]
        L.orc_vndf_g1.restype = C.c_float
        L.orc_correct_specular_normal.argtypes = [f32p, f32p, f32p, f32p]
        L.orc_cartesian_to_spherical.argtypes = [C.c_uint64, f32p, f32p]
        L.orc_prim_bounds.argtypes = [C.c_void_p, f32p, f32p]
        L.orc_atan2_approx.argtypes = [C.c_uint64, f32p, f32p, f32p]
        L.orc_rgb_to_unit.argtypes = [C.c_uint64, f32p, f32p]
        L.orc_uv_to_pixel.argtypes = [C.c_uint64, f32p, u32p, u32p]
        L.orc_texture_lookup.argtypes = [C.POINTER(OrcTexture), C.c_float, C.c_float, f32p]
        L.orc_box_intersect.argtypes = [f32p, f32p, f32p, f32p, C.c_float]
        L.orc_box_intersect.restype = C.c_float
        L.orc_dielectric_lobe.argtypes = [f32p, C.c_float, C.c_float, C.c_float, f32p, C.c_float, f32p, f32p]
        L.orc_dielectric_lobe.restype = C.c_int32
        L.orc_tile_split.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p]
        L.orc_tile_split.restype = C.c_int32
        u8p = C.POINTER(C.c_uint8)
        L.orc_film_accumulate.argtypes = [f32p, f32p, f32p, C.c_uint64, C.c_uint32]
        L.orc_display_blend.argtypes = [f32p, f32p, f32p, C.c_uint64, C.c_uint32]
        L.orc_snapshot.argtypes = [f32p, C.c_int32, C.c_int32, C.c_int32, f32p, C.c_int32, C.c_int32]
        L.orc_rgbe_encode.argtypes = [f32p, C.c_uint64, C.c_int32, u8p]
        L.orc_rgbe_decode.argtypes = [u8p, C.c_uint64, f32p]
        L.orc_hdr_parse.argtypes = [u8p, C.c_uint64, i32p, i32p, u8p]
        L.orc_hdr_parse.restype = C.c_int32
        L.orc_hdr_write.argtypes = [C.c_char_p, f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.orc_hdr_write.restype = C.c_int32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def sobol_table() -> np.ndarray:
    out = np.zeros((256, 32), np.uint32)
    lib().orc_sobol_table(_p(out, u32p))
    return out


def sobol_samples(index, dim, seed: int) -> np.ndarray:
    index = np.ascontiguousarray(index, np.uint32)
    dim = np.ascontiguousarray(dim, np.uint32)
    out = np.zeros(index.shape, np.float32)
    lib().orc_sobol_samples(_p(index, u32p), _p(dim, u32p), index.size, seed, _p(out, f32p))
    return out


def acos_lut(precision: int = 500000) -> np.ndarray:
    out = np.zeros(precision, np.float32)
    lib().orc_acos_lut(_p(out, f32p), precision)
    return out


def options(width, height, spp, max_depth, seed=0, index_mode=0, rr_start=-1, threads=0, tile=20, vertical_invert=0):
    return OrcOptions(width, height, spp, max_depth, seed, index_mode, rr_start, threads, tile, vertical_invert)


def material_table(scene: dict):
    """The scene's materials as an orc_material array."""
    mats = (OrcMaterial * len(scene["materials"]))()
    for i, m in enumerate(scene["materials"]):
        mats[i] = OrcMaterial(m.get("albedo", -1), m.get("metallic", -1), m.get("normalmap", -1),
                              m.get("emissive", -1), (C.c_float * 3)(*m.get("eta", (0, 0, 0))),
                              (C.c_float * 3)(*m.get("k", (0, 0, 0))), m.get("anisotropy", 0.0))
    return mats


def texture_table(scene: dict):
    """The scene's textures as an orc_texture array, and the pixel arrays it points into."""
    texs = (OrcTexture * len(scene["textures"]))()
    keep = []
    for i, t in enumerate(scene["textures"]):
        if t["format"] == "u8":
            px = np.ascontiguousarray(t["pixels"], np.uint32)
            texs[i] = OrcTexture(_p(px, u32p), None, t["width"], t["height"], t.get("channels", 4),
                                 int(t.get("is_rgba", 1)), int(t.get("invert_u", 0)), int(t.get("invert_v", 0)))
        else:
            px = np.ascontiguousarray(t["pixels"], np.float32)
            texs[i] = OrcTexture(None, _p(px, f32p), t["width"], t["height"], t.get("channels", 4),
                                 int(t.get("is_rgba", 1)), int(t.get("invert_u", 0)), int(t.get("invert_v", 0)))
        keep.append(px)
    return texs, keep


class OracleScene:
    """Builds the oracle's scene + reference binary SAH BVH from a scene dictionary
    (see axomae_b200.scenes for the layout)."""

    def __init__(self, scene: dict):
        self._keep = []
        meshes = (OrcMesh * len(scene["meshes"]))()
        for i, m in enumerate(scene["meshes"]):
            arrs = [np.ascontiguousarray(m[k], np.float32) for k in ("vertices", "normals", "tangents", "bitangents",
                                                                      "uv")]
            idx = np.ascontiguousarray(m["indices"], np.uint32)
            self._keep += arrs + [idx]
            meshes[i] = OrcMesh(*[_p(a, f32p) for a in arrs], _p(idx, u32p), arrs[0].size // 3, idx.size // 3)
        insts = (OrcInstance * len(scene["instances"]))()
        for i, x in enumerate(scene["instances"]):
            m = np.asarray(x["m"], np.float32).reshape(16)
            inv = np.asarray(x["inv"], np.float32).reshape(16)
            n = np.asarray(x["n"], np.float32).reshape(9)
            insts[i] = OrcInstance(x["mesh"], x["material"], (C.c_float * 16)(*m), (C.c_float * 16)(*inv),
                                   (C.c_float * 9)(*n))
        mats, texs, keep = material_table(scene), *texture_table(scene)
        self._keep += keep
        sc = OrcScene(meshes, len(scene["meshes"]), insts, len(scene["instances"]), mats, len(scene["materials"]),
                      texs, len(scene["textures"]), scene["envmap"],
                      (C.c_float * 16)(*np.asarray(scene["inv_P"], np.float32).reshape(16)),
                      (C.c_float * 16)(*np.asarray(scene["inv_V"], np.float32).reshape(16)))
        self._keep += [meshes, insts, mats, texs, sc]
        self.n_tris = sum(meshes[x["mesh"]].n_tris for x in scene["instances"])
        self.n_materials = len(scene["materials"])
        self.h = lib().orc_build(C.byref(sc))
        if not self.h:
            raise ValueError("oracle rejected the scene")
        self._keep = []  # the oracle copied everything it needs

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def bvh_info(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        lib().orc_bvh_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def prim_bounds(self):
        """(boxes (n, 6) as min then max, centroids (n, 3)) of every triangle, world space, instance
        by instance and triangle by triangle."""
        boxes = np.zeros((self.n_tris, 6), np.float32)
        cents = np.zeros((self.n_tris, 3), np.float32)
        lib().orc_prim_bounds(self.h, _p(boxes, f32p), _p(cents, f32p))
        return boxes, cents

    def trace(self, orig, dirs):
        orig = np.ascontiguousarray(orig, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = orig.shape[0]
        prim = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n, np.float32) for _ in range(3))
        st = OrcStats()
        lib().orc_trace(self.h, n, _p(orig, f32p), _p(dirs, f32p), _p(prim, i32p), _p(t, f32p), _p(u, f32p),
                        _p(v, f32p), C.byref(st))
        return prim, t, u, v, st

    def camera_rays(self, opt, px, py, ps):
        px, py, ps = (np.ascontiguousarray(a, np.int32) for a in (px, py, ps))
        n = px.size
        o = np.zeros((n, 3), np.float32)
        d = np.zeros((n, 3), np.float32)
        lib().orc_camera_rays(self.h, C.byref(opt), n, _p(px, i32p), _p(py, i32p), _p(ps, i32p), _p(o, f32p),
                              _p(d, f32p))
        return o, d

    def render(self, opt, pixel_ids=None):
        out = np.full((opt.height, opt.width, 4), 0.0, np.float32)  # touched here, not in the timed loop
        st = OrcStats()
        if pixel_ids is None:
            rc = lib().orc_render(self.h, C.byref(opt), _p(out, f32p), None, 0, C.byref(st))
        else:
            ids = np.ascontiguousarray(pixel_ids, np.int32)
            rc = lib().orc_render(self.h, C.byref(opt), _p(out, f32p), _p(ids, i32p), ids.size, C.byref(st))
        if rc != 0:
            raise ValueError("oracle render failed: %d" % rc)
        return out, st

    def sample_path(self, opt, x, y, s, max_segments=64):
        """Segments of one path: (n, 10) float32 rows of origin, direction, hit primitive (int32
        bits), t, u, v; and the path's radiance."""
        out = np.zeros((max_segments, 10), np.float32)
        rad = np.zeros(3, np.float32)
        n = lib().orc_sample_path(self.h, C.byref(opt), x, y, s, _p(out, f32p), max_segments, _p(rad, f32p))
        return out[:n], rad

    def scatter(self, o, d, prim, t, u, v, index, bounce, seed=0):
        """One shading event per hit (orc_scatter): next origin, next direction, weight, emission
        (each (n, 3)) and valid (n,)."""
        n = len(prim)
        f3 = lambda a: np.ascontiguousarray(a, np.float32).reshape(n, 3)
        o, d = f3(o), f3(d)
        prim = np.ascontiguousarray(prim, np.int32)
        t, u, v = (np.ascontiguousarray(a, np.float32) for a in (t, u, v))
        index = np.ascontiguousarray(index, np.uint32)
        bounce = np.ascontiguousarray(bounce, np.int32)
        outs = [np.zeros((n, 3), np.float32) for _ in range(4)]
        valid = np.zeros(n, np.int32)
        lib().orc_scatter(self.h, n, _p(o, f32p), _p(d, f32p), _p(prim, i32p), _p(t, f32p), _p(u, f32p), _p(v, f32p),
                          _p(index, u32p), _p(bounce, i32p), seed, *[_p(a, f32p) for a in outs], _p(valid, i32p))
        return (*outs, valid)

    def render_aov(self, opt, kind, near_plane=0.1, far_plane=1000.0):
        """AOV integrator image (kind 1 normal, 2 depth, 4 emissive), (H, W, 4)."""
        out = np.zeros((opt.height, opt.width, 4), np.float32)
        if lib().orc_render_aov(self.h, C.byref(opt), kind, near_plane, far_plane, _p(out, f32p)) != 0:
            raise ValueError("bad AOV request")
        return out

    def set_diff_params(self, albedo=None, roughness=None):
        """Per-triangle RGB albedo ((n_tris, 3)) / per-material roughness; None = textures."""
        self._alb = None if albedo is None else np.ascontiguousarray(albedo, np.float32).reshape(-1)
        self._rough = None if roughness is None else np.ascontiguousarray(roughness, np.float32)
        lib().orc_set_diff_params(self.h, None if self._alb is None else _p(self._alb, f32p),
                                  None if self._rough is None else _p(self._rough, f32p))

    def set_perturbation(self, kind=0, index=0, channel=0, delta=0.0):
        """Detached perturbation: 1 = albedo of triangle `index` (channel), 2 = roughness of
        material `index`; f is evaluated with the moved parameter, sampling is unperturbed."""
        if lib().orc_set_perturbation(self.h, kind, index, channel, delta) != 0:
            raise ValueError("bad perturbation")

    def _check_sizes(self, opt, d_image, n_tris, n_materials):
        """The C side writes 3 * (scene triangles) and (scene materials) gradients and reads W * H * 4
        image adjoints: refuse buffers of other sizes."""
        if n_tris != self.n_tris or n_materials != self.n_materials:
            raise ValueError("gradient sizes %d / %d do not match the scene's %d triangles / %d materials"
                             % (n_tris, n_materials, self.n_tris, self.n_materials))
        if np.size(d_image) != opt.width * opt.height * 4:
            raise ValueError("d_image must hold width * height * 4 floats")

    def backward(self, opt, d_image, n_tris, n_materials, threads=0):
        """Replay adjoint on the CPU: (grad_albedo (n_tris, 3), grad_roughness (n_materials,))."""
        self._check_sizes(opt, d_image, n_tris, n_materials)
        d_image = np.ascontiguousarray(d_image, np.float32)
        ga = np.zeros(3 * n_tris, np.float32)
        gr = np.zeros(n_materials, np.float32)
        rc = lib().orc_backward(self.h, C.byref(opt), _p(d_image, f32p), _p(ga, f32p), _p(gr, f32p), threads)
        if rc != 0:
            raise ValueError("oracle backward failed")
        return ga.reshape(n_tris, 3), gr

    def backward_range(self, opt, sample_begin, sample_count, d_image, n_tris, n_materials, threads=0):
        """Replay adjoint of the mean over samples [sample_begin, sample_begin + sample_count)."""
        self._check_sizes(opt, d_image, n_tris, n_materials)
        d_image = np.ascontiguousarray(d_image, np.float32)
        ga = np.zeros(3 * n_tris, np.float32)
        gr = np.zeros(n_materials, np.float32)
        rc = lib().orc_backward_range(self.h, C.byref(opt), sample_begin, sample_count, _p(d_image, f32p),
                                      _p(ga, f32p), _p(gr, f32p), threads)
        if rc != 0:
            raise ValueError("oracle backward failed")
        return ga.reshape(n_tris, 3), gr

    def sample_radiance(self, opt, px, py, ps):
        px, py, ps = (np.ascontiguousarray(a, np.int32) for a in (px, py, ps))
        out = np.zeros((px.size, 3), np.float32)
        lib().orc_sample_radiance(self.h, C.byref(opt), px.size, _p(px, i32p), _p(py, i32p), _p(ps, i32p),
                                  _p(out, f32p))
        return out


def bake_irradiance(src: np.ndarray, out_w: int, out_h: int, samples: int, threads: int = 8) -> np.ndarray:
    src = np.ascontiguousarray(src, np.float32)
    h, w, ch = src.shape
    out = np.zeros((out_h, out_w, ch), np.float32)
    rc = lib().orc_bake_irradiance(_p(src, f32p), w, h, ch, out_w, out_h, samples, threads, _p(out, f32p))
    if rc != 0:
        raise ValueError("bake rejected")
    return out


def bake_irradiance_texunit(src: np.ndarray, out_w: int, out_h: int, samples: int, threads: int = 8) -> np.ndarray:
    """The reference's CUDA bake (CubemapProcessing.cu:129-175) restated, texture filter included:
    (out_h, out_w, 4), alpha 1.  The source is made RGBA with alpha 1 first, as the reference does."""
    src = np.asarray(src, np.float32)
    h, w, ch = src.shape
    rgba = np.ones((h, w, 4), np.float32)
    rgba[..., :3] = src[..., :3]
    out = np.zeros((out_h, out_w, 4), np.float32)
    L = lib()
    L.orc_bake_irradiance_texunit.argtypes = [f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                              f32p]
    L.orc_bake_irradiance_texunit.restype = C.c_int32
    if L.orc_bake_irradiance_texunit(_p(rgba, f32p), w, h, out_w, out_h, samples, threads, _p(out, f32p)) != 0:
        raise ValueError("bake rejected")
    return out


def _v(x, n):
    return np.ascontiguousarray(x, np.float32).reshape(n)


def fresnel_real(ior, cos_i):
    """Fresnel::real: (reflectance, the eta used) for the cosine of incidence."""
    e = np.zeros(1, np.float32)
    r = lib().orc_fresnel_real(ior, cos_i, _p(e, f32p))
    return float(r), float(e[0])


def vndf_sample(roughness, wo, uc, anisotropy=0.0):
    wo, uc, wm = _v(wo, 3), _v(uc, 2), np.zeros(3, np.float32)
    lib().orc_vndf_sample(anisotropy, roughness, _p(wo, f32p), _p(uc, f32p), _p(wm, f32p))
    return wm


def vndf_g1(roughness, v, anisotropy=0.0):
    v = _v(v, 3)
    return float(lib().orc_vndf_g1(anisotropy, roughness, _p(v, f32p)))


def correct_specular_normal(ng, wo, ns):
    ng, wo, ns, out = _v(ng, 3), _v(wo, 3), _v(ns, 3), np.zeros(3, np.float32)
    lib().orc_correct_specular_normal(_p(ng, f32p), _p(wo, f32p), _p(ns, f32p), _p(out, f32p))
    return out


def env_sample(pixels, dirs):
    """EnvmapTexture::sample of a float texture (H, W, C) for directions (n, 3): (n, 4)."""
    px = np.ascontiguousarray(pixels, np.float32)
    h, w, ch = px.shape
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    out = np.zeros((d.shape[0], 4), np.float32)
    lib().orc_env_sample(_p(px, f32p), w, h, ch, d.shape[0], _p(d, f32p), _p(out, f32p))
    return out


def texture_lookup(tex, u, v):
    """One lookup of a texture dictionary (scenes layout) at (u, v): RGBA float."""
    if tex["format"] == "u8":
        px = np.ascontiguousarray(tex["pixels"], np.uint32)
        t = OrcTexture(_p(px, u32p), None, tex["width"], tex["height"], tex.get("channels", 4),
                       int(tex.get("is_rgba", 1)), int(tex.get("invert_u", 0)), int(tex.get("invert_v", 0)))
    else:
        px = np.ascontiguousarray(tex["pixels"], np.float32)
        t = OrcTexture(None, _p(px, f32p), tex["width"], tex["height"], tex.get("channels", 4),
                       int(tex.get("is_rgba", 1)), int(tex.get("invert_u", 0)), int(tex.get("invert_v", 0)))
    out = np.zeros(4, np.float32)
    lib().orc_texture_lookup(C.byref(t), u, v, _p(out, f32p))
    return out


MAXFLOAT = float(np.finfo(np.float32).max)


def box_intersect(mn, mx, o, d, dist_min):
    """The traversal's slab test: entry distance of the ray into [mn, mx], MAXFLOAT for a miss."""
    a = [np.ascontiguousarray(x, np.float32).reshape(3) for x in (mn, mx, o, d)]
    return lib().orc_box_intersect(*[_p(x, f32p) for x in a], dist_min)


def dielectric_lobe(albedo, eta, roughness, anisotropy, wo, uc, u):
    """The dielectric lobe alone: (sampled, dict of f, pdf, wi, costheta, f_eval, pdf_eval)."""
    alb = np.ascontiguousarray(albedo, np.float32).reshape(3)
    w = np.ascontiguousarray(wo, np.float32).reshape(3)
    uu = np.ascontiguousarray(u, np.float32).reshape(2)
    out = np.zeros(12, np.float32)
    ok = lib().orc_dielectric_lobe(_p(alb, f32p), eta, roughness, anisotropy, _p(w, f32p), uc, _p(uu, f32p),
                                   _p(out, f32p))
    return bool(ok), {"f": out[0:3], "pdf": float(out[3]), "wi": out[4:7], "costheta": float(out[7]),
                      "f_eval": out[8:11], "pdf_eval": float(out[11])}


def cartesian_to_spherical(xyz):
    """(phi, theta) of unit directions (n, 3) with the reference's fast approximations."""
    d = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    out = np.zeros((d.shape[0], 2), np.float32)
    lib().orc_cartesian_to_spherical(d.shape[0], _p(d, f32p), _p(out, f32p))
    return out


def tile_split(width, height, tiles_w, tiles_h):
    """The frame's split into tiles_w x tiles_h tiles: (n, 4) rows of (x0, x1, y0, y1)."""
    rects = np.zeros((max(tiles_w, 0) * max(tiles_h, 0), 4), np.int32)
    n = lib().orc_tile_split(width, height, tiles_w, tiles_h, _p(rects, i32p))
    if n == 0 and rects.size:
        raise ValueError("bad tile split %dx%d of %dx%d" % (tiles_w, tiles_h, width, height))
    return rects[:n]


# ---- film outputs and the Radiance .hdr format (oracle/film_io.cpp) ----

def film_accumulate(partial, accum, frame_index):
    """Returns (accum + partial, its mean over frame_index + 1 frames); inputs unchanged."""
    partial = np.ascontiguousarray(partial, np.float32).reshape(-1)
    acc = np.array(accum, np.float32).reshape(-1)
    final = np.zeros_like(acc)
    lib().orc_film_accumulate(_p(partial, f32p), _p(acc, f32p), _p(final, f32p), acc.size, frame_index)
    return acc, final


def display_blend(partial, accum, current_frame):
    partial = np.ascontiguousarray(partial, np.float32).reshape(-1)
    accum = np.ascontiguousarray(accum, np.float32).reshape(-1)
    out = np.zeros_like(accum)
    lib().orc_display_blend(_p(partial, f32p), _p(accum, f32p), _p(out, f32p), out.size, current_frame)
    return out


def snapshot(film, dst_w, dst_h, dst_init=None):
    """film: (H, W, C) floats; returns (dst_h, dst_w, C) with channel 3 left as dst_init's (zeros)."""
    film = np.ascontiguousarray(film, np.float32)
    h, w, ch = film.shape
    out = np.zeros((dst_h, dst_w, ch), np.float32) if dst_init is None else np.array(dst_init, np.float32)
    lib().orc_snapshot(_p(film, f32p), w, h, ch, _p(out, f32p), dst_w, dst_h)
    return out


def rgbe_encode(pixels, channels):
    px = np.ascontiguousarray(pixels, np.float32).reshape(-1)
    n = px.size // channels
    out = np.zeros((n, 4), np.uint8)
    lib().orc_rgbe_encode(_p(px, f32p), n, channels, _p(out, C.POINTER(C.c_uint8)))
    return out


def rgbe_decode(rgbe):
    q = np.ascontiguousarray(rgbe, np.uint8).reshape(-1, 4)
    out = np.zeros((q.shape[0], 4), np.float32)
    lib().orc_rgbe_decode(_p(q, C.POINTER(C.c_uint8)), q.shape[0], _p(out, f32p))
    return out


def hdr_parse(data: bytes):
    """(code, width, height, rgbe (H, W, 4) uint8 or None): code 0 on success."""
    buf = np.frombuffer(data, np.uint8).copy() if len(data) else np.zeros(1, np.uint8)
    w, h = C.c_int32(0), C.c_int32(0)
    u8p = C.POINTER(C.c_uint8)
    code = lib().orc_hdr_parse(_p(buf, u8p), len(data), C.byref(w), C.byref(h), None)
    if code:
        return code, 0, 0, None
    rgbe = np.zeros((h.value, w.value, 4), np.uint8)
    code = lib().orc_hdr_parse(_p(buf, u8p), len(data), C.byref(w), C.byref(h), _p(rgbe, u8p))
    return code, w.value, h.value, (rgbe if code == 0 else None)


def hdr_write(path, pixels, width, height, channels, flip=0):
    """Writes path + ".hdr" the way IO::Loader::writeHdr does."""
    px = np.ascontiguousarray(pixels, np.float32).reshape(-1)
    if lib().orc_hdr_write(os.fsencode(path), _p(px, f32p), width, height, channels, flip) != 0:
        raise OSError("cannot write %s.hdr" % path)


def hdr_body(data: bytes) -> bytes:
    """The scanline bytes of a .hdr file (after the resolution line)."""
    head_end = data.index(b"\n\n") + 2
    return data[data.index(b"\n", head_end) + 1:]
