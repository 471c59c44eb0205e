"""ctypes binding of the C ABI in include/nova_b200.h (libnova_b200.so, built in-tree).

The library is the product: a Python caller (tests, bench.py, the smoke check) talks to it only
through the C entry points, exactly as a C++ Nova render call would.  There is no CPU fallback:
importing this module on a machine without the built library, or creating a context without a
GPU, raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnova_b200.so")

f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)

STATUS = ["SUCCESS", "INVALID_ENGINE_STATE", "INVALID_BUFFER_STATE", "INVALID_CHANNEL_DESCRIPTOR", "INVALID_SCENE_TYPE",
          "INVALID_TRANSFORM_TYPE", "RENDER_BUFFER_NOT_INITIALIZED", "RENDER_OPTIONS_NOT_INITIALIZED",
          "RENDER_ENGINE_NOT_INITIALIZED", "SCENE_NOT_PROCESSED", "NOT_GPU_BUILD", "OUT_OF_MEMORY",
          "MULTIPLE_INTEGRATORS_NOT_SUPPORTED", "THREADPOOL_CREATION_ERROR", "THREADPOOL_NOT_INITIALIZED",
          "INVALID_ARGUMENT", "RENDERER_EXCEPTION"]


class NovaError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        name = STATUS[status] if 0 <= status < len(STATUS) else str(status)
        super().__init__("%s: %s" % (name, message))


class Mesh(C.Structure):
    _fields_ = [("vertices", f32p), ("normals", f32p), ("tangents", f32p), ("bitangents", f32p), ("uv", f32p),
                ("indices", u32p), ("n_verts", C.c_uint32), ("n_tris", C.c_uint32)]


class Instance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("material", C.c_uint32), ("m", C.c_float * 16), ("inv", C.c_float * 16),
                ("n", C.c_float * 9)]


class Material(C.Structure):
    _fields_ = [("albedo", C.c_int32), ("metallic", C.c_int32), ("normalmap", C.c_int32), ("emissive", C.c_int32),
                ("eta", C.c_float * 3), ("k", C.c_float * 3), ("anisotropy", C.c_float)]


class Texture(C.Structure):
    _fields_ = [("u8_pixels", u32p), ("f32_pixels", f32p), ("width", C.c_int32), ("height", C.c_int32),
                ("channels", C.c_int32), ("is_rgba", C.c_int32), ("invert_u", C.c_int32), ("invert_v", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(Mesh)), ("n_meshes", C.c_uint32), ("instances", C.POINTER(Instance)),
                ("n_instances", C.c_uint32), ("materials", C.POINTER(Material)), ("n_materials", C.c_uint32),
                ("textures", C.POINTER(Texture)), ("n_textures", C.c_uint32), ("envmap", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("queue_capacity", C.c_uint32), ("trace_block", C.c_uint32), ("shade_block", C.c_uint32),
                ("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("bvh_width", C.c_int32),
                ("trace_mode", C.c_uint32), ("wait_limit_us", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


TUNE_BVH_WIDTH = 1
AOV_NORMAL, AOV_DEPTH, AOV_EMISSIVE = 1, 2, 4
BACKWARD_REUSE_PRIMAL = 1


class BvhOptions(C.Structure):
    _fields_ = [("max_leaf_size", C.c_int32), ("bins", C.c_int32), ("width", C.c_int32),
                ("small_subtree", C.c_int32)]


class Frame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp_total", C.c_int32), ("sample_begin", C.c_int32),
                ("sample_count", C.c_int32), ("max_depth", C.c_int32), ("seed", C.c_uint32), ("rr_start", C.c_int32),
                ("reset", C.c_int32), ("vertical_invert", C.c_int32), ("inv_P", C.c_float * 16),
                ("inv_V", C.c_float * 16)]


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("segments", C.c_uint64), ("traced", C.c_uint64), ("waves", C.c_uint64),
                ("device_ms", C.c_double), ("trace_ms", C.c_double), ("shade_ms", C.c_double),
                ("kernels", C.c_uint64), ("nonfinite", C.c_uint64), ("bad_index", C.c_uint64),
                ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

EXPORTS = ["nova_b200_create", "nova_b200_destroy", "nova_b200_upload_scene", "nova_b200_build_bvh",
           "nova_b200_render", "nova_b200_trace", "nova_b200_sobol", "nova_b200_bake_irradiance",
           "nova_b200_get_error", "nova_b200_scene_info", "nova_b200_synchronize", "nova_b200_render_noalloc", "nova_b200_render_batch",
           "nova_b200_scatter", "nova_b200_set_tuning", "nova_b200_get_tuning", "nova_b200_autotune",
           "nova_b200_set_diff_params", "nova_b200_backward", "nova_b200_upload_scene_batch",
           "nova_b200_build_bvh_batch", "nova_b200_upload_build_batch", "nova_b200_upload_build_render_batch",
           "nova_b200_render_aov",
           "nova_b200_film_accumulate",
           "nova_b200_display_blend", "nova_b200_snapshot", "nova_b200_hdr_info", "nova_b200_hdr_read",
           "nova_b200_hdr_write", "nova_b200_last_call_ms", "nova_b200_bake_texture",
           "nova_b200_trace_host", "nova_b200_cancel", "nova_b200_bake_irradiance_texunit",
           "nova_b200_bake_texture_flags"]


def lib():
    """Loads libnova_b200.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libnova_b200.so is not built (run __graft_entry__.build() or make -C axomae_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.nova_b200_create.argtypes = [C.POINTER(vp), C.c_int32]
        L.nova_b200_destroy.argtypes = [vp]
        L.nova_b200_upload_scene.argtypes = [vp, C.POINTER(SceneDesc)]
        L.nova_b200_build_bvh.argtypes = [vp, C.POINTER(BvhOptions)]
        L.nova_b200_render.argtypes = [vp, C.POINTER(Frame), vp, vp, C.POINTER(RenderStats)]
        L.nova_b200_trace.argtypes = [vp, C.c_uint64, vp, vp, vp, vp, vp, vp]
        L.nova_b200_sobol.argtypes = [vp, C.c_uint64, vp, vp, C.c_uint32, vp]
        L.nova_b200_render_aov.argtypes = [vp, C.POINTER(Frame), C.c_int32, C.c_float, C.c_float, vp, vp]
        L.nova_b200_upload_scene_batch.argtypes = [C.POINTER(vp), C.POINTER(SceneDesc), C.c_uint32]
        L.nova_b200_build_bvh_batch.argtypes = [C.POINTER(vp), C.c_uint32, C.POINTER(BvhOptions)]
        L.nova_b200_upload_build_batch.argtypes = [C.POINTER(vp), C.POINTER(SceneDesc), C.c_uint32,
                                                   C.POINTER(BvhOptions)]
        L.nova_b200_upload_build_render_batch.argtypes = [C.POINTER(vp), C.POINTER(SceneDesc), C.POINTER(Frame),
                                                          C.c_uint32, C.POINTER(BvhOptions), C.POINTER(vp),
                                                          C.POINTER(vp), C.POINTER(RenderStats)]
        L.nova_b200_set_diff_params.argtypes = [vp, vp, vp]
        L.nova_b200_backward.argtypes = [vp, C.POINTER(Frame), vp, vp, vp, C.c_uint32, C.POINTER(RenderStats)]
        L.nova_b200_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.nova_b200_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.nova_b200_autotune.argtypes = [C.POINTER(vp), C.POINTER(Frame), C.c_uint32, C.c_char_p, C.c_uint32,
                                         C.POINTER(Tuning)]
        L.nova_b200_scatter.argtypes = [vp, C.c_uint64] + [vp] * 8 + [C.c_uint32] + [vp] * 5
        L.nova_b200_bake_irradiance.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                                C.c_int32, vp]
        L.nova_b200_get_error.argtypes = [vp, C.c_char_p, C.POINTER(C.c_size_t)]
        L.nova_b200_get_error.restype = None
        L.nova_b200_scene_info.argtypes = [vp] + [C.POINTER(C.c_uint64)] * 5
        L.nova_b200_synchronize.argtypes = [vp]
        L.nova_b200_render_noalloc.argtypes = [vp, C.POINTER(Frame), vp]
        L.nova_b200_film_accumulate.argtypes = [vp, vp, vp, vp, C.c_uint64, C.c_uint32]
        L.nova_b200_display_blend.argtypes = [vp, vp, vp, vp, C.c_uint64, C.c_uint32]
        L.nova_b200_snapshot.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32, C.c_int32]
        L.nova_b200_hdr_info.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.nova_b200_hdr_read.argtypes = [vp, C.c_char_p, vp, vp, C.c_uint64]
        L.nova_b200_hdr_write.argtypes = [vp, C.c_char_p, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.nova_b200_last_call_ms.argtypes = [vp, C.POINTER(C.c_float)]
        L.nova_b200_cancel.argtypes = [vp]
        L.nova_b200_bake_texture.argtypes = [vp, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_char_p,
                                             C.c_char_p]
        L.nova_b200_bake_texture_flags.argtypes = [vp, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_char_p,
                                                   C.c_char_p, C.c_uint32]
        L.nova_b200_bake_irradiance_texunit.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                                        C.c_int32, C.c_int32, vp]
        L.nova_b200_render_batch.argtypes = [C.POINTER(vp), C.POINTER(Frame), C.c_uint32, C.POINTER(vp),
                                             C.POINTER(vp), C.POINTER(RenderStats)]
        for name in EXPORTS:
            if name != "nova_b200_get_error":
                getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _np_dtype(struct):
    """numpy dtype with the layout of a ctypes Structure (pointer fields as uint64 addresses)."""
    names, formats, offsets = [], [], []
    for name, ctype in struct._fields_:
        names.append(name)
        offsets.append(getattr(struct, name).offset)
        if issubclass(ctype, C._Pointer):
            formats.append(np.uint64)
        elif issubclass(ctype, C.Array):
            formats.append((np.dtype(ctype._type_), ctype._length_))
        else:
            formats.append(np.dtype(ctype))
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": C.sizeof(struct)})


def _addr(a) -> int:
    return a.ctypes.data


def make_scene_desc(scene: dict):
    """Builds the C scene descriptor for a scene dictionary (axomae_b200.scenes layout), filling the
    descriptor tables as numpy records with the C layout.  Returns (desc, keepalive) — keep
    `keepalive` referenced until the upload call returns."""
    keep = []
    ms = scene["meshes"]
    mt = np.zeros(len(ms), _np_dtype(Mesh))

    def as_c(a, dtype):
        if not (type(a) is np.ndarray and a.dtype == dtype and a.flags.c_contiguous):
            a = np.ascontiguousarray(a, dtype)
        keep.append(a)
        return a

    f32, u32 = np.dtype(np.float32), np.dtype(np.uint32)
    cols = {k: [] for k in ("vertices", "normals", "tangents", "bitangents", "uv", "indices", "n_verts", "n_tris")}
    for m in ms:
        for k in ("vertices", "normals", "tangents", "bitangents", "uv"):
            cols[k].append(as_c(m[k], f32).__array_interface__["data"][0])
        idx = as_c(m["indices"], u32)
        cols["indices"].append(idx.__array_interface__["data"][0])
        cols["n_verts"].append(np.size(m["vertices"]) // 3)
        cols["n_tris"].append(idx.size // 3)
    for k, v in cols.items():
        mt[k] = v
    xs = scene["instances"]
    it = np.zeros(len(xs), _np_dtype(Instance))
    it["mesh"] = [x["mesh"] for x in xs]
    it["material"] = [x["material"] for x in xs]
    it["m"] = np.asarray([x["m"] for x in xs], np.float32).reshape(-1, 16)
    it["inv"] = np.asarray([x["inv"] for x in xs], np.float32).reshape(-1, 16)
    it["n"] = np.asarray([x["n"] for x in xs], np.float32).reshape(-1, 9)
    mats = scene["materials"]
    mat = np.zeros(len(mats), _np_dtype(Material))
    for k in ("albedo", "metallic", "normalmap", "emissive"):
        mat[k] = [m.get(k, -1) for m in mats]
    mat["eta"] = np.asarray([m.get("eta", (0, 0, 0)) for m in mats], np.float32).reshape(-1, 3)
    mat["k"] = np.asarray([m.get("k", (0, 0, 0)) for m in mats], np.float32).reshape(-1, 3)
    mat["anisotropy"] = [m.get("anisotropy", 0.0) for m in mats]
    ts = scene["textures"]
    tt = np.zeros(len(ts), _np_dtype(Texture))
    for i, t in enumerate(ts):
        want = np.uint32 if t["format"] == "u8" else np.float32
        px = t["pixels"]
        if not (isinstance(px, np.ndarray) and px.dtype == want and px.flags.c_contiguous):
            px = np.ascontiguousarray(px, want)
        keep.append(px)
        tt["u8_pixels" if t["format"] == "u8" else "f32_pixels"][i] = _addr(px)
    tt["width"] = [t["width"] for t in ts]
    tt["height"] = [t["height"] for t in ts]
    tt["channels"] = [t.get("channels", 4) for t in ts]
    tt["is_rgba"] = [int(t.get("is_rgba", 1)) for t in ts]
    tt["invert_u"] = [int(t.get("invert_u", 0)) for t in ts]
    tt["invert_v"] = [int(t.get("invert_v", 0)) for t in ts]
    keep += [mt, it, mat, tt]
    desc = SceneDesc(C.cast(_addr(mt), C.POINTER(Mesh)), len(ms), C.cast(_addr(it), C.POINTER(Instance)), len(xs),
                     C.cast(_addr(mat), C.POINTER(Material)), len(mats), C.cast(_addr(tt), C.POINTER(Texture)),
                     len(ts), scene["envmap"])
    return desc, keep


def make_frame(scene: dict, width, height, spp_total, max_depth, seed=0, sample_begin=0, sample_count=None,
               rr_start=-1, reset=1, vertical_invert=0) -> Frame:
    return Frame(width, height, spp_total, sample_begin, spp_total if sample_count is None else sample_count,
                 max_depth, seed, rr_start, reset, vertical_invert,
                 (C.c_float * 16)(*np.asarray(scene["inv_P"], np.float32).reshape(16)),
                 (C.c_float * 16)(*np.asarray(scene["inv_V"], np.float32).reshape(16)))


def render_batch(contexts, frames, films_host=None, films_device=None) -> "RenderStats":
    """Renders frames[j] of contexts[j] for every j in one wavefront (nova_b200_render_batch)."""
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    fs = (Frame * n)(*frames)
    fh = None if films_host is None else (C.c_void_p * n)(*[None if a is None else a.ctypes.data for a in films_host])
    fd = None if films_device is None else (C.c_void_p * n)(*films_device)
    st = RenderStats()
    rc = lib().nova_b200_render_batch(hs, fs, n, fh, fd, C.byref(st))
    if rc != 0:
        raise NovaError(rc, contexts[0].error())
    return st


class PreparedScene:
    """A scene's C descriptor built once (make_scene_desc) for repeated uploads: it points at the
    scene's arrays, which it keeps alive, so the arrays must not be modified in place between an
    upload and the next (their contents are copied to the device at every upload)."""

    def __init__(self, scene: dict):
        self.desc, self._keep = make_scene_desc(scene)


def prepare_scene(scene: dict) -> PreparedScene:
    return PreparedScene(scene)


def _desc_of(scene):
    if isinstance(scene, PreparedScene):
        return scene.desc, scene
    return make_scene_desc(scene)


def upload_batch(contexts, scenes):
    """nova_b200_upload_scene_batch: uploads scenes[k] (a scene dictionary or a PreparedScene) to
    contexts[k], the contexts concurrently."""
    n = len(contexts)
    keep, descs = [], (SceneDesc * n)()
    for k, sc in enumerate(scenes):
        d, kp = _desc_of(sc)
        descs[k] = d
        keep.append(kp)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    rc = lib().nova_b200_upload_scene_batch(hs, descs, n)
    del keep
    if rc != 0:
        raise NovaError(rc, contexts[0].error())


def build_batch(contexts, max_leaf=0, bins=0, width=0, small_subtree=0):
    """nova_b200_build_bvh_batch: builds every context's BVH, the contexts concurrently."""
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    rc = lib().nova_b200_build_bvh_batch(hs, n, C.byref(BvhOptions(max_leaf, bins, width, small_subtree)))
    if rc != 0:
        raise NovaError(rc, contexts[0].error())


def upload_build_batch(contexts, scenes, max_leaf=0, bins=0, width=0, small_subtree=0):
    """nova_b200_upload_build_batch: uploads scenes[k] to contexts[k] and builds its BVH, the
    contexts concurrently (one scene's copies overlap another's build)."""
    n = len(contexts)
    keep, descs = [], (SceneDesc * n)()
    for k, sc in enumerate(scenes):
        d, kp = _desc_of(sc)
        descs[k] = d
        keep.append(kp)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    rc = lib().nova_b200_upload_build_batch(hs, descs, n, C.byref(BvhOptions(max_leaf, bins, width, small_subtree)))
    del keep
    if rc != 0:
        raise NovaError(rc, contexts[0].error())


def upload_build_render_batch(contexts, scenes, frames, films_host=None, films_device=None, max_leaf=0, bins=0,
                              width=0, small_subtree=0) -> "RenderStats":
    """nova_b200_upload_build_render_batch: uploads and builds every context's scene on host threads
    while the calling thread renders frames[j] of contexts[j], each chunk starting once its scenes
    are built."""
    n = len(contexts)
    keep, descs = [], (SceneDesc * n)()
    for k, sc in enumerate(scenes):
        d, kp = _desc_of(sc)
        descs[k] = d
        keep.append(kp)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    fs = (Frame * n)(*frames)
    fh = None if films_host is None else (C.c_void_p * n)(*[None if a is None else a.ctypes.data for a in films_host])
    fd = None if films_device is None else (C.c_void_p * n)(*films_device)
    st = RenderStats()
    rc = lib().nova_b200_upload_build_render_batch(hs, descs, fs, n, C.byref(BvhOptions(max_leaf, bins, width,
                                                                                          small_subtree)),
                                                   fh, fd, C.byref(st))
    del keep
    if rc != 0:
        raise NovaError(rc, contexts[0].error())
    return st


def autotune(contexts, frames, cache_path=None, flags=0) -> Tuning:
    """nova_b200_autotune: picks and applies the fastest launch tuning for these frames."""
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    fs = (Frame * n)(*frames)
    out = Tuning()
    path = None if cache_path is None else os.fsencode(cache_path)
    rc = lib().nova_b200_autotune(hs, fs, n, path, flags, C.byref(out))
    if rc != 0:
        raise NovaError(rc, contexts[0].error())
    return out


class Context:
    """One device context: scene upload, BVH build, render, queries."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        st = lib().nova_b200_create(C.byref(self.h), device)
        if st != 0:
            raise NovaError(st, "nova_b200_create failed")

    def close(self):
        if self.h:
            lib().nova_b200_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def error(self) -> str:
        buf = C.create_string_buffer(1024)
        n = C.c_size_t()
        lib().nova_b200_get_error(self.h, buf, C.byref(n))
        return buf.value.decode()

    def _check(self, st):
        if st != 0:
            raise NovaError(st, self.error())

    def upload(self, scene):
        """nova_b200_upload_scene of a scene dictionary or a PreparedScene."""
        desc, keep = _desc_of(scene)
        self._check(lib().nova_b200_upload_scene(self.h, C.byref(desc)))
        del keep

    def build(self, max_leaf=0, bins=0, width=0, small_subtree=0):
        self._check(lib().nova_b200_build_bvh(self.h, C.byref(BvhOptions(max_leaf, bins, width, small_subtree))))

    def info(self) -> dict:
        vals = [C.c_uint64() for _ in range(5)]
        self._check(lib().nova_b200_scene_info(self.h, *[C.byref(v) for v in vals]))
        return dict(zip(["triangles", "instances", "nodes", "leaves", "device_bytes"], [v.value for v in vals]))

    def render(self, frame: Frame, film_host: np.ndarray = None, film_device_ptr: int = None) -> RenderStats:
        st = RenderStats()
        host = None if film_host is None else film_host.ctypes.data_as(C.c_void_p)
        dev = None if film_device_ptr is None else C.c_void_p(film_device_ptr)
        self._check(lib().nova_b200_render(self.h, C.byref(frame), host, dev, C.byref(st)))
        return st

    def render_noalloc(self, frame: Frame, film_device_ptr: int):
        """Allocation-free render into a device film (mean of the frame's sample range)."""
        self._check(lib().nova_b200_render_noalloc(self.h, C.byref(frame), C.c_void_p(film_device_ptr)))

    def trace(self, orig_ptr, dir_ptr, n, prim_ptr, t_ptr, u_ptr, v_ptr):
        """Device pointers (e.g. torch CUDA tensors' data_ptr())."""
        self._check(lib().nova_b200_trace(self.h, n, C.c_void_p(orig_ptr), C.c_void_p(dir_ptr), C.c_void_p(prim_ptr),
                                          C.c_void_p(t_ptr), C.c_void_p(u_ptr), C.c_void_p(v_ptr)))

    def scatter(self, n, o_ptr, d_ptr, prim_ptr, t_ptr, u_ptr, v_ptr, index_ptr, bounce_ptr, seed, out_o_ptr,
                out_d_ptr, weight_ptr, emissive_ptr, valid_ptr):
        """One shading event per hit (nova_b200_scatter); device pointers."""
        ptrs = [o_ptr, d_ptr, prim_ptr, t_ptr, u_ptr, v_ptr, index_ptr, bounce_ptr]
        outs = [out_o_ptr, out_d_ptr, weight_ptr, emissive_ptr, valid_ptr]
        self._check(lib().nova_b200_scatter(self.h, n, *[C.c_void_p(p) for p in ptrs], seed,
                                            *[C.c_void_p(p) for p in outs]))

    def render_aov(self, frame, kind, near_plane=0.1, far_plane=1000.0, film_host=None, film_device_ptr=None):
        """AOV integrator image (AOV_NORMAL, AOV_DEPTH, AOV_EMISSIVE) into a host and/or device film."""
        fh = film_host.ctypes.data_as(C.c_void_p) if film_host is not None else None
        fd = C.c_void_p(film_device_ptr) if film_device_ptr else None
        self._check(lib().nova_b200_render_aov(self.h, C.byref(frame), kind, near_plane, far_plane, fh, fd))

    def set_diff_params(self, albedo_ptr=None, roughness_ptr=None):
        """Per-triangle RGB albedo / per-material roughness in device memory (None: textures)."""
        self._check(lib().nova_b200_set_diff_params(self.h, C.c_void_p(albedo_ptr) if albedo_ptr else None,
                                                    C.c_void_p(roughness_ptr) if roughness_ptr else None))

    def backward(self, frame, d_image_ptr, grad_albedo_ptr=None, grad_roughness_ptr=None,
                 reuse_primal=False) -> "RenderStats":
        """Replay adjoint: adds dLoss/dparams to the gradient buffers (device pointers)."""
        st = RenderStats()
        self._check(lib().nova_b200_backward(self.h, C.byref(frame), C.c_void_p(d_image_ptr),
                                             C.c_void_p(grad_albedo_ptr) if grad_albedo_ptr else None,
                                             C.c_void_p(grad_roughness_ptr) if grad_roughness_ptr else None,
                                             BACKWARD_REUSE_PRIMAL if reuse_primal else 0, C.byref(st)))
        return st

    def set_tuning(self, tuning=None, **kw):
        """Sets the launch tuning (a Tuning, or keyword fields; nothing = defaults)."""
        t = tuning if tuning is not None else Tuning(**kw)
        self._check(lib().nova_b200_set_tuning(self.h, C.byref(t) if (tuning is not None or kw) else None))

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self._check(lib().nova_b200_get_tuning(self.h, C.byref(t)))
        return t

    def sobol(self, idx_ptr, dim_ptr, n, seed, out_ptr):
        self._check(lib().nova_b200_sobol(self.h, n, C.c_void_p(idx_ptr), C.c_void_p(dim_ptr), seed,
                                          C.c_void_p(out_ptr)))

    def bake_irradiance(self, src_ptr, sw, sh, ch, ow, oh, samples, out_ptr):
        self._check(lib().nova_b200_bake_irradiance(self.h, C.c_void_p(src_ptr), sw, sh, ch, ow, oh, samples,
                                                    C.c_void_p(out_ptr)))

    def bake_irradiance_texunit(self, src_ptr, sw, sh, ch, ow, oh, samples, out_ptr):
        """The bake of the reference's CUDA kernel (texture-unit filtering); out: ow * oh * 4 floats."""
        self._check(lib().nova_b200_bake_irradiance_texunit(self.h, C.c_void_p(src_ptr), sw, sh, ch, ow, oh, samples,
                                                            C.c_void_p(out_ptr)))

    def film_accumulate(self, partial_ptr, accum_ptr, final_ptr, n, frame_index):
        """accum += partial; final = accum / (frame_index + 1) over n device floats."""
        self._check(lib().nova_b200_film_accumulate(self.h, C.c_void_p(partial_ptr), C.c_void_p(accum_ptr),
                                                    C.c_void_p(final_ptr) if final_ptr else None, n, frame_index))

    def display_blend(self, partial_ptr, accum_ptr, out_ptr, n, current_frame):
        """The editor's display value over n device floats."""
        self._check(lib().nova_b200_display_blend(self.h, C.c_void_p(partial_ptr), C.c_void_p(accum_ptr),
                                                  C.c_void_p(out_ptr), n, current_frame))

    def snapshot(self, film_ptr, width, height, channels, dst_ptr, dst_width, dst_height):
        """The film resampled to dst_width x dst_height (device buffers)."""
        self._check(lib().nova_b200_snapshot(self.h, C.c_void_p(film_ptr), width, height, channels,
                                             C.c_void_p(dst_ptr), dst_width, dst_height))

    def hdr_read(self, path, rgba_host=None, rgba_device_ptr=None, capacity=None):
        """Reads a .hdr file as (height, width, 4) floats into a host array and / or device buffer."""
        w, h = hdr_info(path)
        cap = capacity if capacity is not None else w * h * 4
        if rgba_host is not None and rgba_host.size < cap:
            raise ValueError("host array too small")
        fh = rgba_host.ctypes.data_as(C.c_void_p) if rgba_host is not None else None
        fd = C.c_void_p(rgba_device_ptr) if rgba_device_ptr else None
        self._check(lib().nova_b200_hdr_read(self.h, os.fsencode(path), fh, fd, cap))
        return w, h

    def hdr_write(self, path, width, height, channels, pixels_host=None, pixels_device_ptr=None, flip=False):
        """Writes path + ".hdr" from host or device pixels (width * height * channels floats)."""
        if pixels_host is not None:
            pixels_host = np.ascontiguousarray(pixels_host, np.float32)
            if pixels_host.size < width * height * channels:
                raise ValueError("pixel array too small")
        fh = pixels_host.ctypes.data_as(C.c_void_p) if pixels_host is not None else None
        fd = C.c_void_p(pixels_device_ptr) if pixels_device_ptr else None
        self._check(lib().nova_b200_hdr_write(self.h, os.fsencode(path), fh, fd, width, height, channels,
                                              1 if flip else 0))

    def bake_texture(self, kind, width, height, samples, path_in, path_out, gpu_kernel=False):
        """The bake command: path_in (.hdr) -> irradiance map path_out + ".hdr" (gpu_kernel: the
        reference's --gpu bake)."""
        self._check(lib().nova_b200_bake_texture_flags(self.h, kind.encode(), width, height, samples,
                                                       os.fsencode(path_in), os.fsencode(path_out),
                                                       1 if gpu_kernel else 0))

    def cancel(self):
        """Stops the render / backward call running on this context in another thread."""
        self._check(lib().nova_b200_cancel(self.h))

    def last_call_ms(self) -> float:
        """Device time of the kernel of the last film / .hdr call."""
        ms = C.c_float(0.0)
        self._check(lib().nova_b200_last_call_ms(self.h, C.byref(ms)))
        return ms.value

    def synchronize(self):
        self._check(lib().nova_b200_synchronize(self.h))


def hdr_info(path):
    """(width, height) of a Radiance .hdr file (header only; no device needed)."""
    w, h = C.c_int32(0), C.c_int32(0)
    st = lib().nova_b200_hdr_info(None, os.fsencode(path), C.byref(w), C.byref(h))
    if st != 0:
        raise NovaError(st, "not a readable Radiance .hdr file: %s" % path)
    return w.value, h.value
