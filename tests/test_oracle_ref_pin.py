"""The oracle's restatements of the reference's header-only arithmetic, held bit for bit to those
headers compiled as they are (oracle/ref_pieces.cpp -> oracle/_ref/libref_pieces.so, built by
`make -C oracle ref` from the reference tree): the fast atan2 polynomial of the environment lookup
(corelib/internal/common/math/math_utils_approx.h:13-40), rgb_uint2float and uvToPixel
(corelib/internal/common/math/math_texturing.h:8-21), and the CPU path's tile split
(corelib/nova/utils/nova_utils.h:34-53).  The device computes the same functions bit
for bit (test_scatter_bit_exact compares environment lookups and texel reads with the oracle's),
so this pins that part of the device path to the reference's own code.  Skipped where neither the
reference tree nor a prebuilt pin library is present."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PIN = os.path.join(ROOT, "oracle", "_ref", "libref_pieces.so")
f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)


@pytest.fixture(scope="module")
def pin():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], capture_output=True)
    if not os.path.exists(PIN):
        pytest.skip("the reference tree is not here and no pin library was built")
    L = C.CDLL(PIN)
    L.ref_atan2_approx.argtypes = [C.c_uint64, f32p, f32p, f32p]
    L.ref_rgb_uint2float.argtypes = [C.c_uint64, f32p, f32p]
    L.ref_uv_to_pixel.argtypes = [C.c_uint64, f32p, u32p, u32p]
    L.ref_divide_by_tiles.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]
    L.ref_divide_by_tiles.restype = C.c_int32
    return L


def _p(a, t):
    return a.ctypes.data_as(t)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_atan2_approx_matches_reference_header(oracle, pin):
    rng = np.random.default_rng(21)
    y = np.concatenate([rng.standard_normal(200000), rng.uniform(-1e-30, 1e-30, 1000),
                        [0.0, 0.0, -0.0, 1.0, -1.0, 0.0, 1.0, -1.0, 1e30, -1e30]]).astype(np.float32)
    x = np.concatenate([rng.standard_normal(200000), rng.uniform(-1e-30, 1e-30, 1000),
                        [1.0, -1.0, 1.0, 0.0, 0.0, 0.0, 1.0, -1.0, 1.0, -1.0]]).astype(np.float32)
    want, got = np.zeros_like(y), np.zeros_like(y)
    pin.ref_atan2_approx(y.size, _p(y, f32p), _p(x, f32p), _p(want, f32p))
    lib = oracle.lib()
    lib.orc_atan2_approx(y.size, _p(y, f32p), _p(x, f32p), _p(got, f32p))
    same = (_bits(got) == _bits(want)) | (np.isnan(got) & np.isnan(want))
    assert same.all(), np.flatnonzero(~same)[:10]


def test_texel_conversions_match_reference_header(oracle, pin):
    rng = np.random.default_rng(22)
    v = np.concatenate([np.arange(256), rng.uniform(0.0, 255.0, 100000)]).astype(np.float32)
    want, got = np.zeros_like(v), np.zeros_like(v)
    pin.ref_rgb_uint2float(v.size, _p(v, f32p), _p(want, f32p))
    lib = oracle.lib()
    lib.orc_rgb_to_unit(v.size, _p(v, f32p), _p(got, f32p))
    np.testing.assert_array_equal(_bits(got), _bits(want))

    t = np.concatenate([rng.uniform(0.0, 1.0, 100000), [0.0, 1.0, 0.5, np.nextafter(1.0, 0.0)]]).astype(np.float32)
    dim = rng.integers(1, 65537, t.size).astype(np.uint32)
    dim[-4:] = [1, 4096, 3, 65535]
    want_i, got_i = np.zeros_like(dim), np.zeros_like(dim)
    pin.ref_uv_to_pixel(t.size, _p(t, f32p), _p(dim, u32p), _p(want_i, u32p))
    lib.orc_uv_to_pixel(t.size, _p(t, f32p), _p(dim, u32p), _p(got_i, u32p))
    np.testing.assert_array_equal(got_i, want_i)


def test_tile_split_matches_reference_header(oracle, pin):
    rng = np.random.default_rng(23)
    cases = [(50, 50, 5, 5), (97, 61, 6, 4), (1920, 1080, 60, 33), (7, 5, 7, 5), (8, 8, 1, 1)]
    cases += [(int(w), int(h), int(rng.integers(1, min(w, 64) + 1)), int(rng.integers(1, min(h, 64) + 1)))
              for w, h in rng.integers(1, 4000, (200, 2))]
    for w, h, tw, th in cases:
        want = np.zeros((tw * th, 4), np.int32)
        n = pin.ref_divide_by_tiles(w, h, tw, th, want.ctypes.data_as(C.POINTER(C.c_int32)))
        assert n == tw * th
        np.testing.assert_array_equal(oracle.tile_split(w, h, tw, th), want)


def _fixture(pin, shape):
    """A mesh fixture of the reference's unit tests (geometry_shapes.h), compiled into the pin."""
    pin.ref_fixture_floats.restype = C.c_int64
    pin.ref_fixture_indices.restype = C.c_int64
    out = {}
    for attr in ("vertices", "normals", "uv", "tangents", "bitangents"):
        n = pin.ref_fixture_floats(shape.encode(), attr.encode(), None, 0)
        a = np.zeros(n, np.float32)
        pin.ref_fixture_floats(shape.encode(), attr.encode(), _p(a, f32p), n)
        out[attr] = a
    n = pin.ref_fixture_indices(shape.encode(), None, 0)
    idx = np.zeros(n, np.uint32)
    pin.ref_fixture_indices(shape.encode(), _p(idx, u32p), n)
    out["indices"] = idx
    return out


@pytest.mark.parametrize("shape", ["CUBE", "QUAD", "TRIANGLE"])
def test_triangle_bounds_on_reference_fixtures(oracle, pin, shape):
    """TriangleTest.computeAABB / centroid (shape/TriangleTest.cpp:25-62) on the reference's own
    fixture meshes, every face: the oracle's box is the min / max of the face's vertices and its
    centroid their mean within 1e-5 (identity transform, as the reference test builds it)."""
    from axomae_b200 import scenes
    mesh = _fixture(pin, shape)
    nv = mesh["vertices"].size // 3
    for attr in ("normals", "tangents", "bitangents"):  # one record per vertex (CUBE's lists are per face corner)
        mesh[attr] = mesh[attr][:3 * nv]
    mesh["uv"] = mesh["uv"][:2 * nv]
    b = scenes._Builder()
    b.add(mesh, b.lambert((0.5, 0.5, 0.5)))
    env = b.tex(scenes.f32_texture(np.ones((2, 2, 4), np.float32)))
    scene = b.finish(env, scenes.camera((0.0, 0.0, 5.0), (0.0, 0.0, 0.0), 8, 8))
    boxes, cents = oracle.OracleScene(scene).prim_bounds()
    tri = mesh["vertices"].reshape(-1, 3)[mesh["indices"].reshape(-1, 3)]
    assert boxes.shape[0] == tri.shape[0] == mesh["indices"].size // 3
    np.testing.assert_array_equal(boxes[:, :3], tri.min(axis=1))
    np.testing.assert_array_equal(boxes[:, 3:], tri.max(axis=1))
    assert np.abs(cents - tri.mean(axis=1)).max() <= 1e-5
