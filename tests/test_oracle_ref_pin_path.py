"""The oracle's restatement of the Nova path past the sampler, held bit for bit to the reference's own
code compiled as it is (oracle/ref_nova_path.cpp -> oracle/_ref/libref_pieces.so, built from the
reference tree by `make -C oracle ref`): PrincipledBSDF::sample_f with its lobe weights, lobe choice
and shading frame (corelib/nova/material/BSDF.h:22-162), the Disney diffuse, GGX specular and
dielectric lobes' sample_f and the dielectric's f / pdf (material/BxDF.h:252-608), the VNDF, Fresnel
and specular-normal correction (material/BxDF_math.h:26-343), Triangle::hit's Moller-Trumbore
(shape/Triangle.h:146-177), the traversal's slab test (internal/geometry/BoundingBox.cpp:150-160),
Ray::spawn (ray/Ray.h:22-27) and the frame helpers gram_shmidt / make_onb
(internal/common/math/utils_3D.h:52-81).

Those headers need glm, an empty submodule in the reference tree; oracle/glm_shim stands in for it
with glm's evaluation order.  The pin library links correctly rounded float transcendentals (each
evaluated in double and rounded once), the convention the oracle and the device share; the last test
measures how far glibc's own cosf / powf / ... move the reference's samples.

The device is held bit for bit to the oracle on the same functions (test_gpu_parity.py:
test_scatter_bit_exact, test_random_ray_hits), so these cases pin the device path to the reference's
code through the oracle.  Skipped where neither the reference tree nor a prebuilt pin library is
present."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PIN = os.path.join(ROOT, "oracle", "_ref", "libref_pieces.so")
f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
vp = C.c_void_p

CASE = np.dtype([("ns", "<f4", 3), ("ng", "<f4", 3), ("dpdu", "<f4", 3), ("dpdv", "<f4", 3), ("wo_dot_ng", "<f4"),
                 ("roughness", "<f4"), ("metal", "<f4"), ("transmission", "<f4"), ("anisotropy", "<f4"),
                 ("eta", "<f4"), ("albedo", "<f4", 3), ("wo", "<f4", 3), ("uc", "<f4"), ("u", "<f4", 2),
                 ("weight", "<f4"), ("probability", "<f4"), ("thin", "<i4")])
RESULT = np.dtype([("f", "<f4", 3), ("wi", "<f4", 3), ("pdf", "<f4"), ("costheta", "<f4"), ("flags", "<u4"),
                   ("valid", "<i4")])
assert CASE.itemsize == 120 and RESULT.itemsize == 40  # orc_bsdf_case / orc_bsdf_result (oracle/oracle.h)

N = 200000


@pytest.fixture(scope="module")
def pin():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], capture_output=True)
    if not os.path.exists(PIN):
        pytest.skip("the reference tree is not here and no pin library was built")
    L = C.CDLL(PIN)
    L.ref_principled_sample.argtypes = [C.c_uint64, vp, vp]
    L.ref_lobe_sample.argtypes = [C.c_int32, C.c_uint64, vp, vp]
    L.ref_dielectric_eval.argtypes = [C.c_uint64, vp, f32p, f32p, f32p]
    L.ref_triangle_hits.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, C.c_float, C.c_float, i32p, f32p, f32p, f32p]
    L.ref_box_intersect.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, f32p, f32p]
    L.ref_spawn.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, f32p]
    L.ref_gram_shmidt.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p]
    L.ref_make_onb.argtypes = [C.c_uint64, f32p, f32p]
    L.ref_fresnel_real.argtypes = [C.c_float, C.c_float, f32p]
    L.ref_fresnel_real.restype = C.c_float
    L.ref_vndf.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, f32p, f32p]
    L.ref_correct_specular_normal.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p]
    L.ref_libm_glibc.argtypes = [C.c_int32]
    L.ref_libm_glibc(0)
    return L


@pytest.fixture(scope="module")
def orc(oracle):
    L = oracle.lib()
    L.orc_principled_sample.argtypes = [C.c_uint64, vp, vp]
    L.orc_lobe_sample.argtypes = [C.c_int32, C.c_uint64, vp, vp]
    L.orc_dielectric_eval.argtypes = [C.c_uint64, vp, f32p, f32p, f32p]
    L.orc_triangle_hits.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, C.c_float, C.c_float, i32p, f32p, f32p, f32p]
    L.orc_spawn.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p, f32p]
    L.orc_gram_shmidt.argtypes = [C.c_uint64, f32p, f32p, f32p, f32p]
    L.orc_make_onb.argtypes = [C.c_uint64, f32p, f32p]
    return L


def _p(a, t=f32p):
    return a.ctypes.data_as(t)


def _same(a, b):
    """Bit-equal, NaN equal to NaN."""
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _uniforms(rng, n):
    """Uniforms in [0, 1) as float32, with the ends and values one ulp from them mixed in."""
    u = rng.random(n).astype(np.float32)
    edge = np.array([0.0, np.nextafter(np.float32(0), np.float32(1)), 0.5, np.nextafter(np.float32(1), np.float32(0))],
                    np.float32)
    pick = rng.random(n) < 0.02
    u[pick] = rng.choice(edge, pick.sum())
    return u


def _cases(rng, n, local):
    c = np.zeros(n, CASE)
    ns = _unit(rng, n)
    c["ns"] = ns
    c["ng"] = (ns + 0.3 * _unit(rng, n)).astype(np.float32)
    c["ng"] /= np.linalg.norm(c["ng"], axis=1, keepdims=True)
    c["dpdu"] = _unit(rng, n) * rng.uniform(0.1, 4.0, (n, 1)).astype(np.float32)
    c["dpdv"] = _unit(rng, n) * rng.uniform(0.1, 4.0, (n, 1)).astype(np.float32)
    if local:  # a direction in the lobe's own frame, mostly above the surface
        wo = _unit(rng, n)
        wo[:, 2] = np.where(rng.random(n) < 0.8, np.abs(wo[:, 2]), wo[:, 2])
        c["wo"] = wo
    else:
        c["wo"] = _unit(rng, n)
    c["wo_dot_ng"] = np.einsum("ij,ij->i", c["wo"], c["ng"]).astype(np.float32)
    r = rng.random(n).astype(np.float32)
    r[rng.random(n) < 0.05] = 0.0
    r[rng.random(n) < 0.05] = 1.0
    c["roughness"] = r
    c["metal"] = rng.choice(np.array([0.0, 1.0, 0.3, 0.75], np.float32), n)
    c["transmission"] = rng.choice(np.array([0.0, 1.0], np.float32), n)
    c["anisotropy"] = np.where(rng.random(n) < 0.7, 0.0, rng.uniform(-1.2, 1.2, n)).astype(np.float32)
    c["eta"] = rng.choice(np.array([0.0, 1.0, 1.5, 1.33, 2.4], np.float32), n)
    c["albedo"] = rng.random((n, 3)).astype(np.float32)
    c["uc"] = _uniforms(rng, n)
    c["u"][:, 0] = _uniforms(rng, n)
    c["u"][:, 1] = _uniforms(rng, n)
    c["weight"] = rng.uniform(0.0, 1.0, n).astype(np.float32)
    c["probability"] = rng.uniform(0.05, 1.0, n).astype(np.float32)
    c["thin"] = (rng.random(n) < 0.1).astype(np.int32)
    return c


def _compare_samples(want, got):
    assert (want["valid"] == got["valid"]).all(), np.flatnonzero(want["valid"] != got["valid"])[:10]
    ok = want["valid"] == 1
    assert ok.sum() > 0.2 * ok.size  # the cases exercise the sampled branch
    assert (want["flags"][ok] == got["flags"][ok]).all()
    for k in ("f", "wi", "pdf", "costheta"):
        same = _same(want[k][ok], got[k][ok])
        assert same.all(), (k, np.flatnonzero(~same.reshape(same.shape[0], -1).all(axis=1))[:10])


def test_principled_bsdf_sample_matches_reference(pin, orc):
    """PrincipledBSDF(params, uc).sample_f in world space: lobe weights (BSDF.h:43-67), the lobe
    choice with no fallback (:69-79), the frame and its flip with 1/eta (:87-97), sample_f (:107-130)."""
    rng = np.random.default_rng(101)
    cases = _cases(rng, N, local=False)
    want, got = np.zeros(N, RESULT), np.zeros(N, RESULT)
    pin.ref_principled_sample(N, cases.ctypes.data, want.ctypes.data)
    orc.orc_principled_sample(N, cases.ctypes.data, got.ctypes.data)
    _compare_samples(want, got)
    for flag in (4 | 1, 8 | 1, 8 | 2, 16 | 1, 16 | 2):  # diffuse, glossy R/T, specular R/T all reached
        assert (want["flags"][want["valid"] == 1] == flag).any(), flag


@pytest.mark.parametrize("lobe,name", [(1, "DisneyDiffuseBxDF"), (2, "SpecularBxDF"), (3, "DielectricBxDF")])
def test_lobe_sample_matches_reference(pin, orc, lobe, name):
    """<lobe>::sample_f in the local frame with its construction weight and probability (BxDF.h)."""
    rng = np.random.default_rng(110 + lobe)
    cases = _cases(rng, N, local=True)
    if lobe == 3:
        cases["eta"] = np.where(cases["eta"] == 0.0, np.float32(1.5), cases["eta"])
    want, got = np.zeros(N, RESULT), np.zeros(N, RESULT)
    pin.ref_lobe_sample(lobe, N, cases.ctypes.data, want.ctypes.data)
    orc.orc_lobe_sample(lobe, N, cases.ctypes.data, got.ctypes.data)
    _compare_samples(want, got)


def test_dielectric_f_pdf_match_reference(pin, orc):
    """DielectricBxDF::f / ::pdf (BxDF.h:497-545) at directions in both hemispheres."""
    rng = np.random.default_rng(120)
    cases = _cases(rng, N, local=True)
    cases["eta"] = np.where(cases["eta"] == 0.0, np.float32(1.5), cases["eta"])
    wi = _unit(rng, N)
    fw, fg = np.zeros((N, 3), np.float32), np.zeros((N, 3), np.float32)
    pw, pg = np.zeros(N, np.float32), np.zeros(N, np.float32)
    pin.ref_dielectric_eval(N, cases.ctypes.data, _p(wi), _p(fw), _p(pw))
    orc.orc_dielectric_eval(N, cases.ctypes.data, _p(wi), _p(fg), _p(pg))
    assert _same(fw, fg).all() and _same(pw, pg).all()
    assert (pw > 0).mean() > 0.3


def _triangle_cases(rng, n):
    tri = rng.uniform(-2.0, 2.0, (n, 9)).astype(np.float32)
    # inverse transforms: identity, translations, rotations with scale
    inv = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (n, 1))
    kind = rng.integers(0, 3, n)
    for i in np.flatnonzero(kind > 0):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        m = np.eye(4)
        m[:3, :3] = q * rng.uniform(0.3, 3.0) if kind[i] == 2 else np.eye(3)
        m[:3, 3] = rng.uniform(-5, 5, 3)
        inv[i] = np.linalg.inv(m).T.reshape(16).astype(np.float32)  # column-major
    # rays: aimed at a random barycentric point (with the edges and vertices mixed in), or random
    bary = rng.random((n, 3))
    pick = rng.random(n)
    bary[pick < 0.05, 0] = 0.0
    bary[(pick >= 0.05) & (pick < 0.1), 1] = 0.0
    bary[(pick >= 0.1) & (pick < 0.12)] = [1.0, 0.0, 0.0]
    bary /= bary.sum(axis=1, keepdims=True)
    t3 = tri.reshape(n, 3, 3).astype(np.float64)
    target_obj = np.einsum("nk,nkj->nj", bary, t3)
    minv = inv.reshape(n, 4, 4).transpose(0, 2, 1).astype(np.float64)
    m = np.linalg.inv(minv)
    target = np.einsum("nij,nj->ni", m[:, :3, :3], target_obj) + m[:, :3, 3]
    o = (target + rng.standard_normal((n, 3)) * 3.0).astype(np.float32)
    d = (target - o).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rnd = rng.random(n) < 0.15
    d[rnd] = _unit(rng, rnd.sum())
    deg = rng.random(n) < 0.01  # a repeated vertex position: det == 0
    tri[deg, 3:6] = tri[deg, 0:3]
    return tri, inv, o, d


def test_triangle_hit_matches_reference(pin, orc):
    """Triangle::hit (Triangle.h:146-177) on one triangle per ray: hit flag, t and barycentrics, with
    object-space rays through random rigid / scaled inverse transforms, edge and vertex hits and
    misses."""
    rng = np.random.default_rng(130)
    tri, inv, o, d = _triangle_cases(rng, N)
    out = []
    for fn in (pin.ref_triangle_hits, orc.orc_triangle_hits):
        hit = np.zeros(N, np.int32)
        t, u, v = (np.zeros(N, np.float32) for _ in range(3))
        fn(N, _p(tri), _p(inv), _p(o), _p(d), 1e-6, 1e30, _p(hit, i32p), _p(t), _p(u), _p(v))
        out.append((hit, t, u, v))
    (hw, tw, uw, vw), (hg, tg, ug, vg) = out
    assert (hw == hg).all(), np.flatnonzero(hw != hg)[:10]
    h = hw == 1
    assert 0.5 < h.mean() < 0.95
    assert _same(tw[h], tg[h]).all()
    # the reference stores the interpolated uv, which equals the barycentrics up to the sign of zero
    assert (uw[h] == ug[h]).all() and (vw[h] == vg[h]).all()


def test_box_slab_test_matches_reference(pin, oracle):
    """BoundingBox::intersect(dir, origin, dist_min) (BoundingBox.cpp:150-160): the division slab test
    the native traversal culls with, incl. rays along the axes and origins inside the box."""
    rng = np.random.default_rng(140)
    n = 20000
    c = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
    e = rng.uniform(0.01, 5, (n, 3)).astype(np.float32)
    mn, mx = c - e, c + e
    o = rng.uniform(-20, 20, (n, 3)).astype(np.float32)
    o[: n // 10] = c[: n // 10]  # inside
    d = _unit(rng, n)
    axis = rng.integers(0, 3, n // 10)
    d[n // 10: n // 5] = 0.0
    d[np.arange(n // 10, n // 5), axis] = rng.choice([-1.0, 1.0], n // 10)
    dist = np.where(rng.random(n) < 0.5, np.float32(3.4028234663852886e38), rng.uniform(0, 30, n)).astype(np.float32)
    want = np.zeros(n, np.float32)
    pin.ref_box_intersect(n, _p(mn), _p(mx), _p(o), _p(d), _p(dist), _p(want))
    lib = oracle.lib()
    got = np.array([lib.orc_box_intersect(_p(mn[i]), _p(mx[i]), _p(o[i]), _p(d[i]), float(dist[i])) for i in range(n)],
                   np.float32)
    assert _same(want, got).all()
    assert (want < 3e38).mean() > 0.1


def test_spawn_and_frames_match_reference(pin, orc):
    """Ray::spawn (Ray.h:22-27), gram_shmidt and make_onb (utils_3D.h:52-81)."""
    rng = np.random.default_rng(150)
    wi, nrm = _unit(rng, N), _unit(rng, N)
    wi[: N // 20] *= rng.uniform(0.5, 3, (N // 20, 1)).astype(np.float32)  # not yet normalised
    pos = rng.uniform(-50, 50, (N, 3)).astype(np.float32)
    res = []
    for fn in (pin.ref_spawn, orc.orc_spawn):
        oo, dd = np.zeros((N, 3), np.float32), np.zeros((N, 3), np.float32)
        fn(N, _p(wi), _p(nrm), _p(pos), _p(oo), _p(dd))
        res.append((oo, dd))
    assert _same(res[0][0], res[1][0]).all() and _same(res[0][1], res[1][1]).all()

    tan = (_unit(rng, N) * rng.uniform(0.1, 3, (N, 1))).astype(np.float32)
    bit = _unit(rng, N)
    a, b = np.zeros((N, 9), np.float32), np.zeros((N, 9), np.float32)
    pin.ref_gram_shmidt(N, _p(nrm), _p(tan), _p(bit), _p(a))
    orc.orc_gram_shmidt(N, _p(nrm), _p(tan), _p(bit), _p(b))
    assert _same(a, b).all()
    a, b = np.zeros((N, 6), np.float32), np.zeros((N, 6), np.float32)
    pin.ref_make_onb(N, _p(nrm), _p(a))
    orc.orc_make_onb(N, _p(nrm), _p(b))
    assert _same(a, b).all()


def test_fresnel_vndf_and_normal_correction_match_reference(pin, oracle):
    """Fresnel::real, VNDF::sampleGGXVNDF / G1 and correct_specular_shading_normal (BxDF_math.h)."""
    rng = np.random.default_rng(160)
    lib = oracle.lib()
    n = 20000
    ior = rng.choice(np.array([1.0, 1.5, 1.33, 2.4, 0.7], np.float32), n)
    cs = rng.uniform(-1.2, 1.2, n).astype(np.float32)
    e1, e2 = C.c_float(), C.c_float()
    for i in range(n):
        a = pin.ref_fresnel_real(float(ior[i]), float(cs[i]), C.byref(e1))
        b = lib.orc_fresnel_real(float(ior[i]), float(cs[i]), C.byref(e2))
        assert _same(np.float32(a), np.float32(b)) and _same(np.float32(e1.value), np.float32(e2.value)), i

    aniso = np.where(rng.random(n) < 0.6, 0.0, rng.uniform(-1.2, 1.2, n)).astype(np.float32)
    rough = rng.random(n).astype(np.float32)
    rough[:50] = 0.0
    wo = _unit(rng, n)
    wo[:, 2] = np.abs(wo[:, 2])
    uc = rng.random((n, 2)).astype(np.float32)
    v = _unit(rng, n)
    out = np.zeros((n, 6), np.float32)
    pin.ref_vndf(n, _p(aniso), _p(rough), _p(wo), _p(uc), _p(v), _p(out))
    wm = np.zeros(3, np.float32)
    for i in range(n):
        lib.orc_vndf_sample(float(aniso[i]), float(rough[i]), _p(wo[i]), _p(uc[i]), _p(wm))
        assert _same(wm, out[i, :3]).all(), i
        g1 = lib.orc_vndf_g1(float(aniso[i]), float(rough[i]), _p(v[i]))
        assert _same(np.float32(g1), out[i, 3]), i

    ng, ns = _unit(rng, n), _unit(rng, n)
    want = np.zeros((n, 3), np.float32)
    pin.ref_correct_specular_normal(n, _p(ng), _p(wo), _p(ns), _p(want))
    got = np.zeros(3, np.float32)
    for i in range(n):
        lib.orc_correct_specular_normal(_p(ng[i]), _p(wo[i]), _p(ns[i]), _p(got))
        assert _same(got, want[i]).all(), i


def test_glibc_transcendentals_move_few_samples(pin, orc):
    """With glibc's own cosf / sinf / powf / ... (not correctly rounded) in place of the correctly
    rounded ones, the reference's principled samples still agree with the oracle on all but a small
    fraction, and those differ in the last bits: the one place the pin's libm convention matters."""
    rng = np.random.default_rng(170)
    cases = _cases(rng, N, local=False)
    want, got = np.zeros(N, RESULT), np.zeros(N, RESULT)
    pin.ref_libm_glibc(1)
    try:
        pin.ref_principled_sample(N, cases.ctypes.data, want.ctypes.data)
    finally:
        pin.ref_libm_glibc(0)
    orc.orc_principled_sample(N, cases.ctypes.data, got.ctypes.data)
    ok = (want["valid"] == 1) & (got["valid"] == 1)
    differ = ~np.all(np.concatenate([_same(want["f"], got["f"]), _same(want["wi"], got["wi"]),
                                     _same(want["pdf"], got["pdf"])[:, None]], axis=1), axis=1)
    frac = float(differ[ok].mean())
    print("glibc libm: %.3f%% of valid samples differ from the correctly rounded convention" % (100 * frac))
    assert (want["valid"] != got["valid"]).mean() < 1e-3
    assert frac < 0.05
    fw, fg = want["f"][ok], got["f"][ok]
    fin = np.isfinite(fw).all(axis=1) & np.isfinite(fg).all(axis=1)  # non-finite f: DENANed by the path
    rel = np.abs(fw[fin] - fg[fin]) / np.maximum(np.abs(fg[fin]), 1e-30)
    assert np.quantile(rel, 0.999) < 1e-5


def _lib_pin_extra(pin):
    u32p = C.POINTER(C.c_uint32)
    pin.ref_sobol.argtypes = [C.c_uint64, u32p, u32p, C.c_uint32, f32p]
    pin.ref_env_sample.argtypes = [vp, C.c_uint32, C.c_int32, C.c_uint64, f32p, f32p]
    pin.ref_material_scatter.argtypes = [C.c_uint64, f32p, f32p, u32p, vp, C.c_uint32, vp, C.c_uint32, u32p, i32p,
                                         C.c_uint32, f32p, f32p, f32p, f32p, i32p]
    return u32p


@pytest.mark.parametrize("seed", [0, 0xDEADBEEF, 12345])
def test_sobol_generator_matches_reference(pin, oracle, seed):
    """SobolGenerator(seed).generate(index, dim) (math_random.h:37-98) with the direction-vector table
    the reference's generator script writes, for every dimension the path uses and indices up to 2^32-2."""
    u32p = _lib_pin_extra(pin)
    rng = np.random.default_rng(180)
    n = 300000
    idx = np.concatenate([np.arange(4096, dtype=np.uint32), rng.integers(0, 2 ** 32 - 1, n - 4096, dtype=np.uint32)])
    idx[-3:] = [2 ** 32 - 2, 2 ** 31, 2 ** 31 - 1]
    dim = rng.integers(0, 255, n).astype(np.uint32)
    want, got = np.zeros(n, np.float32), np.zeros(n, np.float32)
    pin.ref_sobol(n, _p(idx, u32p), _p(dim, u32p), seed, _p(want))
    oracle.lib().orc_sobol_samples(_p(idx, u32p), _p(dim, u32p), n, seed, _p(got))
    assert _same(want, got).all()


def test_env_lookup_matches_reference(pin, oracle):
    """EnvmapTexture::sample (NovaTextureInterface.h:152-174): cartesianToSpherical with the fast
    atan2 and the acos table of math_acos_lt.cpp, sphericalToUv, wrap, the nearest-texel float fetch
    (TextureContext.h:196-223), on a 2048 x 1024 map, incl. the poles and the seam."""
    _lib_pin_extra(pin)
    rng = np.random.default_rng(190)
    h, w = 1024, 2048
    px = rng.lognormal(0.0, 1.5, (h, w, 4)).astype(np.float32)
    scene = {"textures": [{"format": "f32", "pixels": px, "width": w, "height": h, "channels": 4}]}
    texs, keep = oracle.texture_table(scene)
    n = 200000
    d = _unit(rng, n)
    d[:6] = [[0, 1, 0], [0, -1, 0], [0, 0, -1], [0, 0, 1], [-1, 0, 0], [1e-8, 0.3, -1]]
    d[6:1000] *= rng.uniform(0.1, 10, (994, 1)).astype(np.float32)  # not normalised
    want, got = np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)
    pin.ref_env_sample(C.cast(texs, vp), 1, 0, n, _p(d), _p(want))
    oracle.lib().orc_env_sample(_p(px), w, h, 4, n, _p(d), _p(got))
    assert _same(want, got).all()


def _scatter_scene():
    """40 small spheres and boxes on a tessellated ground, materials cycling through Lambert, GGX
    conductor, GGX dielectric and Burley diffuse; every third with a bumpy normal map, every fourth
    emissive."""
    from axomae_b200 import scenes
    rng = np.random.default_rng(41)
    b = scenes._Builder()
    b.add(scenes.grid_quad(30.0, 16), b.lambert((0.6, 0.6, 0.6)))
    for i in range(40):
        kind = i % 4
        if kind == 0:
            mat = b.lambert(rng.uniform(0.1, 0.9, 3))
        elif kind == 1:
            mat = b.conductor(rng.uniform(0.5, 1.0, 3), rng.uniform(0.0, 0.8))
        elif kind == 2:
            mat = b.dielectric(rng.uniform(0.0, 0.5))
        else:
            mat = b.burley(rng.uniform(0.1, 0.9, 3), rng.uniform(0.2, 1.0))
        c = np.array([rng.uniform(-8, 8), rng.uniform(0.5, 2.5), rng.uniform(-8, 8)])
        mesh = (scenes.uv_sphere(c, rng.uniform(0.4, 1.2), 16, 8) if rng.uniform() < 0.6
                else scenes.box(c, rng.uniform(0.3, 1.0, 3), scenes.random_rotation(rng)))
        b.add(mesh, mat)
    mats = b.materials
    for i, m in enumerate(mats):
        if i % 4 == 1:
            m["emissive"] = b.tex(scenes.solid_u8(rng.uniform(0.2, 1.0, 3)))
        if i % 3 == 2:
            nm = np.concatenate([rng.integers(90, 166, (8, 8, 2)), rng.integers(200, 256, (8, 8, 1)),
                                 np.full((8, 8, 1), 255)], -1).astype(np.uint8)
            m["normalmap"] = b.tex(scenes.u8_texture(nm))
    env = np.concatenate([rng.lognormal(0.0, 1.0, (64, 128, 3)), np.ones((64, 128, 1))], -1).astype(np.float32)
    return b.finish(b.tex(scenes.f32_texture(env)), scenes.camera((0.0, 10.0, 18.0), (0.0, 0.0, 0.0), 64, 48))


def test_material_scatter_matches_reference(pin, oracle):
    """PrincipledMaterial::scatter (NovaMaterials.h:89-137) on traced hits of a mixed Lambert / GGX
    conductor / dielectric scene with normal maps and emissive textures: the textures through
    ImageTexture<u32>'s bilinear CPU fetch, roughness = metallic.g and metal = .b, transmission when eta
    is set and k is not, the sampler's dimension order (uc, u0, u1, then uc again after the
    specular-normal correction) from a SobolSampler at the integrator's dimension 2 + 4 * bounce, then
    Ray::spawn and the path weight f * costheta / pdf.  The hit record (Embree semantics, the one step
    whose reference code needs Embree) comes from the oracle and is fed to both."""
    u32p = _lib_pin_extra(pin)
    scene = _scatter_scene()
    osc = oracle.OracleScene(scene)
    lib = oracle.lib()
    lib.orc_hit_record.argtypes = [vp, C.c_uint64, f32p, f32p, i32p, f32p, f32p, f32p, f32p]
    rng = np.random.default_rng(200)
    W, H = 64, 48
    opt = oracle.options(W, H, 4, 6)
    n = 60000
    px, py, ps = rng.integers(0, W, n), rng.integers(0, H, n), rng.integers(0, 4, n)
    o, d = osc.camera_rays(opt, px, py, ps)
    # second half: random rays from above the scene, so grazing and backface hits are in the mix
    o[n // 2:] = rng.uniform(-8, 8, (n - n // 2, 3)).astype(np.float32) + np.float32([0, 6, 0])
    d[n // 2:] = _unit(rng, n - n // 2)
    prim, t, u, v, _ = osc.trace(o, d)
    keep = prim >= 0
    o, d, prim, t, u, v = o[keep], d[keep], prim[keep], t[keep], u[keep], v[keep]
    m = prim.size
    assert m > 20000
    # material of each primitive: primitives are numbered instance by instance
    tri_counts = [np.asarray(scene["meshes"][x["mesh"]]["indices"]).size // 3 for x in scene["instances"]]
    first = np.cumsum([0] + tri_counts)
    inst = np.searchsorted(first, prim, side="right") - 1
    mat_of = np.array([x["material"] for x in scene["instances"]], np.uint32)[inst]
    index = rng.integers(0, 2 ** 31, m).astype(np.uint32)
    bounce = rng.integers(0, 8, m).astype(np.int32)
    seed = 7
    rec = np.zeros((m, 23), np.float32)
    lib.orc_hit_record(osc.h, m, _p(o), _p(d), _p(prim, i32p), _p(t), _p(u), _p(v), _p(rec))
    outs_ref = [np.zeros((m, 3), np.float32) for _ in range(4)] + [np.zeros(m, np.int32)]
    mats = oracle.material_table(scene)
    texs, keep_px = oracle.texture_table(scene)
    pin.ref_material_scatter(m, _p(rec), _p(d), _p(mat_of, u32p), C.cast(mats, vp), len(scene["materials"]),
                             C.cast(texs, vp), len(scene["textures"]), _p(index, u32p), _p(bounce, i32p), seed,
                             *[_p(a) for a in outs_ref[:4]], _p(outs_ref[4], i32p))
    no, nd, w, e, ok = osc.scatter(o, d, prim, t, u, v, index, bounce, seed=seed)
    assert (ok == outs_ref[4]).all(), np.flatnonzero(ok != outs_ref[4])[:10]
    valid = ok == 1
    assert 0.5 < valid.mean() < 1.0
    for got, want in zip((no, nd, w), outs_ref[:3]):
        assert _same(got[valid], want[valid]).all()
    assert _same(e, outs_ref[3]).all()
    # every material feature is exercised: emissive, normal-mapped, dielectric (eta set, k not)
    mm = scene["materials"]
    feats = {"emissive": [x.get("emissive", -1) >= 0 for x in mm],
             "normalmap": [i % 3 == 2 for i in range(len(mm))],
             "dielectric": [any(x.get("eta", (0, 0, 0))) and not any(x.get("k", (0, 0, 0))) for x in mm]}
    for name, flag in feats.items():
        assert np.asarray(flag)[mat_of].sum() > 100, name
    assert (e.max(axis=1) > 0).sum() > 100
