"""The Nova engine API re-stated in C++ (include/nova_b200_api.hpp, libnova_b200_engine.so), through
its own test program tests/cpp/engine_test.cpp (built by tests/cpp/Makefile):

- `cpu`: transforms, cameras, render options, render buffers, scenes and the engine's error codes,
  with no GPU;
- `accel` (GPU): the reference's acceleration tests (inside a cube every ray hits; in front of it,
  looking at it, every ray hits; just outside, looking away, none does; with the cube moved 3 units
  to the right, none does) on DeviceAcceleratorInterface::make()'s B200 accelerator;
- `render` (GPU): a progressive nova::Engine render equals a one-shot C-ABI render of the same
  scene bit for bit, its NORMAL pass equals nova_b200_render_aov, a failing frame stops the render
  with a message; the image is then compared here with the oracle's render of the same scene."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "_build", "engine_test")


@pytest.fixture(scope="module")
def engine_test():
    if not os.path.exists(os.path.join(ROOT, "axomae_b200", "libnova_b200_engine.so")):
        pytest.fail("build the libraries first (make -C axomae_b200/csrc)")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    return EXE


def _run(exe, *args, timeout=600):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def test_engine_api_without_device(engine_test):
    _run(engine_test, "cpu")


@pytest.mark.gpu
def test_engine_accelerator_cube_hits(engine_test):
    _run(engine_test, "accel")


@pytest.mark.gpu
def test_engine_render_matches_c_abi_and_oracle(engine_test, oracle, tmp_path):
    _run(engine_test, "render", str(tmp_path))
    d = str(tmp_path)
    lines = open(os.path.join(d, "meta.txt")).read().split("\n")
    W, H, spp, depth, n_meshes, n_u8 = (int(x) for x in lines[0].split())
    eye16 = np.eye(4, dtype=np.float32).reshape(-1)
    eye9 = np.eye(3, dtype=np.float32).reshape(-1)
    meshes, instances, materials = [], [], []
    for i in range(n_meshes):
        f = lambda k, t=np.float32: np.fromfile(os.path.join(d, "mesh%d_%s.bin" % (i, k)), t)
        meshes.append({"vertices": f("v"), "normals": f("n"), "tangents": f("t"), "bitangents": f("b"),
                       "uv": f("uv"), "indices": f("idx", np.uint32)})
        instances.append({"mesh": i, "material": i, "m": eye16, "inv": eye16, "n": eye9})
        a, m, nm, eta = lines[1 + i].split()
        e = float(eta)
        materials.append({"albedo": int(a), "metallic": int(m), "normalmap": int(nm), "emissive": -1,
                          "eta": (e, e, e), "k": (0.0, 0.0, 0.0), "anisotropy": 0.0})
    textures = [{"format": "u8", "pixels": np.fromfile(os.path.join(d, "tex%d.bin" % k), np.uint32), "width": 2,
                 "height": 2, "channels": 4, "is_rgba": 1, "invert_u": 0, "invert_v": 0} for k in range(n_u8)]
    textures.append({"format": "f32", "pixels": np.fromfile(os.path.join(d, "env.bin"), np.float32), "width": 16,
                     "height": 8, "channels": 4, "is_rgba": 1, "invert_u": 0, "invert_v": 0})
    scene = {"meshes": meshes, "instances": instances, "materials": materials, "textures": textures,
             "envmap": n_u8, "inv_P": np.fromfile(os.path.join(d, "inv_P.bin"), np.float32),
             "inv_V": np.fromfile(os.path.join(d, "inv_V.bin"), np.float32)}
    image = np.fromfile(os.path.join(d, "image.bin"), np.float32).reshape(H, W, 4)
    ref, _ = oracle.OracleScene(scene).render(oracle.options(W, H, spp, depth))
    rel = (image[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
    assert np.isfinite(image).all() and image[..., :3].max() > 0
    assert float(np.sqrt(np.mean(rel * rel))) <= 1e-3


def test_api_caller_builds_against_reference_headers_and_here(engine_test):
    """tests/cpp/api_caller.cpp, a caller of every scene / camera / transform / mesh / material /
    texture / render-option / render-buffer method and of NovaException, compiles unchanged against
    the reference's own API headers and against include/nova_b200_api.hpp, runs its checks here,
    and both builds print the same enum values (ERROR_STATE, integrator flags, texture formats and
    channels, mesh types, exception bits)."""
    build = os.path.join(ROOT, "tests", "cpp", "_build")
    ours = _run(os.path.join(build, "api_caller"))
    assert "0 failed checks" in ours.stdout
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp"), "ref"], capture_output=True)
    ref_exe = os.path.join(build, "api_caller_ref")
    if not os.path.exists(ref_exe):
        pytest.skip("the reference's API headers are not here")
    ref = _run(ref_exe)
    enum_lines = lambda out: [l for l in out.splitlines() if not l.startswith("api caller")]
    assert enum_lines(ours.stdout) == enum_lines(ref.stdout)
    assert len(enum_lines(ref.stdout)) == 5
