"""Film outputs and Radiance .hdr files through the C ABI on the GPU, against the CPU oracle
(oracle/film_io.cpp).  All of this is float / byte arithmetic without accumulation order, so the
bar is bit-exact (NaN compared as NaN, whatever its payload); the bake command line is compared
with the oracle's bake within one RGBE mantissa step, the bake itself being held to 1e-4."""
import os
import subprocess

import numpy as np
import pytest

from test_film_io import header, make_file

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def ctx(torch_cuda):
    from axomae_b200 import native
    c = native.Context(0)
    yield c
    c.close()


def same_bits(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    assert a.shape == b.shape
    na, nb = np.isnan(a), np.isnan(b)
    np.testing.assert_array_equal(na, nb)
    np.testing.assert_array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


def special_values(rng, shape):
    x = rng.lognormal(0, 3, shape).astype(np.float32) * rng.choice([1, -1], shape).astype(np.float32)
    flat = x.reshape(-1)
    k = flat.size
    idx = rng.choice(k, min(k, 64), replace=False)
    flat[idx[:8]] = 0.0
    flat[idx[8:16]] = -0.0
    flat[idx[16:20]] = np.inf
    flat[idx[20:24]] = -np.inf
    flat[idx[24:28]] = np.nan
    flat[idx[28:36]] = 1e-35
    flat[idx[36:44]] = 3e38
    return x


@pytest.mark.parametrize("n", [4096, 4 * 1001 + 3], ids=["aligned", "ragged"])
@pytest.mark.parametrize("frame", [0, 7])
def test_accumulate_and_display_blend_bit_exact(ctx, oracle, torch_cuda, n, frame):
    torch = torch_cuda
    rng = np.random.default_rng(n + frame)
    partial = special_values(rng, n)
    accum = rng.lognormal(0, 2, n).astype(np.float32)
    ref_acc, ref_final = oracle.film_accumulate(partial, accum, frame)
    ref_disp = oracle.display_blend(partial, accum, frame)
    tp, ta = torch.from_numpy(partial).cuda(), torch.from_numpy(accum).cuda()
    tf, td = torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")
    ctx.display_blend(tp.data_ptr(), ta.data_ptr(), td.data_ptr(), n, frame)
    ctx.film_accumulate(tp.data_ptr(), ta.data_ptr(), tf.data_ptr(), n, frame)
    same_bits(td.cpu().numpy(), ref_disp)
    same_bits(ta.cpu().numpy(), ref_acc)
    same_bits(tf.cpu().numpy(), ref_final)
    assert ctx.last_call_ms() >= 0.0


@pytest.mark.parametrize("size", [(64, 48, 64, 48), (64, 48, 37, 23), (64, 48, 200, 150), (13, 9, 1, 1),
                                  (300, 7, 64, 64)], ids=["same", "down", "up", "one", "wide"])
@pytest.mark.parametrize("channels", [3, 4])
def test_snapshot_bit_exact(ctx, oracle, torch_cuda, size, channels):
    torch = torch_cuda
    w, h, dw, dh = size
    rng = np.random.default_rng(w * 7 + dw)
    film = special_values(rng, (h, w, channels))
    init = np.full((dh, dw, channels), 5.5, np.float32)
    ref = oracle.snapshot(film, dw, dh, dst_init=init)
    tf = torch.from_numpy(film).cuda()
    to = torch.from_numpy(init).cuda()
    ctx.snapshot(tf.data_ptr(), w, h, channels, to.data_ptr(), dw, dh)
    same_bits(to.cpu().numpy(), ref)


@pytest.mark.parametrize("w,h", [(5, 3), (8, 2), (37, 11), (300, 4)])
@pytest.mark.parametrize("channels", [1, 2, 3, 4])
@pytest.mark.parametrize("flip", [0, 1])
def test_hdr_write_matches_oracle(ctx, oracle, torch_cuda, tmp_path, w, h, channels, flip):
    """The written file, read by the oracle's parser, holds exactly the oracle's RGBE encoding of the
    pixels in file row order, from host pixels and from device pixels alike."""
    torch = torch_cuda
    rng = np.random.default_rng(w * 31 + channels + flip)
    px = special_values(rng, (h, w, channels))
    px[0, : min(w, 30)] = 0.75  # runs for the run-length packets
    rows = px[::-1] if flip else px
    want = oracle.rgbe_encode(rows, channels).reshape(h, w, 4)
    for src in ("host", "device"):
        base = str(tmp_path / ("img_" + src))
        if src == "host":
            ctx.hdr_write(base, w, h, channels, pixels_host=px, flip=flip)
        else:
            t = torch.from_numpy(np.ascontiguousarray(px)).cuda()
            ctx.hdr_write(base, w, h, channels, pixels_device_ptr=t.data_ptr(), flip=flip)
        data = open(base + ".hdr", "rb").read()
        code, fw, fh, got = oracle.hdr_parse(data)
        assert (code, fw, fh) == (0, w, h)
        np.testing.assert_array_equal(got, want)
        if 8 <= w < 32768:
            assert data.count(b"\x02\x02" + bytes([w >> 8, w & 255])) >= h  # run-length rows
        # the packets themselves: the same greedy packing as the oracle's writer, byte for byte
        oracle.hdr_write(str(tmp_path / "oracle"), px, w, h, channels, flip)
        assert oracle.hdr_body(data) == oracle.hdr_body(open(str(tmp_path / "oracle.hdr"), "rb").read())


@pytest.mark.parametrize("w", [300, 32767, 32768], ids=["w300", "max-rle-width", "flat-width"])
def test_hdr_runs_round_trip(ctx, oracle, torch_cuda, tmp_path, w):
    """Rows of long and short runs (lengths 1-3, 127-129, 254-256, a whole row) between literal
    stretches: the written packets equal the oracle writer's, and reading them back gives exactly
    the decoded RGBE pixels, on the host and on the device."""
    torch = torch_cuda
    rng = np.random.default_rng(w)
    h = 3
    px = np.zeros((h, w, 4), np.float32)
    px[0] = 1.0
    pieces, x = [], 0
    for n in (1, 2, 3, 127, 128, 129, 254, 255, 256, 5, 40):
        pieces.append((x, n))
        x += n + 7
    for k, (x0, n) in enumerate(pieces):
        if x0 + n <= w:
            px[1, x0:x0 + n] = [0.5, 1.0, 0.0, 1.0][k % 4]
    px[2] = rng.lognormal(0, 1, (w, 4))
    px[2, w // 3: w // 3 + 200] = 0.0
    base = str(tmp_path / "runs")
    ctx.hdr_write(base, w, h, 4, pixels_host=px)
    data = open(base + ".hdr", "rb").read()
    oracle.hdr_write(str(tmp_path / "oracle"), px, w, h, 4)
    assert oracle.hdr_body(data) == oracle.hdr_body(open(str(tmp_path / "oracle.hdr"), "rb").read())
    code, fw, fh, q = oracle.hdr_parse(data)
    assert (code, fw, fh) == (0, w, h)
    want = oracle.rgbe_decode(q.reshape(-1, 4)).reshape(h, w, 4)
    host = np.zeros((h, w, 4), np.float32)
    dev = torch.zeros((h, w, 4), device="cuda")
    ctx.hdr_read(base + ".hdr", rgba_host=host, rgba_device_ptr=dev.data_ptr())
    same_bits(host, want)
    same_bits(dev.cpu().numpy(), want)


def test_hdr_read_matches_oracle(ctx, oracle, torch_cuda, tmp_path):
    torch = torch_cuda
    from axomae_b200 import native
    rng = np.random.default_rng(8)
    files = {}
    rgbe = rng.integers(0, 256, (7, 50, 4), dtype=np.uint8)
    rgbe[1, 3:40] = [200, 100, 50, 140]
    rgbe[5, :, 3] = 0
    files["rle"] = make_file(rgbe)
    files["flat_wide"] = make_file(rgbe, rle=False)
    files["small"] = make_file(rng.integers(0, 256, (4, 6, 4), dtype=np.uint8), rle=False)
    files["truncated"] = make_file(rgbe, rle=False)[:-300]
    px = np.abs(special_values(rng, (9, 33, 4)))
    ctx.hdr_write(str(tmp_path / "own"), 33, 9, 4, pixels_host=px)
    files["own"] = open(str(tmp_path / "own.hdr"), "rb").read()
    for name, data in files.items():
        path = tmp_path / (name + ".hdr")
        path.write_bytes(data)
        code, w, h, q = oracle.hdr_parse(data)
        assert code == 0, name
        want = oracle.rgbe_decode(q.reshape(-1, 4)).reshape(h, w, 4)
        host = np.zeros((h, w, 4), np.float32)
        dev = torch.zeros((h, w, 4), device="cuda")
        ctx.hdr_read(str(path), rgba_host=host, rgba_device_ptr=dev.data_ptr())
        same_bits(host, want)
        same_bits(dev.cpu().numpy(), want)
    bad = tmp_path / "bad.hdr"
    bad.write_bytes(header(50, 7) + bytes([2, 2, 0, 50, 0]) + bytes(100))  # a zero packet count
    assert oracle.hdr_parse(bad.read_bytes())[0] != 0
    with pytest.raises(native.NovaError) as e:
        ctx.hdr_read(str(bad), rgba_host=np.zeros(7 * 50 * 4, np.float32))
    assert e.value.status == 15
    with pytest.raises(native.NovaError):
        ctx.hdr_read(str(tmp_path / "rle.hdr"), rgba_host=np.zeros(100, np.float32), capacity=100)


def test_bake_cli_matches_oracle(oracle, torch_cuda, tmp_path):
    """nova_b200_bake reads the map, bakes on the GPU and writes the .hdr; the oracle decodes the
    input file, bakes it on the CPU and encodes the result: the two files' pixels agree within one
    RGBE mantissa step (the two bakes agree to 1e-4 before encoding)."""
    rng = np.random.default_rng(12)
    env = np.concatenate([rng.lognormal(0, 1, (64, 128, 3)), np.ones((64, 128, 1))], -1).astype(np.float32)
    src = tmp_path / "env.hdr"
    src.write_bytes(make_file(oracle.rgbe_encode(env, 4).reshape(64, 128, 4)))
    exe = os.path.join(ROOT, "axomae_b200", "nova_b200_bake")
    r = subprocess.run([exe, "--bake", "irradiance", "32", "16", "64", str(src), str(tmp_path / "irr")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    code, w, h, q = oracle.hdr_parse((tmp_path / "irr.hdr").read_bytes())
    assert (code, w, h) == (0, 32, 16)
    got = oracle.rgbe_decode(q.reshape(-1, 4)).reshape(h, w, 4)
    _, _, _, qin = oracle.hdr_parse(src.read_bytes())
    env_dec = oracle.rgbe_decode(qin.reshape(-1, 4)).reshape(64, 128, 4)
    ref = oracle.bake_irradiance(env_dec, 32, 16, 64)
    ref_q = oracle.rgbe_encode(ref, 4).reshape(h, w, 4)
    step = np.ldexp(1.0, ref_q[..., 3].astype(np.int32) - 136)[..., None]
    assert np.all(np.abs(got[..., :3] - ref[..., :3]) <= 2 * step)
    assert np.mean(np.all(q.reshape(h, w, 4) == ref_q, -1)) > 0.95
    r = subprocess.run([exe, "--bake", "irradiance", "30", "16", "64", str(src), str(tmp_path / "bad")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "power of two" in r.stderr
    r = subprocess.run([exe, "--bake", "irradiance", "32", "16", "64", str(tmp_path / "none.hdr"),
                        str(tmp_path / "bad")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_bake_cli_gpu_flag_uses_the_cuda_kernel(oracle, torch_cuda, tmp_path):
    """nova_b200_bake --gpu bakes with the reference's CUDA kernel, as the reference's --gpu option
    selects it (ProgramOptionsManager.cpp:39-40): the file agrees with the oracle's restatement of that
    kernel within the RGBE encoding and the texture filter's tolerance, and differs from the CPU-path
    bake of the same map."""
    rng = np.random.default_rng(14)
    env = np.concatenate([rng.lognormal(0, 1, (64, 128, 3)), np.ones((64, 128, 1))], -1).astype(np.float32)
    src = tmp_path / "env.hdr"
    src.write_bytes(make_file(oracle.rgbe_encode(env, 4).reshape(64, 128, 4)))
    exe = os.path.join(ROOT, "axomae_b200", "nova_b200_bake")
    r = subprocess.run([exe, "--bake", "irradiance", "32", "16", "64", str(src), str(tmp_path / "irr"), "--gpu"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    code, w, h, q = oracle.hdr_parse((tmp_path / "irr.hdr").read_bytes())
    assert (code, w, h) == (0, 32, 16)
    got = oracle.rgbe_decode(q.reshape(-1, 4)).reshape(h, w, 4)
    _, _, _, qin = oracle.hdr_parse(src.read_bytes())
    env_dec = oracle.rgbe_decode(qin.reshape(-1, 4)).reshape(64, 128, 4)
    ref = oracle.bake_irradiance_texunit(env_dec, 32, 16, 64)
    d = (got[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
    assert float(np.sqrt(np.mean(d * d))) <= 1e-2
    cpu = oracle.bake_irradiance(env_dec, 32, 16, 64)
    d2 = (got[..., :3].astype(np.float64) - cpu[..., :3]) / np.maximum(cpu[..., :3], 1e-3)
    assert float(np.sqrt(np.mean(d2 * d2))) > 2e-2
