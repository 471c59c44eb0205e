"""Film outputs and the Radiance .hdr format on the CPU: the oracle (oracle/film_io.cpp) against
known answers of the RGBE format and hand-packed files, and the library's host-only header logic
(nova_b200_hdr_info) and bake command line against the oracle.  No GPU is used here.

The known answers follow from the format's definition (a pixel is 3 mantissa bytes and a shared
exponent byte: value = byte * 2^(e - 136); encoding takes m = max component, m = f 2^k with f in
[0.5, 1), scale = f * 256 / m, byte = trunc(c * scale), e = k + 128), as the reference's writer
(stbi_write_hdr in IO::Loader::writeHdr) and reader (stbi_loadf in IO::Loader::loadRadianceFile)
implement it.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle_binding as ob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header(w, h, first="#?RADIANCE", fmt="FORMAT=32-bit_rle_rgbe", extra=()):
    lines = [first] + list(extra) + ([fmt] if fmt else [])
    return ("\n".join(lines) + "\n\n-Y %d +X %d\n" % (h, w)).encode()


def pack_rle_row(row):
    """One run-length scanline (row: (w, 4) uint8): header, then per component greedy packets
    (runs of >= 3 equal bytes as run packets, other bytes as dumps).  Test-side packer."""
    w = row.shape[0]
    out = bytearray([2, 2, w >> 8, w & 255])
    for k in range(4):
        p = row[:, k].tolist()
        x = 0
        lit = []
        while x < w:
            r = x
            while r < w and p[r] == p[x] and r - x < 127:
                r += 1
            if r - x >= 3:
                while lit:
                    out += bytes([min(len(lit), 128)]) + bytes(lit[:128])
                    lit = lit[128:]
                out += bytes([128 + r - x, p[x]])
                x = r
            else:
                lit.append(p[x])
                x += 1
        while lit:
            out += bytes([min(len(lit), 128)]) + bytes(lit[:128])
            lit = lit[128:]
    return bytes(out)


def make_file(rgbe, rle=True, **kw):
    h, w, _ = rgbe.shape
    body = b"".join(pack_rle_row(rgbe[j]) for j in range(h)) if rle else rgbe.tobytes()
    return header(w, h, **kw) + body


def test_rgbe_known_answers(oracle):
    px = np.array([[1.0, 1.0, 1.0], [0.5, 0.25, 0.125], [0.999, 0.5, 0.0], [0, 0, 0], [1e-33, 0, 0],
                   [-1, -2, -3], [np.inf, 0, 0], [3.0, 1.0, 0.0], [2.0 ** 127, 1.0, 0.0]], np.float32)
    want = np.array([[128, 128, 128, 129], [128, 64, 32, 128], [255, 128, 0, 128], [0, 0, 0, 0], [0, 0, 0, 0],
                     [0, 0, 0, 0], [0, 0, 0, 128], [192, 64, 0, 130], [128, 0, 0, 0]], np.uint8)
    np.testing.assert_array_equal(ob.rgbe_encode(px, 3), want)
    # one and two channels: the first channel as grey
    np.testing.assert_array_equal(ob.rgbe_encode(np.array([0.5, 7.0], np.float32), 1),
                                  [[128, 128, 128, 128], [224, 224, 224, 131]])
    np.testing.assert_array_equal(ob.rgbe_encode(np.array([0.5, 9.0], np.float32), 2), [[128, 128, 128, 128]])
    dec = ob.rgbe_decode(np.array([[128, 128, 128, 129], [128, 64, 32, 128], [255, 1, 0, 128], [7, 7, 7, 0],
                                   [1, 0, 0, 1]], np.uint8))
    np.testing.assert_array_equal(dec, np.array([[1, 1, 1, 1], [0.5, 0.25, 0.125, 1], [255 / 256, 1 / 256, 0, 1],
                                                 [0, 0, 0, 1], [2.0 ** -135, 0, 0, 1]], np.float32))


def test_rgbe_round_trip_bounds(oracle):
    """decode(encode(x)) <= x and within one mantissa step (2^(e-136)) of x for non-negative x."""
    rng = np.random.default_rng(3)
    px = rng.lognormal(0, 4, (20000, 3)).astype(np.float32)
    q = ob.rgbe_encode(px, 3)
    dec = ob.rgbe_decode(q)[:, :3]
    step = np.ldexp(1.0, q[:, 3].astype(np.int32) - 136)[:, None]
    assert np.all(dec <= px) and np.all(px - dec < step)
    # the largest component keeps 8 significant bits: its byte is in [128, 255]
    assert np.all(q[:, :3].max(1) >= 128)


def test_hdr_parse_rle_and_flat(oracle):
    rng = np.random.default_rng(4)
    rgbe = rng.integers(0, 256, (6, 40, 4), dtype=np.uint8)
    rgbe[2, 5:30] = [9, 9, 9, 130]  # long runs in every plane
    rgbe[4, :, 3] = 129
    for rle in (True, False):
        code, w, h, got = ob.hdr_parse(make_file(rgbe, rle=rle))
        assert (code, w, h) == (0, 40, 6)
        np.testing.assert_array_equal(got, rgbe)
    # widths outside [8, 32768) are always flat
    small = rng.integers(0, 256, (3, 5, 4), dtype=np.uint8)
    code, w, h, got = ob.hdr_parse(make_file(small, rle=False, first="#?RADIANCE", extra=("# comment",)))
    assert (code, w, h) == (0, 5, 3)
    np.testing.assert_array_equal(got, small)


def test_hdr_parse_rules(oracle):
    rgbe = np.full((2, 8, 4), 128, np.uint8)
    ok = make_file(rgbe)
    assert ob.hdr_parse(ok)[0] == 0
    assert ob.hdr_parse(make_file(rgbe, first="#?RGBE"))[0] == 1  # the loader's magic check wants #?RADIANCE
    assert ob.hdr_parse(make_file(rgbe, first="#?RADIANCE x"))[0] == 1  # first line must be exact
    assert ob.hdr_parse(make_file(rgbe, fmt=None))[0] == 2
    assert ob.hdr_parse(make_file(rgbe, fmt="FORMAT=32-bit_rle_xyze"))[0] == 2
    assert ob.hdr_parse(b"\x76\x2f\x31\x01" + bytes(40))[0] == 6  # OpenEXR
    bad_res = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n+Y 2 +X 8\n" + bytes(64)
    assert ob.hdr_parse(bad_res)[0] == 3
    hdr = header(8, 2)
    assert ob.hdr_parse(hdr + bytes([2, 2, 0, 9]) + bytes(64))[0] == 4  # scanline length != width
    assert ob.hdr_parse(hdr + bytes([2, 2, 0, 8, 0]) + bytes(64))[0] == 5  # zero count
    assert ob.hdr_parse(hdr + bytes([2, 2, 0, 8, 128 + 9, 1]) + bytes(64))[0] == 5  # run past the row
    # a first row without a run-length header: the whole image is flat from there
    flat = np.arange(2 * 8 * 4, dtype=np.uint8).reshape(2, 8, 4)
    code, w, h, got = ob.hdr_parse(hdr + flat.tobytes())
    assert code == 0
    np.testing.assert_array_equal(got, flat)
    # reading past the end gives zeros
    code, w, h, got = ob.hdr_parse(hdr + flat.tobytes()[:20])
    assert code == 0 and got.reshape(-1)[20:].max() == 0


def test_snapshot_oracle_properties(oracle):
    rng = np.random.default_rng(5)
    film = rng.standard_normal((9, 13, 4)).astype(np.float32)
    same = ob.snapshot(film, 13, 9)
    np.testing.assert_array_equal(same[..., :3], film[..., :3])  # whole-pixel weights: a copy
    assert np.all(same[..., 3] == 0)  # channel 3 is never written
    down = ob.snapshot(film, 5, 4)
    for j in range(4):
        for i in range(5):
            x = int(np.float32(i / 5) * np.float32(13))
            y = int(np.float32(j / 4) * np.float32(9))
            np.testing.assert_array_equal(down[j, i, :3], film[y, x, :3])
    acc, final = ob.film_accumulate(np.ones(8, np.float32), np.full(8, 3.0, np.float32), 3)
    np.testing.assert_array_equal(acc, 4.0)
    np.testing.assert_array_equal(final, 1.0)
    np.testing.assert_allclose(ob.display_blend(np.full(4, 2.0, np.float32), np.full(4, 3.0, np.float32), 2),
                               1.0 + 0.8 * (2.0 - 1.0))


def test_hdr_info_header_logic(tmp_path):
    """nova_b200_hdr_info is host-only: same size and same accept / reject decisions as the oracle."""
    from axomae_b200 import native
    rgbe = np.full((3, 17, 4), 130, np.uint8)
    cases = {"ok": make_file(rgbe), "flat": make_file(rgbe, rle=False), "rgbe_magic": make_file(rgbe, first="#?RGBE"),
             "no_format": make_file(rgbe, fmt=None), "exr": b"\x76\x2f\x31\x01" + bytes(40),
             "bad_res": b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 3 -X 17\n",
             "long_header": make_file(rgbe, extra=["# " + "x" * 2000] * 80)}  # 160 KB of comment lines
    for name, data in cases.items():
        p = tmp_path / (name + ".hdr")
        p.write_bytes(data)
        code, w, h, _ = ob.hdr_parse(data)
        if code == 0:
            assert native.hdr_info(str(p)) == (w, h) == (17, 3)
        else:
            with pytest.raises(native.NovaError) as e:
                native.hdr_info(str(p))
            assert e.value.status == 15  # INVALID_ARGUMENT
    with pytest.raises(native.NovaError):
        native.hdr_info(str(tmp_path / "missing.hdr"))


def test_bake_cli_usage_errors():
    exe = os.path.join(ROOT, "axomae_b200", "nova_b200_bake")
    assert os.path.exists(exe), "build the library first (make -C axomae_b200/csrc)"
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "missing argument" in r.stderr
    r = subprocess.run([exe, "--bake", "irradiance", "32", "16"], capture_output=True, text=True)
    assert r.returncode == 1 and "missing argument" in r.stderr
    r = subprocess.run([exe, "--bake", "irradiance", "3x", "16", "8", "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1 and "integers" in r.stderr
    r = subprocess.run([exe, "--bake", "prefilter", "32", "16", "8", "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1 and "only \"irradiance\"" in r.stderr


def _rows_strategy():
    from hypothesis import strategies as st
    # rows built from runs: (length, value) pieces so long runs, short runs and literals all occur
    piece = st.tuples(st.integers(1, 140), st.integers(0, 255))
    return st.tuples(st.integers(8, 300), st.integers(1, 4), st.lists(piece, min_size=1, max_size=12),
                     st.integers(0, 2**32 - 1))


def test_hdr_rle_round_trip_fuzz(oracle):
    """Random run structures (runs up to 140 bytes, so past the 127-byte packet limit, literals,
    widths 8..300): the test-side packer's file parses back to the same pixels, flat files too,
    and the oracle's own writer emits files its parser reads back to the encoder's bytes."""
    from hypothesis import given, settings, HealthCheck

    @settings(max_examples=60, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(_rows_strategy())
    def check(case):
        w, h, pieces, seed = case
        rng = np.random.default_rng(seed)
        rgbe = np.zeros((h, w, 4), np.uint8)
        for j in range(h):
            for k in range(4):
                plane, x = [], 0
                order = rng.permutation(len(pieces))
                while len(plane) < w:
                    n, v = pieces[order[x % len(pieces)]]
                    plane += [v] * n if rng.random() < 0.7 else list(rng.integers(0, 256, n))
                    x += 1
                rgbe[j, :, k] = plane[:w]
        # a flat file's first pixel must not read as a run-length row header (2, 2, < 128): a
        # normalised RGBE pixel never does (its largest mantissa byte is >= 128)
        rgbe[0, 0, 0] = max(rgbe[0, 0, 0], 128)
        for rle in (True, False):
            code, gw, gh, got = ob.hdr_parse(make_file(rgbe, rle=rle))
            assert (code, gw, gh) == (0, w, h)
            np.testing.assert_array_equal(got, rgbe)

    check()


def test_hdr_writer_output_parses_back(oracle, tmp_path):
    rng = np.random.default_rng(9)
    for w, h in ((8, 3), (37, 5), (300, 2), (5, 4)):
        px = rng.lognormal(0.0, 2.0, (h, w, 4)).astype(np.float32)
        px[0, : w // 2] = 1.5  # a run
        base = str(tmp_path / ("img%dx%d" % (w, h)))
        ob.hdr_write(base, px, w, h, 4)
        data = open(base + ".hdr", "rb").read()
        code, gw, gh, got = ob.hdr_parse(data)
        assert (code, gw, gh) == (0, w, h)
        np.testing.assert_array_equal(got.reshape(-1, 4), ob.rgbe_encode(px, 4))


def test_hdr_info_header_fuzz(tmp_path):
    """Random headers (magic lines, extra lines, FORMAT lines, resolution strings with odd spacing,
    signs and sizes): the library's host-only header parse accepts exactly what the oracle's
    header rules accept, with the same size.  The body is valid, so only the header decides."""
    from hypothesis import given, settings, HealthCheck, strategies as st
    from axomae_b200 import native
    line = st.sampled_from(["# comment", "EXPOSURE=1.0", "GAMMA=2.2", "FORMAT=32-bit_rle_xyze", "", "x" * 300,
                            "FORMAT=32-bit_rle_rgbe"])
    size = st.one_of(st.integers(1, 64), st.integers(-2, 70000))
    res = st.tuples(st.sampled_from(["-Y", "-Y", "-Y", "+Y", "-X", "Y"]), size, st.sampled_from([" ", " ", "  ", ""]),
                    st.sampled_from(["+X", "+X", "-X", "X"]), size)
    lines = st.one_of(st.just(["FORMAT=32-bit_rle_rgbe"]), st.lists(line, max_size=5))
    case = st.tuples(st.sampled_from(["#?RADIANCE", "#?RADIANCE", "#?RGBE", "#?RADIANCE ", "#?radiance"]), lines, res)
    counter = [0]

    @settings(max_examples=120, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(case)
    def check(c):
        first, lines, (ys, h, sp, xs, w) = c
        head = (first + "\n" + "".join(l + "\n" for l in lines if l) + "\n" + "%s %d%s%s %d\n" % (ys, h, sp, xs, w))
        body = bytes(4 * 8 * 2)  # enough flat zeros for the smallest valid sizes; larger ones read zeros
        data = head.encode() + body
        small = w <= 64 and h <= 64  # the oracle decodes what it accepts: keep its images small
        code, ow, oh, _ = ob.hdr_parse(data) if small or "-Y" not in ys else (None, 0, 0, None)
        p = tmp_path / ("h%d.hdr" % counter[0])
        counter[0] += 1
        p.write_bytes(data)
        try:
            got = native.hdr_info(str(p))
        except native.NovaError as e:
            assert e.status == 15
            got = None
        if code is None:  # a large image: the oracle is not asked to decode it, only the header matters
            return
        assert (got is not None) == (code == 0), (head, code, got)
        if got is not None:
            assert got == (ow, oh)
            accepted[0] += 1
        else:
            rejected[0] += 1

    accepted, rejected = [0], [0]
    check()
    assert accepted[0] > 0 and rejected[0] > 0
