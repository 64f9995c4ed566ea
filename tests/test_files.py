"""Asset and image files of the small_pt task, checked on the CPU:

  * OpenEXR: the interval images (composite_and_save_to_exr, render_target.cpp:181-208, through
    save_to_exr, image_util.cpp:101-190) read back bit-exactly by OpenCV's OpenEXR reader, FP32
    and FP16 (rounded to nearest even); the reader takes OpenCV's NONE / RLE / ZIPS / ZIP files,
    FP32 and FP16, and reports PIZ as unsupported;
  * Radiance .hdr sky maps (SkyLight through stb_image, light.cpp:19-31): the same floats as
    OpenCV's RGBE decoder;
  * mesh assets (create_mesh_asset, mesh_asset.cpp:243-266): OBJ with texcoords and normals, the
    binary mesh asset (load_from_binary / write_to_binary, mesh_asset.cpp:180-240) through the
    convert_mesh_asset task (mesh_asset.cpp:301-311), the to_world transform
    (MeshData::transform, geometry.cpp:15-32).  The binary files are parsed here by a reader that
    follows load_from_binary's read order.
"""
import os
import struct

import numpy as np
import pytest

os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")


def _ks():
    import keepsake_b200 as ks
    return ks


def _cv2():
    cv2 = pytest.importorskip("cv2")
    return cv2


def _pixels(h=37, w=53, c=3, seed=0):
    rng = np.random.default_rng(seed)
    a = (rng.random((h, w, c)) * 10).astype(np.float32)
    a[0, 0, :min(c, 3)] = [0.0, 1e-8, 65504.0][:min(c, 3)]
    return a


@pytest.mark.parametrize("half", [False, True])
def test_exr_written_reads_back_in_opencv(tmp_path, half):
    ks, cv2 = _ks(), _cv2()
    a = _pixels()
    f = tmp_path / "a.exr"
    ks.save_exr(f, a, half=half)
    b = cv2.imread(str(f), cv2.IMREAD_UNCHANGED)
    assert b is not None and b.dtype == np.float32 and b.shape == a.shape
    want = a.astype(np.float16).astype(np.float32) if half else a
    assert np.array_equal(b[:, :, ::-1], want)  # OpenCV returns B, G, R
    assert np.array_equal(ks.load_image(f), want)


@pytest.mark.parametrize("channels", [1, 2, 4])
def test_exr_channel_counts(tmp_path, channels):
    """save_to_exr's channel sets: R; G, R; A, B, G, R (sorted by name in the file)."""
    ks, cv2 = _ks(), _cv2()
    a = _pixels(c=channels, seed=channels)
    f = tmp_path / "c.exr"
    ks.save_exr(f, a)
    raw = f.read_bytes()
    names = {1: [b"R"], 2: [b"G", b"R"], 4: [b"A", b"B", b"G", b"R"]}[channels]
    chl = raw[raw.index(b"channels\0chlist\0") + 16 + 4:]
    for n in names:
        assert chl.startswith(n + b"\0")
        chl = chl[len(n) + 1 + 16:]
    assert chl[0] == 0
    b = cv2.imread(str(f), cv2.IMREAD_UNCHANGED)
    if channels == 1:
        # OpenCV puts a lone R channel in red; load_from_exr (tinyexr) reads one channel as grey
        assert np.array_equal(b[:, :, 2], a[:, :, 0]) and not b[:, :, :2].any()
        assert np.array_equal(ks.load_image(f), np.repeat(a, 3, axis=2))
    elif channels == 4:
        assert np.array_equal(b, a[:, :, [2, 1, 0, 3]])  # B, G, R, A
        assert np.array_equal(ks.load_image(f), a[:, :, :3])


@pytest.mark.parametrize("comp", ["NO", "RLE", "ZIPS", "ZIP"])
@pytest.mark.parametrize("half", [False, True])
def test_exr_reader_on_opencv_files(tmp_path, comp, half):
    ks, cv2 = _ks(), _cv2()
    a = _pixels(h=41, w=29, seed=3)
    a[5:9, :, :] = 1.0  # runs for RLE
    f = tmp_path / "o.exr"
    flags = [cv2.IMWRITE_EXR_COMPRESSION, getattr(cv2, "IMWRITE_EXR_COMPRESSION_" + comp)]
    if half:
        flags += [cv2.IMWRITE_EXR_TYPE, cv2.IMWRITE_EXR_TYPE_HALF]
    assert cv2.imwrite(str(f), a[:, :, ::-1], flags)
    want = a.astype(np.float16).astype(np.float32) if half else a
    assert np.array_equal(ks.load_image(f), want)


def test_exr_unsupported_and_bad_files(tmp_path):
    ks, cv2 = _ks(), _cv2()
    f = tmp_path / "p.exr"
    cv2.imwrite(str(f), _pixels()[:, :, ::-1], [cv2.IMWRITE_EXR_COMPRESSION, cv2.IMWRITE_EXR_COMPRESSION_PIZ])
    with pytest.raises(ks.KsError) as e:
        ks.load_image(f)
    assert e.value.status == 7 and "compression 4" in str(e.value)
    g = tmp_path / "bad.exr"
    g.write_bytes(b"\x76\x2f\x31\x01" + b"\x02\0\0\0" + b"chan")
    with pytest.raises(ks.KsError) as e:
        ks.load_image(g)
    assert e.value.status == 9
    with pytest.raises(ks.KsError) as e:
        ks.load_image(tmp_path / "missing.exr")
    assert e.value.status == 9
    with pytest.raises(ks.KsError) as e:
        ks.load_image(tmp_path / "x.png")
    assert e.value.status == 7


def test_half_rounding_is_nearest_even(tmp_path):
    """Every finite half, the midpoints between neighbours (ties round to even), values past the
    largest half and below the smallest subnormal: the FP16 file holds numpy's float16 rounding."""
    ks = _ks()
    h = np.arange(0, 0x7c00, dtype=np.uint16).view(np.float16).astype(np.float64)
    mids = (h[:-1] + h[1:]) / 2.0
    vals = np.concatenate([h, mids, np.nextafter(mids, 0), np.nextafter(mids, 1e9), [65519.99, 65520.0, 7e4],
                           [2.0 ** -25, 2.0 ** -25 * 1.0000001, 2.0 ** -26]]).astype(np.float32)
    vals = np.concatenate([vals, -vals])
    n = len(vals)
    w = 256
    rows = -(-n // w)
    a = np.zeros(rows * w, np.float32)
    a[:n] = vals
    f = tmp_path / "h.exr"
    ks.save_exr(f, a.reshape(rows, w, 1), half=True)
    got = ks.load_image(f)[:, :, 0].reshape(-1)[:n]
    with np.errstate(over="ignore"):
        want = vals.astype(np.float16).astype(np.float32)
    assert np.array_equal(got, want)


def test_hdr_reader_matches_opencv(tmp_path):
    ks, cv2 = _ks(), _cv2()
    a = _pixels(h=19, w=70, seed=5)  # >= 8 wide: run-length scanlines
    f = tmp_path / "s.hdr"
    assert cv2.imwrite(str(f), a[:, :, ::-1])
    b = cv2.imread(str(f), cv2.IMREAD_UNCHANGED)[:, :, ::-1]
    got = ks.load_image(f)
    assert np.array_equal(got, b)
    # RGBE keeps 8 bits of mantissa relative to a pixel's largest component
    assert (np.abs(got - a) <= a.max(axis=2, keepdims=True) / 128.0).all()
    # flat (uncompressed) scanlines: 4-wide image written by hand
    rgbe = np.array([[[128, 64, 32, 129], [0, 0, 0, 0], [255, 255, 255, 136], [1, 2, 3, 100]]], np.uint8)
    g = tmp_path / "flat.hdr"
    g.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 1 +X 4\n" + rgbe.tobytes())
    e = rgbe[..., 3].astype(np.int32)
    want = np.where(e[..., None] > 0, rgbe[..., :3] * np.ldexp(1.0, e - 136)[..., None], 0.0).astype(np.float32)
    assert np.array_equal(ks.load_image(g), want)


# ---- mesh assets ---------------------------------------------------------------------------
OBJ = """# two shapes: a textured quad with normals, a plain triangle
o quad
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
f 1/1/1 2/2/1 3/3/1 4/4/1
o tri
v 2 0 0
v 3 0 0
v 2 1 0
f -3 -2 -1
"""


def read_bin(path):
    """load_from_binary's read order (mesh_asset.cpp:182-218)."""
    b = open(path, "rb").read()
    assert b[:24] == b"i_am_a_binary_mesh_asset"
    p = 24
    (n,) = struct.unpack_from("<i", b, p)
    p += 4
    out = []
    for _ in range(n):
        twosided, smooth, nv, nt, has_tc, has_n = struct.unpack_from("<??ii??", b, p)
        p += 12
        m = dict(twosided=twosided, smooth=smooth)
        m["vertices"] = np.frombuffer(b, np.float32, 3 * nv + 1, p)
        p += 4 * (3 * nv + 1)
        m["indices"] = np.frombuffer(b, np.uint32, 3 * nt, p).reshape(-1, 3)
        p += 4 * 3 * nt
        if has_tc:
            m["texcoords"] = np.frombuffer(b, np.float32, 2 * nv + 2, p)
            p += 4 * (2 * nv + 2)
        if has_n:
            m["normals"] = np.frombuffer(b, np.float32, 3 * nv + 1, p)
            p += 4 * (3 * nv + 1)
        out.append(m)
    assert p == len(b)
    return out


def _convert(tmp_path, asset_toml, name="m"):
    ks = _ks()
    doc = asset_toml + f'\n[[task]]\ntype = "convert_mesh_asset"\ntask_dir = "conv"\nassets = ["mesh_asset.{name}"]\n'
    ks.config_run(doc, str(tmp_path / "out"), str(tmp_path))
    return tmp_path / "out" / "conv" / f"{name}.bin"


def test_obj_to_binary_mesh_asset(tmp_path):
    (tmp_path / "a.obj").write_text(OBJ)
    f = _convert(tmp_path, '[mesh_asset.m]\npath = "a.obj"\n')
    quad, tri = read_bin(f)
    # create_mesh_asset's OBJ defaults: one-sided, smooth normals
    assert not quad["twosided"] and quad["smooth"] and not tri["twosided"]
    assert np.array_equal(quad["vertices"][:-1].reshape(-1, 3), [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]])
    assert np.isnan(quad["vertices"][-1])
    assert np.array_equal(quad["indices"], [[0, 1, 2], [0, 2, 3]])  # the quad fanned
    assert np.array_equal(quad["texcoords"][:-2].reshape(-1, 2), [[0, 0], [1, 0], [1, 1], [0, 1]])
    assert np.array_equal(quad["normals"][:-1].reshape(-1, 3), [[0, 0, 1]] * 4)
    assert np.array_equal(tri["vertices"][:-1].reshape(-1, 3), [[2, 0, 0], [3, 0, 0], [2, 1, 0]])
    assert "texcoords" not in tri and "normals" not in tri
    # flags from the asset table
    f2 = _convert(tmp_path, '[mesh_asset.m]\npath = "a.obj"\ntwosided = true\nuse_smooth_normal = false\n')
    q2, _ = read_bin(f2)
    assert q2["twosided"] and not q2["smooth"]


def test_obj_vertices_split_by_attribute_triples(tmp_path):
    """A position used with two different texcoords becomes two vertices (tinyobj's index triple)."""
    (tmp_path / "s.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvt 0.5 0.5\n"
                                    "f 1/1 2/2 3/3\nf 1/4 3/3 2/2\n")
    (m,) = read_bin(_convert(tmp_path, '[mesh_asset.m]\npath = "s.obj"\n'))
    v = m["vertices"][:-1].reshape(-1, 3)
    assert len(v) == 4 and np.array_equal(v[3], [0, 0, 0])
    assert np.array_equal(m["indices"], [[0, 1, 2], [3, 2, 1]])


def test_binary_asset_round_trip_and_to_world(tmp_path):
    (tmp_path / "a.obj").write_text(OBJ)
    first = _convert(tmp_path, '[mesh_asset.m]\npath = "a.obj"\ntwosided = true\n').read_bytes()
    (tmp_path / "m.bin").write_bytes(first)
    again = _convert(tmp_path, '[mesh_asset.m]\npath = "m.bin"\nformat = "bin"\n')
    assert again.read_bytes() == first
    # to_world: points through the affine map, normals through its inverse transpose, normalised
    moved = _convert(tmp_path, '[mesh_asset.m]\npath = "m.bin"\nformat = "bin"\n'
                               'to_world = { scale = [2.0, 1.0, 0.5], translation = [1.0, 2.0, 3.0] }\n')
    quad, tri = read_bin(moved)
    v0 = read_bin(tmp_path / "m.bin")[0]["vertices"][:-1].reshape(-1, 3)
    assert np.allclose(quad["vertices"][:-1].reshape(-1, 3), v0 * [2.0, 1.0, 0.5] + [1.0, 2.0, 3.0])
    assert np.allclose(quad["normals"][:-1].reshape(-1, 3), [[0, 0, 1]] * 4)
    (tmp_path / "n.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 1 1 0\nf 1//1 2//1 3//1\n")
    (m,) = read_bin(_convert(tmp_path, '[mesh_asset.m]\npath = "n.obj"\nto_world = { scale = [2.0, 1.0, 1.0] }\n'))
    n = np.array([0.5, 1.0, 0.0]) / np.linalg.norm([0.5, 1.0, 0.0])
    assert np.allclose(m["normals"][:-1].reshape(-1, 3), [n] * 3, atol=1e-6)


def test_mesh_asset_errors(tmp_path):
    ks = _ks()
    (tmp_path / "bad.bin").write_bytes(b"not_a_binary_mesh_asset_at_all")
    with pytest.raises(ks.KsError) as e:
        _convert(tmp_path, '[mesh_asset.m]\npath = "bad.bin"\nformat = "bin"\n')
    assert e.value.status == 9 and "invalid binary mesh asset" in str(e.value)
    (tmp_path / "a.obj").write_text(OBJ)
    with pytest.raises(ks.KsError) as e:
        _convert(tmp_path, '[mesh_asset.m]\npath = "a.obj"\nload_materials = true\n')
    assert e.value.status == 7
    with pytest.raises(ks.KsError) as e:
        _convert(tmp_path, '[mesh_asset.m]\npath = "a.obj"\nformat = "ply"\n')
    assert e.value.status == 7
    (tmp_path / "mixed.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/1 2/1 3/1\nf 1 2 3\n")
    with pytest.raises(ks.KsError) as e:
        _convert(tmp_path, '[mesh_asset.m]\npath = "mixed.obj"\n')
    assert e.value.status == 9 and "texcoords" in str(e.value)
