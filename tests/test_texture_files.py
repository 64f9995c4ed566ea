"""Texture files and the loaders that bind them: PNG decoding and channel conversion
(create_texture_from_image, texture.cpp:922-944, through stb_image; glTF images through tinygltf,
create_texture_from_gltf, mesh_asset.cpp:370-388), float textures from .exr / .hdr
(load_from_exr / load_from_hdr, image_util.cpp:54-100), glTF material textures
(mesh_asset.cpp:694-950) and the TOML task's texture shader fields and normal maps
(create_texture_shader_field_color, shader_field.h:107-156; create_texture_sampler,
texture.cpp:1086-1121; create_normal_map, normal_map.cpp:40-55).

The PNG files are written here from the PNG specification (all colour types and bit depths,
every scanline filter, Adam7 interlacing, palette and colour-key transparency) and by OpenCV; the
expected samples are the ones written, converted with stb_image's published rules in numpy."""
import base64
import json
import struct
import zlib

import numpy as np
import pytest

from imaging import composite


def _ks():
    import keepsake_b200 as ks
    return ks


# ---- a PNG writer (ISO/IEC 15948) ------------------------------------------------------------
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def _chunk(t, body):
    return struct.pack(">I", len(body)) + t + body + struct.pack(">I", zlib.crc32(t + body) & 0xFFFFFFFF)


def _pack_rows(samples, depth):
    """samples [h, w, c] (ints) -> list of raw scanline bytes at `depth` bits per sample."""
    rows = []
    for r in samples:
        flat = r.reshape(-1).astype(np.int64)
        if depth == 16:
            rows.append(b"".join(struct.pack(">H", int(v)) for v in flat))
        elif depth == 8:
            rows.append(bytes(int(v) for v in flat))
        else:
            bits = "".join(format(int(v), "0%db" % depth) for v in flat)
            bits += "0" * (-len(bits) % 8)
            rows.append(bytes(int(bits[i:i + 8], 2) for i in range(0, len(bits), 8)))
    return rows


def _filter_rows(rows, bpp, first_filter):
    out, prev = b"", bytes(len(rows[0])) if rows else b""
    for k, row in enumerate(rows):
        t = (first_filter + k) % 5
        f = bytearray(len(row))
        for i in range(len(row)):
            a = row[i - bpp] if i >= bpp else 0
            b = prev[i]
            c = prev[i - bpp] if i >= bpp else 0
            if t == 0:
                p = 0
            elif t == 1:
                p = a
            elif t == 2:
                p = b
            elif t == 3:
                p = (a + b) >> 1
            else:
                pp = a + b - c
                pa, pb, pc = abs(pp - a), abs(pp - b), abs(pp - c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            f[i] = (row[i] - p) & 0xFF
        out += bytes([t]) + bytes(f)
        prev = row
    return out


def write_png(path, samples, color, depth, interlace=False, palette=None, trns=None):
    """samples [h, w, c] as stored (palette indices for colour type 3)."""
    h, w, c = samples.shape
    bpp = max(1, c * depth // 8)
    raw = b""
    if interlace:
        for k, (x0, y0, dx, dy) in enumerate(ADAM7):
            sub = samples[y0::dy, x0::dx]
            if sub.size:
                raw += _filter_rows(_pack_rows(sub, depth), bpp, k)
    else:
        raw = _filter_rows(_pack_rows(samples, depth), bpp, 0)
    data = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color, 0, 0, int(interlace)))
    if palette is not None:
        data += _chunk(b"PLTE", bytes(np.asarray(palette, np.uint8).reshape(-1)))
    if trns is not None:
        data += _chunk(b"tRNS", bytes(trns))
    data += _chunk(b"tEXt", b"Comment\x00ancillary chunks are skipped")
    # two IDAT chunks: the zlib stream is their concatenation
    z = zlib.compress(raw, 6)
    data += _chunk(b"IDAT", z[:len(z) // 2]) + _chunk(b"IDAT", z[len(z) // 2:]) + _chunk(b"IEND", b"")
    path.write_bytes(data)
    return data


CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


@pytest.mark.parametrize("color,depth,interlace", [
    (0, 1, False), (0, 2, True), (0, 4, False), (0, 8, True), (0, 16, False),
    (2, 8, False), (2, 16, True), (3, 1, True), (3, 4, False), (3, 8, False),
    (4, 8, True), (4, 16, False), (6, 8, False), (6, 16, True)])
def test_png_decoding(tmp_path, color, depth, interlace):
    ks = _ks()
    rng = np.random.default_rng(color * 100 + depth + 7 * interlace)
    h, w = 13, 11
    c = CHANNELS[color]
    if color == 3:
        n_pal = min(1 << depth, 40)
        pal = rng.integers(0, 256, (n_pal, 3))
        idx = rng.integers(0, n_pal, (h, w, 1))
        write_png(tmp_path / "p.png", idx, 3, depth, interlace, palette=pal)
        want = pal[idx[..., 0]]
    else:
        s = rng.integers(0, 1 << depth, (h, w, c))
        write_png(tmp_path / "p.png", s, color, depth, interlace)
        want = s * (255 // ((1 << depth) - 1)) if depth < 8 else s
    nat = 3 if color == 3 else c
    keep16 = depth == 16
    got, srgb = ks.load_texture(tmp_path / "p.png", nat, keep_16bit=keep16)
    assert got.dtype == (np.uint16 if keep16 else np.uint8) and not srgb
    assert np.array_equal(got, want)
    if keep16:
        got8, _ = ks.load_texture(tmp_path / "p.png", nat)
        assert np.array_equal(got8, want >> 8)


def test_png_transparency(tmp_path):
    """tRNS: palette alpha entries (RGBA), and a grey / RGB colour key (an alpha channel, 0 where the
    pixel equals the key)."""
    ks = _ks()
    rng = np.random.default_rng(3)
    pal = rng.integers(0, 256, (6, 3))
    idx = rng.integers(0, 6, (9, 10, 1))
    write_png(tmp_path / "a.png", idx, 3, 8, palette=pal, trns=[10, 200, 0])
    got, _ = ks.load_texture(tmp_path / "a.png", 4)
    alpha = np.array([10, 200, 0, 255, 255, 255])[idx[..., 0]]
    assert np.array_equal(got, np.concatenate([pal[idx[..., 0]], alpha[..., None]], -1))
    s = rng.integers(0, 4, (9, 10, 3))
    write_png(tmp_path / "k.png", s, 2, 8, trns=struct.pack(">HHH", 1, 2, 3))
    got, _ = ks.load_texture(tmp_path / "k.png", 4)
    key = (s == [1, 2, 3]).all(-1)
    assert np.array_equal(got[..., :3], s) and np.array_equal(got[..., 3], np.where(key, 0, 255))
    g = rng.integers(0, 4, (9, 10, 1)) * 85
    write_png(tmp_path / "g.png", g // 85, 0, 2, trns=struct.pack(">H", 2))
    got, _ = ks.load_texture(tmp_path / "g.png", 2)
    assert np.array_equal(got[..., 0], g[..., 0]) and np.array_equal(got[..., 1], np.where(g[..., 0] == 170, 0, 255))


def _stb_convert(s, n, c, opaque):
    """stb_image's conversion of n-channel samples to c channels."""
    s = s.astype(np.int64)
    grey = s[..., 0] if n <= 2 else (s[..., 0] * 77 + s[..., 1] * 150 + s[..., 2] * 29) >> 8
    alpha = s[..., n - 1] if n in (2, 4) else np.full(s.shape[:2], opaque)
    if c == 1:
        return grey[..., None]
    if c == 2:
        return np.stack([grey, alpha], -1)
    rgb = np.repeat(s[..., :1], 3, -1) if n <= 2 else s[..., :3]
    return rgb if c == 3 else np.concatenate([rgb, alpha[..., None]], -1)


@pytest.mark.parametrize("color,depth", [(0, 8), (2, 8), (4, 16), (6, 8), (6, 16)])
def test_png_channel_conversion(tmp_path, color, depth):
    ks = _ks()
    rng = np.random.default_rng(color + depth)
    n = CHANNELS[color]
    s = rng.integers(0, 1 << depth, (7, 9, n))
    write_png(tmp_path / "c.png", s, color, depth)
    for c in (1, 2, 3, 4):
        got, _ = ks.load_texture(tmp_path / "c.png", c)
        assert np.array_equal(got, _stb_convert(s >> (depth - 8), n, c, 255)), c
        if depth == 16:
            got16, _ = ks.load_texture(tmp_path / "c.png", c, keep_16bit=True)
            assert np.array_equal(got16, _stb_convert(s, n, c, 65535)), c


def test_png_against_opencv(tmp_path):
    """PNG files written by OpenCV (its own zlib and filter choices) decode to OpenCV's samples."""
    cv2 = pytest.importorskip("cv2")
    ks = _ks()
    rng = np.random.default_rng(11)
    cases = [rng.integers(0, 256, (37, 29, 3), dtype=np.uint8), rng.integers(0, 65536, (21, 33, 4), dtype=np.uint16),
             rng.integers(0, 256, (17, 16), dtype=np.uint8)]
    for k, img in enumerate(cases):
        f = tmp_path / f"cv{k}.png"
        assert cv2.imwrite(str(f), img)
        back = cv2.imread(str(f), cv2.IMREAD_UNCHANGED)
        if back.ndim == 3:
            back = back[..., [2, 1, 0, 3][:back.shape[2]]]
        else:
            back = back[..., None]
        got, _ = ks.load_texture(f, back.shape[2], keep_16bit=True)
        assert np.array_equal(got, back), k


def test_png_errors(tmp_path):
    ks = _ks()
    (tmp_path / "x.png").write_bytes(b"\x89PNG\r\n\x1a\nnot really")
    with pytest.raises(ks.KsError) as e:
        ks.load_texture(tmp_path / "x.png", 3)
    assert e.value.status == 9
    data = bytearray(write_png(tmp_path / "ok.png", np.zeros((4, 4, 3), np.int64), 2, 8))
    (tmp_path / "t.png").write_bytes(bytes(data[:-30]))
    with pytest.raises(ks.KsError):
        ks.load_texture(tmp_path / "t.png", 3)
    (tmp_path / "a.jpg").write_bytes(b"\xff\xd8\xff\xe0")
    with pytest.raises(ks.KsError) as e:
        ks.load_texture(tmp_path / "a.jpg", 3)
    assert e.value.status == 7


def test_float_textures(tmp_path):
    """.exr: the first channels of R, G, B, A (A = 1 without it; a one-channel file in all four);
    .hdr: RGB, or the mean of R, G and B for one or two channels (then alpha 1)."""
    ks = _ks()
    rng = np.random.default_rng(2)
    rgba = rng.random((6, 5, 4)).astype(np.float32)
    ks.save_exr(tmp_path / "a.exr", rgba)
    for c in (1, 2, 3, 4):
        got, _ = ks.load_texture(tmp_path / "a.exr", c)
        assert got.dtype == np.float32 and np.array_equal(got, rgba[..., :c])
    ks.save_exr(tmp_path / "rgb.exr", rgba[..., :3])
    got, _ = ks.load_texture(tmp_path / "rgb.exr", 4, srgb=True)
    assert np.array_equal(got[..., :3], rgba[..., :3]) and (got[..., 3] == 1.0).all()
    ks.save_exr(tmp_path / "y.exr", rgba[..., :1])
    got, _ = ks.load_texture(tmp_path / "y.exr", 4)
    assert np.array_equal(got, np.repeat(rgba[..., :1], 4, -1))
    cv2 = pytest.importorskip("cv2")
    assert cv2.imwrite(str(tmp_path / "s.hdr"), (rgba[..., 2::-1] * 4.0).astype(np.float32))
    rgb = ks.load_image(tmp_path / "s.hdr")
    got, _ = ks.load_texture(tmp_path / "s.hdr", 3)
    assert np.array_equal(got, rgb)
    got, _ = ks.load_texture(tmp_path / "s.hdr", 2)
    assert np.array_equal(got[..., 0], (rgb[..., 0] + rgb[..., 1] + rgb[..., 2]) / np.float32(3.0))
    assert (got[..., 1] == 1.0).all()


# ---- glTF material textures --------------------------------------------------------------------
def _png_bytes(tmp_path, name, samples, color, depth=8):
    return write_png(tmp_path / name, samples, color, depth)


def _textured_document(tmp_path, alpha_mode="OPAQUE", min_filter=None, image_kind="png", emissive_tex=False):
    from test_gltf import _document
    doc, buf = _document()
    rng = np.random.default_rng(4)
    base = rng.integers(0, 256, (8, 8, 4))
    mr = rng.integers(0, 65536, (4, 4, 3))
    nrm = rng.integers(0, 256, (4, 4, 3))
    pngs = [_png_bytes(tmp_path, "base.png", base, 6), _png_bytes(tmp_path, "mr.png", mr, 2, 16),
            _png_bytes(tmp_path, "n.png", nrm, 2)]
    if image_kind == "jpeg":
        pngs[0] = b"\xff\xd8\xff\xe0" + b"\0" * 32
    # image 0 in a buffer view of a second buffer, image 1 as a data URI, image 2 a file
    doc["buffers"].append(dict(byteLength=len(pngs[0]),
                               uri="data:application/octet-stream;base64," + base64.b64encode(pngs[0]).decode()))
    doc["bufferViews"].append(dict(buffer=1, byteOffset=0, byteLength=len(pngs[0])))
    doc["images"] = [dict(bufferView=len(doc["bufferViews"]) - 1, mimeType="image/png"),
                     dict(uri="data:image/png;base64," + base64.b64encode(pngs[1]).decode()),
                     dict(uri="n.png")]
    sampler = dict(magFilter=9729)
    if min_filter is not None:
        sampler["minFilter"] = min_filter
    doc["samplers"] = [sampler]
    doc["textures"] = [dict(source=0, sampler=0), dict(source=1, sampler=0), dict(source=2)]
    m0 = doc["materials"][0]
    m0["pbrMetallicRoughness"]["baseColorTexture"] = dict(
        index=0, extensions=dict(KHR_texture_transform=dict(scale=[2.0, 3.0], offset=[0.25, -0.5])))
    m0["pbrMetallicRoughness"]["metallicRoughnessTexture"] = dict(index=1)
    m0["normalTexture"] = dict(index=2, scale=0.6)
    m0["alphaMode"] = alpha_mode
    if emissive_tex:
        doc["materials"][1]["emissiveTexture"] = dict(index=2)
    return doc, buf, base, mr, nrm


def test_gltf_material_textures(tmp_path):
    from test_gltf import write_glb
    ks = _ks()
    doc, buf, base, mr, nrm = _textured_document(tmp_path, alpha_mode="MASK")
    write_glb(tmp_path / "t.glb", doc, buf)
    g = ks.Generated.load_compound(tmp_path / "t.glb")
    # images in order of first use, four channels (16-bit kept), sRGB for the base colour only
    (t0, s0), (t1, s1), (t2, s2) = g.textures
    assert s0 and not s1 and not s2
    assert t0.dtype == np.uint8 and np.array_equal(t0, base)
    assert t1.dtype == np.uint16 and np.array_equal(t1[..., :3], mr) and (t1[..., 3] == 65535).all()
    assert t2.dtype == np.uint8 and np.array_equal(t2[..., :3], nrm) and (t2[..., 3] == 255).all()
    b = {(x.material, x.field): x for x in g.bindings}
    assert sorted(b) == [(0, 0), (0, 1), (0, 2), (0, 9), (0, 10)]
    bc, op, ro, me, nm = b[0, 0], b[0, 10], b[0, 1], b[0, 2], b[0, 9]
    assert bc.texture == 0 and list(bc.scale) == pytest.approx([0.9, 0.5, 0.25, 1.0])
    assert list(bc.uv_scale) == [2.0, 3.0] and list(bc.uv_offset) == [0.25, -0.5]
    assert bc.filter == 0 and bc.flip_v == 0 and bc.wrap_u == 0 and bc.wrap_v == 0
    assert op.texture == 0 and op.swizzle[0] == 3 and op.scale[0] == 1.0
    assert ro.texture == 1 and ro.swizzle[0] == 1 and ro.scale[0] == pytest.approx(0.3)
    assert me.texture == 1 and me.swizzle[0] == 2 and me.scale[0] == pytest.approx(0.2)
    assert nm.texture == 2 and nm.strength == pytest.approx(0.6) and nm.normal_space == 0 and nm.range01 == 1
    # a constant alpha (no base colour texture): a one-texel opacity texture scaled by the factor
    doc, buf, *_ = _textured_document(tmp_path, alpha_mode="BLEND")
    del doc["materials"][0]["pbrMetallicRoughness"]["baseColorTexture"]
    doc["materials"][0]["pbrMetallicRoughness"]["baseColorFactor"][3] = 0.4
    write_glb(tmp_path / "c.glb", doc, buf)
    g = ks.Generated.load_compound(tmp_path / "c.glb")
    op = [x for x in g.bindings if x.field == 10][0]
    t, _ = g.textures[op.texture]
    assert t.shape == (1, 1, 1) and t.dtype == np.float32 and t[0, 0, 0] == 1.0
    assert op.scale[0] == pytest.approx(0.4)
    # without materials the textures are not read
    g = ks.Generated.load_compound(tmp_path / "t.glb", load_materials=False)
    assert g.textures == [] and g.bindings == []


def test_gltf_emissive_texture(tmp_path):
    """An emitter's emissiveTexture becomes its emission (x emissive strength x emissiveFactor, sRGB
    image)."""
    from test_gltf import write_glb
    ks = _ks()
    doc, buf, *_ = _textured_document(tmp_path, emissive_tex=True)
    write_glb(tmp_path / "e.glb", doc, buf)
    g = ks.Generated.load_compound(tmp_path / "e.glb")
    em = [b for b in g.bindings if b.field == 11]
    assert len(em) == 1 and em[0].material == 1
    assert list(em[0].scale) == pytest.approx([4.0, 2.0, 1.0, 1.0])
    assert g.textures[em[0].texture][1]  # the normal-map image, now also an emissive one: sRGB
    assert g.materials[1].has_emission


@pytest.mark.parametrize("change", [dict(min_filter=9987), dict(image_kind="jpeg")])
def test_gltf_unsupported_textures(tmp_path, change):
    from test_gltf import write_glb
    ks = _ks()
    doc, buf, *_ = _textured_document(tmp_path, **change)
    write_glb(tmp_path / "u.glb", doc, buf)
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(tmp_path / "u.glb")
    assert e.value.status == 7


@pytest.mark.gpu
def test_gltf_textured_render_through_task(ctx, tmp_path):
    """A textured glTF asset renders the same through the TOML task (compound_object) and through
    ks_compound_asset_load + the C ABI; opacity maps in instanced scenes are refused."""
    from test_gltf import write_glb
    ks = _ks()
    doc, buf, *_ = _textured_document(tmp_path)
    write_glb(tmp_path / "t.glb", doc, buf)
    c2w = [1.0, 0.0, 0.0, 1.2, 0.0, 1.0, 0.0, 3.0, 0.0, 0.0, 1.0, 9.0, 0.0, 0.0, 0.0, 1.0]
    cfg = f"""
[compound_mesh_asset.t]
path = "t.glb"
load_materials = true

[[task]]
type = "small_pt_b200"
compound_object = "compound_mesh_asset.t"
sky = {{ ambient = [0.4, 0.5, 0.6] }}
bounces = 4
render_width = 40
render_height = 32
spp = 8
spp_prog_interval = 8
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = 40.0, aspect = 1.25 }}
"""
    ks.config_run(cfg, str(tmp_path / "out"), str(tmp_path))
    img = ks.load_image(tmp_path / "out" / "task_0" / "small_pt_spp8.exr")
    g = ks.Generated.load_compound(tmp_path / "t.glb")
    g.desc.contents.sky.kind = 1
    g.desc.contents.sky.ambient[:] = (0.4, 0.5, 0.6)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    vfov = np.float32(40.0) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.25)
    p = ks.SmallPTParams.make(render_width=40, render_height=32, spp=8, bounces=4, spp_prog_interval=8)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert ref.mean() > 0.0
    assert np.array_equal(img, ref)
    doc, buf, *_ = _textured_document(tmp_path, alpha_mode="MASK")
    write_glb(tmp_path / "m.glb", doc, buf)
    g = ks.Generated.load_compound(tmp_path / "m.glb")
    import ctypes
    h = ctypes.c_void_p()
    assert ks.lib.ks_scene_create(ctx.handle, g.desc, ctypes.byref(h)) == 7


# ---- the TOML task's texture fields -------------------------------------------------------------
@pytest.mark.gpu
def test_task_texture_fields_equal_c_abi(ctx, tmp_path):
    """Texture assets (PNG in sRGB, EXR), texture shader fields (nearest / linear / cubic lookups,
    wrap modes, flip_v, swizzle, uv transform, scale) and a normal-map asset through the TOML task
    render what the C ABI renders with the same textures and bindings."""
    ks = _ks()
    rng = np.random.default_rng(9)
    checker = ((np.add.outer(np.arange(16) // 4, np.arange(16) // 4) % 2) * 180 + 40).astype(np.int64)
    tex0 = np.stack([checker, 255 - checker, rng.integers(0, 256, (16, 16))], -1)
    write_png(tmp_path / "albedo.png", tex0, 2, 8)
    rough = rng.random((8, 8, 3)).astype(np.float32)
    ks.save_exr(tmp_path / "rough.exr", rough)
    nrm = np.stack([np.full((8, 8), 0.6), np.full((8, 8), 0.5), np.full((8, 8), 0.9)], -1).astype(np.float32)
    ks.save_exr(tmp_path / "nrm.exr", nrm)
    c2w = [1.0, 0.0, 0.0, 0.0, 0.0, 0.9578, 0.2873, 1.8, 0.0, -0.2873, 0.9578, 3.0, 0.0, 0.0, 0.0, 1.0]
    cfg = f"""
[texture.albedo]
path = "albedo.png"
channels = 3
build_mipmaps = false
colorspace = "sRGB"

[texture.rough]
path = "rough.exr"
channels = 3
build_mipmaps = false

[texture.nrm]
path = "nrm.exr"
channels = 3
build_mipmaps = true

[bsdf.floor]
type = "principled_bsdf"
basecolor = {{ type = "texture", map = "texture.albedo", sampler = {{ type = "linear", wrap_mode_u = "clamp" }}, uv_scale = [2.0, 1.5], uv_offset = [0.1, 0.0] }}
roughness = {{ type = "texture", map = "texture.rough", sampler = {{ type = "cubic", kernel = "catmull_rom" }}, swizzle = 1, scale = 0.8 }}
metallic = {{ type = "constant", value = 0.1 }}

[bsdf.lamp]
type = "lambertian"
albedo = {{ type = "constant", value = [0.3, 0.3, 0.3] }}

[bsdf.box]
type = "principled_brdf"
basecolor = {{ type = "texture", map = "texture.albedo", sampler = {{ type = "nearest" }}, flip_v = false, swizzle = [2, 1, 0] }}

[normal_map.bump]
map = {{ type = "texture", map = "texture.nrm", sampler = {{ type = "nearest" }} }}
strength = 0.7

[material.floor]
bsdf = "bsdf.floor"
normal_map = "normal_map.bump"

[material.lamp]
bsdf = "bsdf.lamp"
emission = [17.0, 12.0, 4.0]

[material.box]
bsdf = "bsdf.box"

[mesh_asset.trio]
type = "inline"
geometry = [
  {{ vertices = [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], indices = [[0, 2, 1], [0, 3, 2]], texcoords = [[0, 0], [1, 0], [1, 1], [0, 1]] }},
  {{ vertices = [[-0.3, 1.5, -0.3], [0.3, 1.5, -0.3], [0.3, 1.5, 0.3], [-0.3, 1.5, 0.3]], indices = [[0, 1, 2], [0, 2, 3]] }},
  {{ vertices = [[-0.2, 0.0, 0.0], [0.2, 0.0, 0.0], [0.0, 0.5, 0.1]], indices = [[0, 1, 2]] }},
]

[[task]]
type = "small_pt_b200"
object = "mesh_asset.trio"
material = [["material.floor", "material.lamp", "material.box"]]
sky = {{ ambient = [0.1, 0.2, 0.3] }}
bounces = 4
clamp_indirect = 0.0
render_width = 48
render_height = 32
spp = 8
spp_prog_interval = 8
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = 45.0, aspect = 1.5 }}
"""
    ks.config_run(cfg, str(tmp_path / "out"), str(tmp_path))
    img = ks.load_image(tmp_path / "out" / "task_0" / "small_pt_spp8.exr")

    def mat(**kw):
        m = ks.MaterialDesc()
        m.basecolor[:] = kw.pop("basecolor", (0.8, 0.8, 0.8))
        m.roughness, m.ior, m.specular_r0_mul, m.diffuse_trans_fwd, m.specular = 1.0, 1.5, 0.5, 0.5, 0.5
        for k, v in kw.items():
            setattr(m, k, v)
        return m
    mats = [mat(metallic=0.1, specular=0.0), mat(basecolor=(0.3, 0.3, 0.3), bsdf=2, has_emission=1, specular=0.0),
            mat(bsdf=1)]
    mats[1].emission[:] = (17.0, 12.0, 4.0)
    tc = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    meshes = [(np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float32), np.array([[0, 2, 1], [0, 3, 2]]), 0,
               {"texcoords": tc}),
              (np.array([[-0.3, 1.5, -0.3], [0.3, 1.5, -0.3], [0.3, 1.5, 0.3], [-0.3, 1.5, 0.3]], np.float32),
               np.array([[0, 1, 2], [0, 2, 3]]), 1),
              (np.array([[-0.2, 0, 0], [0.2, 0, 0], [0, 0.5, 0.1]], np.float32), np.array([[0, 1, 2]]), 2)]
    sky = ks.SkyDesc()
    sky.kind = 1
    sky.ambient[:] = (0.1, 0.2, 0.3)
    desc, keep = ks.scene_desc(meshes, mats, sky)
    B = ks.TextureBinding.make
    textures = [ks.load_texture(tmp_path / "albedo.png", 3, srgb=True), ks.load_texture(tmp_path / "rough.exr", 3),
                ks.load_texture(tmp_path / "nrm.exr", 3)]
    binds = [B(0, "basecolor", 0, filter=1, wrap_u=1, uv_scale=(2.0, 1.5), uv_offset=(0.1, 0.0)),
             B(0, "roughness", 1, filter=2, cubic_kernel=2, swizzle=(1, -1, -1, -1), scale=(0.8, 1, 1, 1)),
             B(0, "normal_map", 2, filter=0, strength=0.7),
             B(2, "basecolor", 0, filter=0, flip_v=0, swizzle=(2, 1, 0, -1))]
    keep2 = ks.attach_textures(desc, textures, binds)
    s = ks.Scene(ctx, desc, (keep, keep2))
    s.build_bvh()
    vfov = np.float32(45.0) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.5)
    p = ks.SmallPTParams.make(render_width=48, render_height=32, spp=8, bounces=4, clamp_indirect=0.0,
                              spp_prog_interval=8)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert ref.mean() > 0.0
    assert np.array_equal(img, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("field,status", [
    ('{ type = "texture", map = "texture.t", sampler = { type = "ewa" } }', 7),
    ('{ type = "texture", map = "texture.m", sampler = { type = "linear" } }', 7),
    ('{ type = "texture", map = "texture.missing", sampler = { type = "nearest" } }', 8),
])
def test_task_texture_field_errors(ctx, tmp_path, field, status):
    ks = _ks()
    write_png(tmp_path / "t.png", np.zeros((4, 4, 3), np.int64), 2, 8)
    cfg = f"""
[texture.t]
path = "t.png"
channels = 3
build_mipmaps = false

[texture.m]
path = "t.png"
channels = 3
build_mipmaps = true

[bsdf.b]
type = "principled_bsdf"
basecolor = {field}

[material.m]
bsdf = "bsdf.b"

[mesh_asset.q]
type = "inline"
geometry = [ {{ vertices = [[-1, 0, -1], [1, 0, -1], [1, 0, 1]], indices = [[0, 2, 1]] }} ]

[[task]]
type = "small_pt_b200"
object = "mesh_asset.q"
material = [["material.m"]]
sky = {{ ambient = [0.1, 0.2, 0.3] }}
render_width = 8
render_height = 8
spp = 1
camera = {{ type = "perspective", to_world = {{ matrix_rm = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 1.0, 3.0, 0.0, 0.0, 0.0, 1.0] }}, vfov = 45.0, aspect = 1.0 }}
"""
    with pytest.raises(ks.KsError) as e:
        ks.config_run(cfg, str(tmp_path / "out"), str(tmp_path))
    assert e.value.status == status, str(e.value)
