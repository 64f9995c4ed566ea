"""glTF 2.0 compound mesh assets (CompoundMeshAsset::load_from_gltf, mesh_asset.cpp:551-1091):
meshes -> prototypes (primitives -> meshes with normals and texcoords), nodes of the default
scene -> instances under their world transforms (traverse_gltf_scene_graph,
mesh_asset.cpp:466-520), metallic-roughness materials -> constant principled materials with the
reference's extension handling (emissive strength, ior, specular, transmission).

The files are written here from the glTF 2.0 specification (JSON + binary buffer, .glb container,
base64 data URIs, external buffers); the expected transforms and materials are computed in
numpy from the same numbers.
"""
import base64
import json
import struct

import numpy as np
import pytest


def _ks():
    import keepsake_b200 as ks
    return ks


def _quat_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _trs(t=(0, 0, 0), q=(0, 0, 0, 1), s=(1, 1, 1)):
    m = np.eye(4)
    m[:3, :3] = _quat_matrix(q) * np.asarray(s)[None, :]
    m[:3, 3] = t
    return m


QUAD_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
QUAD_N = np.array([[0, 0, 1], [0, 0.6, 0.8], [0, 0, 1], [0.6, 0, 0.8]], np.float32)
QUAD_T = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
QUAD_I = np.array([[0, 1, 2], [0, 2, 3]], np.uint16)
TRI_V = np.array([[0, 0, 0], [2, 0, 0], [0, 2, 0]], np.float32)
TRI_I = np.array([[0, 1, 2]], np.uint32)
ROOT_TRS = dict(t=(1.0, 2.0, 3.0), q=(0.0, np.sin(0.35), 0.0, np.cos(0.35)), s=(2.0, 2.0, 2.0))
A_MATRIX = _trs(t=(0.5, 0.0, -1.0), q=(np.sin(0.2), 0.0, 0.0, np.cos(0.2)), s=(1.0, 0.5, 1.5))
B_T = (0.0, 4.0, 0.0)


def _document(materials=True, extra_material=None, mode=None):
    """(gltf dict, binary buffer): the quad (interleaved POSITION / NORMAL / TEXCOORD_0 with a
    byte stride, uint16 indices), the triangle (uint32 indices), two materials, a node tree."""
    inter = np.zeros(4, dtype=[("p", "<f4", 3), ("n", "<f4", 3), ("t", "<f4", 2)])
    inter["p"], inter["n"], inter["t"] = QUAD_V, QUAD_N, QUAD_T
    parts = [inter.tobytes(), QUAD_I.tobytes() + b"\0\0", TRI_V.tobytes(), TRI_I.tobytes()]
    offs = np.cumsum([0] + [len(p) for p in parts])
    buf = b"".join(parts)
    views = [dict(buffer=0, byteOffset=int(offs[0]), byteLength=len(parts[0]), byteStride=32),
             dict(buffer=0, byteOffset=int(offs[1]), byteLength=12),
             dict(buffer=0, byteOffset=int(offs[2]), byteLength=len(parts[2])),
             dict(buffer=0, byteOffset=int(offs[3]), byteLength=len(parts[3]))]
    accs = [dict(bufferView=0, byteOffset=0, componentType=5126, count=4, type="VEC3"),
            dict(bufferView=0, byteOffset=12, componentType=5126, count=4, type="VEC3"),
            dict(bufferView=0, byteOffset=24, componentType=5126, count=4, type="VEC2"),
            dict(bufferView=1, componentType=5123, count=6, type="SCALAR"),
            dict(bufferView=2, componentType=5126, count=3, type="VEC3"),
            dict(bufferView=3, componentType=5125, count=3, type="SCALAR")]
    quad = dict(attributes=dict(POSITION=0, NORMAL=1, TEXCOORD_0=2), indices=3, material=0)
    if mode is not None:
        quad["mode"] = mode
    mats = [dict(pbrMetallicRoughness=dict(baseColorFactor=[0.9, 0.5, 0.25, 1.0], roughnessFactor=0.3,
                                           metallicFactor=0.2),
                 extensions=dict(KHR_materials_ior=dict(ior=1.33),
                                 KHR_materials_specular=dict(specularFactor=0.8, specularColorFactor=[1.0, 0.5, 0.0]))),
            dict(emissiveFactor=[1.0, 0.5, 0.25],
                 extensions=dict(KHR_materials_emissive_strength=dict(emissiveStrength=4.0),
                                 KHR_materials_transmission=dict(transmissionFactor=0.7)))]
    if extra_material:
        mats[0].update(extra_material)
    doc = dict(asset=dict(version="2.0"), buffers=[dict(byteLength=len(buf))], bufferViews=views, accessors=accs,
               meshes=[dict(name="quad", primitives=[quad]),
                       dict(name="tri", primitives=[dict(attributes=dict(POSITION=4), indices=5, material=1)])],
               nodes=[dict(translation=list(ROOT_TRS["t"]), rotation=list(ROOT_TRS["q"]), scale=list(ROOT_TRS["s"]),
                           children=[1, 2]),
                      dict(mesh=0, matrix=[float(x) for x in A_MATRIX.T.reshape(-1)]),
                      dict(mesh=1, translation=list(B_T)),
                      dict(mesh=0)],
               scenes=[dict(nodes=[3]), dict(nodes=[0, 3])], scene=1)
    if not materials:
        for m in doc["meshes"]:
            for p in m["primitives"]:
                del p["material"]
    else:
        doc["materials"] = mats
    return doc, buf


def write_glb(path, doc, buf):
    j = json.dumps(doc).encode()
    j += b" " * (-len(j) % 4)
    b = buf + b"\0" * (-len(buf) % 4)
    body = struct.pack("<II", len(j), 0x4E4F534A) + j + struct.pack("<II", len(b), 0x004E4942) + b
    path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)


def expected_instances():
    root = _trs(**ROOT_TRS)
    return [(0, root @ A_MATRIX), (1, root @ _trs(t=B_T)), (0, np.eye(4))]


def _check(g, materials=True):
    assert len(g.prototypes) == 2 and g.prototypes == [(0, 1), (1, 1)]
    quad, tri = g.meshes
    assert np.array_equal(quad["vertices"], QUAD_V) and np.array_equal(quad["indices"], QUAD_I)
    assert np.array_equal(quad["normals"], QUAD_N) and np.array_equal(quad["texcoords"], QUAD_T)
    assert np.array_equal(tri["vertices"], TRI_V) and np.array_equal(tri["indices"], TRI_I)
    assert tri["normals"] is None and tri["texcoords"] is None
    assert quad["twosided"] == 1 and quad["smooth"] == 1
    want = expected_instances()
    assert len(g.instances) == len(want)
    for (p, xf), (wp, wm) in zip(g.instances, want):
        assert p == wp
        assert np.allclose(xf, wm[:3, :], atol=1e-6), (xf, wm)
    if materials:
        m0, m1 = g.materials
        assert np.allclose(m0.basecolor[:], [0.9, 0.5, 0.25]) and np.isclose(m0.roughness, 0.3)
        assert np.isclose(m0.metallic, 0.2) and np.isclose(m0.ior, 1.33)
        assert np.isclose(m0.specular_r0_mul, 0.8 * 0.5) and m0.specular_trans == 0.0 and not m0.has_emission
        assert m0.diffuse_trans == 0.0 and m0.diffuse_trans_fwd == 0.0
        # glTF defaults: white, roughness 1, metallic 1; emission = strength x factor; transmission
        # makes the mesh one-sided
        assert np.allclose(m1.basecolor[:], [1, 1, 1]) and m1.roughness == 1.0 and m1.metallic == 1.0
        assert m1.has_emission and np.allclose(m1.emission[:], [4.0, 2.0, 1.0])
        assert np.isclose(m1.specular_trans, 0.7) and tri["twosided"] == 0
        assert np.isclose(m1.ior, 1.5) and np.isclose(m1.specular_r0_mul, 0.5)
        assert (quad["material"], tri["material"]) == (0, 1)
    else:
        assert g.materials == [] and tri["twosided"] == 1


def test_glb(tmp_path):
    ks = _ks()
    f = tmp_path / "a.glb"
    write_glb(f, *_document())
    g = ks.Generated.load_compound(f)
    _check(g)


def test_gltf_with_data_uri_and_external_buffer(tmp_path):
    ks = _ks()
    doc, buf = _document()
    doc["buffers"][0]["uri"] = "data:application/octet-stream;base64," + base64.b64encode(buf).decode()
    (tmp_path / "d.gltf").write_text(json.dumps(doc, indent=1))
    _check(ks.Generated.load_compound(tmp_path / "d.gltf"))
    doc["buffers"][0]["uri"] = "my%20data.bin"
    (tmp_path / "my data.bin").write_bytes(buf)
    (tmp_path / "e.gltf").write_text(json.dumps(doc))
    _check(ks.Generated.load_compound(tmp_path / "e.gltf"))


def test_without_materials(tmp_path):
    ks = _ks()
    f = tmp_path / "n.glb"
    write_glb(f, *_document(materials=False))
    _check(ks.Generated.load_compound(f, load_materials=False), materials=False)
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(f, load_materials=True)
    assert e.value.status == 7 and "material" in str(e.value)


@pytest.mark.parametrize("change,status", [
    # a texture index without a textures array (textured materials: tests/test_texture_files.py)
    (dict(extra_material=dict(pbrMetallicRoughness=dict(baseColorTexture=dict(index=0)))), 9),
    (dict(mode=1), 7),
])
def test_unsupported_features(tmp_path, change, status):
    ks = _ks()
    f = tmp_path / "u.glb"
    write_glb(f, *_document(**change))
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(f)
    assert e.value.status == status


def test_bad_files(tmp_path):
    ks = _ks()
    (tmp_path / "bad.gltf").write_text('{"asset": {"version": "2.0"}, "meshes": [}')
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(tmp_path / "bad.gltf")
    assert e.value.status == 9 and "JSON" in str(e.value)
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(tmp_path / "missing.glb")
    assert e.value.status == 9
    doc, buf = _document()
    doc["accessors"][0]["count"] = 40  # past the buffer view
    write_glb(tmp_path / "over.glb", doc, buf)
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(tmp_path / "over.glb")
    assert e.value.status == 9 and "past its buffer view" in str(e.value)
    doc, buf = _document()
    doc["nodes"][1]["children"] = [0]  # a cycle
    write_glb(tmp_path / "cycle.glb", doc, buf)
    with pytest.raises(ks.KsError) as e:
        ks.Generated.load_compound(tmp_path / "cycle.glb")
    assert "cycle" in str(e.value)


@pytest.mark.gpu
def test_compound_object_through_config_task(ctx, tmp_path):
    """The glTF scene through the TOML small_pt task (`compound_object`, materials from the file)
    renders the same image as the C ABI on the loaded description (two prototypes, three
    instances, an ambient sky and the emissive glTF primitive as a mesh light)."""
    from imaging import composite
    ks = _ks()
    f = tmp_path / "s.glb"
    write_glb(f, *_document())
    c2w = [1.0, 0.0, 0.0, 1.5, 0.0, 1.0, 0.0, 3.0, 0.0, 0.0, 1.0, 9.0, 0.0, 0.0, 0.0, 1.0]
    doc = f"""
[compound_mesh_asset.s]
path = "s.glb"
load_materials = true

[[task]]
type = "small_pt"
compound_object = "compound_mesh_asset.s"
sky = {{ ambient = [0.3, 0.3, 0.3] }}
bounces = 4
render_width = 40
render_height = 32
spp = 8
spp_prog_interval = 8
rng_seed = 4
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = 60.0, aspect = 1.25 }}
"""
    ks.config_run(doc, str(tmp_path / "out"), str(tmp_path))
    img = ks.load_image(tmp_path / "out" / "task_0" / "small_pt_spp8.exr")
    g = ks.Generated.load_compound(f)
    sky = g.desc.contents.sky
    sky.kind = 1
    sky.ambient[:] = [0.3, 0.3, 0.3]
    sky.to_world[:] = [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]
    sky.transform_y_up = 1
    sky.strength = 1.0
    g.desc.contents.sky = sky
    s = ks.Scene(ctx, g.desc, keepalive=g)
    s.build_bvh()
    vfov = np.float32(60.0) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.25)
    p = ks.SmallPTParams.make(render_width=40, render_height=32, spp=8, bounces=4, spp_prog_interval=8, rng_seed=4)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert img.mean() > 0.0
    assert np.array_equal(img, ref)


# ---- camera animation ----------------------------------------------------------------------
T_KEYS = np.array([0.0, 1.0, 2.5], np.float32)
T_VALS = np.array([[0, 1, 8], [1, 1, 7], [2, 2, 5]], np.float32)
R_KEYS = np.array([0.0, 2.5], np.float32)
R_VALS = np.array([[0, 0, 0, 1], [0, np.sin(0.3), 0, np.cos(0.3)]], np.float32)  # x y z w


def _anim_document(camera_type="perspective", with_anim=True):
    parts = [T_KEYS.tobytes(), T_VALS.tobytes(), R_KEYS.tobytes(), R_VALS.tobytes()]
    offs = np.cumsum([0] + [len(p) for p in parts])
    buf = b"".join(parts)
    views = [dict(buffer=0, byteOffset=int(offs[i]), byteLength=len(parts[i])) for i in range(4)]
    accs = [dict(bufferView=0, componentType=5126, count=3, type="SCALAR"),
            dict(bufferView=1, componentType=5126, count=3, type="VEC3"),
            dict(bufferView=2, componentType=5126, count=2, type="SCALAR"),
            dict(bufferView=3, componentType=5126, count=2, type="VEC4")]
    cam = dict(name="shot", type=camera_type)
    if camera_type == "perspective":
        cam["perspective"] = dict(yfov=0.8, aspectRatio=1.5, znear=0.1)
    else:
        cam["orthographic"] = dict(xmag=1, ymag=1, znear=0.1, zfar=10)
    doc = dict(asset=dict(version="2.0"), buffers=[dict(byteLength=len(buf))], bufferViews=views, accessors=accs,
               cameras=[dict(name="other", type="perspective", perspective=dict(yfov=1.0, aspectRatio=1.0,
                                                                                 znear=0.1)), cam],
               nodes=[dict(children=[1, 2]), dict(camera=0), dict(camera=1, translation=[9, 9, 9])],
               scenes=[dict(nodes=[0])])
    if with_anim:
        doc["animations"] = [dict(channels=[dict(sampler=0, target=dict(node=2, path="translation")),
                                            dict(sampler=1, target=dict(node=2, path="rotation"))],
                                  samplers=[dict(input=0, output=1), dict(input=2, output=3)])]
    return doc, buf


def _slerp(a, b, t):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = float(a @ b)
    if d < 0:
        b, d = -b, -d
    if d > 1 - 1e-7:
        q = (1 - t) * a + t * b
    else:
        th = np.arccos(d)
        q = (np.sin((1 - t) * th) * a + np.sin(t * th) * b) / np.sin(th)
    return q / np.linalg.norm(q)


def _expected_camera(time, yup=False):
    def seg(keys, t):
        i = int(np.searchsorted(keys, t, side="right"))
        r = min(i, len(keys) - 1)
        lo = max(r - 1, 0)
        if keys[r] == keys[lo]:
            return lo, r, 0.0
        return lo, r, float(np.clip((t - keys[lo]) / (keys[r] - keys[lo]), 0, 1))
    lo, r, d = seg(T_KEYS, time)
    t = (1 - d) * T_VALS[lo].astype(np.float64) + d * T_VALS[r]
    lo, r, d = seg(R_KEYS, time)
    q = _slerp(R_VALS[lo], R_VALS[r], d)
    if yup:
        t = np.array([t[0], -t[2], t[1]])
        s = np.sqrt(0.5)
        rq = np.array([s, 0, 0, s])  # x y z w
        x1, y1, z1, w1 = rq
        x2, y2, z2, w2 = q
        q = np.array([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                      w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2])
    m = np.eye(4)
    m[:3, :3] = _quat_matrix(q)
    m[:3, 3] = t
    return m


@pytest.mark.parametrize("yup", [False, True])
def test_camera_animation(tmp_path, yup):
    ks = _ks()
    f = tmp_path / "cam.glb"
    write_glb(f, *_anim_document())
    a = ks.CameraAnimation(f, "shot", convert_y_up_to_z_up=yup)
    assert a.frames == 3 and np.isclose(a.duration, 2.5)
    for time in (-1.0, 0.0, 0.4, 1.0, 1.7, 2.5, 3.0, a.frame_time(0), a.frame_time(2)):
        m, vfov, aspect = a.eval(time)
        assert np.isclose(vfov, 0.8) and np.isclose(aspect, 1.5)
        assert np.allclose(m, _expected_camera(time, yup), atol=2e-6), (time, m, _expected_camera(time, yup))
    assert np.isclose(a.frame_time(1), 2.5 * 1.5 / 3)
    a.close()


def test_camera_animation_errors(tmp_path):
    ks = _ks()
    f = tmp_path / "cam.glb"
    write_glb(f, *_anim_document())
    with pytest.raises(ks.KsError) as e:
        ks.CameraAnimation(f, "nobody")
    assert e.value.status == 9 and "nobody" in str(e.value)
    write_glb(f, *_anim_document(camera_type="orthographic"))
    with pytest.raises(ks.KsError) as e:
        ks.CameraAnimation(f, "shot")
    assert e.value.status == 7
    write_glb(f, *_anim_document(with_anim=False))
    with pytest.raises(ks.KsError) as e:
        ks.CameraAnimation(f, "shot")
    assert e.value.status == 9 and "animation" in str(e.value)


@pytest.mark.gpu
def test_camera_animation_through_config_task(ctx, tmp_path):
    """small_pt with camera_animation renders the requested frames (offset 1, count 2) to
    small_pt_spp<N>_<frame>.exr, each equal to the C-ABI render from the animation's camera at
    duration x (frame + 0.5) / frames."""
    from imaging import composite
    ks = _ks()
    write_glb(tmp_path / "cam.glb", *_anim_document())
    g = ks.Generated("box_room", 0)
    doc = """
[camera_animation.walk]
path = "cam.glb"
camera_name = "shot"
convert_y_up_to_z_up = false

[mesh_asset.room]
type = "procedural"
kind = "box_room"
seed = 0

[[task]]
type = "small_pt"
object = "mesh_asset.room"
camera_animation = "camera_animation.walk"
camera_animation_offset = 1
camera_animation_count = 2
bounces = 4
render_width = 24
render_height = 16
spp = 4
spp_prog_interval = 4
"""
    ks.config_run(doc, str(tmp_path / "out"), str(tmp_path))
    anim = ks.CameraAnimation(tmp_path / "cam.glb", "shot")
    s = ks.Scene(ctx, g.desc, keepalive=g)
    s.build_bvh()
    for frame in (1, 2):
        img = ks.load_image(tmp_path / "out" / "task_0" / f"small_pt_spp4_{frame:06d}.exr")
        m, vfov, aspect = anim.eval(anim.frame_time(frame))
        cam = ks.camera_perspective(m, vfov, aspect)
        p = ks.SmallPTParams.make(render_width=24, render_height=16, spp=4, bounces=4, spp_prog_interval=4)
        ref = composite(*s.render(cam, p)).astype(np.float32)
        assert np.array_equal(img, ref), frame
    assert not (tmp_path / "out" / "task_0" / "small_pt_spp4_000000.exr").exists()
    s.close()
