"""TOML task boundary (ks_config_run / ks_config_parse): the small_pt task driven by keepsake's
configuration format renders the same image as the programmatic C ABI."""
import os

import numpy as np
import pytest

from imaging import composite

DOC = """
# assets
[bsdf.white]
type = "principled_bsdf"
basecolor = { type = "constant", value = [0.8, 0.8, 0.8] }
roughness = { type = "constant", value = 1.0 }

[material.white]
bsdf = "bsdf.white"

[material.lamp]
bsdf = "bsdf.white"
emission = [17.0, 12.0, 4.0]

[mesh_asset.inline_pair]
type = "inline"
geometry = [
  { vertices = [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], indices = [[0, 2, 1], [0, 3, 2]] },
  { vertices = [[-0.3, 1.5, -0.3], [0.3, 1.5, -0.3], [0.3, 1.5, 0.3], [-0.3, 1.5, 0.3]], indices = [[0, 1, 2], [0, 2, 3]] },
]

[mesh_asset.obj_pair]
path = "pair.obj"
twosided = true

[[task]]
type = "small_pt_b200"
task_dir = "inline"
object = "mesh_asset.inline_pair"
material = [["material.white", "material.lamp"]]
sky = { ambient = [0.1, 0.2, 0.3] }
bounces = 4
render_width = 48
render_height = 32
spp = 8
spp_prog_interval = 4
camera = { type = "perspective", pos = [0.0, 1.0, 3.0], target = [0.0, 0.5, 0.0], up = [0.0, 1.0, 0.0], vfov = 45.0, aspect = 1.5 }

[[task]]
override = 0
task_dir = "obj"
object = "mesh_asset.obj_pair"
"""

OBJ = """o floor
v -1 0 -1
v 1 0 -1
v 1 0 1
v -1 0 1
f 1 3 2
f 1 4 3
o lamp
v -0.3 1.5 -0.3
v 0.3 1.5 -0.3
v 0.3 1.5 0.3
v -0.3 1.5 0.3
f -4 -3 -2 -1
"""


def _ks():
    import keepsake_b200 as ks
    return ks


def test_parse_normalises_and_round_trips():
    ks = _ks()
    n = ks.config_parse(DOC)
    assert 'task = [{ bounces = 4' in n and 'override = 0' in n
    assert ks.config_parse(n) == n
    assert ks.config_parse("a = 0x1F\nb = -1_000\nc = 1e3\nd = 'lit\\\\'\ne = \"\\u00e9\"\n") == \
        'a = 31\nb = -1000\nc = 1000.0\nd = "lit\\\\\\\\"\ne = "\u00e9"\n'


@pytest.mark.parametrize("bad,line", [
    ("a = 1\na = 2\n", 2),
    ("[t]\nx = 1\n[t]\n", 3),
    ("s = \"open\n", 1),
    ("x = 1 2\n", 1),
    ("x = [1, 2\n", 2),
    ("x = 1.2.3\n", 1),
    ("[[t]]\n[t.a]\nb = 1\n[t]\n", 4),
])
def test_parse_errors_name_the_line(bad, line):
    ks = _ks()
    with pytest.raises(ks.KsError) as e:
        ks.config_parse(bad)
    assert e.value.status == 8 and f"line {line}:" in str(e.value)


def test_task_errors_before_any_device_work(tmp_path):
    """Unknown task types, unsupported assets and missing keys fail with a status (no GPU needed:
    the scene description is resolved before a context is created)."""
    ks = _ks()
    with pytest.raises(ks.KsError) as e:
        ks.config_run('[[task]]\ntype = "gpu_small_pt"\n', str(tmp_path))
    assert e.value.status == 7
    doc = DOC.replace('type = "principled_bsdf"', 'type = "oren_nayar"')
    with pytest.raises(ks.KsError) as e:
        ks.config_run(doc, str(tmp_path))
    assert e.value.status == 7 and "oren_nayar" in str(e.value)
    with pytest.raises(ks.KsError) as e:
        ks.config_run(DOC.replace("spp = 8\n", ""), str(tmp_path))
    assert e.value.status == 8 and "spp" in str(e.value)
    with pytest.raises(ks.KsError) as e:  # an unknown distribution is an error, not GGX
        ks.config_run(DOC.replace('type = "principled_bsdf"', 'type = "principled_bsdf"\nmicrofacet = "phong"'),
                      str(tmp_path))
    assert e.value.status == 7 and "phong" in str(e.value)
    with pytest.raises(ks.KsError) as e:
        ks.config_run(DOC.replace('"material.white", "material.lamp"', '"material.white"'), str(tmp_path))
    assert "mismatch" in str(e.value)
    # each task's merged table is written next to its outputs (the override copies task 0)
    with pytest.raises(ks.KsError):
        ks.config_run(DOC.replace("spp = 8\n", ""), str(tmp_path))
    assert (tmp_path / "inline" / "config.toml").exists()


@pytest.mark.gpu
def test_config_inline_and_obj_match(tmp_path):
    ks = _ks()
    (tmp_path / "pair.obj").write_text(OBJ)
    ks.config_run(DOC, str(tmp_path / "out"), str(tmp_path))
    for d in ("inline", "obj"):
        for spp in (4, 8):
            assert (tmp_path / "out" / d / f"small_pt_spp{spp}.exr").exists()
    a = ks.load_image(tmp_path / "out" / "inline" / "small_pt_spp8.exr")
    b = ks.load_image(tmp_path / "out" / "obj" / "small_pt_spp8.exr")
    assert a.shape == (32, 48, 3) and a.mean() > 0.0
    assert np.array_equal(a, b)
    merged = (tmp_path / "out" / "obj" / "config.toml").read_text()
    assert 'object = "mesh_asset.obj_pair"' in merged and "bounces = 4" in merged


@pytest.mark.gpu
def test_config_render_equals_c_abi(ctx, tmp_path):
    """A procedural box room through the TOML task equals the same render through the C ABI."""
    ks = _ks()
    g = ks.Generated("box_room", 0)
    c2w = [float(x) for x in g.camera_to_world]
    deg = float(np.float32(np.degrees(g.vfov)))
    aspect = float(np.float32(g.aspect))
    doc = f"""
[mesh_asset.room]
type = "procedural"
kind = "box_room"
seed = 0

[[task]]
type = "small_pt"
object = "mesh_asset.room"
bounces = 8
clamp_indirect = 0.0
render_width = 64
render_height = 48
spp = 16
spp_prog_interval = 8
rng_seed = 3
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = {deg!r}, aspect = {aspect!r} }}
"""
    ks.config_run(doc, str(tmp_path))
    img = ks.load_image(tmp_path / "task_0" / "small_pt_spp16.exr")
    vfov = np.float32(deg) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), aspect)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    p = ks.SmallPTParams.make(render_width=64, render_height=48, spp=16, bounces=8, clamp_indirect=0.0,
                              spp_prog_interval=8, rng_seed=3)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert np.array_equal(img, ref)


@pytest.mark.gpu
def test_config_bsdf_types_equal_c_abi(ctx, tmp_path):
    """principled_brdf (Beckmann), lambertian and a Beckmann principled_bsdf through the TOML task
    (create_bsdf, bsdf.cpp:50-62) equal the same materials through the C ABI."""
    ks = _ks()
    c2w = [1.0, 0.0, 0.0, 0.0, 0.0, 0.9578, 0.2873, 1.8, 0.0, -0.2873, 0.9578, 3.0, 0.0, 0.0, 0.0, 1.0]
    doc = f"""
[bsdf.floor]
type = "principled_brdf"
basecolor = {{ type = "constant", value = [0.6, 0.5, 0.4] }}
roughness = {{ type = "constant", value = 0.4 }}
metallic = {{ type = "constant", value = 0.2 }}
specular = {{ type = "constant", value = 0.7 }}
microfacet = "beckmann"

[bsdf.lamp]
type = "lambertian"
albedo = {{ type = "constant", value = [0.3, 0.3, 0.3] }}

[bsdf.box]
type = "principled_bsdf"
basecolor = {{ type = "constant", value = [0.2, 0.7, 0.3] }}
roughness = {{ type = "constant", value = 0.3 }}
microfacet = "beckmann"

[material.floor]
bsdf = "bsdf.floor"

[material.lamp]
bsdf = "bsdf.lamp"
emission = [17.0, 12.0, 4.0]

[material.box]
bsdf = "bsdf.box"

[mesh_asset.trio]
type = "inline"
geometry = [
  {{ vertices = [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], indices = [[0, 2, 1], [0, 3, 2]] }},
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
    ks.config_run(doc, str(tmp_path))
    img = ks.load_image(tmp_path / "task_0" / "small_pt_spp8.exr")

    def mat(**kw):
        m = ks.MaterialDesc()
        m.basecolor[:] = kw.pop("basecolor")
        m.roughness, m.ior, m.specular_r0_mul, m.diffuse_trans_fwd = 1.0, 1.5, 0.5, 0.5
        for k, v in kw.items():
            setattr(m, k, v)
        return m
    mats = [mat(basecolor=(0.6, 0.5, 0.4), roughness=0.4, metallic=0.2, specular=0.7, bsdf=1, microfacet=1),
            mat(basecolor=(0.3, 0.3, 0.3), bsdf=2, has_emission=1),
            mat(basecolor=(0.2, 0.7, 0.3), roughness=0.3, microfacet=1)]
    mats[1].emission[:] = (17.0, 12.0, 4.0)
    meshes = [(np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float32), np.array([[0, 2, 1], [0, 3, 2]]), 0),
              (np.array([[-0.3, 1.5, -0.3], [0.3, 1.5, -0.3], [0.3, 1.5, 0.3], [-0.3, 1.5, 0.3]], np.float32),
               np.array([[0, 1, 2], [0, 2, 3]]), 1),
              (np.array([[-0.2, 0, 0], [0.2, 0, 0], [0, 0.5, 0.1]], np.float32), np.array([[0, 1, 2]]), 2)]
    sky = ks.SkyDesc()
    sky.kind = 1
    sky.ambient[:] = (0.1, 0.2, 0.3)
    desc, keep = ks.scene_desc(meshes, mats, sky)
    s = ks.Scene(ctx, desc, keep)
    s.build_bvh()
    vfov = np.float32(45.0) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.5)
    p = ks.SmallPTParams.make(render_width=48, render_height=32, spp=8, bounces=4, clamp_indirect=0.0,
                              spp_prog_interval=8)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert ref.mean() > 0.0
    assert np.array_equal(img, ref)
