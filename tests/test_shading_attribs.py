"""Per-vertex shading attributes of MeshGeometry::compute_intersection (geometry.cpp:68-163):
smooth vertex normals (the shading frame follows the interpolated normal, flipped to the side of
the face normal; geometry.cpp:139-156) and texture coordinates (the frame's tangent is dP/du of
the uv parameterisation; geometry.cpp:94-116).

The scene is the seeded box room with two coarse UV spheres, a glossy metal one and a diffuse
one, both with normals and texcoords (the walls and boxes stay flat).  The metal's GGX sampling
of visible normals only depends on the normal and wo; the diffuse lobe's cosine sampling turns
with the tangent.  The GPU
render matches the oracle's on the same Sobol samples, smooth shading changes the image against
flat shading of the same triangles, and an instanced copy of the spheres renders like the
flattened scene (normals carried to world space by the cofactor matrix of each transform).
"""
import numpy as np
import pytest

from imaging import composite, rel_mse

SAME_SEED_RELMSE = 2e-3
W, H = 64, 64


def uv_sphere(center, radius, nu=16, nv=8):
    """A latitude-longitude sphere: vertices [V,3], indices [T,3], unit normals [V,3], texcoords
    [V,2]; the seam column is duplicated (u = 0 and u = 1), pole quads give one triangle."""
    th = np.pi * np.arange(nv + 1) / nv
    ph = 2.0 * np.pi * np.arange(nu + 1) / nu
    T, P = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    uv = np.stack(np.meshgrid(np.arange(nv + 1) / nv, np.arange(nu + 1) / nu, indexing="ij")[::-1], -1)
    uv = uv.reshape(-1, 2)
    idx = []
    for j in range(nv):
        for i in range(nu):
            a = j * (nu + 1) + i
            b, c = a + 1, a + nu + 1
            d = c + 1
            if j > 0:
                idx.append((a, b, c))
            if j < nv - 1:
                idx.append((b, d, c))
    v = np.asarray(center, np.float32) + np.float32(radius) * n.astype(np.float32)
    return v.astype(np.float32), np.asarray(idx, np.uint32), n.astype(np.float32), uv.astype(np.float32)


def _material(basecolor, roughness, metallic):
    import keepsake_b200 as ks
    return ks.MaterialDesc(tuple(basecolor), roughness, metallic, 1.5, 0.5, 0.0, 0.0, 0.5, (0, 0, 0), 0, 0,
                           (0, 0, 0))


def _spheres(g):
    """The room spans [-1, 1] x [0, 2] x [-1, 1] (camera at z = 3.4 looking down -z, the tall box
    at the back left, the short box, 0.6 high, at the front right): one sphere on the floor at the
    front left, a smaller one on the short box."""
    lo, hi = g.bound
    assert np.allclose(lo, (-1, 0, -1)) and np.allclose(hi, (1, 2, 1))
    return uv_sphere((-0.5, 0.3, 0.55), 0.3), uv_sphere((0.4, 0.82, 0.35), 0.2, nu=12, nv=6)


def box_room_with_spheres(normals=True, texcoords=True, twosided=1):
    """(Generated box room, mesh list for ks.scene_desc, materials)."""
    import keepsake_b200 as ks
    g = ks.Generated("box_room", 0)
    meshes = [(m["vertices"], m["indices"], m["material"], dict(twosided=m["twosided"])) for m in g.meshes]
    mats = list(g.materials) + [_material((0.95, 0.7, 0.35), 0.2, 1.0), _material((0.3, 0.6, 0.8), 1.0, 0.0)]
    for (v, i, n, t), mat in zip(_spheres(g), (len(mats) - 2, len(mats) - 1)):
        meshes.append((v, i, mat, dict(twosided=twosided, normals=n if normals else None,
                                       texcoords=t if texcoords else None)))
    return g, meshes, mats


def _params(spp, seed=0):
    import keepsake_b200 as ks
    return ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=8, rng_seed=seed,
                                 clamp_indirect=0.0)


def _camera(g):
    import keepsake_b200 as ks
    return ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)


def test_uv_sphere_normals_and_winding():
    v, idx, n, uv = uv_sphere((1.0, 2.0, 3.0), 0.5)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6)
    assert np.allclose(v - np.float32((1.0, 2.0, 3.0)), 0.5 * n, atol=1e-6)
    assert idx.max() < len(v) and len(idx) == 16 * 8 * 2 - 2 * 16
    # every triangle is non-degenerate and faces outwards
    p0, p1, p2 = v[idx[:, 0]], v[idx[:, 1]], v[idx[:, 2]]
    ng = np.cross(p1 - p0, p2 - p0)
    assert (np.linalg.norm(ng, axis=1) > 1e-6).all()
    assert (np.einsum("ij,ij->i", ng, (p0 + p1 + p2) / 3 - np.float32((1.0, 2.0, 3.0))) > 0).all()
    assert uv.min() == 0.0 and uv.max() == 1.0


def test_oracle_smooth_normals_change_the_image(oracle):
    """Same samples, same triangles: the sphere pixels change when the shading frame follows the
    vertex normals; texcoords alone only turn the tangent, which changes the diffuse sphere's
    sampled directions (an isotropic BSDF's image keeps its expectation)."""
    import keepsake_b200 as ks
    imgs = {}
    for key, (nrm, tc) in {"flat": (False, False), "smooth": (True, True), "uv": (False, True)}.items():
        g, meshes, mats = box_room_with_spheres(normals=nrm, texcoords=tc)
        d, keep = ks.scene_desc(meshes, mats, g.desc.contents.sky)
        a, w, _ = oracle.scene(d, keepalive=keep).render(_camera(g), _params(4), threads=4)
        imgs[key] = (composite(a, w), w)
    assert np.array_equal(imgs["flat"][1], imgs["smooth"][1])
    rel = np.abs(imgs["smooth"][0] - imgs["flat"][0]) / (np.abs(imgs["flat"][0]) + 1e-3)
    assert (rel > 1e-2).mean() > 0.05
    rel_uv = np.abs(imgs["uv"][0] - imgs["flat"][0]) / (np.abs(imgs["flat"][0]) + 1e-3)
    assert (rel_uv > 1e-2).mean() > 0.005


@pytest.mark.gpu
@pytest.mark.parametrize("normals,texcoords", [(True, True), (True, False), (False, True)])
def test_attribs_same_seed_matches_oracle(ctx, oracle, normals, texcoords):
    import keepsake_b200 as ks
    g, meshes, mats = box_room_with_spheres(normals=normals, texcoords=texcoords)
    d, keep = ks.scene_desc(meshes, mats, g.desc.contents.sky)
    s = ks.Scene(ctx, d, keepalive=keep)
    s.build_bvh()
    cam, p = _camera(g), _params(16, seed=3)
    acc, w = s.render(cam, p)
    s.close()
    oacc, ow, ocnt = oracle.scene(d, keepalive=keep).render(cam, p)
    assert np.array_equal(w, ow), "hit/miss weights differ"
    img, ref = composite(acc, w), composite(oacc, ow)
    assert np.isfinite(img).all()
    err = rel_mse(img, ref)
    assert err < SAME_SEED_RELMSE, f"relMSE(gpu, oracle) = {err}"
    rel = np.abs(img - ref) / (np.abs(ref) + 1e-3)
    assert np.median(rel) < 1e-4


@pytest.mark.gpu
def test_smooth_shading_differs_from_flat_on_gpu(ctx):
    import keepsake_b200 as ks
    out = []
    for nrm in (False, True):
        g, meshes, mats = box_room_with_spheres(normals=nrm, texcoords=False)
        d, keep = ks.scene_desc(meshes, mats, g.desc.contents.sky)
        s = ks.Scene(ctx, d, keepalive=keep)
        s.build_bvh()
        out.append(composite(*s.render(_camera(g), _params(8))))
        s.close()
    rel = np.abs(out[1] - out[0]) / (np.abs(out[0]) + 1e-3)
    assert (rel > 1e-2).mean() > 0.05


def _cofactor(m):
    c0, c1, c2 = m[:, 0].astype(np.float64), m[:, 1].astype(np.float64), m[:, 2].astype(np.float64)
    return np.stack([np.cross(c1, c2), np.cross(c2, c0), np.cross(c0, c1)], axis=1)


@pytest.mark.gpu
def test_instanced_smooth_spheres_match_flattened(ctx):
    """Two prototypes (the two textured smooth spheres) under rotations about random axes, uniform
    scales and translations: the two-level render equals the render of the scene with the
    instances flattened (vertices through the transform, normals through its cofactor matrix)."""
    import keepsake_b200 as ks
    g, meshes, mats = box_room_with_spheres()
    n_room = len(g.meshes)
    rng = np.random.default_rng(7)
    # (prototype, scale, new centre on the floor or on the short box)
    place = [(1, 0.8, (-0.6, 0.0, 0.6)), (2, 0.9, (-0.1, 0.0, 0.75)), (1, 0.6, (0.35, 0.6, 0.35)),
             (2, 0.7, (0.8, 0.0, 0.85))]
    centres, radii = [(-0.5, 0.3, 0.55), (0.4, 0.82, 0.35)], [0.3, 0.2]
    xfs = []
    for pr, sc, (x, y, z) in place:
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        a = rng.uniform(0, 2 * np.pi)
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
        rot = np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K
        c_new = np.array([x, y + sc * radii[pr - 1], z])
        xf = np.zeros((3, 4))
        xf[:, :3] = sc * rot
        xf[:, 3] = c_new - sc * rot @ np.array(centres[pr - 1])
        xfs.append((pr, xf.astype(np.float32)))
    protos = [(0, n_room), (n_room, 1), (n_room + 1, 1)]
    insts = [(0, np.eye(3, 4, dtype=np.float32))] + xfs
    # the instanced description
    d, keep = ks.scene_desc(meshes, mats, g.desc.contents.sky)
    pd = (ks.PrototypeDesc * len(protos))(*[ks.PrototypeDesc(a, b) for a, b in protos])
    idesc = (ks.InstanceDesc * len(insts))()
    for k, (pr, xf) in enumerate(insts):
        idesc[k].prototype = pr
        idesc[k].to_world[:] = [float(x) for x in xf.reshape(12)]
    d.prototypes, d.n_prototypes = pd, len(protos)
    d.instances, d.n_instances = idesc, len(insts)
    inst = ks.Scene(ctx, d, keepalive=(keep, pd, idesc))
    inst.build_bvh()
    # the flattened description: room meshes as they are, each sphere instance in world space
    flat = list(meshes[:n_room])
    for pr, xf in insts[1:]:
        v, idx, mat, extra = meshes[protos[pr][0]]
        w = np.empty_like(v)
        for r in range(3):
            w[:, r] = ((xf[r, 0] * v[:, 0] + xf[r, 1] * v[:, 1]) + xf[r, 2] * v[:, 2]) + xf[r, 3]
        e = dict(extra)
        e["normals"] = (extra["normals"].astype(np.float64) @ _cofactor(xf).T).astype(np.float32)
        flat.append((w, idx, mat, e))
    fd, fkeep = ks.scene_desc(flat, mats, g.desc.contents.sky)
    fs = ks.Scene(ctx, fd, keepalive=fkeep)
    fs.build_bvh()
    cam, p = _camera(g), _params(32, seed=5)
    a = composite(*inst.render(cam, p))
    b = composite(*fs.render(cam, p))
    inst.close()
    fs.close()
    assert a.mean() > 0.0
    assert rel_mse(a, b) < SAME_SEED_RELMSE, rel_mse(a, b)


def _obj_text(meshes):
    """Wavefront OBJ of [(vertices, indices, normals or None, texcoords or None)], one `o` per mesh,
    a corner's vt / vn the ones of its vertex (floats printed to round-trip exactly)."""
    out, vb, tb, nb = [], 1, 1, 1
    for k, (v, idx, n, t) in enumerate(meshes):
        out.append(f"o mesh{k}")
        out += ["v %.9g %.9g %.9g" % tuple(map(float, p)) for p in v]
        if t is not None:
            out += ["vt %.9g %.9g" % tuple(map(float, p)) for p in t]
        if n is not None:
            out += ["vn %.9g %.9g %.9g" % tuple(map(float, p)) for p in n]
        for tri in idx.astype(np.int64):
            corners = []
            for i in tri:
                c = str(i + vb)
                if t is not None or n is not None:
                    c += "/" + (str(i + tb) if t is not None else "")
                if n is not None:
                    c += "/" + str(i + nb)
                corners.append(c)
            out.append("f " + " ".join(corners))
        vb += len(v)
        tb += 0 if t is None else len(t)
        nb += 0 if n is None else len(n)
    return "\n".join(out) + "\n"


@pytest.mark.gpu
def test_obj_normals_and_texcoords_through_config_task(ctx, tmp_path):
    """An OBJ mesh asset with vt / vn lines, rendered by the TOML small_pt task, equals the C-ABI
    render of the same meshes with the same normals and texcoords (bit-exact image)."""
    import keepsake_b200 as ks
    ground = (np.array([[-2, 0, -2], [2, 0, -2], [2, 0, 2], [-2, 0, 2]], np.float32),
              np.array([[0, 2, 1], [0, 3, 2]], np.uint32), None, None)
    s1 = uv_sphere((-0.5, 0.3, 0.55), 0.3)
    s2 = uv_sphere((0.4, 0.25, 0.0), 0.25, nu=12, nv=6)
    s1 = (s1[0], s1[1], s1[2], s1[3])
    s2 = (s2[0], s2[1], None, s2[3])  # texcoords only: flat shading, uv tangents
    (tmp_path / "spheres.obj").write_text(_obj_text([ground, s1, s2]))
    c2w = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.6, 0.0, 0.0, 1.0, 3.0, 0.0, 0.0, 0.0, 1.0]
    doc = f"""
[bsdf.white]
type = "principled_bsdf"

[bsdf.gold]
type = "principled_bsdf"
basecolor = {{ type = "constant", value = [0.95, 0.7, 0.35] }}
roughness = {{ type = "constant", value = 0.2 }}
metallic = {{ type = "constant", value = 1.0 }}

[bsdf.blue]
type = "principled_bsdf"
basecolor = {{ type = "constant", value = [0.3, 0.6, 0.8] }}

[material.white]
bsdf = "bsdf.white"
[material.gold]
bsdf = "bsdf.gold"
[material.blue]
bsdf = "bsdf.blue"

[mesh_asset.spheres]
path = "spheres.obj"
twosided = true

[[task]]
type = "small_pt"
object = "mesh_asset.spheres"
material = [["material.white", "material.gold", "material.blue"]]
sky = {{ ambient = [0.6, 0.7, 0.9] }}
bounces = 6
render_width = 48
render_height = 48
spp = 8
spp_prog_interval = 8
rng_seed = 2
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = 40.0, aspect = 1.0 }}
"""
    ks.config_run(doc, str(tmp_path / "out"), str(tmp_path))
    img = ks.load_image(tmp_path / "out" / "task_0" / "small_pt_spp8.exr")
    mats = [_material((0.8, 0.8, 0.8), 1.0, 0.0), _material((0.95, 0.7, 0.35), 0.2, 1.0),
            _material((0.3, 0.6, 0.8), 1.0, 0.0)]
    meshes = [(v, i, k, dict(twosided=1, normals=n, texcoords=t)) for k, (v, i, n, t) in enumerate([ground, s1, s2])]
    sky = ks.SkyDesc()
    sky.kind = 1
    sky.ambient[:] = [0.6, 0.7, 0.9]
    sky.to_world[:] = [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]
    sky.transform_y_up = 1
    sky.strength = 1.0
    d, keep = ks.scene_desc(meshes, mats, sky)
    s = ks.Scene(ctx, d, keepalive=keep)
    s.build_bvh()
    vfov = np.float32(40.0) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.0)
    p = ks.SmallPTParams.make(render_width=48, render_height=48, spp=8, bounces=6, spp_prog_interval=8, rng_seed=2)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert img.mean() > 0.0
    assert np.array_equal(img, ref)
