"""keepsake_b200: B200-native (sm_100a) small_pt path tracer behind a C ABI.

This Python module is a thin ctypes binding of ``libks_b200.so`` (declared in
``include/ks_b200.h``) used by the test-suite and ``bench.py``.  The library is the product;
there is no Python or CPU fallback: importing this module raises if the shared library has not
been built (``python -c "import __graft_entry__ as g; g.build()"`` or ``make -C keepsake_b200``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libks_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"keepsake_b200: {LIB_PATH} is missing; build it with `make -C keepsake_b200` "
        "(the CUDA library is the only implementation)")

lib = ctypes.CDLL(LIB_PATH)

KS_OK = 0
STATUS_NAMES = {
    0: "KS_OK", 1: "KS_ERR_INVALID_ARGUMENT", 2: "KS_ERR_OUT_OF_MEMORY", 3: "KS_ERR_CUDA",
    4: "KS_ERR_QUEUE_OVERFLOW", 5: "KS_ERR_WATCHDOG", 6: "KS_ERR_NOT_BUILT",
    7: "KS_ERR_UNSUPPORTED", 8: "KS_ERR_PARSE", 9: "KS_ERR_IO",
}

_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_i32 = ctypes.c_int32
_f32 = ctypes.c_float

lib.ks_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
lib.ks_context_create.restype = ctypes.c_int
lib.ks_context_destroy.argtypes = [_vp]
lib.ks_context_destroy.restype = None
lib.ks_status_string.argtypes = [ctypes.c_int]
lib.ks_status_string.restype = ctypes.c_char_p
lib.ks_last_error.argtypes = [_vp]
lib.ks_last_error.restype = ctypes.c_char_p
lib.ks_sobol_points.argtypes = [_vp] + [_u32] * 11 + [_vp]
lib.ks_sobol_points.restype = ctypes.c_int
lib.ks_sobol_bounce.argtypes = [_vp] + [_u32] * 11 + [_vp]
lib.ks_sobol_bounce.restype = ctypes.c_int


class KsError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {detail}" if detail else name)


def ptr(a) -> ctypes.c_void_p:
    """Address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """One CUDA device + stream (ks_context)."""

    def __init__(self, device: int = 0):
        import weakref
        h = _vp()
        st = lib.ks_context_create(device, ctypes.byref(h))
        if st != KS_OK:
            raise KsError(st, "ks_context_create")
        self.handle = h
        # scenes must be destroyed before their context (ks_scene_destroy uses the context)
        self._scenes = weakref.WeakSet()

    def check(self, st: int, what: str = ""):
        if st != KS_OK:
            raise KsError(st, f"{what}: {lib.ks_last_error(self.handle).decode()}")

    def close(self):
        if self.handle:
            for sc in list(self._scenes):
                sc.close()
            lib.ks_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rel_mse_device(self, accum_ptr: int, weights_ptr: int, ref_ptr: int, n_pixels: int, eps=1e-2,
                       backdrop=None) -> float:
        """ks_image_rel_mse_device on device buffers (raw pointers)."""
        out = np.zeros(1, np.float64)
        bd = None if backdrop is None else np.asarray(backdrop, np.float32)
        self.check(lib.ks_image_rel_mse_device(self.handle, ctypes.c_void_p(accum_ptr), ctypes.c_void_p(weights_ptr),
                                               ctypes.c_void_p(ref_ptr), n_pixels, eps, ptr(bd), ptr(out)),
                   "ks_image_rel_mse_device")
        return float(out[0])

    def set_limits(self, sbvh_max_levels=0, wavefront_max_iterations=0):
        """ks_context_set_limits: failure-detection limits (0 = the library's own bound)."""
        lim = ContextLimits(sbvh_max_levels, wavefront_max_iterations)
        self.check(lib.ks_context_set_limits(self.handle, ctypes.byref(lim)), "ks_context_set_limits")

    def mbarrier_probe(self, max_polls, arrive) -> int:
        """ks_mbarrier_wait_probe: the status (KS_OK or KS_ERR_WATCHDOG) of a bounded mbarrier wait."""
        return lib.ks_mbarrier_wait_probe(self.handle, max_polls, int(arrive))

    def bsdf_eval(self, material, wo, wi):
        """ks_bsdf_eval: (f cos [n, 3], pdf [n]) of the device BSDF code for local directions."""
        wo = np.ascontiguousarray(wo, np.float32)
        wi = np.ascontiguousarray(wi, np.float32)
        n = len(wo)
        f = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.check(lib.ks_bsdf_eval(self.handle, ctypes.byref(material), ptr(wo), ptr(wi), n, ptr(f), ptr(pdf)),
                   "ks_bsdf_eval")
        return f, pdf

    def bsdf_sample(self, material, wo, u):
        """ks_bsdf_sample: (wi [n, 3], weight f cos / pdf [n, 3], pdf [n]) for u = (u_lobe, u0, u1)."""
        wo = np.ascontiguousarray(wo, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        n = len(wo)
        wi = np.empty((n, 3), np.float32)
        beta = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.check(lib.ks_bsdf_sample(self.handle, ctypes.byref(material), ptr(wo), ptr(u), n, ptr(wi), ptr(beta),
                                      ptr(pdf)), "ks_bsdf_sample")
        return wi, beta, pdf

    def sobol_points(self, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd) -> np.ndarray:
        out = np.empty((ny, nx, ns, nd, 3), dtype=np.float32)
        st = lib.ks_sobol_points(self.handle, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd, ptr(out))
        self.check(st, "ks_sobol_points")
        return out

    def sobol_bounce(self, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, dim) -> np.ndarray:
        """The seven values one path vertex draws from dimension dim (the sampling kernel's code)."""
        out = np.empty((ny, nx, ns, 7), dtype=np.float32)
        st = lib.ks_sobol_bounce(self.handle, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, dim, ptr(out))
        self.check(st, "ks_sobol_bounce")
        return out


# ---------------------------------------------------------------------------------------------
# Scene description structs (mirror include/ks_b200.h)
# ---------------------------------------------------------------------------------------------
class MeshDesc(ctypes.Structure):
    _fields_ = [("vertices", _vp), ("n_vertices", _u32), ("indices", _vp), ("n_triangles", _u32),
                ("vertex_normals", _vp), ("material", _u32), ("twosided", _i32), ("use_smooth_normal", _i32),
                ("texcoords", _vp)]


class MaterialDesc(ctypes.Structure):
    _fields_ = [("basecolor", _f32 * 3), ("roughness", _f32), ("metallic", _f32), ("ior", _f32),
                ("specular_r0_mul", _f32), ("specular_trans", _f32), ("diffuse_trans", _f32),
                ("diffuse_trans_fwd", _f32), ("emissive", _f32 * 3), ("microfacet", _i32),
                ("has_emission", _i32), ("emission", _f32 * 3), ("bsdf", _i32), ("specular", _f32),
                ("has_subsurface", _i32), ("ss_albedo", _f32 * 3), ("ss_radius", _f32 * 3), ("ss_anisotropy", _f32),
                ("ss_ior", _f32), ("ss_rfr_entry_prob", _f32)]


class SkyDesc(ctypes.Structure):
    _fields_ = [("kind", _i32), ("ambient", _f32 * 3), ("map_rgb", _vp), ("width", _u32), ("height", _u32),
                ("to_world", _f32 * 16), ("transform_y_up", _i32), ("strength", _f32)]


class PrototypeDesc(ctypes.Structure):
    _fields_ = [("first_mesh", _u32), ("n_meshes", _u32)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("prototype", _u32), ("to_world", _f32 * 12)]


class LightDesc(ctypes.Structure):
    _fields_ = [("type", _i32), ("color", _f32 * 3), ("vec", _f32 * 3)]


class TextureDesc(ctypes.Structure):
    _fields_ = [("texels", _vp), ("width", _u32), ("height", _u32), ("channels", _u32), ("format", _i32),
                ("srgb", _i32)]


FIELDS = {"basecolor": 0, "roughness": 1, "metallic": 2, "ior": 3, "specular_r0_mul": 4, "specular_trans": 5,
          "diffuse_trans": 6, "diffuse_trans_fwd": 7, "specular": 8, "normal_map": 9, "opacity_map": 10, "emission": 11}


class TextureBinding(ctypes.Structure):
    _fields_ = [("material", _u32), ("field", _i32), ("texture", _u32), ("filter", _i32), ("cubic_kernel", _i32),
                ("wrap_u", _i32), ("wrap_v", _i32), ("flip_v", _i32), ("swizzle", _i32 * 4), ("uv_scale", _f32 * 2),
                ("uv_offset", _f32 * 2), ("scale", _f32 * 4), ("normal_space", _i32), ("range01", _i32),
                ("strength", _f32), ("to_world", _f32 * 16)]

    @classmethod
    def make(cls, material, field, texture, **kw):
        """A binding with the reference's defaults (flip_v, identity swizzle and scale, uv_scale 1,
        range01, strength 1, identity to_world), then the given fields; `field` by name or id."""
        b = cls()
        b.material, b.texture = material, texture
        b.field = FIELDS[field] if isinstance(field, str) else field
        b.flip_v, b.range01, b.strength = 1, 1, 1.0
        b.swizzle[:] = (0, 1, 2, 3)
        b.uv_scale[:] = (1.0, 1.0)
        b.scale[:] = (1.0, 1.0, 1.0, 1.0)
        b.to_world[:] = [float(x) for x in np.eye(4).reshape(16)]
        for k, v in kw.items():
            if k in ("swizzle", "uv_scale", "uv_offset", "scale", "to_world"):
                getattr(b, k)[:] = [float(x) if k != "swizzle" else int(x) for x in np.asarray(v).reshape(-1)]
            else:
                setattr(b, k, v)
        return b


class SceneDesc(ctypes.Structure):
    _fields_ = [("meshes", ctypes.POINTER(MeshDesc)), ("n_meshes", _u32),
                ("materials", ctypes.POINTER(MaterialDesc)), ("n_materials", _u32), ("sky", SkyDesc),
                ("prototypes", ctypes.POINTER(PrototypeDesc)), ("n_prototypes", _u32),
                ("instances", ctypes.POINTER(InstanceDesc)), ("n_instances", _u32),
                ("lights", ctypes.POINTER(LightDesc)), ("n_lights", _u32),
                ("textures", ctypes.POINTER(TextureDesc)), ("n_textures", _u32),
                ("bindings", ctypes.POINTER(TextureBinding)), ("n_bindings", _u32)]


def attach_textures(desc, textures, bindings):
    """Sets the textures (numpy arrays [H, W, C] of uint8, uint16 or float32, with an `srgb` flag:
    (array, srgb)) and bindings (TextureBinding) of a SceneDesc; returns what must stay alive."""
    keep = []
    td = (TextureDesc * max(len(textures), 1))()
    for k, (arr, srgb) in enumerate(textures):
        a = np.ascontiguousarray(arr)
        if a.ndim == 2:
            a = a[..., None]
        fmt = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2}[a.dtype]
        keep.append(a)
        td[k] = TextureDesc(a.ctypes.data, a.shape[1], a.shape[0], a.shape[2], fmt, int(srgb))
    bd = (TextureBinding * max(len(bindings), 1))(*bindings)
    keep += [td, bd]
    d = desc.contents if isinstance(desc, ctypes._Pointer) else desc
    d.textures, d.n_textures = td, len(textures)
    d.bindings, d.n_bindings = bd, len(bindings)
    return keep


class ContextLimits(ctypes.Structure):
    _fields_ = [("sbvh_max_levels", _u32), ("wavefront_max_iterations", _u32)]


class SBVHOptions(ctypes.Structure):
    _fields_ = [("max_prims_in_node", _u32), ("bucket_count", _u32), ("trav_weight", _f32), ("alpha", _f32)]


class CameraDesc(ctypes.Structure):
    _fields_ = [("camera_to_world", _f32 * 16), ("proj_to_camera", _f32 * 16), ("proj_to_world", _f32 * 16),
                ("orthographic", _i32)]


class ProceduralOptions(ctypes.Structure):
    _fields_ = [("level", _i32), ("roughness_min", _f32), ("roughness_max", _f32), ("occluder", _i32),
                ("sky_width", _u32), ("sky_height", _u32), ("width", _u32), ("height", _u32),
                ("prototypes", _u32), ("instances", _u32), ("frequency", _u32), ("emitters", _u32)]


class SmallPTParams(ctypes.Structure):
    _fields_ = [("include_background", _i32), ("backdrop", _f32 * 3), ("bounces", _i32), ("render_width", _i32),
                ("render_height", _i32), ("crop_start_x", _i32), ("crop_start_y", _i32), ("crop_width", _i32),
                ("crop_height", _i32), ("spp", _i32), ("rng_seed", _i32), ("scale_ray_diff", _i32),
                ("clamp_direct", _f32), ("clamp_indirect", _f32), ("spp_prog_interval", _i32),
                ("pixel_filter_width", _f32), ("pixel_filter", _i32), ("pixel_filter_sigma", _f32)]

    @classmethod
    def make(cls, **kw):
        p = cls()
        lib.ks_small_pt_params_default(ctypes.byref(p))
        for k, v in kw.items():
            if k == "backdrop":
                p.backdrop[:] = v
            else:
                setattr(p, k, v)
        return p


def _sig(name, args, res=ctypes.c_int):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res


_sig("ks_scene_create", [_vp, ctypes.POINTER(SceneDesc), ctypes.POINTER(_vp)])
_sig("ks_bsdf_eval", [_vp, ctypes.POINTER(MaterialDesc), _vp, _vp, _u32, _vp, _vp])
_sig("ks_context_set_limits", [_vp, ctypes.POINTER(ContextLimits)])
_sig("ks_mbarrier_wait_probe", [_vp, _u32, ctypes.c_int])
_sig("ks_bsdf_sample", [_vp, ctypes.POINTER(MaterialDesc), _vp, _vp, _u32, _vp, _vp, _vp])
_sig("ks_scene_destroy", [_vp], None)
_sig("ks_scene_build_bvh", [_vp, ctypes.POINTER(SBVHOptions), ctypes.POINTER(_f32)])
_sig("ks_sbvh_counts", [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u32)])
_sig("ks_sbvh_export", [_vp, _vp, _vp, _vp, _vp, _vp])
_sig("ks_trace_rays", [_vp, _vp, _u32, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp])
_sig("ks_trace_rays_wide", [_vp, _vp, _u32, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp])
_sig("ks_camera_perspective", [ctypes.POINTER(_f32), _f32, _f32, ctypes.POINTER(CameraDesc)])
_sig("ks_camera_orthographic", [ctypes.POINTER(_f32), _f32, _f32, _f32, _f32, _f32, _f32, ctypes.POINTER(CameraDesc)])
_sig("ks_procedural_scene", [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ProceduralOptions),
                             ctypes.POINTER(_vp)])
_sig("ks_generated_scene_desc", [_vp], ctypes.POINTER(SceneDesc))
_sig("ks_generated_camera", [_vp, ctypes.POINTER(_f32), ctypes.POINTER(_f32), ctypes.POINTER(_f32)])
_sig("ks_generated_destroy", [_vp], None)
_sig("ks_compound_asset_load", [ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(_vp)])
_sig("ks_camera_animation_load", [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(_vp)])
_sig("ks_camera_animation_frames", [_vp], ctypes.c_uint32)
_sig("ks_camera_animation_duration", [_vp], _f32)
_sig("ks_camera_animation_eval", [_vp, _f32, ctypes.POINTER(_f32), ctypes.POINTER(_f32), ctypes.POINTER(_f32)])
_sig("ks_camera_animation_destroy", [_vp], None)


class CameraAnimation:
    """A glTF camera animation (ks_camera_animation_*)."""

    def __init__(self, path, camera_name, convert_y_up_to_z_up=False):
        h = _vp()
        st = lib.ks_camera_animation_load(str(path).encode(), camera_name.encode(), int(convert_y_up_to_z_up),
                                          ctypes.byref(h))
        if st != KS_OK:
            raise KsError(st, lib.ks_config_last_error().decode())
        self.handle = h
        self.frames = lib.ks_camera_animation_frames(h)
        self.duration = lib.ks_camera_animation_duration(h)

    def eval(self, time):
        """(camera_to_world [4, 4] row-major, vfov radians, aspect) at `time`."""
        m = (_f32 * 16)()
        vfov, aspect = _f32(), _f32()
        st = lib.ks_camera_animation_eval(self.handle, time, m, ctypes.byref(vfov), ctypes.byref(aspect))
        if st != KS_OK:
            raise KsError(st, "ks_camera_animation_eval")
        return np.array(m[:], np.float32).reshape(4, 4), vfov.value, aspect.value

    def frame_time(self, frame):
        """The time the small_pt task renders frame `frame` at: duration x (frame + 0.5) / frames."""
        return float(np.float32(self.duration) * (np.float32(frame) + np.float32(0.5)) / np.float32(self.frames))

    def close(self):
        if self.handle:
            lib.ks_camera_animation_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
_sig("ks_small_pt_params_default", [ctypes.POINTER(SmallPTParams)], None)


class RenderStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("extension_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("iterations", _u32), ("kernel_launches", _u32), ("ms_total", _f32), ("ms_extend", _f32),
                ("ms_shade", _f32), ("ms_shadow", _f32), ("ext_nodes", ctypes.c_uint64),
                ("ext_tris", ctypes.c_uint64), ("shadow_nodes", ctypes.c_uint64), ("shadow_tris", ctypes.c_uint64),
                ("ms_guide_infer", _f32), ("ms_guide_train", _f32), ("guide_records", ctypes.c_uint64),
                ("guide_train_steps", _u32), ("guide_rows", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PROGRESS_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), _vp)
_sig("ks_small_pt_render", [_vp, ctypes.POINTER(CameraDesc), ctypes.POINTER(SmallPTParams), PROGRESS_FN, _vp,
                            _vp, _vp])
_sig("ks_small_pt_render_device", [_vp, ctypes.POINTER(CameraDesc), ctypes.POINTER(SmallPTParams), _vp, _vp])
_sig("ks_render_stats_last", [_vp, ctypes.POINTER(RenderStats)])
DEVICE_PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, _vp)
_sig("ks_image_rel_mse_device", [_vp, _vp, _vp, _vp, _u32, ctypes.c_double, _vp, _vp])


def _arr(p, n, dtype):
    """Copy n elements of a C array into numpy."""
    if not p or n == 0:
        return np.zeros(0, dtype=dtype)
    ct = {np.float32: ctypes.c_float, np.uint32: ctypes.c_uint32, np.uint16: ctypes.c_uint16,
          np.uint8: ctypes.c_uint8}[dtype]
    buf = (ct * n).from_address(ctypes.cast(p, ctypes.c_void_p).value)
    return np.frombuffer(buf, dtype=dtype).copy()


class Generated:
    """A seeded procedural scene (ks_procedural_scene) with numpy views of its arrays."""

    def __init__(self, kind: str, seed: int = 0, level: int = 8, roughness=(0.05, 1.0), occluder=False,
                 sky=(2048, 1024), resolution=(1024, 1024), prototypes=0, instances=0, frequency=0, emitters=0):
        o = ProceduralOptions(level, roughness[0], roughness[1], int(occluder), sky[0], sky[1],
                              resolution[0], resolution[1], prototypes, instances, frequency, emitters)
        h = _vp()
        st = lib.ks_procedural_scene(kind.encode(), seed, ctypes.byref(o), ctypes.byref(h))
        if st != KS_OK:
            raise KsError(st, "ks_procedural_scene")
        self._adopt(h)

    @classmethod
    def load_compound(cls, path, load_materials=True):
        """A glTF compound mesh asset as a scene description (ks_compound_asset_load)."""
        h = _vp()
        st = lib.ks_compound_asset_load(str(path).encode(), int(load_materials), ctypes.byref(h))
        if st != KS_OK:
            raise KsError(st, lib.ks_config_last_error().decode())
        g = cls.__new__(cls)
        g._adopt(h)
        return g

    def _adopt(self, h):
        self.handle = h
        self.desc = lib.ks_generated_scene_desc(h)
        d = self.desc.contents
        self.meshes = []
        for m in range(d.n_meshes):
            md = d.meshes[m]
            self.meshes.append(dict(
                vertices=_arr(md.vertices, 3 * md.n_vertices, np.float32).reshape(-1, 3),
                indices=_arr(md.indices, 3 * md.n_triangles, np.uint32).reshape(-1, 3),
                normals=(_arr(md.vertex_normals, 3 * md.n_vertices, np.float32).reshape(-1, 3)
                         if md.vertex_normals else None),
                texcoords=(_arr(md.texcoords, 2 * md.n_vertices, np.float32).reshape(-1, 2)
                           if md.texcoords else None),
                material=md.material, twosided=md.twosided, smooth=md.use_smooth_normal))
        self.materials = [d.materials[k] for k in range(d.n_materials)]
        c2w = (_f32 * 16)()
        vfov, aspect = _f32(), _f32()
        lib.ks_generated_camera(h, c2w, ctypes.byref(vfov), ctypes.byref(aspect))
        self.camera_to_world = np.array(c2w[:], dtype=np.float32)
        self.vfov, self.aspect = vfov.value, aspect.value
        self.prototypes = [(d.prototypes[k].first_mesh, d.prototypes[k].n_meshes) for k in range(d.n_prototypes)]
        self.instances = [(d.instances[k].prototype, np.array(d.instances[k].to_world[:], np.float32).reshape(3, 4))
                          for k in range(d.n_instances)]
        self.textures = []
        for k in range(d.n_textures):
            t = d.textures[k]
            dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[t.format]
            self.textures.append((_arr(t.texels, t.height * t.width * t.channels, dt)
                                  .reshape(t.height, t.width, t.channels), bool(t.srgb)))
        self.bindings = [d.bindings[k] for k in range(d.n_bindings)]
        self.sky_kind = d.sky.kind
        self.sky_map = (_arr(d.sky.map_rgb, 3 * d.sky.width * d.sky.height, np.float32)
                        .reshape(d.sky.height, d.sky.width, 3) if d.sky.kind == 2 else None)

    def flat_geometry(self):
        """All meshes concatenated in mesh order: (vertices [V,3], indices [T,3] global)."""
        vs, ids, off = [], [], 0
        for m in self.meshes:
            vs.append(m["vertices"])
            ids.append(m["indices"].astype(np.uint64) + off)
            off += len(m["vertices"])
        return np.concatenate(vs).astype(np.float32), np.concatenate(ids).astype(np.uint32)

    def flattened(self):
        """Instanced scenes: every instance's meshes transformed to world space (float32, the
        product's own arithmetic order), as a list of (vertices [V,3], indices [T,3], material)."""
        if not self.instances:
            return [(m["vertices"], m["indices"], m["material"]) for m in self.meshes]
        out = []
        for proto, xf in self.instances:
            first, n = self.prototypes[proto]
            for m in self.meshes[first:first + n]:
                v = m["vertices"]
                w = np.empty_like(v)
                for r in range(3):
                    w[:, r] = ((xf[r, 0] * v[:, 0] + xf[r, 1] * v[:, 1]) + xf[r, 2] * v[:, 2]) + xf[r, 3]
                out.append((w, m["indices"], m["material"]))
        return out

    @property
    def bound(self):
        """Axis-aligned bound of the scene in world space: (min [3], max [3]) (instances: the
        transformed corners of each prototype's box)."""
        if not self.instances:
            lo = np.min([m["vertices"].min(0) for m in self.meshes], axis=0)
            hi = np.max([m["vertices"].max(0) for m in self.meshes], axis=0)
            return lo, hi
        boxes = []
        for first, n in self.prototypes:
            v = np.concatenate([m["vertices"] for m in self.meshes[first:first + n]])
            boxes.append((v.min(0), v.max(0)))
        pts = []
        for proto, xf in self.instances:
            lo, hi = boxes[proto]
            c = np.array([[(hi if k & 1 else lo)[0], (hi if k & 2 else lo)[1], (hi if k & 4 else lo)[2]]
                          for k in range(8)], np.float64)
            pts.append(c @ xf[:, :3].T.astype(np.float64) + xf[:, 3])
        pts = np.concatenate(pts)
        return pts.min(0).astype(np.float32), pts.max(0).astype(np.float32)

    @property
    def n_triangles(self):
        return sum(len(m["indices"]) for m in self.meshes)

    def close(self):
        if self.handle:
            lib.ks_generated_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scene_desc(meshes, materials, sky=None):
    """A SceneDesc over Python arrays: meshes = [(vertices [V,3], indices [T,3], material[, extra])]
    with the optional dict `extra` holding "normals" [V,3], "texcoords" [V,2], "twosided" (default
    1) and "smooth" (use_smooth_normal, default 1); materials = [MaterialDesc].  Returns
    (desc, keepalive)."""
    keep = []
    md = (MeshDesc * len(meshes))()
    for k, mesh in enumerate(meshes):
        v, idx, mat = mesh[:3]
        extra = mesh[3] if len(mesh) > 3 else {}
        v = np.ascontiguousarray(v, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        keep += [v, idx]
        md[k].vertices = v.ctypes.data
        md[k].n_vertices = len(v)
        md[k].indices = idx.ctypes.data
        md[k].n_triangles = len(idx)
        md[k].material = mat
        md[k].twosided = int(extra.get("twosided", 1))
        md[k].use_smooth_normal = int(extra.get("smooth", 1))
        for key, field, width in (("normals", "vertex_normals", 3), ("texcoords", "texcoords", 2)):
            if extra.get(key) is not None:
                a = np.ascontiguousarray(extra[key], np.float32).reshape(len(v), width)
                keep.append(a)
                setattr(md[k], field, a.ctypes.data)
    mats = (MaterialDesc * len(materials))(*materials)
    keep += [md, mats]
    d = SceneDesc()
    d.meshes = md
    d.n_meshes = len(meshes)
    d.materials = mats
    d.n_materials = len(materials)
    if sky is not None:
        d.sky = sky
    return d, keep


def camera_perspective(camera_to_world, vfov, aspect) -> CameraDesc:
    c = CameraDesc()
    m = (_f32 * 16)(*[float(x) for x in np.asarray(camera_to_world).reshape(16)])
    st = lib.ks_camera_perspective(m, vfov, aspect, ctypes.byref(c))
    if st != KS_OK:
        raise KsError(st, "ks_camera_perspective")
    return c


def camera_orthographic(camera_to_world, left, right, bottom, top, near_clip, far_clip) -> CameraDesc:
    c = CameraDesc()
    m = (_f32 * 16)(*[float(x) for x in np.asarray(camera_to_world).reshape(16)])
    st = lib.ks_camera_orthographic(m, left, right, bottom, top, near_clip, far_clip, ctypes.byref(c))
    if st != KS_OK:
        raise KsError(st, "ks_camera_orthographic")
    return c


def triangle_soup_desc(vertices, indices, material=None):
    """Builds a one-mesh SceneDesc over numpy arrays; returns (desc, keepalive)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
    mesh = MeshDesc(ptr(v), len(v), ptr(i), len(i), None, 0, 1, 1, None)
    mat = material or MaterialDesc((0.8, 0.8, 0.8), 1.0, 0.0, 1.5, 0.5, 0.0, 0.0, 0.5, (0, 0, 0), 0, 0, (0, 0, 0))
    meshes = (MeshDesc * 1)(mesh)
    mats = (MaterialDesc * 1)(mat)
    d = SceneDesc(meshes, 1, mats, 1, SkyDesc())
    return d, (v, i, meshes, mats)


class Scene:
    """A device-resident scene (ks_scene)."""

    def __init__(self, ctx: Context, desc, keepalive=None):
        self.ctx = ctx
        self._keep = keepalive
        h = _vp()
        dp = desc if isinstance(desc, ctypes.POINTER(SceneDesc)) else ctypes.byref(desc)
        ctx.check(lib.ks_scene_create(ctx.handle, dp, ctypes.byref(h)), "ks_scene_create")
        self.handle = h
        ctx._scenes.add(self)

    def build_bvh(self, max_prims=4, buckets=12, trav_weight=1.0, alpha=1e-5) -> float:
        o = SBVHOptions(max_prims, buckets, trav_weight, alpha)
        ms = _f32()
        self.ctx.check(lib.ks_scene_build_bvh(self.handle, ctypes.byref(o), ctypes.byref(ms)), "ks_scene_build_bvh")
        return ms.value

    def export_sbvh(self):
        nn, npr = _u32(), _u32()
        self.ctx.check(lib.ks_sbvh_counts(self.handle, ctypes.byref(nn), ctypes.byref(npr)), "ks_sbvh_counts")
        n, m = nn.value, npr.value
        bounds = np.empty((n, 6), np.float32)
        axis = np.empty(n, np.uint32)
        right = np.empty(n, np.uint32)
        off = np.empty(n, np.uint32)
        prims = np.empty(m, np.uint32)
        self.ctx.check(lib.ks_sbvh_export(self.handle, ptr(bounds), ptr(axis), ptr(right), ptr(off), ptr(prims)),
                       "ks_sbvh_export")
        return dict(bounds=bounds, axis=axis, right=right, prim_offset=off, prims=prims)

    def trace(self, rays, any_hit=False, culling=2, wide=False):
        """ks_trace_rays (wide=True: ks_trace_rays_wide, the renderer's 4-wide traversal)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        tri = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        bary = np.empty((n, 3), np.float32)
        fn, name = (lib.ks_trace_rays_wide, "ks_trace_rays_wide") if wide else (lib.ks_trace_rays, "ks_trace_rays")
        self.ctx.check(fn(self.handle, ptr(rays), n, int(any_hit), culling, ptr(tri), ptr(t), ptr(bary)), name)
        return (tri.astype(bool), None, None) if any_hit else (tri, t, bary)

    def render(self, camera: CameraDesc, params: SmallPTParams, callback=None):
        """ks_small_pt_render into fresh host FP64 buffers; returns (accum [H,W,3], weights [H,W,2])."""
        W, H = params.render_width, params.render_height
        accum = np.zeros((H, W, 3), np.float64)
        weights = np.zeros((H, W, 2), np.float64)
        cb = PROGRESS_FN(0)
        if callback is not None:
            def _cb(spp, a, w, user):
                callback(spp, np.ctypeslib.as_array(a, (H, W, 3)).copy(), np.ctypeslib.as_array(w, (H, W, 2)).copy())
            cb = PROGRESS_FN(_cb)
        self.ctx.check(lib.ks_small_pt_render(self.handle, ctypes.byref(camera), ctypes.byref(params), cb, None,
                                              ptr(accum), ptr(weights)), "ks_small_pt_render")
        return accum, weights

    def render_guided(self, camera: CameraDesc, params: SmallPTParams, guide, options=None, callback=None):
        """ks_small_pt_render_guided into fresh host FP64 buffers (see render)."""
        options = options or GuideRenderOptions.make()
        W, H = params.render_width, params.render_height
        accum = np.zeros((H, W, 3), np.float64)
        weights = np.zeros((H, W, 2), np.float64)
        cb = PROGRESS_FN(0)
        if callback is not None:
            def _cb(spp, a, w, user):
                callback(spp, np.ctypeslib.as_array(a, (H, W, 3)).copy(), np.ctypeslib.as_array(w, (H, W, 2)).copy())
            cb = PROGRESS_FN(_cb)
        self.ctx.check(lib.ks_small_pt_render_guided(self.handle, ctypes.byref(camera), ctypes.byref(params),
                                                     guide.handle, ctypes.byref(options), cb, None, ptr(accum),
                                                     ptr(weights)), "ks_small_pt_render_guided")
        return accum, weights

    def render_guided_device(self, camera: CameraDesc, params: SmallPTParams, guide, options, accum_ptr: int,
                             weights_ptr: int):
        self.ctx.check(lib.ks_small_pt_render_guided_device(self.handle, ctypes.byref(camera), ctypes.byref(params),
                                                            guide.handle, ctypes.byref(options),
                                                            ctypes.c_void_p(accum_ptr), ctypes.c_void_p(weights_ptr)),
                       "ks_small_pt_render_guided_device")

    def render_device_progress(self, camera: CameraDesc, params: SmallPTParams, accum_ptr: int, weights_ptr: int,
                               callback, guide=None, options=None):
        """ks_small_pt_render_device_progress: callback(spp_done) after every pass; a true return
        value stops the render."""
        if guide is not None and options is None:
            options = GuideRenderOptions.make()
        cb = DEVICE_PROGRESS_FN(lambda spp, user: int(bool(callback(spp))))
        self.ctx.check(lib.ks_small_pt_render_device_progress(
            self.handle, ctypes.byref(camera), ctypes.byref(params), guide.handle if guide is not None else None,
            ctypes.byref(options) if options is not None else None, cb, None, ctypes.c_void_p(accum_ptr),
            ctypes.c_void_p(weights_ptr)), "ks_small_pt_render_device_progress")

    def render_device(self, camera: CameraDesc, params: SmallPTParams, accum_ptr: int, weights_ptr: int):
        self.ctx.check(lib.ks_small_pt_render_device(self.handle, ctypes.byref(camera), ctypes.byref(params),
                                                     ctypes.c_void_p(accum_ptr), ctypes.c_void_p(weights_ptr)),
                       "ks_small_pt_render_device")

    def stats(self) -> RenderStats:
        s = RenderStats()
        self.ctx.check(lib.ks_render_stats_last(self.handle, ctypes.byref(s)), "ks_render_stats_last")
        return s

    def close(self):
        if self.handle:
            lib.ks_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# Learned guiding network (ks_guide_*)
# ---------------------------------------------------------------------------------------------
GUIDE_LEVELS = 16
GUIDE_TABLE_SIZE = 1 << 19
GUIDE_WEIGHTS = 19456
GUIDE_OUTPUTS = 41
GUIDE_LAYERS = [(64, 64), (64, 64), (64, 64), (64, 64), (48, 64)]  # (out, in) of each W; 41 of 48 rows used


class GuideParams(ctypes.Structure):
    _fields_ = [("bound", _f32 * 6), ("base_res", _f32), ("max_res", _f32), ("learning_rate", _f32),
                ("alpha_max", _f32), ("seed", ctypes.c_uint64)]


_sig("ks_guide_create", [_vp, ctypes.POINTER(GuideParams), ctypes.POINTER(_vp)])
_sig("ks_guide_destroy", [_vp], None)
_sig("ks_guide_level_res", [_vp, _vp])
_sig("ks_guide_get_weights", [_vp, _vp, _vp])
_sig("ks_guide_last_loss", [_vp, _vp])
_sig("ks_guide_set_weights", [_vp, _vp, _vp])
_sig("ks_guide_infer", [_vp, _vp, _vp, _vp, _u32, _vp])
_sig("ks_guide_gradients", [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, ctypes.c_int, _vp, _vp, _vp])


class GuideRenderOptions(ctypes.Structure):
    _fields_ = [("guide_from_pass", _i32), ("train_passes", _i32),
                ("max_records", _u32), ("train_batch", _u32), ("record_bounces", _i32), ("min_roughness", _f32)]

    @staticmethod
    def make(**kw):
        o = GuideRenderOptions()
        lib.ks_guide_render_options_default(ctypes.byref(o))
        for k, v in kw.items():
            if not hasattr(o, k):
                raise AttributeError(k)
            setattr(o, k, v)
        return o


_sig("ks_guide_render_options_default", [ctypes.POINTER(GuideRenderOptions)], None)
_sig("ks_small_pt_render_guided", [_vp, ctypes.POINTER(CameraDesc), ctypes.POINTER(SmallPTParams), _vp,
                                   ctypes.POINTER(GuideRenderOptions), PROGRESS_FN, _vp, _vp, _vp])
_sig("ks_small_pt_render_guided_device", [_vp, ctypes.POINTER(CameraDesc), ctypes.POINTER(SmallPTParams), _vp,
                                          ctypes.POINTER(GuideRenderOptions), _vp, _vp])
_sig("ks_small_pt_render_device_progress", [_vp, ctypes.POINTER(CameraDesc), ctypes.POINTER(SmallPTParams), _vp,
                                            _vp, DEVICE_PROGRESS_FN, _vp, _vp, _vp])


def split_guide_weights(flat):
    """Splits the flat weight vector into the per-layer [out][in] matrices (views)."""
    out, o = [], 0
    for n, k in GUIDE_LAYERS:
        out.append(flat[o:o + n * k].reshape(n, k))
        o += n * k
    return out


class Guide:
    """The guiding network (ks_guide): hash grid + MLP + vMF mixture head, trained with Adam."""

    def __init__(self, ctx: Context, bound, base_res=16.0, max_res=2048.0, learning_rate=1e-2, alpha_max=0.8,
                 seed=1):
        self.ctx = ctx
        p = GuideParams()
        p.bound[:] = [float(x) for x in bound]
        p.base_res, p.max_res, p.learning_rate, p.alpha_max, p.seed = base_res, max_res, learning_rate, alpha_max, seed
        h = _vp()
        ctx.check(lib.ks_guide_create(ctx.handle, ctypes.byref(p), ctypes.byref(h)), "ks_guide_create")
        self.handle = h
        ctx._scenes.add(self)

    def level_res(self) -> np.ndarray:
        r = np.empty(GUIDE_LEVELS, np.uint32)
        self.ctx.check(lib.ks_guide_level_res(self.handle, ptr(r)), "ks_guide_level_res")
        return r

    def last_loss(self) -> float:
        out = np.zeros(1, np.float64)
        self.ctx.check(lib.ks_guide_last_loss(self.handle, ptr(out)), "ks_guide_last_loss")
        return float(out[0])

    def get_weights(self, grid=True):
        w = np.empty(GUIDE_WEIGHTS, np.float32)
        g = np.empty((GUIDE_LEVELS, GUIDE_TABLE_SIZE, 2), np.float32) if grid else None
        self.ctx.check(lib.ks_guide_get_weights(self.handle, ptr(w), ptr(g)), "ks_guide_get_weights")
        return w, g

    def set_weights(self, w=None, grid=None):
        w = None if w is None else np.ascontiguousarray(w, np.float32)
        grid = None if grid is None else np.ascontiguousarray(grid, np.float32)
        self.ctx.check(lib.ks_guide_set_weights(self.handle, ptr(w), ptr(grid)), "ks_guide_set_weights")

    def infer(self, pos, wo, normal) -> np.ndarray:
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
        normal = np.ascontiguousarray(normal, np.float32).reshape(-1, 3)
        out = np.empty((len(pos), GUIDE_OUTPUTS), np.float32)
        self.ctx.check(lib.ks_guide_infer(self.handle, ptr(pos), ptr(wo), ptr(normal), len(pos), ptr(out)),
                       "ks_guide_infer")
        return out

    def gradients(self, pos, wo, normal, wi, target, bsdf_pdf=None, apply_adam=False, want_grads=True):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
        normal = np.ascontiguousarray(normal, np.float32).reshape(-1, 3)
        wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
        target = np.ascontiguousarray(target, np.float32).reshape(-1)
        pb = None if bsdf_pdf is None else np.ascontiguousarray(bsdf_pdf, np.float32).reshape(-1)
        loss = np.zeros(1, np.float64)
        gw = np.empty(GUIDE_WEIGHTS, np.float32) if want_grads else None
        gg = np.empty((GUIDE_LEVELS, GUIDE_TABLE_SIZE, 2), np.float32) if want_grads else None
        self.ctx.check(lib.ks_guide_gradients(self.handle, ptr(pos), ptr(wo), ptr(normal), ptr(wi), ptr(target), ptr(pb),
                                              len(pos), int(apply_adam), ptr(loss), ptr(gw), ptr(gg)),
                       "ks_guide_gradients")
        return float(loss[0]), gw, gg

    def train_step(self, pos, wo, normal, wi, target, bsdf_pdf=None) -> float:
        return self.gradients(pos, wo, normal, wi, target, bsdf_pdf, apply_adam=True, want_grads=False)[0]

    def close(self):
        if self.handle:
            lib.ks_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# TOML tasks (ks_config_*)
# ---------------------------------------------------------------------------------------------
_sig("ks_config_run", [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p])
_sig("ks_config_last_error", [], ctypes.c_char_p)
_sig("ks_config_parse", [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)])


def config_parse(text: str) -> str:
    """Normalised form of a TOML task document (raises KsError with the line on errors)."""
    n = ctypes.c_size_t()
    st = lib.ks_config_parse(text.encode(), None, 0, ctypes.byref(n))
    if st != KS_OK:
        raise KsError(st, lib.ks_config_last_error().decode())
    buf = ctypes.create_string_buffer(n.value + 1)
    lib.ks_config_parse(text.encode(), buf, n.value + 1, None)
    return buf.value.decode()


def config_run(text: str, output_dir: str, asset_root: str = None):
    """Runs every [[task]] of a TOML document (ks_config_run)."""
    st = lib.ks_config_run(text.encode(), asset_root.encode() if asset_root else None, output_dir.encode())
    if st != KS_OK:
        raise KsError(st, lib.ks_config_last_error().decode())


def read_pfm(path):
    """RGB PFM file -> float32 array [H, W, 3] (top row first)."""
    with open(path, "rb") as f:
        magic = f.readline().strip()
        w, h = (int(x) for x in f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4")
    assert magic == b"PF"
    return data.reshape(h, w, 3)[::-1].astype(np.float32)


_sig("ks_image_save_exr", [ctypes.c_char_p, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32])
_sig("ks_image_load_rgb", [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(_f32)), ctypes.POINTER(ctypes.c_int32),
                           ctypes.POINTER(ctypes.c_int32)])
_sig("ks_image_free", [ctypes.POINTER(_f32)], None)


def save_exr(path, pixels, half=False):
    """float array [H, W, C] (C = 1..4, R G B A) -> OpenEXR file (ks_image_save_exr)."""
    a = np.ascontiguousarray(pixels, np.float32)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, c = a.shape
    st = lib.ks_image_save_exr(str(path).encode(), a.ctypes.data, w, h, c, int(half))
    if st != KS_OK:
        raise KsError(st, lib.ks_config_last_error().decode())


def load_image(path) -> np.ndarray:
    """RGB pixels of an .exr, .hdr or .pfm file -> float32 [H, W, 3] (ks_image_load_rgb)."""
    buf = ctypes.POINTER(_f32)()
    w, h = ctypes.c_int32(), ctypes.c_int32()
    st = lib.ks_image_load_rgb(str(path).encode(), ctypes.byref(buf), ctypes.byref(w), ctypes.byref(h))
    if st != KS_OK:
        raise KsError(st, lib.ks_config_last_error().decode())
    try:
        return np.ctypeslib.as_array(buf, shape=(h.value, w.value, 3)).copy()
    finally:
        lib.ks_image_free(buf)


_sig("ks_texture_load", [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                         ctypes.POINTER(TextureDesc)])
_sig("ks_texture_free", [ctypes.POINTER(TextureDesc)], None)


def load_texture(path, channels, srgb=False, keep_16bit=False):
    """A texture file (ks_texture_load) -> (array [H, W, channels] of uint8, uint16 or float32, srgb),
    the form attach_textures takes."""
    t = TextureDesc()
    st = lib.ks_texture_load(str(path).encode(), int(channels), int(srgb), int(keep_16bit), ctypes.byref(t))
    if st != KS_OK:
        raise KsError(st, lib.ks_config_last_error().decode())
    try:
        dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[t.format]
        n = t.height * t.width * t.channels
        buf = ctypes.cast(t.texels, ctypes.POINTER({0: ctypes.c_uint8, 1: ctypes.c_uint16, 2: _f32}[t.format]))
        a = np.ctypeslib.as_array(buf, shape=(n,)).astype(dt, copy=True)
        return a.reshape(t.height, t.width, t.channels), bool(t.srgb)
    finally:
        lib.ks_texture_free(ctypes.byref(t))


# ---------------------------------------------------------------------------------------------
# Batched rendering (ks_batch_*)
# ---------------------------------------------------------------------------------------------
class BatchJob(ctypes.Structure):
    _fields_ = [("scene", _vp), ("camera", CameraDesc), ("params", SmallPTParams), ("accum_rgb_device", _vp),
                ("weights_device", _vp)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("capacity", _u32), ("grid_per_sm", _u32), ("use_graph", _i32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("extension_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("iterations", _u32), ("graph_launches", _u32), ("ms_total", _f32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_sig("ks_batch_render_device", [_vp, ctypes.POINTER(BatchJob), _u32, ctypes.POINTER(BatchOptions),
                                ctypes.POINTER(BatchStats)])
_sig("ks_batch_autotune", [_vp, ctypes.POINTER(BatchJob), _u32, ctypes.POINTER(BatchOptions),
                           ctypes.POINTER(_f32)])


def _batch_jobs(jobs):
    arr = (BatchJob * len(jobs))()
    for k, (scene, camera, params, acc_ptr, wts_ptr) in enumerate(jobs):
        arr[k].scene = scene.handle
        arr[k].camera = camera
        arr[k].params = params
        arr[k].accum_rgb_device = acc_ptr
        arr[k].weights_device = wts_ptr
    return arr


def batch_render(ctx: Context, jobs, capacity=0, grid_per_sm=0, use_graph=True) -> BatchStats:
    """ks_batch_render_device; jobs = [(Scene, CameraDesc, SmallPTParams, accum_ptr, weights_ptr)]
    with device buffers (raw pointers)."""
    arr = _batch_jobs(jobs)
    o = BatchOptions(capacity, grid_per_sm, int(bool(use_graph)))
    st = BatchStats()
    ctx.check(lib.ks_batch_render_device(ctx.handle, arr, len(jobs), ctypes.byref(o), ctypes.byref(st)),
              "ks_batch_render_device")
    return st


def batch_autotune(ctx: Context, jobs, use_graph=True):
    """ks_batch_autotune: returns (BatchOptions, ms of the best sample run)."""
    arr = _batch_jobs(jobs)
    o = BatchOptions(0, 0, int(bool(use_graph)))
    ms = _f32()
    ctx.check(lib.ks_batch_autotune(ctx.handle, arr, len(jobs), ctypes.byref(o), ctypes.byref(ms)),
              "ks_batch_autotune")
    return o, ms.value
