"""ctypes binding of the ORACLE (oracle/liboracle.so, oracle/_ref/libksref_sbvh.so).

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
this; the product never does.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libksref_sbvh.so")

_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32


def P(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


# Mirrors of include/ks_b200.h's camera and render-parameter structs, so that CPU-only callers of
# the oracle (bench.py's reference arm) need not load the CUDA library.
class CameraDesc(ctypes.Structure):
    _fields_ = [("camera_to_world", ctypes.c_float * 16), ("proj_to_camera", ctypes.c_float * 16),
                ("proj_to_world", ctypes.c_float * 16), ("orthographic", ctypes.c_int32)]


class SmallPTParams(ctypes.Structure):
    _fields_ = [("include_background", ctypes.c_int32), ("backdrop", ctypes.c_float * 3),
                ("bounces", ctypes.c_int32), ("render_width", ctypes.c_int32), ("render_height", ctypes.c_int32),
                ("crop_start_x", ctypes.c_int32), ("crop_start_y", ctypes.c_int32), ("crop_width", ctypes.c_int32),
                ("crop_height", ctypes.c_int32), ("spp", ctypes.c_int32), ("rng_seed", ctypes.c_int32),
                ("scale_ray_diff", ctypes.c_int32), ("clamp_direct", ctypes.c_float),
                ("clamp_indirect", ctypes.c_float), ("spp_prog_interval", ctypes.c_int32),
                ("pixel_filter_width", ctypes.c_float), ("pixel_filter", ctypes.c_int32),
                ("pixel_filter_sigma", ctypes.c_float)]


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(ORACLE_SO)
        L = self.lib
        L.oracle_sobol_points.argtypes = [_u32] * 11 + [_vp]
        L.oracle_sobol_points.restype = ctypes.c_int
        L.oracle_sobol_matrices01.argtypes = [_vp]
        L.oracle_sobol_matrices01.restype = None

        L.oracle_scene_create.argtypes = [_vp, _vp]
        L.oracle_scene_create.restype = _vp
        L.oracle_scene_destroy.argtypes = [_vp]
        L.oracle_scene_destroy.restype = None
        L.oracle_light_table.argtypes = [_vp, _vp, _vp]
        L.oracle_light_table.restype = _u32
        L.oracle_sky_tables.argtypes = [_vp, _vp, _vp]
        L.oracle_render.argtypes = [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]
        L.oracle_render_range.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp]
        L.oracle_render_range.restype = ctypes.c_int
        L.oracle_sky_sample.argtypes = [_vp, _vp, _u32, _vp, _vp, _vp]
        L.oracle_sky_sample.restype = ctypes.c_int
        L.oracle_sky_eval.argtypes = [_vp, _vp, _u32, _vp, _vp]
        L.oracle_sky_eval.restype = ctypes.c_int
        L.oracle_bsdf_eval.argtypes = [_vp, _vp, _vp, _u32, _vp, _vp]
        L.oracle_bsdf_eval.restype = None
        L.oracle_bsdf_sample.argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp]
        L.oracle_bsdf_sample.restype = None
        L.oracle_generate.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_int, _u32, _u32, _u32, _u32]
        L.oracle_generate.restype = _vp
        L.oracle_generated_desc.argtypes = [_vp]
        L.oracle_generated_desc.restype = _vp
        L.oracle_generated_camera.argtypes = [_vp, _vp, _vp, _vp]
        L.oracle_generated_camera.restype = None
        L.oracle_generated_destroy.argtypes = [_vp]
        L.oracle_generated_destroy.restype = None
        L.oracle_camera_perspective.argtypes = [_vp, ctypes.c_float, ctypes.c_float, _vp]
        L.oracle_camera_perspective.restype = ctypes.c_int
        L.oracle_params_default.argtypes = [_vp]
        L.oracle_params_default.restype = None

    def generate(self, kind, seed=0, level=8, roughness=(0.05, 1.0), occluder=False, sky=(2048, 1024),
                 resolution=(1024, 1024)):
        """A seeded synthetic scene (the library's generator, compiled into the oracle library) with
        its camera: (OracleGenerated, CameraDesc)."""
        return OracleGenerated(self, kind, seed, level, roughness, occluder, sky, resolution)

    def params(self, **kw):
        """SmallPTParams with the small_pt task's defaults, then the given fields."""
        p = SmallPTParams()
        self.lib.oracle_params_default(ctypes.byref(p))
        for k, v in kw.items():
            if k == "backdrop":
                p.backdrop[:] = v
            else:
                setattr(p, k, v)
        return p

    def scene(self, desc, keepalive=None):
        return OracleScene(self, desc, keepalive)

    def bsdf_eval(self, material, wo, wi):
        wo = np.ascontiguousarray(wo, np.float32)
        wi = np.ascontiguousarray(wi, np.float32)
        n = len(wo)
        f = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.lib.oracle_bsdf_eval(ctypes.byref(material), P(wo), P(wi), n, P(f), P(pdf))
        return f, pdf

    def bsdf_sample(self, material, wo, u):
        wo = np.ascontiguousarray(wo, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        n = len(wo)
        wi = np.empty((n, 3), np.float32)
        beta = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.lib.oracle_bsdf_sample(ctypes.byref(material), P(wo), P(u), n, P(wi), P(beta), P(pdf))
        return wi, beta, pdf

    def sobol_points(self, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd):
        out = np.empty((ny, nx, ns, nd, 3), dtype=np.float32)
        self.lib.oracle_sobol_points(full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd, P(out))
        return out

    def sobol_matrices01(self):
        out = np.empty(104, dtype=np.uint32)
        self.lib.oracle_sobol_matrices01(P(out))
        return out


class OracleScene:
    """CPU restatement of the small_pt scene + render (oracle/src/o_small_pt.cpp)."""

    def __init__(self, oracle, desc, keepalive=None):
        self.o = oracle
        self._keep = keepalive
        if isinstance(desc, (int, _vp)):
            dp = desc
        elif isinstance(desc, ctypes._Pointer):
            dp = ctypes.cast(desc, _vp)
        else:
            dp = ctypes.cast(ctypes.pointer(desc), _vp)
        self.h = oracle.lib.oracle_scene_create(dp, None)
        assert self.h, "oracle_scene_create failed"

    def light_table(self):
        n = self.o.lib.oracle_light_table(self.h, None, None)
        powers = np.empty(n, np.float32)
        cdf = np.empty(n + 1, np.float32)
        self.o.lib.oracle_light_table(self.h, P(powers), P(cdf))
        return powers, cdf

    def sky_tables(self, w, h):
        cond = np.empty((h, w + 1), np.float32)
        margin = np.empty(h + 1, np.float32)
        assert self.o.lib.oracle_sky_tables(self.h, P(cond), P(margin)) == 0
        return cond, margin

    def render(self, camera, params, threads=None):
        W, H = params.render_width, params.render_height
        accum = np.zeros((H, W, 3), np.float64)
        weights = np.zeros((H, W, 2), np.float64)
        counts = np.zeros(2, np.uint64)
        threads = threads or os.cpu_count() or 1
        self.o.lib.oracle_render(self.h, ctypes.byref(camera), ctypes.byref(params), P(accum), P(weights),
                                 threads, P(counts))
        return accum, weights, counts

    def sky_sample(self, u):
        """The sky light's sample for each row of u (n x 2): (wi [n, 3], pdf [n], Le / pdf [n, 3])."""
        u = np.ascontiguousarray(u, np.float32)
        n = len(u)
        wi, pdf, lb = np.empty((n, 3), np.float32), np.empty(n, np.float32), np.empty((n, 3), np.float32)
        assert self.o.lib.oracle_sky_sample(self.h, P(u), n, P(wi), P(pdf), P(lb)) == 0
        return wi, pdf, lb

    def sky_eval(self, wi):
        """The sky light's pdf [n] and radiance [n, 3] in the directions wi (n x 3)."""
        wi = np.ascontiguousarray(wi, np.float32)
        n = len(wi)
        pdf, le = np.empty(n, np.float32), np.empty((n, 3), np.float32)
        assert self.o.lib.oracle_sky_eval(self.h, P(wi), n, P(pdf), P(le)) == 0
        return pdf, le

    def render_range(self, camera, params, s_begin, s_end, threads=None, count_work=False, accum=None,
                     weights=None):
        """Samples [s_begin, s_end) of the params.spp samples per pixel, accumulated into accum /
        weights (fresh zero arrays when None).  Returns (accum, weights, counts, work): counts =
        (extension, shadow) queries; work (count_work) = dict of the queries' nodes and triangles
        counted by the restatement of the reference traversal, and its disagreements with the
        reference's own queries."""
        W, H = params.render_width, params.render_height
        if accum is None:
            accum = np.zeros((H, W, 3), np.float64)
        if weights is None:
            weights = np.zeros((H, W, 2), np.float64)
        counts = np.zeros(2, np.uint64)
        work = np.zeros(7, np.uint64) if count_work else None
        threads = threads or os.cpu_count() or 1
        st = self.o.lib.oracle_render_range(self.h, ctypes.byref(camera), ctypes.byref(params), s_begin, s_end,
                                            P(accum), P(weights), threads, P(counts), P(work))
        assert st == 0, "oracle_render_range: bad sample range"
        wd = None
        if count_work:
            wd = dict(ext_nodes=int(work[0]), ext_tris=int(work[1]), ext_overflows=int(work[2]),
                      shadow_nodes=int(work[3]), shadow_tris=int(work[4]), shadow_overflows=int(work[5]),
                      mismatches=int(work[6]))
        return accum, weights, counts, wd

    def __del__(self):
        try:
            self.o.lib.oracle_scene_destroy(self.h)
        except Exception:
            pass


class OracleGenerated:
    def __init__(self, oracle, kind, seed, level, roughness, occluder, sky, resolution):
        self.o = oracle
        self.h = oracle.lib.oracle_generate(kind.encode(), seed, level, roughness[0], roughness[1], int(occluder),
                                            sky[0], sky[1], resolution[0], resolution[1])
        assert self.h, f"oracle_generate({kind}) failed"
        self.desc = oracle.lib.oracle_generated_desc(self.h)
        c2w = (ctypes.c_float * 16)()
        vfov, aspect = ctypes.c_float(), ctypes.c_float()
        oracle.lib.oracle_generated_camera(self.h, c2w, ctypes.byref(vfov), ctypes.byref(aspect))
        self.camera = CameraDesc()
        assert oracle.lib.oracle_camera_perspective(c2w, vfov.value, aspect.value, ctypes.byref(self.camera)) == 0

    def __del__(self):
        try:
            self.o.lib.oracle_generated_destroy(self.h)
        except Exception:
            pass


class RefSBVH:
    """The reference's own SBVH builder + traversal (cuda/sbvh.cu), compiled host-side."""

    def __init__(self):
        self.lib = ctypes.CDLL(REF_SO)
        L = self.lib
        L.ksref_sbvh_build.argtypes = [_vp, _u32, _vp, _u32, _u32, _u32, ctypes.c_float, ctypes.c_float,
                                       ctypes.POINTER(_vp), ctypes.POINTER(_u32), ctypes.POINTER(_u32)]
        L.ksref_sbvh_export.argtypes = [_vp] * 6
        L.ksref_sbvh_intersect.argtypes = [_vp, _vp, _u32, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int]
        L.ksref_sbvh_destroy.argtypes = [_vp]
        L.ksref_tri_test.argtypes = [_vp, _vp, _vp, _u32, _vp, _vp]
        L.ksref_tri_test.restype = None

    def build(self, verts, idx, max_prims=4, buckets=12, trav_weight=1.0, alpha=1e-5):
        verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(idx, dtype=np.uint32).reshape(-1)
        h, nn, npr = _vp(), _u32(), _u32()
        st = self.lib.ksref_sbvh_build(P(verts), len(verts), P(idx), len(idx) // 3, max_prims, buckets,
                                       trav_weight, alpha, ctypes.byref(h), ctypes.byref(nn), ctypes.byref(npr))
        assert st == 0
        n, m = nn.value, npr.value
        bounds = np.empty((n, 6), np.float32)
        axis = np.empty(n, np.uint32)
        right = np.empty(n, np.uint32)
        off = np.empty(n, np.uint32)
        prims = np.empty(m, np.uint32)
        self.lib.ksref_sbvh_export(h, P(bounds), P(axis), P(right), P(off), P(prims))
        return RefTree(self, h, bounds, axis, right, off, prims)


class RefTree:
    def __init__(self, owner, h, bounds, axis, right, off, prims):
        self.owner, self.h = owner, h
        self.bounds, self.axis, self.right, self.prim_offset, self.prims = bounds, axis, right, off, prims

    def intersect(self, rays, any_hit=False, culling=2, threads=8):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        tri = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        bary = np.empty((n, 3), np.float32)
        self.owner.lib.ksref_sbvh_intersect(self.h, P(rays), n, int(any_hit), culling, P(tri), P(t), P(bary),
                                            threads)
        return (tri.astype(bool), None, None) if any_hit else (tri, t, bary)

    def tri_test(self, rays, tri):
        """The reference's watertight test of triangle tri[i] against ray i: (hit [n] bool, t [n])."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        tri = np.ascontiguousarray(tri, dtype=np.uint32)
        n = len(rays)
        t = np.zeros(n, np.float32)
        hit = np.zeros(n, np.uint32)
        self.owner.lib.ksref_tri_test(self.h, P(rays), P(tri), n, P(t), P(hit))
        return hit.astype(bool), t

    def __del__(self):
        try:
            self.owner.lib.ksref_sbvh_destroy(self.h)
        except Exception:
            pass


_oracle = None


def load():
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


def ref_sbvh():
    return RefSBVH()
