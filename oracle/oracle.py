"""TEST INFRASTRUCTURE: ctypes access to the CPU oracles.

* ``liboracle.so`` -- the C restatement of the reference's GPU builders
  (engine/gpu/shaders/trace/trace_build.wgsl, trace_ploc.wgsl; engine/gpu/trace_gpu.c:546-805).
* ``_ref/libref_f.so`` / ``_ref/libref_d.so`` -- the reference's own CPU engine (float and
  double builds) with ``ref_bridge.c``: ``scene_intersect`` (engine/rt/accel.c:252),
  ``trace_image`` (engine/rt/tracer.c:329), ``triangle_bounds`` (engine/scene/scene.c:65).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this module,
always as the checker or the timed CPU baseline, never as the product path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")


def build():
    """Builds liboracle.so and, where the reference sources are present, _ref/*.so."""
    import subprocess
    make = ["make", "-s", "-C", HERE, "all"]
    ref = os.environ.get("LR_REFERENCE", "/root/reference")   # the reference's checkout, where present
    if os.path.isfile(os.path.join(ref, "engine", "rt", "tracer.c")):
        make.append(f"REF={ref}")
    subprocess.run(make, check=True)


def _load(name):
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        raise RuntimeError(f"oracle library {path} is not built (make -C oracle)")
    lib = C.CDLL(path)
    _libs[name] = lib
    return lib


def oracle_lib():
    lib = _load("liboracle.so")
    if not getattr(lib, "_typed", False):
        lib.or_params.argtypes = [_f32p, _f32p, _f32p, _f32p]
        lib.or_morton.argtypes = [_f32p, C.c_int, _f32p, _f32p, C.c_int, _u32p]
        lib.or_bitonic.argtypes = [_u32p, C.c_uint32, C.c_int]
        lib.or_lbvh.argtypes = [_f32p, C.c_int, _f32p, _f32p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                _u32p, _u32p, C.c_void_p]
        lib.or_ploc.argtypes = [_f32p, C.c_int, _f32p, _f32p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_int, _u32p, _u32p]
        lib.or_check_tree.argtypes = [_u32p, C.c_int, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.or_trace_tree.argtypes = [_u32p, _u32p, C.c_uint32, _f32p, _f32p, _f32p, C.c_longlong, C.c_float,
                                      C.c_float, _i32p, _f32p, _i64p]
        lib.or_refit.argtypes = [_u32p, C.c_int, _u32p, C.c_uint32, _f32p, C.c_int]
        lib._typed = True
    return lib


def pow2_at_least(n):
    p = 2
    while p < n:
        p <<= 1
    return p


def params(bounds_lo, bounds_hi):
    """build_queue's lo and ext = 1 / extent (0 on a flat axis), trace_gpu.c:605-611."""
    lo = np.zeros(3, np.float32)
    ext = np.zeros(3, np.float32)
    oracle_lib().or_params(np.ascontiguousarray(bounds_lo, np.float32), np.ascontiguousarray(bounds_hi, np.float32),
                           lo, ext)
    return lo, ext


def morton(boxes, lo, ext, bits=30):
    n = boxes.shape[0]
    p = pow2_at_least(n)
    w = 3 if bits == 63 else 2
    keys = np.zeros(p * w, np.uint32)
    oracle_lib().or_morton(np.ascontiguousarray(boxes, np.float32).reshape(-1), n, lo, ext, bits, keys)
    return keys.reshape(p, w)


def bitonic(keys, bits=30):
    k = np.ascontiguousarray(keys, np.uint32).copy()
    oracle_lib().or_bitonic(k.reshape(-1), k.shape[0], bits)
    return k


def lbvh(boxes, lo, ext, bits=30, node0=0, ref0=0, ref_add=0, want_keys=False):
    """The reference LBVH (morton, bitonic sort, hier, leaves, up). nodes: (node0 + 2n - 1, 8) u32."""
    n = boxes.shape[0]
    nodes = np.zeros((node0 + max(2 * n - 1, 1), 8), np.uint32)
    aux = np.zeros(ref0 + n, np.uint32)
    w = 3 if bits == 63 else 2
    keys = np.zeros(pow2_at_least(n) * w, np.uint32) if want_keys else None
    rc = oracle_lib().or_lbvh(np.ascontiguousarray(boxes, np.float32).reshape(-1), n, lo, ext, bits, node0, ref0,
                              ref_add, nodes.reshape(-1), aux, keys.ctypes.data if want_keys else None)
    if rc:
        raise MemoryError("or_lbvh")
    return (nodes, aux, keys.reshape(-1, w)) if want_keys else (nodes, aux)


def ploc(boxes, lo, ext, bits=30, node0=0, ref0=0, ref_add=0, small=1024):
    """The reference PLOC (morton, bitonic, leaves, init/nn/mark/top/scatter rounds, small)."""
    n = boxes.shape[0]
    nodes = np.zeros((node0 + 2 * n - 1, 8), np.uint32)
    aux = np.zeros(ref0 + n, np.uint32)
    rc = oracle_lib().or_ploc(np.ascontiguousarray(boxes, np.float32).reshape(-1), n, lo, ext, bits, node0, ref0,
                              ref_add, small, nodes.reshape(-1), aux)
    if rc:
        raise ValueError("or_ploc: n < 3 or out of memory")
    return nodes, aux


def refit(nodes, aux, boxes, ref_add=0):
    """bvh_refit_boxes (bvh.c:471-485) restated for a GPU-layout tree (root at node 0): a copy of
    nodes with every box made again for the items' new boxes (n x 8 floats)."""
    out = np.array(nodes, np.uint32, copy=True).reshape(-1, 8)
    boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 8)
    ok = oracle_lib().or_refit(out.reshape(-1), out.shape[0], np.ascontiguousarray(aux, np.uint32), ref_add,
                               boxes.reshape(-1), boxes.shape[0])
    if not ok:
        raise ValueError("or_refit: not a tree over these items")
    return out


def ref_bvh_refit(boxes, moved):
    """The reference's own refit: bvh_build_boxes (SAH, leaves of up to 4) over boxes, then
    bvh_refit_boxes for moved. Returns (nodes in the GPU layout, refs, cost)."""
    boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 8)
    moved = np.ascontiguousarray(moved, np.float32).reshape(-1, 8)
    n = boxes.shape[0]
    nodes = np.zeros((2 * n - 1, 8), np.uint32)
    refs = np.zeros(n, np.uint32)
    cost = C.c_float()
    nn = ref_lib().rb_bvh_refit(boxes.reshape(-1), moved.reshape(-1), n, nodes.reshape(-1), refs, C.byref(cost))
    return nodes[:nn], refs, cost.value


def check_tree(nodes, n, node0=0):
    cost = C.c_double()
    depth = C.c_int()
    ok = oracle_lib().or_check_tree(np.ascontiguousarray(nodes, np.uint32).reshape(-1), n, node0, C.byref(cost),
                                    C.byref(depth))
    return bool(ok), cost.value, depth.value


def trace_tree(nodes, aux, tris_quv, orig, dirs, tmin=0.0, tmax=1e30, node0=0):
    """Closest hit through a built binary tree; returns prim, t, (box tests, triangle tests)."""
    n = orig.shape[0]
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    counts = np.zeros(2, np.int64)
    oracle_lib().or_trace_tree(np.ascontiguousarray(nodes, np.uint32).reshape(-1),
                               np.ascontiguousarray(aux, np.uint32), node0,
                               np.ascontiguousarray(tris_quv, np.float32).reshape(-1),
                               np.ascontiguousarray(orig, np.float32).reshape(-1),
                               np.ascontiguousarray(dirs, np.float32).reshape(-1), n, tmin, tmax, prim, t, counts)
    return prim, t, counts


# ---- the reference's own CPU engine ---------------------------------------------------------------------
def ref_lib(double=False, gpu=False):
    """The reference's CPU engine (float, or double); gpu: the float build linked with the engine's
    gpu_frame.c and the CUDA backend (shim/gpu_cuda.c on liblrc), for the drop-in checks."""
    name = os.path.join("_ref", "libref_gpu.so" if gpu else ("libref_d.so" if double else "libref_f.so"))
    lib = _load(name)
    if gpu and not getattr(lib, "_gpu_typed", False):
        lib.rb_gpu_frame_trace.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_int, _f32p]
        lib.rb_scene_tree.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib._gpu_typed = True
    if not getattr(lib, "_typed", False):
        vp = C.c_void_p
        lib.rb_scene_new.restype = vp
        lib.rb_scene_free.argtypes = [vp]
        lib.rb_add_material.argtypes = [vp, C.c_int, _f32p, _f32p, C.c_float, C.c_float, C.c_float, C.c_float]
        lib.rb_add_material_preset.argtypes = [vp, C.c_int, _f32p, C.c_float, C.c_float]
        lib.rb_add_triangles.argtypes = [vp, _f32p, _i32p, C.c_int]
        lib.rb_add_quad.argtypes = [vp, _f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.rb_add_sphere.argtypes = [vp, _f32p, C.c_float, C.c_int]
        lib.rb_add_mesh.argtypes = [vp, _f32p, _i32p, C.c_int]
        lib.rb_add_instance.argtypes = [vp, C.c_int, _f32p, C.c_int]
        lib.rb_move_instance.argtypes = [vp, C.c_int, _f32p]
        lib.rb_update_instances.argtypes = [vp]
        lib.rb_bvh_refit.argtypes = [_f32p, _f32p, C.c_int, _u32p, _u32p, C.POINTER(C.c_float)]
        lib.rb_instance_data.argtypes = [vp, C.c_int, _f32p, _f32p]
        lib.rb_mesh_box.argtypes = [vp, C.c_int, _f32p]
        lib.rb_set_env.argtypes = [vp, _f32p, C.c_int, C.c_int]
        lib.rb_set_accel.argtypes = [vp]
        lib.rb_tri_data.argtypes = [vp, _f32p, C.c_void_p]
        lib.rb_num_tris.argtypes = [vp]
        lib.rb_num_prims.argtypes = [vp]
        lib.rb_triangle_bounds.argtypes = [_f32p, C.c_int, _f32p]
        lib.rb_intersect.argtypes = [vp, _f32p, _f32p, C.c_longlong, C.c_float, C.c_float, _i32p, _i32p, _f32p]
        lib.rb_occluded.argtypes = [vp, _f32p, _f32p, C.c_longlong, C.c_float, C.c_float, _i32p]
        lib.rb_trace_image.argtypes = [vp, _f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        lib.rb_set_indirect_clamp.argtypes = [C.c_float]
        lib.rb_volume_majorants.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.rb_srgb_table.argtypes = [_f32p]
        lib.rb_add_texmap.argtypes = [vp, _u32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.rb_material_textures.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                             C.c_float]
        lib.rb_set_texcoords.argtypes = [vp, _i32p, C.c_int, _f32p, _f32p, C.c_int]
        lib.rb_add_volume.argtypes = [vp, C.c_int, C.c_int, C.c_int, _f32p, C.c_float, _f32p, C.c_float, _f32p]
        lib.rb_guide.argtypes = [vp, _f32p, C.c_float, C.c_int, C.c_int, _f32p, _f32p]
        lib.rb_light_trace_caustics.argtypes = [vp, _f32p, C.c_float, C.c_int, C.c_int, C.c_longlong, C.c_int,
                                                C.c_ulonglong, _f32p]
        lib.rb_rays.argtypes = [_i64p]
        lib.rb_blue_noise.argtypes = [_u16p]
        lib.rb_sampler_owen.argtypes = [C.c_uint32, C.c_uint32]
        lib.rb_sampler_owen.restype = C.c_uint32
        lib.rb_sampler_sobol1.argtypes = [C.c_uint32]
        lib.rb_sampler_sobol1.restype = C.c_uint32
        lib.rb_sampler_hash.argtypes = [C.c_uint32]
        lib.rb_sampler_hash.restype = C.c_uint32
        lib.rb_set_threads.argtypes = [C.c_int]
        lib.rb_bsdf_tables.argtypes = [_f32p]
        lib.rb_prim_data.argtypes = [vp, _f32p]
        lib.rb_camera.argtypes = [_f32p, C.c_float, C.c_float, _f32p]
        lib.rb_env_tables.argtypes = [vp, _f32p, _f32p, _f32p]
        lib._typed = True
    return lib


def bsdf_tables():
    """scene/brdf_tables.h packed as gpu_bsdf_tables packs it (2112 floats)."""
    out = np.zeros(2112, np.float32)
    ref_lib().rb_bsdf_tables(out)
    return out


def blue_noise():
    out = np.zeros(4096, np.uint16)
    ref_lib().rb_blue_noise(out)
    return out


def camera(from_at_up, vfov, aspect):
    """camera_make (camera.h:21-36): (origin, upper_left, horizontal, vertical) as 12 floats."""
    out = np.zeros(12, np.float32)
    ref_lib().rb_camera(np.ascontiguousarray(from_at_up, np.float32).reshape(-1), vfov, aspect, out)
    return out


def triangle_bounds(quv):
    """The reference's triangle_bounds (scene.c:65-74): (n, 8) float32 boxes, padded by 1e-3."""
    quv = np.ascontiguousarray(quv, np.float32).reshape(-1, 9)
    out = np.zeros((quv.shape[0], 8), np.float32)
    ref_lib().rb_triangle_bounds(quv.reshape(-1), quv.shape[0], out.reshape(-1))
    return out


class RefScene:
    """A reference Scene made through its public API (scene_add_triangle, make_quad, ...)."""

    def __init__(self, double=False, gpu=False):
        self.lib = ref_lib(double, gpu)
        self.s = self.lib.rb_scene_new()

    def gpu_frame_trace(self, from_at_up, vfov, w, h, spp, max_depth, mis=1, sampler=1):
        """The engine's gpu_frame_trace (engine/app/gpu_frame.c:49) through the CUDA backend (a RefScene
        made with gpu=True): (status, (h, w, 3) mean image)."""
        out = np.zeros((h, w, 3), np.float32)
        rc = self.lib.rb_gpu_frame_trace(self.s, np.ascontiguousarray(from_at_up, np.float32).reshape(-1), vfov, w, h,
                                         spp, max_depth, mis, sampler, out.reshape(-1))
        return rc, out

    def tree(self):
        """The scene's own tree (scene_set_accel made it) in put_nodes' layout: ((n, 8) uint32 nodes, refs)."""
        nn, nr = C.c_int(), C.c_int()
        if not self.lib.rb_scene_tree(self.s, None, None, C.byref(nn), C.byref(nr)):
            return None
        nodes = np.zeros((nn.value, 8), np.uint32)
        refs = np.zeros(nr.value, np.uint32)
        self.lib.rb_scene_tree(self.s, nodes.ctypes.data, refs.ctypes.data, C.byref(nn), C.byref(nr))
        return nodes, refs

    def close(self):
        if self.s:
            self.lib.rb_scene_free(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def material(self, type_, albedo=(0, 0, 0), emission=(0, 0, 0), ior=1.5, metallic=0.0, roughness=1.0,
                 transmission=0.0):
        return self.lib.rb_add_material(self.s, int(type_), np.asarray(albedo, np.float32),
                                        np.asarray(emission, np.float32), ior, metallic, roughness, transmission)

    def triangles(self, corners, mats):
        corners = np.ascontiguousarray(corners, np.float32).reshape(-1, 9)
        self.lib.rb_add_triangles(self.s, corners.reshape(-1), np.ascontiguousarray(mats, np.int32),
                                  corners.shape[0])

    def quad(self, q, u, v, mat, light=False):
        f = lambda a: np.asarray(a, np.float32)
        return self.lib.rb_add_quad(self.s, f(q), f(u), f(v), mat, int(light))

    def sphere(self, c, r, mat):
        return self.lib.rb_add_sphere(self.s, np.asarray(c, np.float32), r, mat)

    def mesh(self, corners, mats):
        corners = np.ascontiguousarray(corners, np.float32).reshape(-1, 9)
        return self.lib.rb_add_mesh(self.s, corners.reshape(-1), np.ascontiguousarray(mats, np.int32),
                                    corners.shape[0])

    def instance(self, mesh, xf12, material=-1):
        return self.lib.rb_add_instance(self.s, mesh, np.ascontiguousarray(xf12, np.float32).reshape(-1),
                                        material)

    def instance_data(self, i):
        box = np.zeros(6, np.float32)
        inv = np.zeros(12, np.float32)
        self.lib.rb_instance_data(self.s, i, box, inv)
        return box, inv

    def mesh_box(self, m):
        box = np.zeros(6, np.float32)
        self.lib.rb_mesh_box(self.s, m, box)
        return box

    def env(self, rgb):
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = rgb.shape[:2]
        if not self.lib.rb_set_env(self.s, rgb.reshape(-1), w, h):
            raise MemoryError("env")

    def env_tables(self, w, h):
        marg = np.zeros(h + 1, np.float32)
        cond = np.zeros(h * (w + 1), np.float32)
        prob = np.zeros(w * h, np.float32)
        self.lib.rb_env_tables(self.s, marg, cond, prob)
        return marg, cond, prob

    def set_accel(self):
        self.lib.rb_set_accel(self.s)

    def move_instance(self, i, xf12):
        """scene_move_instance (scene.c:743); update_instances then makes the top level again."""
        self.lib.rb_move_instance(self.s, i, np.ascontiguousarray(xf12, np.float32).reshape(-1))

    def update_instances(self):
        self.lib.rb_update_instances(self.s)

    def prim_data(self):
        n = self.lib.rb_num_prims(self.s)
        out = np.zeros((max(n, 1), 24), np.float32)
        self.lib.rb_prim_data(self.s, out.reshape(-1))
        return out[:n]

    def tri_data(self):
        n = self.lib.rb_num_tris(self.s)
        quv = np.zeros((n, 9), np.float32)
        mats = np.zeros(n, np.int32)
        self.lib.rb_tri_data(self.s, quv.reshape(-1), mats.ctypes.data)
        return quv, mats

    def intersect(self, orig, dirs, tmin=0.0, tmax=1e30):
        n = orig.shape[0]
        prim = np.zeros(n, np.int32)
        inst = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        self.lib.rb_intersect(self.s, np.ascontiguousarray(orig, np.float32).reshape(-1),
                              np.ascontiguousarray(dirs, np.float32).reshape(-1), n, tmin, tmax, prim, inst, t)
        return prim, inst, t

    def occluded(self, orig, dirs, tmin, tmax):
        n = orig.shape[0]
        out = np.zeros(n, np.int32)
        self.lib.rb_occluded(self.s, np.ascontiguousarray(orig, np.float32).reshape(-1),
                             np.ascontiguousarray(dirs, np.float32).reshape(-1), n, tmin, tmax, out)
        return out

    def trace_image(self, cam, vfov, w, h, spp, seed, max_depth, mis=1, sampler=1, y0=0, rows=None, skip_caustics=0,
                    indirect_clamp=0.0):
        """trace_image: (rows, w, 3) mean radiance; returns (image, (closest rays, shadow rays))."""
        rows = h if rows is None else rows
        out = np.zeros((rows, w, 3), np.float32)
        self.lib.rb_rays_reset()
        self.lib.rb_set_indirect_clamp(indirect_clamp)
        try:
            self.lib.rb_trace_image(self.s, np.ascontiguousarray(cam, np.float32).reshape(-1), vfov, w, h, y0, rows,
                                    spp, seed, max_depth, mis, sampler, skip_caustics, out.reshape(-1))
        finally:
            self.lib.rb_set_indirect_clamp(0.0)
        cnt = np.zeros(2, np.int64)
        self.lib.rb_rays(cnt)
        return out, (int(cnt[0]), int(cnt[1]))

    def texmap(self, rgba, srgb, wrap_u=0, wrap_v=0):
        """texmap_make + scene_add_texmap of (h, w) uint32 RGBA8 texels: the texture's number."""
        px = np.ascontiguousarray(rgba, np.uint32)
        return self.lib.rb_add_texmap(self.s, px.reshape(-1), px.shape[1], px.shape[0], srgb, wrap_u, wrap_v)

    def material_textures(self, mat, base=0, mr=0, normal=0, emissive=0, occlusion=0, uv_scale=0.0, normal_scale=0.0):
        self.lib.rb_material_textures(self.s, mat, base, mr, normal, emissive, occlusion, uv_scale, normal_scale)

    def texcoords(self, tri_uv, uvs, tangents):
        tri_uv = np.ascontiguousarray(tri_uv, np.int32)
        self.lib.rb_set_texcoords(self.s, tri_uv.reshape(-1), tri_uv.shape[0], np.ascontiguousarray(uvs, np.float32).reshape(-1),
                                  np.ascontiguousarray(tangents, np.float32).reshape(-1), len(uvs))

    def volume(self, density, lo, hi, sigma_t, albedo, g):
        """scene_add_volume of a (nz, ny, nx) density grid filling the box lo..hi."""
        den = np.ascontiguousarray(density, np.float32)
        nz, ny, nx = den.shape
        box = np.array([*lo, *hi], np.float32)
        return self.lib.rb_add_volume(self.s, nx, ny, nz, box, sigma_t, np.asarray(albedo, np.float32), g, den.reshape(-1))

    def guide(self, cam, vfov, w, h):
        """The denoiser's guide planes 2 and 3 ((h, w, 4) each) restated on this scene."""
        n4 = np.zeros((h, w, 4), np.float32)
        a4 = np.zeros((h, w, 4), np.float32)
        self.lib.rb_guide(self.s, np.ascontiguousarray(cam, np.float32).reshape(-1), vfov, w, h, n4.reshape(-1),
                          a4.reshape(-1))
        return n4, a4

    def light_trace_caustics(self, cam, vfov, w, h, photons, max_depth, seed):
        """light_trace_caustics (tracer.c:553-665): the (h, w, 3) caustic image of `photons` light
        paths; returns (image, (closest rays, shadow rays))."""
        out = np.zeros((h, w, 3), np.float32)
        self.lib.rb_rays_reset()
        self.lib.rb_light_trace_caustics(self.s, np.ascontiguousarray(cam, np.float32).reshape(-1), vfov, w, h,
                                         photons, max_depth, seed, out.reshape(-1))
        cnt = np.zeros(2, np.int64)
        self.lib.rb_rays(cnt)
        return out, (int(cnt[0]), int(cnt[1]))
