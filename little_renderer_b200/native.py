"""Build recipe and ctypes binding of the CUDA backend's C ABI (include/lrc.h).

The library is built in-tree (``little_renderer_b200/liblrc.so``) with nvcc for sm_100a only.
Loading it never falls back to anything: a missing or unloadable library raises.
"""
import ctypes as C
import os
import subprocess

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "liblrc.so")
SOURCES = ["api.cu", "build.cu", "traverse.cu", "static_build.cu", "pathtrace.cu", "host_tables.cu", "batch.cu", "wavefront.cu", "refit.cu", "serve.cu", "caustics.cu", "denoise.cu", "media.cu", "textures.cu", "wide.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC"]
OBJ_DIR = os.path.join(PKG, "_build")

LRC_OK, LRC_RETRY, LRC_E_INVALID, LRC_E_CUDA, LRC_E_TIMEOUT, LRC_E_STACK, LRC_E_NODEVICE = 0, 1, -1, -2, -3, -4, -5
LRC_DEVICE = 1
LRC_TRACE_GUIDED = 64
LRC_TRACE_MEGAKERNEL = 256
LRC_REPROJECT_EDIT = 128
LRC_SERVE_DENOISE = 16
LRC_WAVEFRONT_DEFAULT_VARIANT = 9      # (include/lrc.h)
LRC_BATCH_BUILD, LRC_BATCH_GRAPH, LRC_BATCH_ZERO, LRC_BATCH_STEPPED, LRC_BATCH_COUNT = 4, 8, 16, 32, 64


def nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.sep not in p or os.path.exists(p)):
            return p
    return "nvcc"


def build(force=False, verbose=False):
    """Compiles liblrc.so for sm_100a: each source to an object of its own (in parallel, again
    only when it or a header is newer than the object), then one link. Returns the library's path."""
    from concurrent.futures import ThreadPoolExecutor
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(ROOT, "include", "lrc.h"))
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs = []
    objs = []
    for src in SOURCES:
        s_path = os.path.join(CSRC, src)
        o_path = os.path.join(OBJ_DIR, src[:-3] + ".o")
        d_path = o_path[:-2] + ".d"
        objs.append(o_path)
        deps = _deps(d_path) if os.path.exists(d_path) else headers
        deps = [d for d in deps if os.path.exists(d)] + [s_path]
        if force or not os.path.exists(o_path) or os.path.getmtime(o_path) < max(os.path.getmtime(d) for d in deps):
            jobs.append([nvcc()] + NVCC_FLAGS + ["-MD", "-MF", d_path, "-c", s_path, "-o", o_path])
    if not jobs and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, cwd=CSRC)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs)
    return LIB


def _deps(d_path):
    """The files an object depends on, from its make-style dependency file (nvcc -MD)."""
    with open(d_path) as f:
        text = f.read().replace("\\\n", " ")
    paths = [os.path.normpath(os.path.join(CSRC, t)) for t in text.split(":", 1)[-1].split()]
    return [t for t in paths if t.startswith(ROOT + os.sep)]     # the project's own files only


_lib = None


class LrcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lrc error {code}: {msg}")
        self.code = code


def lib():
    """The loaded liblrc.so (raises if it is missing: there is no other path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise RuntimeError(f"{LIB} is not built: the CUDA backend is required (python -c 'import "
                           "__graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB)
    vp, u32, u64, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float
    L.lrc_open.argtypes = [C.c_int, C.POINTER(vp)]
    L.lrc_close.argtypes = [vp]
    L.lrc_message.argtypes = [vp]
    L.lrc_message.restype = C.c_char_p
    L.lrc_sync.argtypes = [vp]
    L.lrc_set_stream.argtypes = [vp, vp]
    L.lrc_status.argtypes = [vp]
    L.lrc_status.restype = u32
    L.lrc_num_sms.argtypes = [vp]
    L.lrc_params_from_bounds.argtypes = [vp, vp, vp]
    L.lrc_build.argtypes = [vp, vp, vp, vp, vp, C.c_uint]
    L.lrc_build_scratch_bytes.argtypes = [u32, C.c_int, C.c_int]
    L.lrc_build_scratch_bytes.restype = C.c_size_t
    L.lrc_triangle_boxes.argtypes = [vp, vp, u32, vp, vp, C.c_uint]
    L.lrc_build_static.argtypes = [vp, vp, vp, vp, vp]
    L.lrc_scene_create.argtypes = [vp, C.POINTER(vp)]
    L.lrc_scene_destroy.argtypes = [vp]
    L.lrc_scene_set_triangles.argtypes = [vp, vp, u32, C.c_uint]
    L.lrc_scene_build.argtypes = [vp, C.c_int, C.c_int]
    L.lrc_scene_tree.argtypes = [vp, vp, vp, C.c_uint]
    L.lrc_scene_tree_device.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(u32)]
    L.lrc_scene_intersect.argtypes = [vp, vp, vp, u64, f32, f32, vp, vp, C.c_uint]
    L.lrc_scene_occluded.argtypes = [vp, vp, vp, vp, u64, f32, vp, C.c_uint]
    L.lrc_scene_trace_stats.argtypes = [vp, vp, vp, u64, f32, f32, vp, C.c_uint]
    L.lrc_scene_set_walk.argtypes = [vp, C.c_int]
    L.lrc_scene_set_prims.argtypes = [vp, vp, u32, C.c_uint]
    L.lrc_scene_set_normals.argtypes = [vp, vp, u32, C.c_uint]
    L.lrc_scene_set_materials.argtypes = [vp, vp, u32]
    L.lrc_scene_set_light.argtypes = [vp, C.c_int32]
    L.lrc_scene_set_tables.argtypes = [vp, vp, vp]
    L.lrc_default_blue_noise.argtypes = [vp]
    L.lrc_default_bsdf_tables.argtypes = [vp]
    L.lrc_trace.argtypes = [vp, vp, C.c_int32, C.c_int32, u32, u32, vp, vp, C.c_uint]
    L.lrc_caustics.argtypes = [vp, vp, C.c_uint64, C.c_uint64, vp, vp, C.c_uint]
    L.lrc_caustics_sums.argtypes = [vp, vp, C.c_uint64, C.c_uint64, vp, vp, C.c_uint]
    L.lrc_caustics_variant.argtypes = [vp, C.c_int]
    L.lrc_guide.argtypes = [vp, vp, vp, C.c_uint]
    L.lrc_reproject.argtypes = [vp, vp, vp, vp, vp, C.c_int32, C.c_uint]
    L.lrc_reproject_gradients.argtypes = [vp, vp, vp, u32, vp, vp, C.c_int32, C.c_int32, vp, C.c_uint]
    L.lrc_trace_frame.argtypes = [vp, vp, vp, u32, u32, vp, vp, C.c_int32, C.c_int32, C.c_uint]
    L.lrc_scene_set_volumes.argtypes = [vp, vp, u32]
    L.lrc_volume_majorants.argtypes = [vp, vp, vp, vp]
    L.lrc_srgb_table.argtypes = [vp]
    L.lrc_scene_set_texmaps.argtypes = [vp, vp, u32]
    L.lrc_scene_set_texcoords.argtypes = [vp, vp, u32, vp, vp, u32]
    L.lrc_denoise.argtypes = [vp, C.c_int32, C.c_int32, vp, C.c_int32, vp, C.c_uint]
    L.lrc_scene_set_meshes.argtypes = [vp, vp, vp, u32, C.c_uint]
    L.lrc_scene_set_instances.argtypes = [vp, vp, u32, C.c_uint]
    L.lrc_scene_build_instances.argtypes = [vp, C.c_int, C.c_int]
    L.lrc_scene_set_sky.argtypes = [vp, vp, C.c_int32, C.c_int32, vp, vp, vp, f32]
    L.lrc_scene_intersect_ex.argtypes = [vp, vp, vp, u64, f32, f32, vp, vp, vp, C.c_uint]
    L.lrc_sky_tables.argtypes = [vp, C.c_int32, C.c_int32, vp, vp, vp]
    L.lrc_set_timing.argtypes = [vp, C.c_int]
    L.lrc_timings.argtypes = [vp, vp, vp]
    L.lrc_batch_create.argtypes = [vp, C.POINTER(vp)]
    L.lrc_batch_destroy.argtypes = [vp]
    L.lrc_batch_add.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, u32, u32, vp, C.c_int32, C.c_int32]
    L.lrc_batch_add_guided.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, u32, u32, vp, C.c_int32, C.c_int32]
    L.lrc_batch_clear.argtypes = [vp]
    L.lrc_batch_jobs.argtypes = [vp]
    L.lrc_batch_run.argtypes = [vp, C.c_uint]
    L.lrc_batch_rays.argtypes = [vp, vp, vp]
    L.lrc_batch_shape.argtypes = [C.c_int32, vp, vp, vp]
    L.lrc_batch_set_shape.argtypes = [vp, C.c_int32, C.c_int32]
    L.lrc_batch_tune.argtypes = [vp, u64, vp, vp, vp]
    L.lrc_batch_info.argtypes = [vp, vp, vp, vp, vp, vp]
    L.lrc_scene_move_instances.argtypes = [vp, vp, u32, C.c_int, C.c_uint]
    L.lrc_scene_tlas_cost.argtypes = [vp, vp]
    L.lrc_refit.argtypes = [vp, vp, vp, u32, u32, vp, C.c_uint]
    L.lrc_server_create.argtypes = [vp, u64, u64, C.POINTER(vp)]
    L.lrc_server_destroy.argtypes = [vp]
    L.lrc_server_submit.argtypes = [vp, vp, vp, u32, vp, u32, C.c_int, C.POINTER(u64)]
    L.lrc_server_step.argtypes = [vp, C.POINTER(C.c_int32)]
    L.lrc_server_result.argtypes = [vp, u64, C.POINTER(vp), C.POINTER(u64), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.lrc_server_release.argtypes = [vp, u64]
    L.lrc_server_read.argtypes = [vp, u64, vp]
    L.lrc_server_state.argtypes = [vp, vp, vp, vp, vp]
    L.lrc_server_clock.restype = C.c_double
    L.lrc_server_batch.argtypes = [vp]
    L.lrc_server_batch.restype = vp
    L.lrc_server_set_wavefront.argtypes = [vp, u32, C.c_int32]
    L.lrc_batch_set_engine.argtypes = [vp, C.c_int32]
    L.lrc_batch_set_wavefront.argtypes = [vp, u32, C.c_int32]
    L.lrc_batch_wavefront_shape.argtypes = [C.c_int32, vp, vp, vp]
    L.lrc_batch_engine.argtypes = [vp, vp, vp, vp]
    _lib = L
    return L


class BuildParams(C.Structure):
    """lrc_build_params (build_queue's BuildParams, engine/gpu/trace_gpu.c:546)."""
    _fields_ = [("n", C.c_uint32), ("node0", C.c_uint32), ("ref0", C.c_uint32), ("ref_add", C.c_uint32),
                ("lo", C.c_float * 3), ("ext", C.c_float * 3), ("key_bits", C.c_int32), ("builder", C.c_int32)]


class Volume(C.Structure):
    """lrc_volume (engine/scene/volume.h's Volume: grid, box, optics)."""
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("lo", C.c_float * 3), ("hi", C.c_float * 3),
                ("sigma_t", C.c_float), ("albedo", C.c_float * 3), ("g", C.c_float), ("density", C.c_void_p)]


class TexMap(C.Structure):
    """lrc_texmap (level 0 of the reference's TexMap)."""
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("srgb", C.c_int32), ("wrap_u", C.c_int32), ("wrap_v", C.c_int32),
                ("rgba", C.c_void_p)]


class TraceParams(C.Structure):
    """lrc_trace_params (the Camera of engine/scene/camera.h and GpuTraceParams' numbers)."""
    _fields_ = [("origin", C.c_float * 3), ("upper_left", C.c_float * 3), ("horizontal", C.c_float * 3),
                ("vertical", C.c_float * 3), ("width", C.c_int32), ("height", C.c_int32), ("max_depth", C.c_int32),
                ("mis", C.c_int32), ("sampler", C.c_int32), ("exact", C.c_int32), ("seed", C.c_uint64),
                ("clamp", C.c_float), ("skip_caustics", C.c_int32), ("indirect_clamp", C.c_float)]


def trace_params(cam12, width, height, max_depth=8, mis=1, sampler=1, exact=0, seed=0, clamp=0.0, skip_caustics=0,
                 indirect_clamp=0.0):
    p = TraceParams()
    cam12 = np.asarray(cam12, np.float32).reshape(4, 3)
    for i, name in enumerate(("origin", "upper_left", "horizontal", "vertical")):
        getattr(p, name)[:] = cam12[i].tolist()
    p.width, p.height, p.max_depth, p.mis, p.sampler, p.exact, p.seed, p.clamp, p.skip_caustics = (
        width, height, max_depth, mis, sampler, exact, seed, clamp, skip_caustics)
    p.indirect_clamp = indirect_clamp
    return p


def volume_majorants(density, lo, hi):
    """lrc_volume_majorants (host): (largest density, active box (6,), brick maxima (bz, by, bx))."""
    den = np.ascontiguousarray(density, np.float32)
    v = Volume()
    v.nz, v.ny, v.nx = den.shape
    v.lo[:] = list(map(float, lo))
    v.hi[:] = list(map(float, hi))
    v.sigma_t, v.g = 0.1, 0.0
    v.albedo[:] = [1.0, 1.0, 1.0]
    v.density = den.ctypes.data
    mx = np.zeros(1, np.float32)
    act = np.zeros(6, np.float32)
    b = [(n + 7) // 8 for n in den.shape]
    bricks = np.zeros(b, np.float32)
    rc = lib().lrc_volume_majorants(C.byref(v), _ptr(mx), _ptr(act), _ptr(bricks))
    if rc:
        raise LrcError(rc, "lrc_volume_majorants")
    return float(mx[0]), act, bricks


def srgb_table():
    out = np.zeros(256, np.float32)
    lib().lrc_srgb_table(_ptr(out))
    return out


def sky_tables(rgb):
    """lrc_sky_tables (host): (marg, cond, prob) of an (h, w, 3) sky."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    marg = np.zeros(h + 1, np.float32)
    cond = np.zeros(h * (w + 1), np.float32)
    prob = np.zeros(w * h, np.float32)
    lib().lrc_sky_tables(_ptr(rgb), w, h, _ptr(marg), _ptr(cond), _ptr(prob))
    return marg, cond, prob


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray) else C.c_void_p(int(a))


class Context:
    """An lrc context on one CUDA device (lrc_open)."""

    def __init__(self, device=0):
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.lrc_open(device, C.byref(h))
        if rc:
            raise LrcError(rc, "lrc_open failed (no CUDA device?)")
        self.h = h

    def check(self, rc):
        if rc:
            raise LrcError(rc, self.L.lrc_message(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.lrc_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        return self.check(self.L.lrc_sync(self.h))

    def set_stream(self, stream_ptr):
        self.check(self.L.lrc_set_stream(self.h, C.c_void_p(stream_ptr)))

    def denoise(self, planes, passes=5, out=None):
        """lrc_denoise with host arrays: planes (4, h, w, 4) -> the denoised image (h, w, 4)."""
        planes = np.ascontiguousarray(planes, np.float32)
        h, w = planes.shape[1:3]
        if out is None:
            out = np.zeros((h, w, 4), np.float32)
        self.check(self.L.lrc_denoise(self.h, w, h, _ptr(planes), passes, _ptr(out), 0))
        return out

    def reproject(self, old_params, new_params, old_planes, new_planes, history):
        """lrc_reproject with host planes (4, h, w, 4): new_planes' planes 0 and 1 from old_planes."""
        old_planes = np.ascontiguousarray(old_planes, np.float32)
        self.check(self.L.lrc_reproject(self.h, C.byref(old_params), C.byref(new_params), _ptr(old_planes),
                                        _ptr(new_planes), history, 0))
        return new_planes

    def denoise_device(self, width, height, d_planes, d_out, passes=5):
        self.check(self.L.lrc_denoise(self.h, width, height, C.c_void_p(d_planes), passes, C.c_void_p(d_out),
                                      LRC_DEVICE))

    def caustics_variant(self, variant=-1):
        """lrc_caustics_variant: the light tracer's launch variant; returns how many there are."""
        n = self.L.lrc_caustics_variant(self.h, variant)
        if n < 0:
            raise ValueError(f"no light tracer variant {variant}")
        return n

    def num_sms(self):
        return self.L.lrc_num_sms(self.h)

    STAGES = ("boxes", "morton", "sort", "hierarchy", "trace", "shade")

    def set_timing(self, on=True):
        self.check(self.L.lrc_set_timing(self.h, int(on)))

    def timings(self):
        """{stage: (ms, launches)} since the last call (lrc_timings)."""
        ms = np.zeros(8, np.float64)
        cnt = np.zeros(8, np.int32)
        self.check(self.L.lrc_timings(self.h, _ptr(ms), _ptr(cnt)))
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(self.STAGES)}

    def params(self, n, lo, hi, key_bits=30, builder=0, node0=0, ref0=0, ref_add=0):
        p = BuildParams()
        p.n, p.node0, p.ref0, p.ref_add, p.key_bits, p.builder = n, node0, ref0, ref_add, key_bits, builder
        lo = np.ascontiguousarray(lo, np.float32)
        hi = np.ascontiguousarray(hi, np.float32)
        self.L.lrc_params_from_bounds(_ptr(lo), _ptr(hi), C.byref(p))
        return p

    def build(self, params, boxes, nodes=None, aux=None):
        """lrc_build with host arrays: returns (nodes (node0 + 2n - 1, 8) u32, aux (ref0 + n) u32)."""
        n = params.n
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 8)
        if nodes is None:
            nodes = np.zeros((params.node0 + max(2 * n - 1, 1), 8), np.uint32)
        if aux is None:
            aux = np.zeros(params.ref0 + n, np.uint32)
        self.check(self.L.lrc_build(self.h, C.byref(params), _ptr(boxes), _ptr(nodes), _ptr(aux), 0))
        return nodes, aux

    def build_device(self, params, d_boxes, d_nodes, d_aux):
        """lrc_build with device pointers (ints): enqueued on the context's stream."""
        self.check(self.L.lrc_build(self.h, C.byref(params), C.c_void_p(d_boxes), C.c_void_p(d_nodes),
                                    C.c_void_p(d_aux), LRC_DEVICE))

    def refit(self, nodes, aux, boxes, ref_add=0):
        """lrc_refit with host arrays: the tree's boxes made again for new item boxes (a copy)."""
        nodes = np.array(nodes, np.uint32, copy=True).reshape(-1, 8)
        aux = np.ascontiguousarray(aux, np.uint32)
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 8)
        n = boxes.shape[0]
        self.check(self.L.lrc_refit(self.h, _ptr(nodes), _ptr(aux), n, ref_add, _ptr(boxes), 0))
        return nodes

    def triangle_boxes(self, tris12):
        tris12 = np.ascontiguousarray(tris12, np.uint32).reshape(-1, 12)
        n = tris12.shape[0]
        boxes = np.zeros((n, 8), np.float32)
        bounds = np.zeros(6, np.float32)
        self.check(self.L.lrc_triangle_boxes(self.h, _ptr(tris12), n, _ptr(boxes), _ptr(bounds), 0))
        return boxes, bounds


class Scene:
    """A device-resident scene (lrc_scene_*)."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.L.lrc_scene_create(ctx.h, C.byref(h)))
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.lrc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_triangles(self, tris12, device_ptr=None, n=None):
        L = self.ctx.L
        if device_ptr is not None:
            self.ctx.check(L.lrc_scene_set_triangles(self.h, C.c_void_p(device_ptr), n, LRC_DEVICE))
            self.n = n
            return
        tris12 = np.ascontiguousarray(tris12, np.uint32).reshape(-1, 12)
        self.n = tris12.shape[0]
        self.ctx.check(L.lrc_scene_set_triangles(self.h, _ptr(tris12), self.n, 0))

    def build(self, builder=0, key_bits=30):
        self.ctx.check(self.ctx.L.lrc_scene_build(self.h, builder, key_bits))

    def set_tree(self, nodes, aux):
        """lrc_scene_set_tree: the world tree given (put_nodes' layout, shape ids in aux), not built."""
        nodes = np.ascontiguousarray(nodes, np.uint32).reshape(-1, 8)
        aux = np.ascontiguousarray(aux, np.uint32)
        self.ctx.check(self.ctx.L.lrc_scene_set_tree(self.h, _ptr(nodes), nodes.shape[0], _ptr(aux), aux.shape[0], 0))

    def set_walk(self, mode):
        """lrc_scene_set_walk: ray queries over a copy of the tree with tight boxes (1, the default),
        that copy as 8-wide quantised nodes (2), or the tree as built (0)."""
        self.ctx.check(self.ctx.L.lrc_scene_set_walk(self.h, int(mode)))

    def tree(self):
        nodes = np.zeros((2 * self.n - 1, 8), np.uint32)
        aux = np.zeros(self.n, np.uint32)
        self.ctx.check(self.ctx.L.lrc_scene_tree(self.h, _ptr(nodes), _ptr(aux), 0))
        return nodes, aux

    def intersect(self, orig, dirs, tmin=0.0, tmax=1e30):
        orig = np.ascontiguousarray(orig, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = orig.shape[0]
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        self.ctx.check(self.ctx.L.lrc_scene_intersect(self.h, _ptr(orig), _ptr(dirs), n, tmin, tmax, _ptr(prim),
                                                      _ptr(t), 0))
        return prim, t

    def intersect_device(self, d_orig, d_dir, n, d_prim, d_t, tmin=0.0, tmax=1e30):
        self.ctx.check(self.ctx.L.lrc_scene_intersect(self.h, C.c_void_p(d_orig), C.c_void_p(d_dir), n, tmin, tmax,
                                                      C.c_void_p(d_prim), C.c_void_p(d_t), LRC_DEVICE))

    def set_prims(self, prims24):
        prims24 = np.ascontiguousarray(prims24, np.float32).reshape(-1, 24)
        self.ctx.check(self.ctx.L.lrc_scene_set_prims(self.h, _ptr(prims24), prims24.shape[0], 0))

    def set_normals(self, normals):
        normals = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        self.ctx.check(self.ctx.L.lrc_scene_set_normals(self.h, _ptr(normals), normals.shape[0], 0))

    def set_materials(self, recs16):
        recs16 = np.ascontiguousarray(recs16, np.float32).reshape(-1, 16)
        self.ctx.check(self.ctx.L.lrc_scene_set_materials(self.h, _ptr(recs16), recs16.shape[0]))

    def set_light(self, prim):
        self.ctx.check(self.ctx.L.lrc_scene_set_light(self.h, prim))

    def set_tables(self, blue_noise=None, bsdf_tables=None):
        bn = None if blue_noise is None else np.ascontiguousarray(blue_noise, np.uint16)
        tb = None if bsdf_tables is None else np.ascontiguousarray(bsdf_tables, np.float32)
        self.ctx.check(self.ctx.L.lrc_scene_set_tables(self.h, None if bn is None else _ptr(bn),
                                                       None if tb is None else _ptr(tb)))

    def set_meshes(self, meshes_tris12):
        """meshes_tris12: a list of (n_m, 12) u32 arrays (the GPU triangle layout)."""
        counts = np.array([t.shape[0] for t in meshes_tris12], np.uint32)
        allt = np.ascontiguousarray(np.concatenate(meshes_tris12), np.uint32) if len(meshes_tris12) else np.zeros((1, 12), np.uint32)
        self.ctx.check(self.ctx.L.lrc_scene_set_meshes(self.h, _ptr(allt), _ptr(counts), counts.shape[0], 0))

    def set_instances(self, records32):
        records32 = np.ascontiguousarray(records32, np.float32).reshape(-1, 32)
        self.ctx.check(self.ctx.L.lrc_scene_set_instances(self.h, _ptr(records32), records32.shape[0], 0))

    def build_instances(self, mesh_builder=1, key_bits=30):
        self.ctx.check(self.ctx.L.lrc_scene_build_instances(self.h, mesh_builder, key_bits))

    def move_instances(self, records, mode=0):
        """lrc_scene_move_instances: 0 refit, 1 rebuild, 2 auto (the reference's refit policy)."""
        records = np.ascontiguousarray(records, np.float32).reshape(-1, 32)
        self.ctx.check(self.ctx.L.lrc_scene_move_instances(self.h, _ptr(records), records.shape[0], mode, 0))

    def tlas_cost(self):
        c = C.c_double()
        self.ctx.check(self.ctx.L.lrc_scene_tlas_cost(self.h, C.byref(c)))
        return c.value

    def set_sky(self, rgb, scale=1.0, marg=None, cond=None, prob=None):
        if rgb is None:
            self.ctx.check(self.ctx.L.lrc_scene_set_sky(self.h, None, 0, 0, None, None, None, 1.0))
            return
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = rgb.shape[:2]
        arr = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (marg, cond, prob)]
        self.ctx.check(self.ctx.L.lrc_scene_set_sky(self.h, _ptr(rgb), w, h, *[None if a is None else _ptr(a) for a in arr],
                                                    scale))

    def intersect_ex(self, orig, dirs, tmin=0.0, tmax=1e30):
        """(prim, inst, t) as scene_intersect's Hit."""
        orig = np.ascontiguousarray(orig, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = orig.shape[0]
        prim = np.zeros(n, np.int32)
        inst = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        self.ctx.check(self.ctx.L.lrc_scene_intersect_ex(self.h, _ptr(orig), _ptr(dirs), n, tmin, tmax, _ptr(prim),
                                                         _ptr(inst), _ptr(t), 0))
        return prim, inst, t

    def trace(self, params, spp, accum=None, y0=0, rows=None, spp0=0, flags=0):
        """lrc_trace with a host image: returns (accum (h, w, 4) sum + count, rays traced)."""
        rows = params.height if rows is None else rows
        if accum is None:
            accum = np.zeros((params.height, params.width, 4), np.float32)
        rays = C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_trace(self.h, C.byref(params), y0, rows, spp0, spp, _ptr(accum),
                                            C.byref(rays), flags))
        return accum, rays.value

    def trace_device(self, params, spp, d_accum, y0=0, rows=None, spp0=0, flags=0):
        rows = params.height if rows is None else rows
        self.ctx.check(self.ctx.L.lrc_trace(self.h, C.byref(params), y0, rows, spp0, spp, C.c_void_p(d_accum), None,
                                            LRC_DEVICE | flags))

    def set_volumes(self, vols):
        """lrc_scene_set_volumes: vols = [(density (nz, ny, nx) float32, lo, hi, sigma_t, albedo, g), ...]."""
        arr = (Volume * max(len(vols), 1))()
        self._vol_keep = []
        for i, (den, lo, hi, sigma_t, albedo, g) in enumerate(vols):
            den = np.ascontiguousarray(den, np.float32)
            self._vol_keep.append(den)
            v = arr[i]
            v.nz, v.ny, v.nx = den.shape
            v.lo[:] = list(map(float, lo))
            v.hi[:] = list(map(float, hi))
            v.sigma_t, v.g = float(sigma_t), float(g)
            v.albedo[:] = list(map(float, albedo))
            v.density = den.ctypes.data
        self.ctx.check(self.ctx.L.lrc_scene_set_volumes(self.h, arr, len(vols)))

    def set_texmaps(self, maps):
        """lrc_scene_set_texmaps: maps = [(rgba (h, w) uint32, srgb, wrap_u, wrap_v), ...]."""
        arr = (TexMap * max(len(maps), 1))()
        self._tex_keep = []
        for i, (px, srgb, wu, wv) in enumerate(maps):
            px = np.ascontiguousarray(px, np.uint32)
            self._tex_keep.append(px)
            arr[i].h, arr[i].w = px.shape
            arr[i].srgb, arr[i].wrap_u, arr[i].wrap_v = int(srgb), int(wu), int(wv)
            arr[i].rgba = px.ctypes.data
        self.ctx.check(self.ctx.L.lrc_scene_set_texmaps(self.h, arr, len(maps)))

    def set_texcoords(self, tri_uv, uvs, tangents):
        """lrc_scene_set_texcoords: tri_uv (ntris, 3) int32, uvs (n, 2), tangents (n, 4)."""
        tri_uv = np.ascontiguousarray(tri_uv, np.int32)
        uvs = np.ascontiguousarray(uvs, np.float32)
        tangents = np.ascontiguousarray(tangents, np.float32)
        self.ctx.check(self.ctx.L.lrc_scene_set_texcoords(self.h, _ptr(tri_uv), tri_uv.shape[0], _ptr(uvs), _ptr(tangents),
                                                          uvs.shape[0]))

    def guide(self, params, planes=None):
        """lrc_guide with host planes (4, h, w, 4): planes 2 and 3 written; returns the planes."""
        if planes is None:
            planes = np.zeros((4, params.height, params.width, 4), np.float32)
        self.ctx.check(self.ctx.L.lrc_guide(self.h, C.byref(params), _ptr(planes), 0))
        return planes

    def guide_device(self, params, d_planes):
        self.ctx.check(self.ctx.L.lrc_guide(self.h, C.byref(params), C.c_void_p(d_planes), LRC_DEVICE))

    def trace_guided(self, params, spp, planes, spp0=0, flags=0):
        """lrc_trace with LRC_TRACE_GUIDED on host planes (4, h, w, 4): samples into plane 0, the
        luminance moments into plane 1; returns (planes, rays)."""
        rays = C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_trace(self.h, C.byref(params), 0, params.height, spp0, spp, _ptr(planes),
                                            C.byref(rays), LRC_TRACE_GUIDED | flags))
        return planes, rays.value

    def reproject_gradients(self, old_params, new_params, spp0, old_planes, new_planes, history_max, history,
                            edit=False):
        """lrc_reproject_gradients with host planes (4, h, w, 4): new_planes' planes 0 and 1 from
        old_planes, each pixel's history from its tile's temporal gradient; returns the tiles
        ((h + 3) // 4, (w + 3) // 4, 4): new pixel, old pixel, the sample's lambda, the filtered
        lambda (-1: none)."""
        old_planes = np.ascontiguousarray(old_planes, np.float32)
        h, w = new_planes.shape[1:3]
        tiles = np.zeros(((h + 3) // 4, (w + 3) // 4, 4), np.float32)
        self.ctx.check(self.ctx.L.lrc_reproject_gradients(
            self.h, C.byref(old_params), C.byref(new_params), spp0, _ptr(old_planes), _ptr(new_planes), history_max,
            history, _ptr(tiles), LRC_REPROJECT_EDIT if edit else 0))
        return tiles

    def reproject_gradients_device(self, old_params, new_params, spp0, d_old, d_new, history_max, history, d_tiles=0,
                                   edit=False):
        """lrc_reproject_gradients with device planes (and tiles, 0: none); returns at once."""
        self.ctx.check(self.ctx.L.lrc_reproject_gradients(
            self.h, C.byref(old_params), C.byref(new_params), spp0, C.c_void_p(d_old), C.c_void_p(d_new), history_max,
            history, C.c_void_p(d_tiles) if d_tiles else None, LRC_DEVICE | (LRC_REPROJECT_EDIT if edit else 0)))

    def trace_frame(self, old_params, new_params, spp0, spp, old_planes, history_max, history, edit=False):
        """lrc_trace_frame with host planes: the new frame's 4 planes (h, w) from old_planes (4, h, w,
        4) or None (the first frame)."""
        new = np.zeros((4, new_params.height, new_params.width, 4), np.float32)
        old = None if old_planes is None else np.ascontiguousarray(old_planes, np.float32)
        self.ctx.check(self.ctx.L.lrc_trace_frame(
            self.h, C.byref(old_params) if old_params is not None else None, C.byref(new_params), spp0, spp,
            _ptr(old) if old is not None else None, _ptr(new), history_max, history,
            LRC_REPROJECT_EDIT if edit else 0))
        return new

    def trace_frame_device(self, old_params, new_params, spp0, spp, d_old, d_new, history_max, history, edit=False):
        """lrc_trace_frame with device planes (d_old 0: the first frame); returns at once."""
        self.ctx.check(self.ctx.L.lrc_trace_frame(
            self.h, C.byref(old_params) if old_params is not None else None, C.byref(new_params), spp0, spp,
            C.c_void_p(d_old) if d_old else None, C.c_void_p(d_new), history_max, history,
            LRC_DEVICE | (LRC_REPROJECT_EDIT if edit else 0)))

    def trace_guided_device(self, params, spp, d_planes, spp0=0):
        self.ctx.check(self.ctx.L.lrc_trace(self.h, C.byref(params), 0, params.height, spp0, spp, C.c_void_p(d_planes),
                                            None, LRC_TRACE_GUIDED | LRC_DEVICE))

    def caustics(self, params, photons, seed, image=None):
        """lrc_caustics with a host image: returns (image (h, w, 3) += the caustic image of `photons`
        light paths, rays traced)."""
        if image is None:
            image = np.zeros((params.height, params.width, 3), np.float32)
        rays = C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_caustics(self.h, C.byref(params), photons, seed, _ptr(image), C.byref(rays), 0))
        return image, rays.value

    def caustics_device(self, params, photons, seed, d_image):
        self.ctx.check(self.ctx.L.lrc_caustics(self.h, C.byref(params), photons, seed, C.c_void_p(d_image), None,
                                               LRC_DEVICE))

    def caustics_sums_device(self, params, photons, seed, d_sums):
        self.ctx.check(self.ctx.L.lrc_caustics_sums(self.h, C.byref(params), photons, seed, C.c_void_p(d_sums), None,
                                                    LRC_DEVICE))

    def caustics_sums(self, params, photons, seed, sums=None):
        """lrc_caustics_sums with host sums: returns (sums (h, w, 3) uint64 += the 32.32 values, rays)."""
        if sums is None:
            sums = np.zeros((params.height, params.width, 3), np.uint64)
        rays = C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_caustics_sums(self.h, C.byref(params), photons, seed, _ptr(sums), C.byref(rays),
                                                    0))
        return sums, rays.value

    def trace_stats(self, orig, dirs=None, tmin=0.0, tmax=1e30):
        """(box tests, triangle tests) of the closest-hit walk over these rays: host arrays
        (orig, dirs), or device rays as orig = (count, origins pointer, directions pointer)."""
        stats = np.zeros(2, np.uint64)
        if isinstance(orig, np.ndarray):
            orig = np.ascontiguousarray(orig, np.float32)
            dirs = np.ascontiguousarray(dirs, np.float32)
            self.ctx.check(self.ctx.L.lrc_scene_trace_stats(self.h, _ptr(orig), _ptr(dirs), orig.shape[0], tmin, tmax,
                                                            _ptr(stats), 0))
        else:
            n, po, pd = orig
            self.ctx.check(self.ctx.L.lrc_scene_trace_stats(self.h, C.c_void_p(po), C.c_void_p(pd), n, tmin, tmax,
                                                            _ptr(stats), LRC_DEVICE))
        return int(stats[0]), int(stats[1])

    def occluded(self, orig, dirs, tmax, tmin=0.0):
        orig = np.ascontiguousarray(orig, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        n = orig.shape[0]
        out = np.zeros(n, np.uint8)
        self.ctx.check(self.ctx.L.lrc_scene_occluded(self.h, _ptr(orig), _ptr(dirs), _ptr(tmax), n, tmin, _ptr(out),
                                                     0))
        return out


def pack_tris(quv, mats=None):
    """(n, 9) q, u, v float32 -> (n, 12) u32 words in the reference's GPU layout (put_tris,
    engine/gpu/trace_gpu.c:898-911): flat triangles (n0 = 0xffffffff), material in the top 6 bits."""
    quv = np.ascontiguousarray(quv, np.float32).reshape(-1, 9)
    n = quv.shape[0]
    out = np.zeros((n, 12), np.uint32)
    f = out.view(np.float32)
    f[:, 0:3] = quv[:, 0:3]
    f[:, 4:7] = quv[:, 3:6]
    f[:, 8:11] = quv[:, 6:9]
    out[:, 3] = 0xFFFFFFFF
    out[:, 7] = 0
    m = np.zeros(n, np.uint32) if mats is None else (np.asarray(mats, np.uint32) & 63)
    out[:, 11] = m << 26
    return out


class Batch:
    """A batch of jobs (lrc_batch_*): each job traces a band of one scene's image into a device
    image; a run drains all of them through one persistent kernel (optionally building the scenes
    first, optionally as one CUDA graph)."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.L.lrc_batch_create(ctx.h, C.byref(h)))
        self.h = h
        self.keep = []        # the scenes and parameters the jobs name

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.lrc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, scene, params, spp, d_accum, y0=0, rows=None, spp0=0, builder=-1, key_bits=30, guided=False):
        """lrc_batch_add (guided: lrc_batch_add_guided, d_accum the 4 planes)."""
        rows = params.height if rows is None else rows
        fn = self.ctx.L.lrc_batch_add_guided if guided else self.ctx.L.lrc_batch_add
        self.ctx.check(fn(self.h, scene.h, C.byref(params), y0, rows, spp0, spp, C.c_void_p(d_accum), builder, key_bits))
        self.keep.append((scene, params))
        return len(self.keep) - 1

    def clear(self):
        self.ctx.check(self.ctx.L.lrc_batch_clear(self.h))
        self.keep = []

    def run(self, build=False, graph=False, zero=False, stepped=False, count=False):
        flags = (LRC_BATCH_BUILD if build else 0) | (LRC_BATCH_GRAPH if graph else 0) | (LRC_BATCH_ZERO if zero else 0)
        flags |= (LRC_BATCH_STEPPED if stepped else 0) | (LRC_BATCH_COUNT if count else 0)
        self.ctx.check(self.ctx.L.lrc_batch_run(self.h, flags))

    def step_stats(self):
        """The last stepped run: {intersect_ms, intersect_rays, box_tests, tri_tests, kernels}."""
        ms, rays, bt, tt, k = C.c_double(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_batch_step_stats(self.h, C.byref(ms), C.byref(rays), C.byref(bt), C.byref(tt),
                                                       C.byref(k)))
        return {"intersect_ms": ms.value, "intersect_rays": rays.value, "box_tests": bt.value, "tri_tests": tt.value,
                "kernels": k.value}

    def rays(self):
        """(rays per job, total) of the last run (waits for it)."""
        per = np.zeros(max(len(self.keep), 1), np.uint64)
        tot = C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_batch_rays(self.h, _ptr(per), C.byref(tot)))
        return per[:len(self.keep)], tot.value

    def tune(self, sample_tasks=0):
        v, g, ns = C.c_int32(), C.c_int32(), C.c_double()
        self.ctx.check(self.ctx.L.lrc_batch_tune(self.h, sample_tasks, C.byref(v), C.byref(g), C.byref(ns)))
        return v.value, g.value, ns.value

    def set_shape(self, variant, grid=0):
        self.ctx.check(self.ctx.L.lrc_batch_set_shape(self.h, variant, grid))

    def set_engine(self, engine):
        """0: the persistent megakernel, 1: the wavefront (the default)."""
        self.ctx.check(self.ctx.L.lrc_batch_set_engine(self.h, engine))

    def set_wavefront(self, slots, variant=None):
        variant = LRC_WAVEFRONT_DEFAULT_VARIANT if variant is None else variant
        self.ctx.check(self.ctx.L.lrc_batch_set_wavefront(self.h, slots, variant))

    def engine(self):
        e, m, v = C.c_int32(), C.c_uint32(), C.c_int32()
        self.ctx.check(self.ctx.L.lrc_batch_engine(self.h, C.byref(e), C.byref(m), C.byref(v)))
        return {"engine": e.value, "slots": m.value, "wf_variant": v.value}

    def info(self):
        t, p, v, g, u = C.c_uint64(), C.c_uint64(), C.c_int32(), C.c_int32(), C.c_int32()
        self.ctx.check(self.ctx.L.lrc_batch_info(self.h, C.byref(t), C.byref(p), C.byref(v), C.byref(g), C.byref(u)))
        return {"tasks": t.value, "pixels": p.value, "variant": v.value, "grid": g.value, "graph_used": u.value}


def wavefront_shapes():
    """[(threads per block, register-cap blocks per SM, resident blocks per SM)] of the wavefront's
    closest-hit / shadow kernels' launch shapes."""
    L = lib()
    out = []
    b, m, r = C.c_int32(), C.c_int32(), C.c_int32()
    n = L.lrc_batch_wavefront_shape(0, C.byref(b), C.byref(m), C.byref(r))
    for v in range(max(n, 0)):
        L.lrc_batch_wavefront_shape(v, C.byref(b), C.byref(m), C.byref(r))
        out.append((b.value, m.value, r.value))
    return out


def batch_shapes():
    """[(threads per block, register-cap blocks per SM, resident blocks per SM)] of the batch
    kernel's launch shapes (needs a device for the last)."""
    L = lib()
    out = []
    b, m, r = C.c_int32(), C.c_int32(), C.c_int32()
    n = L.lrc_batch_shape(0, C.byref(b), C.byref(m), C.byref(r))
    for v in range(max(n, 0)):
        L.lrc_batch_shape(v, C.byref(b), C.byref(m), C.byref(r))
        out.append((b.value, m.value, r.value))
    return out


class Server:
    """A render server (lrc_server_*): submit jobs as they arrive, step waves, collect results."""

    def __init__(self, ctx, budget_bytes, wave_paths=1 << 22):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.L.lrc_server_create(ctx.h, budget_bytes, wave_paths, C.byref(h)))
        self.h = h
        self.keep = {}

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.lrc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, scene, params, spp, records=None, tlas_mode=0, denoise=False):
        jid = C.c_uint64()
        mode = tlas_mode | (LRC_SERVE_DENOISE if denoise else 0)
        if records is None:
            rc = self.ctx.L.lrc_server_submit(self.h, scene.h, C.byref(params), spp, None, 0, mode, C.byref(jid))
        else:
            records = np.ascontiguousarray(records, np.float32).reshape(-1, 32)
            rc = self.ctx.L.lrc_server_submit(self.h, scene.h, C.byref(params), spp, _ptr(records), records.shape[0],
                                              mode, C.byref(jid))
        self.ctx.check(rc)
        self.keep[jid.value] = (scene, params)
        return jid.value

    def step(self):
        n = C.c_int32()
        self.ctx.check(self.ctx.L.lrc_server_step(self.h, C.byref(n)))
        return n.value

    def result(self, jid):
        """(device image pointer, rays, t_submit, t_admit, t_done) of a finished job, or None."""
        img, rays = C.c_void_p(), C.c_uint64()
        t0, t1, t2 = C.c_double(), C.c_double(), C.c_double()
        rc = self.ctx.L.lrc_server_result(self.h, jid, C.byref(img), C.byref(rays), C.byref(t0), C.byref(t1),
                                          C.byref(t2))
        if rc == LRC_RETRY:
            return None
        self.ctx.check(rc)
        return img.value, rays.value, t0.value, t1.value, t2.value

    def image(self, jid):
        """A finished job's image as a host array (h, w, 4): the sum of its samples and their count."""
        _, p = self.keep[jid]
        out = np.zeros((p.height, p.width, 4), np.float32)
        self.ctx.check(self.ctx.L.lrc_server_read(self.h, jid, _ptr(out)))
        return out

    def release(self, jid):
        self.ctx.check(self.ctx.L.lrc_server_release(self.h, jid))
        self.keep.pop(jid, None)

    def state(self):
        q, a, f, b = C.c_int32(), C.c_int32(), C.c_int32(), C.c_uint64()
        self.ctx.check(self.ctx.L.lrc_server_state(self.h, C.byref(q), C.byref(a), C.byref(f), C.byref(b)))
        return {"queued": q.value, "active": a.value, "finished": f.value, "bytes": b.value}

    def batch_handle(self):
        return self.ctx.L.lrc_server_batch(self.h)

    def stats(self):
        """(waves run, trace kernels launched, the waves' device ms) so far (lrc_server_stats)."""
        w, k, ms = C.c_uint64(), C.c_uint64(), C.c_double()
        self.ctx.check(self.ctx.L.lrc_server_stats(self.h, C.byref(w), C.byref(k), C.byref(ms)))
        return w.value, k.value, ms.value

    def set_policy(self, policy):
        self.ctx.check(self.ctx.L.lrc_server_set_policy(self.h, policy))

    def set_wavefront(self, slots, variant=None):
        """The waves' wavefront size (paths in flight) and launch shape (None: the default)."""
        variant = LRC_WAVEFRONT_DEFAULT_VARIANT if variant is None else variant
        self.ctx.check(self.ctx.L.lrc_server_set_wavefront(self.h, slots, variant))


def clock_ms():
    return lib().lrc_server_clock()

