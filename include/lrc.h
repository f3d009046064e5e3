/* lrc.h - the C ABI of little_renderer's CUDA backend (B200, sm_100a).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes. It replaces the
 * WebGPU-typed private layer of the reference's GPU path tracer (engine/gpu/gpu_internal.h:
 * 260-313, gpu_trace_*) so that a `cuda` backend implementing the public, WebGPU-free headers
 * engine/gpu/gpu.h:17-71 and engine/gpu/view_gpu.h:49-176 drops in beside the WebGPU/Vulkan one
 * (as NOGPU=1 swaps in stubs, engine/gpu/view_gpu.c:5-46).
 *
 * Status codes follow the reference's conventions (view_gpu.h:65-74): 0 = done; > 0 = this
 * cannot be held now, retry after a change (as gpu_view_trace_start's 0); < 0 = failed for good
 * (as gpu_view_trace_failed). No exception crosses the ABI. lrc_message() says why.
 *
 * Memory: unless LRC_DEVICE is given, every array argument is host memory, copied in and out
 * inside the call. With LRC_DEVICE every array argument is a device pointer of the context's
 * device and nothing is copied.
 */
#ifndef LRC_H
#define LRC_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LRC_OK 0
#define LRC_RETRY 1            /* refusable: out of device memory for this size; retry after a change */
#define LRC_E_INVALID (-1)     /* a bad argument */
#define LRC_E_CUDA (-2)        /* a CUDA error (lrc_message has it); the context may be lost */
#define LRC_E_TIMEOUT (-3)     /* a bounded device wait ran out (the device status word says which) */
#define LRC_E_STACK (-4)       /* a traversal stack would have overflowed (never dropped silently) */
#define LRC_E_NODEVICE (-5)    /* no CUDA device (the caller then path traces on the CPU, gpu.h:32-35) */

#define LRC_DEVICE 1u          /* flag: array arguments are device pointers */
#define LRC_SORT_RAYS 2u       /* flag (ray queries): reorder a large batch by a coherence key first */

typedef struct lrc_ctx lrc_ctx;

/* ---- device and context: replaces gpu_create / gpu_state / gpu_wait / gpu_message /
 * gpu_destroy (engine/gpu/gpu.h:17-71) ------------------------------------------------------- */
/* A context on CUDA device `device`, with its own stream. */
int lrc_open(int device, lrc_ctx **out);
void lrc_close(lrc_ctx *ctx);
/* the last error's text (gpu_message, gpu.h) */
const char *lrc_message(const lrc_ctx *ctx);
/* waits for the context's work (gpu_wait, gpu.h) */
int lrc_sync(lrc_ctx *ctx);
/* later work goes to this CUDA stream (a cudaStream_t; NULL: the context's own) */
int lrc_set_stream(lrc_ctx *ctx, void *cuda_stream);
/* the device status word: bits of bounded waits that ran out (1 sort, 2 PLOC, 8 grid barrier)
 * and of a traversal stack that would have overflowed (4). Read and cleared. */
uint32_t lrc_status(lrc_ctx *ctx);
/* the CUDA device's SM count (for callers sizing their own work) */
int lrc_num_sms(const lrc_ctx *ctx);
/* 1: all the context's work is done, 0: some is still running (does not wait), < 0: an error */
int lrc_query(lrc_ctx *ctx);
/* Device memory for callers without the CUDA runtime (the engine's GPU backend, gpu_cuda.c): an
 * allocation on the context's device (LRC_RETRY when out of memory), its release (after the
 * context's work), a copy that waits for the context's work and itself (kind below), and a
 * zeroing enqueued on the context's stream. */
#define LRC_COPY_H2D 0
#define LRC_COPY_D2H 1
#define LRC_COPY_D2D 2
int lrc_device_alloc(lrc_ctx *ctx, size_t bytes, void **out);
void lrc_device_free(lrc_ctx *ctx, void *p);
int lrc_device_copy(lrc_ctx *ctx, void *dst, const void *src, size_t bytes, int kind);
int lrc_device_zero(lrc_ctx *ctx, void *p, size_t bytes);
/* GPU time by stage (gpu_set_timing, gpu.h; the reference's GpuTimer stages, trace_gpu.c:330-333):
 * on = 1 records CUDA events around each stage of later calls */
#define LRC_TS_BOXES 0       /* triangle boxes and the mesh box */
#define LRC_TS_MORTON 1      /* Morton codes and the radix histograms */
#define LRC_TS_SORT 2        /* the radix sort's passes */
#define LRC_TS_HIERARCHY 3   /* LBVH hierarchy and boxes, or PLOC */
#define LRC_TS_TRACE 4       /* ray queries */
#define LRC_TS_SHADE 5       /* path tracing */
#define LRC_TS_LIGHT 6       /* light tracing (caustics) */
#define LRC_TS_DENOISE 7     /* the denoiser's passes */
#define LRC_NUM_STAGES 8
int lrc_set_timing(lrc_ctx *ctx, int on);
/* milliseconds of each stage (ms[LRC_NUM_STAGES]) and launches of each (optional) since the last
 * call; waits for the context's work */
int lrc_timings(lrc_ctx *ctx, double *ms, int *launches);

/* ---- the BVH builder: replaces build_queue + gpu_trace_build (engine/gpu/trace_gpu.c:587-764;
 * shaders trace_build.wgsl and trace_ploc.wgsl) ----------------------------------------------- */
typedef struct {
    uint32_t n;          /* items (boxes) */
    uint32_t node0;      /* the tree's root goes to nodes[node0]; internal i at node0 + i, leaf j at
                            node0 + n - 1 + j (LBVH); PLOC: internal k's children at node0 + 1 + 2k, + 2 + 2k */
    uint32_t ref0;       /* leaf j's entry in aux: ref0 + j */
    uint32_t ref_add;    /* aux[ref0 + j] = item + ref_add */
    float lo[3];         /* the bounds' low corner (BuildParams.lo) */
    float ext[3];        /* 1 / the bounds' size per axis, 0 on a flat axis (BuildParams.ext) */
    int32_t key_bits;    /* 30: the reference's Morton codes (10 bits per axis); 63: 21 bits per axis */
    int32_t builder;     /* 0 LBVH (Karras), 1 PLOC */
} lrc_build_params;

/* build_queue's parameters from a bounds box (trace_gpu.c:605-611): lo, and ext = 1 / size in float */
void lrc_params_from_bounds(const float lo[3], const float hi[3], lrc_build_params *p);
/* Builds a BVH over n boxes (8 floats each: lo.xyz, -, hi.xyz, -, as build_queue's boxes) into
 * nodes (8 words each: node0 + 2n - 1 of them) and aux (ref0 + n words), node for node and bit
 * for bit the tree the reference's builders make. PLOC needs n >= 3 (as build_queue). */
int lrc_build(lrc_ctx *ctx, const lrc_build_params *p, const float *boxes, uint32_t *nodes, uint32_t *aux,
              unsigned flags);
/* The device scratch memory lrc_build uses for n items (it is the context's, grown as needed). */
size_t lrc_build_scratch_bytes(uint32_t n, int key_bits, int builder);

/* A build that allocates nothing. It has no counterpart in the reference.
 * Some callers cannot call cudaMalloc: a host program that gives out all its device memory up
 * front from its own pool cannot let a library allocate behind its back (the allocation may fail
 * against that budget), and a frame loop that rebuilds a top-level tree every frame cannot afford
 * cudaMalloc's implicit device synchronisation. This is lrc_build with LRC_DEVICE (every array a
 * device pointer of the current device), the same trees bit for bit, its scratch memory in one
 * fixed device array of LRC_STATIC_SCRATCH_BYTES; it calls no cudaMalloc, cudaFree or other
 * allocating routine itself. n above LRC_STATIC_MAX_ITEMS: LRC_E_TOO_BIG, nothing done.
 * The first call on a device sets it up: it finds the array's device address, and since CUDA
 * loads a library's kernels lazily, that is when the driver loads this part of the library and
 * reserves the array on that device (held from then until the process exits; the load may
 * synchronise the device). Make that first call at initialisation, outside the frame loop. The
 * kernels' attributes are set on the first use of each key width and of PLOC. Calls cannot be
 * captured into a CUDA graph: each one waits for its work and reads the status word back.
 * Every call shares the array: calls that overlap on the GPU (other streams, other host threads)
 * race and must not be made. The work goes to cuda_stream (a cudaStream_t; NULL: the default
 * stream) and the call waits for it, returning LRC_OK, LRC_E_TIMEOUT (a bounded device wait ran
 * out) or LRC_E_CUDA. */
#define LRC_E_TOO_BIG (-6)
#define LRC_STATIC_MAX_ITEMS 65536
#define LRC_STATIC_SCRATCH_BYTES (6u << 20)
int lrc_build_static(const lrc_build_params *p, const float *boxes, uint32_t *nodes, uint32_t *aux, void *cuda_stream);

/* triangle_bounds (engine/scene/scene.c:65-74) of n triangles in the reference's GPU layout
 * (12 words each: q.xyz, n0, u.xyz, n1, v.xyz, material << 26 | n2; put_tris, trace_gpu.c:898-911)
 * into boxes (8 floats each), and the mesh box of their corners (SceneMesh.box, scene.c:638-646)
 * into bounds6 (lo.xyz, hi.xyz). */
int lrc_triangle_boxes(lrc_ctx *ctx, const uint32_t *tris, uint32_t n, float *boxes, float *bounds6, unsigned flags);

/* ---- a scene resident on the device: replaces GpuTrace's buffers and uploads
 * (gpu_trace_sync, trace_gpu.c:1571; upload_tris :913, build_queue for meshes :1497-1512) ---- */
typedef struct lrc_scene lrc_scene;
int lrc_scene_create(lrc_ctx *ctx, lrc_scene **out);
void lrc_scene_destroy(lrc_scene *s);
/* the scene's triangles (12 words each, the reference GPU layout). Replaces what it held. */
int lrc_scene_set_triangles(lrc_scene *s, const uint32_t *tris, uint32_t n, unsigned flags);
/* Builds the scene's BVH over its triangles on the device: boxes = triangle_bounds, bounds = the
 * mesh box (as upload_instances queues a dynamic mesh, trace_gpu.c:1497-1512), builder 0 LBVH /
 * 1 PLOC, key_bits 30 or 63. */
int lrc_scene_build(lrc_scene *s, int builder, int key_bits);
/* the scene's nodes (2n - 1) and aux (n) copied out (host), or their device addresses */
int lrc_scene_tree(lrc_scene *s, uint32_t *nodes, uint32_t *aux, unsigned flags);
int lrc_scene_tree_device(lrc_scene *s, const uint32_t **nodes, const uint32_t **aux, uint32_t *n);
/* The scene's world tree given, not built: nnodes nodes in put_nodes' layout (trace_gpu.c:883-896:
 * lo.xyz, a, hi.xyz, b; inner: a, b the children; leaf: a its first aux entry, b = 0x80000000 |
 * count, up to any count) with the root at 0, and naux shape ids (primitives, then triangles) -
 * the engine's own SAH tree (scene_bvh, engine/rt/accel.h:32; Bvh.nodes and .refs), which the
 * reference's GPU path tracer traces (upload_world, trace_gpu.c:1103-1112). Host arrays are
 * checked (children, leaf ranges and shape ids in range). The scene's next lrc_scene_build, or a
 * change of its shapes, replaces it. lrc_scene_tree then copies out nnodes and naux entries. */
int lrc_scene_set_tree(lrc_scene *s, const uint32_t *nodes, uint32_t nnodes, const uint32_t *aux, uint32_t naux,
                       unsigned flags);
/* The walk's tree of a scene of triangles alone (no primitives). mode 1 (the default): after each
 * lrc_scene_build or lrc_scene_set_tree, the ray queries below (closest hit, any hit, walk
 * statistics) follow a copy of the tree - the same nodes and leaves - whose boxes are the
 * triangles' own bounds widened by 2^-17 of the root box's largest coordinate (at most the 1e-3
 * of triangle_bounds, scene.c:65-74), inner boxes their unions: the same hits as the padded tree,
 * fewer box tests where the padding is large beside the triangles. mode 2: that tree collapsed
 * into 8-wide nodes with their children's boxes quantised to bytes (80 bytes a node; a tree whose
 * leaves hold more triangles than a node's slots keeps mode 1). mode 0: the tree as built.
 * lrc_scene_tree always gives the tree as built (the reference's); the path tracer walks that. */
int lrc_scene_set_walk(lrc_scene *s, int mode);

/* Closest hits of nrays rays (origins, directions: 3 floats each) in (tmin, tmax) through the
 * scene's BVH: prim = the triangle hit (-1: none), t. The reference's Moller-Trumbore arithmetic
 * (engine/rt/intersect.h:96-112), bit for bit. Replaces traverse (trace.wgsl:270-392) for
 * closest hits; the CPU counterpart is scene_intersect (engine/rt/accel.c:252). */
int lrc_scene_intersect(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                        int32_t *prim, float *t, unsigned flags);
/* Any hit in (tmin, tmax[i]) (shadow rays; scene_occluded, accel.c:280): out[i] = 1 if blocked */
int lrc_scene_occluded(lrc_scene *s, const float *orig, const float *dir, const float *tmax, uint64_t nrays,
                       float tmin, uint8_t *out, unsigned flags);
/* The closest-hit walk of lrc_scene_intersect, counting instead of answering: stats[0] = box tests
 * (32-byte node records read; with the 8-wide walk, each 80-byte node read counts 2.5), stats[1] =
 * triangle tests (48-byte triangles read), over all rays.
 * The traversal's algorithmic bytes (as the reference's tree statistics, LR_GPU_BVH_CHECK's cost
 * and depth, trace_gpu.c:768-805, describe a tree). stats: host. */
int lrc_scene_trace_stats(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                          uint64_t *stats, unsigned flags);

/* ---- the world besides its triangles: replaces upload_world / upload_layout's primitives,
 * normals and the parameters' materials (trace_gpu.c:1098-1171, 1597-1678) ------------------ */
/* Spheres and quads, 24 floats each as upload_world packs them (trace_gpu.c:1145-1154):
 * center.xyz, radius | q.xyz, 1 for a quad (0 a sphere) | u.xyz, material | v.xyz, area |
 * normal.xyz, plane_d | w.xyz, 0. With primitives the world's shapes are numbered as the
 * reference numbers them (scene.h:101-106): primitives, then triangles; lrc_scene_build builds
 * over both and lrc_scene_intersect returns shape ids. */
int lrc_scene_set_prims(lrc_scene *s, const float *prims, uint32_t n, unsigned flags);
/* vertex normals (3 floats each) that triangles' normal indices (put_tris words 3, 7, 11) refer to */
int lrc_scene_set_normals(lrc_scene *s, const float *normals, uint32_t n, unsigned flags);
/* Materials (engine/scene/scene.h:31-51), 16 floats each: albedo.xyz, type (MatType, as the int's
 * bits) | emission.xyz, 0 | ior, metallic, roughness, transmission | 0, 0, 0, 0. At most 64. Host. */
int lrc_scene_set_materials(lrc_scene *s, const float *mats, uint32_t n);
/* Scene.light: the lamp, a quad primitive sampled by next event estimation (-1: none) */
int lrc_scene_set_light(lrc_scene *s, int32_t prim);
/* Instanced meshes (SceneMesh, scene.h:181-194): nmeshes meshes of tri_counts[m] triangles each,
 * their triangles one mesh after another (12 words each, the GPU layout; flat). Replaces the
 * scene's meshes (and drops their trees: lrc_scene_build_instances builds them again). */
int lrc_scene_set_meshes(lrc_scene *s, const uint32_t *tris, const uint32_t *tri_counts, uint32_t nmeshes, unsigned flags);
/* Instances (scene.h:202-209), 32 floats each: the object-to-world transform (3 x 4, row-major),
 * its inverse (xform_inverse, scene.c:606-623), the world box's lo.xyz and the mesh's index (the
 * int's bits), its hi.xyz and the material (the int's bits; -1: the triangles' own). Host. */
int lrc_scene_set_instances(lrc_scene *s, const float *records, uint32_t n, unsigned flags);
/* Each mesh's BVH (builder 0 LBVH / 1 PLOC, key_bits 30 / 63; built once per lrc_scene_set_meshes)
 * and the top level over the instances' boxes (LBVH, 30-bit keys, the reference's GPU top level,
 * trace_gpu.c:459-460, 1462-1463): after moving instances, only the top level is built again. */
int lrc_scene_build_instances(lrc_scene *s, int mesh_builder, int key_bits);
/* Moved instances (scene_update_instances, engine/rt/accel.c:197-207; the reference's top level
 * follows them in build_tlas, accel.c:154-173): new records for the same n instances (host, or
 * device with LRC_DEVICE), and the top level made again for them - LRC_TLAS_REFIT: the built
 * tree's boxes from its leaves up (bvh_refit_boxes, engine/rt/bvh.c:471-485); LRC_TLAS_REBUILD:
 * built again (LBVH); LRC_TLAS_AUTO: refit while the tree's SAH cost stays within 1.1x of its cost
 * as built, else built again (the reference's TLAS_REFIT_GROWTH policy). */
#define LRC_TLAS_REFIT 0
#define LRC_TLAS_REBUILD 1
#define LRC_TLAS_AUTO 2
int lrc_scene_move_instances(lrc_scene *s, const float *records, uint32_t n, int mode, unsigned flags);
/* The top level's SAH cost (bvh_cost, bvh.c:463-468: the nodes' surface areas over the root's). */
int lrc_scene_tlas_cost(lrc_scene *s, double *cost);
/* The bottom-up refit of any tree these builders made (root at nodes[0], node0 = 0): every box made
 * again from the n items' new boxes (8 floats each, as lrc_build's), the topology kept; boxes to
 * the bit bvh_refit_boxes' on that topology. Host arrays, or device ones with LRC_DEVICE. */
int lrc_refit(lrc_ctx *ctx, uint32_t *nodes, const uint32_t *aux, uint32_t n, uint32_t ref_add, const float *boxes,
              unsigned flags);
/* Materials' textures (the reference's PBR5: Scene.texmaps, Material.tex_*; engine/scene/texture.h,
 * scene.h:42-50): up to 255 RGBA8 images (level 0; the path tracers sample it bilinearly), colour
 * ones sRGB-decoded when read, wrapping as glTF's samplers (0 repeat, 1 clamp, 2 mirror). A
 * material names them in its fourth 4 floats as the GPU backend packs them (gpu_tex_pack,
 * engine/gpu/tex_gpu.c:19-29, as uint32 bits): [12] base | emissive << 8, [13] metal-rough
 * (roughness in green, metallic in blue) | occlusion << 8 | its strength x 255 << 16, [14] normal
 * map | normal scale x 4096 << 8, [15] uv scale (float; 0 = 1); each 1 + a texmap's index, 0
 * none. Replaces the scene's texmaps (n = 0: none). Host arrays. */
typedef struct {
    int32_t w, h;                /* level 0's size */
    int32_t srgb;                /* 1: colour (sRGB-encoded texels) */
    int32_t wrap_u, wrap_v;      /* 0 repeat, 1 clamp, 2 mirror */
    const uint32_t *rgba;        /* w x h texels r | g << 8 | b << 16 | a << 24, rows top to bottom */
} lrc_texmap;
int lrc_scene_set_texmaps(lrc_scene *s, const lrc_texmap *t, uint32_t n);
/* the sRGB decoding table the texmaps use (texmap_srgb_table, texture.c:64-73), host only */
void lrc_srgb_table(float *out256);
/* The world triangles' texture coordinates (Triangle.t, Scene.uvs / .tangents): tri_uv 3 indices
 * per triangle into uvs (2 floats each) and tangents (xyz + handedness w), -1 none (the triangle's
 * barycentrics then, as tri_texcoords' fallback). ntris must be the scene's triangle count when it
 * is traced (else they are not used). Instances' meshes carry none here. Host arrays. */
int lrc_scene_set_texcoords(lrc_scene *s, const int32_t *tri_uv, uint32_t ntris, const float *uvs, const float *tangents,
                            uint32_t nuv);
/* Participating media (engine/scene/volume.h: Volume; scene_add_volume, scene.c:575-583): up to 8
 * voxel grids of density (trilinear between voxel centres, 0 outside), each with its extinction
 * at density 1, single-scattering albedo and Henyey-Greenstein g. Replaces the scene's media (n = 0:
 * none); the majorants (largest density, active box, 8^3-voxel brick maxima) are made here as
 * volume_update makes them. lrc_trace (both modes) and the batch's engine 0 trace them with delta
 * and ratio tracking (engine/rt/medium.c); lrc_caustics stops light paths that scatter in them and
 * dims camera connections through them; the wavefront engine and the server refuse such scenes.
 * Host arrays. */
typedef struct {
    int32_t nx, ny, nz;          /* voxels per axis */
    float lo[3], hi[3];          /* the world box the grid fills */
    float sigma_t;               /* extinction at density 1, per scene unit */
    float albedo[3];             /* single-scattering albedo (sigma_s / sigma_t) */
    float g;                     /* Henyey-Greenstein anisotropy, in (-1, 1) */
    const float *density;        /* nx * ny * nz values >= 0, x fastest: index (z * ny + y) * nx + x */
} lrc_volume;
int lrc_scene_set_volumes(lrc_scene *s, const lrc_volume *v, uint32_t n);
/* The majorants lrc_scene_set_volumes derives for a volume, on the host (volume_update,
 * volume.c:47-108): the largest density, the active box (lo xyz, hi xyz) and the 8^3-voxel bricks'
 * maxima (ceil(nx/8) x ceil(ny/8) x ceil(nz/8), x fastest; NULL: not wanted). */
int lrc_volume_majorants(const lrc_volume *v, float *max_density, float *active6, float *brick_max);
/* The sky (Env, env.h:29-53; upload_sky, trace_gpu.c:1522-1569): w x h linear RGB, rows top to
 * bottom, times scale; its sampling tables (marg: h + 1 floats, cond: h x (w + 1), prob: w x h =
 * env_pixel_prob) or NULL: made here as env_prepare makes them (env.c:116-167, 341-363). Host.
 * rgb NULL: no sky. */
int lrc_scene_set_sky(lrc_scene *s, const float *rgb, int32_t w, int32_t h, const float *marg, const float *cond,
                      const float *prob, float scale);
/* The sky's sampling tables as env_prepare makes them (host only, no device): marg h + 1, cond
 * h x (w + 1), prob w x h. Returns 1, or 0 when no pixel weighs anything. */
int lrc_sky_tables(const float *rgb, int32_t w, int32_t h, float *marg, float *cond, float *prob);
/* Closest hits as scene_intersect's Hit (accel.c:252): prim = the world's shape id (primitives,
 * then triangles) or, on an instance, the triangle's index in its mesh; inst = the instance or -1 */
int lrc_scene_intersect_ex(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                           int32_t *prim, int32_t *inst, float *t, unsigned flags);
/* The blue-noise mask (64 x 64 ranks; blue_noise_mask(), engine/base/sampler.c) and the BSDF tables
 * (2112 floats packed as gpu_bsdf_tables packs scene/brdf_tables.h, engine/gpu/brdf_gpu.c:20-25),
 * both host. NULL: the ones lrc_default_blue_noise / lrc_default_bsdf_tables make. */
int lrc_scene_set_tables(lrc_scene *s, const uint16_t *blue_noise, const float *bsdf_tables);
/* the mask and the tables made here by the reference's published methods (void-and-cluster;
 * the GGX albedo integrals): the same mask as the reference's, the tables within 1e-6 */
void lrc_default_blue_noise(uint16_t *out4096);
void lrc_default_bsdf_tables(float *out2112);

/* ---- the path tracer: replaces gpu_trace_encode + the megakernel `main` / `trace()`
 * (trace_gpu.c:1935-2031; trace.wgsl:1125-1316); the CPU counterpart is trace_image /
 * trace_path_sampled (engine/rt/tracer.c:329-545) -------------------------------------------- */
typedef struct {
    float origin[3], upper_left[3], horizontal[3], vertical[3];   /* Camera (engine/scene/camera.h:15-20) */
    int32_t width, height;
    int32_t max_depth;     /* bounces per path */
    int32_t mis;           /* next event estimation weighted by the power heuristic */
    int32_t sampler;       /* 1: Owen-scrambled Sobol + blue noise; 0: plain random (GpuTraceParams.random) */
    int32_t exact;         /* 1: trace_image's random streams (per pixel, samples in order): the CPU's image
                              up to transcendental rounding; 0: a stream per sample (faster) */
    uint64_t seed;         /* the image's seed (trace_image's) */
    float clamp;           /* largest sample value, 0: none */
    int32_t skip_caustics; /* 1: leave out the paths light tracing covers (camera -> diffuse first,
                              then the lamp right after a mirror / glass vertex; TraceParams.skip_caustics,
                              engine/rt/tracer.h:16-20): set it when lrc_caustics adds them */
    float indirect_clamp;  /* after a path's first rough bounce, each light it brings is held to this
                              much (its largest channel); 0: no limit (TraceParams.indirect_clamp,
                              engine/rt/tracer.h:35; GpuTraceParams.indirect_clamp, view_gpu.h:62) */
} lrc_trace_params;
/* Samples [spp0, spp0 + spp) of every pixel of rows [y0, y0 + rows), added into accum (width x
 * height x 4 floats: the sum of the samples' linear RGB and their count, as gpu_view_trace_read
 * gives them, view_gpu.h:118-124). exact = 1 needs spp0 = 0 (the streams start at each pixel's
 * first sample). rays (optional, host): the closest-hit and shadow rays traced.
 * A call of at least LRC_TRACE_WAVEFRONT_PATHS paths (width x rows x spp) on a scene without media
 * runs as a one-job batch on the wavefront engine (the batch's image is this call's to the bit);
 * smaller ones, scenes with media and calls with LRC_TRACE_MEGAKERNEL run the one-kernel path. */
int lrc_trace(lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0, uint32_t spp,
              float *accum, uint64_t *rays, unsigned flags);
#define LRC_TRACE_GUIDED 64u  /* flag: accum is the denoiser's 4 planes (below); each sample's luminance
                                 over the guide's albedo is added to plane 1's (sum l, sum l^2) */
#define LRC_TRACE_MEGAKERNEL 256u  /* flag: the one-kernel path tracer whatever the size */
#define LRC_TRACE_WAVEFRONT_PATHS (1u << 20)

/* ---- the denoiser: replaces gpu_denoise_create / gpu_denoise_encode (engine/gpu/denoise_gpu.c;
 * denoise.wgsl `prep`, `atrous`) and the guide pass `gbuf` (trace.wgsl:1045-1104, 1319-1337) ----
 * Planes: 4 arrays of width x height float4 back to back, as the reference's path tracer keeps
 * them: 0 the samples' sum and count (lrc_trace's accum), 1 the luminance moments, 2 the guide's
 * normal and distance, 3 its albedo and kind (0 a rough surface, 1 a lamp / the sky / nothing,
 * 2 a medium; + 4 (instance + 1)). A new image: planes 0 and 1 zeroed, lrc_guide, then lrc_trace
 * with LRC_TRACE_GUIDED, then lrc_denoise whenever an image is wanted.
 * lrc_guide: planes 2 and 3 from the ray through each pixel's centre to its first rough surface,
 *   through mirrors and glass (the whole image; planes 0 and 1 are not touched).
 * lrc_denoise: out (width x height float4: rgb, 1) = the edge-avoiding a-trous filter of the
 *   planes, steered by each pixel's variance (passes 1-5, the hole sizes 1, 2, 4, 8, 16; other
 *   values: 5). Arrays are host memory, or device memory with LRC_DEVICE. */
int lrc_guide(lrc_scene *s, const lrc_trace_params *p, float *planes, unsigned flags);
/* A new image's samples carried over from the previous one (gpu_trace_begin_image with history > 0,
 * trace_gpu.c:2020-2060; trace_reproject.wgsl `main`), without temporal gradients: each new pixel's
 * first surface (its guide, planes 2 and 3 of new_planes, made by lrc_guide) is placed in the old
 * camera's image, and the old pixels around that point that saw the same surface (kind and
 * object, distance within 2 % plus its local change, normal within ~25 degrees) give it their
 * samples and moments, bilinearly weighted, at most `history` samples' worth. Writes planes 0 and
 * 1 of new_planes (cleared where nothing matched). Both images of the same size. */
int lrc_reproject(lrc_ctx *ctx, const lrc_trace_params *old_cam, const lrc_trace_params *new_cam, const float *old_planes,
                  float *new_planes, int32_t history, unsigned flags);
/* The same with temporal gradients (A-SVGF; gpu_trace_begin_image with history_max > 0,
 * trace_gpu.c:2081-2114; trace_reproject.wgsl gmatch, gfilter and main with dims.w = 1;
 * trace.wgsl main's gradient branch, :1231-1293): each pixel keeps a history of its own, from how
 * much the light changed where it is.
 *   - per tile of 4 x 4 new pixels one surface pixel k (the first from a point that moves each
 *     image) whose place in the old image is an old pixel o that saw the same surface, and o's last
 *     sample (plane 1's z and w of old_planes: lrc_trace with LRC_TRACE_GUIDED in fast mode keeps
 *     them);
 *   - that sample traced again in s (the new scene, new_p's camera) from the same random numbers
 *     (old_p's seed and sampler, o's stream, its sample number from its low 24 bits and spp0's
 *     high bits) through k moved by o's offset: lambda = |l - old l| / max(l, old l) of the two
 *     samples' luminance over the albedo;
 *   - lambda filtered over the tiles (3 a-trous passes, 1, 2 and 4 tiles apart, weighted by the
 *     tiles' first pixels' distance and normal);
 *   - each pixel keeps floor((1 - lambda) / lambda + 1/2) samples' worth of its old ones, at most
 *     history_max (all where nothing changed, none where a shadow moved); `history` where no tile
 *     near had a lambda. With LRC_REPROJECT_EDIT (the scene was edited: colours may have changed,
 *     which lambda does not see) lambda counts 4 times, a surface's samples are kept only where
 *     its albedo is the same, and lamps, the sky and media keep `history`.
 * new_planes: planes 2 and 3 made by lrc_guide for new_p; planes 0 and 1 are written. spp0: the
 * new image's first sample number (sample numbers keep counting from image to image). tiles_out
 * (optional): per tile (row-major) 4 floats (k, o, the sample's lambda, the filtered lambda), -1
 * for none (k and o exact below 2^24 pixels). old_p in fast mode (exact = 0); history_max > 0. */
#define LRC_REPROJECT_EDIT 128u
int lrc_reproject_gradients(lrc_scene *s, const lrc_trace_params *old_p, const lrc_trace_params *new_p, uint32_t spp0,
                            const float *old_planes, float *new_planes, int32_t history_max, int32_t history,
                            float *tiles_out, unsigned flags);
/* A viewer's frame in one call (gpu_trace_begin_image with its reprojection and gradients, then
 * the frame's samples; trace_gpu.c:2040-2114): new_planes (4 planes) = lrc_guide(new_p), then
 * lrc_reproject_gradients (history_max > 0) or lrc_reproject (history_max = 0) from old_planes
 * (null: the first frame, no history), then lrc_trace(new_p, spp0, spp, LRC_TRACE_GUIDED) - the
 * same planes to the bit, in one stream of launches with host copies (without LRC_DEVICE) of
 * the old planes in and the new ones out only. Fast mode only (new_p and old_p with exact = 0). */
int lrc_trace_frame(lrc_scene *s, const lrc_trace_params *old_p, const lrc_trace_params *new_p, uint32_t spp0,
                    uint32_t spp, const float *old_planes, float *new_planes, int32_t history_max, int32_t history,
                    unsigned flags);
int lrc_denoise(lrc_ctx *ctx, int32_t width, int32_t height, const float *planes, int32_t passes, float *out,
                unsigned flags);

/* ---- light-traced caustics: replaces light_trace_caustics (engine/rt/tracer.c:553-665) and the
 * GPU backend's `ltrace` pass into its 64-bit caustic sums (gpu_trace_light, trace_gpu.c:1946-1954;
 * trace.wgsl:1415-1511) ------------------------------------------------------------------------
 * `photons` light paths from the scene's lamp through mirrors / glass onto rough surfaces, each
 * such vertex joined to the camera of p (width, height, max_depth, exact: the random streams as
 * lrc_trace's modes; the other fields are not read). Light tracing covers exactly the paths
 * lrc_trace leaves out with p->skip_caustics = 1, so the two images added are the full image.
 * Contributions are summed as 32.32 fixed-point integers (value * 2^32 / photons, rounded to the
 * nearest) with integer atomics: the result does not depend on the order or the launch.
 * No lamp, or no material with a perfectly smooth (mirror / glass) part: nothing is added.
 * lrc_caustics: image (width x height x 3 floats, linear RGB) += the caustic image (the sums /
 *   2^32, light_trace_caustics' `out +=`).
 * lrc_caustics_sums: sums (width x height x 3 uint64, 32.32) += the fixed-point values, the GPU
 *   backend's `caus` buffer; after passes of equal photon counts the image is sums / 2^32 / passes.
 * Arrays are host memory, or device memory with LRC_DEVICE. rays (optional, host): the closest-hit
 * and shadow rays traced. */
int lrc_caustics(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, uint64_t seed, float *image,
                 uint64_t *rays, unsigned flags);
int lrc_caustics_sums(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, uint64_t seed, uint64_t *sums,
                      uint64_t *rays, unsigned flags);
/* the light tracer's launch variant for later calls on ctx (its register cap as blocks of 128
 * threads per SM: 4, 5, 6, 7, 8, 10; -1 the default, 8): returns how many there are. Results do
 * not depend on it. */
int lrc_caustics_variant(lrc_ctx *ctx, int variant);

/* ---- batches: many jobs over many resident scenes, built and traced together --------------
 * No counterpart in the reference, which traces one scene per dispatch and sizes its submits by
 * the band scheduler (gpu_view_trace_more, engine/gpu/view_gpu.c:1081-1190); a batch replaces a
 * sequence of lrc_trace calls. Every job's samples are the ones lrc_trace draws for the same
 * arguments and are added into its image in lrc_trace's order: a batched image equals the
 * lrc_trace image to the bit, in exact and fast mode. Images are device arrays; the scenes and
 * images a batch names must outlive it (or its lrc_batch_clear). */
typedef struct lrc_batch lrc_batch;
#define LRC_BATCH_BUILD 4u    /* build each job's scene first (its builder and key bits; once per scene) */
#define LRC_BATCH_GRAPH 8u    /* run as one CUDA graph: captured after the first such run (which runs
                                 uncaptured, sizing every buffer), replayed while nothing it names changed
                                 (the wavefront keeps its graph before too, and goes back to it when runs
                                 alternate: jobs with instances, then without) */
#define LRC_BATCH_ZERO 16u    /* clear each job's band of its image first */
#define LRC_BATCH_STEPPED 32u /* wavefront: launch each pass's kernels from the host, no graph (slower;
                                 for profilers that cannot see into a graph's loop); not with GRAPH */
#define LRC_BATCH_COUNT 64u   /* with STEPPED: the closest-hit walks count their box and triangle tests
                                 (lrc_batch_step_stats) */
int lrc_batch_create(lrc_ctx *c, lrc_batch **out);
void lrc_batch_destroy(lrc_batch *b);
/* A job: lrc_trace(s, p, y0, rows, spp0, spp, d_accum, ..., LRC_DEVICE) as part of the batch;
 * builder 0 (LBVH) / 1 (PLOC) / 2 (LBVH, then PLOC: the PLOC tree is traced) with key_bits 30 / 63
 * builds the scene's world tree in a LRC_BATCH_BUILD run, -1 traces the tree it has (instanced
 * scenes: -1). A scene in several jobs is built once, by its first job's builder. */
int lrc_batch_add(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0,
                  uint32_t spp, float *d_accum, int32_t builder, int32_t key_bits);
/* The same with the denoiser's 4 planes (device; the guide made by lrc_guide): lrc_trace with
 * LRC_TRACE_GUIDED as part of the batch (the moments added as the plain call adds them, to the
 * bit; LRC_BATCH_ZERO clears the band's planes 0 and 1). */
int lrc_batch_add_guided(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows,
                         uint32_t spp0, uint32_t spp, float *d_planes, int32_t builder, int32_t key_bits);
int lrc_batch_clear(lrc_batch *b);
int lrc_batch_jobs(const lrc_batch *b);
/* Enqueues the run on the context's stream (lrc_sync or lrc_batch_rays wait for it). */
int lrc_batch_run(lrc_batch *b, unsigned flags);
/* After a run (synchronises): rays traced per job (in lrc_batch_add order) and in all; either NULL. */
int lrc_batch_rays(lrc_batch *b, uint64_t *per_job, uint64_t *total);
/* After a run (synchronises): the wavefront's passes (bounces of the paths in flight, 0 for the
 * megakernel engine) and the trace kernels the run launched (optional, either NULL). */
int lrc_batch_passes(lrc_batch *b, uint32_t *passes, uint64_t *kernels);
/* The last LRC_BATCH_STEPPED run of the wavefront (each optional): its closest-hit kernel's device
 * time (CUDA events around each launch) and the rays it traced; with LRC_BATCH_COUNT its walks' box
 * tests (32-byte node records read) and triangle tests (48-byte triangles read), counted by a
 * counting build of that kernel (for the launch shapes of 128 threads, registers capped for 4 or 8
 * blocks an SM, the default's among them; with other shapes the counts are 0; it tests what the
 * plain one does: the same hits, the images the same to the bit); and the kernels the run
 * launched. */
int lrc_batch_step_stats(const lrc_batch *b, double *intersect_ms, uint64_t *intersect_rays, uint64_t *box_tests,
                         uint64_t *tri_tests, uint64_t *kernels);
/* The trace kernel's launch shapes: shape `variant`'s threads per block, the blocks per SM its
 * registers are capped for, and the blocks that fit per SM; returns the number of shapes, or -1. */
int lrc_batch_shape(int32_t variant, int32_t *block, int32_t *minb, int32_t *per_sm);
/* Sets the launch shape: variant, grid blocks (0: as many as are resident at once). */
int lrc_batch_set_shape(lrc_batch *b, int32_t variant, int32_t grid);
/* The engine: 1 (the default) the wavefront - a pool of paths in flight advanced by four kernels
 * per bounce (advance / closest hit / shade / shadow rays) looped inside one CUDA graph; 0 the
 * persistent megakernel (one path per lane, the next sample started when a path ends). Both give
 * the same images. */
int lrc_batch_set_engine(lrc_batch *b, int32_t engine);
/* The wavefront's size (paths in flight: a multiple of 256) and its kernels' launch shape
 * (lrc_batch_wavefront_shape describes the closest-hit / shadow kernels' as lrc_batch_shape does;
 * each shape also caps the shading kernel's registers). LRC_WAVEFRONT_DEFAULT_VARIANT is the shape
 * a batch starts with, and the one lrc_trace and the server use: 128 threads a block, the
 * closest-hit and shadow kernels' registers capped for 8 blocks an SM, the shading kernel's for 4
 * (the fastest of the shapes on a served stream of path-traced jobs). */
#define LRC_WAVEFRONT_DEFAULT_VARIANT 9
int lrc_batch_set_wavefront(lrc_batch *b, uint32_t slots, int32_t variant);
int lrc_batch_wavefront_shape(int32_t variant, int32_t *block, int32_t *minb, int32_t *per_sm);
int lrc_batch_engine(const lrc_batch *b, int32_t *engine, uint32_t *slots, int32_t *wf_variant);
/* The autotuner: times the engine's shapes on the first sample_tasks tasks of the queue (0: a
 * sixteenth; for the wavefront at least 2^24 tasks, or all) and keeps the fastest - the megakernel's launch shape (variant, grid blocks), or the
 * wavefront's size and launch shape (variant, grid = paths in flight) - and the ns per task (each
 * optional). Changes no image. */
int lrc_batch_tune(lrc_batch *b, uint64_t sample_tasks, int32_t *variant, int32_t *grid, double *ns_per_task);
/* The last prepared run: its tasks ((pixel, lane slot) pairs), pixels, shape, grid and whether it
 * replayed a graph. */
int lrc_batch_info(const lrc_batch *b, uint64_t *tasks, uint64_t *pixels, int32_t *variant, int32_t *grid,
                   int32_t *graph_used);

/* ---- a render server: jobs admitted as they arrive, traced together in waves --------------
 * No counterpart in the reference (its GPU view traces one scene at a time, paced by the band
 * scheduler, engine/gpu/view_gpu.c:1081-1190). Jobs are admitted in arrival order while their
 * device bytes (the image; for moved instances, their own records and top level) fit the budget;
 * each wave traces the next band of rows of every admitted job as one batch (the wavefront), the
 * wave's paths shared evenly, so jobs that arrive join at the next wave and small jobs finish in a
 * wave or two. A band holds all of its pixels' samples: a job's image is the lrc_trace image of it
 * alone, to the bit. One host thread drives a server. */
typedef struct lrc_server lrc_server;
int lrc_server_create(lrc_ctx *c, uint64_t hbm_budget_bytes, uint64_t wave_paths, lrc_server **out);
void lrc_server_destroy(lrc_server *sv);
/* Queues a job: the whole image p (fast mode) of scene s at spp samples per pixel. records (host, n
 * x 32 floats as lrc_scene_set_instances's; n = the scene's instance count) moves its instances for
 * this job only: the job gets its own copy of the instance layer, its top level refit
 * (LRC_TLAS_REFIT) or built again (LRC_TLAS_REBUILD) on the device when admitted; NULL: the scene
 * as it is. tlas_mode | LRC_SERVE_DENOISE: the job is traced with the denoiser's planes (lrc_guide
 * at admission, the moments with its samples) and its result is lrc_denoise's image (rgb, 1); it
 * holds 80 bytes a pixel while traced, 16 once done. A job larger than the whole budget:
 * LRC_E_TOO_BIG. */
#define LRC_SERVE_DENOISE 16
int lrc_server_submit(lrc_server *sv, lrc_scene *s, const lrc_trace_params *p, uint32_t spp, const float *records,
                      uint32_t n, int tlas_mode, uint64_t *id);
/* One step: admission, then the next wave (bands of the admitted jobs with rows left, as the
 * policy below makes them) planned and launched as one batch run, then the wave launched by the
 * step before waited for and the jobs whose last band it held finished; *finished: those jobs. The
 * waves alternate between two batches, so the device runs one wave while the host plans the next. */
int lrc_server_step(lrc_server *sv, int32_t *finished);
/* A finished job (LRC_RETRY while not): its image (device, W x H x 4 floats: sum and count; complete
 * on the context's stream, or through lrc_server_read), its rays, and the server clock's times (ms)
 * of its submit, admission and end. */
int lrc_server_result(lrc_server *sv, uint64_t id, const float **d_image, uint64_t *rays, double *t_submit,
                      double *t_admit, double *t_done);
/* A finished job's image copied to host memory (W x H x 4 floats; gpu_view_trace_read's sum and
 * count, view_gpu.h:118-124); waits. LRC_RETRY while the job is not finished. */
int lrc_server_read(lrc_server *sv, uint64_t id, float *out);
/* Frees a finished job (its image) and its bytes in the budget. */
int lrc_server_release(lrc_server *sv, uint64_t id);
int lrc_server_state(const lrc_server *sv, int32_t *queued, int32_t *active, int32_t *finished, uint64_t *bytes);
/* The server's clock (ms; monotonic). */
double lrc_server_clock(void);
/* The first of the two batches a server runs its waves with (do not add jobs). */
lrc_batch *lrc_server_batch(lrc_server *sv);
/* The waves' wavefront size (paths in flight) and closest-hit / shadow launch shape, both batches
 * (lrc_batch_set_wavefront). */
int lrc_server_set_wavefront(lrc_server *sv, uint32_t slots, int32_t variant);
/* waves run so far, the trace kernels they launched and their device time (CUDA events from each
 * wave's launch to its end), each optional */
int lrc_server_stats(const lrc_server *sv, uint64_t *waves, uint64_t *kernels, double *gpu_ms);
/* How a wave is made from the admitted jobs: 0 the next band of every job, the wave's paths shared
 * evenly; 1 the oldest jobs first, each band as large as the wave's paths left allow (fewer scenes a
 * wave); 2 (the default) as 1 with the jobs that have the fewest paths left first. */
int lrc_server_set_policy(lrc_server *sv, int32_t policy);

#ifdef __cplusplus
}
#endif
#endif
