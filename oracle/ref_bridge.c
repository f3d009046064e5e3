// ref_bridge.c - TEST INFRASTRUCTURE (the oracle). Compiled together with the reference's own
// CPU engine (engine/{base,formats,scene,rt}/*.c, by oracle/Makefile) into _ref/libref_f.so
// (float build) and _ref/libref_d.so (double build, -DLR_DOUBLE). It turns flat arrays into a
// reference Scene through the reference's public API and runs the reference's own code on it:
//   closest hit  scene_intersect   (engine/rt/accel.c:252)
//   any hit      scene_occluded    (engine/rt/accel.c:280)
//   image        trace_image       (engine/rt/tracer.c:329)
//   caustics     light_trace_caustics (engine/rt/tracer.c:553)
//   guide        the denoiser's guide of the GPU path tracer (trace.wgsl guide(): it has no CPU
//                counterpart), restated here on the reference's Scene, scene_intersect and BSDF
//   boxes        triangle_bounds   (engine/scene/scene.c:65)
// and counts the tracer's rays through link-time --wrap of scene_intersect/scene_occluded
// (no edit of the reference). Nothing of the product path calls this file.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "scene/scene.h"
#include "scene/env.h"
#include "rt/accel.h"
#include "rt/bvh.h"
#include "rt/tracer.h"
#include "rt/intersect.h"
#include "scene/brdf.h"
#include "scene/volume.h"
#include "scene/texture.h"
#include "base/sampler.h"
#include "scene/brdf_tables.h"

// ---- ray counters: one slot per OpenMP thread, 64 bytes apart ----------------------------
#define RB_MAX_THREADS 256
static long long rb_cnt[RB_MAX_THREADS * 8][2];

int __real_scene_intersect(const Scene *s, const Ray *ray, real tmin, real tmax, Hit *h);
int __real_scene_occluded(const Scene *s, const Ray *ray, real tmin, real tmax);

int __wrap_scene_intersect(const Scene *s, const Ray *ray, real tmin, real tmax, Hit *h){
    rb_cnt[(omp_get_thread_num() & (RB_MAX_THREADS - 1)) * 8][0]++;
    return __real_scene_intersect(s, ray, tmin, tmax, h);
}
int __wrap_scene_occluded(const Scene *s, const Ray *ray, real tmin, real tmax){
    rb_cnt[(omp_get_thread_num() & (RB_MAX_THREADS - 1)) * 8][1]++;
    return __real_scene_occluded(s, ray, tmin, tmax);
}
void rb_rays_reset(void){ memset(rb_cnt, 0, sizeof(rb_cnt)); }
// out[0] closest-hit rays, out[1] shadow rays since the last reset
void rb_rays(long long *out){
    out[0] = out[1] = 0;
    for (int i = 0; i < RB_MAX_THREADS; i++){ out[0] += rb_cnt[i * 8][0]; out[1] += rb_cnt[i * 8][1]; }
}
int rb_real_is_double(void){ return sizeof(real) == sizeof(double); }
int rb_max_threads(void){ return omp_get_max_threads(); }
void rb_set_threads(int n){ if (n > 0) omp_set_num_threads(n); }

// ---- scenes ---------------------------------------------------------------------------------
static Vec3 v3f(const float *p){ return vec3(p[0], p[1], p[2]); }

void *rb_scene_new(void){
    Scene *s = calloc(1, sizeof(Scene));
    if (s) s->light = -1;
    return s;
}
void rb_scene_free(void *sp){
    Scene *s = sp;
    if (!s) return;
    scene_free(s);
    free(s);
}

// a material: type (MatType), albedo, emission, ior, metallic, roughness, transmission
int rb_add_material(void *sp, int type, const float *albedo, const float *emission, float ior, float metallic,
                    float roughness, float transmission){
    Material m;
    memset(&m, 0, sizeof(m));
    m.type = (MatType)type;
    m.albedo = v3f(albedo);
    m.emission = v3f(emission);
    m.ior = ior; m.metallic = metallic; m.roughness = roughness; m.transmission = transmission;
    return scene_add_material(sp, m);
}
// the reference's presets (scene.h:48-70), for scene generators that name them
int rb_add_material_preset(void *sp, int kind, const float *rgb, float a, float b){
    Vec3 c = v3f(rgb);
    Material m;
    switch (kind){
    case 0: m = material_diffuse(c); break;
    case 1: m = material_mirror(c); break;
    case 2: m = material_glass(c, a); break;
    case 3: m = material_light(c); break;
    case 4: m = material_pbr(c, a, b, 1.5, 0); break;          // metal: metallic a, roughness b
    default: m = material_pbr(c, 0, b, a, 1); break;            // rough glass: ior a, roughness b
    }
    return scene_add_material(sp, m);
}

// n triangles by their corners (9 floats each: a, b, c), flat (no vertex normals)
void rb_add_triangles(void *sp, const float *corners, const int *mats, int n){
    for (int i = 0; i < n; i++){
        const float *c = corners + 9 * (size_t)i;
        scene_add_triangle(sp, v3f(c), v3f(c + 3), v3f(c + 6), NULL, mats[i]);
    }
}
// a quad primitive (make_quad); light = 1 makes it Scene.light. Returns its index.
int rb_add_quad(void *sp, const float *q, const float *u, const float *v, int mat, int light){
    Scene *s = sp;
    int i = scene_add_prim(s, make_quad(v3f(q), v3f(u), v3f(v), mat));
    if (light) s->light = i;
    return i;
}
int rb_add_sphere(void *sp, const float *c, float r, int mat){ return scene_add_prim(sp, make_sphere(v3f(c), r, mat)); }

// an instanced mesh from corners (9 floats per triangle), flat, material per triangle
int rb_add_mesh(void *sp, const float *corners, const int *mats, int n){
    Triangle *t = malloc((size_t)(n ? n : 1) * sizeof(Triangle));
    Vec3 *nrm = malloc(sizeof(Vec3));
    for (int i = 0; i < n; i++){
        const float *c = corners + 9 * (size_t)i;
        Vec3 a = v3f(c), b = v3f(c + 3), d = v3f(c + 6);
        t[i].q = a; t[i].u = v_sub(b, a); t[i].v = v_sub(d, a);
        for (int k = 0; k < 3; k++){ t[i].n[k] = -1; t[i].t[k] = -1; }
        t[i].material = mats[i];
    }
    return scene_add_mesh_arrays(sp, t, n, nrm, 0, NULL, NULL, 0);
}
// an instance of mesh `mesh` by its 3x4 row-major transform
int rb_add_instance(void *sp, int mesh, const float *xf12, int material){
    Xform x;
    for (int r = 0; r < 3; r++) for (int k = 0; k < 4; k++) x.m[r][k] = xf12[4 * r + k];
    return scene_add_instance(sp, mesh, x, material);
}
void rb_move_instance(void *sp, int inst, const float *xf12){
    Xform x;
    for (int r = 0; r < 3; r++) for (int k = 0; k < 4; k++) x.m[r][k] = xf12[4 * r + k];
    scene_move_instance(sp, inst, x);
}
// instance i's world box (6 floats) and inverse transform (12)
void rb_instance_data(const void *sp, int i, float *box6, float *inv12){
    const Scene *s = sp;
    const Instance *in = &s->insts[i];
    box6[0] = in->box.lo.x; box6[1] = in->box.lo.y; box6[2] = in->box.lo.z;
    box6[3] = in->box.hi.x; box6[4] = in->box.hi.y; box6[5] = in->box.hi.z;
    for (int r = 0; r < 3; r++) for (int k = 0; k < 4; k++) inv12[4 * r + k] = in->inv.m[r][k];
}
void rb_mesh_box(const void *sp, int mesh, float *box6){
    const Scene *s = sp;
    const Aabb *b = &s->meshes[mesh].box;
    box6[0] = b->lo.x; box6[1] = b->lo.y; box6[2] = b->lo.z; box6[3] = b->hi.x; box6[4] = b->hi.y; box6[5] = b->hi.z;
}
// a sky from w x h linear RGB floats (copied; the scene owns it)
// a material's texture map (the reference's TexMap: texmap_make from w x h RGBA8 texels, its wrap
// modes; scene_add_texmap): returns its number (1 + index) or 0
int rb_add_texmap(void *sp, const uint32_t *rgba, int w, int h, int srgb, int wrap_u, int wrap_v){
    TexMap t;
    memset(&t, 0, sizeof(t));
    if (texmap_make(&t, (const unsigned char *)rgba, w, h, srgb)) return 0;
    t.wrap_u = wrap_u;
    t.wrap_v = wrap_v;
    return scene_add_texmap(sp, &t);
}
// material mat's textures (Material.tex_*, uv_scale, normal_scale)
void rb_material_textures(void *sp, int mat, int base, int mr, int normal, int emissive, int occlusion, float uv_scale,
                          float normal_scale){
    Material *m = &((Scene *)sp)->mats[mat];
    m->tex_base = base; m->tex_mr = mr; m->tex_normal = normal; m->tex_emissive = emissive; m->tex_occlusion = occlusion;
    m->uv_scale = uv_scale;
    m->normal_scale = normal_scale;
}
// the world triangles' texture coordinates: Triangle.t (3 per triangle, -1 none), Scene.uvs and
// .tangents (nuv each)
void rb_set_texcoords(void *sp, const int *tri_uv, int ntris, const float *uvs, const float *tangents, int nuv){
    Scene *s = sp;
    s->uvs = malloc(sizeof(Vec2) * (size_t)(nuv > 0 ? nuv : 1));
    s->tangents = malloc(sizeof(Vec4) * (size_t)(nuv > 0 ? nuv : 1));
    for (int i = 0; i < nuv; i++){
        s->uvs[i] = (Vec2){uvs[2 * i], uvs[2 * i + 1]};
        s->tangents[i] = (Vec4){tangents[4 * i], tangents[4 * i + 1], tangents[4 * i + 2], tangents[4 * i + 3]};
    }
    s->nuvs = s->cap_uvs = nuv;
    for (int i = 0; i < ntris && i < s->ntris; i++)
        for (int k = 0; k < 3; k++) s->tris[i].t[k] = tri_uv[3 * i + k];
}

// a volume's majorants as volume_update makes them (volume_create + the density + volume_update):
// the largest density, the active box (lo, hi) and the bricks' maxima
void rb_volume_majorants(int nx, int ny, int nz, const float *box6, const float *density, float *max_density,
                         float *active6, float *brick_max){
    Aabb b = {v3f(box6), v3f(box6 + 3)};
    Volume *v = volume_create(nx, ny, nz, b);
    if (!v) return;
    memcpy(v->density, density, sizeof(float) * (size_t)nx * ny * nz);
    volume_update(v);
    *max_density = (float)v->max_density;
    active6[0] = (float)v->active.lo.x; active6[1] = (float)v->active.lo.y; active6[2] = (float)v->active.lo.z;
    active6[3] = (float)v->active.hi.x; active6[4] = (float)v->active.hi.y; active6[5] = (float)v->active.hi.z;
    memcpy(brick_max, v->brick_max, sizeof(float) * (size_t)v->bnx * v->bny * v->bnz);
    volume_free(v);
}
// the sRGB table texmap_srgb_table makes
void rb_srgb_table(float *out){ memcpy(out, texmap_srgb_table(), sizeof(float) * 256); }

// a participating medium: volume_create + the density + its optics + volume_update + scene_add_volume
// (box6: lo, hi; albedo3; density nz * ny * nx, x fastest). Returns its index or -1.
int rb_add_volume(void *sp, int nx, int ny, int nz, const float *box6, float sigma_t, const float *albedo3, float g,
                  const float *density){
    Aabb b = {v3f(box6), v3f(box6 + 3)};
    Volume *v = volume_create(nx, ny, nz, b);
    if (!v) return -1;
    memcpy(v->density, density, sizeof(float) * (size_t)nx * ny * nz);
    v->sigma_t = sigma_t;
    v->albedo = v3f(albedo3);
    v->g = g;
    volume_update(v);
    return scene_add_volume(sp, v);
}

int rb_set_env(void *sp, const float *rgb, int w, int h){
    Scene *s = sp;
    float *c = malloc(sizeof(float) * 3 * (size_t)w * h);
    if (!c) return 0;
    memcpy(c, rgb, sizeof(float) * 3 * (size_t)w * h);
    s->env = env_from_rgb(c, w, h);
    return s->env != NULL;
}
void rb_set_accel(void *sp){ scene_set_accel(sp, ACCEL_BVH, NULL); }
// after instances moved: the top level made again (scene_update_instances, accel.c:197)
void rb_update_instances(void *sp){ scene_update_instances(sp, NULL); }

// the world's triangles as stored (q, u, v: 9 floats each) and their materials
void rb_tri_data(const void *sp, float *quv, int *mats){
    const Scene *s = sp;
    for (int i = 0; i < s->ntris; i++){
        const Triangle *t = &s->tris[i];
        float *o = quv + 9 * (size_t)i;
        o[0] = t->q.x; o[1] = t->q.y; o[2] = t->q.z;
        o[3] = t->u.x; o[4] = t->u.y; o[5] = t->u.z;
        o[6] = t->v.x; o[7] = t->v.y; o[8] = t->v.z;
        if (mats) mats[i] = t->material;
    }
}
int rb_num_tris(const void *sp){ return ((const Scene *)sp)->ntris; }
int rb_num_prims(const void *sp){ return ((const Scene *)sp)->nprims; }

// triangle_bounds (scene.c:65) of n triangles given as q, u, v (9 floats each): 8 floats per box
// (lo.xyz, 0, hi.xyz, 0), the GPU builder's input layout
// bvh_build_boxes (binned SAH, leaves of up to 4, 16 bins) over n boxes (8 floats each: lo, -, hi,
// -), then bvh_refit_boxes (bvh.c:471) for the moved boxes; out: the refit tree in the GPU node
// layout (8 words: lo, a, hi, b; inner: a / b the children; leaf: a its first ref, b 0x80000000 |
// count), its refs, and the cost the refit returns. Returns the node count (nodes8: 2n - 1 room).
int rb_bvh_refit(const float *boxes, const float *moved, int n, uint32_t *nodes8, uint32_t *refs, float *cost){
    Aabb *a = malloc((size_t)n * sizeof(Aabb)), *m = malloc((size_t)n * sizeof(Aabb));
    for (int i = 0; i < n; i++){
        const float *p = boxes + 8 * (size_t)i, *q = moved + 8 * (size_t)i;
        a[i].lo = v3f(p); a[i].hi = v3f(p + 4);
        m[i].lo = v3f(q); m[i].hi = v3f(q + 4);
    }
    Bvh b;
    memset(&b, 0, sizeof(b));
    bvh_build_boxes(&b, a, n, 4, 16, BVH_SPLIT_SAH);
    *cost = (float)bvh_refit_boxes(&b, m);
    for (int i = 0; i < b.nnodes; i++){
        const BvhNode *d = &b.nodes[i];
        float *f = (float *)(nodes8 + 8 * (size_t)i);
        f[0] = (float)d->box.lo.x; f[1] = (float)d->box.lo.y; f[2] = (float)d->box.lo.z;
        f[4] = (float)d->box.hi.x; f[5] = (float)d->box.hi.y; f[6] = (float)d->box.hi.z;
        nodes8[8 * (size_t)i + 3] = d->count > 0 ? (uint32_t)d->start : (uint32_t)d->left;
        nodes8[8 * (size_t)i + 7] = d->count > 0 ? 0x80000000u | (uint32_t)d->count : (uint32_t)d->right;
    }
    for (int i = 0; i < b.nrefs; i++) refs[i] = (uint32_t)b.refs[i];
    int nn = b.nnodes;
    bvh_free(&b);
    free(a);
    free(m);
    return nn;
}

void rb_triangle_bounds(const float *quv, int n, float *boxes){
    for (int i = 0; i < n; i++){
        const float *p = quv + 9 * (size_t)i;
        Triangle t;
        memset(&t, 0, sizeof(t));
        t.q = v3f(p); t.u = v3f(p + 3); t.v = v3f(p + 6);
        Aabb b = triangle_bounds(&t);
        float *o = boxes + 8 * (size_t)i;
        o[0] = b.lo.x; o[1] = b.lo.y; o[2] = b.lo.z; o[3] = 0;
        o[4] = b.hi.x; o[5] = b.hi.y; o[6] = b.hi.z; o[7] = 0;
    }
}

// ---- queries ----------------------------------------------------------------------------------
// Closest hits of n rays (origins, directions: 3 floats each) in (tmin, tmax): prim = shape id
// (-1: none), inst, t. OpenMP over the rays.
void rb_intersect(const void *sp, const float *orig, const float *dir, long long n, float tmin, float tmax,
                  int *prim, int *inst, float *t){
    const Scene *s = sp;
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long i = 0; i < n; i++){
        Ray r = {v3f(orig + 3 * i), v3f(dir + 3 * i)};
        Hit h;
        if (__real_scene_intersect(s, &r, tmin, tmax, &h)){ prim[i] = h.prim; inst[i] = h.inst; t[i] = (float)h.t; }
        else { prim[i] = -1; inst[i] = -1; t[i] = -1; }
    }
}
void rb_occluded(const void *sp, const float *orig, const float *dir, long long n, float tmin, float tmax, int *out){
    const Scene *s = sp;
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long i = 0; i < n; i++){
        Ray r = {v3f(orig + 3 * i), v3f(dir + 3 * i)};
        out[i] = __real_scene_occluded(s, &r, tmin, tmax);
    }
}

// TraceParams.indirect_clamp of the next rb_trace_image calls (0: off, trace_default_params')
static float g_indirect_clamp = 0;
void rb_set_indirect_clamp(float v){ g_indirect_clamp = v; }

// trace_image over rows [y0, y0 + rows) of a w x h image (rows = h: all of it); rgb: rows * w * 3
// floats (the mean of each pixel's spp samples). cam: from, at, up (9 floats), vfov in degrees.
void rb_trace_image(const void *sp, const float *cam, float vfov, int w, int h, int y0, int rows, int spp,
                    unsigned long long seed, int max_depth, int mis, int sampler, int skip_caustics, float *rgb){
    const Scene *s = sp;
    Camera c = camera_make(v3f(cam), v3f(cam + 3), v3f(cam + 6), vfov, (real)w / (real)h);
    TraceParams tp = trace_default_params();
    tp.max_depth = max_depth;
    tp.mis = mis;
    tp.sampler = sampler;
    tp.skip_caustics = skip_caustics;
    tp.indirect_clamp = g_indirect_clamp;
    Vec3 *px = malloc(sizeof(Vec3) * (size_t)w * h);
    if (!px) return;
    if (rows == h && y0 == 0) trace_image(s, &c, &tp, w, h, spp, seed, 0, px, NULL, NULL);
    else {
        // the same pixels as trace_image's (its per-pixel seeding), for a band of rows
#pragma omp parallel for schedule(dynamic, 1)
        for (int y = y0; y < y0 + rows; y++)
            for (int x = 0; x < w; x++){
                uint64_t pixel = (uint64_t)y * w + x;
                Rng rng;
                rng_seed(&rng, 0x853c49e6748fea9bULL ^ (pixel * 0x9E3779B97F4A7C15ULL) ^ (seed * 0xD1B54A32D192ED03ULL), pixel);
                Vec3 sum = vec3(0, 0, 0);
                for (int k = 0; k < spp; k++){
                    Sampler sm = sampler_make(&rng, x, y, (uint32_t)k, (uint32_t)seed * 0x9e3779b9u, tp.sampler);
                    real jx, jy;
                    sampler_2d(&sm, SAMPLE_CAMERA, &jx, &jy);
                    Vec3 col = trace_path_sampled(s, camera_ray(&c, (x + jx) / w, (y + jy) / h), &sm, &tp);
                    if (!(col.x == col.x && col.y == col.y && col.z == col.z)) continue;
                    sum = v_add(sum, col);
                }
                px[pixel] = v_scale(sum, (real)1 / spp);
            }
    }
    for (int y = y0; y < y0 + rows; y++)
        for (int x = 0; x < w; x++){
            const Vec3 *p = &px[(size_t)y * w + x];
            float *o = rgb + 3 * ((size_t)(y - y0) * w + x);
            o[0] = (float)p->x; o[1] = (float)p->y; o[2] = (float)p->z;
        }
    free(px);
}

// light_trace_caustics of `photons` light paths over a w x h image, added into rgb (w * h * 3
// floats). cam: from, at, up (9 floats), vfov in degrees.
void rb_light_trace_caustics(const void *sp, const float *cam, float vfov, int w, int h, long long photons,
                             int max_depth, unsigned long long seed, float *rgb){
    const Scene *s = sp;
    Camera c = camera_make(v3f(cam), v3f(cam + 3), v3f(cam + 6), vfov, (real)w / (real)h);
    TraceParams tp = trace_default_params();
    tp.max_depth = max_depth;
    Vec3 *px = calloc((size_t)w * h, sizeof(Vec3));
    if (!px) return;
    light_trace_caustics(s, &c, w, h, photons, &tp, seed, px);
    for (size_t i = 0; i < (size_t)w * h; i++){
        rgb[3 * i] += (float)px[i].x; rgb[3 * i + 1] += (float)px[i].y; rgb[3 * i + 2] += (float)px[i].z;
    }
    free(px);
}

// The denoiser's guide (trace.wgsl:1045-1104 without media; gbuf's ray through the pixel centre,
// trace.wgsl:1330-1332): per pixel, through mirrors and glass (refracting unless the glass reflects
// all), the first rough surface's normal and distance (n4: x y z, distance) and the albedo of the
// way with the kind (a4: r g b, kind + 4 (instance + 1); kind 0 a rough surface, 1 a lamp, a bright
// glow or nothing). bsdf_rough_part is tracer.c:258's (static there).
#ifdef LR_DOUBLE
#define RB_EPS 1e-4
#else
#define RB_EPS 2e-3
#endif
void rb_guide(const void *sp, const float *cam, float vfov, int w, int h, float *n4, float *a4){
    const Scene *s = sp;
    Camera c = camera_make(v3f(cam), v3f(cam + 3), v3f(cam + 6), vfov, (real)w / (real)h);
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < w * h; k++){
        const int x = k % w, y = k / w;
        Vec3 pc = v_sub(v_add(c.upper_left, v_scale(c.horizontal, (x + 0.5f) / (real)w)),
                        v_scale(c.vertical, (y + 0.5f) / (real)h));
        Ray ray = {c.origin, v_norm(v_sub(pc, c.origin))};
        Vec3 gn = vec3(0, 0, 0), ga = vec3(1, 1, 1), a = vec3(1, 1, 1);
        real gz = 1e30, dist = 0, kind = 1;
        int ginst = -1;
        for (int i = 0; i < 6; i++){
            Hit hit;
            if (!scene_intersect(s, &ray, RB_EPS, 1e30, &hit)) break;
            const Material *m = &s->mats[hit_material(s, &hit)];
            if (m->type == MAT_LIGHT || v_max(m->emission) >= 1){ gn = hit.n; gz = dist + hit.t; ginst = hit.inst; break; }
            Bsdf b = bsdf_make(m, hit.front_face);
            if (!b.smooth || (1 - b.metallic) * (1 - b.transmission) > 0){
                gn = hit.n; gz = dist + hit.t; ga = v_mul(a, m->albedo); kind = 0; ginst = hit.inst;
                break;
            }
            a = v_mul(a, m->albedo);
            dist += hit.t;
            Vec3 nxt = v_reflect(ray.d, hit.n);
            if (b.transmission > 0.5 && b.metallic < 0.5){
                real cos_i = r_fmin(-v_dot(ray.d, hit.n), 1);
                if (b.eta * b.eta * (1 - cos_i * cos_i) <= 1) nxt = v_refract(ray.d, hit.n, b.eta);
            }
            ray.o = hit.p;
            ray.d = v_norm(nxt);
        }
        float *n = n4 + 4 * (size_t)k, *al = a4 + 4 * (size_t)k;
        n[0] = (float)gn.x; n[1] = (float)gn.y; n[2] = (float)gn.z; n[3] = (float)gz;
        al[0] = (float)ga.x; al[1] = (float)ga.y; al[2] = (float)ga.z;
        al[3] = (float)kind + 4.0f * (float)(ginst >= 0 ? (unsigned)ginst + 1u : 0u);
    }
}

// the BSDF's tables (scene/brdf_tables.h) packed as the GPU backend packs them (brdf_gpu.c:20-25)
void rb_bsdf_tables(float *out){
    memcpy(out, BRDF_E, sizeof(BRDF_E));
    memcpy(out + 1024, BRDF_B, sizeof(BRDF_B));
    memcpy(out + 2048, BRDF_E_AVG, sizeof(BRDF_E_AVG));
    memcpy(out + 2080, BRDF_B_AVG, sizeof(BRDF_B_AVG));
}
// the primitives as upload_world packs them (trace_gpu.c:1145-1154): 24 floats each
void rb_prim_data(const void *sp, float *out){
    const Scene *s = sp;
    for (int i = 0; i < s->nprims; i++){
        const Primitive *p = &s->prims[i];
        float *o = out + 24 * (size_t)i;
        o[0] = p->center.x; o[1] = p->center.y; o[2] = p->center.z; o[3] = p->radius;
        o[4] = p->q.x; o[5] = p->q.y; o[6] = p->q.z; o[7] = p->type == PRIM_QUAD ? 1.0f : 0.0f;
        o[8] = p->u.x; o[9] = p->u.y; o[10] = p->u.z; o[11] = (float)p->material;
        o[12] = p->v.x; o[13] = p->v.y; o[14] = p->v.z; o[15] = p->area;
        o[16] = p->normal.x; o[17] = p->normal.y; o[18] = p->normal.z; o[19] = p->plane_d;
        o[20] = p->w.x; o[21] = p->w.y; o[22] = p->w.z; o[23] = 0;
    }
}
// camera_make (camera.h:21-36): origin, upper_left, horizontal, vertical (12 floats)
void rb_camera(const float *from_at_up, float vfov, float aspect, float *out){
    Camera c = camera_make(v3f(from_at_up), v3f(from_at_up + 3), v3f(from_at_up + 6), vfov, aspect);
    Vec3 v[4] = {c.origin, c.upper_left, c.horizontal, c.vertical};
    for (int k = 0; k < 4; k++){ out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z; }
}

// the sky's sampling tables (env.h: marg h + 1, cond h x (w + 1)) and each pixel's probability
void rb_env_tables(const void *sp, float *marg, float *cond, float *prob){
    const Scene *s = sp;
    const Env *e = s->env;
    memcpy(marg, e->marg, sizeof(float) * (size_t)(e->h + 1));
    memcpy(cond, e->cond, sizeof(float) * (size_t)e->h * (e->w + 1));
    for (int y = 0; y < e->h; y++)
        for (int x = 0; x < e->w; x++) prob[(size_t)y * e->w + x] = (float)env_pixel_prob(e, x, y);
}

// the blue-noise mask (sampler.c): 64 x 64 ranks
void rb_blue_noise(uint16_t *out){ memcpy(out, blue_noise_mask(), sizeof(uint16_t) * BLUE_NOISE_SIZE * BLUE_NOISE_SIZE); }
uint32_t rb_sampler_owen(uint32_t x, uint32_t seed){ return sampler_owen(x, seed); }
uint32_t rb_sampler_sobol1(uint32_t i){ return sampler_sobol1(i); }
uint32_t rb_sampler_hash(uint32_t x){ return sampler_hash(x); }
