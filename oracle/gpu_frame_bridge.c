// gpu_frame_bridge.c - test infrastructure only: the reference engine's offline GPU entry point
// (engine/app/gpu_frame.c: gpu_frame_open, gpu_frame_trace, gpu_frame_close) run, unmodified,
// through the CUDA backend (little_renderer_b200/shim/gpu_cuda.c, which implements the engine's
// gpu.h / view_gpu.h on liblrc), on a Scene made by ref_bridge.c; and the scene's own tree
// (scene_bvh) in the layout the reference's GPU path tracer reads (put_nodes,
// engine/gpu/trace_gpu.c:883-896), for the tests to give lrc_scene_set_tree the same tree.
#include "app/gpu_frame.h"
#include "rt/accel.h"
#include "rt/bvh.h"
#include "scene/camera.h"

#include <stdint.h>
#include <string.h>

// gpu_frame_trace of a w x h image at spp samples (depth max_depth, NEE + MIS as mis, sampler 1:
// Owen-Sobol + blue noise) from the camera at from_at_up (9 floats) with vfov degrees; rgb: w x h x 3
// floats, the mean of each pixel's samples as gpu_frame_trace leaves them. Returns its status
// (0 done), or -1 when gpu_frame_open found no GPU.
int rb_gpu_frame_trace(void *sp, const float *from_at_up, float vfov, int w, int h, int spp, int max_depth, int mis,
                       int sampler, float *rgb){
    Scene *s = sp;
    Gpu *g = NULL;
    GpuView *v = NULL;
    if (gpu_frame_open(w, h, &g, &v)) return -1;
    Vec3 from = {from_at_up[0], from_at_up[1], from_at_up[2]};
    Vec3 at = {from_at_up[3], from_at_up[4], from_at_up[5]};
    Vec3 up = {from_at_up[6], from_at_up[7], from_at_up[8]};
    Camera cam = camera_make(from, at, up, vfov, (real)w / (real)h);
    Image img = image_create(w, h);
    int rc = 1;
    if (img.px){
        rc = gpu_frame_trace(g, v, s, &cam, NULL, NULL, spp, max_depth, mis, 0, sampler, 0, &img, 0);
        for (int i = 0; i < w * h; i++){
            rgb[3 * i] = (float)img.px[i].x;
            rgb[3 * i + 1] = (float)img.px[i].y;
            rgb[3 * i + 2] = (float)img.px[i].z;
        }
        image_free(&img);
    }
    gpu_frame_close(g, v);
    return rc;
}

// the scene's own tree (scene_set_accel made it): its node and ref counts; with nodes and refs
// given, the nodes in put_nodes' layout (8 words each, root at 0, refs from 0) and the refs
static int put(uint32_t *o, real x){ float f = (float)x; memcpy(o, &f, 4); return 0; }

int rb_scene_tree(const void *sp, uint32_t *nodes, uint32_t *refs, int *nnodes, int *nrefs){
    const Bvh *b = scene_bvh(sp);
    if (!b) return 0;
    *nnodes = b->nnodes;
    *nrefs = b->nrefs;
    if (!nodes || !refs) return 1;
    for (int i = 0; i < b->nnodes; i++){
        const BvhNode *n = &b->nodes[i];
        uint32_t *o = nodes + 8 * (size_t)i;
        put(o, n->box.lo.x); put(o + 1, n->box.lo.y); put(o + 2, n->box.lo.z);
        put(o + 4, n->box.hi.x); put(o + 5, n->box.hi.y); put(o + 6, n->box.hi.z);
        o[3] = n->count > 0 ? (uint32_t)n->start : (uint32_t)n->left;
        o[7] = n->count > 0 ? (0x80000000u | (uint32_t)n->count) : (uint32_t)n->right;
    }
    for (int i = 0; i < b->nrefs; i++) refs[i] = (uint32_t)b->refs[i];
    return 1;
}
