// media.cuh - participating media on the device: the reference's voxel-grid volumes
// (engine/scene/volume.h) and their tracking (engine/rt/medium.c), restated with the float
// build's roundings (each operation rounded alone, in the C code's order) so that exact-mode paths
// draw the same random numbers and take the same decisions as the CPU's, up to logf's rounding.
//
//   volume_density     trilinear density at a point, 0 outside the grid (volume.h:64-83)
//   walk_init / next   3D DDA over the majorant bricks, or one segment with the global majorant
//                      when the whole segment's optical depth is below 4 (medium.c:47-126)
//   sample_distance    delta tracking (medium.c:136-151)
//   transmittance      ratio tracking with Russian roulette below 0.1 (medium.c:157-176)
//   scene_*            all media at once: the earliest collision; transmittances multiplied
//                      (medium.c:188-203)
//   phase_hg / sample_phase_u  Henyey-Greenstein (volume.h:89-92; medium.c:205-214)
#pragma once
#include "lrc_internal.cuh"
#include "pt_math.cuh"

namespace lrc {
namespace pt {

constexpr float MEDIUM_DDA_MIN_TAU = 4.0f;
constexpr int VOLUME_BRICK = 8;
constexpr float REAL_MAX_F = 3.402823466e+38f;

__device__ __forceinline__ float volume_density(const VolDev &v, V3 p) {
    const float gx = sub(mul(dvd(sub(p.x, v.lo[0]), sub(v.hi[0], v.lo[0])), (float)v.nx), 0.5f);
    const float gy = sub(mul(dvd(sub(p.y, v.lo[1]), sub(v.hi[1], v.lo[1])), (float)v.ny), 0.5f);
    const float gz = sub(mul(dvd(sub(p.z, v.lo[2]), sub(v.hi[2], v.lo[2])), (float)v.nz), 0.5f);
    if (!(gx > -1.0f && gy > -1.0f && gz > -1.0f && gx < (float)v.nx && gy < (float)v.ny && gz < (float)v.nz)) return 0.0f;
    const int x0 = gx < 0.0f ? -1 : (int)gx, y0 = gy < 0.0f ? -1 : (int)gy, z0 = gz < 0.0f ? -1 : (int)gz;
    const float fx = sub(gx, (float)x0), fy = sub(gy, (float)y0), fz = sub(gz, (float)z0);
    float c[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int x = x0 + (k & 1), y = y0 + ((k >> 1) & 1), z = z0 + (k >> 2);
        const bool inside = x >= 0 && y >= 0 && z >= 0 && x < v.nx && y < v.ny && z < v.nz;
        c[k] = inside ? __ldg(&v.density[((size_t)z * v.ny + y) * v.nx + x]) : 0.0f;
    }
    const float c00 = add(c[0], mul(sub(c[1], c[0]), fx)), c10 = add(c[2], mul(sub(c[3], c[2]), fx));
    const float c01 = add(c[4], mul(sub(c[5], c[4]), fx)), c11 = add(c[6], mul(sub(c[7], c[6]), fx));
    const float c0 = add(c00, mul(sub(c10, c00), fy)), c1 = add(c01, mul(sub(c11, c01), fy));
    return add(c0, mul(sub(c1, c0), fz));
}

__device__ __forceinline__ float phase_hg(float cos_theta, float g) {
    const float d = sub(add(1.0f, mul(g, g)), mul(mul(2.0f, g), cos_theta));
    return dvd(sub(1.0f, mul(g, g)), mul(mul(mul(4.0f, PIF), d), __fsqrt_rn(d)));
}

__device__ __forceinline__ V3 sample_phase_u(V3 d, float g, float xi, float u_phi) {
    float cos_t;
    if (fabsf(g) < 1e-3f) {
        cos_t = sub(1.0f, mul(2.0f, xi));
    } else {
        const float sq = dvd(sub(1.0f, mul(g, g)), sub(add(1.0f, g), mul(mul(2.0f, g), xi)));
        cos_t = dvd(sub(add(1.0f, mul(g, g)), mul(sq, sq)), mul(2.0f, g));
    }
    cos_t = cos_t < -1.0f ? -1.0f : (cos_t > 1.0f ? 1.0f : cos_t);
    const float sin_t = __fsqrt_rn(sub(1.0f, mul(cos_t, cos_t)));
    const float phi = mul(mul(2.0f, PIF), u_phi);
    V3 t, b;
    onb(d, t, b);
    return vadd(vadd(vscale(t, mul(sin_t, cosf(phi))), vscale(b, mul(sin_t, sinf(phi)))), vscale(d, cos_t));
}

// the part [t0, t1] of the ray inside the box, clipped to [tmin, tmax]
__device__ __forceinline__ bool clip_to_box(const float *bl, const float *bh, V3 ro, V3 rd, float tmin, float tmax,
                                            float &t0, float &t1) {
    float lo = tmin, hi = tmax;
    const float o[3] = {ro.x, ro.y, ro.z}, d[3] = {rd.x, rd.y, rd.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (d[a] == 0.0f) {
            if (o[a] < bl[a] || o[a] > bh[a]) return false;
            continue;
        }
        const float inv = dvd(1.0f, d[a]);
        float ta = mul(sub(bl[a], o[a]), inv), tb = mul(sub(bh[a], o[a]), inv);
        if (ta > tb) {
            const float t = ta;
            ta = tb;
            tb = t;
        }
        if (ta > lo) lo = ta;
        if (tb < hi) hi = tb;
        if (lo >= hi) return false;
    }
    t0 = lo;
    t1 = hi;
    return true;
}

struct BrickWalk {
    bool global;
    float t, t1;
    int i[3], step[3], n[3];
    float next[3], delta[3];
};

__device__ __forceinline__ bool walk_init(BrickWalk &w, const VolDev &v, V3 ro, V3 rd, float tmin, float tmax) {
    float t0, t1;
    if (!clip_to_box(v.alo, v.ahi, ro, rd, tmin, tmax, t0, t1)) return false;
    w.t = t0;
    w.t1 = t1;
    w.global = mul(mul(v.sigma_t, v.max_density), sub(t1, t0)) < MEDIUM_DDA_MIN_TAU;
    if (w.global) return true;
    const float o[3] = {ro.x, ro.y, ro.z}, d[3] = {rd.x, rd.y, rd.z};
    const int nvox[3] = {v.nx, v.ny, v.nz};
    w.n[0] = v.bnx;
    w.n[1] = v.bny;
    w.n[2] = v.bnz;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float bs = mul(dvd(sub(v.hi[a], v.lo[a]), (float)nvox[a]), (float)VOLUME_BRICK);
        const float p = add(o[a], mul(d[a], t0));
        int i = (int)floorf(dvd(sub(p, v.lo[a]), bs));
        if (i < 0) i = 0;
        if (i > w.n[a] - 1) i = w.n[a] - 1;
        w.i[a] = i;
        if (d[a] > 0.0f) {
            w.step[a] = 1;
            w.next[a] = dvd(sub(add(v.lo[a], mul((float)(i + 1), bs)), o[a]), d[a]);
            w.delta[a] = dvd(bs, d[a]);
        } else if (d[a] < 0.0f) {
            w.step[a] = -1;
            w.next[a] = dvd(sub(add(v.lo[a], mul((float)i, bs)), o[a]), d[a]);
            w.delta[a] = dvd(-bs, d[a]);
        } else {
            w.step[a] = 0;
            w.next[a] = REAL_MAX_F;
            w.delta[a] = REAL_MAX_F;
        }
    }
    return true;
}

// the next segment [ta, tb] and the extinction majorant over it; false: done
__device__ __forceinline__ bool walk_next(BrickWalk &w, const VolDev &v, float &ta, float &tb, float &smax) {
    if (w.t >= w.t1) return false;
    if (w.global) {
        ta = w.t;
        tb = w.t1;
        smax = mul(v.sigma_t, v.max_density);
        w.t = w.t1;
        return true;
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
        if (w.i[a] < 0 || w.i[a] >= w.n[a]) return false;
    const int ax = w.next[0] < w.next[1] ? (w.next[0] < w.next[2] ? 0 : 2) : (w.next[1] < w.next[2] ? 1 : 2);
    float end = w.next[ax] < w.t1 ? w.next[ax] : w.t1;
    if (end < w.t) end = w.t;
    ta = w.t;
    tb = end;
    smax = mul(v.sigma_t, __ldg(&v.brick_max[((size_t)w.i[2] * v.bny + w.i[1]) * v.bnx + w.i[0]]));
    w.t = end;
    w.i[ax] += w.step[ax];
    w.next[ax] = add(w.next[ax], w.delta[ax]);
    return true;
}

// tentative collisions one tracking call may take (far beyond what finite inputs need: the
// expected count is the segment's majorant optical depth); past it the call stops, flags
// ST_MEDIUM and counts as no collision / full transmittance
constexpr uint32_t MEDIUM_MAX_STEPS = 1u << 20;

// The ray's position at t (v_add(o, v_scale(d, t)))
__device__ __forceinline__ V3 at(V3 o, V3 d, float t) { return vadd(o, vscale(d, t)); }

// delta tracking: true and the distance of a real collision before tmax
__device__ __forceinline__ bool medium_sample_distance(const VolDev &v, V3 ro, V3 rd, float tmin, float tmax, Rng &rng,
                                                       float &t_hit, uint32_t *err) {
    if (v.max_density <= 0.0f || v.sigma_t <= 0.0f) return false;
    BrickWalk w;
    if (!walk_init(w, v, ro, rd, tmin, tmax)) return false;
    float ta, tb, smax;
    uint32_t steps = 0;
    while (walk_next(w, v, ta, tb, smax)) {
        if (smax <= 0.0f) continue;
        float t = ta;
        for (;;) {
            if (++steps > MEDIUM_MAX_STEPS) {
                atomicOr(err, ST_MEDIUM);
                return false;
            }
            t = sub(t, dvd(logf(sub(1.0f, rng_real(rng))), smax));
            if (t >= tb) break;
            const float s = mul(v.sigma_t, volume_density(v, at(ro, rd, t)));
            if (mul(rng_real(rng), smax) < s) {
                t_hit = t;
                return true;
            }
        }
    }
    return false;
}

// ratio tracking: the fraction of light that crosses [tmin, tmax]
__device__ __forceinline__ float medium_transmittance(const VolDev &v, V3 ro, V3 rd, float tmin, float tmax, Rng &rng,
                                                     uint32_t *err) {
    if (v.max_density <= 0.0f || v.sigma_t <= 0.0f) return 1.0f;
    BrickWalk w;
    if (!walk_init(w, v, ro, rd, tmin, tmax)) return 1.0f;
    float tr = 1.0f, ta, tb, smax;
    uint32_t steps = 0;
    while (walk_next(w, v, ta, tb, smax)) {
        if (smax <= 0.0f) continue;
        float t = ta;
        for (;;) {
            if (++steps > MEDIUM_MAX_STEPS) {
                atomicOr(err, ST_MEDIUM);
                return tr;
            }
            t = sub(t, dvd(logf(sub(1.0f, rng_real(rng))), smax));
            if (t >= tb) break;
            float s = mul(v.sigma_t, volume_density(v, at(ro, rd, t)));
            if (s > smax) s = smax;
            tr = mul(tr, sub(1.0f, dvd(s, smax)));
            if (tr < 0.1f) {
                if (rng_real(rng) < 0.5f) return 0.0f;
                tr = mul(tr, 2.0f);
            }
        }
    }
    return tr;
}

// The two scene-level calls are compiled once per file (not inlined): the path tracer calls them
// from five places, and inlined copies of the tracking loops overflowed the instruction cache.
// every medium tracked up to the best collision so far: the earliest one and its medium
static __device__ __noinline__ bool scene_medium_collision(const VolDev *vols, uint32_t nvol, V3 ro, V3 rd, float tmin,
                                                           float tmax, Rng &rng, float &t, int &which, uint32_t *err) {
    int w = -1;
    float best = tmax;
    for (uint32_t i = 0; i < nvol; i++) {
        float ti;
        if (medium_sample_distance(vols[i], ro, rd, tmin, best, rng, ti, err)) {
            best = ti;
            w = (int)i;
        }
    }
    if (w < 0) return false;
    t = best;
    which = w;
    return true;
}

static __device__ __noinline__ float scene_medium_transmittance(const VolDev *vols, uint32_t nvol, V3 ro, V3 rd, float tmin,
                                                               float tmax, Rng &rng, uint32_t *err) {
    float tr = 1.0f;
    for (uint32_t i = 0; i < nvol && tr > 0.0f; i++) tr = mul(tr, medium_transmittance(vols[i], ro, rd, tmin, tmax, rng, err));
    return tr;
}

}  // namespace pt
}  // namespace lrc
