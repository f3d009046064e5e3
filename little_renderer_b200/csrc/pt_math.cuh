// pt_math.cuh - the path tracer's arithmetic: the reference's float build (engine/base/lrmath.h,
// -fsingle-precision-constant, no fused multiply-add) restated on the device. Every sum, product
// and quotient is rounded on its own (__fadd_rn, __fmul_rn, __fdiv_rn) in the C code's order, so a
// path's decisions follow the CPU's bit for bit up to the transcendental functions (sinf, cosf,
// tanf, acosf, powf: CUDA's, a few ulp from the C library's). sqrtf is correctly rounded in both.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lrc {
namespace pt {

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return v3(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return v3(sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)); }
__device__ __forceinline__ V3 vmul(V3 a, V3 b) { return v3(mul(a.x, b.x), mul(a.y, b.y), mul(a.z, b.z)); }
__device__ __forceinline__ V3 vscale(V3 a, float s) { return v3(mul(a.x, s), mul(a.y, s), mul(a.z, s)); }
__device__ __forceinline__ V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
// v_dot: a.x*b.x + a.y*b.y + a.z*b.z, left to right
__device__ __forceinline__ float vdot(V3 a, V3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    return v3(sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x)));
}
__device__ __forceinline__ float vlen(V3 a) { return __fsqrt_rn(vdot(a, a)); }
// v_norm: l > 0 ? a * (1 / l) : a
__device__ __forceinline__ V3 vnorm(V3 a) {
    float l = vlen(a);
    return l > 0.0f ? vscale(a, dvd(1.0f, l)) : a;
}
// r_fmin / r_fmax: the other number when b is a NaN
__device__ __forceinline__ float rmin(float a, float b) { return b != b ? a : (a < b ? a : b); }
__device__ __forceinline__ float rmax(float a, float b) { return b != b ? a : (a > b ? a : b); }
__device__ __forceinline__ float vmax3(V3 a) { return rmax(a.x, rmax(a.y, a.z)); }
// v_reflect: d - n * (2 * dot(d, n))
__device__ __forceinline__ V3 vreflect(V3 d, V3 n) { return vsub(d, vscale(n, mul(2.0f, vdot(d, n)))); }
// v_refract (lrmath.h)
__device__ __forceinline__ V3 vrefract(V3 d, V3 n, float eta) {
    float cos_i = rmin(vdot(vneg(d), n), 1.0f);
    V3 perp = vscale(vadd(d, vscale(n, cos_i)), eta);
    V3 para = vscale(n, -__fsqrt_rn(fabsf(sub(1.0f, vdot(perp, perp)))));
    return vadd(perp, para);
}
__device__ __forceinline__ float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

constexpr float PIF = 3.14159265358979323846f;   // PI in the float build

// onb_from_normal (rng.h, Duff et al. 2017)
__device__ __forceinline__ void onb(V3 n, V3 &t, V3 &b) {
    float s = copysignf(1.0f, n.z);
    float a = dvd(-1.0f, add(s, n.z));
    float c = mul(mul(n.x, n.y), a);
    t = v3(add(1.0f, mul(mul(mul(s, n.x), n.x), a)), mul(s, c), -mul(s, n.x));
    b = v3(c, add(s, mul(mul(n.y, n.y), a)), -n.y);
}

// sample_cosine_hemisphere_u (rng.h)
__device__ __forceinline__ V3 cosine_hemisphere(V3 n, float u1, float u2) {
    float phi = mul(mul(2.0f, PIF), u1);
    float rad = __fsqrt_rn(u2);
    float x = mul(rad, cosf(phi)), y = mul(rad, sinf(phi)), z = __fsqrt_rn(rmax(0.0f, sub(1.0f, u2)));
    V3 t, b;
    onb(n, t, b);
    return vadd(vadd(vscale(t, x), vscale(b, y)), vscale(n, z));
}

// ---- random numbers: PCG32 (rng.h), 64-bit state as the CPU's ---------------------------------
struct Rng {
    uint64_t state, inc;
};
__device__ __forceinline__ uint32_t rng_u32(Rng &r) {
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ull + r.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
__device__ __forceinline__ void rng_seed(Rng &r, uint64_t seed, uint64_t stream) {
    r.state = 0;
    r.inc = (stream << 1u) | 1u;
    rng_u32(r);
    r.state += seed;
    rng_u32(r);
}
// rng_real, float build: 24 random bits
__device__ __forceinline__ float rng_real(Rng &r) { return mul((float)(rng_u32(r) >> 8), 1.0f / 16777216.0f); }

// ---- the sampler (engine/base/sampler.c): Owen-scrambled Sobol pairs with blue-noise shifts ----
constexpr int SAMPLER_PAIRS = 13;
__device__ __forceinline__ int SAMPLE_LIGHT(int depth) { return 1 + 3 * depth; }
__device__ __forceinline__ int SAMPLE_DIR(int depth) { return 2 + 3 * depth; }
__device__ __forceinline__ int SAMPLE_MISC(int depth) { return 3 + 3 * depth; }

__device__ __forceinline__ uint32_t s_hash(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t owen_rev(uint32_t x, uint32_t seed) {
    x ^= x * 0x3d20adeau;
    x += seed;
    x *= (seed >> 16) | 1u;
    x ^= x * 0x05526c56u;
    x ^= x * 0x53a22864u;
    return __brev(x);
}
__device__ __forceinline__ uint32_t s_owen(uint32_t x, uint32_t seed) { return owen_rev(__brev(x), seed); }
__device__ __forceinline__ uint32_t sobol1_rev(uint32_t i) {
    i ^= (i >> 1) & 0x55555555u;
    i ^= (i >> 2) & 0x33333333u;
    i ^= (i >> 4) & 0x0f0f0f0fu;
    i ^= (i >> 8) & 0x00ff00ffu;
    i ^= i >> 16;
    return i;
}
__device__ __forceinline__ float unit24(uint32_t v) { return mul((float)(v >> 8), 1.0f / 16777216.0f); }
__device__ __forceinline__ float wrap01(float t) { return t >= 1.0f ? sub(t, 1.0f) : t; }

struct Sampler {
    Rng *rng;
    uint32_t index, seed;
    int x, y, on;
    const uint16_t *mask;    // 64 x 64 blue-noise ranks
};
__device__ __forceinline__ float bn_value(const uint16_t *m, int x, int y) {
    return mul(add((float)__ldg(&m[(y & 63) * 64 + (x & 63)]), 0.5f), 1.0f / 4096.0f);
}
__device__ __forceinline__ void sampler_2d(Sampler &s, int dim, float &a, float &b) {
    if (!s.on || dim >= SAMPLER_PAIRS) {
        a = rng_real(*s.rng);
        b = rng_real(*s.rng);
        return;
    }
    uint32_t tile = s_hash(((uint32_t)(s.x >> 6) * 73856093u) ^ ((uint32_t)(s.y >> 6) * 19349663u));
    uint32_t seed = s_hash(s.seed ^ s_hash(((uint32_t)dim * 0x9e3779b9u) ^ tile));
    uint32_t i = s_owen(s.index, seed);
    uint32_t xa = owen_rev(i, s_hash(seed ^ 0xa511e9b3u));
    uint32_t xb = owen_rev(sobol1_rev(i), s_hash(seed ^ 0x63d83595u));
    int ox = s.x + 23 * dim, oy = s.y + 41 * dim;
    a = wrap01(add(unit24(xa), bn_value(s.mask, ox, oy)));
    b = wrap01(add(unit24(xb), bn_value(s.mask, ox + 32, oy + 17)));
}
__device__ __forceinline__ float sampler_1d(Sampler &s, int dim, int comp) {
    if (!s.on || dim >= SAMPLER_PAIRS) return rng_real(*s.rng);
    float a, b;
    sampler_2d(s, dim, a, b);
    return comp ? b : a;
}

}  // namespace pt
}  // namespace lrc
