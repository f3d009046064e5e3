// denoise.cu - the path tracer's denoiser on sm_100a: the guide pass (`guide` / `gbuf`,
// engine/gpu/shaders/trace/trace.wgsl:1045-1104, 1319-1337) and the edge-avoiding a-trous filter
// steered by each pixel's variance (engine/gpu/denoise_gpu.c; denoise.wgsl `prep`, `atrous`:
// Dammertz et al. 2010 with SVGF's variance, Schied et al. 2017, without its temporal part).
//
// Planes (w x h float4 each, one array): 0 the samples' sum and count (lrc_trace's accum),
// 1 the moments of each sample's luminance over the guide's albedo (sum l, sum l^2; lrc_trace
// with LRC_TRACE_GUIDED adds them), 2 the guide's normal and distance, 3 its albedo and kind
// (0 a rough surface, 1 a lamp / the sky / nothing, 2 a medium; + 4 (instance + 1)).
//
// The filter's passes pass the image packed, as the reference's do: 8 bytes per pixel
// (irradiance and variance as four halves). The guide's normal goes through the reference's
// octahedral snorm16 code once, in prep, and the passes read it decoded (16 bytes: the normal and
// the distance, whose sign gives the kind): the taps are L1 / L2 hits at these image sizes and
// the passes are bound by instructions, not bytes, so decoding once beats reading half as much.
// Blocks are 32 x 8 pixel tiles so that a tile's taps share cache lines.

#include "pt_device.cuh"
#include <cuda_fp16.h>
#include <algorithm>

namespace lrc {
namespace dn {

using pt::V3;
using pt::v3;

// lowbias32 (util.wgsl hash32)
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
// Rec. 709 luminance (util.wgsl luma)
__device__ __forceinline__ float luma(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }
__device__ __forceinline__ float gkind(float w) { return w - 4.0f * floorf(w * 0.25f); }

// an image value: irradiance (each channel at most 6e4) and variance (< 0: no sample) as halves
__device__ __forceinline__ uint32_t half2_bits(float a, float b) {
    return (uint32_t)__half_as_ushort(__float2half_rn(a)) | ((uint32_t)__half_as_ushort(__float2half_rn(b)) << 16);
}
__device__ __forceinline__ uint2 put_iv(float r, float g, float b, float v) {
    return make_uint2(half2_bits(fminf(r, 6e4f), fminf(g, 6e4f)), half2_bits(fminf(b, 6e4f), fminf(fmaxf(v, -1.0f), 6e4f)));
}
__device__ __forceinline__ float4 get_iv(uint2 p) {
    return make_float4(__half2float(__ushort_as_half((unsigned short)(p.x & 0xffff))),
                       __half2float(__ushort_as_half((unsigned short)(p.x >> 16))),
                       __half2float(__ushort_as_half((unsigned short)(p.y & 0xffff))),
                       __half2float(__ushort_as_half((unsigned short)(p.y >> 16))));
}

// the normal on an octahedron, two snorm16
__device__ __forceinline__ uint32_t snorm16x2(float a, float b) {
    int ia = __float2int_rn(fminf(fmaxf(a, -1.0f), 1.0f) * 32767.0f);
    int ib = __float2int_rn(fminf(fmaxf(b, -1.0f), 1.0f) * 32767.0f);
    return (uint32_t)(ia & 0xffff) | ((uint32_t)(ib & 0xffff) << 16);
}
__device__ __forceinline__ float2 unsnorm16x2(uint32_t p) {
    float a = (float)(int16_t)(p & 0xffff), b = (float)(int16_t)(p >> 16);
    return make_float2(fmaxf(a / 32767.0f, -1.0f), fmaxf(b / 32767.0f, -1.0f));
}
__device__ __forceinline__ uint32_t oct(float nx, float ny, float nz) {
    const float s = fmaxf(fabsf(nx) + fabsf(ny) + fabsf(nz), 1e-6f);
    float px = nx / s, py = ny / s;
    if (nz < 0.0f) {
        const float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
        const float qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
        px = qx;
        py = qy;
    }
    return snorm16x2(px, py);
}
__device__ __forceinline__ V3 unoct(float2 e) {
    float x = e.x, y = e.y, z = 1.0f - fabsf(e.x) - fabsf(e.y);
    const float t = fmaxf(-z, 0.0f);
    x += x >= 0.0f ? -t : t;
    y += y >= 0.0f ? -t : t;
    const float l = sqrtf(x * x + y * y + z * z);
    return v3(x / l, y / l, z / l);
}
struct G {
    V3 n;
    float z;
    int kind;
};
// The guide as the passes read it: the normal as its octahedral code decodes (unoct(oct(n)), the
// values the reference's packed guide gives), decoded once by prep instead of at every tap; w the
// distance with the kind in its sign (kind 0: z, kind 2: -(z + 1), kind 1: -2e38)
__device__ __forceinline__ G get_g(float4 p) {
    G g;
    const float e = p.w;
    g.kind = e >= 0.0f ? 0 : (e < -1e37f ? 1 : 2);
    g.z = e >= 0.0f ? e : -e - 1.0f;
    g.n = v3(p.x, p.y, p.z);
    return g;
}

// the mean of a pixel's samples over its guide's albedo (a surface), or the mean
__device__ __forceinline__ V3 irradiance(const float4 *__restrict__ px, size_t N, size_t k) {
    const float4 a = px[k], g = px[3 * N + k];
    const float c = fmaxf(a.w, 1.0f);
    V3 m = v3(a.x / c, a.y / c, a.z / c);
    if (gkind(g.w) == 0.0f) m = v3(m.x / fmaxf(g.x, 1e-3f), m.y / fmaxf(g.y, 1e-3f), m.z / fmaxf(g.z, 1e-3f));
    return m;
}

// prep: the packed guide, and each pixel's irradiance with the variance of its mean (its own
// moments from 4 samples on, else the spread of its 7 x 7 neighbours on the same surface)
__global__ void __launch_bounds__(256) prep_kernel(const float4 *__restrict__ px, int W, int H, uint2 *__restrict__ dst,
                                                   float4 *__restrict__ gd) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= W || y >= H) return;
    const size_t N = (size_t)W * H, k = (size_t)y * W + x;
    const float4 a = px[k], g = px[3 * N + k], n = px[2 * N + k];
    const float gk = gkind(g.w);
    const float e = gk == 0.0f ? n.w : (gk == 1.0f ? -2e38f : -(n.w + 1.0f));
    const V3 nd = unoct(unsnorm16x2(oct(n.x, n.y, n.z)));
    gd[k] = make_float4(nd.x, nd.y, nd.z, e);
    if (a.w == 0.0f) {
        dst[k] = put_iv(0.0f, 0.0f, 0.0f, -1.0f);
        return;
    }
    const V3 irr = irradiance(px, N, k);
    if (gk == 1.0f) {
        dst[k] = put_iv(irr.x, irr.y, irr.z, 0.0f);
        return;
    }
    float v;
    if (a.w >= 4.0f) {
        const float4 m = px[N + k];
        const float el = m.x / a.w;
        v = fmaxf(m.y / a.w - el * el, 0.0f) / a.w;
    } else {
        float s1 = 0.0f, s2 = 0.0f, c = 0.0f;
        for (int dy = -3; dy <= 3; dy++)
            for (int dx = -3; dx <= 3; dx++) {
                const int qx = x + dx, qy = y + dy;
                if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
                const size_t q = (size_t)qy * W + qx;
                if (px[q].w == 0.0f || gkind(px[3 * N + q].w) != gk) continue;
                if (gk == 0.0f) {
                    const float4 nq = px[2 * N + q];
                    if (nq.x * n.x + nq.y * n.y + nq.z * n.z < 0.9f) continue;
                }
                const V3 iq = irradiance(px, N, q);
                const float l = luma(iq.x, iq.y, iq.z);
                s1 += l;
                s2 += l * l;
                c += 1.0f;
            }
        const float el = s1 / c;
        v = fmaxf(s2 / c - el * el, 0.0f);
    }
    dst[k] = put_iv(irr.x, irr.y, irr.z, v);
}

// the B3 spline's weights 1/16, 1/4, 3/8, 1/4, 1/16
__device__ __forceinline__ float b3(int i) { return i == 2 ? 0.375f : (i == 1 || i == 3 ? 0.25f : 0.0625f); }

// One a-trous pass: a 5 x 5 B3 spline with holes `step` apart, each tap jittered within its hole
// (but the centre), weighted by luminance (against the noise of the noisier of the two), normal
// (cos^128) and distance (against how fast it changes here); the variance filtered with the
// squared weights. The last pass writes the image (times the albedo on surfaces).
__global__ void __launch_bounds__(256) atrous_kernel(const float4 *__restrict__ px, int W, int H, int step, int last,
                                                     float sigma_l, float sigma_z, const uint2 *__restrict__ src,
                                                     uint2 *__restrict__ dst, const float4 *__restrict__ gd,
                                                     float4 *__restrict__ outp) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= W || y >= H) return;
    const uint32_t N = (uint32_t)W * (uint32_t)H, k = (uint32_t)y * W + x;
    const float4 c = get_iv(src[k]);
    const G gp = get_g(gd[k]);
    if (c.w < 0.0f || gp.kind == 1) {                // no sample yet; a lamp, the sky: as they are
        if (last) outp[k] = c.w < 0.0f ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : make_float4(c.x, c.y, c.z, 1.0f);
        else dst[k] = src[k];
        return;
    }
    // the variance blurred 3 x 3
    float v = 0.0f, vw = 0.0f;
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
            const int qx = min(max(x + dx, 0), W - 1), qy = min(max(y + dy, 0), H - 1);
            const float4 s = get_iv(src[(uint32_t)qy * W + qx]);
            if (s.w < 0.0f) continue;
            const float w = (dx != 0 ? 0.25f : 0.5f) * (dy != 0 ? 0.25f : 0.5f);
            v += w * s.w;
            vw += w;
        }
    v /= fmaxf(vw, 1e-6f);
    const float lp = luma(c.x, c.y, c.z);
    const bool surface = gp.kind == 0;
    // how fast the distance changes per pixel here (the smaller side)
    float gx = 0.0f, gy = 0.0f;
    if (surface) {
        const float l = get_g(gd[(uint32_t)y * W + max(x - 1, 0)]).z, r = get_g(gd[(uint32_t)y * W + min(x + 1, W - 1)]).z;
        const float d = get_g(gd[(uint32_t)max(y - 1, 0) * W + x]).z, u = get_g(gd[(uint32_t)min(y + 1, H - 1) * W + x]).z;
        gx = fminf(fabsf(gp.z - l), fabsf(gp.z - r));
        gy = fminf(fabsf(gp.z - d), fabsf(gp.z - u));
    }
    uint32_t seed = hash32((k * 0x9e3779b9u) ^ ((uint32_t)step * 0x85ebca6bu));
    const int jit = step / 2;
    const uint32_t jn = (uint32_t)(2 * jit + 1);
    float sr = 0.0f, sg = 0.0f, sb = 0.0f, vsum = 0.0f, wsum = 0.0f;
#pragma unroll 1
    for (int j = 0; j < 5; j++) {
#pragma unroll
        for (int i = 0; i < 5; i++) {
            int ox = (i - 2) * step, oy = (j - 2) * step;
            if (jit > 0 && (i != 2 || j != 2)) {
                seed = hash32(seed);
                ox += (int)(((seed & 0xffffu) * jn) >> 16) - jit;
                oy += (int)(((seed >> 16) * jn) >> 16) - jit;
            }
            const int qx = x + ox, qy = y + oy;
            if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
            const uint32_t q = (uint32_t)qy * W + qx;
            const float4 s = get_iv(src[q]);
            float w = b3(i) * b3(j);
            if (q != k) {
                const G gq = get_g(gd[q]);
                if (s.w < 0.0f || gq.kind != gp.kind) continue;
                w *= __expf(__fdividef(-fabsf(lp - luma(s.x, s.y, s.z)), sigma_l * sqrtf(fmaxf(v, s.w)) + 1e-6f));
                if (surface) {
                    float wn = fmaxf(gp.n.x * gq.n.x + gp.n.y * gq.n.y + gp.n.z * gq.n.z, 0.0f);
#pragma unroll
                    for (int e = 0; e < 7; e++) wn *= wn;   // cos^128
                    w *= wn;
                    const float expect = gx * fabsf((float)ox) + gy * fabsf((float)oy);
                    w *= __expf(__fdividef(-fabsf(gp.z - gq.z), sigma_z * expect + 1e-3f * gp.z + 1e-6f));
                }
            }
            sr += w * s.x;
            sg += w * s.y;
            sb += w * s.z;
            vsum += w * w * s.w;
            wsum += w;
        }
    }
    const float o0 = sr / wsum, o1 = sg / wsum, o2 = sb / wsum;
    if (last) {
        const float4 al = px[3 * (size_t)N + k];
        outp[k] = surface ? make_float4(o0 * al.x, o1 * al.y, o2 * al.z, 1.0f) : make_float4(o0, o1, o2, 1.0f);
    } else {
        dst[k] = put_iv(o0, o1, o2, vsum / (wsum * wsum));
    }
}

// ---- the guide: the ray through the pixel's centre to the first rough surface, through mirrors
// and glass (refracting unless the glass reflects all), with the albedo of the whole way ------
__global__ void __launch_bounds__(128) guide_kernel(PtScene S, PtParams P, float4 *__restrict__ planes,
                                                    uint32_t *err) {
    using namespace pt;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)P.W * P.H;
    if (idx >= N) return;
    const uint32_t x = idx % P.W, y = idx / P.W;
    const V3 pc = vsub(vadd(P.upper_left, vscale(P.horizontal, (x + 0.5f) / (float)P.W)),
                       vscale(P.vertical, (y + 0.5f) / (float)P.H));
    V3 ro = P.origin, rd = vnorm(vsub(pc, P.origin));
    V3 gn = v3(0, 0, 0), ga = v3(1, 1, 1), a = v3(1, 1, 1);
    float gz = 1e30f, dist = 0.0f, kind = 1.0f;
    int ginst = -1;
    for (int i = 0; i < 6; i++) {
        Hit h;
        if (!scene_intersect(S, ro, rd, RT_EPS, 1e30f, h, err)) break;
        Mat m = load_mat(S.mats, hit_material(S, h) & 63);
        if (textured(m)) m = hit_shading(S, h, ro, rd, vneg(rd), m);   // (shade_tex)
        // a lamp, or a surface glowing at least as bright as white paper under a light of 1
        if (m.type == MAT_LIGHT || fmaxf(m.emission.x, fmaxf(m.emission.y, m.emission.z)) >= 1.0f) {
            gn = h.n;
            gz = dist + h.t;
            ginst = h.inst;
            break;
        }
        Bsdf b = bsdf_make(m, h.front, S.tab);
        if (bsdf_rough_part(b)) {                    // a surface the light scatters on
            gn = h.n;
            gz = dist + h.t;
            ga = v3(a.x * m.albedo.x, a.y * m.albedo.y, a.z * m.albedo.z);
            kind = 0.0f;
            ginst = h.inst;
            break;
        }
        a = v3(a.x * m.albedo.x, a.y * m.albedo.y, a.z * m.albedo.z);
        dist += h.t;
        V3 nxt = vreflect(rd, h.n);
        if (b.transmission > 0.5f && b.metallic < 0.5f) {
            const float cos_i = fminf(-vdot(rd, h.n), 1.0f);
            if (b.eta * b.eta * (1.0f - cos_i * cos_i) <= 1.0f) nxt = vrefract(rd, h.n, b.eta);
        }
        ro = h.p;
        rd = vnorm(nxt);
    }
    const float w = kind + 4.0f * (float)(ginst >= 0 ? ((uint32_t)ginst & 0x3fffffu) + 1u : 0u);
    planes[2 * N + idx] = make_float4(gn.x, gn.y, gn.z, gz);
    planes[3 * N + idx] = make_float4(ga.x, ga.y, ga.z, w);
}

// ---- reprojection (trace_reproject.wgsl `main` without temporal gradients): a new image's
// samples from the previous image's, where each pixel still sees the same surface ---------------
struct RpCam {
    float3 o, ul, h, v;
};
__device__ __forceinline__ float3 f3(pt::V3 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sc3(float3 a, float k) { return make_float3(a.x * k, a.y * k, a.z * k); }

// where new pixel k's surface was in the old image (pixel centres at integers; z its distance
// from the old eye, w 1 if in front of it)
__device__ __forceinline__ float4 old_place(const RpCam &oc, const RpCam &nc, int W, int H, uint32_t k, float4 g2) {
    const float x = (float)(k % (uint32_t)W), y = (float)(k / (uint32_t)W);
    float3 d = sub3(sub3(add3(nc.ul, sc3(nc.h, (x + 0.5f) / (float)W)), sc3(nc.v, (y + 0.5f) / (float)H)), nc.o);
    d = sc3(d, rsqrtf(dot3(d, d)));
    const bool far = g2.w > 1e29f;
    const float3 p = add3(nc.o, sc3(d, far ? 1e6f : g2.w));
    const float3 f = sub3(oc.ul, oc.o);
    const float3 c = sub3(add3(f, sc3(oc.h, 0.5f)), sc3(oc.v, 0.5f));
    const float3 q0 = sub3(p, oc.o);
    const float den = dot3(q0, c);
    if (den <= 0.0f) return make_float4(0, 0, 0, 0);
    const float3 q = sub3(sc3(q0, dot3(c, c) / den), f);
    const float fx = dot3(q, oc.h) / dot3(oc.h, oc.h) * (float)W - 0.5f;
    const float fy = -dot3(q, oc.v) / dot3(oc.v, oc.v) * (float)H - 0.5f;
    return make_float4(fx, fy, sqrtf(dot3(q0, q0)), 1.0f);
}

// old pixel o saw what the new one sees: samples, the same kind and object, the distance within
// 2 % (25 % in a medium) plus how fast it changes there, the normal within ~25 degrees
__device__ __forceinline__ bool same_surface(const float4 *__restrict__ old, int W, int H, uint32_t o, float4 g2, float4 g3,
                                             float dist, bool edit) {
    const size_t N = (size_t)W * H;
    if (old[o].w == 0.0f) return false;
    const float4 o3 = old[3 * N + o];
    if (o3.w != g3.w) return false;
    const float gk = gkind(g3.w);
    const float4 o2 = old[2 * N + o];
    if (g2.w <= 1e29f) {
        const uint32_t ux = o % (uint32_t)W, uy = o / (uint32_t)W;
        const float zl = old[2 * N + o - (ux > 0 ? 1 : 0)].w, zr = old[2 * N + o + (ux + 1 < (uint32_t)W ? 1 : 0)].w;
        const float zu = old[2 * N + o - (uy > 0 ? W : 0)].w, zd = old[2 * N + o + (uy + 1 < (uint32_t)H ? W : 0)].w;
        const float grad = fminf(fabsf(zl - o2.w), fabsf(zr - o2.w)) + fminf(fabsf(zu - o2.w), fabsf(zd - o2.w));
        if (fabsf(o2.w - dist) > (gk == 2.0f ? 0.25f : 0.02f) * dist + grad) return false;
    }
    if (gk == 0.0f && o2.x * g2.x + o2.y * g2.y + o2.z * g2.z < 0.9f) return false;
    if (edit && gk == 0.0f) {                       // an edit's: the same colour too
        const float dm = fmaxf(fabsf(o3.x - g3.x), fmaxf(fabsf(o3.y - g3.y), fabsf(o3.z - g3.z)));
        if (dm > 0.02f + 0.1f * fmaxf(g3.x, fmaxf(g3.y, g3.z))) return false;
    }
    return true;
}

// the history a pixel keeps with temporal gradients: its tile's filtered lambda as (1 - lambda) /
// lambda samples' worth (A-SVGF's blend), at most hmax; `fallback` where no tile near had a lambda,
// and with an edit's move (lambda then counted 4 times) for what is not a surface
__device__ __forceinline__ float grad_history(const GradTile *__restrict__ tiles, int W, uint32_t k, float4 g3, float hmax,
                                              float fallback, bool edit) {
    const uint32_t tw = ((uint32_t)W + GRAD_TILE - 1) / GRAD_TILE;
    const uint32_t x = k % (uint32_t)W, y = k / (uint32_t)W;
    const float lam = tiles[(y / GRAD_TILE) * tw + x / GRAD_TILE].lam[3];
    if (edit && gkind(g3.w) != 0.0f) return fallback;
    if (!(lam >= 0.0f)) return fallback;
    const float l = edit ? lam * 4.0f : lam;
    return fminf(floorf((1.0f - fminf(l, 1.0f)) / fmaxf(l, 1e-3f) + 0.5f), hmax);
}

// tiles: null without temporal gradients (history for every pixel), else each pixel's history from
// its tile's lambda (grad_history, history the most)
__global__ void __launch_bounds__(256) reproject_kernel(RpCam oc, RpCam nc, int W, int H, float history,
                                                        const float4 *__restrict__ old, float4 *__restrict__ cur,
                                                        const GradTile *__restrict__ tiles, float fallback, bool edit) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)W * H;
    if (k >= N) return;
    const float4 g2 = cur[2 * N + k], g3 = cur[3 * N + k];
    if (tiles) history = grad_history(tiles, W, k, g3, history, fallback, edit);
    const float4 at = old_place(oc, nc, W, H, k, g2);
    float4 a0 = make_float4(0, 0, 0, 0), a1 = make_float4(0, 0, 0, 0);
    float nsum = 0.0f, wsum = 0.0f;
    if (at.w > 0.0f) {
        const float x0 = floorf(at.x), y0 = floorf(at.y);
        for (int j = 0; j < 4; j++) {
            const float tx = x0 + (float)(j & 1), ty = y0 + (float)(j >> 1);
            if (tx < 0.0f || ty < 0.0f || tx >= (float)W || ty >= (float)H) continue;
            const uint32_t o = (uint32_t)ty * (uint32_t)W + (uint32_t)tx;
            if (!same_surface(old, W, H, o, g2, g3, at.z, edit)) continue;
            const float4 s = old[o], m = old[N + o];
            const float w = (1.0f - fabsf(at.x - tx)) * (1.0f - fabsf(at.y - ty));
            const float ws = w / s.w;
            a0 = make_float4(a0.x + ws * s.x, a0.y + ws * s.y, a0.z + ws * s.z, a0.w + ws * s.w);
            a1 = make_float4(a1.x + ws * m.x, a1.y + ws * m.y, a1.z + ws * m.z, a1.w + ws * m.w);
            nsum += w * s.w;
            wsum += w;
        }
    }
    if (wsum < 0.05f || history < 0.5f) {
        cur[k] = make_float4(0, 0, 0, 0);
        cur[N + k] = make_float4(0, 0, 0, 0);
        return;
    }
    const float n = fminf(nsum / wsum, history);
    cur[k] = make_float4(a0.x / wsum * n, a0.y / wsum * n, a0.z / wsum * n, n);
    cur[N + k] = make_float4(a1.x / wsum * n, a1.y / wsum * n, 0.0f, 0.0f);   // (z, w: no sample of this image yet)
}

// the tiles for the caller: (new pixel, old pixel, the sample's lambda, the filtered lambda)
__global__ void grad_out_kernel(const GradTile *__restrict__ tiles, uint32_t n, float4 *__restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const GradTile T = tiles[t];
    out[t] = make_float4((float)T.k, (float)T.o, T.lam[0], T.lam[3]);
}

__device__ __forceinline__ uint32_t hashr(uint32_t x) {     // lowbias32
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// gmatch: one thread per tile. Its pixels from a different first one each image (`next`: the new
// image's first sample number): the first surface pixel whose place in the old image lies in an
// old pixel that saw the same surface and has a last sample; that sample's number from its low 24
// bits (plane 1's w) and the high bits of `next`
__global__ void __launch_bounds__(128) gmatch_kernel(RpCam oc, RpCam nc, int W, int H, uint32_t next, bool edit,
                                                     const float4 *__restrict__ old, const float4 *__restrict__ cur,
                                                     GradTile *__restrict__ tiles) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tw = ((uint32_t)W + GRAD_TILE - 1) / GRAD_TILE, th = ((uint32_t)H + GRAD_TILE - 1) / GRAD_TILE;
    if (t >= tw * th) return;
    const size_t N = (size_t)W * H;
    const uint32_t tx = t % tw, ty = t / tw;
    constexpr uint32_t TT = GRAD_TILE * GRAD_TILE;
    const uint32_t first = hashr(t ^ hashr(next)) % TT;
    GradTile T;
    T.k = T.o = -1;
    T.dx = T.dy = T.l = 0.0f;
    T.kk = 0;
    for (uint32_t i = 0; i < TT; i++) {
        const uint32_t c = (first + i) % TT;
        const uint32_t px = tx * GRAD_TILE + c % GRAD_TILE, py = ty * GRAD_TILE + c / GRAD_TILE;
        if (px >= (uint32_t)W || py >= (uint32_t)H) continue;
        const uint32_t k = py * (uint32_t)W + px;
        const float4 g2 = cur[2 * N + k], g3 = cur[3 * N + k];
        if (gkind(g3.w) != 0.0f) continue;                       // a surface only
        const float4 at = old_place(oc, nc, W, H, k, g2);
        if (at.w <= 0.0f) continue;
        const float ox = floorf(at.x + 0.5f), oy = floorf(at.y + 0.5f);
        if (ox < 0.0f || oy < 0.0f || ox >= (float)W || oy >= (float)H) continue;
        const uint32_t o = (uint32_t)oy * (uint32_t)W + (uint32_t)ox;
        const float4 last = old[N + o];
        if (last.w < 0.5f || !same_surface(old, W, H, o, g2, g3, at.z, edit)) continue;
        const uint32_t lo = (uint32_t)last.w - 1u;
        uint32_t cnt = (next & 0xff000000u) | lo;
        if (cnt > next) cnt -= 0x1000000u;
        T.k = (int32_t)k;
        T.o = (int32_t)o;
        T.dx = ox - at.x;
        T.dy = oy - at.y;
        T.l = last.z;
        T.kk = cnt;
        break;
    }
    for (int q = 0; q < 4; q++) T.lam[q] = -1.0f;
    tiles[t] = T;
}

// gfilter pass `pass` (0, 1, 2): lam[pass] of the tiles 1, 2, 4 tiles apart (3 x 3, B-spline-like
// weights) weighted by the anchors' (each tile's first pixel's) distance and normal into
// lam[pass + 1]; -1 where no tile near had one
__global__ void __launch_bounds__(128) gfilter_kernel(int W, int H, int pass, const float4 *__restrict__ cur,
                                                      GradTile *__restrict__ tiles) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const int tw = (W + GRAD_TILE - 1) / GRAD_TILE, th = (H + GRAD_TILE - 1) / GRAD_TILE;
    if (t >= (uint32_t)(tw * th)) return;
    const size_t N = (size_t)W * H;
    const int tx = (int)(t % (uint32_t)tw), ty = (int)(t / (uint32_t)tw);
    const int step = 1 << pass;
    const float4 ga = cur[2 * N + (size_t)ty * GRAD_TILE * W + tx * GRAD_TILE];
    float sum = 0.0f, wsum = 0.0f;
    for (int dy = -1; dy <= 1; dy++) {
        for (int dx = -1; dx <= 1; dx++) {
            const int bx = tx + dx * step, by = ty + dy * step;
            if (bx < 0 || by < 0 || bx >= tw || by >= th) continue;
            const float lam = tiles[by * tw + bx].lam[pass];
            if (lam < 0.0f) continue;
            const float4 gb = cur[2 * N + (size_t)by * GRAD_TILE * W + bx * GRAD_TILE];
            float w = (dx == 0 ? 1.0f : 0.5f) * (dy == 0 ? 1.0f : 0.5f);
            if (ga.w < 1e29f && gb.w < 1e29f) {
                float nd = fmaxf(ga.x * gb.x + ga.y * gb.y + ga.z * gb.z, 0.0f);
                nd *= nd;
                nd *= nd;
                nd *= nd;
                w *= expf(-fabsf(ga.w - gb.w) / (0.05f * ga.w + 1e-3f)) * nd;
            }
            sum += w * lam;
            wsum += w;
        }
    }
    tiles[t].lam[pass + 1] = wsum > 1e-4f ? sum / wsum : -1.0f;
}

}  // namespace dn

cudaError_t dn_guide(const PtScene &S, const PtParams &P, float4 *d_planes, uint32_t *d_status, cudaStream_t st) {
    const size_t N = (size_t)P.W * P.H;
    if (!N) return cudaSuccess;
    dn::guide_kernel<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(S, P, d_planes, d_status);
    return cudaGetLastError();
}

size_t dn_scratch_bytes(int W, int H) { return 4 * (size_t)W * H * 8 + 512; }

cudaError_t dn_denoise(const float4 *d_planes, int W, int H, int passes, float4 *d_out, void *scratch,
                       cudaStream_t st) {
    const size_t N = (size_t)W * H;
    if (!N) return cudaSuccess;
    uint2 *a = static_cast<uint2 *>(scratch), *b = a + N;
    float4 *gd = reinterpret_cast<float4 *>(b + N);
    const dim3 grid((unsigned)((W + 31) / 32), (unsigned)((H + 7) / 8));
    dn::prep_kernel<<<grid, 256, 0, st>>>(d_planes, W, H, a, gd);
    // a -> b, b -> a, ...; the last pass into out
    for (int i = 1; i <= passes; i++) {
        const uint2 *in = i % 2 ? a : b;
        uint2 *to = i % 2 ? b : a;
        dn::atrous_kernel<<<grid, 256, 0, st>>>(d_planes, W, H, 1 << (i - 1), i == passes, 4.0f, 1.0f, in, to, gd, d_out);
    }
    return cudaGetLastError();
}

}  // namespace lrc

namespace {
lrc::dn::RpCam rp_cam(const lrc_trace_params *p) {
    lrc::dn::RpCam c;
    c.o = make_float3(p->origin[0], p->origin[1], p->origin[2]);
    c.ul = make_float3(p->upper_left[0], p->upper_left[1], p->upper_left[2]);
    c.h = make_float3(p->horizontal[0], p->horizontal[1], p->horizontal[2]);
    c.v = make_float3(p->vertical[0], p->vertical[1], p->vertical[2]);
    return c;
}
}  // namespace

// ---- the C ABI ------------------------------------------------------------------------------
#include "api_internal.cuh"

using namespace lrcapi;

namespace {
// what a scene needs before its paths are traced (lrc_trace's checks)
int scene_traceable(lrc_scene *s) {
    lrc_ctx *c = s->ctx;
    if (!s->built_n && !s->tlas_n) return fail(c, LRC_E_INVALID, "the scene has nothing built (lrc_scene_build)");
    if (s->ninst && s->tlas_n != s->ninst) return fail(c, LRC_E_INVALID, "instances changed: lrc_scene_build_instances");
    if (!s->d_mats || !s->nmats) return fail(c, LRC_E_INVALID, "the scene has no materials (lrc_scene_set_materials)");
    if (s->light >= (int32_t)s->nprims) return fail(c, LRC_E_INVALID, "the light is not one of the primitives");
    if (!s->tables) return lrc_scene_set_tables(s, nullptr, nullptr);
    return LRC_OK;
}

lrc::PtParams trace_params_of(const lrc_trace_params *p) {
    lrc::PtParams P{};
    P.W = p->width; P.H = p->height; P.y0 = 0; P.rows = p->height;
    P.max_depth = p->max_depth; P.mis = p->mis; P.sampler_on = p->sampler; P.exact = p->exact;
    P.seed = p->seed;
    P.clamp = p->clamp;
    P.skip_caustics = p->skip_caustics != 0;
    P.indirect_clamp = p->indirect_clamp;
    P.origin = {p->origin[0], p->origin[1], p->origin[2]};
    P.upper_left = {p->upper_left[0], p->upper_left[1], p->upper_left[2]};
    P.horizontal = {p->horizontal[0], p->horizontal[1], p->horizontal[2]};
    P.vertical = {p->vertical[0], p->vertical[1], p->vertical[2]};
    return P;
}

uint32_t grad_tiles(int W, int H) {
    return (uint32_t)(((W + lrc::GRAD_TILE - 1) / lrc::GRAD_TILE) * (size_t)((H + lrc::GRAD_TILE - 1) / lrc::GRAD_TILE));
}

// the temporal gradients up to the tiles' filtered lambda: gmatch, the gradient samples (the new
// camera and scene, the old image's random numbers: its seed and sampler), the filter's 3 passes
cudaError_t grad_chain(lrc_scene *s, const lrc_trace_params *old_p, const lrc_trace_params *new_p, uint32_t spp0,
                       const float4 *d_old, float4 *d_new, lrc::GradTile *d_tiles, bool edit, cudaStream_t st) {
    lrc_ctx *c = s->ctx;
    const int W = new_p->width, H = new_p->height;
    const size_t N = (size_t)W * H;
    const uint32_t ntiles = grad_tiles(W, H);
    lrc::PtParams P = trace_params_of(new_p);
    P.spp0 = (int)spp0; P.spp = 1; P.group = 1; P.exact = 0;
    P.sampler_on = old_p->sampler;
    P.seed = old_p->seed;
    lrc::dn::gmatch_kernel<<<(ntiles + 127) / 128, 128, 0, st>>>(rp_cam(old_p), rp_cam(new_p), W, H, spp0, edit, d_old,
                                                                 d_new, d_tiles);
    cudaError_t e = cudaGetLastError();
    if (!e) e = lrc::pt_gradients(pt_scene(s), P, d_tiles, ntiles, d_new + 3 * N, s->d_rays, c->d_status, st);
    for (int pass = 0; pass < 3 && !e; pass++) {
        lrc::dn::gfilter_kernel<<<(ntiles + 127) / 128, 128, 0, st>>>(W, H, pass, d_new, d_tiles);
        e = cudaGetLastError();
    }
    return e;
}
}  // namespace

extern "C" {

int lrc_guide(lrc_scene *s, const lrc_trace_params *p, float *planes, unsigned flags) {
    if (!s || !p || !planes || p->width <= 0 || p->height <= 0) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->built_n && !s->tlas_n) return fail(c, LRC_E_INVALID, "the scene has nothing built (lrc_scene_build)");
    if (s->ninst && s->tlas_n != s->ninst) return fail(c, LRC_E_INVALID, "instances changed: lrc_scene_build_instances");
    if (!s->d_mats || !s->nmats) return fail(c, LRC_E_INVALID, "the scene has no materials (lrc_scene_set_materials)");
    DeviceGuard g(c->device);
    if (!s->tables) {
        int rc = lrc_scene_set_tables(s, nullptr, nullptr);
        if (rc) return rc;
    }
    const size_t N = (size_t)p->width * p->height;
    lrc::PtParams P{};
    P.W = p->width; P.H = p->height; P.rows = p->height;
    P.origin = {p->origin[0], p->origin[1], p->origin[2]};
    P.upper_left = {p->upper_left[0], p->upper_left[1], p->upper_left[2]};
    P.horizontal = {p->horizontal[0], p->horizontal[1], p->horizontal[2]};
    P.vertical = {p->vertical[0], p->vertical[1], p->vertical[2]};
    float4 *d_planes = reinterpret_cast<float4 *>(planes);
    cudaError_t e = cudaSuccess;
    if (!(flags & LRC_DEVICE)) {                     // (planes 2 and 3 are written: only they travel)
        e = reserve(&c->stage, &c->stage_cap, N * 64);
        d_planes = static_cast<float4 *>(c->stage);
    }
    c->timer.begin(LRC_TS_SHADE, c->st);
    if (!e) e = lrc::dn_guide(pt_scene(s), P, d_planes, c->d_status, c->st);
    c->timer.end(c->st);
    if (!e && !(flags & LRC_DEVICE))
        e = cudaMemcpyAsync(planes + 8 * N, d_planes + 2 * N, N * 32, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_guide");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_reproject(lrc_ctx *c, const lrc_trace_params *old_cam, const lrc_trace_params *new_cam, const float *old_planes,
                  float *new_planes, int32_t history, unsigned flags) {
    if (!c || !old_cam || !new_cam || !old_planes || !new_planes || history < 0) return LRC_E_INVALID;
    const int W = new_cam->width, H = new_cam->height;
    if (W <= 0 || H <= 0 || old_cam->width != W || old_cam->height != H)
        return fail(c, LRC_E_INVALID, "reprojection: both images of the same size");
    DeviceGuard g(c->device);
    const size_t N = (size_t)W * H;
    const float4 *d_old = reinterpret_cast<const float4 *>(old_planes);
    float4 *d_new = reinterpret_cast<float4 *>(new_planes);
    cudaError_t e = cudaSuccess;
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, N * 128);
        float4 *st = static_cast<float4 *>(c->stage);
        if (!e) e = cudaMemcpyAsync(st, old_planes, N * 64, cudaMemcpyHostToDevice, c->st);
        if (!e) e = cudaMemcpyAsync(st + 4 * N, new_planes, N * 64, cudaMemcpyHostToDevice, c->st);
        d_old = st;
        d_new = st + 4 * N;
    }
    if (!e) {
        lrc::dn::reproject_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>(rp_cam(old_cam), rp_cam(new_cam), W, H,
                                                                                  (float)history, d_old, d_new, nullptr,
                                                                                  0.0f, false);
        e = cudaGetLastError();
    }
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(new_planes, d_new, N * 32, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_reproject");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_reproject_gradients(lrc_scene *s, const lrc_trace_params *old_p, const lrc_trace_params *new_p, uint32_t spp0,
                            const float *old_planes, float *new_planes, int32_t history_max, int32_t history,
                            float *tiles_out, unsigned flags) {
    if (!s || !old_p || !new_p || !old_planes || !new_planes || history_max <= 0 || history < 0) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    const int W = new_p->width, H = new_p->height;
    if (W <= 0 || H <= 0 || old_p->width != W || old_p->height != H)
        return fail(c, LRC_E_INVALID, "reprojection: both images of the same size");
    if ((uint64_t)W * (uint64_t)H >= (1ull << 31)) return fail(c, LRC_E_INVALID, "image too large (2^31 pixels)");
    if (old_p->exact)
        return fail(c, LRC_E_INVALID, "temporal gradients trace a sample again: the old image in fast mode (exact = 0)");
    DeviceGuard g(c->device);
    int rc = scene_traceable(s);
    if (rc) return rc;
    const size_t N = (size_t)W * H;
    const uint32_t ntiles = grad_tiles(W, H);
    const float4 *d_old = reinterpret_cast<const float4 *>(old_planes);
    float4 *d_new = reinterpret_cast<float4 *>(new_planes);
    float4 *d_tout = reinterpret_cast<float4 *>(tiles_out);
    const size_t tile_bytes = ((size_t)ntiles * sizeof(lrc::GradTile) + 255) / 256 * 256;
    cudaError_t e = reserve(&c->dn, &c->dn_cap, tile_bytes + (size_t)ntiles * 16 + 256);
    if (e) return cuda_status(c, e, "gradient tiles");
    lrc::GradTile *d_tiles = static_cast<lrc::GradTile *>(c->dn);
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, N * 128);
        float4 *st = static_cast<float4 *>(c->stage);
        if (!e) e = cudaMemcpyAsync(st, old_planes, N * 64, cudaMemcpyHostToDevice, c->st);
        if (!e) e = cudaMemcpyAsync(st + 4 * N, new_planes, N * 64, cudaMemcpyHostToDevice, c->st);
        d_old = st;
        d_new = st + 4 * N;
        d_tout = reinterpret_cast<float4 *>(static_cast<char *>(c->dn) + tile_bytes);
    }
    if (!e && !s->d_rays) e = cudaMalloc(&s->d_rays, 256);
    if (!e) e = cudaMemsetAsync(s->d_rays, 0, 8, c->st);
    if (e) return cuda_status(c, e, "lrc_reproject_gradients");
    const bool edit = (flags & LRC_REPROJECT_EDIT) != 0;
    c->timer.begin(LRC_TS_SHADE, c->st);
    e = grad_chain(s, old_p, new_p, spp0, d_old, d_new, d_tiles, edit, c->st);
    if (!e) {
        lrc::dn::reproject_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>(rp_cam(old_p), rp_cam(new_p), W, H,
                                                                                  (float)history_max, d_old, d_new,
                                                                                  d_tiles, (float)history, edit);
        e = cudaGetLastError();
    }
    if (!e && tiles_out) {
        lrc::dn::grad_out_kernel<<<(ntiles + 127) / 128, 128, 0, c->st>>>(d_tiles, ntiles, d_tout);
        e = cudaGetLastError();
    }
    c->timer.end(c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(new_planes, d_new, N * 32, cudaMemcpyDeviceToHost, c->st);
    if (!e && tiles_out && !(flags & LRC_DEVICE))
        e = cudaMemcpyAsync(tiles_out, d_tout, (size_t)ntiles * 16, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_reproject_gradients");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_trace_frame(lrc_scene *s, const lrc_trace_params *old_p, const lrc_trace_params *new_p, uint32_t spp0,
                    uint32_t spp, const float *old_planes, float *new_planes, int32_t history_max, int32_t history,
                    unsigned flags) {
    if (!s || !new_p || !new_planes || !spp || history_max < 0 || history < 0 || (old_planes && !old_p))
        return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    const int W = new_p->width, H = new_p->height;
    if (W <= 0 || H <= 0 || (old_planes && (old_p->width != W || old_p->height != H)))
        return fail(c, LRC_E_INVALID, "reprojection: both images of the same size");
    if ((uint64_t)W * (uint64_t)H >= (1ull << 31)) return fail(c, LRC_E_INVALID, "image too large (2^31 pixels)");
    if (new_p->exact) return fail(c, LRC_E_INVALID, "a frame's samples in fast mode (exact = 0)");
    const bool grads = old_planes && history_max > 0;
    if (grads && old_p->exact)
        return fail(c, LRC_E_INVALID, "temporal gradients trace a sample again: the old image in fast mode (exact = 0)");
    DeviceGuard g(c->device);
    int rc = scene_traceable(s);
    if (rc) return rc;
    const size_t N = (size_t)W * H;
    const uint32_t ntiles = grad_tiles(W, H);
    const float4 *d_old = reinterpret_cast<const float4 *>(old_planes);
    float4 *d_new = reinterpret_cast<float4 *>(new_planes);
    cudaError_t e = cudaSuccess;
    if (grads) e = reserve(&c->dn, &c->dn_cap, ((size_t)ntiles * sizeof(lrc::GradTile) + 255) / 256 * 256 + 256);
    if (!e && !(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, N * 128);
        float4 *st = static_cast<float4 *>(c->stage);
        if (!e && old_planes) e = cudaMemcpyAsync(st, old_planes, N * 64, cudaMemcpyHostToDevice, c->st);
        d_old = old_planes ? st : nullptr;
        d_new = st + 4 * N;
    }
    if (!e && !s->d_rays) e = cudaMalloc(&s->d_rays, 256);
    if (!e) e = cudaMemsetAsync(s->d_rays, 0, 8, c->st);
    if (e) return cuda_status(c, e, "lrc_trace_frame");
    lrc::PtParams P = trace_params_of(new_p);
    P.spp0 = (int)spp0;
    P.spp = (int)spp;
    int gsz = 1;
    while (gsz * 2 <= (int)spp && gsz < 16) gsz *= 2;
    P.group = gsz;
    P.moments = d_new + N;
    P.guide = d_new + 3 * N;
    lrc::GradTile *d_tiles = static_cast<lrc::GradTile *>(c->dn);
    const bool edit = (flags & LRC_REPROJECT_EDIT) != 0;
    c->timer.begin(LRC_TS_SHADE, c->st);
    e = lrc::dn_guide(pt_scene(s), P, d_new, c->d_status, c->st);
    if (!e && grads) e = grad_chain(s, old_p, new_p, spp0, d_old, d_new, d_tiles, edit, c->st);
    if (!e && old_planes) {
        lrc::dn::reproject_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>(
            rp_cam(old_p), rp_cam(new_p), W, H, (float)(grads ? history_max : history), d_old, d_new,
            grads ? d_tiles : nullptr, (float)history, grads && edit);
        e = cudaGetLastError();
    } else if (!e) {
        e = cudaMemsetAsync(d_new, 0, N * 32, c->st);   // (the first frame: no history)
    }
    if (!e) e = lrc::pt_trace(pt_scene(s), P, reinterpret_cast<float *>(d_new), s->d_rays, c->d_status, c->st);
    c->timer.end(c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(new_planes, d_new, N * 64, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_trace_frame");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_denoise(lrc_ctx *c, int32_t width, int32_t height, const float *planes, int32_t passes, float *out,
                unsigned flags) {
    if (!c || !planes || !out || width <= 0 || height <= 0) return LRC_E_INVALID;
    if ((uint64_t)width * (uint64_t)height >= (1ull << 31)) return fail(c, LRC_E_INVALID, "image too large (2^31 pixels)");
    if (passes < 1 || passes > 5) passes = 5;
    DeviceGuard g(c->device);
    const size_t N = (size_t)width * height;
    cudaError_t e = reserve(&c->dn, &c->dn_cap, lrc::dn_scratch_bytes(width, height));
    if (e) return cuda_status(c, e, "denoiser scratch");
    const float4 *d_planes = reinterpret_cast<const float4 *>(planes);
    float4 *d_out = reinterpret_cast<float4 *>(out);
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, N * 80);
        if (e) return cuda_status(c, e, "image staging");
        float4 *st = static_cast<float4 *>(c->stage);
        d_planes = st;
        d_out = st + 4 * N;
        e = cudaMemcpyAsync(st, planes, N * 64, cudaMemcpyHostToDevice, c->st);
    }
    c->timer.begin(LRC_TS_DENOISE, c->st);
    if (!e) e = lrc::dn_denoise(d_planes, width, height, passes, d_out, c->dn, c->st);
    c->timer.end(c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(out, d_out, N * 16, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_denoise");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

}  // extern "C"
