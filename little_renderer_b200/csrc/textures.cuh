// textures.cuh - the materials' textures on the device (the reference's PBR5: engine/scene/texture.c,
// scene.c material_at / material_normal, rt/intersect.c hit_texcoords, rt/tracer.c hit_shading),
// restated with the float build's roundings. The path tracers sample level 0 bilinearly (they pass
// MATERIAL_LOD0: no filtering footprint), so only level 0 of each texmap is kept on the device.
#pragma once
#include "lrc_internal.cuh"
#include "pt_math.cuh"
#include "bsdf.cuh"

namespace lrc {
namespace pt {

enum { TEX_REPEAT = 0, TEX_CLAMP = 1, TEX_MIRROR = 2 };

struct Tex4 {
    float x, y, z, w;
};

// fold (texture.c:245-252): u into [0, 1] by the wrap mode
__device__ __forceinline__ float tex_fold(float u, int mode) {
    if (mode == TEX_CLAMP) return u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
    if (mode == TEX_MIRROR) {
        const float m = sub(u, mul(2.0f, floorf(mul(u, 0.5f))));
        return m > 1.0f ? sub(2.0f, m) : m;
    }
    return u >= 0.0f && u < 1.0f ? u : sub(u, floorf(u));
}
// edge (texture.c:254-257): texel -1 .. n of a row of n
__device__ __forceinline__ int tex_edge(int x, int n, int mode) {
    if (mode == TEX_REPEAT) return x < 0 ? x + n : (x >= n ? x - n : x);
    return x < 0 ? 0 : (x >= n ? n - 1 : x);
}
__device__ __forceinline__ Tex4 tex_decode(uint32_t c, const float *lut) {
    Tex4 r;
    if (lut) {
        r.x = __ldg(&lut[c & 255]);
        r.y = __ldg(&lut[(c >> 8) & 255]);
        r.z = __ldg(&lut[(c >> 16) & 255]);
    } else {
        r.x = mul((float)(c & 255), 1.0f / 255.0f);
        r.y = mul((float)((c >> 8) & 255), 1.0f / 255.0f);
        r.z = mul((float)((c >> 16) & 255), 1.0f / 255.0f);
    }
    r.w = mul((float)(c >> 24), 1.0f / 255.0f);
    return r;
}
__device__ __forceinline__ Tex4 tex_lerp(Tex4 a, Tex4 b, float f) {
    return Tex4{add(a.x, mul(sub(b.x, a.x), f)), add(a.y, mul(sub(b.y, a.y), f)), add(a.z, mul(sub(b.z, a.z), f)),
                add(a.w, mul(sub(b.w, a.w), f))};
}

// texmap_sample at level 0 (texture.c:260-283): texmap k (0-based), bilinear
__device__ __forceinline__ Tex4 tex_sample0(const PtScene &S, uint32_t k, float u, float v) {
    if (!(u > -1e6f && u < 1e6f && v > -1e6f && v < 1e6f)) u = v = 0.0f;
    const uint4 T = __ldg(&S.texs[k]);
    const int w = (int)T.x, h = (int)T.y, wu = (int)((T.z >> 1) & 3), wv = (int)((T.z >> 3) & 3);
    u = tex_fold(u, wu);
    v = tex_fold(v, wv);
    const float x = sub(mul(u, (float)w), 0.5f), y = sub(mul(v, (float)h), 0.5f);
    const float fx0 = floorf(x), fy0 = floorf(y);
    int x0 = (int)fx0, y0 = (int)fy0;
    const float fx = sub(x, fx0), fy = sub(y, fy0);
    if (x0 < -1) x0 = -1;
    if (x0 > w - 1) x0 = w - 1;
    if (y0 < -1) y0 = -1;
    if (y0 > h - 1) y0 = h - 1;
    const int xa = tex_edge(x0, w, wu), xb = tex_edge(x0 + 1, w, wu), ya = tex_edge(y0, h, wv), yb = tex_edge(y0 + 1, h, wv);
    const uint32_t *px = S.texels + T.w;
    const float *lut = (T.z & 1u) ? S.srgb : nullptr;
    const Tex4 a = tex_decode(__ldg(&px[(size_t)ya * w + xa]), lut), b = tex_decode(__ldg(&px[(size_t)ya * w + xb]), lut);
    const Tex4 c = tex_decode(__ldg(&px[(size_t)yb * w + xa]), lut), d = tex_decode(__ldg(&px[(size_t)yb * w + xb]), lut);
    return tex_lerp(tex_lerp(a, b, fx), tex_lerp(c, d, fx), fy);
}

// a texture number (1 + index) that names one of the scene's texmaps
__device__ __forceinline__ bool tex_ok(const PtScene &S, uint32_t t) { return t > 0 && t <= S.ntex; }

// the barycentrics (b1, b2) the triangle test gives for this ray (lr_hit_triangle_t)
__device__ __forceinline__ void tri_bary(const float4 *tp, V3 o, V3 d, float &b1, float &b2) {
    const float4 q = ld4(tp), u = ld4(tp + 1), v = ld4(tp + 2);
    const V3 uu = v3(u.x, u.y, u.z), vv = v3(v.x, v.y, v.z);
    const V3 pvec = vcross(d, vv);
    const float inv = dvd(1.0f, vdot(uu, pvec));
    const V3 tvec = vsub(o, v3(q.x, q.y, q.z));
    b1 = mul(vdot(tvec, pvec), inv);
    b2 = mul(vdot(d, vcross(tvec, uu)), inv);
}
// quad_tangent (intersect.c:84-87)
__device__ __forceinline__ Tex4 quad_tangent(V3 u) {
    const V3 t = vnorm(u);
    return Tex4{t.x, t.y, t.z, -1.0f};
}

// hit_texcoords (intersect.c:89-132) for the hit of the ray (o, d) at h: its texture coordinates and
// tangent (xyz, handedness w)
__device__ __forceinline__ void hit_texcoords(const PtScene &S, const Hit &h, V3 o, V3 d, float &tu, float &tv, Tex4 &tg) {
    if (h.inst < 0) {
        if ((uint32_t)h.prim < S.nprims) {
            const float4 *pr = S.prims + 6 * (size_t)h.prim;
            const float4 c = ld4(pr), qf = ld4(pr + 1);
            if (qf.w == 0.0f) {                      // a sphere: longitude and latitude
                const V3 p = vadd(o, vscale(d, h.t));
                const V3 n = vscale(vsub(p, v3(c.x, c.y, c.z)), dvd(1.0f, c.w));
                const float ny = n.y < -1.0f ? -1.0f : (n.y > 1.0f ? 1.0f : n.y);
                const float uu = add(0.5f, mul(atan2f(n.x, n.z), dvd(0.5f, PIF)));
                tu = sub(uu, floorf(uu));
                tv = mul(acosf(ny), dvd(1.0f, PIF));
                const float ph = mul(sub(tu, 0.5f), mul(2.0f, PIF));
                tg = Tex4{cosf(ph), 0.0f, -sinf(ph), 1.0f};
            } else {                                 // a quad: (a, b)
                const float4 q = ld4(pr + 1), u = ld4(pr + 2), v = ld4(pr + 3), w = ld4(pr + 5);
                const V3 p = vadd(o, vscale(d, h.t));
                const V3 rel = vsub(p, v3(q.x, q.y, q.z));
                const V3 ww = v3(w.x, w.y, w.z);
                tu = vdot(ww, vcross(rel, v3(v.x, v.y, v.z)));
                tv = vdot(ww, vcross(v3(u.x, u.y, u.z), rel));
                tg = quad_tangent(v3(u.x, u.y, u.z));
            }
            return;
        }
        const uint32_t k = (uint32_t)h.prim - S.nprims;
        const float4 *tp = S.tris + 3 * (size_t)k;
        float b1, b2;
        tri_bary(tp, o, d, b1, b2);
        const int t0 = S.tri_uv ? __ldg(&S.tri_uv[3 * (size_t)k]) : -1;
        const int t1 = S.tri_uv ? __ldg(&S.tri_uv[3 * (size_t)k + 1]) : -1;
        const int t2 = S.tri_uv ? __ldg(&S.tri_uv[3 * (size_t)k + 2]) : -1;
        const int n = (int)S.nuv;
        if (t0 < 0 || t0 >= n || t1 >= n || t2 >= n || t1 < 0 || t2 < 0) {   // tri_texcoords' fallback
            tu = b1;
            tv = b2;
            const float4 u = ld4(tp + 1);
            tg = quad_tangent(v3(u.x, u.y, u.z));
            tg.w = 1.0f;
            return;
        }
        const float w0 = sub(sub(1.0f, b1), b2);
        const float2 a0 = __ldg(&S.uvs[t0]), a1 = __ldg(&S.uvs[t1]), a2 = __ldg(&S.uvs[t2]);
        tu = add(add(mul(w0, a0.x), mul(b1, a1.x)), mul(b2, a2.x));
        tv = add(add(mul(w0, a0.y), mul(b1, a1.y)), mul(b2, a2.y));
        const float4 g0 = __ldg(&S.tangents[t0]), g1 = __ldg(&S.tangents[t1]), g2 = __ldg(&S.tangents[t2]);
        tg = Tex4{add(add(mul(w0, g0.x), mul(b1, g1.x)), mul(b2, g2.x)), add(add(mul(w0, g0.y), mul(b1, g1.y)), mul(b2, g2.y)),
                  add(add(mul(w0, g0.z), mul(b1, g1.z)), mul(b2, g2.z)), g0.w};
        return;
    }
    // an instance's mesh triangle (no texture coordinates here: tri_texcoords' fallback), made in
    // the instance's space and its tangent turned into the world
    const float4 *rec = S.inst + 8 * (size_t)h.inst;
    const uint4 mi = __ldg(&S.mesh_info[__float_as_uint(ld4(rec + 6).w)]);
    const float4 *tp = S.mtris + 3 * (size_t)(mi.y + h.prim);
    float b1, b2;
    tri_bary(tp, xpoint(rec + 3, o), xdir(rec + 3, d), b1, b2);
    tu = b1;
    tv = b2;
    const float4 u = ld4(tp + 1);
    const Tex4 t = quad_tangent(v3(u.x, u.y, u.z));
    const V3 dd = vnorm(xdir(rec, v3(t.x, t.y, t.z)));
    tg = Tex4{dd.x, dd.y, dd.z, 1.0f};
}

// uv_scaled (scene.c:244-247)
__device__ __forceinline__ float uv_k(const Mat &m) { return m.uv_scale > 0.0f ? m.uv_scale : 1.0f; }

// material_at (scene.c:259-279) at level 0: the material with its textures applied (type MAT_PBR)
__device__ __forceinline__ Mat material_at(const PtScene &S, const Mat &m, float u, float v) {
    Mat r = resolved(m);
    const float k = uv_k(m);
    u = mul(u, k);
    v = mul(v, k);
    const uint32_t base = m.tex0 & 0xffu, emis = (m.tex0 >> 8) & 0xffu, mr = m.tex1 & 0xffu;
    if (tex_ok(S, base)) {
        const Tex4 c = tex_sample0(S, base - 1, u, v);
        r.albedo = v3(mul(r.albedo.x, c.x), mul(r.albedo.y, c.y), mul(r.albedo.z, c.z));
    }
    if (tex_ok(S, mr)) {
        const Tex4 c = tex_sample0(S, mr - 1, u, v);
        r.roughness = mul(r.roughness, c.y);
        r.metallic = mul(r.metallic, c.z);
    }
    if (tex_ok(S, emis)) {
        const Tex4 c = tex_sample0(S, emis - 1, u, v);
        r.emission = v3(mul(r.emission.x, c.x), mul(r.emission.y, c.y), mul(r.emission.z, c.z));
    }
    r.type = MAT_PBR;
    r.tex0 = r.tex1 = r.tex2 = 0;
    return r;
}

// material_normal (scene.c:288-301): the normal map's normal in the world (tangent space, green up)
__device__ __forceinline__ V3 material_normal(const PtScene &S, const Mat &m, float u, float v, V3 n, Tex4 t) {
    const uint32_t nt = m.tex2 & 0xffu;
    if (!tex_ok(S, nt)) return n;
    const float k = uv_k(m);
    const Tex4 c = tex_sample0(S, nt - 1, mul(u, k), mul(v, k));
    const V3 t3 = v3(t.x, t.y, t.z);
    V3 tt = vsub(t3, vscale(n, vdot(n, t3)));
    const float l = vlen(tt);
    if (!(l > 1e-6f)) return n;
    tt = vscale(tt, dvd(1.0f, l));
    const V3 b = vscale(vcross(n, tt), t.w);
    const uint32_t nsq = m.tex2 >> 8;
    const float ns = (float)nsq * (1.0f / 4096.0f), kk = ns > 0.0f ? ns : 1.0f;
    const V3 out = vadd(vadd(vscale(tt, mul(kk, sub(mul(2.0f, c.x), 1.0f))), vscale(b, mul(kk, sub(mul(2.0f, c.y), 1.0f)))),
                        vscale(n, sub(mul(2.0f, c.z), 1.0f)));
    const float lo = vlen(out);
    return lo > 1e-6f ? vscale(out, dvd(1.0f, lo)) : n;
}

// hit_shading (tracer.c:241-255): the material at the hit with its textures applied, and the
// shading normal bent by its normal map (tilted back towards v, the direction the ray came from,
// when it would face away). m: the hit's material as stored; h: the hit of the ray (o, d)
__device__ __forceinline__ Mat hit_shading(const PtScene &S, Hit &h, V3 o, V3 d, V3 v, const Mat &m) {
    if (!textured(m) || m.type == MAT_LIGHT) return m;
    float u, w;
    Tex4 tg;
    hit_texcoords(S, h, o, d, u, w, tg);
    const Mat r = material_at(S, m, u, w);
    if (m.tex2 & 0xffu) {
        V3 n = material_normal(S, m, u, w, h.n, tg);
        const float c = vdot(n, v);
        if (c < 1e-3f) n = vnorm(vadd(n, vscale(v, sub(1e-3f, c))));
        h.n = n;
    }
    return r;
}

}  // namespace pt
}  // namespace lrc
