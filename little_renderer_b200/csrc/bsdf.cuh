// bsdf.cuh - the reference's BSDF (engine/scene/brdf.h: glTF metallic-roughness with transmission;
// GGX with height-correlated Smith masking, Schlick Fresnel, Kulla-Conty multiple scattering, a
// Lambert layer under the dielectric specular one, Walter et al.'s rough BTDF; roughness <= 0.02
// perfectly smooth), restated for the device with the C code's operation order (pt_math.cuh).
// The albedo tables (scene/brdf_tables.h, 2112 floats: E[32][32], B[32][32], E_avg[32], B_avg[32],
// packed as gpu_bsdf_tables packs them, engine/gpu/brdf_gpu.c:20-25) come from the caller.
#pragma once
#include "pt_math.cuh"

namespace lrc {
namespace pt {

enum { MAT_DIFFUSE = 0, MAT_MIRROR = 1, MAT_GLASS = 2, MAT_LIGHT = 3, MAT_PBR = 4 };
enum { BSDF_SPEC = 0, BSDF_DIFF = 1, BSDF_TRANS = 2, BSDF_MS = 3, BSDF_LOBES = 4 };
constexpr int TAB_N = 32;
constexpr int TAB_E = 0, TAB_B = 1024, TAB_EAVG = 2048, TAB_BAVG = 2080, TAB_FLOATS = 2112;

// a material on the device (16 floats): albedo.xyz, type | emission.xyz, - | ior, metallic,
// roughness, transmission | its textures as gpu_tex_pack packs them (engine/gpu/tex_gpu.c:19-29):
// base | emissive << 8, metal-rough | occlusion << 8 | occlusion strength << 16, normal |
// normal scale x 4096 << 8 (bits), uv scale (float); texture numbers 1 + the texmap's index, 0 none
struct Mat {
    V3 albedo, emission;
    int type;
    float ior, metallic, roughness, transmission;
    uint32_t tex0, tex1, tex2;
    float uv_scale;
};
__device__ __forceinline__ Mat load_mat(const float4 *mats, int i) {
    float4 a = __ldg(&mats[4 * i]), e = __ldg(&mats[4 * i + 1]), p = __ldg(&mats[4 * i + 2]), t = __ldg(&mats[4 * i + 3]);
    Mat m;
    m.albedo = v3(a.x, a.y, a.z);
    m.type = __float_as_int(a.w);
    m.emission = v3(e.x, e.y, e.z);
    m.ior = p.x; m.metallic = p.y; m.roughness = p.z; m.transmission = p.w;
    m.tex0 = __float_as_uint(t.x);
    m.tex1 = __float_as_uint(t.y);
    m.tex2 = __float_as_uint(t.z);
    m.uv_scale = t.w;
    return m;
}
// material_textured (scene.h:76-78): base, metal-rough, normal, emissive or occlusion
__device__ __forceinline__ bool textured(const Mat &m) { return ((m.tex0 | m.tex1) & 0xffffu) || (m.tex2 & 0xffu); }
// material_resolved (scene.h): a preset's parameters filled in
__device__ __forceinline__ Mat resolved(Mat r) {
    switch (r.type) {
    case MAT_DIFFUSE: r.metallic = 0; r.roughness = 1; r.ior = 1.5f; r.transmission = 0; break;
    case MAT_MIRROR: r.metallic = 1; r.roughness = 0; r.ior = 1.5f; r.transmission = 0; break;
    case MAT_GLASS: r.metallic = 0; r.roughness = 0; r.transmission = 1; if (!(r.ior > 0)) r.ior = 1.5f; break;
    case MAT_LIGHT: r.metallic = 0; r.roughness = 1; r.transmission = 0; break;
    default: if (!(r.ior > 0)) r.ior = 1.5f; break;
    }
    return r;
}
__device__ __forceinline__ bool glows(const Mat &m) {
    return m.type != MAT_LIGHT && (m.emission.x > 0 || m.emission.y > 0 || m.emission.z > 0);
}

struct Bsdf {
    V3 base;
    float metallic, transmission, rough, alpha, eta, e_avg, es_avg;
    int smooth;
    V3 ms;
    float kd_norm, kms_norm;
    float cv, p[BSDF_LOBES], es_v, e_v;
    const float *tab;
};

struct BsdfSample {
    V3 l, w;
    float pdf;
    int delta, through;
};

__device__ __forceinline__ float lum(V3 c) { return add(add(mul(0.2126f, c.x), mul(0.7152f, c.y)), mul(0.0722f, c.z)); }

// bsdf_table: bilinear in (roughness, cosine)
__device__ __forceinline__ float table(const float *t, float rough, float mu) {
    float x = mul(rough, (float)(TAB_N - 1)), y = mul(clamp01(mu), (float)(TAB_N - 1));
    int j = (int)x, i = (int)y;
    if (j > TAB_N - 2) j = TAB_N - 2;
    if (i > TAB_N - 2) i = TAB_N - 2;
    float fx = sub(x, (float)j), fy = sub(y, (float)i);
    float t00 = __ldg(&t[j * TAB_N + i]), t01 = __ldg(&t[j * TAB_N + i + 1]);
    float t10 = __ldg(&t[(j + 1) * TAB_N + i]), t11 = __ldg(&t[(j + 1) * TAB_N + i + 1]);
    float e0 = add(t00, mul(fy, sub(t01, t00)));
    float e1 = add(t10, mul(fy, sub(t11, t10)));
    return add(e0, mul(fx, sub(e1, e0)));
}
__device__ __forceinline__ float albedo_e(const Bsdf &b, float mu) { return table(b.tab + TAB_E, b.rough, mu); }
__device__ __forceinline__ float albedo_b(const Bsdf &b, float mu) { return table(b.tab + TAB_B, b.rough, mu); }

__device__ __forceinline__ float fresnel_dielectric(float cos_i, float eta) {
    cos_i = clamp01(cos_i);
    float s2 = mul(mul(eta, eta), sub(1.0f, mul(cos_i, cos_i)));
    if (s2 >= 1.0f) return 1.0f;
    float c = eta > 1.0f ? __fsqrt_rn(sub(1.0f, s2)) : cos_i;
    float f0 = dvd(sub(1.0f, eta), add(1.0f, eta));
    f0 = mul(f0, f0);
    float x = sub(1.0f, c), x2 = mul(x, x);
    return add(f0, mul(mul(mul(sub(1.0f, f0), x2), x2), x));
}
__device__ __forceinline__ float fresnel_dielectric_avg(float eta) {
    float e = eta > 1.0f ? dvd(1.0f, eta) : eta;
    float f0 = dvd(sub(1.0f, e), add(1.0f, e));
    f0 = mul(f0, f0);
    float avg = add(f0, dvd(sub(1.0f, f0), 21.0f));
    return eta > 1.0f ? sub(1.0f, dvd(sub(1.0f, avg), mul(eta, eta))) : avg;
}
__device__ __forceinline__ float spec_albedo(const Bsdf &b, float mu) {
    if (b.smooth || b.eta > 1.0f) return fresnel_dielectric(mu, b.eta);
    float f0 = dvd(sub(1.0f, b.eta), add(1.0f, b.eta)), e = albedo_e(b, mu), bb = albedo_b(b, mu);
    f0 = mul(f0, f0);
    return add(mul(f0, sub(e, bb)), bb);
}
__device__ __forceinline__ float spec_albedo_avg(const Bsdf &b) {
    return b.smooth || b.eta > 1.0f ? fresnel_dielectric_avg(b.eta) : b.es_avg;
}
__device__ __forceinline__ V3 fresnel_metal(V3 f0, float c) {
    float x = sub(1.0f, clamp01(c)), x2 = mul(x, x), x5 = mul(mul(x2, x2), x);
    return v3(add(f0.x, mul(sub(1.0f, f0.x), x5)), add(f0.y, mul(sub(1.0f, f0.y), x5)), add(f0.z, mul(sub(1.0f, f0.z), x5)));
}
__device__ __forceinline__ float ggx_d(float nh, float s2, float a) {
    float a2 = mul(a, a), d = add(s2, mul(mul(a2, nh), nh));
    return dvd(a2, mul(mul(PIF, d), d));
}
__device__ __forceinline__ float ggx_s2(V3 n, V3 h) {
    V3 c = vcross(n, h);
    return vdot(c, c);
}
__device__ __forceinline__ float ggx_g1(float c, float a) {
    c = fabsf(c);
    float aa = mul(a, a);
    return dvd(mul(2.0f, c), add(c, __fsqrt_rn(add(aa, mul(mul(sub(1.0f, aa), c), c)))));
}
__device__ __forceinline__ float ggx_vis(float cv, float cl, float a) {
    cv = fabsf(cv);
    cl = fabsf(cl);
    float a2 = mul(a, a);
    float d = add(mul(cl, __fsqrt_rn(add(mul(mul(cv, cv), sub(1.0f, a2)), a2))),
                  mul(cv, __fsqrt_rn(add(mul(mul(cl, cl), sub(1.0f, a2)), a2))));
    return d > 0.0f ? dvd(0.5f, d) : 0.0f;
}
__device__ __forceinline__ V3 ggx_sample_vndf(V3 n, V3 v, float a, float u1, float u2) {
    V3 t, bt;
    onb(n, t, bt);
    V3 vh = vnorm(v3(mul(a, vdot(v, t)), mul(a, vdot(v, bt)), vdot(v, n)));
    float phi = mul(mul(2.0f, PIF), u1);
    float z = sub(mul(sub(1.0f, u2), add(1.0f, vh.z)), vh.z);
    float st = __fsqrt_rn(rmax(0.0f, sub(1.0f, mul(z, z))));
    V3 hs = v3(add(mul(st, cosf(phi)), vh.x), add(mul(st, sinf(phi)), vh.y), add(z, vh.z));
    V3 hl = vnorm(v3(mul(a, hs.x), mul(a, hs.y), rmax(hs.z, 0.0f)));
    return vadd(vadd(vscale(t, hl.x), vscale(bt, hl.y)), vscale(n, hl.z));
}
__device__ __forceinline__ V3 ms_color(const Bsdf &b) {
    float e = b.e_avg;
    V3 fa = v3(add(b.base.x, dvd(sub(1.0f, b.base.x), 21.0f)), add(b.base.y, dvd(sub(1.0f, b.base.y), 21.0f)),
               add(b.base.z, dvd(sub(1.0f, b.base.z), 21.0f)));
    return v3(dvd(mul(mul(fa.x, fa.x), e), sub(1.0f, mul(fa.x, sub(1.0f, e)))),
              dvd(mul(mul(fa.y, fa.y), e), sub(1.0f, mul(fa.y, sub(1.0f, e)))),
              dvd(mul(mul(fa.z, fa.z), e), sub(1.0f, mul(fa.z, sub(1.0f, e)))));
}

// bsdf_make: outside = v on the side the geometric normal points to
__device__ __forceinline__ Bsdf bsdf_make(const Mat &mat, int outside, const float *tab) {
    Mat m = resolved(mat);
    Bsdf b;
    b.tab = tab;
    b.base = m.albedo;
    b.metallic = clamp01(m.metallic);
    b.transmission = clamp01(m.transmission);
    float r = clamp01(m.roughness);
    b.smooth = r <= 0.02f;
    b.rough = r;
    b.alpha = rmax(mul(r, r), 1e-4f);
    float ior = m.ior > 0.0f ? m.ior : 1.5f;
    b.eta = b.transmission > 0.0f && !outside ? ior : dvd(1.0f, ior);
    float x = mul(r, (float)(TAB_N - 1));
    int j = (int)x;
    if (j > TAB_N - 2) j = TAB_N - 2;
    const float *ea = tab + TAB_EAVG, *ba = tab + TAB_BAVG;
    b.e_avg = add(__ldg(&ea[j]), mul(sub(x, (float)j), sub(__ldg(&ea[j + 1]), __ldg(&ea[j]))));
    float b_avg = add(__ldg(&ba[j]), mul(sub(x, (float)j), sub(__ldg(&ba[j + 1]), __ldg(&ba[j]))));
    float f0 = dvd(sub(1.0f, b.eta), add(1.0f, b.eta));
    f0 = mul(f0, f0);
    b.es_avg = add(mul(f0, sub(b.e_avg, b_avg)), b_avg);
    b.kd_norm = dvd(1.0f, sub(1.0f, spec_albedo_avg(b)));
    b.kms_norm = dvd(1.0f, mul(PIF, sub(1.0f, b.e_avg)));
    b.ms = b.smooth || b.metallic <= 0.0f ? v3(0, 0, 0) : ms_color(b);
    b.cv = -1.0f;
    b.es_v = b.e_v = 0.0f;
    for (int i = 0; i < BSDF_LOBES; i++) b.p[i] = 0.0f;
    return b;
}

// bsdf_view: the lobes' chances and albedos seen from cosine cv
__device__ __forceinline__ void bsdf_view(Bsdf &b, float cv) {
    if (b.cv == cv) return;
    b.cv = cv;
    float fd = fresnel_dielectric(cv, b.eta);
    float fs = b.smooth ? fd : rmin(fd, 0.9f);
    float m = b.metallic, t = b.transmission, lb = lum(b.base);
    b.es_v = mul(sub(1.0f, m), sub(1.0f, t)) > 0.0f ? spec_albedo(b, cv) : 0.0f;
    b.e_v = b.smooth || m <= 0.0f ? 1.0f : albedo_e(b, cv);
    float w0 = add(mul(sub(1.0f, m), fs), mul(m, lum(fresnel_metal(b.base, cv))));
    float w1 = mul(mul(mul(sub(1.0f, m), sub(1.0f, t)), sub(1.0f, b.es_v)), lb);
    float w2 = mul(mul(mul(sub(1.0f, m), t), sub(1.0f, fs)), lb);
    float w3 = mul(mul(m, lum(b.ms)), sub(1.0f, b.e_v));
    float sum = add(add(add(w0, w1), w2), w3);
    b.p[0] = sum > 0.0f ? dvd(w0, sum) : 0.0f;
    b.p[1] = sum > 0.0f ? dvd(w1, sum) : 0.0f;
    b.p[2] = sum > 0.0f ? dvd(w2, sum) : 0.0f;
    b.p[3] = sum > 0.0f ? dvd(w3, sum) : 0.0f;
}

// bsdf_eval: f(v, l) without the delta lobes, and the density bsdf_sample draws l with
__device__ __forceinline__ V3 bsdf_eval(Bsdf &b, V3 n, V3 v, V3 l, float &pdf) {
    V3 f = v3(0, 0, 0);
    pdf = 0.0f;
    float cv = vdot(v, n), cl = vdot(l, n);
    if (cv <= 0.0f) return f;
    bsdf_view(b, cv);
    const float m = b.metallic, t = b.transmission, a = b.alpha;
    if (cl > 0.0f) {
        V3 h = vnorm(vadd(v, l));
        float vh = clamp01(vdot(v, h)), nh = vdot(n, h);
        float fd = fresnel_dielectric(vh, b.eta);
        float kd = mul(sub(1.0f, m), sub(1.0f, t));
        if (kd > 0.0f) {
            kd = mul(kd, mul(mul(sub(1.0f, b.es_v), sub(1.0f, spec_albedo(b, cl))), b.kd_norm));
            f = vscale(b.base, dvd(kd, PIF));
            pdf = add(pdf, dvd(mul(b.p[BSDF_DIFF], cl), PIF));
        }
        if (!b.smooth && m > 0.0f) {
            float k = mul(mul(mul(m, sub(1.0f, b.e_v)), sub(1.0f, albedo_e(b, cl))), b.kms_norm);
            f = vadd(f, vscale(b.ms, k));
            pdf = add(pdf, dvd(mul(b.p[BSDF_MS], cl), PIF));
        }
        if (!b.smooth && nh > 0.0f) {
            float d = ggx_d(nh, ggx_s2(n, h), a);
            V3 fm = fresnel_metal(b.base, vh);
            float s = mul(d, ggx_vis(cv, cl, a));
            f = vadd(f, v3(mul(add(mul(sub(1.0f, m), fd), mul(m, fm.x)), s), mul(add(mul(sub(1.0f, m), fd), mul(m, fm.y)), s),
                           mul(add(mul(sub(1.0f, m), fd), mul(m, fm.z)), s)));
            pdf = add(pdf, dvd(mul(mul(b.p[BSDF_SPEC], ggx_g1(cv, a)), d), mul(4.0f, cv)));
        }
    } else if (cl < 0.0f && !b.smooth && t > 0.0f && m < 1.0f) {
        const float eta = b.eta;
        V3 h = vnorm(vneg(vadd(vscale(v, eta), l)));
        if (vdot(h, n) < 0.0f) h = vneg(h);
        float vh = vdot(v, h), lh = vdot(l, h), nh = vdot(n, h);
        float den = add(mul(eta, vh), lh);
        den = mul(den, den);
        if (vh > 0.0f && lh < 0.0f && nh > 0.0f && den > 1e-12f) {
            float fd = fresnel_dielectric(vh, eta);
            float d = ggx_d(nh, ggx_s2(n, h), a);
            float g2 = mul(mul(mul(ggx_vis(cv, cl, a), 4.0f), cv), -cl);
            float ft = dvd(mul(mul(mul(mul(vh, -lh), sub(1.0f, fd)), d), g2), mul(mul(cv, -cl), den));
            f = vscale(b.base, mul(mul(sub(1.0f, m), t), ft));
            pdf = dvd(mul(dvd(mul(mul(mul(b.p[BSDF_TRANS], ggx_g1(cv, a)), vh), d), cv), -lh), den);
        }
    }
    return f;
}

__device__ __forceinline__ int bsdf_pick(const Bsdf &b, float ul) {
    int lobe = 0;
    for (float acc = b.p[0]; lobe < BSDF_LOBES - 1 && (ul >= acc || b.p[lobe] <= 0.0f);) {
        ++lobe;
        acc = add(acc, b.p[lobe]);
    }
    return b.p[lobe] > 0.0f ? lobe : -1;
}
__device__ __forceinline__ bool bsdf_lobe_delta(const Bsdf &b, int lobe) {
    return b.smooth && (lobe == BSDF_SPEC || lobe == BSDF_TRANS);
}
__device__ __forceinline__ int bsdf_nlobes(const Bsdf &b) {
    return (b.p[0] > 0.0f) + (b.p[1] > 0.0f) + (b.p[2] > 0.0f) + (b.p[3] > 0.0f);
}
__device__ __forceinline__ bool bsdf_rough_part(const Bsdf &b) {
    return !b.smooth || mul(sub(1.0f, b.metallic), sub(1.0f, b.transmission)) > 0.0f;
}

__device__ __forceinline__ bool bsdf_sample_lobe(Bsdf &b, int lobe, V3 n, V3 v, float u1, float u2, BsdfSample &s) {
    float cv = vdot(v, n);
    if (cv <= 0.0f || lobe < 0) return false;
    bsdf_view(b, cv);
    if (b.p[lobe] <= 0.0f) return false;
    const float m = b.metallic, t = b.transmission;
    s.delta = 0;
    s.through = 0;
    if (b.smooth && (lobe == BSDF_SPEC || lobe == BSDF_TRANS)) {
        float fd = fresnel_dielectric(cv, b.eta);
        if (lobe == BSDF_SPEC) {
            V3 fm = fresnel_metal(b.base, cv);
            float k = dvd(1.0f, b.p[lobe]);
            s.l = vreflect(vneg(v), n);
            s.w = v3(mul(add(mul(sub(1.0f, m), fd), mul(m, fm.x)), k), mul(add(mul(sub(1.0f, m), fd), mul(m, fm.y)), k),
                     mul(add(mul(sub(1.0f, m), fd), mul(m, fm.z)), k));
        } else {
            if (fd >= 1.0f) return false;
            s.l = vrefract(vneg(v), n, b.eta);
            s.w = vscale(b.base, dvd(mul(mul(sub(1.0f, m), t), sub(1.0f, fd)), b.p[lobe]));
            s.through = 1;
        }
        s.pdf = 0.0f;
        s.delta = 1;
        return true;
    }
    V3 l;
    if (lobe == BSDF_DIFF || lobe == BSDF_MS) {
        l = cosine_hemisphere(n, u1, u2);
    } else {
        V3 h = ggx_sample_vndf(n, v, b.alpha, u1, u2);
        float vh = vdot(v, h);
        if (vh <= 0.0f) return false;
        if (lobe == BSDF_SPEC) l = vreflect(vneg(v), h);
        else {
            if (mul(mul(b.eta, b.eta), sub(1.0f, mul(vh, vh))) >= 1.0f) return false;
            l = vrefract(vneg(v), h, b.eta);
        }
    }
    if ((lobe == BSDF_TRANS) != (vdot(l, n) < 0.0f)) return false;
    float pdf;
    V3 f = bsdf_eval(b, n, v, l, pdf);
    if (!(pdf > 0.0f)) return false;
    s.l = l;
    s.w = vscale(f, dvd(fabsf(vdot(l, n)), pdf));
    s.pdf = pdf;
    s.through = vdot(l, n) < 0.0f;
    return true;
}

}  // namespace pt
}  // namespace lrc
