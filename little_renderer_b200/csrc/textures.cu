// textures.cu - the materials' textures of a scene (lrc_scene_set_texmaps) and the world triangles'
// texture coordinates (lrc_scene_set_texcoords): the reference's Scene.texmaps (TexMap level 0),
// Triangle.t with Scene.uvs / .tangents (engine/scene/scene.h:134-140, 279-281), and the sRGB table
// texture.c makes (texmap_srgb_table, texture.c:64-73: the sRGB transfer curve per byte).
#include "api_internal.cuh"
#include <cmath>
#include <vector>

using namespace lrcapi;

extern "C" {

void lrc_srgb_table(float *out256) {
    // the sRGB curve per byte as the float build computes it: its constants are single precision
    // (-fsingle-precision-constant), i / 255 a float division, the rest in double
    for (int i = 0; i < 256; i++) {
        const double v = (double)((float)i / 255.0f);
        const double lim = (double)0.04045f, slope = (double)12.92f, a = (double)0.055f, b = (double)1.055f,
                     gamma = (double)2.4f;
        out256[i] = (float)(v <= lim ? v / slope : std::pow((v + a) / b, gamma));
    }
}

int lrc_scene_set_texmaps(lrc_scene *s, const lrc_texmap *t, uint32_t n) {
    if (!s || n > 255 || (n && !t)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    size_t texels = 0;
    for (uint32_t i = 0; i < n; i++) {
        const lrc_texmap &m = t[i];
        if (m.w < 1 || m.h < 1 || !m.rgba || m.wrap_u < 0 || m.wrap_u > 2 || m.wrap_v < 0 || m.wrap_v > 2 ||
            (uint64_t)m.w * m.h > (1ull << 28))
            return fail(c, LRC_E_INVALID, "a texmap needs w, h >= 1, its texels and wraps 0 (repeat), 1 (clamp) or 2 (mirror)");
        texels += (size_t)m.w * m.h;
    }
    DeviceGuard g(c->device);
    cudaError_t e = cudaStreamSynchronize(c->st);      // (the old buffer may still be read)
    if (!e && s->d_tex) e = cudaFree(s->d_tex);
    s->d_tex = nullptr;
    s->ntex = 0;
    if (e) return cuda_status(c, e, "texmaps");
    if (!n) return LRC_OK;
    std::vector<uint32_t> table(4 * (size_t)n);
    size_t at = 0;
    for (uint32_t i = 0; i < n; i++) {
        table[4 * i] = (uint32_t)t[i].w;
        table[4 * i + 1] = (uint32_t)t[i].h;
        table[4 * i + 2] = (t[i].srgb ? 1u : 0u) | (uint32_t)t[i].wrap_u << 1 | (uint32_t)t[i].wrap_v << 3;
        table[4 * i + 3] = (uint32_t)at;
        at += (size_t)t[i].w * t[i].h;
    }
    // the sRGB curve per byte as the float build computes it: its constants are single precision
    // (-fsingle-precision-constant), i / 255 a float division, the rest in double
    float lut[256];
    lrc_srgb_table(lut);
    const size_t tb = al(table.size() * 4), lb = al(256 * 4);
    e = cudaMalloc(&s->d_tex, tb + lb + texels * 4);
    char *base = static_cast<char *>(s->d_tex);
    if (!e) e = cudaMemcpy(base, table.data(), table.size() * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(base + tb, lut, sizeof lut, cudaMemcpyHostToDevice);
    at = 0;
    for (uint32_t i = 0; i < n && !e; i++) {
        e = cudaMemcpy(base + tb + lb + at * 4, t[i].rgba, (size_t)t[i].w * t[i].h * 4, cudaMemcpyHostToDevice);
        at += (size_t)t[i].w * t[i].h;
    }
    if (e) return cuda_status(c, e, "texmaps");
    s->ntex = n;
    s->tex_lut_off = tb;
    s->texel_off = tb + lb;
    return LRC_OK;
}

int lrc_scene_set_texcoords(lrc_scene *s, const int32_t *tri_uv, uint32_t ntris, const float *uvs, const float *tangents,
                            uint32_t nuv) {
    if (!s || (ntris && !tri_uv) || (nuv && (!uvs || !tangents))) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = cudaStreamSynchronize(c->st);
    if (!e && s->d_uv) e = cudaFree(s->d_uv);
    s->d_uv = nullptr;
    s->uv_tris = 0;
    s->nuv = 0;
    if (e) return cuda_status(c, e, "texture coordinates");
    if (!ntris) return LRC_OK;
    const size_t a = al((size_t)ntris * 12), b = al((size_t)nuv * 8);
    e = cudaMalloc(&s->d_uv, a + b + (size_t)nuv * 16 + 256);
    char *base = static_cast<char *>(s->d_uv);
    if (!e) e = cudaMemcpy(base, tri_uv, (size_t)ntris * 12, cudaMemcpyHostToDevice);
    if (!e && nuv) e = cudaMemcpy(base + a, uvs, (size_t)nuv * 8, cudaMemcpyHostToDevice);
    if (!e && nuv) e = cudaMemcpy(base + a + b, tangents, (size_t)nuv * 16, cudaMemcpyHostToDevice);
    if (e) return cuda_status(c, e, "texture coordinates");
    s->uv_tris = ntris;
    s->nuv = nuv;
    s->uv_off = a;
    s->tangent_off = a + b;
    return LRC_OK;
}

}  // extern "C"
