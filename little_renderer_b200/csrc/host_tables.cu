// host_tables.cu - what the path tracer reads besides the scene, for callers that do not pass it
// (the reference's engine passes its own: blue_noise_mask() and gpu_bsdf_tables(), as
// trace_gpu.c:523-532 uploads them). Both are made here by the reference's published methods:
//
//   default_blue_noise   the 64 x 64 void-and-cluster mask (Ulichney 1993) as engine/base/sampler.c
//                        makes it: a Gaussian energy (sigma 1.9, wrapping) over the tile, a tenth of
//                        the points placed at random by PCG32 (seed 0x5eedb10e, stream 7) and relaxed,
//                        ranked by removing the most crowded, the rest ranked by filling the largest
//                        void; float energies, first index on ties. The same ranks as the reference's.
//   default_bsdf_tables  the white GGX lobe's directional albedo E(mu, r) and its Schlick-weighted
//                        twin B (Kulla & Conty 2017; Karis 2013), integrated over the visible normals
//                        (Heitz 2018) with 128 x 128 stratified samples per node on 32 x 32 nodes,
//                        their cosine-weighted means by the trapezoid rule on a 2049-point resampling,
//                        rounded to 6 decimals, as tools/gen_brdf_tables.py made scene/brdf_tables.h.
#include "lrc_internal.cuh"
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace lrc {

namespace {

struct HostPcg {
    uint64_t state, inc;
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((0u - rot) & 31u));
    }
    HostPcg(uint64_t seed, uint64_t stream) {
        state = 0;
        inc = (stream << 1u) | 1u;
        next();
        state += seed;
        next();
    }
};

constexpr int BN = 64, BN_N = BN * BN;

void bn_add(float *energy, const float *kern, int p, float sign) {
    const int px = p % BN, py = p / BN;
    for (int y = 0; y < BN; y++) {
        const float *k = kern + ((y - py) & (BN - 1)) * BN;
        float *e = energy + y * BN;
        for (int x = 0; x < BN; x++) e[x] += sign * k[(x - px) & (BN - 1)];
    }
}

int bn_pick(const float *energy, const unsigned char *on, int want_on, bool want_max) {
    int best = -1;
    for (int i = 0; i < BN_N; i++) {
        if (on[i] != want_on) continue;
        if (best < 0 || (want_max ? energy[i] > energy[best] : energy[i] < energy[best])) best = i;
    }
    return best;
}

}  // namespace

void default_blue_noise(uint16_t *rank) {
    std::vector<float> kern(BN_N), energy(BN_N, 0.0f), e0(BN_N);
    std::vector<unsigned char> on(BN_N, 0), on0(BN_N);
    // sigma 1.9 as the float build has it (-fsingle-precision-constant makes the literal a float)
    const double sigma = (double)1.9f;
    for (int y = 0; y < BN; y++)
        for (int x = 0; x < BN; x++) {
            int dx = x < BN / 2 ? x : x - BN, dy = y < BN / 2 ? y : y - BN;
            kern[y * BN + x] = (float)std::exp(-(dx * dx + dy * dy) / (2 * sigma * sigma));
        }
    HostPcg rng(0x5eedb10eull, 7);
    const int ones = BN_N / 10;
    for (int n = 0; n < ones;) {
        int p = (int)(rng.next() % BN_N);
        if (on[p]) continue;
        on[p] = 1;
        bn_add(energy.data(), kern.data(), p, 1.0f);
        n++;
    }
    for (int it = 0; it < BN_N; it++) {                 // relax: the most crowded to the largest void
        int c = bn_pick(energy.data(), on.data(), 1, true);
        on[c] = 0;
        bn_add(energy.data(), kern.data(), c, -1.0f);
        int v = bn_pick(energy.data(), on.data(), 0, false);
        on[v] = 1;
        bn_add(energy.data(), kern.data(), v, 1.0f);
        if (v == c) break;
    }
    on0 = on;
    e0 = energy;
    for (int r = ones - 1; r >= 0; r--) {               // the first tenth's ranks: most crowded out first
        int c = bn_pick(energy.data(), on.data(), 1, true);
        on[c] = 0;
        bn_add(energy.data(), kern.data(), c, -1.0f);
        rank[c] = (uint16_t)r;
    }
    on = on0;
    energy = e0;
    for (int r = ones; r < BN_N; r++) {                 // the rest: each into the largest void
        int v = bn_pick(energy.data(), on.data(), 0, false);
        on[v] = 1;
        bn_add(energy.data(), kern.data(), v, 1.0f);
        rank[v] = (uint16_t)r;
    }
}

namespace {

double g1(double c, double a) {
    c = std::fabs(c);
    return 2 * c / (c + std::sqrt(a * a + (1 - a * a) * c * c));
}
double vis(double cv, double cl, double a) {
    double a2 = a * a;
    double d = cl * std::sqrt(cv * cv * (1 - a2) + a2) + cv * std::sqrt(cl * cl * (1 - a2) + a2);
    return 0.5 / d;
}

// E and B of a white GGX lobe of roughness r seen at cosine mu: the mean, over microfacet normals
// drawn from the visible normals, of G2 / G1 (the reflection's weight; 0 below the horizon)
void albedo(double mu, double r, double &E, double &B) {
    const int S = 128;
    const double a = std::max(r * r, 1e-4);
    mu = std::max(mu, 1e-4);
    const double v[3] = {std::sqrt(1 - mu * mu), 0.0, mu};
    double vh[3] = {a * v[0], a * v[1], v[2]};
    double ln = std::sqrt(vh[0] * vh[0] + vh[1] * vh[1] + vh[2] * vh[2]);
    for (double &x : vh) x /= ln;
    double se = 0, sb = 0;
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) {
            double u1 = (i + 0.5) / S, u2 = (j + 0.5) / S;
            double phi = 2 * M_PI * u1;
            double z = (1 - u2) * (1 + vh[2]) - vh[2];
            double st = std::sqrt(std::max(0.0, 1 - z * z));
            double hs[3] = {st * std::cos(phi) + vh[0], st * std::sin(phi) + vh[1], z + vh[2]};
            double h[3] = {a * hs[0], a * hs[1], std::max(hs[2], 0.0)};
            double hn = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
            for (double &x : h) x /= hn;
            double vdh = h[0] * v[0] + h[1] * v[1] + h[2] * v[2];
            double cl = 2 * vdh * h[2] - v[2];
            double w = cl > 0 ? vis(mu, std::max(cl, 1e-9), a) * 4 * mu * std::max(cl, 0.0) / g1(mu, a) : 0.0;
            double c = std::min(std::max(vdh, 0.0), 1.0);
            se += w;
            sb += w * std::pow(1 - c, 5);
        }
    E = se / (S * S);
    B = sb / (S * S);
}

// 2 * integral of f(mu) mu dmu, f linear between the 32 nodes, trapezoid rule on 2049 points
double cosine_mean(const double *f) {
    const int N = 32, F = 2049;
    double sum = 0, prev = 0;
    for (int k = 0; k < F; k++) {
        double x = (double)k / (F - 1);
        double pos = x * (N - 1);
        int i = std::min((int)pos, N - 2);
        double y = f[i] + (pos - i) * (f[i + 1] - f[i]);
        double g = y * x;
        if (k) sum += (g + prev) * 0.5 / (F - 1);
        prev = g;
    }
    return 2 * sum;
}

float six(double x) {
    char buf[32];
    snprintf(buf, sizeof(buf), "%.6f", x);
    return strtof(buf, nullptr);
}

}  // namespace

void default_bsdf_tables(float *out) {
    const int N = 32;
    std::vector<double> E(N * N), B(N * N);
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) albedo((double)i / (N - 1), (double)j / (N - 1), E[j * N + i], B[j * N + i]);
    for (int k = 0; k < N * N; k++) {
        out[k] = six(E[k]);
        out[1024 + k] = six(B[k]);
    }
    for (int j = 0; j < N; j++) {
        out[2048 + j] = six(cosine_mean(&E[j * N]));
        out[2080 + j] = six(cosine_mean(&B[j * N]));
    }
}

// The sky's importance-sampling tables, as engine/scene/env.c makes them (make_weights :125-162,
// prepare_base :341-363, pixel_prob :164-167): a pixel's weight is the largest luminance of its
// 3 x 3 neighbourhood (wrapping across, stopping at the poles) times its row's sin(theta); each row's
// cumulative distribution and the rows' are summed in double and stored in float; a pixel's
// probability is its weight over the whole sum.
bool env_tables(const float *rgb, int w, int h, float *marg, float *cond, float *prob) {
    std::vector<float> lum((size_t)w * h), wmax((size_t)w * h);
    std::vector<float> row_sin(h);
    for (int y = 0; y < h; y++) {
        const float *p = rgb + 3 * (size_t)y * w;
        float *l = lum.data() + (size_t)y * w, *o = wmax.data() + (size_t)y * w;
        for (int x = 0; x < w; x++) {
            const float *c = p + 3 * x;
            float a = 0.2126f * c[0];
            float b = 0.7152f * c[1];
            float d = 0.0722f * c[2];
            l[x] = (a + b) + d;
        }
        for (int x = 0; x < w; x++) {
            float a = l[x == 0 ? w - 1 : x - 1], b = l[x], c = l[x + 1 == w ? 0 : x + 1];
            float m = a > b ? a : b;
            o[x] = m > c ? m : c;
        }
        float arg = ((float)y + 0.5f) * 3.14159265358979323846f;
        row_sin[y] = sinf(arg / (float)h);
    }
    lum = wmax;
    for (int y = 0; y < h; y++) {
        const float *a = lum.data() + (size_t)(y > 0 ? y - 1 : y) * w, *b = lum.data() + (size_t)y * w;
        const float *c = lum.data() + (size_t)(y + 1 < h ? y + 1 : y) * w;
        float *o = wmax.data() + (size_t)y * w;
        for (int x = 0; x < w; x++) {
            float m = a[x] > b[x] ? a[x] : b[x];
            m = m > c[x] ? m : c[x];
            o[x] = m > 0 ? m : 0;
        }
    }
    auto weight = [&](int x, int y) { return wmax[(size_t)y * w + x] * row_sin[y]; };
    std::vector<double> rows(h);
    double sum = 0;
    for (int y = 0; y < h; y++) {
        float *c = cond + (size_t)y * (w + 1);
        double acc = 0;
        c[0] = 0;
        for (int x = 0; x < w; x++) {
            acc += weight(x, y);
            c[x + 1] = (float)acc;
        }
        rows[y] = acc;
        for (int x = 1; x <= w; x++) c[x] = acc > 0 ? (float)(c[x] / acc) : (float)x / w;
        c[w] = 1;
        sum += acc;
    }
    double acc = 0;
    marg[0] = 0;
    for (int y = 0; y < h; y++) {
        acc += rows[y];
        marg[y + 1] = sum > 0 ? (float)(acc / sum) : (float)(y + 1) / h;
    }
    marg[h] = 1;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) prob[(size_t)y * w + x] = sum > 0 ? (float)(weight(x, y) / sum) : 0.0f;
    return sum > 0;
}

}  // namespace lrc

extern "C" int lrc_sky_tables(const float *rgb, int32_t w, int32_t h, float *marg, float *cond, float *prob) {
    if (!rgb || w <= 0 || h <= 0 || !marg || !cond || !prob) return 0;
    return lrc::env_tables(rgb, w, h, marg, cond, prob) ? 1 : 0;
}

extern "C" void lrc_default_blue_noise(uint16_t *out) {
    if (out) lrc::default_blue_noise(out);
}
extern "C" void lrc_default_bsdf_tables(float *out) {
    if (out) lrc::default_bsdf_tables(out);
}
