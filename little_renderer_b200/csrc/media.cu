// media.cu - participating media of a scene (lrc_scene_set_volumes): the reference's Volume
// (engine/scene/volume.h) uploaded with its derived majorants, restated from volume_update
// (engine/scene/volume.c:47-108) on the host in the float build's arithmetic: the largest density,
// the active box (the voxels with density, one voxel wider for the interpolation, clipped to the
// bounds) and each brick's majorant (the brick's voxels and one around). Delta tracking draws its
// random numbers per majorant segment, so these must be the reference's to the bit for exact-mode
// paths to follow the CPU's.
#include "api_internal.cuh"
#include <cmath>
#include <cstring>
#include <vector>

using namespace lrcapi;

namespace {

constexpr int kBrick = 8;   // VOLUME_BRICK

float fmax_r(float a, float b) { return b != b ? a : (a > b ? a : b); }   // r_fmax
float fmin_r(float a, float b) { return b != b ? a : (a < b ? a : b); }   // r_fmin

// volume_update for one volume: the VolDev fields but its pointers, and the brick majorants
void derive(const lrc_volume &v, lrc::VolDev &d, std::vector<float> &bricks) {
    for (int a = 0; a < 3; a++) {
        d.lo[a] = v.lo[a];
        d.hi[a] = v.hi[a];
        d.albedo[a] = v.albedo[a];
    }
    d.sigma_t = v.sigma_t;
    d.g = v.g;
    d.nx = v.nx; d.ny = v.ny; d.nz = v.nz;
    d.bnx = (v.nx + kBrick - 1) / kBrick;
    d.bny = (v.ny + kBrick - 1) / kBrick;
    d.bnz = (v.nz + kBrick - 1) / kBrick;
    const float *den = v.density;
    auto at = [&](int x, int y, int z) { return den[((size_t)z * v.ny + y) * v.nx + x]; };
    bricks.assign((size_t)d.bnx * d.bny * d.bnz, 0.0f);
    for (int bz = 0; bz < d.bnz; bz++)
        for (int by = 0; by < d.bny; by++)
            for (int bx = 0; bx < d.bnx; bx++) {
                int x0 = bx * kBrick - 1, x1 = bx * kBrick + kBrick, y0 = by * kBrick - 1, y1 = by * kBrick + kBrick;
                int z0 = bz * kBrick - 1, z1 = bz * kBrick + kBrick;
                if (x0 < 0) x0 = 0;
                if (y0 < 0) y0 = 0;
                if (z0 < 0) z0 = 0;
                if (x1 > v.nx - 1) x1 = v.nx - 1;
                if (y1 > v.ny - 1) y1 = v.ny - 1;
                if (z1 > v.nz - 1) z1 = v.nz - 1;
                float m = 0;
                for (int z = z0; z <= z1; z++)
                    for (int y = y0; y <= y1; y++)
                        for (int x = x0; x <= x1; x++)
                            if (at(x, y, z) > m) m = at(x, y, z);
                bricks[((size_t)bz * d.bny + by) * d.bnx + bx] = m;
            }
    int x0 = v.nx, y0 = v.ny, z0 = v.nz, x1 = -1, y1 = -1, z1 = -1;
    float mx = 0;
    for (int z = 0; z < v.nz; z++)
        for (int y = 0; y < v.ny; y++)
            for (int x = 0; x < v.nx; x++) {
                const float q = at(x, y, z);
                if (!(q > 0)) continue;
                if (q > mx) mx = q;
                x0 = std::min(x0, x); x1 = std::max(x1, x);
                y0 = std::min(y0, y); y1 = std::max(y1, y);
                z0 = std::min(z0, z); z1 = std::max(z1, z);
            }
    d.max_density = mx;
    if (x1 < 0) {                                    // empty: a box nothing can enter
        for (int a = 0; a < 3; a++) {
            d.alo[a] = 1.0f;
            d.ahi[a] = -1.0f;
        }
        return;
    }
    // volume_voxel_center: lo + (i + 0.5) * size / n, each operation rounded in float
    const int n[3] = {v.nx, v.ny, v.nz}, i0[3] = {x0, y0, z0}, i1[3] = {x1, y1, z1};
    for (int a = 0; a < 3; a++) {
        const volatile float size = v.hi[a] - v.lo[a];
        const volatile float vox = size / (float)n[a];
        volatile float c0 = ((float)i0[a] + 0.5f) * size;
        c0 = c0 / (float)n[a];
        c0 = v.lo[a] + c0;
        volatile float c1 = ((float)i1[a] + 0.5f) * size;
        c1 = c1 / (float)n[a];
        c1 = v.lo[a] + c1;
        const volatile float lo = c0 - vox, hi = c1 + vox;
        d.alo[a] = fmax_r(lo, v.lo[a]);
        d.ahi[a] = fmin_r(hi, v.hi[a]);
    }
}

bool valid(const lrc_volume &v) {
    if (v.nx < 1 || v.ny < 1 || v.nz < 1 || !v.density) return false;
    if ((uint64_t)v.nx * v.ny * v.nz > (1ull << 30)) return false;
    for (int a = 0; a < 3; a++)
        if (!std::isfinite(v.lo[a]) || !std::isfinite(v.hi[a]) || !(v.lo[a] < v.hi[a]) || !std::isfinite(v.albedo[a]))
            return false;
    if (!std::isfinite(v.sigma_t) || v.sigma_t < 0 || !(v.g > -1.0f && v.g < 1.0f)) return false;
    const size_t n = (size_t)v.nx * v.ny * v.nz;
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(v.density[i]) || v.density[i] < 0) return false;
    return true;
}

}  // namespace

extern "C" {

int lrc_volume_majorants(const lrc_volume *v, float *max_density, float *active6, float *brick_max) {
    if (!v || !max_density || !active6 || !valid(*v)) return LRC_E_INVALID;
    lrc::VolDev d{};
    std::vector<float> bricks;
    derive(*v, d, bricks);
    *max_density = d.max_density;
    for (int a = 0; a < 3; a++) {
        active6[a] = d.alo[a];
        active6[3 + a] = d.ahi[a];
    }
    if (brick_max) std::memcpy(brick_max, bricks.data(), bricks.size() * 4);
    return LRC_OK;
}

int lrc_scene_set_volumes(lrc_scene *s, const lrc_volume *vols, uint32_t n) {
    if (!s || n > (uint32_t)lrc::kMaxVolumes || (n && !vols)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    for (uint32_t i = 0; i < n; i++)
        if (!valid(vols[i]))
            return fail(c, LRC_E_INVALID, "a volume needs a grid >= 1 voxel, finite bounds lo < hi, finite density >= 0, "
                                          "sigma_t >= 0 and g in (-1, 1)");
    DeviceGuard g(c->device);
    std::vector<lrc::VolDev> dev(n);
    std::vector<std::vector<float>> bricks(n);
    size_t bytes = 0;
    std::vector<size_t> off_den(n), off_br(n);
    for (uint32_t i = 0; i < n; i++) {
        derive(vols[i], dev[i], bricks[i]);
        off_den[i] = bytes;
        bytes += al((size_t)vols[i].nx * vols[i].ny * vols[i].nz * 4);
        off_br[i] = bytes;
        bytes += al(bricks[i].size() * 4);
    }
    cudaError_t e = cudaStreamSynchronize(c->st);     // (the old buffers may still be read)
    if (!e && s->d_vols) e = cudaFree(s->d_vols);
    s->d_vols = nullptr;
    s->nvol = 0;
    if (!e && n) e = cudaMalloc(&s->d_vols, al(n * sizeof(lrc::VolDev)) + bytes);
    if (e) return cuda_status(c, e, "volumes");
    if (!n) return LRC_OK;
    char *base = static_cast<char *>(s->d_vols), *data = base + al(n * sizeof(lrc::VolDev));
    for (uint32_t i = 0; i < n && !e; i++) {
        dev[i].density = reinterpret_cast<const float *>(data + off_den[i]);
        dev[i].brick_max = reinterpret_cast<const float *>(data + off_br[i]);
        e = cudaMemcpy(data + off_den[i], vols[i].density, (size_t)vols[i].nx * vols[i].ny * vols[i].nz * 4,
                       cudaMemcpyHostToDevice);
        if (!e) e = cudaMemcpy(data + off_br[i], bricks[i].data(), bricks[i].size() * 4, cudaMemcpyHostToDevice);
    }
    if (!e) e = cudaMemcpy(base, dev.data(), n * sizeof(lrc::VolDev), cudaMemcpyHostToDevice);
    if (e) return cuda_status(c, e, "volumes");
    s->nvol = n;
    return LRC_OK;
}

}  // extern "C"
