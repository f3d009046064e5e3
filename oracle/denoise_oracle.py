"""TEST INFRASTRUCTURE (the oracle): a numpy restatement of the reference's GPU denoiser
(engine/gpu/denoise_gpu.c: the `prep` and `atrous` passes of engine/gpu/shaders/trace/denoise.wgsl),
which has no CPU counterpart in the reference. Parity unpinned: the reference's WGSL cannot run here
(no graphics stack), so this restatement is checked only against the CUDA kernels it restates.

Planes: (4, h, w, 4) float32 as the reference's path tracer keeps them (denoise.wgsl:8, trace.wgsl
gbuf): 0 the samples' sum and count, 1 the luminance moments (sum l, sum l^2), 2 the guide's normal
and distance, 3 its albedo and kind. Values pass between passes as halves, as the shader packs them
(put_iv, denoise.wgsl:16-19); the guide's normal through its octahedral snorm16 code (oct / unoct,
:25-37). Nothing on the product path imports this file."""
import numpy as np

F = np.float32


def hash32(x):
    """lowbias32 (util.wgsl hash32) on uint32 arrays."""
    x = np.asarray(x, np.uint32).copy()
    with np.errstate(over="ignore"):
        x ^= x >> np.uint32(16)
        x *= np.uint32(0x7FEB352D)
        x ^= x >> np.uint32(15)
        x *= np.uint32(0x846CA68B)
        x ^= x >> np.uint32(16)
    return x


def luma(c):
    return F(0.2126) * c[..., 0] + F(0.7152) * c[..., 1] + F(0.0722) * c[..., 2]


def gkind(w):
    return w - F(4) * np.floor(w * F(0.25))


def halves(x):
    """f32 -> f16 -> f32 (pack2x16float then unpack)."""
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


def put_iv(c, v):
    """irradiance (each channel at most 6e4) and variance (-1 .. 6e4) as halves: (.., 4)."""
    out = np.empty(c.shape[:-1] + (4,), np.float32)
    out[..., :3] = halves(np.minimum(c, F(6e4)))
    out[..., 3] = halves(np.minimum(np.maximum(v, F(-1)), F(6e4)))
    return out


def snorm16(v):
    return np.rint(np.clip(v, F(-1), F(1)) * F(32767)).astype(np.int16)


def oct_code(n):
    s = np.maximum(np.abs(n[..., 0]) + np.abs(n[..., 1]) + np.abs(n[..., 2]), F(1e-6))
    px, py = n[..., 0] / s, n[..., 1] / s
    sx = np.where(px >= 0, F(1), F(-1))
    sy = np.where(py >= 0, F(1), F(-1))
    neg = n[..., 2] < 0
    qx = np.where(neg, (F(1) - np.abs(py)) * sx, px)
    qy = np.where(neg, (F(1) - np.abs(px)) * sy, py)
    return snorm16(qx), snorm16(qy)


def unoct(ax, ay):
    ex = np.maximum(ax.astype(np.float32) / F(32767), F(-1))
    ey = np.maximum(ay.astype(np.float32) / F(32767), F(-1))
    z = F(1) - np.abs(ex) - np.abs(ey)
    t = np.maximum(-z, F(0))
    x = ex + np.where(ex >= 0, -t, t)
    y = ey + np.where(ey >= 0, -t, t)
    ln = np.sqrt(x * x + y * y + z * z)
    return np.stack([x / ln, y / ln, z / ln], -1)


def irradiance(px):
    a, g = px[0], px[3]
    mean = a[..., :3] / np.maximum(a[..., 3:4], F(1))
    surf = (gkind(g[..., 3]) == 0)[..., None]
    return np.where(surf, mean / np.maximum(g[..., :3], F(1e-3)), mean)


def prep(px):
    """prep (denoise.wgsl:58-105): (image (h, w, 4): irradiance + variance as halves, guide dict)."""
    px = np.asarray(px, np.float32)
    H, W = px.shape[1:3]
    a, m, n, g = px[0], px[1], px[2], px[3]
    gk = gkind(g[..., 3])
    e = np.where(gk == 0, n[..., 3], np.where(gk == 1, F(-2e38), -(n[..., 3] + F(1))))
    kind = np.where(e >= 0, 0, np.where(e < F(-1e37), 1, 2))
    guide = {"n": unoct(*oct_code(n[..., :3])), "z": np.where(e >= 0, e, -e - F(1)).astype(np.float32),
             "kind": kind}
    irr = irradiance(px)
    cnt = a[..., 3]
    el = m[..., 0] / np.where(cnt > 0, cnt, F(1))
    v_own = np.maximum(m[..., 1] / np.where(cnt > 0, cnt, F(1)) - el * el, F(0)) / np.where(cnt > 0, cnt, F(1))
    # fewer than 4 samples: the spread of the 7 x 7 neighbours' luminance on the same surface
    lq = luma(irr)
    s1 = np.zeros((H, W), np.float32)
    s2 = np.zeros((H, W), np.float32)
    c = np.zeros((H, W), np.float32)
    ys, xs = np.mgrid[0:H, 0:W]
    for dy in range(-3, 4):
        for dx in range(-3, 4):
            qy, qx = ys + dy, xs + dx
            ok = (qx >= 0) & (qy >= 0) & (qx < W) & (qy < H)
            qyc, qxc = np.clip(qy, 0, H - 1), np.clip(qx, 0, W - 1)
            ok &= (a[qyc, qxc, 3] != 0) & (gkind(g[qyc, qxc, 3]) == gk)
            nd = (n[qyc, qxc, 0] * n[..., 0] + n[qyc, qxc, 1] * n[..., 1]) + n[qyc, qxc, 2] * n[..., 2]
            ok &= ~((gk == 0) & (nd < F(0.9)))
            l = lq[qyc, qxc]
            s1 += np.where(ok, l, F(0))
            s2 += np.where(ok, l * l, F(0))
            c += np.where(ok, F(1), F(0))
    with np.errstate(invalid="ignore", divide="ignore"):
        en = s1 / c
        v_nb = np.maximum(s2 / c - en * en, F(0))
    v = np.where(cnt >= 4, v_own, v_nb)
    v = np.where(gk == 1, F(0), v)
    irr = np.where((gk == 1)[..., None], irr, irr)
    out = put_iv(irr, v)
    empty = cnt == 0
    out[empty] = put_iv(np.zeros(3, np.float32), F(-1))
    return out, guide


def b3(i):
    return F(0.375) if i == 2 else (F(0.25) if i in (1, 3) else F(0.0625))


def atrous(px, src, guide, step, last, sigma_l=4.0, sigma_z=1.0):
    """One a-trous pass (denoise.wgsl:107-205): the next image (halves), or the output image
    (h, w, 4) on the last pass."""
    px = np.asarray(px, np.float32)
    H, W = src.shape[:2]
    sigma_l, sigma_z = F(sigma_l), F(sigma_z)
    ys, xs = np.mgrid[0:H, 0:W]
    k = (ys * W + xs).astype(np.uint32)
    gpn, gpz, gpk = guide["n"], guide["z"], guide["kind"]
    cw = src[..., 3]
    passthrough = (cw < 0) | (gpk == 1)
    # the variance blurred 3 x 3
    v = np.zeros((H, W), np.float32)
    vw = np.zeros((H, W), np.float32)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            qy, qx = np.clip(ys + dy, 0, H - 1), np.clip(xs + dx, 0, W - 1)
            sw = src[qy, qx, 3]
            w = (F(0.25) if dx else F(0.5)) * (F(0.25) if dy else F(0.5))
            v += np.where(sw < 0, F(0), w * sw)
            vw += np.where(sw < 0, F(0), w)
    v = v / np.maximum(vw, F(1e-6))
    lp = luma(src)
    surface = gpk == 0
    zl = gpz[ys, np.maximum(xs - 1, 0)]
    zr = gpz[ys, np.minimum(xs + 1, W - 1)]
    zd = gpz[np.maximum(ys - 1, 0), xs]
    zu = gpz[np.minimum(ys + 1, H - 1), xs]
    gx = np.where(surface, np.minimum(np.abs(gpz - zl), np.abs(gpz - zr)), F(0))
    gy = np.where(surface, np.minimum(np.abs(gpz - zd), np.abs(gpz - zu)), F(0))
    with np.errstate(over="ignore"):
        seed = hash32((k * np.uint32(0x9E3779B9)) ^ np.uint32((step * 0x85EBCA6B) & 0xFFFFFFFF))
    jit = step // 2
    jn = np.uint32(2 * jit + 1)
    sums = np.zeros((H, W, 3), np.float32)
    vsum = np.zeros((H, W), np.float32)
    wsum = np.zeros((H, W), np.float32)
    for j in range(5):
        for i in range(5):
            ox = np.full((H, W), (i - 2) * step, np.int64)
            oy = np.full((H, W), (j - 2) * step, np.int64)
            if jit > 0 and (i != 2 or j != 2):
                seed = hash32(seed)
                with np.errstate(over="ignore"):
                    ox += (((seed & np.uint32(0xFFFF)) * jn) >> np.uint32(16)).astype(np.int64) - jit
                    oy += (((seed >> np.uint32(16)) * jn) >> np.uint32(16)).astype(np.int64) - jit
            qx, qy = xs + ox, ys + oy
            ok = (qx >= 0) & (qy >= 0) & (qx < W) & (qy < H)
            qxc, qyc = np.clip(qx, 0, W - 1), np.clip(qy, 0, H - 1)
            s = src[qyc, qxc]
            w = np.full((H, W), b3(i) * b3(j), np.float32)
            centre = (qx == xs) & (qy == ys)
            gqk = gpk[qyc, qxc]
            ok &= centre | ~((s[..., 3] < 0) | (gqk != gpk))
            with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
                wl = np.exp(-np.abs(lp - luma(s)) / (sigma_l * np.sqrt(np.maximum(v, s[..., 3])) + F(1e-6)))
                gqn = gpn[qyc, qxc]
                wn = np.maximum((gpn[..., 0] * gqn[..., 0] + gpn[..., 1] * gqn[..., 1]) + gpn[..., 2] * gqn[..., 2], F(0))
                for _ in range(7):
                    wn = wn * wn
                expect = gx * np.abs(ox).astype(np.float32) + gy * np.abs(oy).astype(np.float32)
                wz = np.exp(-np.abs(gpz - gpz[qyc, qxc]) / (sigma_z * expect + F(1e-3) * gpz + F(1e-6)))
            wt = np.where(centre, w, w * wl * np.where(surface, wn * wz, F(1)))
            wt = np.where(ok, wt, F(0))
            sums += wt[..., None] * s[..., :3]
            vsum += wt * wt * s[..., 3]
            wsum += wt
    with np.errstate(invalid="ignore", divide="ignore"):
        o = sums / wsum[..., None]
    if last:
        out = np.zeros((H, W, 4), np.float32)
        al = px[3][..., :3]
        out[..., :3] = np.where(surface[..., None], o * al, o)
        out[..., 3] = 1
        out[passthrough] = np.concatenate([src[..., :3], np.ones((H, W, 1), np.float32)], -1)[passthrough]
        out[cw < 0] = 0
        return out
    with np.errstate(invalid="ignore", divide="ignore"):
        nxt = put_iv(o, vsum / (wsum * wsum))
    nxt[passthrough] = src[passthrough]
    return nxt


def denoise(px, passes=5):
    """prep, then `passes` a-trous passes (holes 1, 2, 4, ...): the image (h, w, 4)."""
    img, guide = prep(px)
    for i in range(1, passes + 1):
        img = atrous(px, img, guide, 1 << (i - 1), i == passes)
    return img
