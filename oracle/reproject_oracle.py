"""TEST INFRASTRUCTURE (the oracle): a numpy restatement of the reference's reprojection of a new
image's samples from the previous image's (engine/gpu/shaders/trace/trace_reproject.wgsl `main`,
without temporal gradients and not an edit's move: dims.w = 0, ext.z = 0), which has no CPU
counterpart in the reference. Parity unpinned: the reference's WGSL cannot run here.

Planes (4, h, w, 4) float32 as the path tracer keeps them: 0 samples' sum and count, 1 moments,
2 the guide's normal and distance, 3 its albedo and kind. Cameras: (origin, upper_left,
horizontal, vertical) as 4 x 3 floats. Nothing on the product path imports this file."""
import numpy as np

F = np.float32


def gkind(w):
    return w - F(4) * np.floor(w * F(0.25))


def old_place(oc, nc, W, H, g2):
    """Where each new pixel's surface was in the old image: (fx, fy, distance, in front)."""
    y, x = np.mgrid[0:H, 0:W].astype(np.float32)
    no, nul, nh, nv = (np.asarray(a, np.float32) for a in nc)
    oo, oul, oh, ov = (np.asarray(a, np.float32) for a in oc)
    d = nul + nh * ((x + F(0.5)) / F(W))[..., None] - nv * ((y + F(0.5)) / F(H))[..., None] - no
    d = d / np.sqrt((d * d).sum(-1, keepdims=True))
    far = g2[..., 3] > F(1e29)
    p = no + d * np.where(far, F(1e6), g2[..., 3])[..., None]
    f = oul - oo
    c = f + F(0.5) * oh - F(0.5) * ov
    q0 = p - oo
    den = (q0 * c).sum(-1)
    ok = den > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        q = q0 * (np.dot(c, c) / den)[..., None] - f
    fx = (q * oh).sum(-1) / np.dot(oh, oh) * F(W) - F(0.5)
    fy = -(q * ov).sum(-1) / np.dot(ov, ov) * F(H) - F(0.5)
    return np.where(ok, fx, 0), np.where(ok, fy, 0), np.where(ok, np.sqrt((q0 * q0).sum(-1)), 0), ok


def reproject(old, cur, oc, nc, history):
    """cur's planes 0 and 1 from old's (cur's planes 2 and 3: the new guide). Returns the new
    (4, h, w, 4) planes."""
    old = np.asarray(old, np.float32)
    cur = np.array(cur, np.float32)
    H, W = cur.shape[1:3]
    g2, g3 = cur[2], cur[3]
    fx, fy, dist, front = old_place(oc, nc, W, H, g2)
    x0, y0 = np.floor(fx), np.floor(fy)
    a0 = np.zeros((H, W, 4), np.float32)
    a1 = np.zeros((H, W, 4), np.float32)
    nsum = np.zeros((H, W), np.float32)
    wsum = np.zeros((H, W), np.float32)
    o2all = old[2]
    zs = o2all[..., 3]
    zl = np.concatenate([zs[:, :1], zs[:, :-1]], 1)
    zr = np.concatenate([zs[:, 1:], zs[:, -1:]], 1)
    zu = np.concatenate([zs[:1], zs[:-1]], 0)
    zd = np.concatenate([zs[1:], zs[-1:]], 0)
    grad_all = np.minimum(np.abs(zl - zs), np.abs(zr - zs)) + np.minimum(np.abs(zu - zs), np.abs(zd - zs))
    gk = gkind(g3[..., 3])
    for j in range(4):
        tx, ty = x0 + (j & 1), y0 + (j >> 1)
        inb = front & (tx >= 0) & (ty >= 0) & (tx < W) & (ty < H)
        ox, oy = np.clip(tx, 0, W - 1).astype(np.int64), np.clip(ty, 0, H - 1).astype(np.int64)
        s, m = old[0][oy, ox], old[1][oy, ox]
        o2, o3 = old[2][oy, ox], old[3][oy, ox]
        ok = inb & (s[..., 3] != 0) & (o3[..., 3] == g3[..., 3])
        tol = np.where(gk == 2, F(0.25), F(0.02)) * dist + grad_all[oy, ox]
        ok &= ~((g2[..., 3] <= F(1e29)) & (np.abs(o2[..., 3] - dist) > tol))
        ok &= ~((gk == 0) & ((o2[..., :3] * g2[..., :3]).sum(-1) < F(0.9)))
        w = (F(1) - np.abs(fx - tx)) * (F(1) - np.abs(fy - ty))
        w = np.where(ok, w, F(0))
        with np.errstate(divide="ignore", invalid="ignore"):
            ws = np.where(ok, w / s[..., 3], F(0))
        a0 += ws[..., None] * np.where(ok[..., None], s, 0)
        a1 += ws[..., None] * np.where(ok[..., None], m, 0)
        nsum += w * np.where(ok, s[..., 3], 0)
        wsum += w
    keep = (wsum >= F(0.05)) & (history >= 0.5)
    with np.errstate(divide="ignore", invalid="ignore"):
        n = np.minimum(nsum / wsum, F(history))
        p0 = np.concatenate([a0[..., :3] / wsum[..., None] * n[..., None], n[..., None]], -1)
        p1 = np.stack([a1[..., 0] / wsum * n, a1[..., 1] / wsum * n, np.zeros_like(n), np.zeros_like(n)], -1)
    cur[0] = np.where(keep[..., None], p0, 0)
    cur[1] = np.where(keep[..., None], p1, 0)
    return cur
