"""TEST INFRASTRUCTURE (the oracle): a numpy restatement of the reference's reprojection of a new
image's samples from the previous image's (engine/gpu/shaders/trace/trace_reproject.wgsl `main`),
and of its temporal gradients (`gmatch`, `gfilter`, and `main`'s history from the tiles' lambda,
dims.w = 1), which have no CPU counterpart in the reference. Parity unpinned: the reference's WGSL
cannot run here. The gradient samples themselves are path traced (trace.wgsl main's gradient
branch): the tests take their lambda from the CUDA path and restate what is made of it.

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


def same_surface_at(old, g2, g3, ox, oy, dist, edit=False):
    """same_surface (trace_reproject.wgsl:62-86) of old pixels (oy, ox) (int arrays, in the image)
    for new pixels whose guide is g2, g3 and whose point is `dist` from the old eye."""
    zs = old[2][..., 3]
    zl = np.concatenate([zs[:, :1], zs[:, :-1]], 1)
    zr = np.concatenate([zs[:, 1:], zs[:, -1:]], 1)
    zu = np.concatenate([zs[:1], zs[:-1]], 0)
    zd = np.concatenate([zs[1:], zs[-1:]], 0)
    grad_all = np.minimum(np.abs(zl - zs), np.abs(zr - zs)) + np.minimum(np.abs(zu - zs), np.abs(zd - zs))
    gk = gkind(g3[..., 3])
    s, o2, o3 = old[0][oy, ox], old[2][oy, ox], old[3][oy, ox]
    ok = (s[..., 3] != 0) & (o3[..., 3] == g3[..., 3])
    tol = np.where(gk == 2, F(0.25), F(0.02)) * dist + grad_all[oy, ox]
    ok &= ~((g2[..., 3] <= F(1e29)) & (np.abs(o2[..., 3] - dist) > tol))
    ok &= ~((gk == 0) & ((o2[..., :3] * g2[..., :3]).sum(-1) < F(0.9)))
    if edit:
        dm = np.abs(o3[..., :3] - g3[..., :3]).max(-1)
        ok &= ~((gk == 0) & (dm > F(0.02) + F(0.1) * g3[..., :3].max(-1)))
    return ok


def hashr(x):
    """lowbias32 on a Python int."""
    x &= 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


TILE = 4


def gmatch(old, cur, oc, nc, nxt, edit=False):
    """gmatch (trace_reproject.wgsl:175-214): per tile (th, tw) the new pixel k, the old pixel o
    (-1: none), the offset (dx, dy), the old sample's value and number."""
    old = np.asarray(old, np.float32)
    cur = np.asarray(cur, np.float32)
    H, W = cur.shape[1:3]
    g2, g3 = cur[2], cur[3]
    fx, fy, dist, front = old_place(oc, nc, W, H, g2)
    ox, oy = np.floor(fx + F(0.5)), np.floor(fy + F(0.5))
    inb = front & (gkind(g3[..., 3]) == 0) & (ox >= 0) & (oy >= 0) & (ox < W) & (oy < H)
    oxi, oyi = np.clip(ox, 0, W - 1).astype(np.int64), np.clip(oy, 0, H - 1).astype(np.int64)
    last = old[1][oyi, oxi]
    ok = inb & (last[..., 3] >= F(0.5)) & same_surface_at(old, g2, g3, oxi, oyi, dist, edit)
    tw, th = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    out = {"k": np.full((th, tw), -1, np.int64), "o": np.full((th, tw), -1, np.int64),
           "d": np.zeros((th, tw, 2), np.float32), "l": np.zeros((th, tw), np.float32),
           "kk": np.zeros((th, tw), np.int64)}
    for t in range(tw * th):
        tx, ty = t % tw, t // tw
        first = hashr(t ^ hashr(nxt)) % (TILE * TILE)
        for i in range(TILE * TILE):
            c = (first + i) % (TILE * TILE)
            px, py = tx * TILE + c % TILE, ty * TILE + c // TILE
            if px >= W or py >= H or not ok[py, px]:
                continue
            lo = int(last[py, px, 3]) - 1
            cnt = (nxt & 0xFF000000) | lo
            if cnt > nxt:
                cnt -= 0x1000000
            out["k"][ty, tx] = py * W + px
            out["o"][ty, tx] = oyi[py, px] * W + oxi[py, px]
            out["d"][ty, tx] = (ox[py, px] - fx[py, px], oy[py, px] - fy[py, px])
            out["l"][ty, tx] = last[py, px, 2]
            out["kk"][ty, tx] = cnt
            break
    return out


def gfilter(lam, cur):
    """gfilter's 3 passes (trace_reproject.wgsl:221-269) over the tiles' lambda (th, tw), -1 none:
    the filtered lambda (th, tw). The anchors' guide (plane 2 of cur) weighs the tiles."""
    cur = np.asarray(cur, np.float32)
    th, tw = lam.shape
    ga_all = cur[2][::TILE, ::TILE][:th, :tw]
    lam = np.asarray(lam, np.float32)
    for fpass in range(3):
        step = 1 << fpass
        out = np.full_like(lam, -1)
        for ty in range(th):
            for tx in range(tw):
                ga = ga_all[ty, tx]
                s = ws = F(0)
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        bx, by = tx + dx * step, ty + dy * step
                        if bx < 0 or by < 0 or bx >= tw or by >= th or lam[by, bx] < 0:
                            continue
                        gb = ga_all[by, bx]
                        w = F((1.0 if dx == 0 else 0.5) * (1.0 if dy == 0 else 0.5))
                        if ga[3] < F(1e29) and gb[3] < F(1e29):
                            nd = max(F(ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]), F(0))
                            w = F(w * F(np.exp(-abs(ga[3] - gb[3]) / (F(0.05) * ga[3] + F(1e-3)))) * F(nd ** 8))
                        s = F(s + w * lam[by, bx])
                        ws = F(ws + w)
                out[ty, tx] = s / ws if ws > F(1e-4) else F(-1)
        lam = out
    return lam


def grad_history(lam, cur, hmax, fallback, edit=False):
    """Each pixel's history from its tile's filtered lambda (trace_reproject.wgsl:100-113)."""
    cur = np.asarray(cur, np.float32)
    H, W = cur.shape[1:3]
    lp = np.repeat(np.repeat(lam, TILE, 0), TILE, 1)[:H, :W]
    l = lp * F(4) if edit else lp
    with np.errstate(divide="ignore", invalid="ignore"):
        h = np.minimum(np.floor((F(1) - np.minimum(l, F(1))) / np.maximum(l, F(1e-3)) + F(0.5)), F(hmax))
    h = np.where(lp >= 0, h, F(fallback))
    if edit:
        h = np.where(gkind(cur[3][..., 3]) != 0, F(fallback), h)
    return h.astype(np.float32)


def reproject(old, cur, oc, nc, history, edit=False):
    """cur's planes 0 and 1 from old's (cur's planes 2 and 3: the new guide); history: a number, or
    each pixel's (grad_history). Returns the new (4, h, w, 4) planes."""
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
        if edit:
            dm = np.abs(o3[..., :3] - g3[..., :3]).max(-1)
            ok &= ~((gk == 0) & (dm > F(0.02) + F(0.1) * g3[..., :3].max(-1)))
        w = (F(1) - np.abs(fx - tx)) * (F(1) - np.abs(fy - ty))
        w = np.where(ok, w, F(0))
        with np.errstate(divide="ignore", invalid="ignore"):
            ws = np.where(ok, w / s[..., 3], F(0))
        a0 += ws[..., None] * np.where(ok[..., None], s, 0)
        a1 += ws[..., None] * np.where(ok[..., None], m, 0)
        nsum += w * np.where(ok, s[..., 3], 0)
        wsum += w
    history = np.asarray(history, np.float32)
    keep = (wsum >= F(0.05)) & (history >= 0.5)
    with np.errstate(divide="ignore", invalid="ignore"):
        n = np.minimum(nsum / wsum, history)
        p0 = np.concatenate([a0[..., :3] / wsum[..., None] * n[..., None], n[..., None]], -1)
        p1 = np.stack([a1[..., 0] / wsum * n, a1[..., 1] / wsum * n, np.zeros_like(n), np.zeros_like(n)], -1)
    cur[0] = np.where(keep[..., None], p0, 0)
    cur[1] = np.where(keep[..., None], p1, 0)
    return cur
