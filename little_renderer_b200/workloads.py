"""Seeded synthetic workloads (no public dataset is involved; all inputs are generated here).

Triangles are kept as the reference stores them (engine/scene/scene.h:134-140 ``Triangle``):
corner ``q`` and edges ``u = b - a``, ``v = c - a``, each computed in float32 exactly as
``scene_add_triangle`` (engine/scene/scene.c add_tri) computes them in the float build.
"""
import numpy as np


def corners_to_quv(corners):
    """(n, 3, 3) float32 corners a, b, c -> (n, 9) q, u, v with float32 subtraction."""
    c = np.ascontiguousarray(corners, np.float32).reshape(-1, 3, 3)
    q = c[:, 0]
    u = (c[:, 1] - c[:, 0]).astype(np.float32)
    v = (c[:, 2] - c[:, 0]).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([q, u, v], axis=1), np.float32)


def soup(n, seed=1):
    """The builder workload: n triangles with centroids uniform in the unit cube, edges
    Gaussian with sigma = 0.002 * n^(-1/3), and 2 % of them (a seeded choice) scaled x50 about
    their centroid. Returns (n, 3, 3) float32 corners."""
    rng = np.random.default_rng(seed)
    cen = rng.random((n, 3), dtype=np.float64)
    sigma = 0.002 * n ** (-1.0 / 3.0)
    e1 = rng.normal(0.0, sigma, (n, 3))
    e2 = rng.normal(0.0, sigma, (n, 3))
    big = rng.random(n) < 0.02
    e1[big] *= 50.0
    e2[big] *= 50.0
    a = cen - (e1 + e2) / 3.0
    corners = np.stack([a, a + e1, a + e2], axis=1).astype(np.float32)
    return corners


def rays_at_cube(n, seed=2, radius=2.0, centre=(0.5, 0.5, 0.5), scale=1.0):
    """n rays: origins uniform on the sphere of `radius` about `centre`, unit directions toward
    uniform points of the unit cube; scale: the cube, the sphere and its centre scaled by it (the
    scaled soup's rays). Returns (orig, dir) float32 (n, 3) each."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    o = (np.asarray(centre) * scale + (radius * scale) * g).astype(np.float32)
    target = (rng.random((n, 3), dtype=np.float64) * scale).astype(np.float32)
    d = (target - o).astype(np.float32)
    d = (d / np.linalg.norm(d.astype(np.float64), axis=1, keepdims=True)).astype(np.float32)
    return np.ascontiguousarray(o), np.ascontiguousarray(d)


def mesh_bounds(quv):
    """SceneMesh.box (engine/scene/scene.c:638-646 mesh_bounds): the corners' box, unpadded."""
    quv = np.asarray(quv, np.float32).reshape(-1, 9)
    q = quv[:, 0:3]
    b = (q + quv[:, 3:6]).astype(np.float32)
    c = (q + quv[:, 6:9]).astype(np.float32)
    lo = np.minimum(np.minimum(q.min(0), b.min(0)), c.min(0)).astype(np.float32)
    hi = np.maximum(np.maximum(q.max(0), b.max(0)), c.max(0)).astype(np.float32)
    return lo, hi


# ---- the path tracer's scenes ------------------------------------------------------------------
# material types (engine/scene/scene.h MatType) and the presets' parameters (scene.h:48-70)
MAT_DIFFUSE, MAT_MIRROR, MAT_GLASS, MAT_LIGHT, MAT_PBR = 0, 1, 2, 3, 4


def material(type_, albedo=(0, 0, 0), emission=(0, 0, 0), ior=1.5, metallic=0.0, roughness=1.0, transmission=0.0):
    return {"type": type_, "albedo": tuple(float(x) for x in albedo), "emission": tuple(float(x) for x in emission),
            "ior": float(ior), "metallic": float(metallic), "roughness": float(roughness),
            "transmission": float(transmission)}


def diffuse(c):
    return material(MAT_DIFFUSE, albedo=c, ior=1.5, roughness=1.0)


def glass(tint, ior):
    return material(MAT_GLASS, albedo=tint, ior=ior, roughness=0.0, transmission=1.0)


def light(e):
    return material(MAT_LIGHT, emission=e, ior=1.0, roughness=1.0)


def pbr(base, metallic, roughness, ior, transmission):
    return material(MAT_PBR, albedo=base, ior=ior, metallic=metallic, roughness=roughness, transmission=transmission)


def icosphere(subdiv=2):
    """Unit icosphere: (20 * 4^subdiv, 3, 3) corners, counter-clockwise seen from outside."""
    t = (1.0 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    tri = np.array([[v[a], v[b], v[c]] for a, b, c in f], np.float64)
    tri /= np.linalg.norm(tri, axis=2, keepdims=True)
    for _ in range(subdiv):
        a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tri = np.concatenate([np.stack(s, 1) for s in ((a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca))])
    return tri


def cornell_spheres(seed=7, n_spheres=64, width=256, height=256):
    """The plain render: a box 555 units on a side, open at the front (5 walls of 2 triangles),
    a lamp quad under the ceiling (emission 15, white; Scene.light), and 64 icospheres of
    subdivision 2 (320 flat triangles each) with centres uniform in the box and radii uniform in
    [0.05, 0.15] x 555; each sphere's material one of Lambert (albedo U[0.2, 0.9]^3), GGX metal
    (roughness U[0.05, 0.5]) or dielectric (ior 1.5), at most 60 distinct (MAX_MATS is 64).
    The camera looks into the box from (278, 278, -800), vertical field of view 40 degrees."""
    S = 555.0
    rng = np.random.default_rng(seed)
    mats = [diffuse((0.73, 0.73, 0.73)), diffuse((0.65, 0.05, 0.05)), diffuse((0.12, 0.45, 0.15)),
            light((15.0, 15.0, 15.0))]
    corners, tmat = [], []

    def quad(a, b, c, d, m):
        corners.extend([[a, b, c], [a, c, d]])
        tmat.extend([m, m])

    quad((0, 0, 0), (S, 0, 0), (S, 0, S), (0, 0, S), 0)            # floor
    quad((0, S, 0), (0, S, S), (S, S, S), (S, S, 0), 0)            # ceiling
    quad((0, 0, S), (S, 0, S), (S, S, S), (0, S, S), 0)            # back
    quad((0, 0, 0), (0, 0, S), (0, S, S), (0, S, 0), 1)            # left
    quad((S, 0, 0), (S, S, 0), (S, S, S), (S, 0, S), 2)            # right
    kinds = rng.integers(0, 3, n_spheres)
    sphere_mats = []
    for i in range(min(n_spheres, 60)):
        k = kinds[i]
        if k == 0:
            sphere_mats.append(diffuse(rng.uniform(0.2, 0.9, 3)))
        elif k == 1:
            sphere_mats.append(pbr(rng.uniform(0.5, 0.95, 3), 1.0, rng.uniform(0.05, 0.5), 1.5, 0.0))
        else:
            sphere_mats.append(glass((1.0, 1.0, 1.0), 1.5))
    base = len(mats)
    mats.extend(sphere_mats)
    unit = icosphere(2)
    for i in range(n_spheres):
        r = rng.uniform(0.05, 0.15) * S
        c = rng.uniform(0.0, S, 3)
        tri = c + r * unit
        corners.extend(tri.tolist())
        tmat.extend([base + i % len(sphere_mats)] * len(unit))
    corners = np.asarray(corners, np.float32).reshape(-1, 3, 3)
    return {"corners": corners, "tri_mats": np.asarray(tmat, np.int32), "materials": mats,
            "lamp": {"q": (213.0, 554.0, 227.0), "u": (130.0, 0.0, 0.0), "v": (0.0, 0.0, 105.0), "material": 3},
            "camera": {"from": (278.0, 278.0, -800.0), "at": (278.0, 278.0, 0.0), "up": (0.0, 1.0, 0.0), "vfov": 40.0},
            "width": width, "height": height, "spp": 16, "max_depth": 8}


def cloud_grid(seed=3, res=(40, 32, 40), blobs=6):
    """A cloud-like density grid (nz, ny, nx): a few soft blobs (1 - r^2 / R^2, clipped at 0) with
    uniform centres in the grid's middle half and radii in [0.15, 0.3] of its size, summed and
    clipped to [0, 1.2]; the corners stay empty (an active box smaller than the grid)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = res
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    d = np.zeros(res, np.float64)
    for _ in range(blobs):
        c = rng.uniform(0.3, 0.7, 3)
        r = rng.uniform(0.15, 0.3)
        q = ((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (r * r)
        d += np.clip(1.0 - q, 0.0, None)
    return np.clip(d, 0.0, 1.2).astype(np.float32)


def foggy_cornell(seed=7, width=128, height=128, sigma_t=0.02, g=0.3):
    """The plain render's box (16 spheres) with a cloud of participating medium (cloud_grid, 40 x 32 x
    40 voxels) filling x in [80, 480], y in [60, 380], z in [80, 480]: extinction sigma_t per unit
    at density 1 (optical depth up to about 7 across), albedo (0.9, 0.85, 0.8), Henyey-Greenstein g."""
    sc = cornell_spheres(seed=seed, n_spheres=16, width=width, height=height)
    sc["volumes"] = [(cloud_grid(seed), (80.0, 60.0, 80.0), (480.0, 380.0, 480.0), sigma_t, (0.9, 0.85, 0.8), g)]
    return sc


def texture_maps(n=64):
    """Three procedural RGBA8 maps (uint32 (n, n), r | g << 8 | b << 16 | a << 24): a colour
    checker with value noise (sRGB), a metal-rough map (roughness in green from 0.15 to 1 in
    bands, metallic in blue in stripes), and a normal map of round bumps (tangent space)."""
    rng = np.random.default_rng(17)
    y, x = np.mgrid[0:n, 0:n]
    cell = ((x // (n // 8)) + (y // (n // 8))) % 2
    base = np.where(cell[..., None] == 1, [200, 60, 40], [230, 220, 190]).astype(np.float64)
    base += rng.uniform(-25, 25, (n, n, 1))
    base = np.clip(base, 0, 255).astype(np.uint32)
    checker = base[..., 0] | base[..., 1] << 8 | base[..., 2] << 16 | np.uint32(255) << 24
    rough = (40 + (215 * ((y // (n // 4)) + 1) // 4)).astype(np.uint32)
    metal = np.where((x // (n // 8)) % 2 == 0, 255, 0).astype(np.uint32)
    mr = np.uint32(0) | rough << 8 | metal << 16 | np.uint32(255) << 24
    cx, cy = (x % (n // 4)) - n / 8 + 0.5, (y % (n // 4)) - n / 8 + 0.5
    r2 = (cx * cx + cy * cy) / (n / 8) ** 2
    h = np.where(r2 < 1, np.sqrt(np.clip(1 - r2, 0, 1)), 0.0)
    nx, ny = np.where(r2 < 1, cx / (n / 8) * 0.6, 0.0), np.where(r2 < 1, -cy / (n / 8) * 0.6, 0.0)
    nz = np.sqrt(np.clip(1 - nx * nx - ny * ny, 0, 1)) + 0 * h
    enc = lambda v: np.clip(np.rint((v * 0.5 + 0.5) * 255), 0, 255).astype(np.uint32)   # noqa: E731
    normal = enc(nx) | enc(ny) << 8 | enc(nz) << 16 | np.uint32(255) << 24
    return [(checker.astype(np.uint32), 1, 0, 0), (mr.astype(np.uint32), 0, 0, 0), (normal.astype(np.uint32), 0, 2, 2)]


def textured_cornell(seed=7, width=128, height=128):
    """The plain render's box (16 spheres) with textured materials: the floor diffuse white under a
    colour checker and a bump normal map (4 repeats), the back wall a rough metal with the checker
    and a metal-rough map (2 repeats), one sphere material with the metal-rough map (its triangles
    sample it at their barycentrics: no texture coordinates). Floor and back wall triangles carry
    texture coordinates and tangents along +x."""
    sc = cornell_spheres(seed=seed, n_spheres=16, width=width, height=height)
    mats = sc["materials"]
    mats.append(dict(diffuse((0.8, 0.8, 0.8)), tex={"base": 1, "normal": 3, "uv_scale": 4.0}))
    mats.append(dict(pbr((0.9, 0.9, 0.9), 1.0, 0.6, 1.5, 0.0), tex={"base": 1, "mr": 2, "uv_scale": 2.0}))
    floor_m, back_m = len(mats) - 2, len(mats) - 1
    for i, m in enumerate(mats[4:], 4):
        if m["type"] == MAT_PBR and m.get("tex") is None:
            mats[i] = dict(m, tex={"mr": 2})
            break
    tm = sc["tri_mats"].copy()
    tm[0:2] = floor_m
    tm[4:6] = back_m
    sc["tri_mats"] = tm
    tri_uv = np.full((sc["corners"].shape[0], 3), -1, np.int32)
    tri_uv[0], tri_uv[1] = (0, 1, 2), (0, 2, 3)          # floor a b c, a c d
    tri_uv[4], tri_uv[5] = (4, 5, 6), (4, 6, 7)          # back wall
    uvs = np.array([[0, 0], [1, 0], [1, 1], [0, 1], [0, 1], [1, 1], [1, 0], [0, 0]], np.float32)
    tangents = np.tile(np.array([1, 0, 0, 1], np.float32), (8, 1))
    sc["texmaps"] = texture_maps()
    sc["texcoords"] = (tri_uv, uvs, tangents)
    return sc


def box_scene(seed, n_tris, width=256, height=256, spp=16, max_depth=8):
    """A scene of the plain render's kind with about n_tris triangles: the open box and its lamp,
    then icospheres and bevelled boxes (a quarter of the objects) with centres uniform in the box.
    Objects grow finer with the count (icosphere subdivision 1 to 4) and their radii shrink as
    count^(-1/3), so the box holds the same volume of them as the plain render's 64 spheres.
    Materials as the plain render's (Lambert, GGX metal, dielectric), at most 60 distinct."""
    S = 555.0
    rng = np.random.default_rng(seed)
    sub = 1 if n_tris < 4_000 else 2 if n_tris < 30_000 else 3 if n_tris < 120_000 else 4
    unit = icosphere(sub)
    per = unit.shape[0]
    n_obj = max(1, (n_tris - 12) // per)
    base_sc = cornell_spheres(seed=seed, n_spheres=0, width=width, height=height)
    corners = [base_sc["corners"].astype(np.float64)]
    tmat = [base_sc["tri_mats"]]
    mats = base_sc["materials"]
    kinds = rng.integers(0, 3, min(n_obj, 60))
    for k in kinds:
        if k == 0:
            mats.append(diffuse(rng.uniform(0.2, 0.9, 3)))
        elif k == 1:
            mats.append(pbr(rng.uniform(0.5, 0.95, 3), 1.0, rng.uniform(0.05, 0.5), 1.5, 0.0))
        else:
            mats.append(glass((1.0, 1.0, 1.0), 1.5))
    first = 4
    shrink = (64.0 / n_obj) ** (1.0 / 3.0)
    box_unit = rounded_box(per, rng)
    rots = random_rotations(n_obj, rng)
    radii = rng.uniform(0.05, 0.15, n_obj) * S * shrink
    centres = rng.uniform(0.0, S, (n_obj, 3))
    is_box = rng.random(n_obj) < 0.25
    for i in range(n_obj):
        shape = box_unit @ rots[i].T if is_box[i] else unit
        corners.append(centres[i] + radii[i] * shape)
        tmat.append(np.full(shape.shape[0], first + i % len(kinds), np.int32))
    base_sc["corners"] = np.concatenate(corners).astype(np.float32)
    base_sc["tri_mats"] = np.concatenate(tmat).astype(np.int32)
    base_sc["materials"] = mats
    base_sc["spp"], base_sc["max_depth"] = spp, max_depth
    return base_sc


def batch_scenes(n_scenes=256, seed=11, tri_range=(1_000, 200_000), resolutions=(128, 256, 512), spps=(8, 32, 128),
                 max_depth=8):
    """The multi-scene launch: n_scenes box scenes with triangle counts log-uniform in tri_range,
    each with a square resolution and spp drawn uniformly from the choices, depth max_depth."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(tri_range[0]), np.log(tri_range[1])
    out = []
    for i in range(n_scenes):
        n = int(np.exp(rng.uniform(lo, hi)))
        r = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        out.append(box_scene(seed * 100_003 + i, n, r, r, spp, max_depth))
    return out


def material_records(mats, ntex=0):
    """Materials as the device reads them: 16 floats each (albedo.xyz, type as int bits |
    emission.xyz, 0 | ior, metallic, roughness, transmission | the textures as gpu_tex_pack packs
    them: base | emissive << 8, mr | occlusion << 8 | strength << 16, normal | scale x 4096 << 8
    (uint32 bits), uv scale). A material's "tex" dict names texture numbers (1 + index), 0 none."""
    out = np.zeros((len(mats), 16), np.float32)
    words = out.view(np.uint32)
    for i, m in enumerate(mats):
        out[i, 0:3] = m["albedo"]
        out[i, 3] = np.array([m["type"]], np.int32).view(np.float32)[0]
        out[i, 4:7] = m["emission"]
        out[i, 8:12] = (m["ior"], m["metallic"], m["roughness"], m["transmission"])
        t = m.get("tex")
        if t:
            tx = lambda k: int(t.get(k, 0)) if 0 < int(t.get(k, 0)) <= ntex else 0   # noqa: E731
            os_ = t.get("occlusion_strength", 0.0) or 1.0
            ns = t.get("normal_scale", 0.0) or 1.0
            osq = int(min(os_, 1.0) * 255 + 0.5)
            nsq = int(min(ns, 4000.0) * 4096 + 0.5)
            words[i, 12] = tx("base") | tx("emissive") << 8
            words[i, 13] = tx("mr") | tx("occlusion") << 8 | ((osq << 16) if tx("occlusion") else 0)
            words[i, 14] = (tx("normal") | nsq << 8) if tx("normal") else 0
            out[i, 15] = t.get("uv_scale", 0.0)
    return out


def make_quad(q, u, v, material):
    """make_quad (engine/scene/scene.c:26-39) in float: the 24 floats the device reads
    (upload_world's layout, engine/gpu/trace_gpu.c:1145-1154)."""
    f = np.float32
    q, u, v = (np.asarray(x, f) for x in (q, u, v))
    n = np.array([u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]], f)
    dot = lambda a, b: f(f(f(a[0] * b[0]) + f(a[1] * b[1])) + f(a[2] * b[2]))
    ln = np.sqrt(dot(n, n), dtype=f)
    normal = (n * (f(1) / ln)).astype(f) if ln > 0 else n
    w = (n * (f(1) / dot(n, n))).astype(f)
    out = np.zeros(24, f)
    out[4:7], out[7] = q, 1.0
    out[8:11], out[11] = u, f(material)
    out[12:15], out[15] = v, ln
    out[16:19], out[19] = normal, dot(normal, q)
    out[20:23] = w
    return out


def camera(cam, aspect):
    """camera_make (engine/scene/camera.h:21-36) in float: origin, upper_left, horizontal, vertical."""
    f = np.float32
    frm, at, up = (np.asarray(cam[k], f) for k in ("from", "at", "up"))
    h = np.tan(f(f(f(f(cam["vfov"]) * f(np.pi)) / f(180.0)) / f(2.0)), dtype=f)
    view_h = f(f(2.0) * h)
    view_w = f(f(aspect) * view_h)

    def norm(a):
        ln = np.sqrt(f(f(f(a[0] * a[0]) + f(a[1] * a[1])) + f(a[2] * a[2])), dtype=f)
        return (a * (f(1) / ln)).astype(f)

    def cross(a, b):
        return np.array([f(a[1] * b[2]) - f(a[2] * b[1]), f(a[2] * b[0]) - f(a[0] * b[2]), f(a[0] * b[1]) - f(a[1] * b[0])], f)

    w = norm((frm - at).astype(f))
    u = norm(cross(up, w))
    v = cross(w, u)
    hor = (u * view_w).astype(f)
    ver = (v * view_h).astype(f)
    ul = (((frm - (hor * f(0.5)).astype(f)).astype(f) + (ver * f(0.5)).astype(f)).astype(f) - w).astype(f)
    return np.concatenate([frm, ul, hor, ver]).astype(f)


# ---- the instanced scene -----------------------------------------------------------------------
def rounded_box(target, rng):
    """A box with rounded (bevelled) edges: a subdivided cube pushed onto a rounded box."""
    n = max(2, int(round((target / 12.0) ** 0.5)))
    g = np.linspace(-1, 1, n + 1)
    faces = []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            a, b = np.meshgrid(g, g, indexing="ij")
            p = np.zeros(a.shape + (3,))
            p[..., axis] = sgn
            p[..., (axis + 1) % 3] = a
            p[..., (axis + 2) % 3] = b
            q00, q10, q01, q11 = p[:-1, :-1], p[1:, :-1], p[:-1, 1:], p[1:, 1:]
            t1 = np.stack([q00, q10, q11], -2).reshape(-1, 3, 3)
            t2 = np.stack([q00, q11, q01], -2).reshape(-1, 3, 3)
            tri = np.concatenate([t1, t2])
            if sgn < 0:
                tri = tri[:, ::-1]
            faces.append(tri)
    tri = np.concatenate(faces)
    half = rng.uniform(0.5, 1.0, 3)
    rad = 0.25 * half.min()
    p = tri * half
    core = np.clip(p, -(half - rad), half - rad)
    off = p - core
    ln = np.linalg.norm(off, axis=-1, keepdims=True)
    return core + off / np.maximum(ln, 1e-12) * rad


def convex_hull_mesh(target, rng):
    from scipy.spatial import ConvexHull
    npts = max(8, target // 2 + 2)
    d = rng.normal(size=(npts, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p = d * rng.uniform(0.6, 1.0, 3) * rng.uniform(0.9, 1.0, (npts, 1))
    hull = ConvexHull(p)
    tri = p[hull.simplices]
    # outward: the normal away from the centre
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    flip = (n * tri.mean(axis=1)).sum(1) < 0
    tri[flip] = tri[flip][:, ::-1]
    return tri


def xform_inverse(m):
    """xform_inverse (engine/scene/scene.c:606-623) in float32, for (n, 3, 4) transforms."""
    f = np.float32
    m = np.asarray(m, f)
    M = lambda i, j: m[:, i, j]
    det = (M(0, 0) * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) - M(0, 1) * (M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0))) \
        + M(0, 2) * (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0))
    idt = np.where(det != 0, f(1) / np.where(det != 0, det, f(1)), f(0)).astype(f)
    r = np.zeros_like(m)
    r[:, 0, 0] = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) * idt
    r[:, 0, 1] = (M(0, 2) * M(2, 1) - M(0, 1) * M(2, 2)) * idt
    r[:, 0, 2] = (M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1)) * idt
    r[:, 1, 0] = (M(1, 2) * M(2, 0) - M(1, 0) * M(2, 2)) * idt
    r[:, 1, 1] = (M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0)) * idt
    r[:, 1, 2] = (M(0, 2) * M(1, 0) - M(0, 0) * M(1, 2)) * idt
    r[:, 2, 0] = (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0)) * idt
    r[:, 2, 1] = (M(0, 1) * M(2, 0) - M(0, 0) * M(2, 1)) * idt
    r[:, 2, 2] = (M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0)) * idt
    for i in range(3):
        r[:, i, 3] = -((r[:, i, 0] * M(0, 3) + r[:, i, 1] * M(1, 3)) + r[:, i, 2] * M(2, 3))
    return r


def xform_box(m, lo, hi):
    """xform_box (scene.c:629-636): the world box of a transformed box, float32; m (n, 3, 4), lo/hi (n, 3)."""
    f = np.float32
    m = np.asarray(m, f)
    blo = np.full((m.shape[0], 3), f(1e30), f)
    bhi = np.full((m.shape[0], 3), f(-1e30), f)
    for c in range(8):
        p = np.stack([hi[:, 0] if c & 1 else lo[:, 0], hi[:, 1] if c & 2 else lo[:, 1], hi[:, 2] if c & 4 else lo[:, 2]], 1)
        w = np.stack([((m[:, r, 0] * p[:, 0] + m[:, r, 1] * p[:, 1]) + m[:, r, 2] * p[:, 2]) + m[:, r, 3] for r in range(3)], 1)
        blo = np.where(blo < w, blo, w)
        bhi = np.where(bhi > w, bhi, w)
    return blo.astype(f), bhi.astype(f)


def random_rotations(n, rng):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                     np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                     np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)


def sky(w, h, seed=3, sun_elev=45.0, sun_azim=30.0, sun_radius_deg=0.5, sun=5e4):
    """A synthetic HDR equirect sky (rows top to bottom, as env.h): lognormal luminance (mu 0,
    sigma 1) per pixel, faintly blue, and a sun disc of the given radius at radiance `sun`."""
    rng = np.random.default_rng(seed)
    lum = np.exp(rng.normal(0.0, 1.0, (h, w)))
    rgb = np.stack([lum * 0.8, lum * 0.9, lum * 1.1], -1)
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    ph = (u - 0.5) * 2 * np.pi
    th = v * np.pi
    d = np.stack([np.sin(th)[:, None] * np.sin(ph)[None, :], np.cos(th)[:, None] * np.ones((1, w)),
                  np.sin(th)[:, None] * np.cos(ph)[None, :]], -1)
    el, az = np.radians(sun_elev), np.radians(sun_azim)
    s = np.array([np.cos(el) * np.sin(az), np.sin(el), np.cos(el) * np.cos(az)])
    rgb[(d @ s) > np.cos(np.radians(sun_radius_deg))] = sun
    return np.ascontiguousarray(rgb, np.float32)


def instanced_field(seed=5, n_instances=5000, n_meshes=14, tri_range=(10_000, 100_000), width=1280, height=720,
                    sky_w=2048, sky_h=1024, spp=64, max_depth=12):
    """The instanced scene: n_meshes procedural meshes (icospheres, rounded boxes, convex hulls)
    with triangle counts log-uniform in tri_range, n_instances instances with random rotations at
    positions uniform over a 40 x 40 ground quad, heights U[0, 3]; one material per mesh (GGX metal,
    rough glass or Lambert); a grey ground quad; a synthetic sky; no lamp."""
    rng = np.random.default_rng(seed)
    mats, meshes = [], []
    lo_t, hi_t = np.log(tri_range[0]), np.log(tri_range[1])
    for m in range(n_meshes):
        target = int(np.exp(rng.uniform(lo_t, hi_t)))
        kind = m % 3
        if kind == 0:
            sub = int(np.clip(np.round(np.log(target / 20.0) / np.log(4.0)), 1, 7))
            tri = icosphere(sub) * rng.uniform(0.5, 1.0)
        elif kind == 1:
            tri = rounded_box(target, rng)
        else:
            tri = convex_hull_mesh(target, rng)
        meshes.append(np.ascontiguousarray(tri, np.float32))
        mk = rng.integers(0, 3)
        if mk == 0:
            mats.append(pbr(rng.uniform(0.5, 0.95, 3), 1.0, rng.uniform(0.05, 0.5), 1.5, 0.0))
        elif mk == 1:
            mats.append(pbr(rng.uniform(0.8, 1.0, 3), 0.0, rng.uniform(0.05, 0.3), 1.5, 1.0))
        else:
            mats.append(diffuse(rng.uniform(0.2, 0.9, 3)))
    mats.append(diffuse((0.5, 0.5, 0.5)))                        # the ground
    mesh_of = rng.integers(0, n_meshes, n_instances)
    R = random_rotations(n_instances, rng) * rng.uniform(0.4, 1.0, (n_instances, 1, 1))
    t = np.stack([rng.uniform(0, 40, n_instances), rng.uniform(0, 3, n_instances), rng.uniform(0, 40, n_instances)], 1)
    xf = np.concatenate([R, t[:, :, None]], 2).astype(np.float32)
    return {"meshes": meshes, "mesh_mats": list(range(n_meshes)), "materials": mats, "mesh_of": mesh_of.astype(np.int32),
            "xf": xf, "ground": {"q": (0.0, 0.0, 0.0), "u": (0.0, 0.0, 40.0), "v": (40.0, 0.0, 0.0),
                                 "material": n_meshes},
            "sky": sky(sky_w, sky_h), "camera": {"from": (20.0, 14.0, -18.0), "at": (20.0, 0.0, 20.0),
                                                 "up": (0.0, 1.0, 0.0), "vfov": 40.0},
            "width": width, "height": height, "spp": spp, "max_depth": max_depth}


def instance_records(sc):
    """32 floats per instance (lrc_scene_set_instances): xf, its inverse, box lo + mesh, box hi + material."""
    xf = sc["xf"]
    n = xf.shape[0]
    inv = xform_inverse(xf)
    mlo = np.zeros((len(sc["meshes"]), 3), np.float32)
    mhi = np.zeros((len(sc["meshes"]), 3), np.float32)
    for m, tri in enumerate(sc["meshes"]):
        quv = corners_to_quv(tri)
        mlo[m], mhi[m] = mesh_bounds(quv)
    lo, hi = xform_box(xf, mlo[sc["mesh_of"]], mhi[sc["mesh_of"]])
    rec = np.zeros((n, 32), np.float32)
    rec[:, 0:12] = xf.reshape(n, 12)
    rec[:, 12:24] = inv.reshape(n, 12)
    rec[:, 24:27] = lo
    rec[:, 27] = sc["mesh_of"].view(np.float32)
    rec[:, 28:31] = hi
    rec[:, 31] = np.full(n, -1, np.int32).view(np.float32)
    return rec


def rigid_motion(n, seed, speed=(0.5, 2.0), spin=(0.2, 1.5)):
    """Per-instance rigid motion: a linear velocity (uniform direction, speed uniform in `speed`
    units per frame) and an angular one (uniform axis, rate uniform in `spin` radians per frame)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v *= (rng.uniform(*speed, n) / np.linalg.norm(v, axis=1))[:, None]
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    return {"v": v, "axis": axis, "rate": rng.uniform(*spin, n)}


def moved_xf(xf0, motion, t):
    """The transforms at frame t: each instance turned about its axis by rate * t (after its own
    rotation and scale) and carried by v * t, float32."""
    xf0 = np.asarray(xf0, np.float64)
    a, th = motion["axis"], motion["rate"] * t
    c, s_ = np.cos(th), np.sin(th)
    x, y, z = a.T
    rot = np.stack([np.stack([c + x * x * (1 - c), x * y * (1 - c) - z * s_, x * z * (1 - c) + y * s_], -1),
                    np.stack([y * x * (1 - c) + z * s_, c + y * y * (1 - c), y * z * (1 - c) - x * s_], -1),
                    np.stack([z * x * (1 - c) - y * s_, z * y * (1 - c) + x * s_, c + z * z * (1 - c)], -1)], 1)
    out = np.empty_like(xf0)
    out[:, :, :3] = rot @ xf0[:, :, :3]
    out[:, :, 3] = xf0[:, :, 3] + motion["v"] * t
    return out.astype(np.float32)


def instanced_box(seed, n_instances=2000, n_meshes=4, width=256, height=256, spp=16, max_depth=8):
    """The plain render's box and lamp with n_instances instances of n_meshes meshes inside
    (icospheres of subdivision 2 and bevelled boxes of about 320 triangles), each instance turned
    at random, scaled to a radius uniform in [4, 12] and placed uniformly in the box; one material
    (Lambert, GGX metal or dielectric) per mesh."""
    rng = np.random.default_rng(seed)
    base = cornell_spheres(seed=seed, n_spheres=0, width=width, height=height)
    mats = base["materials"]
    meshes, mesh_mats = [], []
    for m in range(n_meshes):
        k = m % 3
        mats.append(diffuse(rng.uniform(0.2, 0.9, 3)) if k == 0 else
                    pbr(rng.uniform(0.5, 0.95, 3), 1.0, rng.uniform(0.05, 0.5), 1.5, 0.0) if k == 1 else
                    glass((1.0, 1.0, 1.0), 1.5))
        meshes.append((icosphere(2) if m % 2 == 0 else rounded_box(320, rng)).astype(np.float32))
        mesh_mats.append(len(mats) - 1)
    rot = random_rotations(n_instances, rng)
    scale = rng.uniform(4.0, 12.0, n_instances)
    xf = np.zeros((n_instances, 3, 4), np.float32)
    xf[:, :, :3] = rot * scale[:, None, None]
    xf[:, :, 3] = rng.uniform(20.0, 535.0, (n_instances, 3))
    base.update({"meshes": meshes, "mesh_mats": mesh_mats, "xf": xf,
                 "mesh_of": rng.integers(0, n_meshes, n_instances).astype(np.int32),
                 "spp": spp, "max_depth": max_depth})
    return base

