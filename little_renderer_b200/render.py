"""A world scene (primitives, triangles, materials, the lamp) on the device, from the dict the
workload generators return, and the image path tracing through the C ABI gives."""
import numpy as np

from . import native, workloads as W


def world_scene(ctx, sc, builder=1, key_bits=30, blue_noise=None, bsdf_tables=None):
    """lrc_scene with the scene's triangles, its lamp quad (primitive 0, Scene.light), materials
    and the path tracer's tables (None: the library's own), its BVH built (PLOC by default)."""
    s = native.Scene(ctx)
    quv = W.corners_to_quv(sc["corners"])
    s.set_triangles(native.pack_tris(quv, sc["tri_mats"]))
    lamp = sc.get("lamp")
    if lamp is not None:
        s.set_prims(W.make_quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"]))
        s.set_light(0)
    s.set_materials(W.material_records(sc["materials"], len(sc.get("texmaps", []))))
    s.set_tables(blue_noise, bsdf_tables)
    if sc.get("volumes"):
        s.set_volumes(sc["volumes"])
    if sc.get("texmaps"):
        s.set_texmaps(sc["texmaps"])
    if sc.get("texcoords"):
        s.set_texcoords(*sc["texcoords"])
    s.build(builder, key_bits)
    return s


def camera12(sc):
    return W.camera(sc["camera"], sc["width"] / sc["height"])


def render(ctx, scene, sc, spp=None, exact=0, seed=1, max_depth=None, sampler=1):
    """(mean image (h, w, 3), rays traced): spp samples per pixel."""
    spp = sc["spp"] if spp is None else spp
    p = native.trace_params(camera12(sc), sc["width"], sc["height"], sc["max_depth"] if max_depth is None else max_depth,
                            1, sampler, exact, seed)
    acc, rays = scene.trace(p, spp)
    img = acc[..., :3] * (np.float32(1) / np.maximum(acc[..., 3:4], np.float32(1)))
    return img.astype(np.float32), rays


def instanced_scene(ctx, sc, mesh_builder=1, key_bits=30, blue_noise=None, bsdf_tables=None, sky=True):
    """lrc_scene of an instanced field: the ground quad (the world's one primitive), the meshes and
    their trees, the instances and their top level, the sky, no lamp."""
    s = native.Scene(ctx)
    g = sc["ground"]
    s.set_prims(W.make_quad(g["q"], g["u"], g["v"], g["material"]))
    s.set_light(-1)
    s.set_materials(W.material_records(sc["materials"]))
    s.set_tables(blue_noise, bsdf_tables)
    s.build(1, 30)
    s.set_meshes([native.pack_tris(W.corners_to_quv(t), np.full(t.shape[0], m, np.int32))
                  for t, m in zip(sc["meshes"], sc["mesh_mats"])])
    s.set_instances(W.instance_records(sc))
    s.build_instances(mesh_builder, key_bits)
    if sky:
        s.set_sky(sc["sky"])
    return s


def instanced_box_scene(ctx, sc, mesh_builder=1, key_bits=30, blue_noise=None, bsdf_tables=None):
    """lrc_scene of an instanced box: the walls (world triangles) and the lamp (primitive 0,
    Scene.light), the meshes and their trees, the instances and their top level."""
    s = world_scene(ctx, sc, 1, key_bits, blue_noise, bsdf_tables)
    s.set_meshes([native.pack_tris(W.corners_to_quv(t), np.full(t.shape[0], m, np.int32))
                  for t, m in zip(sc["meshes"], sc["mesh_mats"])])
    s.set_instances(W.instance_records(sc))
    s.build_instances(mesh_builder, key_bits)
    return s



def sample_range(rank, world, spp):
    """Rank's share of an image's spp samples split over `world` ranks: (spp0, n), the samples
    [spp0, spp0 + n); the first spp % world ranks take one more. The shares cover [0, spp) once
    each, so the sum of the ranks' accumulation buffers holds every sample of every pixel."""
    if world < 1 or not 0 <= rank < world or spp < 0:
        raise ValueError("sample_range: 0 <= rank < world and spp >= 0")
    base, extra = divmod(spp, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


def trace_split(scene, params, spp, d_accum, dist=None, group=None):
    """One image traced by all ranks of a torch.distributed group (the multi-GPU sample split):
    each rank traces its sample_range of every pixel into d_accum (a device tensor (h, w, 4),
    cleared by the caller), then one sum all-reduce of the W x H x 16-B buffers gives every rank
    the whole image. A fast-mode sample's random numbers depend on its pixel, its number and the
    seed only, so the image has the samples one rank would trace (summed in another order). The
    scene's context must launch on torch's current stream (lrc_set_stream), which the all-reduce
    then follows. Exact mode (one stream per pixel from its first sample) cannot be split.
    Returns this rank's (spp0, n)."""
    world = dist.get_world_size(group) if dist is not None else 1
    rank = dist.get_rank(group) if dist is not None else 0
    if params.exact and world > 1:
        raise ValueError("trace_split: exact mode cannot be split over ranks")
    spp0, n = sample_range(rank, world, spp)
    if n:
        scene.trace_device(params, n, d_accum.data_ptr(), spp0=spp0)
    if world > 1:
        dist.all_reduce(d_accum, op=dist.ReduceOp.SUM, group=group)
    return spp0, n
