"""Makes tests/golden/cornell<size>_fp64_4096spp.npy: the plain render's scene (the open box, its
lamp and 64 icospheres; workloads.cornell_spheres at size x size) rendered by the reference's own
double-precision CPU build (trace_image, engine/rt/tracer.c:329, built with -DLR_DOUBLE) at 4096
samples per pixel, seed 1, depth 8, NEE + MIS, Owen-Sobol sampler: the FP64 oracle images are
measured against. Stored as float32 mean radiance (size, size, 3). Sizes: 128 (the small tests)
and 256 (the plain render's own size).

    python tests/golden/make_fp64_golden.py [size]   # needs the reference's sources (oracle/_ref)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from little_renderer_b200 import workloads as W  # noqa: E402

SPP, SEED, SIZE = 4096, 1, 128


def scene(sc, double):
    ref = O.RefScene(double)
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    ref.triangles(sc["corners"], sc["tri_mats"])
    lamp = sc["lamp"]
    ref.quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"], light=True)
    ref.set_accel()
    return ref


def main(size=SIZE):
    SIZE = size
    sc = W.cornell_spheres(width=SIZE, height=SIZE)
    c = sc["camera"]
    cam = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
    ref = scene(sc, True)
    t0 = time.time()
    img, rays = ref.trace_image(cam, c["vfov"], SIZE, SIZE, SPP, SEED, sc["max_depth"])
    out = os.path.join(HERE, f"cornell{SIZE}_fp64_{SPP}spp.npy")
    np.save(out, img.astype(np.float32))
    print(f"{out}: {time.time() - t0:.1f} s, rays {rays}, mean {img.mean():.5f}")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else SIZE)
