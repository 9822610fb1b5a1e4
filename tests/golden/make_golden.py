"""Generates the golden fixtures of tests/test_oracle_pins.py by running the reference's own code,
built from the reference sources by oracle/ref_harness/Makefile into oracle/_ref/:

  cubic_kernel.npz      W and dW/dx of the reference CubicKernelPerso (FP32) at 257 distances
  neighbors_8x8x8.npz   neighbour sets of a seeded 512-particle scene through the reference's
                        ITER_NEIGHBORS_FROM_STRUCTURE_LINEAR_ADVANCED macro over its 256^3 table
  first_step_8x8x8.npz  fields after one TimeStepDFSPH::step() of the reference CPU solver
                        (analytic cubic kernel, reference default mass) on the same scene

usage: python tests/golden/make_golden.py   (needs oracle/_ref built; run from the repo root)
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import Oracle  # noqa: E402
from oracle.ref_runner import available, ref_cubic_values, ref_neighbor_lists, run_reference_full  # noqa: E402
from splishsplash_for_cuda_b200.scene import synthetic_scene  # noqa: E402

OUT = Path(__file__).resolve().parent


def scene():
    return synthetic_scene(1, counts=(8, 8, 8), jitter=0.01)


def main():
    if not available():
        raise SystemExit("oracle/_ref is not built (make -C oracle/ref_harness)")
    H = np.float32(0.1)
    r = np.linspace(0.0, 0.11, 257).astype(np.float32)
    w, g = ref_cubic_values(float(H), r)
    np.savez_compressed(OUT / "cubic_kernel.npz", H=H, r=r, W=w, gradW_x=g)
    s = scene()
    o = Oracle(s, 64)
    off = np.array([int(o.scalar("grid_offset_" + a)) for a in "xyz"], dtype=np.int32)
    counts, lists = ref_neighbor_lists(s.fluid, s.boundary, 4 * s.config.particleRadius, off, row=96)
    np.savez_compressed(OUT / "neighbors_8x8x8.npz", fluid=s.fluid, boundary=s.boundary, offset=off,
                        counts=counts, lists=lists)
    rr = run_reference_full(s, steps=1, kernel=0)
    np.savez_compressed(OUT / "first_step_8x8x8.npz", fluid=s.fluid, boundary=s.boundary,
                        iterations=rr["iterations"], iterations_v=rr["iterations_v"],
                        position=rr["position"], velocity=rr["velocity"], density=rr["density"],
                        factor=rr["factor"], boundary_psi=rr["boundary_psi"])
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
