"""Generates tests/golden/ref_jacobi*.npz: grids written by the reference's
own single-GPU Jacobi runs (single_gpu() of Stencil/jacobi2D/src/common.cu and
Stencil/jacobi3D/src/common.cu, FP32, the reference's initial state), built
from the reference sources by `make -C oracle ref` into oracle/_ref/.

Needs a CUDA device:  python tests/golden/make_ref_fixtures.py OUTDIR
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

CASES_2D = [(32, 32, 10), (64, 48, 37), (40, 17, 5), (256, 256, 100), (7, 9, 1)]
CASES_2D_MIRROR = [(64, 32, 9), (128, 40, 20)]  # nx multiple of 32 (reference kernel bound)
CASES_3D = [(16, 12, 10, 7), (33, 9, 17, 12), (32, 32, 32, 20), (64, 40, 24, 5), (5, 6, 7, 1)]


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for nx, ny, it in CASES_2D:
        out = oracle.ref_jacobi2d(nx, ny, it)
        np.savez_compressed(os.path.join(outdir, f"ref_jacobi2d_{nx}x{ny}_{it}.npz"), out=out, niter=it,
                            kind="2d")
    for nx, ny, it in CASES_2D_MIRROR:
        out = oracle.ref_jacobi2d(nx, ny, it, mirror=True)
        np.savez_compressed(os.path.join(outdir, f"ref_jacobi2d_mirror_{nx}x{ny}_{it}.npz"), out=out,
                            niter=it, kind="2d_mirror")
    for nx, ny, nz, it in CASES_3D:
        out = oracle.ref_jacobi3d(nx, ny, nz, it)
        np.savez_compressed(os.path.join(outdir, f"ref_jacobi3d_{nx}x{ny}x{nz}_{it}.npz"), out=out,
                            niter=it, kind="3d")
    print("wrote", len(os.listdir(outdir)), "fixtures to", outdir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
