"""Packs the reference-GPU golden vectors into tests/golden/ref_gpu_equations.npz.

The vectors come from oracle/_ref/ref_gpu_golden -- the reference's own GPU
functors (src/equations_cuda.cu) built from its sources by `make -C oracle
ref-golden` and run on a GPU:

    oracle/_ref/ref_gpu_golden <outdir>
    python tests/golden/make_ref_gpu_golden.py <outdir>

The inputs are rebuilt by tests/golden/ref_gpu_inputs.py (the same integer hash
as the harness), so the archive holds the outputs only.
"""
import os
import sys

import numpy as np

NAMES = ["lambda_rhs", "lambda_rho", "lambda_step", "sqrt_rhs", "sqrt_rho", "sqrt_step", "fixed_rhs", "fixed_rho",
         "fixed_step", "kgfrw_dot_rho", "approx_rhs", "approx_fullband_rhs"]


def main(src):
    out = {n: np.fromfile(os.path.join(src, n + ".f64")) for n in NAMES}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_gpu_equations.npz")
    np.savez_compressed(dst, **out)
    print(dst, {k: v.size for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1])
