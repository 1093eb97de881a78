"""Writes tests/golden/growth_and_fs_n384.npz from the reference's published
sample outputs (output/Growth_and_FS/ in the reference tree; produced by the
reference driver src/main.cpp at N=384, L=307.2, seed 0).

Only a compact, deterministic subset is kept so the fixture stays small:
for every spectrum the first 4096 s^2 bins, every 97th bin after that, and the
full-array sum; for the rho slice / axis average the first 4096 values and the
sum.  The parity tests rebuild the same quantities with the oracles and compare
on exactly these entries.

Usage: python tests/golden/make_golden.py <path/to/reference tree>
"""
import os
import sys

import numpy as np

if len(sys.argv) < 2:
    sys.exit("usage: make_golden.py <path/to/reference tree>")
ref = sys.argv[1]
src = os.path.join(ref, "output", "Growth_and_FS")
out = {}
for name in ["initial_R_spectrum", "initial_Psi_spectrum", "rho_spectrum_0", "varphi_plus_spectrum_0",
             "rho_slice_0", "rho_axis_average_0"]:
    a = np.fromfile(os.path.join(src, name + ".dat"))
    if "spectrum" in name:
        idx = np.concatenate([np.arange(4096), np.arange(4096, a.size, 97)])
    else:
        idx = np.arange(4096)
    out[name + "_idx"] = idx.astype(np.int64)
    out[name + "_val"] = a[idx]
    out[name + "_sum"] = np.array([a.sum()])
    out[name + "_size"] = np.array([a.size])
out["t_list"] = np.fromfile(os.path.join(src, "t_list.dat"))
out["N"] = np.array([384])
out["L"] = np.array([384 * 0.8])
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "growth_and_fs_n384.npz")
np.savez_compressed(dst, **out)
print("wrote", dst, os.path.getsize(dst), "bytes")
