"""Inputs and parameters of the reference-GPU golden vectors (ref_gpu_equations.npz).

The same closed-form integer hash as oracle/ref_gpu_golden.cu (mix32 of the site or
mode index), so the arrays here equal the harness's inputs bit for bit:
phi = 0.5 (2u - 1), dphi = 0.3 (2u - 1), Psi = 0.02 (2u - 1) with u = mix32(i * 0x9E3779B9
+ salt) / 2^32, and a band-limited, Hermitian-on-c=0 R_fft.
"""
import numpy as np

T, DT = 1.3, 0.05
FRW = dict(a1=1.0, H1=0.5, t1=1.0)
SMALL = dict(N=8, L=5.0, m=1.0, lam=0.8, f_a=0.7)
APPROX = dict(N=16, L=10.0, m=1.0, M=8)

# case -> (equation code, lattice, band of R_fft or None, with fixed Psi)
CASES = {
    "lambda": (3, SMALL, None, False),
    "sqrt": (4, SMALL, None, False),
    "fixed": (5, SMALL, None, True),
    "approx": (6, APPROX, APPROX["M"] // 2, False),
    "approx_fullband": (6, APPROX, APPROX["N"] // 2 + 1, False),
}


def mix32(x):
    x = np.asarray(x, dtype=np.uint32)
    with np.errstate(over="ignore"):
        x = x ^ (x >> np.uint32(16))
        x = x * np.uint32(0x7FEB352D)
        x = x ^ (x >> np.uint32(15))
        x = x * np.uint32(0x846CA68B)
        x = x ^ (x >> np.uint32(16))
    return x


def u01(i, salt):
    i = np.asarray(i, dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = (i.astype(np.uint32) * np.uint32(0x9E3779B9) + np.uint32(salt)).astype(np.uint32)
    return mix32(v).astype(np.float64) / 4294967296.0


def state(N):
    i = np.arange(N ** 3)
    return np.concatenate([0.5 * (2 * u01(i, 1) - 1), 0.3 * (2 * u01(i, 2) - 1)])


def psi(N):
    return 0.02 * (2 * u01(np.arange(N ** 3), 3) - 1)


def R_fft(N, band):
    nh = N // 2 + 1
    a, b, c = np.meshgrid(np.arange(N), np.arange(N), np.arange(nh), indexing="ij")
    o = (a * N + b) * nh + c
    oc = (((N - a) % N) * N + (N - b) % N) * nh + c
    asf = np.where(a <= N // 2, a, N - a)
    bsf = np.where(b <= N // 2, b, N - b)
    keep = (asf < band) & (bsf < band) & (c < band)
    re = 1e-3 * (2 * u01(o, 4) - 1)
    im = 1e-3 * (2 * u01(o, 5) - 1)
    edge = (c == 0) | (c == N // 2)
    re = np.where(edge, 1e-3 * ((2 * u01(o, 4) - 1) + (2 * u01(oc, 4) - 1)), re)
    im = np.where(edge, 1e-3 * ((2 * u01(o, 5) - 1) - (2 * u01(oc, 5) - 1)), im)
    out = np.zeros((N, N, nh, 2))
    out[..., 0] = np.where(keep, re, 0.0)
    out[..., 1] = np.where(keep, im, 0.0)
    return out.ravel()


def oracle_params(O, case):
    """oracle.make_params for a case (O: the oracle module)."""
    eq, lat, _, fixed = CASES[case]
    kw = dict(lat)
    N, L, m = kw.pop("N"), kw.pop("L"), kw.pop("m")
    if fixed:
        kw["psi_fixed"] = psi(N)
    return O.make_params(N, L, m, eq=eq, **FRW, **kw)


def inputs(case):
    """(state, R_fft or None, Psi or None) of a case."""
    eq, lat, band, fixed = CASES[case]
    N = lat["N"]
    return state(N), (R_fft(N, band) if band is not None else None), (psi(N) if fixed else None)
