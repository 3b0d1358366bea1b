"""TEST INFRASTRUCTURE: how far the reference's own Wen-Yin integration moves under a tiny
perturbation of the sketch, on a scaled-down copy of the 50000 x 50000 TS / WY case (the same
spectrum shape sigma_i = (1 + i)^(-1/2), noise of the same spectral norm relative to sigma_k).

Runs the oracle only (the NumPy restatement of core/stage/@x@_integrate_wen_yin.c and the TS
orthogonalization / Gramian postprocessing), in FP64, twice: on Y = A Omega and on Y perturbed
elementwise by 1e-5 relative noise (about the MIXED sketch's rounding).  Prints both WY iteration
counts and the largest relative difference of the k leading singular values.

    python oracle/wy_sensitivity.py
"""
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import isvd_oracle as O  # noqa: E402


def main(m=4000, r=800, k=32, p=32, N=16, seed=0):
    rng = np.random.default_rng(seed)
    n, l = m, k + p
    u = np.linalg.qr(rng.standard_normal((m, r)))[0]
    v = np.linalg.qr(rng.standard_normal((n, r)))[0]
    sig = (1.0 + np.arange(r)) ** -0.5
    noise = 1e-3 * np.sqrt(50000.0 / m)  # noise spectral norm ~ 2 sqrt(m) noise, as at m = 50000
    a = (u * sig) @ v.T + noise * rng.standard_normal((m, n))
    y = a @ rng.standard_normal((n, l * N))
    out = {}
    for name, yy in (("exact", y), ("perturbed 1e-5", y * (1 + 1e-5 * rng.standard_normal(y.shape)))):
        t = time.time()
        q = O.orthogonalize_tall_skinny_qr(yy, l, N)
        qb, it, mu = O.integrate_wen_yin(q, l, N, maxit=512, tol=1e-4)
        s, _, _ = O.postprocess_gramian(a, qb, k)
        out[name] = s[:k]
        print("%-15s WY iterations %3d, final mu %.2e (%.1f s)" % (name, it, mu, time.time() - t), flush=True)
    d = np.abs(out["exact"] - out["perturbed 1e-5"]).max() / out["exact"].max()
    print("largest relative difference of the %d leading singular values: %.2e" % (k, d))


if __name__ == "__main__":
    main()
