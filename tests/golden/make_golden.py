"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference has no test vectors of its own, so these fixtures are the
outputs of the reference's inline CUDA kernels compiled for the host
(``oracle/_ref``, built by ``python oracle/build_ref.py`` from the reference
tree) on small seeded inputs, glued the way the reference's drivers glue
them.  They pin the oracle (tests/test_oracle_pinning.py) and, through it,
the CUDA product, on machines where the reference tree is absent.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_runner as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def gen_rf(rng):
    N = 6
    ha = rng.uniform(0.08, 0.3, N)
    hl = rng.uniform(0, np.pi, N)
    hx = rng.uniform(-0.3, 0.3, N)
    hy = rng.uniform(-0.3, 0.3, N)
    hab = (np.arange(N) % 2).astype(np.int32)
    gab = R.gabor(ha, hl, hx, hy, hab, 24, 20, 1.0, 0.9, -0.5, -0.45, 2.5)
    cs = R.cs(ha, hx, hy, 24, 20, 1.0, 0.9, -0.5, -0.45, 0.05, 0.15)
    fine = R.gabor(ha, hl, hx, hy, hab, 64, 64, 1.0, 1.0, -0.5, -0.5, 2.5)
    Ds = R.compute_Ds(fine, 3, 2, (1 / 64) ** 2)
    dirich = R.dirich_space_fft(Ds, 3, 2, 16, 14, 16, 16)
    norm = rng.uniform(0.5, 1.0, N)
    Dsw = R.compute_Dsw(Ds, norm)
    np.savez_compressed(os.path.join(OUT, "rf_dirichlet.npz"), h_alpha=ha, h_l=hl, h_x0=hx, h_y0=hy, h_ab=hab,
                        gabor=gab, cs=cs, fine=fine, Ds=Ds, dirich=dirich, norm=norm, Dsw=Dsw)


def gen_iaf(rng):
    N, F = 8, 400
    L = rng.standard_normal((F, N)) * 0.6
    L[150:170, 3] = -2.5            # drive neuron 3 through the negative-slope branch
    kap = rng.uniform(0.8, 1.2, N)
    bia = np.full(N, 0.8)
    dl = rng.uniform(0.008, 0.015, N)
    v0 = rng.uniform(0, 1, N) * dl
    dt = 1e-3
    out = {"L": L, "kappa": kap, "bias": bia, "delta": dl, "v0": v0, "dt": dt}
    a, b = v0.copy(), np.zeros(N)
    sp, cnt = R.iaf_encode(L, dt, kap, bia, dl, a, b)
    out.update(lin_counts=cnt, lin_spikes=np.concatenate(sp), lin_v0=a, lin_tc=b)
    sig = rng.uniform(5e-4, 1.5e-3, N)
    randn = rng.standard_normal((int(np.ceil(F / 0.1)), N))
    dv = dl + sig * rng.standard_normal(N)
    a, b, c = v0.copy(), np.zeros(N), dv.copy()
    sp, cnt = R.iaf_encode(L, dt, kap, bia, dl, a, b, randn=randn, sigma=sig, delta_value=c)
    out.update(sigma=sig, randn=randn, delta_value0=dv, rt_counts=cnt, rt_spikes=np.concatenate(sp), rt_v0=a,
               rt_tc=b, rt_dv=c)
    # two consecutive blocks of VTEM_IAF (101 frames each, one shared frame)
    a, b = v0.copy(), np.zeros(N)
    blocks = []
    for s in (0, 100, 200, 300):
        sp, cnt = R.iaf_encode(L[s:s + 101], dt, kap, bia, dl, a, b)
        blocks.append((cnt, np.concatenate(sp)))
        b[:] = 0
    out.update(blk_counts=np.stack([c for c, _ in blocks]),
               blk_spikes=np.concatenate([s for _, s in blocks]), blk_v0=a)
    np.savez_compressed(os.path.join(OUT, "iaf.npz"), **out)


def gen_decode(rng):
    N, n = 6, 96
    tk1 = np.sort(rng.uniform(0, 0.2, n))
    tk2 = tk1 + rng.uniform(0.005, 0.03, n)
    ind = np.sort(rng.integers(0, N, n)).astype(np.int32)
    kap = rng.uniform(0.8, 1.2, N)
    dl = rng.uniform(0.01, 0.05, N)
    bia = rng.uniform(1, 3, N)
    norm = rng.uniform(0.5, 1.0, N)
    D = rng.standard_normal((N, 9)) + 1j * rng.standard_normal((N, 9))
    Dsw = (np.conj(D) @ D.T).real
    Wt, Mt = 2 * np.pi * 20, 4
    q = R.compute_q(tk1, tk2, ind, kap, dl, bia, norm)
    G = R.compute_G(tk1, tk2, ind, Dsw, Wt, Mt)
    Gl = R.compute_G(tk1, tk2, ind, Dsw, Wt, Mt, lamb=0.05)
    c = R.solve_eq_sym(G.copy(), q, 1e-8)
    cr = R.rnn3(G, q, 1e-6, 5000, 60)
    dirich = rng.standard_normal((N, 5, 7))
    t = np.arange(0, 0.02, 2e-3)
    u = R.reconstruct(dirich, tk1, tk2, c, t, ind, norm, Mt, Wt / Mt)
    np.savez_compressed(os.path.join(OUT, "decode.npz"), tk1=tk1, tk2=tk2, ind=ind, kappa=kap, delta=dl, bias=bia,
                        norm=norm, Dsw=Dsw, Wt=Wt, Mt=Mt, q=q, G=G, G_lamb=Gl, c=c, c_rnn=cr, dirich=dirich, t=t,
                        u=u)


def main():
    if not R.available():
        print("oracle/_ref is not built; run python oracle/build_ref.py first")
        return 1
    rng = np.random.default_rng(20260101)
    gen_rf(rng)
    gen_iaf(rng)
    gen_decode(rng)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
