"""Generate the golden fixtures of the interpolation path from the reference
itself.

Run in a tree where the reference source is present (``make -C oracle ref``
compiles src/gemdyn/src/base/turbo_tricublin.c unchanged into oracle/_ref/).
Outputs, committed next to this script:

* ``selftest_reference.txt`` — stdout of the reference's own SELF_TEST
  (turbo_tricublin.c:1314-1506), AVX2 build, timing line removed.
* ``tricublin_ref_vectors.npz`` — inputs and outputs of the reference's
  Tricublin_zyx1_m_n, Tricublin_mono_zyx_m_n (AVX2 and scalar builds) and
  Tricublin_zyx3_n on a small non-uniform grid, random positions plus the
  boundary cases the reference documents (linear z in the first/last two
  intervals, extrapolation below 1 and above nk, integer positions, x/y at the
  edge of the cubic range).

usage: python tests/golden/make_golden.py
"""
import os
import resource
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def levels_height(nk, top=25000.0, dz0=20.0, seed=0):
    """Decreasing heights (GEM height coordinate: k=1 at the top)."""
    th = np.geomspace(dz0, 1000.0, nk)
    z = np.cumsum(th)[::-1].copy()
    return z * (top / z[0])


def main():
    O.build(ref=True)
    # --- SELF_TEST of the reference ---
    def unlimited():
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    out = subprocess.run([os.path.join(O.REF_DIR, "selftest")], capture_output=True, text=True, check=True,
                         preexec_fn=unlimited).stdout
    lines = [ln for ln in out.splitlines() if "cycles per interpolation" not in ln]
    with open(os.path.join(HERE, "selftest_reference.txt"), "w") as fh:
        fh.write("\n".join(lines) + "\n")

    # --- interpolator vectors ---
    rng = np.random.default_rng(20240611)
    ni, nj, nk = 21, 19, 12            # extended array extents (halo included)
    offi, offj = 3, 2                  # Vsearch_setup_plus offsets
    base = 0                           # kernel pointer = array start (offsets compensate)
    lev = levels_height(nk)
    fields = [(rng.standard_normal(ni * nj * nk) * 5 + 2).astype(np.float32) for _ in range(3)]
    f3 = (rng.standard_normal(3 * ni * nj * nk) * 3).astype(np.float32)
    # global positions: px + offi in [2, ni-2) keeps the 4-wide stencil inside
    n_rand = 3000
    px = rng.uniform(2.0 - offi, ni - 2.0 - offi - 1e-3, n_rand)
    py = rng.uniform(2.0 - offj, nj - 2.0 - offj - 1e-3, n_rand)
    pz = rng.uniform(0.3, nk + 0.7, n_rand)
    pos = np.stack([px, py, pz], 1).astype(np.float32)
    edge = []
    xs = [2.0 - offi, 5.0, 7.5, ni - 2.0 - offi - 2e-3]
    ys = [2.0 - offj, 4.0, 9.25, nj - 2.0 - offj - 2e-3]
    zs = [0.0, 0.5, 1.0, 1.5, 2.0, 2.5, 3.0, nk - 2.0, nk - 1.5, nk - 1.0, nk - 0.5, nk, nk + 0.5, nk + 1.0]
    for x in xs:
        for y in ys:
            for z in zs:
                edge.append((x, y, z))
    pos = np.concatenate([pos, np.array(edge, np.float32)], 0)
    R = O.RefKernels()
    zt = R.setup(lev, ni, nj, offi, offj)
    views = [f[base:] for f in fields]
    d1 = R.zyx1_m_n(views, pos, zt)
    d, lin, mi, ma = R.mono_m_n(views, pos, zt)
    d3 = R.zyx3_n(f3, pos, zt)
    RS = O.RefKernels(scalar=True)
    zs_ = RS.setup(lev, ni, nj, offi, offj)
    sd, slin, smi, sma = RS.mono_m_n(views, pos, zs_)
    np.savez_compressed(os.path.join(HERE, "tricublin_ref_vectors.npz"),
                        ni=ni, nj=nj, nk=nk, offi=offi, offj=offj, levels=lev,
                        fields=np.stack(fields), f3=f3, pos=pos,
                        zyx1=d1, mono_d=d, mono_lin=lin, mono_min=mi, mono_max=ma, zyx3=d3,
                        scalar_mono_d=sd, scalar_mono_lin=slin, scalar_mono_min=smi, scalar_mono_max=sma)
    print("wrote", HERE)


if __name__ == "__main__":
    main()
