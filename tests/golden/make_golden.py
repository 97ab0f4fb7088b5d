"""Generates tests/golden/chlld_golden.npz from the reference's own Riemann solver.

    make -C oracle ref && python tests/golden/make_golden.py

Runs Phys_param::chlld (TITAN/source/Phys_param.cpp:882-1878), compiled
unmodified from the reference tree into oracle/_ref/libtitan_ref.so, on seeded
random face problems covering all four solvers, the four wave-speed estimates,
the null_bn / left_ydar / contact flags and two passive scalars, and stores
inputs and outputs. The GPU and oracle tests compare against this file where
the reference tree is not available.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402


def main(n_per_combo: int = 24, seed: int = 20261203):
    ol.build_oracle(ref=True)
    rng = np.random.default_rng(seed)
    combos = []
    for ns in range(4):
        for nd in range(4):
            combos.append((ns, nd, 0, 0, 0))
        for fl in [(1, 0, 0), (0, 1, 0), (0, 0, 1)]:
            combos.append((ns, 0) + fl)
    n = n_per_combo * len(combos)
    nrm, w, q1, q2 = ol.random_riemann_cases(n, seed=seed)
    rec = {k: [] for k in ["n_state", "n_disc", "null_bn", "left_ydar", "contact", "nk", "kl", "kr", "flux",
                           "kout", "ds"]}
    for c, (ns, nd, nb, ly, ct) in enumerate(combos):
        for j in range(n_per_combo):
            i = c * n_per_combo + j
            nk = int(rng.integers(0, 3))
            kl = np.zeros(2)
            kr = np.zeros(2)
            kl[:nk] = q1[i, 0] * rng.uniform(0.0, 1.0, nk)
            kr[:nk] = q2[i, 0] * rng.uniform(0.0, 1.0, nk)
            out, kout, ds, _ = ol.chlld("ref", ns, nrm[i], w[i], q1[i], q2[i], n_disc=nd, null_bn=nb,
                                        left_ydar=ly, contact=ct, kl=tuple(kl[:nk]), kr=tuple(kr[:nk]))
            ko = np.zeros(2)
            ko[:nk] = kout
            for k, v in zip(["n_state", "n_disc", "null_bn", "left_ydar", "contact", "nk", "kl", "kr", "flux",
                             "kout", "ds"], [ns, nd, nb, ly, ct, nk, kl, kr, out, ko, ds]):
                rec[k].append(v)
    arrs = {k: np.array(v) for k, v in rec.items()}
    np.savez_compressed(os.path.join(HERE, "chlld_golden.npz"), nrm=nrm, w=w, q1=q1, q2=q2, **arrs)
    print("wrote", n, "cases")


if __name__ == "__main__":
    main()
