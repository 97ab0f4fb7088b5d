"""Generates tests/golden/godunov_golden.npz from the reference's own exact
Godunov solver of HP faces (Phys_param::Godunov_Solver_Alexashov,
TITAN/source/Phys_param.cpp:1938-2385), compiled unmodified from the reference
tree into oracle/_ref/libtitan_ref.so:

    make -C oracle ref && python tests/golden/make_godunov_golden.py

Seeded face problems over the four wave patterns (two shocks, shock +
rarefaction, two rarefactions, vacuum), both pressure orders and the contact
flag. The oracle and GPU tests compare against this file.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402


def main(n: int = 2000, seed: int = 20261204):
    ol.build_oracle(ref=True)
    nrm, w, q1, q2 = ol.random_godunov_cases(n, seed=seed)
    contact = (np.arange(n) % 5 == 4).astype(np.int32)
    flux, ds = np.zeros((n, 5)), np.zeros((n, 3))
    for i in range(n):
        flux[i], ds[i], _ = ol.godunov("ref", nrm[i], w[i], q1[i], q2[i], contact=contact[i])
    np.savez_compressed(os.path.join(HERE, "godunov_golden.npz"), nrm=nrm, w=w, q1=q1, q2=q2, contact=contact,
                        flux=flux, ds=ds)
    print(f"{n} cases")


if __name__ == "__main__":
    main()
