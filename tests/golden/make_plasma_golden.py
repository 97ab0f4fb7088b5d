"""Generates tests/golden/plasma_components_golden.npz from the reference's own
thermal-proton split (Phys_param::Plasma_components_1,
TITAN/source/Phys_param.cpp:628-665), compiled unmodified from the reference
tree into oracle/_ref/libtitan_ref.so:

    make -C oracle ref && python tests/golden/make_plasma_golden.py

Seeded cells (density, pressure, helium density) for each of the 0-based zones
0-3 the step calls it with, including helium-rich cells whose proton density
and temperature are floored by the caller. tests/test_oracle_bera_numpy.py
compares its restatement against this file without the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402


def main(n: int = 400, seed: int = 20261205):
    ol.build_oracle(ref=True)
    rng = np.random.default_rng(seed)
    zone = np.repeat(np.arange(4, dtype=np.int32), n)
    rho = 10.0 ** rng.uniform(-4.0, 1.0, 4 * n)
    p = 10.0 ** rng.uniform(-6.0, 1.0, 4 * n)
    rho_he = rho * rng.uniform(0.0, 0.3, 4 * n)
    rho_he[::17] = rho[::17] * rng.uniform(0.9, 1.1, len(rho[::17]))   # helium-rich cells
    out = np.zeros((4 * n, 3))
    L = ol.ref()
    o = np.zeros(3)
    for i in range(4 * n):
        L.titan_ref_plasma_components_1(int(zone[i]), float(rho[i]), float(p[i]), float(rho_he[i]), ol._p(o))
        out[i] = o
    np.savez_compressed(os.path.join(HERE, "plasma_components_golden.npz"), zone=zone, rho=rho, p=p,
                        rho_he=rho_he, out=out)
    print(f"{4 * n} cells")


if __name__ == "__main__":
    main()
