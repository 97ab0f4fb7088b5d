"""Synthetic problems of the benchmark configurations (seeded, no external data).

* ``brio_wu_cube``     — 32^3 unit cube, Brio-Wu Riemann problem along
  (1,1,0)/sqrt(2), zero-gradient boundaries, HLLD on every face, CFL 0.4.
* ``heliosphere_shell`` — cubed-sphere shell r in [1, 100], 6 nq^2 x nlayer
  cells: radial supersonic wind with a Parker-spiral field inside, uniform
  interstellar inflow outside, seeded lognormal perturbation of rho and p,
  HLLD where B^2/(8 pi p) > 0.01 else HLLC, prescribed radial node motion.

Units: the state stores B in the reference's Gaussian form (Cell::parameters);
the solver works with b = B / sqrt(4 pi). Field amplitudes quoted for the
problems are in the solver's units b, so the stored B is sqrt(4 pi) * b.
"""
from __future__ import annotations

import numpy as np

from . import mesh as _mesh

SPI4 = np.sqrt(4.0 * np.pi)
GAMMA = 5.0 / 3.0

# Phys_param defaults (TITAN/source/Phys_param.h:107-114, :118-120)
DEFAULT_PARAMS = dict(
    gamma=GAMMA, KFL=0.4, velosity_inf=-2.54327, omega=2.0 * np.pi, par_a_2=0.102046, par_n_H_LISM=3.0,
    par_Kn=40.0906, beta_switch=0.01, move=0, soft_fixups=1, method_policy=0, npassive=0, nh=0, TS_hard=0,
    contact_hard=0, flux_precision=64, tvd=0, snos_on_hp=0, bn_in_p_on_hp=0,
)


def params(**over) -> dict:
    p = dict(DEFAULT_PARAMS)
    for k, v in over.items():
        if k not in p:
            raise KeyError(k)
        p[k] = v
    return p


def brio_wu_cube(n: int = 32):
    """(mesh, params, state [10, C], face_method [F])."""
    return brio_wu_box(n, n, n)


def brio_wu_box(nx: int, ny: int, nz: int):
    """The Brio-Wu problem of brio_wu_cube on the unit box cut into nx x ny x nz
    hexahedra: (mesh, params, state [10, C], face_method [F])."""
    m = _mesh.box_mesh(nx, ny, nz)
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    nrm = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
    tng = np.array([-1.0, 1.0, 0.0]) / np.sqrt(2.0)
    s = (cc - 0.5) @ nrm
    left = s < 0.0
    C = cc.shape[0]
    st = np.zeros((10, C))
    st[0] = np.where(left, 1.0, 0.125)
    st[4] = np.where(left, 1.0, 0.1)
    bt = np.where(left, 1.0, -1.0)
    B = SPI4 * (0.75 * nrm[None, :] + bt[:, None] * tng[None, :])
    st[5:8] = B.T
    p = params(KFL=0.4, soft_fixups=0, method_policy=0)
    method = np.full(m["face_nodes"].shape[0], 3, dtype=np.int8)
    return m, p, st, method


def _parker_wind(x: np.ndarray, rho0=1.0, u0=1.0, mach=10.0, b0=0.1, gamma=GAMMA):
    """Radial wind with rho ~ r^-2, |u| = u0, p ~ r^-2gamma and a Parker spiral
    (b_r = b0 / r^2, b_phi = -b0 sin(theta) / r)."""
    r = np.linalg.norm(x, axis=1)
    rh = x / r[:, None]
    rho = rho0 / r ** 2
    p0 = rho0 * (u0 / mach) ** 2 / gamma
    p = p0 / r ** (2.0 * gamma)
    V = u0 * rh
    sin_th = np.sqrt(np.maximum(x[:, 0] ** 2 + x[:, 1] ** 2, 0.0)) / r
    ephi = np.stack([-x[:, 1], x[:, 0], np.zeros_like(r)], axis=1)
    nphi = np.linalg.norm(ephi, axis=1)
    ephi = np.where(nphi[:, None] > 0, ephi / np.maximum(nphi[:, None], 1e-300), 0.0)
    b = (b0 / r ** 2)[:, None] * rh - (b0 * sin_th / r)[:, None] * ephi
    return rho, V, p, SPI4 * b


def _lism(n: int, rho=0.06, u=2.6, mach=2.0, b=0.3, angle_deg=60.0, gamma=GAMMA):
    p = rho * (u / mach) ** 2 / gamma
    V = np.tile(np.array([-u, 0.0, 0.0]), (n, 1))
    a = np.deg2rad(angle_deg)
    bv = b * np.array([-np.cos(a), np.sin(a), 0.0])
    return np.full(n, rho), V, np.full(n, p), np.tile(SPI4 * bv, (n, 1))


def heliosphere_shell(nq: int = 96, nlayer: int = 40, seed: int = 20261203, move: bool = True,
                      zones: bool = False, npassive: int = 0, nh: int = 0, flux_precision: int = 64,
                      r_mid: float = 25.0, width: float = 3.0, amp: float = 1e-3, tvd: bool = False,
                      radii: np.ndarray | None = None):
    """(mesh, params, state [10, C], hfluids [5 nh, C] or None); radii: the
    nlayer + 1 node radii of the layers instead of geometric spacing."""
    m = _mesh.shell_mesh(nq, nlayer, radii=radii)
    rng = np.random.default_rng(seed)
    xyz = m["node_xyz"]
    cc = xyz[m["cell_nodes"]].mean(axis=1)
    C = cc.shape[0]
    r = np.linalg.norm(cc, axis=1)

    # boundary values (Init_physics, Setka_physics.cpp:470-568, with this problem's states)
    ftype = m["face_type"]
    hard = np.nonzero((ftype == 1) | (ftype == 2))[0]
    fcen = xyz[m["face_nodes"][hard]].mean(axis=1)
    bc = np.zeros((len(hard), 10))
    inner = ftype[hard] == 1
    rho, V, p, B = _parker_wind(fcen[inner])
    bc[inner, 0], bc[inner, 1:4], bc[inner, 4], bc[inner, 5:8] = rho, V, p, B
    bc[inner, 8] = rho                      # Q = rho on the inner sphere
    rho, V, p, B = _lism(int((~inner).sum()))
    bc[~inner, 0], bc[~inner, 1:4], bc[~inner, 4], bc[~inner, 5:8] = rho, V, p, B
    bc[~inner, 8] = 100.0 * rho             # Q = 100 rho in the interstellar medium
    m["face_bc"][hard] = np.arange(len(hard), dtype=np.int32)
    m["bc_vals"] = np.ascontiguousarray(bc)

    # initial state: wind blended into the interstellar flow around r_mid
    w = 0.5 * (1.0 + np.tanh((r - r_mid) / width))
    rs, Vs, ps, Bs = _parker_wind(cc)
    rl, Vl, pl, Bl = _lism(C)
    st = np.zeros((10, C))
    st[0] = (1 - w) * rs + w * rl
    st[1:4] = ((1 - w)[:, None] * Vs + w[:, None] * Vl).T
    st[4] = (1 - w) * ps + w * pl
    st[5:8] = ((1 - w)[:, None] * Bs + w[:, None] * Bl).T
    st[0] *= np.exp(0.01 * rng.standard_normal(C))
    st[4] *= np.exp(0.01 * rng.standard_normal(C))
    if npassive:
        st[8] = st[0] * ((1 - w) * 1.0 + w * 100.0)
        st[9] = 0.0

    # cells touching the inner sphere keep their field (Init_physics sets is_TVD = false)
    inner_cells = m["face_cells"][ftype == 1, 0]
    m["cell_tvd"][inner_cells] = 0
    if zones:
        ct = np.full(C, 3, dtype=np.int8)
        ct[r < 30.0] = 2
        ct[r < 10.0] = 1
        ct[(r >= 30.0) & (cc[:, 0] > 40.0)] = 4
        m["cell_type"] = ct

    # prescribed radial node motion: interior node layers, phase seeded per ray
    if move:
        layer = m["node_layer"]
        phase_ray = rng.uniform(0.0, 2.0 * np.pi, m["node_ray"].max() + 1)
        a = np.where((layer > 0) & (layer < nlayer), amp, 0.0)
        m["node_amp"] = np.ascontiguousarray(a)
        m["node_phase"] = np.ascontiguousarray(phase_ray[m["node_ray"]])

    prm = params(KFL=0.4, soft_fixups=1, method_policy=1, beta_switch=0.01, move=int(move),
                 npassive=npassive, nh=nh, flux_precision=flux_precision, tvd=int(tvd))
    hf = None
    if nh:
        hf = np.zeros((5 * nh, C))
        for k in range(nh):
            nH = 0.18 if k == nh - 1 else 1e-3 * (k + 1)
            hf[5 * k + 0] = nH * np.exp(0.05 * rng.standard_normal(C))
            hf[5 * k + 1] = -2.6 + 0.1 * rng.standard_normal(C)
            hf[5 * k + 2] = 0.1 * rng.standard_normal(C)
            hf[5 * k + 3] = 0.1 * rng.standard_normal(C)
            hf[5 * k + 4] = 0.5 * hf[5 * k + 0] * (1.0 + 0.1 * k)
    return m, prm, st, hf


def gaussian_to_solver_b(B: np.ndarray) -> np.ndarray:
    return B / SPI4
