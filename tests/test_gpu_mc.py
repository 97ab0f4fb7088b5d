"""Monte-Carlo neutral hydrogen (titan_mc_sources): properties the reference's
MK_fly_immit physics must have. The reference's Monte-Carlo keeps no momentum
or energy tallies and its seeds file is absent, so these are statistical checks,
not a pin: free streaming fills a convex box uniformly; an unperturbed
Maxwellian passing through protons at rest exchanges momentum and energy at
the rates of the Maxwell-averaged Bera formulas, to the accuracy those
averages have; a seed reproduces its tallies."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box(titan, n, rho, p, nh_fluid=0):
    m = titan.mesh.cube_mesh(n)
    C = m["cell_nodes"].shape[0]
    st = np.zeros((10, C))
    st[0], st[4] = rho, p
    prm = titan.problems.params(nh=nh_fluid)
    return m, prm, st


def test_free_streaming_fills_a_convex_box_uniformly(titan):
    m, prm, st = _box(titan, 8, 1e-12, 1e-12)   # no protons: no exchange
    g = titan.PlasmaStep(m, prm)
    g.upload_state(st)
    out, info = g.mc_sources(n_H=0.18, u_H=(-2.6, 0.3, 0.0), cp_H=1.2, n_particles=2_000_000, seed=7,
                             face_types=1 << 3)
    g.close()
    assert info["lost"] == 0
    nH = out[0]
    assert abs(nH.mean() / 0.18 - 1.0) < 0.01
    # each cell: statistical scatter only
    assert np.std(nH / 0.18) < 0.05
    assert np.abs(out[1:]).max() < 1e-12 * 0.18


def test_exchange_rates_agree_with_the_bera_averages(titan, oracle_lib):
    """Thin plasma at rest: the neutrals stay an undisturbed drifting Maxwellian,
    so the MC momentum / energy sources follow the Maxwell-averaged rates of
    Calc_sourse_MF_Bera (Setka_physics.cpp:746-1031) for that Maxwellian."""
    import oracle_lib as ol

    rho, p = 1e-3, 1e-3 * 0.5
    nH, uH, cpH = 0.18, (-2.6, 0.0, 0.0), 1.2
    m, prm, st = _box(titan, 6, rho, p)
    g = titan.PlasmaStep(m, prm)
    g.upload_state(st)
    out, info = g.mc_sources(n_H=nH, u_H=uH, cp_H=cpH, n_particles=4_000_000, seed=3, face_types=1 << 3)
    g.close()
    assert info["lost"] == 0
    # Bera with one H fluid carrying the same Maxwellian (T = cp^2, densities in units of n_H_LISM)
    prm_b = titan.problems.params(nh=1)
    run = ol.OracleRun(m, prm_b)
    C = m["cell_nodes"].shape[0]
    H = np.zeros((5, C))
    H[0] = nH / prm_b["par_n_H_LISM"]
    H[1], H[2], H[3] = uH
    H[4] = 0.5 * H[0] * cpH ** 2
    S = np.empty((C, 4))
    import ctypes
    ol.oracle().oracle_sources(ctypes.byref(run.mesh), ctypes.byref(run.params), ol._p(np.ascontiguousarray(st)),
                               ol._p(np.ascontiguousarray(H)), ol._p(S))
    mc_mx = out[1].mean()
    bera_mx = S[:, 0].mean()
    assert np.sign(mc_mx) == np.sign(bera_mx)
    assert abs(mc_mx / bera_mx - 1.0) < 0.25, (mc_mx, bera_mx)
    mc_e = out[4].mean()
    bera_e = S[:, 3].mean()
    assert abs(mc_e / bera_e - 1.0) < 0.35, (mc_e, bera_e)


def test_seed_reproduces_and_seeds_agree_statistically(titan):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=8, move=False)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    kw = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=1.3, n_particles=400_000)
    a, ia = g.mc_sources(seed=11, **kw)
    b, _ = g.mc_sources(seed=11, **kw)
    c, _ = g.mc_sources(seed=12, **kw)
    g.close()
    # the same seed: the same histories; only the order of the atomic tallies varies
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14 * np.abs(a).max())
    assert ia["lost"] == 0
    # a different seed: the same density field within Monte-Carlo noise
    tot_a, tot_c = a[0].sum(), c[0].sum()
    assert abs(tot_a / tot_c - 1.0) < 0.02


def test_inflow_rate_is_the_maxwellian_flux_through_the_open_faces(titan):
    """The device's inflow split (a fixed-order scan over all faces) totals the
    drifting Maxwellian's flux through the inward normal of every face whose
    type is open, n [cp e^{-s^2} / (2 sqrt(pi)) + u_n (1 + erf s) / 2] times the
    area (s = u_n / cp), as numpy sums it from the downloaded geometry; a second
    pass gives the identical total."""
    from scipy.special import erf

    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=8, move=False)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    nH, uH, cpH, types = 0.18, np.array([-2.6, 0.3, 0.1]), 1.3, (1 << 2) | (1 << 3)
    kw = dict(n_H=nH, u_H=tuple(uH), cp_H=cpH, n_particles=50_000, seed=1, face_types=types)
    _, info = g.mc_sources(**kw)
    _, info2 = g.mc_sources(**kw)
    geo = g.geometry()
    g.close()
    ft = m["face_type"].astype(np.int64)
    open_ = (ft > 0) & (((types >> np.clip(ft, 0, 31)) & 1) == 1)
    assert open_.any() and not open_.all()
    un = -(geo["face_normal"][open_] @ uH)
    sr = un / cpH
    flux = nH * (cpH * np.exp(-sr * sr) / (2.0 * np.sqrt(np.pi)) + 0.5 * un * (1.0 + erf(sr)))
    expected = float((flux * geo["face_area"][open_]).sum())
    assert info["inflow_rate"] == pytest.approx(expected, rel=1e-12)
    assert info2["inflow_rate"] == info["inflow_rate"]
