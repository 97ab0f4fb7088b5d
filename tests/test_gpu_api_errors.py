"""The C ABI refuses what it cannot do with TITAN_EINVAL and a message, and the
context stays usable afterwards (the reference's convention is print and
exit; here the caller decides)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _shell(titan, move):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=move)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    return m, g


def _refused(titan, fn, text):
    with pytest.raises(titan.native.TitanError) as e:
        fn()
    assert "TITAN_EINVAL" in str(e.value) and text in str(e.value), str(e.value)


def test_refusals_leave_the_context_usable(titan):
    m, g = _shell(titan, move=False)
    rays = titan.mesh.shell_rays(m)
    # surface tracking needs a moving mesh
    _refused(titan, lambda: g.set_surface_motion(rays, move_HP=1, velocity_HP=1.0), "move = 1")
    # the device fallback needs an envelope and a pass
    _refused(titan, lambda: titan.native.check(titan.native.lib().titan_closure_fallback_from_mc(g.ctx)),
             "envelope")
    # no face of the requested types lets neutrals in
    _refused(titan, lambda: g.mc_sources(n_H=0.18, u_H=(-2.6, 0, 0), cp_H=1.3, n_particles=1000,
                                         face_types=1 << 7), "no inflow")
    # halo ids out of range
    _refused(titan, lambda: g.set_halo(np.array([g.ncell], np.int32), np.zeros(0, np.int32)), "out of range")
    g.go(3)
    assert np.isfinite(g.download_state()).all()
    g.close()


def test_bad_rays_are_refused(titan):
    m, g = _shell(titan, move=True)
    rays = titan.mesh.shell_rays(m)
    short = rays[:, :1].copy()
    _refused(titan, lambda: g.set_surface_motion(short, move_HP=1, velocity_HP=1.0), "ray")
    gap = rays.copy()
    gap[0, 2] = -1                          # padding must run to the end of the row
    _refused(titan, lambda: g.set_surface_motion(gap, move_HP=1, velocity_HP=1.0), "padding")
    far = rays.copy()
    far[0, 1] = g.nnode
    _refused(titan, lambda: g.set_surface_motion(far, move_HP=1, velocity_HP=1.0), "out of range")
    g.go(2)
    assert np.isfinite(g.download_state()).all()
    g.close()
