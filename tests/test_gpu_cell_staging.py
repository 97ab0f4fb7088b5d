"""The staged cell update (face records in shared memory) against the plain one.

The staged launch shapes (cell variants 6-8) copy the face records owned by a
block's cells with one bulk copy into shared memory and the records of the
cells' other faces with per-thread cp.async into slots; records beyond the
stage's capacity or the slots are read from global memory. The sums run in
the same face order as the plain kernel, so every result must be identical:
state, dt and time, after several steps, in every source mode and with the
passive scalars. The meshes are chosen so that each fallback runs: the 1x1x300
column owns 5 faces per cell (more than the 4.25 the stage holds), the
variant with one slot per thread sends many records to global memory, and the
cell counts leave a partial last block.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NET = os.path.join(ROOT, "titan_c-_b200", "data", "closure_shell.npz")
PLAIN = (0, 3)
STAGED = (6, 7, 8)


def _column(T, n=300):
    """A shock tube along z in a 1 x 1 x n column of cells."""
    m = T.mesh.box_mesh(1, 1, n, (1.0 / n, 1.0 / n, 1.0))
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    left = cc[:, 2] < 0.5
    st = np.zeros((10, n))
    st[0] = np.where(left, 1.0, 0.125)
    st[4] = np.where(left, 1.0, 0.1)
    st[5] = np.sqrt(4.0 * np.pi) * np.where(left, 1.0, -1.0)
    st[7] = np.sqrt(4.0 * np.pi) * 0.75
    p = T.problems.params(KFL=0.4, soft_fixups=0, method_policy=0)
    return m, p, st, np.full(m["face_nodes"].shape[0], 3, dtype=np.int8)


def _run(T, m, p, st, cv, steps, method=None, hf=None, net=None):
    g = T.PlasmaStep(m, p)
    if method is not None:
        g.set_face_method(method)
    g.set_tuning(0, cv)
    g.upload_state(st)
    if hf is not None:
        g.upload_hfluids(hf)
    if net is not None:
        net.install(g)
    info = g.go(steps)
    assert info["steps_done"] == steps
    out = (g.download_state(), g.dt, info["t"])
    g.close()
    return out


def _same(a, b):
    assert np.array_equal(a[0], b[0])
    assert a[1] == b[1] and a[2] == b[2]


def _check(T, m, p, st, steps=4, **kw):
    ref = _run(T, m, p, st, PLAIN[0], steps, **kw)
    for cv in PLAIN[1:] + STAGED:
        _same(_run(T, m, p, st, cv, steps, **kw), ref)


def test_staged_update_column_beyond_stage_capacity(titan):
    m, p, st, meth = _column(titan)
    _check(titan, m, p, st, steps=6, method=meth)


def test_staged_update_moving_shell_with_zones_and_passive_scalars(titan):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=6, move=True, zones=True, npassive=2)
    _check(titan, m, p, st)


def test_staged_update_with_bera_sources(titan):
    m, p, st, hf = titan.problems.heliosphere_shell(nq=8, nlayer=5, move=True, zones=True, nh=2)
    _check(titan, m, p, st, hf=hf)


def test_staged_update_with_closure_sources_mixed_step(titan):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=10, nlayer=6, move=True, flux_precision=32)
    net = titan.closure.Closure.load(NET)
    _check(titan, m, p, st, net=net)


def test_staged_variant_is_picked_by_the_autotuner_or_timed(titan):
    """The autotuner times the staged shapes beside the plain ones on a shell."""
    m, p, st, _ = titan.problems.heliosphere_shell(nq=16, nlayer=10, move=True)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    t = g.autotune(reps=2)
    assert 0 <= t["cell_variant"] < 9
    g.go(2)
    g.close()
