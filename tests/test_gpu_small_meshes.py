"""Edge cases of mesh size and shape, through the C ABI against the oracle.

* A single cell: all six faces lie on the boundary, so no face bounds the CFL
  step and the next dt is a face's initial candidate, 1e7 (Setka::
  Culc_Gran_Potok, Setka_physics.cpp:2296); the closed box's fluxes cancel and
  the steps taken with that dt must agree bit for bit.
* A one-cell-thick column and ragged boxes whose cell and face counts fill
  neither a warp nor a block (the renumbering's space-filling curve over
  non-power-of-two extents, partial 32-cell chunks of the staged cell update).
* The ragged box under every launch shape the autotuner can choose, the
  staged cell update included: identical states.

The Brio-Wu problem (HLLD on every face, no transcendental function) keeps
every comparison bit-exact."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _pair(T, dims):
    m, p, st, meth = T.problems.brio_wu_box(*dims)
    gpu = T.PlasmaStep(m, p)
    gpu.set_face_method(meth)
    run = ol.OracleRun(m, p)
    run.set_face_method(meth)
    return gpu, run, st


@pytest.mark.parametrize("dims,steps", [((1, 1, 1), 3), ((1, 40, 1), 6), ((3, 1, 2), 6), ((5, 7, 3), 6),
                                        ((33, 2, 5), 6)])
def test_small_and_ragged_boxes_match_oracle_bit_for_bit(titan, oracle_lib, dims, steps):
    gpu, run, st = _pair(titan, dims)
    gpu.upload_state(st)
    s_or = np.ascontiguousarray(st.copy())
    info = gpu.go(steps)
    oi = run.go(s_or, steps)
    assert info["steps_done"] == steps and oi.err_code == 0
    s_gpu = gpu.download_state()
    assert np.array_equal(s_gpu[:8].view(np.uint64), s_or[:8].view(np.uint64))
    assert gpu.dt == run.clock[0] and gpu.t == run.clock[1]
    if dims == (1, 1, 1):
        assert gpu.dt == 1e7
    gpu.close()


def test_ragged_box_under_every_launch_shape(titan):
    m, p, st, meth = titan.problems.brio_wu_box(33, 2, 5)
    outs = []
    for fv in range(7):
        for cv in range(9):
            if cv and fv:
                continue
            g = titan.PlasmaStep(m, p)
            g.set_face_method(meth)
            g.set_tuning(fv, cv)
            g.upload_state(st)
            g.go(5)
            outs.append(g.download_state())
            g.close()
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint64), outs[0].view(np.uint64))
