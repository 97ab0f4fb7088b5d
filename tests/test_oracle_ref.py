"""Pins the oracle's Riemann solver to the reference's own compiled Phys_param::chlld.

The reference solver (TITAN/source/Phys_param.cpp:882-1878) is compiled
unmodified by `make -C oracle ref` where the reference tree exists; elsewhere
the committed golden vectors (tests/golden/chlld_golden.npz, produced by the
same compiled solver) stand in for it.
"""
import numpy as np
import pytest

import oracle_lib as ol


def _cases():
    return ol.random_riemann_cases(600, seed=11)


@pytest.mark.skipif(not ol.ref_available(), reason="reference solver not built (no reference tree)")
@pytest.mark.parametrize("n_state", [0, 1, 2, 3])
@pytest.mark.parametrize("n_disc", [0, 1, 2, 3])
def test_oracle_chlld_bitwise_vs_reference(oracle_lib, n_state, n_disc):
    nrm, w, q1, q2 = _cases()
    for i in range(0, 600, 3):
        kl = (q1[i, 0] * 0.3, q1[i, 0] * 0.1)
        kr = (q2[i, 0] * 0.5, q2[i, 0] * 0.2)
        a = ol.chlld("ref", n_state, nrm[i], w[i], q1[i], q2[i], n_disc=n_disc, kl=kl, kr=kr)
        b = ol.chlld("oracle", n_state, nrm[i], w[i], q1[i], q2[i], n_disc=n_disc, kl=kl, kr=kr)
        assert b[3] == 0
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.skipif(not ol.ref_available(), reason="reference solver not built (no reference tree)")
@pytest.mark.parametrize("flags", [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)])
def test_oracle_chlld_flags_vs_reference(oracle_lib, flags):
    nrm, w, q1, q2 = _cases()
    for ns in range(4):
        for i in range(0, 600, 13):
            kw = dict(null_bn=flags[0], left_ydar=flags[1], contact=flags[2], kl=(0.4,), kr=(0.7,))
            a = ol.chlld("ref", ns, nrm[i], w[i], q1[i], q2[i], **kw)
            b = ol.chlld("oracle", ns, nrm[i], w[i], q1[i], q2[i], **kw)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])
            np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.skipif(not ol.ref_available(), reason="reference solver not built (no reference tree)")
def test_reference_raspad_testing_case(oracle_lib):
    """The fixed states of Phys_param::raspad_testing (Phys_param.cpp:1880-1935)."""
    q1 = [1.0, 1.0, 1.0, 1.0, 1.0, 1.1, 1.2, 1.3]
    q2 = [2.0, -1.0, 1.0, 1.0, 6.0, 3.1, 1.2, 1.3]
    for ns in range(4):
        a = ol.chlld("ref", ns, [1.0, 0.0, 0.0], -4.0, q1, q2, kl=(10.0,), kr=(20.0,))
        b = ol.chlld("oracle", ns, [1.0, 0.0, 0.0], -4.0, q1, q2, kl=(10.0,), kr=(20.0,))
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_oracle_chlld_vs_golden(oracle_lib):
    g = np.load(ol.ROOT + "/tests/golden/chlld_golden.npz")
    n = g["q1"].shape[0]
    for i in range(n):
        nk = int(g["nk"][i])
        out, kout, ds, rc = ol.chlld("oracle", int(g["n_state"][i]), g["nrm"][i], g["w"][i], g["q1"][i], g["q2"][i],
                                     n_disc=int(g["n_disc"][i]), null_bn=int(g["null_bn"][i]),
                                     left_ydar=int(g["left_ydar"][i]), contact=int(g["contact"][i]),
                                     kl=tuple(g["kl"][i, :nk]), kr=tuple(g["kr"][i, :nk]))
        assert rc == 0
        np.testing.assert_array_equal(out, g["flux"][i])
        np.testing.assert_array_equal(kout, g["kout"][i, :nk])
        np.testing.assert_array_equal(ds, g["ds"][i])


@pytest.mark.skipif(not ol.ref_available(), reason="reference solver not built (no reference tree)")
@pytest.mark.parametrize("kw", [dict(), dict(zones=True, npassive=2, nh=2)])
def test_oracle_step_with_the_reference_solver_is_identical(titan, oracle_lib, kw):
    """The oracle step with the reference's own compiled chlld on every face
    (the CPU baseline's timed form) against the oracle step with its
    restatement: the same states, dt and time, bit for bit."""
    m, p, st, hf = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=True, **kw)
    out = []
    for use_ref in (False, True):
        run = ol.OracleRun(m, p)
        if hf is not None:
            run.hf = np.ascontiguousarray(hf)
        s = np.ascontiguousarray(st.copy())
        try:
            assert ol.use_reference_riemann(p["gamma"] if use_ref else None) == use_ref
            assert run.go(s, 4).err_code == 0
        finally:
            ol.use_reference_riemann(None)
        out.append((s, run.clock.copy()))
    assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
    assert np.array_equal(out[0][1], out[1][1])
