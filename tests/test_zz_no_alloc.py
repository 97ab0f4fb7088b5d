"""titan_step_noalloc: the step for callers that cannot call cudaMalloc.

Some callers step the plasma where they may not allocate device memory — their
own allocator owns the GPU, or allocation is forbidden after start-up. The
no-allocation entry point takes device arrays the caller already owns and keeps
the step's scratch in a fixed array inside the library. These tests call it
through the C ABI on a Brio-Wu cube twice in a row (the second call starts from
the first call's output and dt) and compare each result with titan_step on the
same mesh, within the parity tolerance used by the other GPU tests (1e-12
relative per cell per step): FP64 and FP32 Riemann arithmetic, with and without
the two passive scalars (whose 96-byte flux records fill the scratch's record
slot exactly), and with Bera charge-exchange sources from frozen neutral fluids.
Device arrays for the tests are made with torch; the entry point itself
allocates nothing.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12


def _rel(a, b):
    scale = np.maximum(np.abs(b), 1e-12 * np.max(np.abs(b)))
    return float(np.max(np.abs(a - b) / scale))


def _hfluids(C, nh, seed=5):
    """Frozen neutral fluids [5 nh][C]: density, velocity, pressure (positive)."""
    rng = np.random.default_rng(seed)
    h = np.empty((5 * nh, C))
    for k in range(nh):
        h[5 * k] = 0.1 + 0.2 * rng.random(C)
        h[5 * k + 1:5 * k + 4] = 0.5 * rng.standard_normal((3, C))
        h[5 * k + 4] = 0.05 + 0.1 * rng.random(C)
    return h


CASES = [
    pytest.param(64, 0, 0, id="fp64"),
    pytest.param(32, 0, 0, id="fp32"),
    pytest.param(64, 2, 0, id="fp64-passive"),
    pytest.param(32, 2, 0, id="fp32-passive"),
    pytest.param(64, 0, 2, id="fp64-bera-sources"),
]


@pytest.mark.parametrize("flux,npassive,nh", CASES)
def test_noalloc_step_matches_titan_step_twice(titan, flux, npassive, nh):
    import torch

    N = titan.native
    L = N.lib()
    m, p, st, meth = titan.problems.brio_wu_cube(14)
    p = dict(p, flux_precision=flux, npassive=npassive, nh=nh)
    C, F = m["cell_nodes"].shape[0], m["face_nodes"].shape[0]
    assert F <= 131072
    ns = 8 + npassive
    st = st.copy()
    if npassive:
        st[8] = 0.3 * st[0]           # Q
        st[9] = 0.05 * st[0]          # rho_He
    hfl = _hfluids(C, nh) if nh else None

    # reference: the allocating entry points (titan_create / titan_step)
    ref = titan.PlasmaStep(m, p)
    ref.set_face_method(meth)
    ref.upload_state(st)
    if nh:
        ref.upload_hfluids(hfl)
    g = ref.geometry()
    ref.go(1)
    ref1, dt1 = ref.download_state(), ref.dt
    ref.go(1)
    ref2, dt2 = ref.download_state(), ref.dt
    ref.close()

    # the same mesh as device arrays in the kernels' layout (original numbering)
    dev = torch.device("cuda:0")
    fc = m["face_cells"]
    own = fc[m["cell_faces"]][:, :, 0] == np.arange(C)[:, None]
    cell_faces = (m["cell_faces"].astype(np.int64) | np.where(own, 0, 1 << 31)).astype(np.uint32).view(np.int32)
    cc = g["cell_center"]
    half = np.zeros(F)
    inner = fc[:, 1] >= 0
    d = cc[fc[inner, 0]] - cc[fc[inner, 1]]
    half[inner] = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]) / 2.0
    arrays = dict(
        face_c0=fc[:, 0].copy(), face_c1=fc[:, 1].copy(), face_type=m["face_type"], face_surf=m["face_surf"],
        face_method=meth, face_bc=m["face_bc"], bc_vals=np.zeros((10, 1)), cell_faces=cell_faces.T.copy(),
        cell_type=m["cell_type"], cell_tvd=m["cell_tvd"], cell_center=cc.T.copy(),
        cell_volume=g["cell_volume"], face_center=g["face_center"].T.copy(),
        face_normal=g["face_normal"].T.copy(), face_area=g["face_area"], face_half_dist=half)
    if nh:
        arrays["hfluids"] = hfl
    keep = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in arrays.items()}
    dm = N.TitanDevMesh()
    dm.ncell, dm.nface, dm.nbc = C, F, 0
    for k, t in keep.items():
        setattr(dm, k, t.data_ptr())
    if not nh:
        dm.hfluids = None
    prm = N.TitanParams()
    for k, _ in N.TitanParams._fields_:
        setattr(prm, k, p[k])

    s0 = torch.from_numpy(np.ascontiguousarray(st[:ns])).to(dev)
    s1 = torch.empty_like(s0)
    s2 = torch.empty_like(s0)
    torch.cuda.synchronize()
    dt_next = ctypes.c_double(0.0)
    kind = ctypes.c_int32(-1)
    rc = L.titan_step_noalloc(ctypes.byref(dm), ctypes.byref(prm), 1e-5, s0.data_ptr(), s1.data_ptr(),
                              ctypes.byref(dt_next), ctypes.byref(kind), None)
    N.check(rc)
    assert kind.value == 0
    out1 = s1.cpu().numpy()
    assert _rel(out1, ref1[:ns]) <= REL
    assert abs(dt_next.value - dt1) <= REL * dt1

    rc = L.titan_step_noalloc(ctypes.byref(dm), ctypes.byref(prm), dt_next.value, s1.data_ptr(), s2.data_ptr(),
                              ctypes.byref(dt_next), ctypes.byref(kind), None)
    N.check(rc)
    out2 = s2.cpu().numpy()
    assert _rel(out2, ref2[:ns]) <= REL
    assert abs(dt_next.value - dt2) <= REL * dt2

    # sizes beyond the fixed scratch, and inconsistent cell counts, are refused
    # with a clear error before any launch
    dm.nface = 131073
    rc = L.titan_step_noalloc(ctypes.byref(dm), ctypes.byref(prm), 1e-5, s0.data_ptr(), s1.data_ptr(),
                              ctypes.byref(dt_next), None, None)
    assert rc == -1
    assert b"exceed" in L.titan_last_error()
    dm.nface = F
    dm.ncell = F  # more cells than F / 3 faces can bound
    rc = L.titan_step_noalloc(ctypes.byref(dm), ctypes.byref(prm), 1e-5, s0.data_ptr(), s1.data_ptr(),
                              ctypes.byref(dt_next), None, None)
    assert rc == -1
    assert b"ncell" in L.titan_last_error()
