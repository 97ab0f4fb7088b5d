"""Sharded plasma step: the mesh split over ranks (one GPU each), one halo
exchange per step and a minimum of dt over the ranks.

The reference runs one OpenMP process per mesh (Setka::Go,
TITAN/source/Setka_physics.cpp:1484-2278); this is the multi-GPU layout of the
same step:

* cells go to ranks in contiguous ranges of the Morton order of their centres;
* a rank's sub-mesh holds its own cells, one layer of copies of the cells
  across their faces (the halo), every face of those cells and their nodes.
  A face of a halo cell whose other cell is not on the rank becomes an
  Outer_Soft boundary face there: the halo cells' own update is thrown away,
  since the next exchange overwrites them; only faces with an owned cell
  enter the rank's CFL minimum (titan_set_cfl_faces), and every face of the
  mesh has an owned cell on some rank;
* each step: the owners send their halo cells' states, every rank steps its
  sub-mesh with the dt of the previous step's global minimum, then the ranks
  take the minimum of their CFL candidates.

Every face of an owned cell is on the rank with both its cells' true states,
and the cell update gathers the faces in the cell's own order, so the owned
cells come out bit for bit as in a single-domain step, whatever the split.
Second-order faces take two halo layers: the cells beyond both sides of every
face of an owned cell, and all their faces, are then on the rank, so the
second-order neighbours (chosen on the rank's sub-mesh) are the global ones.
Surface tracking (rays that cross ranks) and Monte-Carlo passes are not
sharded.
"""
from __future__ import annotations

import numpy as np

NV = 10


def _morton3(p: np.ndarray) -> np.ndarray:
    """63-bit Morton keys of points, 21 bits per axis over their bounding box."""
    lo, hi = p.min(axis=0), p.max(axis=0)
    q = np.floor((p - lo) / np.maximum(hi - lo, 1e-300) * ((1 << 21) - 1)).astype(np.uint64)
    key = np.zeros(len(p), dtype=np.uint64)
    for b in range(21):
        for a in range(3):
            key |= ((q[:, a] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + a)
    return key


def partition(mesh: dict, nranks: int) -> np.ndarray:
    """Owner rank of every cell: equal contiguous ranges of the Morton order of the centres."""
    cc = mesh["node_xyz"][mesh["cell_nodes"]].mean(axis=1)
    if not 1 <= nranks <= len(cc):
        raise ValueError(f"cannot split {len(cc)} cells over {nranks} ranks")
    order = np.argsort(_morton3(cc), kind="stable")
    owner = np.empty(len(cc), dtype=np.int32)
    for r, idx in enumerate(np.array_split(order, nranks)):
        owner[idx] = r
    return owner


def build_shard(mesh: dict, owner: np.ndarray, rank: int, layers: int = 1) -> dict:
    """Rank `rank`'s sub-mesh and halo plan, with `layers` layers of halo cells
    (2 for second-order faces, whose reconstruction reaches the cells beyond
    both sides of a face).

    Returns dict(mesh=local mesh dict, cells=global ids of the local cells
    (owned first, ascending, then the halo, ascending), n_owned, faces, nodes
    (global ids), recv={peer: local ids of the halo cells peer owns},
    send={peer: local ids of owned cells peer keeps copies of}); in both plans
    the cells run in ascending global id, the order both sides use."""
    fc = mesh["face_cells"]
    cf = mesh["cell_faces"]
    owned = np.nonzero(owner == rank)[0]
    inner = owned
    for _ in range(layers):
        nb = fc[np.unique(cf[inner].ravel())].ravel()
        inner = np.union1d(inner, nb[nb >= 0])
    halo = np.setdiff1d(inner, owned)
    cells = np.concatenate([owned, halo]).astype(np.int64)
    lc = -np.ones(len(owner), dtype=np.int64)
    lc[cells] = np.arange(len(cells))
    faces = np.unique(cf[cells].ravel())
    lf = -np.ones(len(fc), dtype=np.int64)
    lf[faces] = np.arange(len(faces))
    nodes = np.unique(mesh["cell_nodes"][cells].ravel())
    ln = -np.ones(len(mesh["node_xyz"]), dtype=np.int64)
    ln[nodes] = np.arange(len(nodes))

    c0 = lc[np.maximum(fc[faces, 0], 0)]
    c0[fc[faces, 0] < 0] = -1
    c1 = lc[np.maximum(fc[faces, 1], 0)]
    c1[fc[faces, 1] < 0] = -1
    ftype = mesh["face_type"][faces].copy()
    fsurf = mesh["face_surf"][faces].copy()
    fbc = mesh["face_bc"][faces].copy()
    # a halo cell's face whose other cell is off this rank: Outer_Soft with the halo cell as cells[0]
    cut = (c0 < 0) != (c1 < 0)
    cut &= ftype == 0
    only = np.where(c0 >= 0, c0, c1)
    c0 = np.where(cut, only, c0)
    c1 = np.where(cut, -1, c1)
    ftype[cut] = 3
    fsurf[cut] = 0
    fbc[cut] = -1
    # boundary values of the hard faces kept
    rows = np.unique(fbc[fbc >= 0])
    lrow = -np.ones(max(len(mesh["bc_vals"]), 1), dtype=np.int64)
    lrow[rows] = np.arange(len(rows))
    fbc = np.where(fbc >= 0, lrow[np.maximum(fbc, 0)], -1)

    def sub(key, idx):
        a = mesh.get(key)
        return None if a is None else np.ascontiguousarray(a[idx])

    local = dict(
        node_xyz=np.ascontiguousarray(mesh["node_xyz"][nodes]),
        cell_nodes=np.ascontiguousarray(ln[mesh["cell_nodes"][cells]].astype(np.int32)),
        cell_faces=np.ascontiguousarray(lf[cf[cells]].astype(np.int32)),
        cell_type=sub("cell_type", cells),
        cell_tvd=sub("cell_tvd", cells),
        face_nodes=np.ascontiguousarray(ln[mesh["face_nodes"][faces]].astype(np.int32)),
        face_cells=np.ascontiguousarray(np.stack([c0, c1], axis=1).astype(np.int32)),
        face_type=np.ascontiguousarray(ftype.astype(np.int8)),
        face_surf=np.ascontiguousarray(fsurf.astype(np.int8)),
        face_bc=np.ascontiguousarray(fbc.astype(np.int32)),
        bc_vals=np.ascontiguousarray(mesh["bc_vals"][rows]) if len(rows) else np.zeros((0, NV)),
        node_amp=sub("node_amp", nodes),
        node_phase=sub("node_phase", nodes),
    )
    recv, send = {}, {}
    n_owned = len(owned)
    for peer in np.unique(owner[halo]):
        recv[int(peer)] = lc[halo[owner[halo] == peer]]
    # cells of mine in another rank's halo: within `layers` faces of that rank's cells
    for peer in range(int(owner.max()) + 1):
        if peer == rank:
            continue
        reach = np.nonzero(owner == peer)[0]
        for _ in range(layers):
            nbp = fc[np.unique(cf[reach].ravel())].ravel()
            reach = np.union1d(reach, nbp[nbp >= 0])
        mine = reach[owner[reach] == rank]
        if len(mine):
            send[peer] = lc[mine]
    # faces with no owned cell: their stencils can reach past the halo, and the
    # rank owning a side supplies their CFL candidate
    nodt = ((c0 < 0) | (c0 >= n_owned)) & ((c1 < 0) | (c1 >= n_owned))
    return dict(mesh=local, cells=cells, n_owned=n_owned, faces=faces, nodes=nodes, recv=recv, send=send,
                nodt=np.ascontiguousarray(nodt.astype(np.int8)))


def local_face_method(shard: dict, method: np.ndarray) -> np.ndarray:
    """Per-face n_state of the sub-mesh from the global array."""
    return np.ascontiguousarray(np.asarray(method, dtype=np.int8)[shard["faces"]])


class DeviceStepper:
    """A PlasmaStep on a sub-mesh, with the halo copies through device tensors.
    Its halo copies, steps and clock are ordered on the context's stream, so
    ShardedStep drives it without host waits (device_paced)."""

    device_paced = True

    def __init__(self, pkg, mesh: dict, params: dict):
        self.step = pkg.PlasmaStep(mesh, params)

    @property
    def dt(self) -> float:
        return self.step.dt

    @dt.setter
    def dt(self, v: float):
        self.step.dt = v

    def set_halo(self, send, recv):
        self.step.set_halo(send, recv)

    def set_face_method(self, m):
        self.step.set_face_method(m)

    def set_cfl_faces(self, exclude):
        self.step.set_cfl_faces(exclude)

    def pack(self, buf):
        self.step.pack_halo(buf.data_ptr())

    def unpack(self, buf):
        self.step.unpack_halo(buf.data_ptr())

    def upload_state(self, st):
        self.step.upload_state(st)

    def download_state(self):
        return self.step.download_state()

    def go(self, n: int):
        return self.step.go(n)

    def close(self):
        self.step.close()


class ShardedStep:
    """The plasma step of one rank over torch.distributed: a stepper on the
    rank's sub-mesh (DeviceStepper: a PlasmaStep on this rank's GPU), the halo
    exchange through buffers of whole cells (NCCL on GPUs, point to point with
    each neighbour rank), dt as the minimum over the ranks. All ranks call
    every method together."""

    def __init__(self, pkg, mesh: dict, params: dict, rank: int, world: int, device, stepper=None,
                 method: np.ndarray | None = None):
        import torch

        self.torch = torch
        self.rank, self.world, self.device = rank, world, device
        owner = partition(mesh, world)
        # second-order faces reconstruct from the cells beyond both sides: two halo layers
        self.shard = build_shard(mesh, owner, rank, layers=2 if params.get("tvd") else 1)
        self.step = (stepper or DeviceStepper)(pkg, self.shard["mesh"], params)
        self.step.set_cfl_faces(self.shard["nodt"])
        if method is not None:
            self.step.set_face_method(local_face_method(self.shard, method))
        self.ns = 8 + params["npassive"]
        self.peers_send = sorted(self.shard["send"])
        self.peers_recv = sorted(self.shard["recv"])
        send = np.concatenate([self.shard["send"][p] for p in self.peers_send]) if self.peers_send else \
            np.zeros(0, np.int64)
        recv = np.concatenate([self.shard["recv"][p] for p in self.peers_recv]) if self.peers_recv else \
            np.zeros(0, np.int64)
        self.step.set_halo(send, recv)
        self.sbuf = torch.empty((max(len(send), 1), self.ns), dtype=torch.float64, device=device)
        self.rbuf = torch.empty((max(len(recv), 1), self.ns), dtype=torch.float64, device=device)
        self.n_send, self.n_recv = len(send), len(recv)
        if torch.distributed.is_initialized():
            # every rank meets here before the first point-to-point exchange
            torch.distributed.barrier()

    def upload_state(self, state: np.ndarray):
        """The global state [10, C]; each rank takes its local cells."""
        self.step.upload_state(np.ascontiguousarray(state[:, self.shard["cells"]]))

    def owned_state(self) -> np.ndarray:
        return self.step.download_state()[:, : self.shard["n_owned"]]

    def exchange(self):
        """The halo exchange of the host-paced loop (steppers without a device
        stream, e.g. the oracle on CPU ranks)."""
        if self.n_send:
            self.step.pack(self.sbuf)
        self._p2p()
        if self.device.type == "cuda":
            self.torch.cuda.current_stream(self.device).synchronize()
        if self.n_recv:
            self.step.unpack(self.rbuf)

    def _p2p(self):
        """The point-to-point halo messages on the current stream."""
        dist = self.torch.distributed
        ops, off = [], 0
        for p in self.peers_send:
            n = len(self.shard["send"][p])
            ops.append(dist.P2POp(dist.isend, self.sbuf[off:off + n], p))
            off += n
        off = 0
        for p in self.peers_recv:
            n = len(self.shard["recv"][p])
            ops.append(dist.P2POp(dist.irecv, self.rbuf[off:off + n], p))
            off += n
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()  # NCCL: the current stream waits; the host does not

    def go(self, steps: int):
        """`steps` steps; dt after each is the minimum over the ranks."""
        if getattr(self.step, "device_paced", False) and self.device.type == "cuda":
            return self._go_device(steps)
        dist = self.torch.distributed
        for _ in range(steps):
            self.exchange()
            self.step.go(1)
            if self.world > 1:
                t = self.torch.tensor([self.step.dt], dtype=self.torch.float64, device=self.device)
                dist.all_reduce(t, op=dist.ReduceOp.MIN)
                self.step.dt = float(t.item())

    def _go_device(self, steps: int):
        """The loop paced by the device: every step's pack, NCCL exchange,
        unpack, step and all-reduce(min) of dt run on the context's stream in
        order, and the host waits once, at the end (titan_get_clock)."""
        torch = self.torch
        dist = torch.distributed
        ps = self.step.step
        stream = torch.cuda.ExternalStream(ps.stream(), device=self.device)
        reduce_dt = dist.is_initialized()
        if reduce_dt and not hasattr(self, "dt_buf"):
            self.dt_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
        with torch.cuda.stream(stream):
            ps.set_clock()
            for _ in range(steps):
                if self.n_send:
                    ps.pack_halo(self.sbuf.data_ptr())
                self._p2p()
                if self.n_recv:
                    ps.unpack_halo(self.rbuf.data_ptr())
                ps.step_async(1)
                if reduce_dt:
                    ps.dt_copy(self.dt_buf.data_ptr(), into_clock=False)
                    dist.all_reduce(self.dt_buf, op=dist.ReduceOp.MIN)
                    ps.dt_copy(self.dt_buf.data_ptr(), into_clock=True)
        return ps.get_clock()

    def close(self):
        self.step.close()
