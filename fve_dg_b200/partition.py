"""One mesh across several GPUs: element partition, local meshes with ghost cells, and the per-stage
halo exchange of coefficient blocks.

Each rank owns a contiguous range of the mesh's elements (on the box meshes, slabs). Its local mesh
holds the owned elements first, then the ghost elements: the face neighbours of owned elements
that another rank owns. The local faces are the faces that touch an owned element, with their
cells renumbered and their orientation unchanged, so an owned element sees exactly the faces,
normals and face maps it has in the whole mesh. A ghost keeps only the faces it shares with owned
elements (the mesh's `nghost` marks the ghosts: the library computes no residual, limiting or
reduction for them), and its state is overwritten by its owner's before every stage.

Before each RK stage the stage input's ghost entries are refreshed: every rank sends, to each
neighbouring rank, the coefficient blocks of its owned elements that are ghosts there, and
unpacks what it receives into its ghost slots (one send and one receive per neighbour,
`torch.distributed.batch_isend_irecv`, NCCL between GPUs; on CUDA the gathers and scatters are the
library's own kernels, dg_halo_pack and dg_halo_unpack). Owned results then equal the whole-mesh
results: the same faces, in the same order, see the same inputs. The library builds the same plan
natively (dg_partition_create, NativePlan) for drivers in C or C++.
"""
import ctypes

import numpy as np

from . import _lib as L
from .mesh import Mesh


def partition_elements(mesh, nparts):
    """Owner of every element: nparts contiguous, balanced ranges of the element numbering."""
    return (np.arange(mesh.ncell, dtype=np.int64) * nparts) // mesh.ncell


class LocalMesh:
    """Rank `rank`'s part of `mesh` under the ownership `part` (see the module docstring)."""

    def __init__(self, mesh, part, rank):
        part = np.asarray(part, dtype=np.int64)
        nparts = int(part.max()) + 1
        self.rank, self.nparts = rank, nparts
        fc = mesh.face_cells
        c0, c1 = fc[:, 0], fc[:, 1]
        own = part == rank
        c1s = np.where(c1 >= 0, c1, c0)
        touch = own[c0] | ((c1 >= 0) & own[c1s])
        other = np.where(own[c0], c1, c0)[touch]
        owned = np.flatnonzero(own)
        ghosts = np.unique(other[(other >= 0) & ~own[np.maximum(other, 0)]])
        self.owned, self.ghosts = owned, ghosts
        self.n_owned = len(owned)
        self.l2g = np.concatenate([owned, ghosts])
        g2l = np.full(mesh.ncell, -1, dtype=np.int64)
        g2l[self.l2g] = np.arange(len(self.l2g))
        # the faces touching owned elements, with their orientation and order; a ghost keeps only
        # these (the mesh's last nghost cells need not be closed)
        tf = np.flatnonzero(touch)
        fn1 = mesh.face_nodes1[tf] if mesh.face_nodes1 is not None else None
        per = mesh.periodic[tf] if mesh.periodic is not None else None
        bcs = mesh.bc[tf] if mesh.bc is not None else None
        fcs = np.stack([g2l[c0[tf]], np.where(c1[tf] >= 0, g2l[c1s[tf]], -1)], axis=1)
        self.mesh = Mesh(mesh.points, mesh.cells[self.l2g], mesh.faces[tf], fcs, fn1, per, bcs,
                         nghost=len(ghosts))
        self.global_face = tf  # local face i is global face tf[i]
        # exchange plan: what this rank sends to / receives from every other rank, by global id
        ghost_owner = part[ghosts]
        self.recv = {int(q): g2l[ghosts[ghost_owner == q]] for q in np.unique(ghost_owner)}
        self.send = {}
        for q in range(nparts):
            if q == rank:
                continue
            theirs = LocalMesh.ghost_set(mesh, part, q)
            mine = theirs[part[theirs] == rank]
            if len(mine):
                self.send[q] = g2l[mine]

    @staticmethod
    def ghost_set(mesh, part, rank):
        """Global ids of rank `rank`'s ghost elements, sorted."""
        fc = mesh.face_cells
        c0, c1 = fc[:, 0], fc[:, 1]
        own = np.asarray(part) == rank
        c1s = np.where(c1 >= 0, c1, c0)
        touch = own[c0] | ((c1 >= 0) & own[c1s])
        other = np.where(own[c0], c1, c0)[touch]
        return np.unique(other[(other >= 0) & ~own[np.maximum(other, 0)]])

    @property
    def ncell(self):
        return len(self.l2g)


def halo_exchange(state, lm, dist):
    """Fill the ghost rows of `state` (a torch tensor [local cells][...]) from their owners: one
    send and one receive per neighbouring rank. Every rank calls it with the same sequence."""
    import torch
    cache = lm.__dict__.setdefault("_index_cache", {})
    key = str(state.device)
    if key not in cache:
        cache[key] = ({q: torch.as_tensor(i, device=state.device) for q, i in lm.send.items()},
                      {q: torch.as_tensor(i, device=state.device) for q, i in lm.recv.items()})
    send_idx, recv_idx = cache[key]
    ops, bufs = [], []
    for q in sorted(send_idx):
        buf = state.index_select(0, send_idx[q])
        bufs.append(buf)
        ops.append(dist.P2POp(dist.isend, buf, q))
    recvs = []
    for q in sorted(recv_idx):
        buf = torch.empty((len(recv_idx[q]),) + tuple(state.shape[1:]), dtype=state.dtype, device=state.device)
        recvs.append((recv_idx[q], buf))
        ops.append(dist.P2POp(dist.irecv, buf, q))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    for idx, buf in recvs:
        state.index_copy_(0, idx, buf)


class _DeviceArray:
    """A device buffer of the library, viewed by torch through __cuda_array_interface__."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class PartitionedConvection:
    """ExplicitConvection on rank `rank`'s part of one mesh: SSP-RK3 with a halo exchange before
    every stage, all of it ordered on the context's CUDA stream (the exchange's gathers, the NCCL
    sends and receives and the scatters run on that stream; the host never waits between stages).
    `dist` is torch.distributed with a process group over the parts; single-process users pass
    `exchange` instead, a callable (which) that fills the ghost rows of state buffer `which` on
    the context's stream."""

    def __init__(self, mesh, part, rank, dist=None, exchange=None, device=0, **kw):
        from .convection import ExplicitConvection
        if (dist is None) == (exchange is None):
            raise ValueError("give exactly one of dist and exchange")
        self.lm = LocalMesh(mesh, part, rank)
        self.conv = ExplicitConvection(self.lm.mesh, device=device, **kw)
        self.dist, self._exchange, self.device = dist, exchange, device
        self.mixed = self.conv.precision == "mixed"
        self._comm = None  # the exchange's stream when it overlaps the stage's first phase

    def torch_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.conv.stream, device=torch.device("cuda", self.device))

    def state_view(self, which):
        """Torch view of device state buffer `which` (0 = U^n, 1 = U^(1), 2 = U^(2))."""
        import torch
        ptr = L.lib().dg_state_device(self.conv._ctx, int(which))
        if not ptr:
            raise ValueError(f"no state buffer {which}")
        with torch.cuda.device(self.device):
            return torch.as_tensor(_DeviceArray(ptr, self.conv.shape), device=torch.device("cuda", self.device))

    def set_state(self, U_global):
        self.conv.set_state(np.asarray(U_global)[self.lm.l2g])

    def get_owned(self):
        return self.conv.get_state()[: self.lm.n_owned]

    def rows_dev(self, kind, q):
        """Device copy of the local rows this part sends to ("send") or receives from ("recv") q."""
        import torch
        cache = self.__dict__.setdefault("_rows_cache", {})
        if (kind, q) not in cache:
            rows = (self.lm.send if kind == "send" else self.lm.recv)[q]
            cache[kind, q] = torch.as_tensor(np.ascontiguousarray(rows, dtype=np.int64),
                                             device=torch.device("cuda", self.device))
        return cache[kind, q]

    def pack(self, which, q, buf, stream):
        """Rows of state buffer `which` that peer q needs, into buf, by the library's gather kernel
        (dg_halo_pack) on `stream`."""
        idx = self.rows_dev("send", q)
        L.check(L.lib().dg_halo_pack(self.conv._ctx, int(which), ctypes.c_void_p(idx.data_ptr()), int(idx.numel()),
                                     ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(stream)), "dg_halo_pack")

    def unpack(self, which, q, buf, stream):
        """buf (peer q's rows) into this part's ghost rows of state buffer `which` (dg_halo_unpack)."""
        idx = self.rows_dev("recv", q)
        L.check(L.lib().dg_halo_unpack(self.conv._ctx, int(which), ctypes.c_void_p(idx.data_ptr()), int(idx.numel()),
                                       ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(stream)), "dg_halo_unpack")

    def _halo(self, which):
        """The NCCL halo exchange of state buffer `which` on the current torch stream: the library's
        gather kernel per peer, one send and one receive per neighbouring rank, its scatter kernel."""
        import torch
        stream = torch.cuda.current_stream().cuda_stream
        dev = torch.device("cuda", self.device)
        row = 5 * self.conv.num_basis
        ops, recvs = [], []
        for q in sorted(self.lm.send):
            buf = torch.empty((len(self.lm.send[q]), row), dtype=torch.float64, device=dev)
            self.pack(which, q, buf, stream)
            ops.append(self.dist.P2POp(self.dist.isend, buf, q))
        for q in sorted(self.lm.recv):
            buf = torch.empty((len(self.lm.recv[q]), row), dtype=torch.float64, device=dev)
            recvs.append((q, buf))
            ops.append(self.dist.P2POp(self.dist.irecv, buf, q))
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        for q, buf in recvs:
            self.unpack(which, q, buf, stream)

    def exchange(self, which):
        """Fill the ghost rows of state buffer `which` from their owners (stream-ordered)."""
        import torch
        with torch.cuda.stream(self.torch_stream()):
            if self._exchange is not None:
                self._exchange(which)
            else:
                self._halo(which)

    def stage(self, dt, st):
        L.check(L.lib().dg_ssprk3_stage(self.conv._ctx, float(dt), int(st)), "dg_ssprk3_stage")

    def phase(self, dt, st, ph):
        """Phase 0 of stage st reads no ghost row (the faces between owned elements), phase 1 is the
        rest (dg_ssprk3_stage_phase)."""
        L.check(L.lib().dg_ssprk3_stage_phase(self.conv._ctx, float(dt), int(st), int(ph)),
                "dg_ssprk3_stage_phase")

    def overlapped_stage(self, dt, st):
        """Stage st with the halo exchange of its input on a second stream, concurrent with phase 0
        on the context's stream; phase 1 waits for the exchange (CUDA events, no host wait)."""
        import torch
        main = self.torch_stream()
        if self._comm is None:
            self._comm = torch.cuda.Stream(device=torch.device("cuda", self.device))
        ready = torch.cuda.Event()
        ready.record(main)              # the stage input is complete
        self.phase(dt, st, 0)
        self._comm.wait_event(ready)
        with torch.cuda.stream(self._comm):
            if self._exchange is not None:
                self._exchange(st)
            else:
                self._halo(st)
        done = torch.cuda.Event()
        done.record(self._comm)
        main.wait_event(done)
        self.phase(dt, st, 1)

    def wait(self):
        """Wait for the context's stream; reports a watchdog error of the persistent schedule."""
        L.check(L.lib().dg_ssprk3(self.conv._ctx, 0.0, 0), "dg_ssprk3")

    def ssprk3(self, dt, nsteps=1, overlap=True):
        """SSP-RK3 steps; with overlap the exchange of each stage runs beside its first phase."""
        for _ in range(nsteps):
            for st in range(3):
                if overlap:
                    self.overlapped_stage(dt, st)
                else:
                    self.exchange(st)
                    self.stage(dt, st)
        self.wait()


def emulated_ranks(mesh, nparts, **kw):
    """nparts PartitionedConvection objects in one process on one GPU, exchanging ghost rows through
    the library's gather and scatter kernels (the owner's dg_halo_pack, then dg_halo_unpack); step
    them together with `step_emulated` (the decomposition on one GPU)."""
    import torch
    part = partition_elements(mesh, nparts)
    ranks = []

    def make_exchange(r):
        def ex(which):  # the owner's gather kernel into a buffer, then this part's scatter kernel
            dst = ranks[r]
            stream = torch.cuda.current_stream().cuda_stream
            for q in sorted(dst.lm.recv):
                src = ranks[q]
                buf = torch.empty((len(dst.lm.recv[q]), 5 * dst.conv.num_basis), dtype=torch.float64,
                                  device=torch.device("cuda", dst.device))
                src.pack(which, r, buf, stream)
                dst.unpack(which, q, buf, stream)
        return ex

    for r in range(nparts):
        ranks.append(PartitionedConvection(mesh, part, r, exchange=make_exchange(r), **kw))
    return ranks


def step_emulated(ranks, dt, nsteps=1, phased=False):
    """SSP-RK3 on emulated ranks: all parts finish a stage before any exchange reads it. phased
    runs each stage as its two phases with the exchange between them."""
    import torch
    for _ in range(nsteps):
        for st in range(3):
            torch.cuda.synchronize()
            if phased:
                for r in ranks:
                    r.phase(dt, st, 0)
            for r in ranks:
                r.exchange(st)
            torch.cuda.synchronize()
            for r in ranks:
                if phased:
                    r.phase(dt, st, 1)
                else:
                    r.stage(dt, st)
    for r in ranks:
        r.wait()


class NativePlan:
    """The same part and exchange plan built by the library (dg_partition_create), for drivers in
    C or C++; read back into numpy arrays named as in LocalMesh."""

    def __init__(self, mesh, part, rank):
        lib = L.lib()
        owner = np.ascontiguousarray(part, dtype=np.int32)
        d = mesh.desc()
        err = ctypes.c_int(0)
        h = lib.dg_partition_create(ctypes.byref(d), owner.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(rank),
                                    ctypes.byref(err))
        if not h:
            raise L.DGError(err.value, "dg_partition_create")
        try:
            no, ng = ctypes.c_int64(), ctypes.c_int64()
            ns, nr = ctypes.c_int(), ctypes.c_int()
            L.check(lib.dg_partition_counts(h, ctypes.byref(no), ctypes.byref(ng), ctypes.byref(ns), ctypes.byref(nr)),
                    "dg_partition_counts")
            self.n_owned, self.n_ghost = no.value, ng.value
            nloc = no.value + ng.value
            self.l2g = np.ctypeslib.as_array(lib.dg_partition_l2g(h), shape=(nloc,)).copy()
            ld = L.MeshDesc()
            L.check(lib.dg_partition_local_mesh(h, ctypes.byref(ld)), "dg_partition_local_mesh")
            nf = ld.nface

            def arr(p, n_):
                return np.ctypeslib.as_array(p, shape=(n_,)).copy() if p else None

            self.global_face = np.ctypeslib.as_array(lib.dg_partition_global_faces(h), shape=(nf,)).copy()
            self.face_cells = arr(ld.face_cells, 2 * nf).reshape(nf, 2)
            self.cells = arr(ld.cell_nodes, 4 * nloc).reshape(nloc, 4)
            self.faces = arr(ld.face_nodes, 3 * nf).reshape(nf, 3)
            fn1 = arr(ld.face_nodes1, 3 * nf)
            self.face_nodes1 = fn1.reshape(nf, 3) if fn1 is not None else None
            self.periodic = arr(ld.face_periodic, nf)
            self.bc = arr(ld.face_bc, nf)
            self.nghost = ld.nghost
            self.send, self.recv = {}, {}
            for count, fn, out in ((ns.value, lib.dg_partition_send, self.send), (nr.value, lib.dg_partition_recv, self.recv)):
                for i in range(count):
                    peer, n = ctypes.c_int(), ctypes.c_int64()
                    rows = L.c_int64_p()
                    L.check(fn(h, i, ctypes.byref(peer), ctypes.byref(n), ctypes.byref(rows)), "dg_partition_send/recv")
                    out[peer.value] = np.ctypeslib.as_array(rows, shape=(n.value,)).copy()
        finally:
            lib.dg_partition_destroy(h)
