"""CPU: one mesh split across ranks (fve_dg_b200/partition.py): the element partition, the local meshes
with ghost elements, the exchange plan, and SSP-RK3 on 2 gloo ranks with a halo exchange before
every stage, checked bit for bit against the whole mesh with the oracle's residual."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fve_dg_b200 import box_mesh, problems
from fve_dg_b200.partition import LocalMesh, halo_exchange, partition_elements
from oracle.pyoracle import Oracle

P, QV, QF = 2, 1, 2


def meshes():
    return [box_mesh(4, jitter=0.1, seed=3),
            box_mesh(4, jitter=0.1, seed=4, periodic=(1, 1, 0), bc="Pseudo3DZ")]


def initial(m):
    return problems.project(m, P, problems.density_wave(A=0.3, vel=(1.0, 0.5, 0.25)))


@pytest.mark.parametrize("mi", [0, 1])
@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_local_meshes_cover_and_agree(mi, nparts):
    m = meshes()[mi]
    g = m.compute_geometry()
    part = partition_elements(m, nparts)
    assert np.bincount(part).min() >= m.ncell // nparts
    lms = [LocalMesh(m, part, r) for r in range(nparts)]
    owned = np.concatenate([lm.owned for lm in lms])
    assert np.array_equal(np.sort(owned), np.arange(m.ncell))
    nbr = m.face_cells
    for lm in lms:
        assert np.all(part[lm.owned] == lm.rank) and np.all(part[lm.ghosts] != lm.rank)
        # every ghost is a face neighbour of an owned element, and every neighbour is present
        c0, c1 = nbr[:, 0], nbr[:, 1]
        mine = (part[c0] == lm.rank) | ((c1 >= 0) & (part[np.maximum(c1, 0)] == lm.rank))
        need = np.unique(np.concatenate([c0[mine], c1[mine][c1[mine] >= 0]]))
        assert np.array_equal(np.sort(lm.l2g), need)
        # owned elements see the whole mesh's faces and geometry (the local mesh's geometry is
        # recomputed from its topology, so it is built the same way for the faces kept)
        lg = lm.mesh.compute_geometry()
        tf = lm.global_face
        for k in ("normal", "area", "natural"):
            assert np.array_equal(lg[k][: len(tf)], g[k][tf]), k
        for k in ("invjac", "detj"):
            assert np.array_equal(lg[k], g[k][lm.l2g]), k
        # the plan: what p sends to q is exactly what q receives from p, in the same order
        for q, idx in lm.send.items():
            assert np.array_equal(lm.l2g[idx], lms[q].l2g[lms[q].recv[lm.rank]])
            assert np.all(idx < lm.n_owned)
        assert sum(len(v) for v in lm.recv.values()) == len(lm.ghosts)


def test_ghost_count_is_validated():
    m = meshes()[0]
    lm = LocalMesh(m, partition_elements(m, 2), 0)
    lm.mesh.compute_geometry()  # ghosts with fewer than four faces are accepted
    assert lm.mesh.nghost == len(lm.ghosts) and np.bincount(lm.mesh.face_cells[lm.mesh.face_cells >= 0],
                                                            minlength=lm.ncell)[lm.n_owned:].min() < 4
    for bad, code in ((len(lm.ghosts) - 1, "DG_E_MESH"), (-1, "DG_E_ARG"), (lm.ncell, "DG_E_ARG")):
        lm.mesh.nghost = bad  # an owned cell without four faces, or a count out of range
        with pytest.raises(Exception, match=code):
            lm.mesh.compute_geometry()
    lm.mesh.nghost = len(lm.ghosts)


@pytest.mark.parametrize("mi", [0, 1])
def test_owned_residual_equals_whole_mesh(mi):
    m = meshes()[mi]
    U = initial(m)
    R = Oracle.from_mesh(m).residual(U, P, QV, QF)
    part = partition_elements(m, 3)
    for r in range(3):
        lm = LocalMesh(m, part, r)
        Rl = Oracle.from_mesh(lm.mesh).residual(U[lm.l2g], P, QV, QF)
        assert np.array_equal(Rl[: lm.n_owned], R[lm.owned])


def ssprk3(o, U, b, dt, nsteps, exchange=lambda U: None):
    """Shu-Osher SSP-RK3 with L(U) = -R(U) / mass; `exchange` fills ghost rows of each stage input."""
    def L(V):
        return -o.residual(V, P, QV, QF) / b
    for _ in range(nsteps):
        exchange(U)
        U1 = U + dt * L(U)
        exchange(U1)
        U2 = 0.75 * U + 0.25 * (U1 + dt * L(U1))
        exchange(U2)
        U = U / 3.0 + 2.0 / 3.0 * (U2 + dt * L(U2))
    return U


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, mi, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = meshes()[mi]
        part = partition_elements(m, world)
        lm = LocalMesh(m, part, rank)
        o = Oracle.from_mesh(lm.mesh)
        b = o.mass(P, QV)
        U0 = initial(m)
        U = U0[lm.l2g].copy()
        U[lm.n_owned:] = np.nan  # ghosts hold nothing until the first exchange

        def exchange(V):
            halo_exchange(torch.from_numpy(V), lm, dist)

        U = ssprk3(o, U, b, 2e-3, 2, exchange)
        q.put((rank, lm.owned, U[: lm.n_owned]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("mi", [0, 1])
def test_two_rank_ssprk3_over_gloo_equals_whole_mesh(mi):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mi, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=150) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    m = meshes()[mi]
    o = Oracle.from_mesh(m)
    want = ssprk3(o, initial(m), o.mass(P, QV), 2e-3, 2)
    got = np.empty_like(want)
    for _, owned, Uo in res:
        got[owned] = Uo
    assert np.array_equal(got, want)


@pytest.mark.parametrize("nparts,kw", [(2, dict(n=3)), (3, dict(n=4, jitter=0.1, seed=3)),
                                       (4, dict(n=3, periodic=(1, 1, 0), bc="Pseudo3DZ"))])
def test_native_plan_is_the_python_plan(nparts, kw):
    """dg_partition_create (native, for C/C++ drivers) builds exactly LocalMesh's part: the same
    local elements, faces (nodes, cells, orientation data) and exchange lists, for every rank."""
    from fve_dg_b200.partition import LocalMesh, NativePlan, partition_elements
    m = box_mesh(**kw)
    part = partition_elements(m, nparts)
    for r in range(nparts):
        lm, nat = LocalMesh(m, part, r), NativePlan(m, part, r)
        assert nat.n_owned == lm.n_owned and nat.n_ghost == len(lm.ghosts) == nat.nghost
        assert np.array_equal(nat.l2g, lm.l2g)
        assert np.array_equal(nat.global_face, lm.global_face)
        lmm = lm.mesh
        assert np.array_equal(nat.face_cells, lmm.face_cells.reshape(-1, 2))
        assert np.array_equal(nat.cells, lmm.cells.reshape(-1, 4))
        assert np.array_equal(nat.faces, lmm.faces.reshape(-1, 3))
        assert np.array_equal(nat.face_nodes1, lmm.face_nodes1.reshape(-1, 3))
        assert np.array_equal(nat.periodic, lmm.periodic.reshape(-1))
        assert np.array_equal(nat.bc, lmm.bc.reshape(-1))
        assert sorted(nat.send) == sorted(lm.send) and sorted(nat.recv) == sorted(lm.recv)
        for q in lm.send:
            assert np.array_equal(nat.send[q], lm.send[q])
        for q in lm.recv:
            assert np.array_equal(nat.recv[q], lm.recv[q])


def test_native_plan_rejects_bad_input():
    import ctypes
    from fve_dg_b200 import _lib as L
    m = box_mesh(2)
    lib = L.lib()
    d = m.desc()
    err = ctypes.c_int(0)
    owner = np.zeros(m.ncell, dtype=np.int32)
    op = owner.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    assert not lib.dg_partition_create(ctypes.byref(d), op, 1, ctypes.byref(err))  # rank beyond the parts
    assert err.value == -1
    owner[3] = -2
    assert not lib.dg_partition_create(ctypes.byref(d), op, 0, ctypes.byref(err))  # negative owner
    assert err.value == -1
    assert not lib.dg_partition_create(None, op, 0, ctypes.byref(err))
    owner[:] = 0
    h = lib.dg_partition_create(ctypes.byref(d), op, 0, ctypes.byref(err))  # one part: no ghosts, no peers
    assert h and err.value == 0
    no, ng = ctypes.c_int64(), ctypes.c_int64()
    ns, nr = ctypes.c_int(), ctypes.c_int()
    assert lib.dg_partition_counts(h, ctypes.byref(no), ctypes.byref(ng), ctypes.byref(ns), ctypes.byref(nr)) == 0
    assert (no.value, ng.value, ns.value, nr.value) == (m.ncell, 0, 0, 0)
    assert lib.dg_partition_send(h, 0, None, None, None) == -1
    lib.dg_partition_destroy(h)
