// Host side of one mesh split across processes: rank r's local mesh (owned elements first, then
// the ghost elements it needs) and its halo-exchange plan. The same rules as
// fve_dg_b200/partition.py (LocalMesh), in native code for drivers that exchange with MPI or NCCL
// from C or C++:
//   - the local faces are the faces that touch an owned element, in the global order and with their
//     orientation, so an owned element sees the faces, normals and face maps it has in the whole mesh;
//   - a ghost is a face neighbour of an owned element owned by another rank, kept with only the
//     faces it shares with owned elements (the mesh's nghost marks them);
//   - rank r sends to rank q the rows of its owned elements that are ghosts of q, in ascending global
//     order, and receives from q its ghosts that q owns, in the same order.
// New: the reference runs one mesh per process.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "dg_gpu.h"

struct dg_partition {
    int rank = 0, nparts = 0;
    int64_t n_owned = 0, n_ghost = 0;
    std::vector<int64_t> l2g, global_face;
    std::vector<int64_t> cell_nodes, face_cells, face_nodes, face_nodes1;
    std::vector<uint8_t> face_bc, face_periodic;
    bool has_nodes1 = false, has_bc = false, has_periodic = false;
    const double* points = nullptr;
    int64_t npts = 0;
    std::vector<int> send_peer, recv_peer;
    std::vector<std::vector<int64_t>> send_rows, recv_rows;
};

namespace {

// Global ids of rank r's ghost elements, ascending.
std::vector<int64_t> ghost_set(const dg_mesh_desc* m, const int32_t* owner, int r) {
    std::vector<int64_t> g;
    for (int64_t f = 0; f < m->nface; ++f) {
        const int64_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
        if (c1 == DG_NO_CELL) continue;
        const bool o0 = owner[c0] == r, o1 = owner[c1] == r;
        if (o0 && !o1) g.push_back(c1);
        if (o1 && !o0) g.push_back(c0);
    }
    std::sort(g.begin(), g.end());
    g.erase(std::unique(g.begin(), g.end()), g.end());
    return g;
}

}  // namespace

extern "C" {

dg_partition* dg_partition_create(const dg_mesh_desc* m, const int32_t* owner, int rank, int* err) {
    auto fail = [&](int rc) -> dg_partition* {
        if (err) *err = rc;
        return nullptr;
    };
    if (!m || !owner || !m->face_cells || !m->cell_nodes || !m->face_nodes || !m->points || m->ncell <= 0 ||
        m->nface <= 0 || m->nghost != 0)
        return fail(DG_E_ARG);
    int nparts = 0;
    for (int64_t e = 0; e < m->ncell; ++e) {
        if (owner[e] < 0) return fail(DG_E_ARG);
        nparts = std::max(nparts, owner[e] + 1);
    }
    if (rank < 0 || rank >= nparts) return fail(DG_E_ARG);
    for (int64_t f = 0; f < m->nface; ++f) {
        const int64_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
        if (c0 < 0 || c0 >= m->ncell || (c1 != DG_NO_CELL && (c1 < 0 || c1 >= m->ncell))) return fail(DG_E_MESH);
    }
    dg_partition* p = new (std::nothrow) dg_partition;
    if (!p) return fail(DG_E_NOMEM);
    p->rank = rank;
    p->nparts = nparts;
    p->points = m->points;
    p->npts = m->npts;
    for (int64_t e = 0; e < m->ncell; ++e)
        if (owner[e] == rank) p->l2g.push_back(e);
    p->n_owned = (int64_t)p->l2g.size();
    const std::vector<int64_t> ghosts = ghost_set(m, owner, rank);
    p->n_ghost = (int64_t)ghosts.size();
    p->l2g.insert(p->l2g.end(), ghosts.begin(), ghosts.end());
    std::vector<int64_t> g2l(m->ncell, -1);
    for (size_t i = 0; i < p->l2g.size(); ++i) g2l[p->l2g[i]] = (int64_t)i;
    for (int64_t e : p->l2g)
        for (int k = 0; k < 4; ++k) p->cell_nodes.push_back(m->cell_nodes[4 * e + k]);
    p->has_nodes1 = m->face_nodes1 != nullptr;
    p->has_bc = m->face_bc != nullptr;
    p->has_periodic = m->face_periodic != nullptr;
    for (int64_t f = 0; f < m->nface; ++f) {
        const int64_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
        const bool touch = owner[c0] == rank || (c1 != DG_NO_CELL && owner[c1] == rank);
        if (!touch) continue;
        p->global_face.push_back(f);
        p->face_cells.push_back(g2l[c0]);
        p->face_cells.push_back(c1 == DG_NO_CELL ? (int64_t)DG_NO_CELL : g2l[c1]);
        for (int k = 0; k < 3; ++k) p->face_nodes.push_back(m->face_nodes[3 * f + k]);
        if (p->has_nodes1)
            for (int k = 0; k < 3; ++k) p->face_nodes1.push_back(m->face_nodes1[3 * f + k]);
        if (p->has_bc) p->face_bc.push_back(m->face_bc[f]);
        if (p->has_periodic) p->face_periodic.push_back(m->face_periodic[f]);
    }
    // receive: my ghosts grouped by owner (ascending global id within a peer)
    for (int q = 0; q < nparts; ++q) {
        if (q == rank) continue;
        std::vector<int64_t> rows;
        for (int64_t g : ghosts)
            if (owner[g] == q) rows.push_back(g2l[g]);
        if (!rows.empty()) {
            p->recv_peer.push_back(q);
            p->recv_rows.push_back(std::move(rows));
        }
        std::vector<int64_t> send;
        for (int64_t g : ghost_set(m, owner, q))
            if (owner[g] == rank) send.push_back(g2l[g]);
        if (!send.empty()) {
            p->send_peer.push_back(q);
            p->send_rows.push_back(std::move(send));
        }
    }
    if (err) *err = DG_OK;
    return p;
}

void dg_partition_destroy(dg_partition* p) { delete p; }

int dg_partition_local_mesh(const dg_partition* p, dg_mesh_desc* out) {
    if (!p || !out) return DG_E_ARG;
    std::memset(out, 0, sizeof(*out));
    out->ncell = (int64_t)p->l2g.size();
    out->nface = (int64_t)p->global_face.size();
    out->face_cells = p->face_cells.data();
    out->face_bc = p->has_bc ? p->face_bc.data() : nullptr;
    out->npts = p->npts;
    out->points = p->points;
    out->cell_nodes = p->cell_nodes.data();
    out->face_nodes = p->face_nodes.data();
    out->face_nodes1 = p->has_nodes1 ? p->face_nodes1.data() : nullptr;
    out->face_periodic = p->has_periodic ? p->face_periodic.data() : nullptr;
    out->nghost = p->n_ghost;
    return DG_OK;
}

int dg_partition_counts(const dg_partition* p, int64_t* n_owned, int64_t* n_ghost, int* n_send, int* n_recv) {
    if (!p) return DG_E_ARG;
    if (n_owned) *n_owned = p->n_owned;
    if (n_ghost) *n_ghost = p->n_ghost;
    if (n_send) *n_send = (int)p->send_peer.size();
    if (n_recv) *n_recv = (int)p->recv_peer.size();
    return DG_OK;
}

const int64_t* dg_partition_l2g(const dg_partition* p) { return p ? p->l2g.data() : nullptr; }
const int64_t* dg_partition_global_faces(const dg_partition* p) { return p ? p->global_face.data() : nullptr; }

int dg_partition_send(const dg_partition* p, int i, int* peer, int64_t* n, const int64_t** rows) {
    if (!p || i < 0 || i >= (int)p->send_peer.size()) return DG_E_ARG;
    if (peer) *peer = p->send_peer[i];
    if (n) *n = (int64_t)p->send_rows[i].size();
    if (rows) *rows = p->send_rows[i].data();
    return DG_OK;
}

int dg_partition_recv(const dg_partition* p, int i, int* peer, int64_t* n, const int64_t** rows) {
    if (!p || i < 0 || i >= (int)p->recv_peer.size()) return DG_E_ARG;
    if (peer) *peer = p->recv_peer[i];
    if (n) *n = (int64_t)p->recv_rows[i].size();
    if (rows) *rows = p->recv_rows[i].data();
    return DG_OK;
}

}  // extern "C"
