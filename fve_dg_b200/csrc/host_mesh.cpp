// Host side: periodic box mesh generator, mesh validation, geometry with the reference's formulas
// and operation order, and face maps. Connectivity, orientation and face maps come out bit for bit;
// normals, areas, det J and J^-T agree with the reference to a few ulp, because GCC decides per
// expression where to contract a*b+c into an FMA (both builds use -mfma) and those choices differ
// between the two code bases. Given the reference's own geometry (dg_mesh_desc form (a)) the device
// numbers are the reference's exactly.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <unordered_map>

#include "dg_internal.h"

namespace fvedg {

const int kPermSlots[kNumPerms][3] = {
    {0, 1, 2}, {0, 1, 3}, {0, 2, 1}, {0, 2, 3}, {0, 3, 1}, {0, 3, 2},
    {1, 0, 2}, {1, 0, 3}, {1, 2, 0}, {1, 2, 3}, {1, 3, 0}, {1, 3, 2},
    {2, 0, 1}, {2, 0, 3}, {2, 1, 0}, {2, 1, 3}, {2, 3, 0}, {2, 3, 1},
    {3, 0, 1}, {3, 0, 2}, {3, 1, 0}, {3, 1, 2}, {3, 2, 0}, {3, 2, 1}};

int perm_code(int s0, int s1, int s2) {
    for (int p = 0; p < kNumPerms; ++p)
        if (kPermSlots[p][0] == s0 && kPermSlots[p][1] == s1 && kPermSlots[p][2] == s2) return p;
    return -1;
}

namespace {

// vec_dot for N = 3 (include/base/vector_op.h:121-141 takes the scalar branch): left to right from 0.
inline double dot3(const double* a, const double* b) {
    double s = 0.0;
    s += a[0] * b[0];
    s += a[1] * b[1];
    s += a[2] * b[2];
    return s;
}
inline void cross3(const double* a, const double* b, double* c) {  // vector_op.h:155-161
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
inline void sub3(const double* a, const double* b, double* c) {
    c[0] = a[0] - b[0];
    c[1] = a[1] - b[1];
    c[2] = a[2] - b[2];
}

// CompTetrahedron::compute_geometry, ComputingMesh.cpp:113-125, and the 3x3 inverse of
// DenseMatrix.h:519-538 applied to the row-stacked edges (compute_jacobian_mat, :149-164).
void tet_geometry(const double* p0, const double* p1, const double* p2, const double* p3,
                  double* invj, double* detj, double* cen) {
    for (int i = 0; i < 3; ++i) cen[i] = (((p0[i] + p1[i]) + p2[i]) + p3[i]) / 4.0;
    double v1[3], v2[3], v3[3], cr[3];
    sub3(p1, p0, v1);
    sub3(p2, p0, v2);
    sub3(p3, p0, v3);
    cross3(v2, v3, cr);
    const double vol = std::fabs(dot3(v1, cr)) / 6.0;
    *detj = vol * 6.0;
    const double A[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
    double r[3][3];
    r[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    r[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    r[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    r[0][1] = A[2][1] * A[0][2] - A[2][2] * A[0][1];
    r[1][1] = A[2][2] * A[0][0] - A[2][0] * A[0][2];
    r[2][1] = A[2][0] * A[0][1] - A[2][1] * A[0][0];
    r[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    r[1][2] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
    r[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    double det = 0.0;
    det += A[0][0] * r[0][0];
    det += A[1][0] * r[0][1];
    det += A[2][0] * r[0][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) invj[3 * i + j] = r[i][j] / det;
}

bool in_range(int64_t v, int64_t n) { return v >= 0 && v < n; }

// Slot (0..3) of each face node in a cell, or -1 when a node is not a vertex of the cell.
bool face_slots(const int64_t* cell_nodes4, const int64_t* fn, int slots[3]) {
    for (int k = 0; k < 3; ++k) {
        slots[k] = -1;
        for (int s = 0; s < 4; ++s)
            if (cell_nodes4[s] == fn[k]) slots[k] = s;
        if (slots[k] < 0) return false;
    }
    return slots[0] != slots[1] && slots[0] != slots[2] && slots[1] != slots[2];
}

// Face map code from the reference's natural coordinates m_natural_coords[side]
// (entries e_{slot-1} or the zero vector for slot 0, ComputingMesh.cpp:67-75).
int perm_from_natural(const double* nc9) {
    int slots[3];
    for (int k = 0; k < 3; ++k) {
        int s = 0, ones = 0;
        for (int c = 0; c < 3; ++c) {
            const double v = nc9[3 * k + c];
            if (v == 1.0) { s = c + 1; ++ones; }
            else if (v != 0.0) return -1;
        }
        if (ones > 1) return -1;
        slots[k] = s;
    }
    if (slots[0] == slots[1] || slots[0] == slots[2] || slots[1] == slots[2]) return -1;
    return perm_code(slots[0], slots[1], slots[2]);
}

}  // namespace

int build_geometry(const dg_mesh_desc* d, Geometry* g) {
    if (!d || !g || d->ncell <= 0 || d->nface <= 0 || !d->face_cells) return DG_E_ARG;
    const int64_t nc = d->ncell, nf = d->nface;
    const bool given = d->face_natural && d->face_normal && d->face_area && d->cell_invjac && d->cell_detj;
    const bool raw = d->points && d->cell_nodes && d->face_nodes && d->npts > 0;
    if (!given && !raw) return DG_E_ARG;
    g->normal.assign(3 * nf, 0.0);
    g->area.assign(nf, 0.0);
    g->perm.assign(2 * nf, -1);
    g->invjac.assign(9 * nc, 0.0);
    g->detj.assign(nc, 0.0);
    // face -> cell incidence must be consistent: every cell has exactly four face slots (a ghost
    // cell, one of the last nghost, only those it shares with owned cells: one to four)
    if (d->nghost < 0 || d->nghost >= nc) return DG_E_ARG;
    const int64_t nowned = nc - d->nghost;
    std::vector<int> deg(nc, 0);
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t c0 = d->face_cells[2 * f], c1 = d->face_cells[2 * f + 1];
        if (!in_range(c0, nc)) return DG_E_MESH;
        if (c1 != DG_NO_CELL && !in_range(c1, nc)) return DG_E_MESH;
        ++deg[c0];
        if (c1 != DG_NO_CELL) ++deg[c1];
    }
    for (int64_t c = 0; c < nc; ++c)
        if (c < nowned ? deg[c] != 4 : (deg[c] < 1 || deg[c] > 4)) return DG_E_MESH;

    if (given) {
        std::memcpy(g->normal.data(), d->face_normal, sizeof(double) * 3 * nf);
        std::memcpy(g->area.data(), d->face_area, sizeof(double) * nf);
        std::memcpy(g->invjac.data(), d->cell_invjac, sizeof(double) * 9 * nc);
        std::memcpy(g->detj.data(), d->cell_detj, sizeof(double) * nc);
        for (int64_t f = 0; f < nf; ++f) {
            const int64_t c1 = d->face_cells[2 * f + 1];
            const int p0 = perm_from_natural(d->face_natural + 18 * f);
            if (p0 < 0) return DG_E_MESH;
            g->perm[2 * f] = (int8_t)p0;
            if (c1 != DG_NO_CELL) {
                const int p1 = perm_from_natural(d->face_natural + 18 * f + 9);
                if (p1 < 0) return DG_E_MESH;
                g->perm[2 * f + 1] = (int8_t)p1;
            }
        }
        return DG_OK;
    }

    const int64_t np = d->npts;
    for (int64_t i = 0; i < 4 * nc; ++i)
        if (!in_range(d->cell_nodes[i], np)) return DG_E_MESH;
    for (int64_t i = 0; i < 3 * nf; ++i)
        if (!in_range(d->face_nodes[i], np)) return DG_E_MESH;
    std::vector<double> cen(3 * nc);
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t* cn = d->cell_nodes + 4 * c;
        tet_geometry(d->points + 3 * cn[0], d->points + 3 * cn[1], d->points + 3 * cn[2],
                     d->points + 3 * cn[3], &g->invjac[9 * c], &g->detj[c], &cen[3 * c]);
    }
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t* fn = d->face_nodes + 3 * f;
        const int64_t c0 = d->face_cells[2 * f], c1 = d->face_cells[2 * f + 1];
        const double* p0 = d->points + 3 * fn[0];
        const double* p1 = d->points + 3 * fn[1];
        const double* p2 = d->points + 3 * fn[2];
        double e1[3], e2[3], n[3];
        sub3(p1, p0, e1);
        sub3(p2, p0, e2);
        cross3(e1, e2, n);  // CompTriangleFace::compute_geometry, ComputingMesh.cpp:46
        const bool periodic = d->face_periodic && d->face_periodic[f];
        if (c1 == DG_NO_CELL || periodic) {
            // boundary rule (:47-60): orient away from the cell's fourth vertex
            const double* p3 = nullptr;
            for (int k = 0; k < 4; ++k) {
                const int64_t v = d->cell_nodes[4 * c0 + k];
                if (v == fn[0] || v == fn[1] || v == fn[2]) continue;
                p3 = d->points + 3 * v;
            }
            if (!p3) return DG_E_MESH;
            double v3[3], cr[3];
            sub3(p3, p0, v3);
            cross3(e1, e2, cr);
            if (dot3(cr, v3) * dot3(cr, n) > 0) { n[0] *= -1; n[1] *= -1; n[2] *= -1; }
        } else {
            // interior rule (:61-64): orient from cells[0]'s centroid to cells[1]'s
            double dc[3];
            sub3(&cen[3 * c1], &cen[3 * c0], dc);
            if (dot3(n, dc) < 0) { n[0] *= -1; n[1] *= -1; n[2] *= -1; }
        }
        g->area[f] = std::sqrt(dot3(n, n)) * 0.5;            // :65
        const double len = std::sqrt(dot3(n, n));            // :66 vec_unit
        for (int i = 0; i < 3; ++i) g->normal[3 * f + i] = n[i] / len;
        int s[3];
        if (!face_slots(d->cell_nodes + 4 * c0, fn, s)) return DG_E_MESH;
        g->perm[2 * f] = (int8_t)perm_code(s[0], s[1], s[2]);
        if (c1 != DG_NO_CELL) {
            const int64_t* fn1 = d->face_nodes1 ? d->face_nodes1 + 3 * f : fn;
            if (!face_slots(d->cell_nodes + 4 * c1, fn1, s)) return DG_E_MESH;
            g->perm[2 * f + 1] = (int8_t)perm_code(s[0], s[1], s[2]);
        }
    }
    return DG_OK;
}

}  // namespace fvedg

using namespace fvedg;

// ------------------------------------------------------------------------------------------------
// Periodic box mesh
// ------------------------------------------------------------------------------------------------
struct dg_box_mesh {
    int n = 0;
    std::vector<double> points;
    std::vector<int64_t> cells, faces, face_cells, face_nodes1, cell_faces, cell_cells;
    std::vector<uint8_t> periodic, bc;
};

namespace {
struct KeyHash {
    size_t operator()(const std::array<int64_t, 3>& k) const {
        uint64_t h = 1469598103934665603ull;
        for (int64_t v : k) { h ^= (uint64_t)v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); }
        return (size_t)h;
    }
};
std::array<int64_t, 3> sorted_key(const int64_t* a) {
    std::array<int64_t, 3> k = {a[0], a[1], a[2]};
    std::sort(k.begin(), k.end());
    return k;
}
}  // namespace

extern "C" dg_box_mesh* dg_box_mesh_create(int n, const double lo[3], const double hi[3], double jitter,
                                           uint64_t seed, const int periodic[3], int bc, int* err) {
    auto fail = [&](int e) -> dg_box_mesh* { if (err) *err = e; return nullptr; };
    if (n < 1 || n > 2048 || !lo || !hi || jitter < 0 || jitter >= 0.25) return fail(DG_E_ARG);
    dg_box_mesh* m = new (std::nothrow) dg_box_mesh;
    if (!m) return fail(DG_E_NOMEM);
    m->n = n;
    const int64_t nv = n + 1;
    auto pid = [&](int64_t i, int64_t j, int64_t k) { return i + nv * (j + nv * k); };
    auto ijk = [&](int64_t p, int64_t* c) { c[0] = p % nv; c[1] = (p / nv) % nv; c[2] = p / (nv * nv); };
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = (hi[d] - lo[d]) / n;
    m->points.resize(3 * nv * nv * nv);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    for (int64_t k = 0; k < nv; ++k)
        for (int64_t j = 0; j < nv; ++j)
            for (int64_t i = 0; i < nv; ++i) {
                const int64_t c[3] = {i, j, k};
                double* x = &m->points[3 * pid(i, j, k)];
                for (int d = 0; d < 3; ++d) x[d] = (c[d] == n) ? hi[d] : lo[d] + h[d] * (double)c[d];
                const bool interior = i > 0 && i < n && j > 0 && j < n && k > 0 && k < n;
                if (interior && jitter > 0)
                    for (int d = 0; d < 3; ++d) x[d] += jitter * h[d] * uni(rng);
            }
    // Kuhn split: the six monotone lattice paths from (i,j,k) to (i+1,j+1,k+1).
    static const int sig[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
    const int64_t ncell = (int64_t)6 * n * n * n;
    m->cells.resize(4 * ncell);
    int64_t c = 0;
    for (int64_t k = 0; k < n; ++k)
        for (int64_t j = 0; j < n; ++j)
            for (int64_t i = 0; i < n; ++i)
                for (int s = 0; s < 6; ++s, ++c) {
                    int64_t a[3] = {i, j, k};
                    int64_t nodes[4];
                    nodes[0] = pid(a[0], a[1], a[2]);
                    a[sig[s][0]] += 1;
                    nodes[1] = pid(a[0], a[1], a[2]);
                    a[sig[s][1]] += 1;
                    nodes[2] = pid(a[0], a[1], a[2]);
                    nodes[3] = pid(i + 1, j + 1, k + 1);
                    if (s >= 3) std::swap(nodes[1], nodes[2]);  // odd paths: keep det > 0
                    for (int q = 0; q < 4; ++q) m->cells[4 * c + q] = nodes[q];
                }
    // faces: local face f of a cell omits local node f; nodes kept in ascending local order
    static const int lf[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    std::unordered_map<std::array<int64_t, 3>, int64_t, KeyHash> map;
    map.reserve(3 * ncell);
    std::vector<int64_t> faces, fcells, cfaces(4 * ncell);
    faces.reserve(7 * ncell);
    fcells.reserve(5 * ncell);
    for (int64_t cc = 0; cc < ncell; ++cc)
        for (int f = 0; f < 4; ++f) {
            int64_t fn[3];
            for (int q = 0; q < 3; ++q) fn[q] = m->cells[4 * cc + lf[f][q]];
            auto key = sorted_key(fn);
            auto it = map.find(key);
            if (it == map.end()) {
                const int64_t id = (int64_t)fcells.size() / 2;
                map.emplace(key, id);
                faces.insert(faces.end(), fn, fn + 3);
                fcells.push_back(cc);
                fcells.push_back(DG_NO_CELL);
                cfaces[4 * cc + f] = id;
            } else {
                if (fcells[2 * it->second + 1] != DG_NO_CELL) { delete m; return fail(DG_E_MESH); }
                fcells[2 * it->second + 1] = cc;
                cfaces[4 * cc + f] = it->second;
            }
        }
    const int64_t nf0 = (int64_t)fcells.size() / 2;
    std::vector<int64_t> fn1(faces);
    std::vector<uint8_t> per(nf0, 0), bcv(nf0, (uint8_t)bc);
    std::vector<char> drop(nf0, 0);
    for (int64_t f = 0; f < nf0; ++f) {
        if (fcells[2 * f + 1] != DG_NO_CELL || drop[f]) continue;
        int64_t cq[3][3];
        for (int q = 0; q < 3; ++q) ijk(faces[3 * f + q], cq[q]);
        for (int d = 0; d < 3; ++d) {
            const bool low = cq[0][d] == 0 && cq[1][d] == 0 && cq[2][d] == 0;
            const bool high = cq[0][d] == n && cq[1][d] == n && cq[2][d] == n;
            if (!(low || high) || !periodic || !periodic[d]) continue;
            int64_t moved[3];
            for (int q = 0; q < 3; ++q) {
                int64_t t[3] = {cq[q][0], cq[q][1], cq[q][2]};
                t[d] += low ? n : -n;
                moved[q] = pid(t[0], t[1], t[2]);
            }
            auto it = map.find(sorted_key(moved));
            if (it == map.end()) { delete m; return fail(DG_E_MESH); }
            const int64_t g = it->second;
            if (fcells[2 * g + 1] != DG_NO_CELL || g == f) { delete m; return fail(DG_E_MESH); }
            // keep f (created first, since later ids are skipped once dropped); pair it with g
            fcells[2 * f + 1] = fcells[2 * g];
            for (int q = 0; q < 3; ++q) fn1[3 * f + q] = moved[q];
            per[f] = 1;
            drop[g] = 1;
            // the partner cell's face slot now points at f
            const int64_t gc = fcells[2 * g];
            for (int q = 0; q < 4; ++q)
                if (cfaces[4 * gc + q] == g) cfaces[4 * gc + q] = f;
        }
    }
    std::vector<int64_t> remap(nf0, -1);
    int64_t nf = 0;
    for (int64_t f = 0; f < nf0; ++f)
        if (!drop[f]) remap[f] = nf++;
    m->faces.resize(3 * nf);
    m->face_nodes1.resize(3 * nf);
    m->face_cells.resize(2 * nf);
    m->periodic.resize(nf);
    m->bc.resize(nf);
    for (int64_t f = 0; f < nf0; ++f) {
        if (drop[f]) continue;
        const int64_t r = remap[f];
        for (int q = 0; q < 3; ++q) {
            m->faces[3 * r + q] = faces[3 * f + q];
            m->face_nodes1[3 * r + q] = fn1[3 * f + q];
        }
        m->face_cells[2 * r] = fcells[2 * f];
        m->face_cells[2 * r + 1] = fcells[2 * f + 1];
        m->periodic[r] = per[f];
        m->bc[r] = bcv[f];
    }
    m->cell_faces.resize(4 * ncell);
    m->cell_cells.resize(4 * ncell);
    for (int64_t cc = 0; cc < ncell; ++cc)
        for (int q = 0; q < 4; ++q) {
            const int64_t r = remap[cfaces[4 * cc + q]];
            if (r < 0) { delete m; return fail(DG_E_MESH); }
            m->cell_faces[4 * cc + q] = r;
            const int64_t a = m->face_cells[2 * r], b = m->face_cells[2 * r + 1];
            m->cell_cells[4 * cc + q] = (b == DG_NO_CELL) ? DG_NO_CELL : (a == cc ? b : a);
        }
    if (err) *err = DG_OK;
    return m;
}

extern "C" void dg_box_mesh_destroy(dg_box_mesh* m) { delete m; }

extern "C" int dg_box_mesh_view(const dg_box_mesh* m, dg_mesh_desc* d, const int64_t** cell_faces,
                                const int64_t** cell_cells) {
    if (!m || !d) return DG_E_ARG;
    std::memset(d, 0, sizeof(*d));
    d->ncell = (int64_t)m->cells.size() / 4;
    d->nface = (int64_t)m->face_cells.size() / 2;
    d->face_cells = m->face_cells.data();
    d->face_bc = m->bc.data();
    d->npts = (int64_t)m->points.size() / 3;
    d->points = m->points.data();
    d->cell_nodes = m->cells.data();
    d->face_nodes = m->faces.data();
    d->face_nodes1 = m->face_nodes1.data();
    d->face_periodic = m->periodic.data();
    if (cell_faces) *cell_faces = m->cell_faces.data();
    if (cell_cells) *cell_cells = m->cell_cells.data();
    return DG_OK;
}

extern "C" int dg_mesh_geometry(const dg_mesh_desc* d, double* normal, double* area, double* natural,
                                double* invjac, double* detj, double* centroid) {
    Geometry g;
    const int rc = build_geometry(d, &g);
    if (rc != DG_OK) return rc;
    const int64_t nf = d->nface, nc = d->ncell;
    if (normal) std::memcpy(normal, g.normal.data(), sizeof(double) * 3 * nf);
    if (area) std::memcpy(area, g.area.data(), sizeof(double) * nf);
    if (invjac) std::memcpy(invjac, g.invjac.data(), sizeof(double) * 9 * nc);
    if (detj) std::memcpy(detj, g.detj.data(), sizeof(double) * nc);
    if (natural) {
        for (int64_t f = 0; f < nf; ++f)
            for (int s = 0; s < 2; ++s) {
                double* nc9 = natural + 18 * f + 9 * s;
                std::memset(nc9, 0, sizeof(double) * 9);
                const int p = g.perm[2 * f + s];
                if (p < 0) continue;
                for (int k = 0; k < 3; ++k) {
                    const int slot = kPermSlots[p][k];
                    if (slot > 0) nc9[3 * k + slot - 1] = 1.0;
                }
            }
    }
    if (centroid) {
        if (!d->points || !d->cell_nodes) return DG_E_ARG;
        for (int64_t c = 0; c < nc; ++c) {
            const int64_t* cn = d->cell_nodes + 4 * c;
            for (int i = 0; i < 3; ++i)
                centroid[3 * c + i] = (((d->points[3 * cn[0] + i] + d->points[3 * cn[1] + i]) +
                                        d->points[3 * cn[2] + i]) + d->points[3 * cn[3] + i]) / 4.0;
        }
    }
    return DG_OK;
}

extern "C" int dg_face_perms(const dg_mesh_desc* d, int8_t* perm) {
    Geometry g;
    const int rc = build_geometry(d, &g);
    if (rc != DG_OK) return rc;
    if (perm) std::memcpy(perm, g.perm.data(), g.perm.size());
    return DG_OK;
}
