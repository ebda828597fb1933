/* Test infrastructure (oracle): a plain-C restatement of the reference's explicit DG operator for
 * the 3D compressible Euler equations on affine tetrahedra, plus the SSP-RK3 loop, the diagonal
 * mass and the conservation sums. Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and only as the checker. The product never calls it.
 *
 * Parity is pinned against the reference itself: tests compare this restatement with the
 * reference's own ExplicitConvection::eval compiled from source (oracle/_ref) and with the golden
 * vectors under tests/golden/ that were produced from it.
 *
 * Mesh arguments (all row-major, int64 indices):
 *   pts[npts*3], cells[ncell*4] (tet nodes), faces[nface*3] (face nodes),
 *   face_cells[nface*2] (cells[1] = -1 on a boundary face),
 *   face_nodes1[nface*3]: the face's nodes as numbered in cells[1] (equal to faces[] for an
 *   interior face; the translated partner nodes for a periodic face),
 *   periodic[nface]: 1 when the face pairs two cells across a periodic boundary,
 *   bc[nface]: BoundaryType of include/Mesh/ComputingMesh.h:71-86 for boundary faces.
 */
#ifndef FVEDG_ORACLE_H
#define FVEDG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t npts;
    const double* pts;
    int64_t ncell;
    const int64_t* cells;
    int64_t nface;
    const int64_t* faces;
    const int64_t* face_cells;
    const int64_t* face_nodes1;
    const uint8_t* periodic;
    const uint8_t* bc;
} orc_mesh;

enum { ORC_FLUX_LF = 0, ORC_FLUX_ROE = 1 };

int orc_num_basis(int order);
int orc_basis(int order, int npts, const double* xyz, double* phi, double* grad);
int orc_geometry(const orc_mesh* m, double* normals, double* areas, double* natc, double* invjac,
                 double* detj, double* centroid);
int orc_residual(const orc_mesh* m, int order, double gamma, int flux, int qv, int qf,
                 const double* U, double* R, double t, const double* dirichlet10, int part);
int orc_mass(const orc_mesh* m, int order, int qv, double* mass);
int orc_ssprk3(const orc_mesh* m, int order, double gamma, int flux, int qv, int qf, double* U,
               const double* mass, double dt, int nsteps, double t0, const double* dirichlet10);
int orc_conservation(const orc_mesh* m, int order, int qv, double gamma, const double* U,
                     double out6[6]);
/* The numerical flux 2A-free F^(UL, UR, n) of one face point (ORC_FLUX_LF or ORC_FLUX_ROE). */
int orc_numerical_flux(int kind, const double* UL, const double* UR, const double* n, double gamma, double* Fh);

#ifdef __cplusplus
}
#endif
#endif
