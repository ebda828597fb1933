// Internal declarations shared by the host-side C++ (mesh, geometry, tables) and the CUDA side.
#pragma once
#include <cstdint>
#include <vector>

#include "dg_gpu.h"

namespace fvedg {

constexpr int kMaxOrder = 5;
constexpr int kNumPerms = 24;

inline int num_basis(int order) { return (order + 1) * (order + 2) * (order + 3) / 6; }

// The reference's AutoQuadSelector choices (AutoQuadSelectorTet.h:2-50, AutoQuadSelectorTri.h:1-45)
// mapped to this library's rule ids.
int auto_tet_rule(int order);
int auto_tri_rule(int order);
int tet_rule_npts(int id);
int tri_rule_npts(int id);
const double* tet_rule(int id);  // npts rows of (x, y, z, w)
const double* tri_rule(int id);  // npts rows of (x, y, w)

// Ordered vertex triples (slot of face node 0, 1, 2 in the cell, slots 0..3) for codes 0..23.
extern const int kPermSlots[kNumPerms][3];
int perm_code(int s0, int s1, int s2);

// Basis values and reference gradients at one point (Dubiner-type modal basis of
// include/DG/DG_Basis/DG_Basis_Func.h, evaluated from its Jacobi-polynomial definition).
void basis_eval(int order, double x, double y, double z, double* phi, double* grad);

// Geometry of one mesh, computed with the reference's arithmetic (ComputingMesh.cpp:27-171).
struct Geometry {
    std::vector<double> normal;   // [nface][3]
    std::vector<double> area;     // [nface]
    std::vector<int8_t> perm;     // [nface][2]
    std::vector<double> invjac;   // [ncell][9]
    std::vector<double> detj;     // [ncell]
};
// Validates the description and fills g. Returns DG_OK or an error code.
int build_geometry(const dg_mesh_desc* d, Geometry* g);

// Device-side constant tables for one (order, rules) choice.
struct Tables {
    int order = 0, nb = 0, nqv = 0, nqf = 0;
    std::vector<double> phi_v;      // [nqv][nb]
    std::vector<double> phi_vT;     // [nb][nqv]
    std::vector<double> dphi_vw;    // [nqv][nb][3] reference gradients times w_g
    std::vector<double> dphi_v;     // [nqv][nb][3] reference gradients
    std::vector<double> dphi_f;     // [24][nqf][nb][3] reference gradients at the face points
    std::vector<double> w_v;        // [nqv]
    std::vector<double> phi_f;      // [24][nqf][nb] face point basis values per face map
    std::vector<double> phi_fT;     // [24][nb][nqf]
    std::vector<double> w_f;        // [nqf]
    std::vector<double> mass_ref;   // [nb] sum_g w_g phi_i(x_g)^2 on the reference tet
};
void build_tables(int order, int qv, int qf, Tables* t);

}  // namespace fvedg
