// Test infrastructure (oracle): a stand-in for the reference's Mesh/MeshGenerator.h.
//
// The reference header (include/Mesh/MeshGenerator.h:1-119) pulls in CGAL, which needs Boost,
// which this image lacks. ComputingMesh.h only needs `struct DGMesh` from it
// (include/Mesh/MeshGenerator.h:46-57, consumed by ComputingMesh(const DGMesh&) in
// src/Mesh/ComputingMesh.cpp:268-298), so this shim declares that struct alone with the same
// field order and types. It sits ahead of the reference include path in oracle/Makefile.
#pragma once
#include <array>
#include <cstddef>
#include <vector>

struct DGMesh {
    std::vector<std::array<double, 3>> points;
    std::vector<std::array<size_t, 3>> faces;
    std::vector<std::array<size_t, 4>> cells;
    std::vector<std::array<size_t, 4>> cell_faces;
    std::vector<std::array<size_t, 4>> cell_cells;
    std::vector<std::array<size_t, 2>> face_cells;
    std::vector<bool> is_boundary_face;
};
