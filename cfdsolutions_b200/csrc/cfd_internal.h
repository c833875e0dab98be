// Internal types of the B200 edge-based finite-volume library.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"

namespace cfd {

// Host mesh produced by the builder (mesh.cpp).
struct HostMesh {
    int nnode = 0, nghost = 0, nedge = 0, nbedge = 0;
    std::vector<double> coords;      // [3*nnode] xyz interleaved
    std::vector<int> tets;           // [4*ntet]
    std::vector<int> tris;           // [3*ntri]
    std::vector<int> tri_bc;         // [ntri]
    std::vector<int> edge_nodes;     // [2*nedge]
    std::vector<double> edge_areav;  // [3*nedge]
    std::vector<int> bedge_nodes;    // [2*nbedge]
    std::vector<double> bedge_areav; // [3*nbedge]
    std::vector<int> bedge_type;     // [nbedge]
    std::vector<double> cvol;        // [nnode]
    std::vector<int> n2n_ia, n2n_ja; // node graph without diagonal
};

int build_box(HostMesh &m, int nx, int ny, int nz, double lx, double ly, double lz, double jitter,
              uint64_t seed, int renumber, const int face_bc[6]);
int build_from_cells(HostMesh &m, int nnode, const double *coords, int64_t ntet, const int *tets,
                     int64_t ntri, const int *tris, const int *tri_bc);
int write_ugrid(const HostMesh &m, const char *path, const int *tri_tag);

void set_error(const char *fmt, ...);

}  // namespace cfd

struct cfd_mesh {
    cfd::HostMesh m;
};
