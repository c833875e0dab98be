// Internal types of the B200 edge-based finite-volume library.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"

namespace cfd {

// Threads the host mesh builder may use on the calling thread (0: up to 16).
// The serving workers set a small number, so that a request's mesh build
// does not take the cores the other workers' launches run on.
inline thread_local int g_host_threads = 0;

// Host mesh produced by the builder (mesh.cpp).
struct HostMesh {
    int nnode = 0, nghost = 0, nedge = 0, nbedge = 0;
    std::vector<double> coords;      // [3*nnode] xyz interleaved
    std::vector<int> tets;           // [4*ntet]
    std::vector<int> pyrs;           // [5*npyr]   base quad 0-3, apex 4
    std::vector<int> prisms;         // [6*nprism] triangles 0-1-2 and 3-4-5, sides 0-3, 1-4, 2-5
    std::vector<int> hexes;          // [8*nhex]   bottom 0-1-2-3, top 4-5-6-7, sides i - i+4
    std::vector<int> tris;           // [3*ntri]   boundary, outward right-hand normal
    std::vector<int> tri_bc;         // [ntri]
    std::vector<int> quads;          // [4*nquad]  boundary, outward right-hand normal
    std::vector<int> quad_bc;        // [nquad]
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
int read_ugrid(HostMesh &m, const char *path, int ntag, const int *tag_bc, int renumber);

void set_error(const char *fmt, ...);

}  // namespace cfd

struct cfd_mesh {
    cfd::HostMesh m;
};
