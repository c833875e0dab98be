// VTK legacy ASCII solution writer in the layout of the reference's
// VTK_Writer (Euler3D/src/MeshIO.cpp:219-372), conservative variables:
// points, cells (surface triangles, then tetrahedra), cell types, boundary
// ids, then density, velocity components, pressure, temperature, Mach number
// and the velocity vector of every physical node.  Host code; the derived
// fields are formed in the reference's operation order (Get_Pressure,
// Get_Temperature, Get_Mach of Material.cpp:701-1080 under the generic
// non-dimensionalisation, R = 1/gamma), so an ideal-gas file is byte-identical
// to the reference's for the same mesh and state.  With the stiffened-gas
// constant pinf the pressure is (gamma - 1)(rho et - rho q^2/2) - gamma pinf,
// the temperature (p + pinf)/(R rho) and the sound speed sqrt(gamma (p + pinf)/rho).
//
// Surface triangles are written in the orientation the reference gives them
// after reading (Verify_Surface_Connectivity, Euler3D/src/Connectivity_Maps.cpp:
// 782-899): reversed when their normal (n1-n0) x (n2-n0) points away from the
// centroid of the tetrahedron they bound.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <unordered_map>
#include <vector>

#include "cfd_internal.h"

namespace {

struct TriKeyHash {
    size_t operator()(const std::array<int, 3> &k) const {
        uint64_t h = (uint64_t)(uint32_t)k[0] * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)k[1] + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k[2] + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

// flip[t] = 1 where surface triangle t must be reversed so that its normal
// points into its tetrahedron (the reference's surface-orientation check).
std::vector<char> inward_flips(int nnode, const double *xyz, int64_t ntri, const int *tris, int64_t ntet,
                               const int *tets) {
    std::vector<char> flip((size_t)ntri, 0);
    if (!ntri || !ntet) return flip;
    std::unordered_map<std::array<int, 3>, int64_t, TriKeyHash> face;
    face.reserve((size_t)ntri * 2);
    for (int64_t t = 0; t < ntri; t++) {
        std::array<int, 3> k = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(k.begin(), k.end());
        face.emplace(k, t);
    }
    std::vector<int64_t> owner((size_t)ntri, -1);
    static const int fv[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (int64_t c = 0; c < ntet; c++)
        for (int f = 0; f < 4; f++) {
            std::array<int, 3> k = {tets[4 * c + fv[f][0]], tets[4 * c + fv[f][1]], tets[4 * c + fv[f][2]]};
            std::sort(k.begin(), k.end());
            auto it = face.find(k);
            if (it != face.end() && owner[it->second] < 0) owner[it->second] = c;
        }
    auto unit = [](double v[3]) {
        const double m = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (m > 1.0e-20) { v[0] = v[0] / m; v[1] = v[1] / m; v[2] = v[2] / m; }
    };
    for (int64_t t = 0; t < ntri; t++) {
        const int64_t c = owner[t];
        if (c < 0) continue;
        const int *s = tris + 3 * t;
        const double *p0 = xyz + 3 * (size_t)s[0], *p1 = xyz + 3 * (size_t)s[1], *p2 = xyz + 3 * (size_t)s[2];
        const double a[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        const double b[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        double nv[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        unit(nv);
        double sc[3] = {0.0, 0.0, 0.0}, vc[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 3; i++)
            for (int d = 0; d < 3; d++) sc[d] += xyz[3 * (size_t)s[i] + d];
        for (int d = 0; d < 3; d++) sc[d] /= 3.0;
        for (int i = 0; i < 4; i++)
            for (int d = 0; d < 3; d++) vc[d] += xyz[3 * (size_t)tets[4 * c + i] + d];
        for (int d = 0; d < 3; d++) vc[d] /= 4.0;
        double r[3] = {vc[0] - sc[0], vc[1] - sc[1], vc[2] - sc[2]};
        unit(r);
        if (r[0] * nv[0] + r[1] * nv[1] + r[2] * nv[2] < 0.0) flip[t] = 1;
    }
    (void)nnode;
    return flip;
}

}  // namespace

extern "C" int cfd_vtk_write(const char *path, int nnode, const double *coords, int64_t ntri, const int *tris,
                             const int *tri_tag, int64_t ntet, const int *tets, const cfd_params *p, const double *Q,
                             int64_t ld) {
    if (!path || nnode < 0 || ntri < 0 || ntet < 0 || !p || ld < nnode || (nnode && (!coords || !Q)) ||
        (ntri && !tris) || (ntet && !tets) || !(p->gamma > 1.0)) {
        cfd::set_error("cfd_vtk_write: bad arguments");
        return CFD_ERR_ARG;
    }
    FILE *fp = std::fopen(path, "w");
    if (!fp) {
        cfd::set_error("cfd_vtk_write: cannot write %s", path);
        return CFD_ERR_IO;
    }
    const double g = p->gamma, pinf = p->pinf, R = 1.0 / g;
    const double *Q1 = Q, *Q2 = Q + ld, *Q3 = Q + 2 * ld, *Q4 = Q + 3 * ld, *Q5 = Q + 4 * ld;
    // a (rho, u, v, w, p) state (CFD_VARS_RUP) is written through its conservative form
    std::vector<double> qc;
    if (p->variables == CFD_VARS_RUP) {
        qc.resize((size_t)5 * nnode);
        for (int i = 0; i < nnode; i++) {
            const double r = Q1[i], u = Q2[i], v = Q3[i], w = Q4[i];
            qc[i] = r;
            qc[(size_t)nnode + i] = r * u;
            qc[(size_t)2 * nnode + i] = r * v;
            qc[(size_t)3 * nnode + i] = r * w;
            qc[(size_t)4 * nnode + i] = (Q5[i] + g * pinf) / (g - 1.0) + 0.5 * r * (u * u + v * v + w * w);
        }
        Q1 = qc.data(); Q2 = Q1 + nnode; Q3 = Q2 + nnode; Q4 = Q3 + nnode; Q5 = Q4 + nnode;
    }
    std::fprintf(fp, "# vtk DataFile Version 2.0\n");
    std::fprintf(fp, "Solver solution data\n");
    std::fprintf(fp, "ASCII \n");
    std::fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    std::fprintf(fp, "POINTS %d double\n", nnode);
    for (int i = 0; i < nnode; i++)
        std::fprintf(fp, "%f %f %f\n", coords[3 * (size_t)i], coords[3 * (size_t)i + 1], coords[3 * (size_t)i + 2]);
    const long long ncell = (long long)(ntri + ntet);
    const std::vector<char> flip = inward_flips(nnode, coords, ntri, tris, ntet, tets);
    std::fprintf(fp, "CELLS %lld %lld\n", ncell, (long long)(4 * ntri + 5 * ntet));
    for (int64_t t = 0; t < ntri; t++) {
        if (flip[t]) std::fprintf(fp, "3 %d %d %d\n", tris[3 * t + 2], tris[3 * t + 1], tris[3 * t]);
        else std::fprintf(fp, "3 %d %d %d\n", tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]);
    }
    for (int64_t t = 0; t < ntet; t++)
        std::fprintf(fp, "4 %d %d %d %d\n", tets[4 * t], tets[4 * t + 1], tets[4 * t + 2], tets[4 * t + 3]);
    std::fprintf(fp, "CELL_TYPES %lld\n", ncell);
    for (int64_t t = 0; t < ntri; t++) std::fprintf(fp, "5\n");
    for (int64_t t = 0; t < ntet; t++) std::fprintf(fp, "10\n");
    std::fprintf(fp, "CELL_DATA %lld\n", ncell);
    std::fprintf(fp, "SCALARS BoundaryIds Int 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int64_t t = 0; t < ntri; t++) std::fprintf(fp, "%d\n", tri_tag ? tri_tag[t] : 1);
    for (int64_t t = 0; t < ntet; t++) std::fprintf(fp, "0\n");
    std::fprintf(fp, "POINT_DATA %d\n", nnode);
    const char *names[4] = {"Density", "X_Velocity", "Y_Velocity", "Z_Velocity"};
    for (int v = 0; v < 4; v++) {
        std::fprintf(fp, "SCALARS %s double 1\n", names[v]);
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (int i = 0; i < nnode; i++) {
            const double x = v == 0 ? Q1[i] : (v == 1 ? Q2[i] / Q1[i] : (v == 2 ? Q3[i] / Q1[i] : Q4[i] / Q1[i]));
            std::fprintf(fp, "%22.15e\n", x);
        }
    }
    std::fprintf(fp, "SCALARS Pressure double 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < nnode; i++) {
        const double pr = (g - 1.0) * (Q5[i] - 0.5 * (Q2[i] * Q2[i] + Q3[i] * Q3[i] + Q4[i] * Q4[i]) / Q1[i]);
        std::fprintf(fp, "%22.15e\n", pinf != 0.0 ? pr - g * pinf : pr);
    }
    std::fprintf(fp, "SCALARS Temperature double 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < nnode; i++) {
        const double pr = (g - 1.0) * (Q5[i] - 0.5 * (Q2[i] * Q2[i] + Q3[i] * Q3[i] + Q4[i] * Q4[i]) / Q1[i]);
        // p + pinf = (g - 1)(rho et - rho q^2/2) - (g - 1) pinf
        const double pp = pinf != 0.0 ? pr - (g - 1.0) * pinf : pr;
        std::fprintf(fp, "%22.15e\n", pp / (R * Q1[i]));
    }
    std::fprintf(fp, "SCALARS Mach double 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < nnode; i++) {
        const double q2 = (Q2[i] * Q2[i] + Q3[i] * Q3[i] + Q4[i] * Q4[i]) / (Q1[i] * Q1[i]);
        const double pr = (g - 1.0) * (Q5[i] - 0.5 * Q1[i] * q2);
        const double pp = pinf != 0.0 ? pr - (g - 1.0) * pinf : pr;
        std::fprintf(fp, "%22.15e\n", std::sqrt(q2 * Q1[i] / (g * pp)));
    }
    std::fprintf(fp, "VECTORS Velocity double \n");
    for (int i = 0; i < nnode; i++)
        std::fprintf(fp, "%22.15e \t %22.15e \t %22.15e\n", Q2[i] / Q1[i], Q3[i] / Q1[i], Q4[i] / Q1[i]);
    const bool bad = std::ferror(fp) != 0;
    std::fclose(fp);
    if (bad) {
        cfd::set_error("cfd_vtk_write: write error on %s", path);
        return CFD_ERR_IO;
    }
    return CFD_OK;
}
