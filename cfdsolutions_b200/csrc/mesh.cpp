// Host-side median-dual mesh builder, O(N + E): tet-split box generator,
// reverse Cuthill-McKee renumbering, node-centred median-dual metrics, ghost
// nodes for boundary edges, and the node-to-node CRS graph.
//
// It produces exactly the arrays the reference's pre-processing produces, in
// the reference's conventions:
//   * interior edges (node_L < node_R), area vector pointing from node_L to
//     node_R, summed over the two dual-face triangles of every cell edge
//     (Euler3D/src/Area_Volume.cpp:659-800);
//   * one boundary edge and one private ghost node per boundary-triangle
//     vertex, ghost index = nNode + boundary-edge index, area = one third of
//     the triangle's outward area vector (Area_Volume.cpp:461-556, flipped
//     outward at :912-913);
//   * control volume = sum of median-dual sub-volumes (V_tet / 4 per vertex);
//   * node2node CRS without the diagonal (Connectivity_Maps.cpp:915-985).
// The reference builds node2Edge in O(N*E) (Connectivity_Maps.cpp:766-780) and
// renumbers with an O(N^2) Cuthill-McKee (Cuthill_Mckee_Reorder.cpp:17-155);
// this builder is linear in the mesh size so 128^3-hex meshes build in seconds.
// The node graph and the dual are gathered per node from node -> element
// incidence lists, on up to 16 threads, in the order one loop over the
// elements would sum them (the same bits); the renumbering's bisection and
// patch graph run on threads too.
#include "cfd_internal.h"
#include "host_par.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace cfd {

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform in [-1, 1)
    double sym() { return ((next() >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0; }
};

inline void sub3(const double *a, const double *b, double *o) {
    o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2];
}
inline void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Local edges and faces of the volume element types in the node orders
// above (the geometry of each type; the reference lists the same edges with
// their two faces in Get_Edge_Nodes_Faces_Connectivity, Area_Volume.cpp:20-458).
const int kTetEdges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
const int kPyrEdges[8][2] = {{0, 1}, {0, 3}, {0, 4}, {1, 2}, {1, 4}, {2, 3}, {2, 4}, {3, 4}};
const int kPrismEdges[9][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 4}, {2, 5}, {3, 4}, {3, 5}, {4, 5}};
const int kHexEdges[12][2] = {{0, 1}, {0, 3}, {0, 4}, {1, 2}, {1, 5}, {2, 3},
                              {2, 6}, {3, 7}, {4, 5}, {4, 7}, {5, 6}, {6, 7}};
struct ElemType {
    int nnode, nedge, nface;
    const int (*edges)[2];
    int face[6][4];  // node lists, -1 padded (triangles)
};
const ElemType kPyr = {5, 8, 5, kPyrEdges, {{0, 1, 2, 3}, {0, 1, 4, -1}, {1, 2, 4, -1}, {2, 3, 4, -1}, {3, 0, 4, -1}}};
const ElemType kPrism = {6, 9, 5, kPrismEdges,
                         {{0, 1, 2, -1}, {3, 4, 5, -1}, {0, 1, 4, 3}, {1, 2, 5, 4}, {2, 0, 3, 5}}};
const ElemType kHex = {8, 12, 6, kHexEdges,
                       {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}}};

// The volume elements of a mesh as one sequence of keys: tetrahedra, then
// pyramids, prisms and hexahedra, each in its own order (the order the
// element loops of the dual visit them), with each node's incident elements
// in increasing key order.
struct Cells {
    const int *v[4];     // node lists per type
    int nn[4];           // nodes per element
    int64_t off[5];      // first key of each type; off[4] = elements
    const int (*edges[4])[2];
    int nedge[4];
    std::vector<int64_t> ptr;  // [nnode+1] into key
    std::vector<int> key;

    explicit Cells(const HostMesh &m) {
        const std::vector<int> *lists[4] = {&m.tets, &m.pyrs, &m.prisms, &m.hexes};
        const int nns[4] = {4, kPyr.nnode, kPrism.nnode, kHex.nnode};
        const int (*eds[4])[2] = {kTetEdges, kPyrEdges, kPrismEdges, kHexEdges};
        const int nes[4] = {6, kPyr.nedge, kPrism.nedge, kHex.nedge};
        off[0] = 0;
        for (int t = 0; t < 4; t++) {
            v[t] = lists[t]->data();
            nn[t] = nns[t];
            edges[t] = eds[t];
            nedge[t] = nes[t];
            off[t + 1] = off[t] + (int64_t)lists[t]->size() / nns[t];
        }
        ptr.assign((size_t)m.nnode + 1, 0);
        for (int t = 0; t < 4; t++)
            for (int64_t e = 0; e < off[t + 1] - off[t]; e++)
                for (int k = 0; k < nn[t]; k++) ptr[v[t][e * nn[t] + k] + 1]++;
        for (int a = 0; a < m.nnode; a++) ptr[a + 1] += ptr[a];
        key.resize(ptr[m.nnode]);
        std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
        for (int t = 0; t < 4; t++)
            for (int64_t e = 0; e < off[t + 1] - off[t]; e++)
                for (int k = 0; k < nn[t]; k++) key[fill[v[t][e * nn[t] + k]]++] = (int)(off[t] + e);
    }
    int type_of(int k) const {
        int t = 0;
        while (k >= off[t + 1]) t++;
        return t;
    }
};

// Symmetric node graph of a mesh: CRS without diagonal, rows sorted.  Each
// row is gathered from the node's incident elements (their edges through the
// node), in parallel over node ranges.
void build_graph(const HostMesh &msh, const Cells &cells, std::vector<int> &ia, std::vector<int> &ja) {
    const int nnode = msh.nnode;
    auto row = [&](int a, std::vector<int> &nb) {
        nb.clear();
        for (int64_t q = cells.ptr[a]; q < cells.ptr[a + 1]; q++) {
            const int k = cells.key[q], t = cells.type_of(k);
            const int *v = cells.v[t] + (int64_t)(k - cells.off[t]) * cells.nn[t];
            for (int p = 0; p < cells.nedge[t]; p++) {
                const int x = v[cells.edges[t][p][0]], y = v[cells.edges[t][p][1]];
                if (x == a) nb.push_back(y);
                else if (y == a) nb.push_back(x);
            }
        }
        std::sort(nb.begin(), nb.end());
        nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
    };
    // rows of each range into that range's own buffer, then placed in one copy
    ia.assign(nnode + 1, 0);
    const int nt = range_count(nnode);
    std::vector<std::vector<int>> part(nt);
    std::vector<int> part_lo(nt, 0);
    parallel_ranges(nnode, [&](int t, int lo, int hi) {
        std::vector<int> nb, buf;
        for (int a = lo; a < hi; a++) {
            row(a, nb);
            ia[a + 1] = (int)nb.size();
            buf.insert(buf.end(), nb.begin(), nb.end());
        }
        part[t].swap(buf);
        part_lo[t] = lo;
    });
    for (int a = 0; a < nnode; a++) ia[a + 1] += ia[a];
    ja.assign(ia[nnode], 0);
    for (int t = 0; t < nt; t++) std::copy(part[t].begin(), part[t].end(), ja.begin() + ia[part_lo[t]]);
}

void build_graph(const HostMesh &msh, std::vector<int> &ia, std::vector<int> &ja) {
    const Cells cells(msh);
    build_graph(msh, cells, ia, ja);
}

// Reverse Cuthill-McKee, O(N + E log d).  Start node: a pseudo-peripheral node
// found by repeated BFS from a minimum-degree node.  Returns perm[new] = old.
std::vector<int> rcm_order(int n, const std::vector<int> &ia, const std::vector<int> &ja) {
    std::vector<int> order;
    order.reserve(n);
    std::vector<char> seen(n, 0);
    std::vector<int> level(n, -1), q;
    auto deg = [&](int v) { return ia[v + 1] - ia[v]; };
    auto bfs_last = [&](int s, int &depth) {
        std::fill(level.begin(), level.end(), -1);
        q.clear();
        q.push_back(s);
        level[s] = 0;
        size_t h = 0;
        int last = s;
        while (h < q.size()) {
            int v = q[h++];
            for (int k = ia[v]; k < ia[v + 1]; k++) {
                int w = ja[k];
                if (level[w] < 0) {
                    level[w] = level[v] + 1;
                    q.push_back(w);
                    // deepest level, minimum degree
                    if (level[w] > level[last] || (level[w] == level[last] && deg(w) < deg(last))) last = w;
                }
            }
        }
        depth = level[last];
        return last;
    };
    for (int comp_seed = 0; comp_seed < n; comp_seed++) {
        if (seen[comp_seed]) continue;
        int s = comp_seed, d0 = -1;
        for (int it = 0; it < 4; it++) {
            int d;
            int far = bfs_last(s, d);
            if (d <= d0) break;
            d0 = d;
            s = far;
        }
        size_t base = order.size();
        order.push_back(s);
        seen[s] = 1;
        std::vector<int> nb;
        for (size_t h = base; h < order.size(); h++) {
            int v = order[h];
            nb.clear();
            for (int k = ia[v]; k < ia[v + 1]; k++)
                if (!seen[ja[k]]) { nb.push_back(ja[k]); seen[ja[k]] = 1; }
            std::sort(nb.begin(), nb.end(), [&](int x, int y) { return deg(x) < deg(y) || (deg(x) == deg(y) && x < y); });
            order.insert(order.end(), nb.begin(), nb.end());
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// Recursive coordinate bisection into patches of exactly `psz` nodes (the last
// one may be smaller): split the longest extent at a multiple of psz near the
// middle.  Returns nodes in patch-major order.
void rcb_patches(const std::vector<double> &xyz, int psz, std::vector<int> &idx, int lo, int hi, int depth = 0) {
    const int n = hi - lo;
    if (n <= psz) return;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int k = lo; k < hi; k++)
        for (int d = 0; d < 3; d++) {
            const double v = xyz[3 * (size_t)idx[k] + d];
            mn[d] = std::min(mn[d], v);
            mx[d] = std::max(mx[d], v);
        }
    int ax = 0;
    for (int d = 1; d < 3; d++)
        if (mx[d] - mn[d] > mx[ax] - mn[ax]) ax = d;
    const int npatch = (n + psz - 1) / psz;
    const int mid = lo + ((npatch + 1) / 2) * psz;
    std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int a, int b) {
        const double va = xyz[3 * (size_t)a + ax], vb = xyz[3 * (size_t)b + ax];
        return va < vb || (va == vb && a < b);
    });
    // the halves are independent: the first levels split across threads
    if (depth < 3 && (1 << (depth + 1)) <= range_count(n) && n >= 65536) {
        std::thread left([&] { rcb_patches(xyz, psz, idx, lo, mid, depth + 1); });
        rcb_patches(xyz, psz, idx, mid, hi, depth + 1);
        left.join();
        return;
    }
    rcb_patches(xyz, psz, idx, lo, mid, depth + 1);
    rcb_patches(xyz, psz, idx, mid, hi, depth + 1);
}

// Blocked reverse Cuthill-McKee: RCB patches of psz nodes, patches ordered by
// RCM of the patch adjacency graph, nodes inside a patch in their original
// order.  Every patch is then a contiguous, spatially compact node range
// (what the patch residual kernel works on) and the matrix stays banded at the
// patch level.  Returns perm[new] = old.
std::vector<int> patch_rcm_order(int n, const std::vector<double> &xyz, const std::vector<int> &ia,
                                 const std::vector<int> &ja, int psz) {
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    rcb_patches(xyz, psz, idx, 0, n);
    const int np = (n + psz - 1) / psz;
    std::vector<int> pid(n);
    for (int k = 0; k < n; k++) pid[idx[k]] = k / psz;
    // patch graph, each patch's row from its own nodes (patch p = idx[p*psz ..])
    std::vector<std::vector<int>> adj(np);
    parallel_ranges(np, [&](int, int lo, int hi) {
        for (int p = lo; p < hi; p++) {
            std::vector<int> &r = adj[p];
            for (int q = p * psz; q < std::min(n, (p + 1) * psz); q++) {
                const int a = idx[q];
                for (int k = ia[a]; k < ia[a + 1]; k++)
                    if (pid[ja[k]] != p) r.push_back(pid[ja[k]]);
            }
            std::sort(r.begin(), r.end());
            r.erase(std::unique(r.begin(), r.end()), r.end());
        }
    });
    std::vector<int> pia(np + 1, 0), pja;
    for (int p = 0; p < np; p++) {
        pia[p + 1] = pia[p] + (int)adj[p].size();
        pja.insert(pja.end(), adj[p].begin(), adj[p].end());
    }
    std::vector<int> porder = rcm_order(np, pia, pja);  // porder[new] = old patch
    std::vector<int> perm;
    perm.reserve(n);
    for (int q = 0; q < np; q++) {
        const int p = porder[q];
        const int b = p * psz, e = std::min(n, b + psz);
        std::vector<int> nodes(idx.begin() + b, idx.begin() + e);
        std::sort(nodes.begin(), nodes.end());
        perm.insert(perm.end(), nodes.begin(), nodes.end());
    }
    return perm;
}

}  // namespace

// Build the median-dual metrics of a tet mesh into m (coords/tets/tris set).
static int build_dual(HostMesh &m) {
    const int nnode = m.nnode;
    const Cells cells(m);
    build_graph(m, cells, m.n2n_ia, m.n2n_ja);

    // Interior edges = upper half of the graph, ordered by (L, R).
    std::vector<int> eoff(nnode + 1, 0);  // first edge of each L
    parallel_ranges(nnode, [&](int, int lo, int hi) {
        for (int a = lo; a < hi; a++) {
            const int *r = &m.n2n_ja[m.n2n_ia[a]], *r1 = &m.n2n_ja[0] + m.n2n_ia[a + 1];
            eoff[a + 1] = (int)(r1 - std::upper_bound(r, r1, a));  // rows are sorted
        }
    });
    for (int a = 0; a < nnode; a++) eoff[a + 1] += eoff[a];
    const int nedge = eoff[nnode];
    m.edge_nodes.assign((size_t)2 * nedge, 0);
    parallel_ranges(nnode, [&](int, int lo, int hi) {
        for (int a = lo; a < hi; a++) {
            int e = eoff[a];
            for (int k = m.n2n_ia[a]; k < m.n2n_ia[a + 1]; k++)
                if (m.n2n_ja[k] > a) {
                    m.edge_nodes[2 * (size_t)e] = a;
                    m.edge_nodes[2 * (size_t)e + 1] = m.n2n_ja[k];
                    e++;
                }
        }
    });
    m.nedge = nedge;
    m.edge_areav.assign((size_t)3 * nedge, 0.0);
    m.cvol.assign(nnode, 0.0);

    auto edge_id = [&](int a, int b) {
        // a < b; upper neighbours of a are sorted within [eoff[a], eoff[a+1])
        int lo = eoff[a], hi = eoff[a + 1];
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (m.edge_nodes[2 * mid + 1] < b) lo = mid + 1; else hi = mid;
        }
        return lo;
    };

    // The dual is gathered per node, in parallel over node ranges: node a
    // visits its incident elements in element order and adds, for every
    // element edge (a, b) with b > a, the edge's dual-face area to edge (a, b),
    // and its own share of every element to its control volume.  Each edge and
    // each volume receives the same terms, formed by the same operations, in
    // the same order as one loop over the elements would add them, so the
    // results are the same bit for bit.
    std::vector<int> bad_in(range_count(nnode), 0);  // tetrahedra with non-positive volume, per range
    static const int pairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    static const int others[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
    // the two faces of each local edge of the pyramid, prism and hexahedron
    const ElemType *types[4] = {nullptr, &kPyr, &kPrism, &kHex};
    int ef[4][12][2];
    for (int tt = 1; tt < 4; tt++) {
        const ElemType &T = *types[tt];
        for (int p = 0; p < T.nedge; p++) {
            int k = 0;
            for (int f = 0; f < T.nface && k < 2; f++) {
                bool ha = false, hb = false;
                for (int q = 0; q < 4 && T.face[f][q] >= 0; q++) {
                    ha |= T.face[f][q] == T.edges[p][0];
                    hb |= T.face[f][q] == T.edges[p][1];
                }
                if (ha && hb) ef[tt][p][k++] = f;
            }
        }
    }
    parallel_ranges(nnode, [&](int rt, int lo_node, int hi_node) {
        for (int a = lo_node; a < hi_node; a++) {
            double cv = 0.0;
            for (int64_t q = cells.ptr[a]; q < cells.ptr[a + 1]; q++) {
                const int key = cells.key[q], tt = cells.type_of(key);
                const int *v = cells.v[tt] + (int64_t)(key - cells.off[tt]) * cells.nn[tt];
                if (tt == 0) {
                    // tetrahedron (Area_Volume.cpp:659-800): V/4 per vertex; per edge the
                    // two triangles mid-edge -> face centroid -> tet centroid
                    const double *x[4];
                    for (int k = 0; k < 4; k++) x[k] = &m.coords[3 * (size_t)v[k]];
                    double g[3];
                    for (int d = 0; d < 3; d++) g[d] = 0.25 * (x[0][d] + x[1][d] + x[2][d] + x[3][d]);
                    double e1[3], e2[3], e3[3], c[3];
                    sub3(x[1], x[0], e1); sub3(x[2], x[0], e2); sub3(x[3], x[0], e3);
                    cross3(e2, e3, c);
                    const double vol = dot3(e1, c) / 6.0;
                    if (!(vol > 0.0) && a == std::min(std::min(v[0], v[1]), std::min(v[2], v[3]))) bad_in[rt]++;
                    cv += 0.25 * std::fabs(vol);
                    for (int p = 0; p < 6; p++) {
                        const int ia_ = pairs[p][0], ib = pairs[p][1];
                        const int ea = v[ia_], eb = v[ib];
                        if (std::min(ea, eb) != a) continue;  // the edge's lower node gathers it
                        const int ic = others[p][0], id = others[p][1];
                        double mid[3], f1[3], f2[3];
                        for (int d = 0; d < 3; d++) {
                            mid[d] = 0.5 * (x[ia_][d] + x[ib][d]);
                            f1[d] = (x[ia_][d] + x[ib][d] + x[ic][d]) / 3.0;
                            f2[d] = (x[ia_][d] + x[ib][d] + x[id][d]) / 3.0;
                        }
                        double r1[3], r2[3], rg[3], s1[3], s2[3], S[3];
                        sub3(f1, mid, r1); sub3(g, mid, rg); sub3(f2, mid, r2);
                        cross3(r1, rg, s1);
                        cross3(rg, r2, s2);
                        for (int d = 0; d < 3; d++) S[d] = 0.5 * (s1[d] + s2[d]);
                        // orient from the lower to the higher node index
                        double ab[3];
                        sub3(&m.coords[3 * (size_t)std::max(ea, eb)], &m.coords[3 * (size_t)std::min(ea, eb)], ab);
                        const double sgn = dot3(S, ab) >= 0.0 ? 1.0 : -1.0;
                        const int e = edge_id(a, std::max(ea, eb));
                        for (int d = 0; d < 3; d++) m.edge_areav[3 * (size_t)e + d] += sgn * S[d];
                    }
                    continue;
                }
                // pyramid, prism, hexahedron (Area_Volume.cpp:659-822): per element edge
                // (a, b) the two triangles mid-edge -> face centroid -> element centroid
                // over the two faces sharing the edge, S = (g - m) x (f1 - m) / 2 +
                // (f2 - m) x (g - m) / 2, oriented from the lower to the higher node
                // index; each end node gets the small tetrahedra (node, m, f, g).
                const ElemType &T = *types[tt];
                double g[3] = {0, 0, 0};
                for (int k = 0; k < T.nnode; k++)
                    for (int d = 0; d < 3; d++) g[d] += m.coords[3 * (size_t)v[k] + d];
                for (int d = 0; d < 3; d++) g[d] /= T.nnode;
                for (int p = 0; p < T.nedge; p++) {
                    const int ea = v[T.edges[p][0]], eb = v[T.edges[p][1]];
                    if (ea != a && eb != a) continue;
                    const double *xa = &m.coords[3 * (size_t)ea], *xb = &m.coords[3 * (size_t)eb];
                    double mid[3], fc[2][3], rg[3], r1[3], r2[3], s1[3], s2[3], S[3];
                    for (int d = 0; d < 3; d++) mid[d] = (xa[d] + xb[d]) / 2.0;
                    for (int k = 0; k < 2; k++) {
                        const int *fn = T.face[ef[tt][p][k]];
                        const int nf = fn[3] >= 0 ? 4 : 3;
                        for (int d = 0; d < 3; d++) {
                            double acc = 0.0;
                            for (int r = 0; r < nf; r++) acc += m.coords[3 * (size_t)v[fn[r]] + d];
                            fc[k][d] = acc / (double)nf;
                        }
                    }
                    sub3(g, mid, rg); sub3(fc[0], mid, r1); sub3(fc[1], mid, r2);
                    cross3(rg, r1, s1);
                    cross3(r2, rg, s2);
                    for (int d = 0; d < 3; d++) S[d] = 0.5 * s1[d] + 0.5 * s2[d];
                    const int lo = std::min(ea, eb), hi = std::max(ea, eb);
                    if (lo == a) {
                        double ab[3];
                        sub3(&m.coords[3 * (size_t)hi], &m.coords[3 * (size_t)lo], ab);
                        const double sgn = dot3(S, ab) >= 0.0 ? 1.0 : -1.0;
                        const int e = edge_id(lo, hi);
                        for (int d = 0; d < 3; d++) m.edge_areav[3 * (size_t)e + d] += sgn * S[d];
                    }
                    if (ea == a) {
                        double da[3];
                        sub3(xa, mid, da);
                        cv += (std::fabs(dot3(da, s1)) + std::fabs(dot3(da, s2))) / 6.0;
                    } else {
                        double db[3];
                        sub3(xb, mid, db);
                        cv += (std::fabs(dot3(db, s1)) + std::fabs(dot3(db, s2))) / 6.0;
                    }
                }
            }
            m.cvol[a] = cv;
        }
    });
    int bad = 0;
    for (int b : bad_in) bad += b;
    if (bad) {
        std::fprintf(stderr, "cfd mesh: %d tetrahedra with non-positive volume\n", bad);
        return CFD_ERR_MESH;
    }

    // Boundary edges: one per boundary-triangle (then -quadrilateral) vertex, own ghost node.
    const int64_t ntri = (int64_t)m.tris.size() / 3, nquad = (int64_t)m.quads.size() / 4;
    m.nbedge = (int)(3 * ntri + 4 * nquad);
    m.nghost = m.nbedge;
    m.bedge_nodes.resize((size_t)2 * m.nbedge);
    m.bedge_areav.resize((size_t)3 * m.nbedge);
    m.bedge_type.resize(m.nbedge);
    for (int64_t t = 0; t < ntri; t++) {
        const int *v = &m.tris[3 * t];
        double e1[3], e2[3], nrm[3];
        sub3(&m.coords[3 * (size_t)v[1]], &m.coords[3 * (size_t)v[0]], e1);
        sub3(&m.coords[3 * (size_t)v[2]], &m.coords[3 * (size_t)v[0]], e2);
        cross3(e1, e2, nrm);  // right-hand normal = outward by construction
        // the reference's UGRID reader reverses triangle winding (MeshIO.cpp:22-45),
        // so its boundary edges of a triangle run over (v2, v1, v0)
        for (int k = 0; k < 3; k++) {
            int64_t be = 3 * t + k;
            m.bedge_nodes[2 * be] = v[2 - k];
            m.bedge_nodes[2 * be + 1] = nnode + (int)be;
            for (int d = 0; d < 3; d++) m.bedge_areav[3 * be + d] = nrm[d] / 6.0;  // (|n|/2)/3
            m.bedge_type[be] = m.tri_bc[t];
        }
    }
    // Quadrilaterals (Area_Volume.cpp:556-656): in the reader's reversed order
    // r = (q3, q2, q1, q0), vertex k gets -(V1 x V2 + V2 x V3) / 2 with V1, V3 to
    // the midpoints of its edges to r[k+1] and r[k-1] and V2 to the centroid.
    for (int64_t t = 0; t < nquad; t++) {
        const int r[4] = {m.quads[4 * t + 3], m.quads[4 * t + 2], m.quads[4 * t + 1], m.quads[4 * t]};
        double cen[3];
        for (int d = 0; d < 3; d++)
            cen[d] = (m.coords[3 * (size_t)r[0] + d] + m.coords[3 * (size_t)r[1] + d] +
                      m.coords[3 * (size_t)r[2] + d] + m.coords[3 * (size_t)r[3] + d]) / 4.0;
        for (int k = 0; k < 4; k++) {
            const double *xn = &m.coords[3 * (size_t)r[k]];
            const double *xp = &m.coords[3 * (size_t)r[(k + 1) & 3]];
            const double *xq = &m.coords[3 * (size_t)r[(k + 3) & 3]];
            double V1[3], V2[3], V3[3], c1[3], c2[3];
            for (int d = 0; d < 3; d++) {
                V1[d] = (xn[d] + xp[d]) / 2.0 - xn[d];
                V2[d] = cen[d] - xn[d];
                V3[d] = (xn[d] + xq[d]) / 2.0 - xn[d];
            }
            cross3(V1, V2, c1);
            cross3(V2, V3, c2);
            const int64_t be = 3 * ntri + 4 * t + k;
            m.bedge_nodes[2 * be] = r[k];
            m.bedge_nodes[2 * be + 1] = nnode + (int)be;
            // the reference negates every boundary area afterwards (outward, Area_Volume.cpp:913-915)
            for (int d = 0; d < 3; d++) m.bedge_areav[3 * be + d] = -1.0 * (0.5 * (c1[d] + c2[d]));
            m.bedge_type[be] = m.quad_bc[t];
        }
    }
    return CFD_OK;
}

// Node renumbering of a cell mesh (CFD_NUMBERING_*) before its dual is built.
static void renumber_nodes(HostMesh &m, int renumber) {
    if (!renumber) return;
    std::vector<int> ia, ja;
    build_graph(m, ia, ja);
    // perm[new] = old
    std::vector<int> perm = renumber == CFD_NUMBERING_PATCH_RCM
                                ? patch_rcm_order(m.nnode, m.coords, ia, ja, CFD_PATCH_NODES)
                                : rcm_order(m.nnode, ia, ja);
    std::vector<int> inv(m.nnode);
    for (int i = 0; i < m.nnode; i++) inv[perm[i]] = i;
    std::vector<double> c2(m.coords.size());
    for (int i = 0; i < m.nnode; i++)
        for (int d = 0; d < 3; d++) c2[3 * (size_t)i + d] = m.coords[3 * (size_t)perm[i] + d];
    m.coords.swap(c2);
    for (std::vector<int> *cells : {&m.tets, &m.pyrs, &m.prisms, &m.hexes, &m.tris, &m.quads})
        for (auto &v : *cells) v = inv[v];
}

// Freudenthal split of hex (i,j,k) into 6 positive tets sharing the diagonal
// v000 -> v111; every face gets the diagonal through its lowest corner, so
// neighbouring hexes agree on shared faces.
int build_box(HostMesh &m, int nx, int ny, int nz, double lx, double ly, double lz, double jitter,
              uint64_t seed, int renumber, const int face_bc[6]) {
    if (nx < 1 || ny < 1 || nz < 1) return CFD_ERR_ARG;
    const int px = nx + 1, py = ny + 1, pz = nz + 1;
    const int64_t nn = (int64_t)px * py * pz;
    if (nn > 0x7fffffff / 8) return CFD_ERR_ARG;
    m = HostMesh();
    m.nnode = (int)nn;
    m.coords.resize(3 * (size_t)nn);
    const double hx = lx / nx, hy = ly / ny, hz = lz / nz;
    SplitMix64 rng(seed);
    auto nid = [&](int i, int j, int k) { return i + px * (j + py * k); };
    for (int k = 0; k < pz; k++)
        for (int j = 0; j < py; j++)
            for (int i = 0; i < px; i++) {
                size_t id = (size_t)nid(i, j, k);
                double x = i * hx, y = j * hy, z = k * hz;
                double jx = rng.sym(), jy = rng.sym(), jz = rng.sym();
                bool interior = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
                if (interior) {
                    x += jitter * hx * jx;
                    y += jitter * hy * jy;
                    z += jitter * hz * jz;
                }
                m.coords[3 * id] = x;
                m.coords[3 * id + 1] = y;
                m.coords[3 * id + 2] = z;
            }
    // 6 tets per hex: paths 000 -> +a -> +a+b -> 111 over permutations (a,b,c)
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    m.tets.resize((size_t)24 * nx * ny * nz);
    size_t tp = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                for (int p = 0; p < 6; p++) {
                    int o[3] = {0, 0, 0};
                    int v[4];
                    v[0] = nid(i, j, k);
                    for (int s = 0; s < 3; s++) {
                        o[perms[p][s]] = 1;
                        v[s + 1] = nid(i + o[0], j + o[1], k + o[2]);
                    }
                    // orient positively: swap last two if the permutation is odd
                    bool odd = (p == 1 || p == 2 || p == 5);
                    if (odd) std::swap(v[2], v[3]);
                    for (int s = 0; s < 4; s++) m.tets[tp++] = v[s];
                }
    // Boundary triangles with outward right-hand normals, 2 per face quad,
    // split along the diagonal through the quad's lowest corner.
    auto add_quad = [&](int a, int b, int c, int d, int bc) {
        // quad a-b-c-d counter-clockwise seen from outside; diagonal a-c
        m.tris.push_back(a); m.tris.push_back(b); m.tris.push_back(c); m.tri_bc.push_back(bc);
        m.tris.push_back(a); m.tris.push_back(c); m.tris.push_back(d); m.tri_bc.push_back(bc);
    };
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            // x = 0 face, outward -x: (j,k) plane seen from -x
            add_quad(nid(0, j, k), nid(0, j, k + 1), nid(0, j + 1, k + 1), nid(0, j + 1, k), face_bc[0]);
            add_quad(nid(nx, j, k), nid(nx, j + 1, k), nid(nx, j + 1, k + 1), nid(nx, j, k + 1), face_bc[1]);
        }
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
            add_quad(nid(i, 0, k), nid(i + 1, 0, k), nid(i + 1, 0, k + 1), nid(i, 0, k + 1), face_bc[2]);
            add_quad(nid(i, ny, k), nid(i, ny, k + 1), nid(i + 1, ny, k + 1), nid(i + 1, ny, k), face_bc[3]);
        }
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            add_quad(nid(i, j, 0), nid(i, j + 1, 0), nid(i + 1, j + 1, 0), nid(i + 1, j, 0), face_bc[4]);
            add_quad(nid(i, j, nz), nid(i + 1, j, nz), nid(i + 1, j + 1, nz), nid(i, j + 1, nz), face_bc[5]);
        }
    renumber_nodes(m, renumber);
    return build_dual(m);
}

int build_from_cells(HostMesh &m, int nnode, const double *coords, int64_t ntet, const int *tets,
                     int64_t ntri, const int *tris, const int *tri_bc) {
    m = HostMesh();
    m.nnode = nnode;
    m.coords.assign(coords, coords + 3 * (size_t)nnode);
    m.tets.assign(tets, tets + 4 * ntet);
    m.tris.assign(tris, tris + 3 * ntri);
    m.tri_bc.assign(tri_bc, tri_bc + ntri);
    for (int v : m.tets)
        if (v < 0 || v >= nnode) return CFD_ERR_MESH;
    for (int v : m.tris)
        if (v < 0 || v >= nnode) return CFD_ERR_MESH;
    return build_dual(m);
}

// UGRID ASCII (Euler3D/src/MeshIO.cpp:50-216): counts line
// "nNode nTri nQuad nTet nPyr nPrism nHex", coordinates, 1-based triangles,
// quadrilaterals, their boundary tags, then the volume cells.  The reader
// reverses the boundary faces' winding and permutes the pyramid's nodes
// (UGrid_Translate_Winding, MeshIO.cpp:22-45): a file pyramid (p0..p4) is
// (p0, p3, p4, p1, p2) in the base-then-apex order used here.  Boundary faces
// are written with their outward right-hand normal, as this builder stores them.
namespace {
const int kPyrFromFile[5] = {0, 3, 4, 1, 2};  // internal[kPyrFromFile[k]] = file[k]
}

int write_ugrid(const HostMesh &m, const char *path, const int *tri_tag) {
    FILE *f = std::fopen(path, "w");
    if (!f) return CFD_ERR_IO;
    const int64_t ntri = (int64_t)m.tris.size() / 3, nquad = (int64_t)m.quads.size() / 4;
    const int64_t ntet = (int64_t)m.tets.size() / 4, npyr = (int64_t)m.pyrs.size() / 5;
    const int64_t npri = (int64_t)m.prisms.size() / 6, nhex = (int64_t)m.hexes.size() / 8;
    std::fprintf(f, "%d %lld %lld %lld %lld %lld %lld\n", m.nnode, (long long)ntri, (long long)nquad, (long long)ntet,
                 (long long)npyr, (long long)npri, (long long)nhex);
    for (int i = 0; i < m.nnode; i++)
        std::fprintf(f, "%.17g %.17g %.17g\n", m.coords[3 * (size_t)i], m.coords[3 * (size_t)i + 1],
                     m.coords[3 * (size_t)i + 2]);
    for (int64_t t = 0; t < ntri; t++)
        std::fprintf(f, "%d %d %d\n", m.tris[3 * t] + 1, m.tris[3 * t + 1] + 1, m.tris[3 * t + 2] + 1);
    for (int64_t t = 0; t < nquad; t++)
        std::fprintf(f, "%d %d %d %d\n", m.quads[4 * t] + 1, m.quads[4 * t + 1] + 1, m.quads[4 * t + 2] + 1,
                     m.quads[4 * t + 3] + 1);
    for (int64_t t = 0; t < ntri; t++) std::fprintf(f, "%d\n", tri_tag ? tri_tag[t] : 1);
    for (int64_t t = 0; t < nquad; t++) std::fprintf(f, "%d\n", 1);
    for (int64_t t = 0; t < ntet; t++)
        std::fprintf(f, "%d %d %d %d\n", m.tets[4 * t] + 1, m.tets[4 * t + 1] + 1, m.tets[4 * t + 2] + 1,
                     m.tets[4 * t + 3] + 1);
    for (int64_t t = 0; t < npyr; t++) {
        int fp[5];
        for (int k = 0; k < 5; k++) fp[k] = m.pyrs[5 * t + kPyrFromFile[k]] + 1;
        std::fprintf(f, "%d %d %d %d %d\n", fp[0], fp[1], fp[2], fp[3], fp[4]);
    }
    for (int64_t t = 0; t < npri; t++) {
        const int *v = &m.prisms[6 * t];
        std::fprintf(f, "%d %d %d %d %d %d\n", v[0] + 1, v[1] + 1, v[2] + 1, v[3] + 1, v[4] + 1, v[5] + 1);
    }
    for (int64_t t = 0; t < nhex; t++) {
        const int *v = &m.hexes[8 * t];
        std::fprintf(f, "%d %d %d %d %d %d %d %d\n", v[0] + 1, v[1] + 1, v[2] + 1, v[3] + 1, v[4] + 1, v[5] + 1,
                     v[6] + 1, v[7] + 1);
    }
    std::fclose(f);
    return CFD_OK;
}

int read_ugrid(HostMesh &m, const char *path, int ntag, const int *tag_bc, int renumber) {
    FILE *f = std::fopen(path, "r");
    if (!f) {
        set_error("cfd_mesh_read_ugrid: cannot read %s", path);
        return CFD_ERR_IO;
    }
    m = HostMesh();
    long long n[7];
    int st = CFD_OK;
    auto fail = [&](const char *what) {
        set_error("cfd_mesh_read_ugrid: %s: %s", path, what);
        st = CFD_ERR_MESH;
    };
    if (std::fscanf(f, "%lld %lld %lld %lld %lld %lld %lld", &n[0], &n[1], &n[2], &n[3], &n[4], &n[5], &n[6]) != 7) {
        fail("bad counts line");
    } else if (n[0] <= 0 || n[0] > 0x7fffffff / 8 || n[1] < 0 || n[2] < 0 || n[3] < 0 || n[4] < 0 || n[5] < 0 ||
               n[6] < 0 || (n[3] + n[4] + n[5] + n[6]) == 0) {
        fail("counts out of range or no volume cells");
    }
    auto ints = [&](std::vector<int> &dst, long long count, int per) {
        dst.resize((size_t)count * per);
        for (auto &v : dst) {
            int x;
            if (std::fscanf(f, "%d", &x) != 1 || x < 1 || x > n[0]) { fail("bad node index"); return; }
            v = x - 1;
        }
    };
    if (st == CFD_OK) {
        m.nnode = (int)n[0];
        m.coords.resize(3 * (size_t)n[0]);
        for (auto &x : m.coords)
            if (std::fscanf(f, "%lf", &x) != 1) { fail("bad coordinates"); break; }
    }
    if (st == CFD_OK) ints(m.tris, n[1], 3);
    if (st == CFD_OK) ints(m.quads, n[2], 4);
    std::vector<int> tags((size_t)(n[1] + n[2]));
    for (size_t k = 0; st == CFD_OK && k < tags.size(); k++) {
        if (std::fscanf(f, "%d", &tags[k]) != 1) { fail("bad boundary tag"); break; }
        if (tag_bc && (tags[k] < 1 || tags[k] > ntag)) { fail("boundary tag without a BC type"); break; }
    }
    if (st == CFD_OK) ints(m.tets, n[3], 4);
    std::vector<int> pf;
    if (st == CFD_OK) ints(pf, n[4], 5);
    if (st == CFD_OK) ints(m.prisms, n[5], 6);
    if (st == CFD_OK) ints(m.hexes, n[6], 8);
    std::fclose(f);
    if (st) return st;
    m.pyrs.resize(pf.size());
    for (size_t c = 0; c < pf.size(); c += 5)
        for (int k = 0; k < 5; k++) m.pyrs[c + kPyrFromFile[k]] = pf[c + k];
    m.tri_bc.resize((size_t)n[1]);
    m.quad_bc.resize((size_t)n[2]);
    for (long long k = 0; k < n[1]; k++) m.tri_bc[k] = tag_bc ? tag_bc[tags[k] - 1] : CFD_BC_FAR_FIELD;
    for (long long k = 0; k < n[2]; k++) m.quad_bc[k] = tag_bc ? tag_bc[tags[n[1] + k] - 1] : CFD_BC_FAR_FIELD;
    renumber_nodes(m, renumber);
    return build_dual(m);
}

}  // namespace cfd
