// MsFEM Order1 cell bases on the GPU (Grid_forMech_Poly_Order1::CreateFunctionalSpaces,
// MsFEM/MsFEM_Grid.h:4795-5759), and the C ABI of the batched cell problems.
//
// Per macro cell (an axis-aligned box with its own fine tetrahedral mesh) the
// reference solves, one cell per OpenMP thread:
//   - 24 edge problems (FEM_1D_forElasticDeformation, FEM/FEM.h:3796): on each of the
//     12 box edges, elasticity over the fine segments with the Point (1,1,1) at one
//     end and 0 at the other (MsFEM_Grid.h:5061-5200);
//   - 24 face problems (FEM_2D_forElasticDeformation, :4367): on each face, for each
//     of its 4 vertices v, elasticity over the face triangles with the two edge
//     solutions of v on the edges through v and 0 on the other two (:5205-5340);
//   - 8 volume problems (FEM_3D_forElasticDeformation, :2970): for each vertex v,
//     elasticity over the tetrahedra with the face solutions of v on the three faces
//     through v and 0 on the others (:5380-5510).
// Here the edges are solved in closed form (a segment's block is
// ((lambda+mu) d d^T + mu I)/L, so along the edge direction d the problem is a 1-D
// Laplacian with coefficient lambda + 2 mu and across it one with mu; the P1
// solution at the nodes is the normalised cumulative compliance sum L/k, exact),
// all face problems of all cells go to one persistent batched MINRES launch
// (4 right-hand sides per face), then all volume problems to another (8 per cell).
//
// Cell conventions: vertex b at (x_{b&1}, y_{(b>>1)&1}, z_{(b>>2)&1}); face f
// (0..5) = x0, x1, y0, y1, z0, z1; the vertices of a face in increasing b.  Materials of the
// face and edge problems: by default material 0 on both, as the reference's construction computes
// (its Salome face meshes carry no material ids, Library/Math.h:91-147, MsFEM_Grid.h:4848, and the
// edge segments copy the face ids, :4905); msfem_cells_set_face_material(c, 0) instead gives a
// face triangle the material of the tetrahedron it bounds and an edge segment that of its triangle
// on the lower-numbered of the edge's two faces.
#include <cub/cub.cuh>

#include <algorithm>
#include <utility>
#include <cstring>
#include <memory>
#include <new>

#include "batch.cuh"
#include "cells.cuh"
#include "devutil.cuh"
#include "element.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

constexpr int kMaxEdgeNodes = 1024;  // nodes on one box edge

__device__ __forceinline__ unsigned kFullMask() { return 0xffffffffu; }

__host__ __device__ __forceinline__ int vertex_face_mask(int v)
{
    return (1 << (0 + (v & 1))) | (1 << (2 + ((v >> 1) & 1))) | (1 << (4 + ((v >> 2) & 1)));
}

// edge e (0..11): axis = e / 4, the two other axes (o0 < o1) at sides (s, t) = ((e>>1)&1, e&1)
__host__ __device__ __forceinline__ void edge_info(int e, int& axis, int& fa, int& fb, int& vl, int& vh)
{
    axis = e / 4;
    const int s = (e >> 1) & 1, t = e & 1;
    const int o0 = axis == 0 ? 1 : 0, o1 = axis == 2 ? 1 : 2;
    fa = 2 * o0 + s;
    fb = 2 * o1 + t;
    vl = (s << o0) | (t << o1);
    vh = vl | (1 << axis);
}

// index of vertex v among the 4 vertices of face f (increasing b), or -1
__host__ __device__ __forceinline__ int face_vertex_index(int f, int v)
{
    const int a = f >> 1, side = f & 1;
    if (((v >> a) & 1) != side) return -1;
    int k = 0;
    for (int b = 0; b < v; b++)
        if (((b >> a) & 1) == side) k++;
    return k;
}

__host__ __device__ __forceinline__ int face_vertex(int f, int k)
{
    const int a = f >> 1, side = f & 1;
    for (int b = 0; b < 8; b++)
        if (((b >> a) & 1) == side && k-- == 0) return b;
    return -1;
}

inline unsigned blocks_for(int64_t n, int threads = 256)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 32));
}

// ---- topology kernels (one block per cell where the work is per cell)

// tets: cell-local -> global ids (range checked)
__global__ void k_globalize(int n_cells, const int64_t* __restrict__ node_off, const int64_t* __restrict__ tet_off,
                            int32_t* __restrict__ tets, int* bad)
{
    const int c = blockIdx.x;
    const int64_t n0 = node_off[c], nn = node_off[c + 1] - n0;
    for (int64_t e = tet_off[c] + threadIdx.x; e < tet_off[c + 1]; e += blockDim.x)
        for (int a = 0; a < 4; a++) {
            const int64_t v = tets[4 * e + a];
            if (v < 0 || v >= nn) {
                atomicExch(bad, 1);
                tets[4 * e + a] = (int32_t)n0;
            } else {
                tets[4 * e + a] = (int32_t)(n0 + v);
            }
        }
}

__global__ void k_face_mask(int n_cells, const int64_t* __restrict__ node_off, const double* __restrict__ xyz,
                            const double* __restrict__ box, int32_t* __restrict__ mask, int32_t* __restrict__ vert,
                            int* bad)
{
    const int c = blockIdx.x;
    const double* bx = box + 6 * c;
    const double size = fmax(bx[1] - bx[0], fmax(bx[3] - bx[2], bx[5] - bx[4]));
    const double tol = 1e-9 * size;
    for (int64_t i = node_off[c] + threadIdx.x; i < node_off[c + 1]; i += blockDim.x) {
        int m = 0;
        for (int f = 0; f < 6; f++)
            if (fabs(xyz[3 * i + (f >> 1)] - bx[f]) <= tol) m |= 1 << f;
        mask[i] = m;
        if (__popc(m) == 3) {
            // a corner: which vertex
            const int v = ((m >> 1) & 1) | (((m >> 3) & 1) << 1) | (((m >> 5) & 1) << 2);
            if (vertex_face_mask(v) == m) {
                if (atomicCAS(&vert[8 * c + v], -1, (int32_t)i) != -1) atomicExch(bad, 2);
            } else {
                atomicExch(bad, 3);
            }
        } else if (__popc(m) > 3) {
            atomicExch(bad, 3);
        }
    }
}

__global__ void k_face_flags(int64_t n, const int32_t* __restrict__ mask, int f, int32_t* __restrict__ flag)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = (mask[i] >> f) & 1;
}

__global__ void k_tri_flags(int64_t n_tets, const int32_t* __restrict__ tets, const int32_t* __restrict__ mask, int f,
                            int32_t* __restrict__ flag)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_tets; e += (int64_t)gridDim.x * blockDim.x) {
        int k = 0;
        for (int a = 0; a < 4; a++) k += (mask[tets[4 * e + a]] >> f) & 1;
        flag[e] = k == 3 ? 1 : 0;
    }
}

// face nodes of face f: global face-node index, its cell node and coordinates
__global__ void k_face_nodes(int n_cells, int f, const int64_t* __restrict__ node_off, const int32_t* __restrict__ mask,
                             const int32_t* __restrict__ pos, const int64_t* __restrict__ fsys_node_off,
                             const double* __restrict__ xyz, int32_t* __restrict__ fidx, int32_t* __restrict__ fcell_node,
                             double* __restrict__ fxyz, uint8_t* __restrict__ ffixed)
{
    const int c = blockIdx.x;
    const int64_t first = pos[node_off[c]];
    const int64_t base = fsys_node_off[6 * c + f];
    for (int64_t i = node_off[c] + threadIdx.x; i < node_off[c + 1]; i += blockDim.x) {
        const int m = mask[i];
        if (!((m >> f) & 1)) {
            fidx[i] = -1;
            continue;
        }
        const int64_t k = base + (pos[i] - first);
        fidx[i] = (int32_t)k;
        fcell_node[k] = (int32_t)i;
        for (int a = 0; a < 3; a++) fxyz[3 * k + a] = xyz[3 * i + a];
        ffixed[k] = (m & ~(1 << f)) ? 1 : 0;  // the face border: nodes on another face too
    }
}

// face triangles of face f (tet-local node order), in tet order
__global__ void k_face_tris(int n_cells, int f, const int64_t* __restrict__ tet_off, const int32_t* __restrict__ tets,
                            const int32_t* __restrict__ mat, const int32_t* __restrict__ mask,
                            const int32_t* __restrict__ tpos, const int32_t* __restrict__ tflag,
                            const int64_t* __restrict__ fsys_elem_off, const int32_t* __restrict__ fidx,
                            int32_t* __restrict__ tri, int32_t* __restrict__ tri_mat)
{
    const int c = blockIdx.x;
    const int64_t first = tpos[tet_off[c]];
    const int64_t base = fsys_elem_off[6 * c + f];
    for (int64_t e = tet_off[c] + threadIdx.x; e < tet_off[c + 1]; e += blockDim.x) {
        if (!tflag[e]) continue;
        const int64_t t = base + (tpos[e] - first);
        int k = 0;
        for (int a = 0; a < 4; a++) {
            const int v = tets[4 * e + a];
            if ((mask[v] >> f) & 1) tri[3 * t + k++] = fidx[v];
        }
        tri_mat[t] = mat ? mat[e] : 0;
    }
}

// per (cell, edge): the nodes on the edge sorted along it, and for each segment the
// face triangle (of the edge's lower face) that holds it.  One warp per edge.
__global__ void k_edges(int n_cells, const int64_t* __restrict__ node_off, const int32_t* __restrict__ mask,
                        const double* __restrict__ xyz, const int32_t* __restrict__ vert,
                        const int32_t* __restrict__ fidx_all /* [6][n_nodes] */, int64_t n_nodes,
                        const int64_t* __restrict__ fsys_elem_off, const int32_t* __restrict__ tri, int cap,
                        int32_t* __restrict__ edge_nodes, int32_t* __restrict__ edge_len, int32_t* __restrict__ seg_tri,
                        int* bad)
{
    __shared__ int32_t s_nodes[12][kMaxEdgeNodes];
    const int c = blockIdx.x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w >= 12) return;
    int axis, fa, fb, vl, vh;
    edge_info(w, axis, fa, fb, vl, vh);
    const int want = (1 << fa) | (1 << fb);
    int cnt = 0;
    for (int64_t base = node_off[c]; base < node_off[c + 1]; base += 32) {
        const int64_t i = base + lane;
        const bool on = i < node_off[c + 1] && (mask[i] & want) == want;
        const unsigned bal = __ballot_sync(kFullMask(), on);
        if (on) {
            const int k = cnt + __popc(bal & ((1u << lane) - 1));
            if (k < kMaxEdgeNodes) s_nodes[w][k] = (int32_t)i;
        }
        cnt += __popc(bal);
    }
    __syncwarp();
    const int64_t eid = 12 * (int64_t)c + w;
    if (cnt > kMaxEdgeNodes || cnt > cap || cnt < 2) {
        if (lane == 0) {
            atomicExch(bad, 4);
            edge_len[eid] = 0;
        }
        return;
    }
    // rank sort by the coordinate along the edge (ties by list position)
    for (int i = lane; i < cnt; i += 32) {
        const double xi = xyz[3 * (int64_t)s_nodes[w][i] + axis];
        int rank = 0;
        for (int j = 0; j < cnt; j++) {
            const double xj = xyz[3 * (int64_t)s_nodes[w][j] + axis];
            rank += (xj < xi || (xj == xi && j < i)) ? 1 : 0;
        }
        edge_nodes[eid * cap + rank] = s_nodes[w][i];
    }
    __syncwarp();
    if (lane == 0) {
        edge_len[eid] = cnt;
        if (edge_nodes[eid * cap] != vert[8 * c + vl] || edge_nodes[eid * cap + cnt - 1] != vert[8 * c + vh])
            atomicExch(bad, 5);
    }
    __syncwarp();
    // segment k = (node k, node k+1): the first triangle of face fa holding both
    const int64_t t0 = fsys_elem_off[6 * c + fa], t1 = fsys_elem_off[6 * c + fa + 1];
    const int32_t* fidx = fidx_all + (int64_t)fa * n_nodes;
    for (int k = 0; k + 1 < cnt; k++) {
        const int32_t a = fidx[edge_nodes[eid * cap + k]], b = fidx[edge_nodes[eid * cap + k + 1]];
        int best = 0x7fffffff;
        for (int64_t t = t0 + lane; t < t1; t += 32) {
            const int32_t* q = tri + 3 * t;
            const bool ha = q[0] == a || q[1] == a || q[2] == a;
            const bool hb = q[0] == b || q[1] == b || q[2] == b;
            if (ha && hb) best = min(best, (int)(t - t0));
        }
        best = __reduce_min_sync(kFullMask(), best);
        if (lane == 0) {
            if (best == 0x7fffffff) atomicExch(bad, 6);
            seg_tri[eid * cap + k] = best == 0x7fffffff ? -1 : (int32_t)(t0 + best);
        }
    }
}

// ---- per-build kernels

// exact edge solutions at the edge nodes: prof[node][0] (value 1 at the low end), prof[node][1] (1 at the high end)
__global__ void k_edge_profiles(int n_edges, int cap, const int32_t* __restrict__ edge_nodes,
                                const int32_t* __restrict__ edge_len, const int32_t* __restrict__ seg_tri,
                                const int32_t* __restrict__ tri_mat, const double* __restrict__ lame, int n_mat,
                                const double* __restrict__ xyz, double* __restrict__ prof, int* bad)
{
    for (int eid = blockIdx.x * blockDim.x + threadIdx.x; eid < n_edges; eid += gridDim.x * blockDim.x) {
        const int n = edge_len[eid];
        if (n < 2) continue;
        const int32_t* nodes = edge_nodes + (int64_t)eid * cap;
        const int64_t a0 = nodes[0], a1 = nodes[n - 1];
        double d[3], len = 0.0;
        for (int k = 0; k < 3; k++) {
            d[k] = xyz[3 * a1 + k] - xyz[3 * a0 + k];
            len += d[k] * d[k];
        }
        len = sqrt(len);
        for (int k = 0; k < 3; k++) d[k] /= len;
        const double dd = d[0] + d[1] + d[2];  // d . (1,1,1)
        // totals of the compliance L/k along (lambda + 2 mu) and across (mu)
        double tot_al = 0.0, tot_pe = 0.0;
        for (int k = 0; k + 1 < n; k++) {
            const int t = seg_tri[(int64_t)eid * cap + k];
            const int m = t >= 0 ? tri_mat[t] : -1;
            double L = 0.0;
            for (int q = 0; q < 3; q++) {
                const double u = xyz[3 * (int64_t)nodes[k + 1] + q] - xyz[3 * (int64_t)nodes[k] + q];
                L += u * u;
            }
            L = sqrt(L);
            if (m < 0 || m >= n_mat || !(lame[2 * m + 1] > 0.0)) {
                atomicExch(bad, 7);
                continue;
            }
            tot_al += L / (lame[2 * m] + 2.0 * lame[2 * m + 1]);
            tot_pe += L / lame[2 * m + 1];
        }
        double c_al = 0.0, c_pe = 0.0;
        for (int k = 0; k < n; k++) {
            if (k > 0) {
                const int t = seg_tri[(int64_t)eid * cap + k - 1];
                const int m = t >= 0 ? tri_mat[t] : 0;
                double L = 0.0;
                for (int q = 0; q < 3; q++) {
                    const double u = xyz[3 * (int64_t)nodes[k] + q] - xyz[3 * (int64_t)nodes[k - 1] + q];
                    L += u * u;
                }
                L = sqrt(L);
                if (m >= 0 && m < n_mat && lame[2 * m + 1] > 0.0) {
                    c_al += L / (lame[2 * m] + 2.0 * lame[2 * m + 1]);
                    c_pe += L / lame[2 * m + 1];
                }
            }
            // value at the low end: 1 - C(k)/C_tot; at the high end: C(k)/C_tot (exact ends)
            const double hi_al = k == n - 1 ? 1.0 : c_al / tot_al, hi_pe = k == n - 1 ? 1.0 : c_pe / tot_pe;
            const double lo_al = k == 0 ? 1.0 : (k == n - 1 ? 0.0 : 1.0 - hi_al);
            const double lo_pe = k == 0 ? 1.0 : (k == n - 1 ? 0.0 : 1.0 - hi_pe);
            const double hal = k == 0 ? 0.0 : hi_al, hpe = k == 0 ? 0.0 : hi_pe;
            if (k == 0 || k == n - 1) continue;  // corners: the face problems use the vertex identity
            double* o = prof + 6 * (int64_t)nodes[k];
            for (int q = 0; q < 3; q++) {
                // Point (1,1,1) split into its part along d and across d
                const double along = dd * d[q], across = 1.0 - along;
                o[q] = lo_al * along + lo_pe * across;
                o[3 + q] = hal * along + hpe * across;
            }
        }
    }
}

// Dirichlet data of the face problems: fx[face node][j][3] for the 4 vertices j of the face
__global__ void k_face_dirichlet(int64_t n_fnodes, const int32_t* __restrict__ fcell_node, const uint8_t* __restrict__ ffixed,
                                 const int64_t* __restrict__ fsys_node_off, int n_fsys, const int32_t* __restrict__ mask,
                                 const int32_t* __restrict__ vert, const int64_t* __restrict__ node_off, int n_cells,
                                 const double* __restrict__ prof, double* __restrict__ fx)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_fnodes; k += (int64_t)gridDim.x * blockDim.x) {
        double* o = fx + 12 * k;
        for (int q = 0; q < 12; q++) o[q] = 0.0;
        if (!ffixed[k]) continue;
        // the face system of this node (binary search in fsys_node_off)
        int lo = 0, hi = n_fsys - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (fsys_node_off[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        const int c = lo / 6, f = lo % 6;
        const int64_t i = fcell_node[k];
        const int m = mask[i];
        for (int j = 0; j < 4; j++) {
            const int v = face_vertex(f, j);
            if (__popc(m) == 3) {
                const double val = (i == vert[8 * c + v]) ? 1.0 : 0.0;
                for (int q = 0; q < 3; q++) o[3 * j + q] = val;
                continue;
            }
            // the edge through this node: faces f and g (the other bit)
            const int g = __ffs(m & ~(1 << f)) - 1;
            for (int e = 0; e < 12; e++) {
                int axis, fa, fb, vl, vh;
                edge_info(e, axis, fa, fb, vl, vh);
                if (!((fa == f && fb == g) || (fa == g && fb == f))) continue;
                if (v == vl || v == vh) {
                    const double* p = prof + 6 * i + (v == vl ? 0 : 3);
                    for (int q = 0; q < 3; q++) o[3 * j + q] = p[q];
                }
            }
        }
    }
}

// Dirichlet data of the volume problems: x[node][v][3] from the face solutions
__global__ void k_volume_dirichlet(int64_t n_nodes, const int32_t* __restrict__ mask, const int32_t* __restrict__ fidx_all,
                                   const double* __restrict__ fx, double* __restrict__ x)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const int m = mask[i];
        double* o = x + 24 * i;
        for (int v = 0; v < 8; v++) {
            const int common = m & vertex_face_mask(v);
            double val[3] = {0.0, 0.0, 0.0};
            if (common) {
                const int f = __ffs(common) - 1;  // the lowest face through both
                const int64_t k = fidx_all[(int64_t)f * n_nodes + i];
                const int j = face_vertex_index(f, v);
                for (int q = 0; q < 3; q++) val[q] = fx[12 * k + 3 * j + q];
            }
            for (int q = 0; q < 3; q++) o[3 * v + q] = val[q];
        }
    }
}


// ---- MsFEM macro element matrices (FiniteElement_forMech_Poly_Order1::SolveLocalMatrix,
// MsFEM_Grid.h:3837-3975): the polyhedron quadrature (sub-tetrahedra centroid / face centroid /
// face edge, 4-point rule each, GeometryShape.h:2708-2760, :1754-1851), the basis gradients of
// the micro tetrahedron holding each point (the reference's nearest-element lookup,
// GeometryGrid.h:323-340; the lowest index among ties), and D of material 0 for every cell
// (MsFEM.h:644-647).  K[c][I][J][r][s] = sum_q w_q (B_J^T D B_I)[r][s].

constexpr int kMacroQ = 96;
__constant__ int c_face_cycles[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 1, 3, 2}, {4, 5, 7, 6}};

__device__ __forceinline__ void box_vertex(const double* bx, int v, double p[3])
{
    p[0] = bx[0 + (v & 1)];
    p[1] = bx[2 + ((v >> 1) & 1)];
    p[2] = bx[4 + ((v >> 2) & 1)];
}

// column a of the strain matrix of the component-wise basis e_a psi^a (Voigt xx yy zz xy yz zx,
// engineering shear; the rows of MsFEM_Grid.h:3868-3885), from G[comp][deriv]
__device__ __forceinline__ void strain_column(const double* G, int a, double b[6])
{
    for (int k = 0; k < 6; k++) b[k] = 0.0;
    b[a] = G[3 * a + a];
    if (a == 0) {
        b[3] = G[1];
        b[5] = G[2];
    } else if (a == 1) {
        b[3] = G[3];
        b[4] = G[5];
    } else {
        b[4] = G[7];
        b[5] = G[6];
    }
}

// NB bases per cell ([node][NB][3]); ZREP: every component of basis I is its z component (the
// Order2 macro bases, MsFEM_Grid.h:2978-2979)
template <int NB, bool ZREP>
__global__ void __launch_bounds__(256) k_macro_cells(const int64_t* __restrict__ tet_off, const int32_t* __restrict__ tets,
                                                     const double* __restrict__ xyz, const double* __restrict__ box,
                                                     const double* __restrict__ bases, const double* __restrict__ lame,
                                                     double* __restrict__ K, int* bad)
{
    extern __shared__ double sm[];
    double* sG = sm;                                 // [96][NB][9]
    double* sP = sG + kMacroQ * NB * 9;              // [96][3]
    double* sW = sP + kMacroQ * 3;                   // [96]
    int* sT = reinterpret_cast<int*>(sW + kMacroQ);  // [96]
    const int c = blockIdx.x, tid = threadIdx.x;
    const double* bx = box + 6 * c;
    if (tid < kMacroQ) {
        const int f = tid / 16, i = (tid / 4) % 4, j = tid % 4;
        double C[3] = {0, 0, 0}, F[3] = {0, 0, 0}, a[3], b[3];
        for (int v = 0; v < 8; v++) {
            double p[3];
            box_vertex(bx, v, p);
            for (int d = 0; d < 3; d++) C[d] += 0.125 * p[d];
        }
        for (int k = 0; k < 4; k++) {
            double p[3];
            box_vertex(bx, c_face_cycles[f][k], p);
            for (int d = 0; d < 3; d++) F[d] += 0.25 * p[d];
        }
        box_vertex(bx, c_face_cycles[f][i], a);
        box_vertex(bx, c_face_cycles[f][(i + 1) % 4], b);
        double E1[3], E2[3], E3[3];
        for (int d = 0; d < 3; d++) {
            E1[d] = F[d] - C[d];
            E2[d] = a[d] - C[d];
            E3[d] = b[d] - C[d];
        }
        const double det = E1[0] * (E2[1] * E3[2] - E2[2] * E3[1]) - E1[1] * (E2[0] * E3[2] - E2[2] * E3[0]) +
                           E1[2] * (E2[0] * E3[1] - E2[1] * E3[0]);
        const double u = (5.0 - sqrt(5.0)) / 20.0, vv = 1.0 - 3.0 * u;
        const double bar[3] = {j == 1 ? vv : u, j == 2 ? vv : u, j == 3 ? vv : u};
        for (int d = 0; d < 3; d++) sP[3 * tid + d] = C[d] + bar[0] * E1[d] + bar[1] * E2[d] + bar[2] * E3[d];
        sW[tid] = fabs(det) / 24.0;
        sT[tid] = 0x7fffffff;
    }
    __syncthreads();
    const int64_t t0 = tet_off[c], t1 = tet_off[c + 1];
    for (int64_t e = t0 + tid; e < t1; e += blockDim.x) {
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        const double* p0 = xyz + 3 * (int64_t)v[0];
        for (int q = 0; q < kMacroQ; q++) {
            const double dx[3] = {sP[3 * q] - p0[0], sP[3 * q + 1] - p0[1], sP[3 * q + 2] - p0[2]};
            bool in = true;
            for (int k = 0; k < 4; k++) {
                const double lam = (k == 0 ? 1.0 : 0.0) + G.g[k][0] * dx[0] + G.g[k][1] * dx[1] + G.g[k][2] * dx[2];
                in = in && lam >= -1e-12;
            }
            if (in) atomicMin(&sT[q], (int)(e - t0));
        }
    }
    __syncthreads();
    for (int t = tid; t < kMacroQ * NB; t += blockDim.x) {
        const int q = t / NB, I = t % NB;
        double* out = sG + 9 * NB * q + 9 * I;
        if (sT[q] == 0x7fffffff) {
            atomicExch(bad, 1);
            for (int k = 0; k < 9; k++) out[k] = 0.0;
            continue;
        }
        const int64_t e = t0 + sT[q];
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        for (int cc = 0; cc < 3; cc++)
            for (int d = 0; d < 3; d++) {
                double g = 0.0;
                for (int k = 0; k < 4; k++) g += bases[3 * NB * (int64_t)v[k] + 3 * I + (ZREP ? 2 : cc)] * G.g[k][d];
                out[3 * cc + d] = g;
            }
    }
    __syncthreads();
    // D: lambda on the trace plus 2 mu on the normal strains, mu on the engineering shears
    const double lam = lame[0], mu = lame[1];
    for (int t = tid; t < NB * NB * 9; t += blockDim.x) {
        const int I = t / (9 * NB), J = (t / 9) % NB, r = (t / 3) % 3, cs = t % 3;
        double acc = 0.0;
        for (int q = 0; q < kMacroQ; q++) {
            double bi[6], bj[6];
            strain_column(sG + 9 * NB * q + 9 * I, cs, bi);
            strain_column(sG + 9 * NB * q + 9 * J, r, bj);
            const double tr = bi[0] + bi[1] + bi[2];
            double v = 0.0;
            for (int k = 0; k < 3; k++) v += bj[k] * (lam * tr + 2.0 * mu * bi[k]);
            for (int k = 3; k < 6; k++) v += bj[k] * mu * bi[k];
            acc += sW[q] * v;
        }
        K[NB * NB * 9 * (int64_t)c + t] = acc;
    }
}


// ---- MsFEM macro boundary loads (BoundaryFace_forMech_Poly_Order1::SolveLocalBoundaryVector,
// MsFEM_Grid.h:4104-4135): f[I][a] = sum_q w_q t_a psi_I^a(x_q) over the macro face, with the
// polygon rule of GeometryShape.h:2563-2600 (sub-triangles centroid / face edge) and the triangle
// 4-point rule of :1482-1540; psi from the micro tetrahedron holding each point.
__global__ void __launch_bounds__(128) k_face_loads(int n_items, const int32_t* __restrict__ items,
                                                    const double* __restrict__ traction,
                                                    const int64_t* __restrict__ tet_off, const int32_t* __restrict__ tets,
                                                    const double* __restrict__ xyz, const double* __restrict__ box,
                                                    const double* __restrict__ bases, double* __restrict__ out, int* bad)
{
    __shared__ double sP[16][3], sW[16];
    __shared__ int sT[16];
    const int it = blockIdx.x, tid = threadIdx.x;
    const int c = items[2 * it], f = items[2 * it + 1];
    const double* bx = box + 6 * c;
    if (tid < 16) {
        const int i = tid / 4, j = tid % 4;
        double F[3] = {0, 0, 0}, a[3], b[3];
        for (int k = 0; k < 4; k++) {
            double p[3];
            box_vertex(bx, c_face_cycles[f][k], p);
            for (int d = 0; d < 3; d++) F[d] += 0.25 * p[d];
        }
        box_vertex(bx, c_face_cycles[f][i], a);
        box_vertex(bx, c_face_cycles[f][(i + 1) % 4], b);
        double e1[3], e2[3];
        for (int d = 0; d < 3; d++) {
            e1[d] = a[d] - F[d];
            e2[d] = b[d] - F[d];
        }
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double detD = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        const double xs[4] = {1.0 / 3.0, 3.0 / 5.0, 1.0 / 5.0, 1.0 / 5.0};
        const double ys[4] = {1.0 / 3.0, 1.0 / 5.0, 3.0 / 5.0, 1.0 / 5.0};
        const double ws[4] = {-9.0 / 32.0, 25.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0};
        for (int d = 0; d < 3; d++) sP[tid][d] = F[d] + e1[d] * xs[j] + e2[d] * ys[j];
        sW[tid] = ws[j] * detD;
        sT[tid] = 0x7fffffff;
    }
    __syncthreads();
    const int64_t t0 = tet_off[c], t1 = tet_off[c + 1];
    for (int64_t e = t0 + tid; e < t1; e += blockDim.x) {
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        const double* p0 = xyz + 3 * (int64_t)v[0];
        for (int q = 0; q < 16; q++) {
            const double dx[3] = {sP[q][0] - p0[0], sP[q][1] - p0[1], sP[q][2] - p0[2]};
            bool in = true;
            for (int k = 0; k < 4; k++) {
                const double lam = (k == 0 ? 1.0 : 0.0) + G.g[k][0] * dx[0] + G.g[k][1] * dx[1] + G.g[k][2] * dx[2];
                in = in && lam >= -1e-12;
            }
            if (in) atomicMin(&sT[q], (int)(e - t0));
        }
    }
    __syncthreads();
    if (tid < 24) {
        const int I = tid / 3, a = tid % 3;
        double acc = 0.0;
        for (int q = 0; q < 16; q++) {
            if (sT[q] == 0x7fffffff) {
                atomicExch(bad, 1);
                continue;
            }
            const int64_t e = t0 + sT[q];
            int v[4];
            for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
            TetGeom G;
            tet_geometry(xyz, v, G);
            const double* p0 = xyz + 3 * (int64_t)v[0];
            const double dx[3] = {sP[q][0] - p0[0], sP[q][1] - p0[1], sP[q][2] - p0[2]};
            double psi = 0.0;
            for (int k = 0; k < 4; k++) {
                const double lam = (k == 0 ? 1.0 : 0.0) + G.g[k][0] * dx[0] + G.g[k][1] * dx[1] + G.g[k][2] * dx[2];
                psi += lam * bases[24 * (int64_t)v[k] + 3 * I + a];
            }
            acc += sW[q] * traction[3 * it + a] * psi;
        }
        out[24 * (int64_t)it + tid] = acc;
    }
}

// residual of the current bases in each cell's volume problem: over the free nodes i,
// r_i = sum_j A_ij x_j for the 8 bases (no source term); rel = ||r|| / ||sum_{j fixed} A_ij x_j||
__global__ void __launch_bounds__(256) k_basis_residual(const int64_t* __restrict__ node_off, const int64_t* __restrict__ row_ptr,
                                                        const int32_t* __restrict__ col, const double* __restrict__ val,
                                                        const uint8_t* __restrict__ fixed, const double* __restrict__ x,
                                                        double* __restrict__ rel)
{
    const int c = blockIdx.x;
    double num = 0.0, den = 0.0;
    for (int64_t i = node_off[c] + threadIdx.x; i < node_off[c + 1]; i += blockDim.x) {
        if (fixed[i]) continue;
        double yf[24], yb[24];
        for (int q = 0; q < 24; q++) yf[q] = yb[q] = 0.0;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
            const int64_t j = col[k];
            const double* A = val + 9 * k;
            const double* xj = x + 24 * j;
            double* y = fixed[j] ? yb : yf;
            for (int r = 0; r < 8; r++)
                for (int a = 0; a < 3; a++)
                    y[3 * r + a] += A[3 * a] * xj[3 * r] + A[3 * a + 1] * xj[3 * r + 1] + A[3 * a + 2] * xj[3 * r + 2];
        }
        for (int q = 0; q < 24; q++) {
            num += (yf[q] + yb[q]) * (yf[q] + yb[q]);
            den += yb[q] * yb[q];
        }
    }
    __shared__ double s0[256], s1[256];
    s0[threadIdx.x] = num;
    s1[threadIdx.x] = den;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s0[threadIdx.x] += s0[threadIdx.x + w];
            s1[threadIdx.x] += s1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) rel[c] = s1[0] > 0.0 ? sqrt(s0[0] / s1[0]) : (s0[0] > 0.0 ? INFINITY : 0.0);
}

// fine solution of every cell from the macro one: u[b] = sum_v U[V(c, v)] (.) psi_v(b)
// F[cell_vertex[8 c_i + v]] += loads[i][v] over the items in order (SummPartOfVector item by item,
// the reference's order): one thread per component walks the items, so each vertex sums in order
__global__ void k_macro_load_sum(int n_items, const int32_t* __restrict__ items, const int32_t* __restrict__ cell_vertex,
                                 const double* __restrict__ loads, double* __restrict__ F)
{
    const int a = threadIdx.x;
    if (a >= 3) return;
    for (int i = 0; i < n_items; i++) {
        const int c = items[2 * i];
        for (int v = 0; v < 8; v++) F[3 * (int64_t)cell_vertex[8 * c + v] + a] += loads[24 * (int64_t)i + 3 * v + a];
    }
}

__global__ void k_reconstruct(int n_cells, const int64_t* __restrict__ node_off, const int32_t* __restrict__ cell_vertex,
                              const double* __restrict__ U, const double* __restrict__ bases, double* __restrict__ u)
{
    const int c = blockIdx.x;
    for (int64_t b = node_off[c] + threadIdx.x; b < node_off[c + 1]; b += blockDim.x) {
        double acc[3] = {0, 0, 0};
        for (int v = 0; v < 8; v++) {
            const int64_t V = cell_vertex[8 * c + v];
            for (int a = 0; a < 3; a++) acc[a] += U[3 * V + a] * bases[24 * b + 3 * v + a];
        }
        for (int a = 0; a < 3; a++) u[3 * b + a] = acc[a];
    }
}

}  // namespace

// ------------------------------------------------------------------ handles

namespace {

template <class T>
int copy_in(cudaStream_t st, DBuf<T>& dst, const T* src, size_t n)
{
    MSFEM_TRY(dst.alloc(std::max<size_t>(1, n)));
    if (n) MSFEM_CK(cudaMemcpyAsync(dst.p, src, n * sizeof(T), cudaMemcpyDefault, st));
    return 0;
}

int read_flag(cudaStream_t st, DBuf<int>& flag, int* out)
{
    MSFEM_CK(cudaMemcpyAsync(out, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

int lame_to_device(cudaStream_t st, DBuf<double>& d, const double* E, const double* nu, int n_mat)
{
    std::vector<double> h(2 * (size_t)n_mat);
    std::vector<double> hE(n_mat), hn(n_mat);
    // E and nu may be device pointers: stage through the host
    MSFEM_CK(cudaMemcpyAsync(hE.data(), E, sizeof(double) * n_mat, cudaMemcpyDefault, st));
    MSFEM_CK(cudaMemcpyAsync(hn.data(), nu, sizeof(double) * n_mat, cudaMemcpyDefault, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    lame_params(hE.data(), hn.data(), n_mat, h.data());
    MSFEM_TRY(d.alloc(2 * (size_t)n_mat));
    MSFEM_CK(cudaMemcpyAsync(d.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

int batch_finish(BatchSys& b, int* n_bad, double tol, double* worst)
{
    std::vector<double> rel(b.n_sys);
    if (b.n_sys) MSFEM_CK(cudaMemcpyAsync(rel.data(), b.rel.p, sizeof(double) * b.n_sys, cudaMemcpyDeviceToHost, b.stream));
    MSFEM_CK(cudaStreamSynchronize(b.stream));
    int bad = 0;
    double w = 0.0;
    for (double r : rel) {
        if (!(r <= tol)) bad++;
        if (!(r <= w)) w = r;
    }
    *n_bad = bad;
    if (worst) *worst = w;
    return 0;
}

int cells_create(int n_cells, const int64_t* node_off, const double* xyz, const int64_t* tet_off, const int32_t* tets,
                 const int32_t* material, const double* box, int n_mat, const double* E, const double* nu,
                 CellsHandle& h)
{
    cudaStream_t st = h.stream;
    h.n_cells = n_cells;
    h.n_mat = n_mat;
    h.h_node_off.resize(n_cells + 1);
    h.h_tet_off.resize(n_cells + 1);
    MSFEM_CK(cudaMemcpyAsync(h.h_node_off.data(), node_off, sizeof(int64_t) * (n_cells + 1), cudaMemcpyDefault, st));
    MSFEM_CK(cudaMemcpyAsync(h.h_tet_off.data(), tet_off, sizeof(int64_t) * (n_cells + 1), cudaMemcpyDefault, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (h.h_node_off[0] != 0 || h.h_tet_off[0] != 0) {
        set_error("msfem_cells_create: offsets must start at 0");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int c = 0; c < n_cells; c++)
        if (h.h_node_off[c + 1] < h.h_node_off[c] + 8 || h.h_tet_off[c + 1] <= h.h_tet_off[c]) {
            set_error("msfem_cells_create: cell %d has fewer than 8 nodes or no tetrahedra", c);
            return MSFEM_ERR_ARGUMENT;
        }
    h.n_nodes = h.h_node_off[n_cells];
    h.n_tets = h.h_tet_off[n_cells];
    if (h.n_nodes >= ((int64_t)1 << 31) || h.n_tets >= ((int64_t)1 << 28)) {
        set_error("msfem_cells_create: %lld nodes / %lld tets exceed the int32 / 2^28 limits", (long long)h.n_nodes,
                  (long long)h.n_tets);
        return MSFEM_ERR_LIMIT;
    }
    MSFEM_TRY(copy_in(st, h.node_off, node_off, n_cells + 1));
    MSFEM_TRY(copy_in(st, h.tet_off, tet_off, n_cells + 1));
    MSFEM_TRY(copy_in(st, h.xyz, xyz, 3 * (size_t)h.n_nodes));
    MSFEM_TRY(copy_in(st, h.box, box, 6 * (size_t)n_cells));
    MSFEM_TRY(copy_in(st, h.vols.elems, tets, 4 * (size_t)h.n_tets));
    if (material) {
        MSFEM_TRY(copy_in(st, h.mat, material, (size_t)h.n_tets));
    } else {
        MSFEM_TRY(h.mat.alloc(h.n_tets));
        MSFEM_CK(cudaMemsetAsync(h.mat.p, 0, sizeof(int32_t) * h.n_tets, st));
    }
    MSFEM_TRY(lame_to_device(st, h.lame, E, nu, n_mat));
    MSFEM_TRY(h.flag.alloc(1));
    MSFEM_CK(cudaMemsetAsync(h.flag.p, 0, sizeof(int), st));
    k_globalize<<<n_cells, 256, 0, st>>>(n_cells, h.node_off.p, h.tet_off.p, h.vols.elems.p, h.flag.p);
    MSFEM_TRY(h.mask.alloc(h.n_nodes));
    MSFEM_TRY(h.vert.alloc(8 * (size_t)n_cells));
    MSFEM_CK(cudaMemsetAsync(h.vert.p, 0xff, sizeof(int32_t) * 8 * n_cells, st));
    k_face_mask<<<n_cells, 256, 0, st>>>(n_cells, h.node_off.p, h.xyz.p, h.box.p, h.mask.p, h.vert.p, h.flag.p);
    MSFEM_CK(cudaGetLastError());
    int bad = 0;
    MSFEM_TRY(read_flag(st, h.flag, &bad));
    if (bad) {
        set_error(bad == 1 ? "msfem_cells_create: a tetrahedron node id is outside its cell"
                           : "msfem_cells_create: a cell's corner nodes are missing, repeated or off the box");
        return MSFEM_ERR_ARGUMENT;
    }
    {
        std::vector<int32_t> vh(8 * (size_t)n_cells);
        MSFEM_CK(cudaMemcpyAsync(vh.data(), h.vert.p, sizeof(int32_t) * vh.size(), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        for (size_t q = 0; q < vh.size(); q++)
            if (vh[q] < 0) {
                set_error("msfem_cells_create: cell %zu has no node on its corner %zu", q / 8, q % 8);
                return MSFEM_ERR_ARGUMENT;
            }
    }

    // face nodes and triangles: per face f a scan over all nodes / tets (cell order)
    DBuf<int32_t> flag_n, pos_n, flag_t, pos_t[6], tflag[6];
    DBuf<unsigned char> tmp;
    MSFEM_TRY(flag_n.alloc(h.n_nodes + 1));
    MSFEM_TRY(pos_n.alloc(6 * (h.n_nodes + 1)));
    std::vector<int64_t> fcount(6 * (size_t)n_cells), tcount(6 * (size_t)n_cells);
    std::vector<int32_t> hp(n_cells + 1);
    auto scan = [&](const int32_t* in, int32_t* out, int64_t n) -> int {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, st);
        MSFEM_TRY(tmp.alloc(std::max<size_t>(tb, 1)));
        MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp.p, tb, in, out, (int)n, st));
        return 0;
    };
    // cell boundaries of a scan, to the host
    auto gather_bounds = [&](const int32_t* pos, const std::vector<int64_t>& off, std::vector<int32_t>& out) -> int {
        for (int c = 0; c <= n_cells; c++)
            MSFEM_CK(cudaMemcpyAsync(&out[c], pos + off[c], sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        return 0;
    };
    for (int f = 0; f < 6; f++) {
        k_face_flags<<<blocks_for(h.n_nodes), 256, 0, st>>>(h.n_nodes, h.mask.p, f, flag_n.p);
        MSFEM_CK(cudaMemsetAsync(flag_n.p + h.n_nodes, 0, sizeof(int32_t), st));
        MSFEM_TRY(scan(flag_n.p, pos_n.p + f * (h.n_nodes + 1), h.n_nodes + 1));
        MSFEM_TRY(gather_bounds(pos_n.p + f * (h.n_nodes + 1), h.h_node_off, hp));
        for (int c = 0; c < n_cells; c++) fcount[6 * c + f] = hp[c + 1] - hp[c];
        MSFEM_TRY(tflag[f].alloc(h.n_tets + 1));
        MSFEM_TRY(pos_t[f].alloc(h.n_tets + 1));
        k_tri_flags<<<blocks_for(h.n_tets), 256, 0, st>>>(h.n_tets, h.vols.elems.p, h.mask.p, f, tflag[f].p);
        MSFEM_CK(cudaMemsetAsync(tflag[f].p + h.n_tets, 0, sizeof(int32_t), st));
        MSFEM_TRY(scan(tflag[f].p, pos_t[f].p, h.n_tets + 1));
        MSFEM_TRY(gather_bounds(pos_t[f].p, h.h_tet_off, hp));
        for (int c = 0; c < n_cells; c++) tcount[6 * c + f] = hp[c + 1] - hp[c];
    }
    BatchSys& F = h.faces;
    F.dim = 2;
    F.k1 = 3;
    F.R = 4;
    F.n_sys = 6 * n_cells;
    F.stream = st;
    F.h_node_off.assign(F.n_sys + 1, 0);
    F.h_elem_off.assign(F.n_sys + 1, 0);
    for (int s = 0; s < F.n_sys; s++) {
        if (fcount[s] < 3 || tcount[s] < 1) {
            set_error("msfem_cells_create: face %d of cell %d has %lld nodes and %lld triangles", s % 6, s / 6,
                      (long long)fcount[s], (long long)tcount[s]);
            return MSFEM_ERR_ARGUMENT;
        }
        F.h_node_off[s + 1] = F.h_node_off[s] + fcount[s];
        F.h_elem_off[s + 1] = F.h_elem_off[s] + tcount[s];
    }
    F.n_nodes = F.h_node_off[F.n_sys];
    F.n_elems = F.h_elem_off[F.n_sys];
    MSFEM_TRY(copy_in(st, F.node_off, F.h_node_off.data(), F.n_sys + 1));
    MSFEM_TRY(copy_in(st, F.elem_off, F.h_elem_off.data(), F.n_sys + 1));
    MSFEM_TRY(h.fidx.alloc(6 * h.n_nodes));
    MSFEM_TRY(h.fcell_node.alloc(F.n_nodes));
    MSFEM_TRY(h.fxyz.alloc(3 * F.n_nodes));
    MSFEM_TRY(F.fixed.alloc(F.n_nodes));
    MSFEM_TRY(F.elems.alloc(3 * F.n_elems));
    MSFEM_TRY(F.emat.alloc(F.n_elems));
    for (int f = 0; f < 6; f++)
        k_face_nodes<<<n_cells, 256, 0, st>>>(n_cells, f, h.node_off.p, h.mask.p, pos_n.p + f * (h.n_nodes + 1),
                                               F.node_off.p, h.xyz.p, h.fidx.p + f * h.n_nodes, h.fcell_node.p, h.fxyz.p,
                                               F.fixed.p);
    for (int f = 0; f < 6; f++)
        k_face_tris<<<n_cells, 256, 0, st>>>(n_cells, f, h.tet_off.p, h.vols.elems.p, h.mat.p, h.mask.p, pos_t[f].p,
                                              tflag[f].p, F.elem_off.p, h.fidx.p + f * h.n_nodes, F.elems.p, F.emat.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_TRY(batch_build_pattern(F, h.fxyz.p));

    // edges
    {
        // capacity: the longest edge (count with the same rule the kernel uses)
        int cap = 2;
        std::vector<int32_t> hm(h.n_nodes);
        MSFEM_CK(cudaMemcpyAsync(hm.data(), h.mask.p, sizeof(int32_t) * h.n_nodes, cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        for (int c = 0; c < n_cells; c++) {
            int cnt[12] = {0};
            for (int64_t i = h.h_node_off[c]; i < h.h_node_off[c + 1]; i++)
                for (int e = 0; e < 12; e++) {
                    int axis, fa, fb, vl, vh;
                    edge_info(e, axis, fa, fb, vl, vh);
                    const int want = (1 << fa) | (1 << fb);
                    if ((hm[i] & want) == want) cnt[e]++;
                }
            for (int e = 0; e < 12; e++) cap = std::max(cap, cnt[e]);
        }
        if (cap > kMaxEdgeNodes) {
            set_error("msfem_cells_create: %d nodes on one cell edge (limit %d)", cap, kMaxEdgeNodes);
            return MSFEM_ERR_LIMIT;
        }
        h.cap = cap;
        MSFEM_TRY(h.edge_nodes.alloc(12 * (size_t)n_cells * cap));
        MSFEM_TRY(h.edge_len.alloc(12 * (size_t)n_cells));
        MSFEM_TRY(h.seg_tri.alloc(12 * (size_t)n_cells * cap));
        MSFEM_CK(cudaMemsetAsync(h.flag.p, 0, sizeof(int), st));
        k_edges<<<n_cells, 384, 0, st>>>(n_cells, h.node_off.p, h.mask.p, h.xyz.p, h.vert.p, h.fidx.p, h.n_nodes,
                                         F.elem_off.p, F.elems.p, cap, h.edge_nodes.p, h.edge_len.p, h.seg_tri.p,
                                         h.flag.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_TRY(read_flag(st, h.flag, &bad));
        if (bad) {
            set_error("msfem_cells_create: inconsistent cell edge (code %d: node count, ends or a segment without a "
                      "face triangle)", bad);
            return MSFEM_ERR_ARGUMENT;
        }
    }

    // volumes: the cell meshes themselves
    BatchSys& V = h.vols;
    V.dim = 3;
    V.k1 = 4;
    V.R = 8;
    V.n_sys = n_cells;
    V.stream = st;
    V.h_node_off = h.h_node_off;
    V.h_elem_off = h.h_tet_off;
    V.n_nodes = h.n_nodes;
    V.n_elems = h.n_tets;
    MSFEM_TRY(copy_in(st, V.node_off, h.h_node_off.data(), n_cells + 1));
    MSFEM_TRY(copy_in(st, V.elem_off, h.h_tet_off.data(), n_cells + 1));
    MSFEM_TRY(copy_in(st, V.emat, h.mat.p, (size_t)h.n_tets));
    MSFEM_TRY(V.fixed.alloc(h.n_nodes));
    {
        // Dirichlet nodes: every node on the cell's boundary
        std::vector<int32_t> hm(h.n_nodes);
        std::vector<uint8_t> hf(h.n_nodes);
        MSFEM_CK(cudaMemcpyAsync(hm.data(), h.mask.p, sizeof(int32_t) * h.n_nodes, cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        for (int64_t i = 0; i < h.n_nodes; i++) hf[i] = hm[i] ? 1 : 0;
        MSFEM_CK(cudaMemcpyAsync(V.fixed.p, hf.data(), h.n_nodes, cudaMemcpyHostToDevice, st));
        MSFEM_CK(cudaStreamSynchronize(st));
    }
    MSFEM_TRY(batch_build_pattern(V, h.xyz.p));
    MSFEM_TRY(h.prof.alloc(6 * h.n_nodes));
    MSFEM_TRY(h.fx.alloc(12 * F.n_nodes));
    MSFEM_TRY(h.bx.alloc(24 * h.n_nodes));
    for (auto& e : h.ev) MSFEM_CK(cudaEventCreate(&e));
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

// the face batch's materials for the current face_material mode
int set_face_materials(CellsHandle& h, int mode)
{
    cudaStream_t st = h.stream;
    BatchSys& F = h.faces;
    if (mode == h.face_material) return MSFEM_OK;
    if (mode == 1) {
        MSFEM_TRY(h.face_emat_cells.alloc(F.n_elems));
        MSFEM_CK(cudaMemcpyAsync(h.face_emat_cells.p, F.emat.p, sizeof(int32_t) * F.n_elems, cudaMemcpyDeviceToDevice, st));
        MSFEM_CK(cudaMemsetAsync(F.emat.p, 0, sizeof(int32_t) * F.n_elems, st));
    } else {
        MSFEM_CK(cudaMemcpyAsync(F.emat.p, h.face_emat_cells.p, sizeof(int32_t) * F.n_elems, cudaMemcpyDeviceToDevice, st));
    }
    MSFEM_CK(cudaStreamSynchronize(st));
    h.face_material = mode;
    return MSFEM_OK;
}

// The launches of one stage of the Order1 build: 0 both assemblies, 1 the closed-form edges and
// the face problems' Dirichlet data, 2 the face batch, 3 the volume problems' Dirichlet data and
// the volume batch.  `tf` / `tv`: the face / volume CTA sizes (0: batch_solve autotunes, which
// synchronises).
int cells_stage(CellsHandle& h, int stage, int precision, double tol, int maxiter, int tf, int tv)
{
    cudaStream_t st = h.stream;
    BatchSys& F = h.faces;
    BatchSys& V = h.vols;
    switch (stage) {
    case 0:
        MSFEM_TRY(batch_assemble_enqueue(F, h.fxyz.p, h.lame.p, h.n_mat));
        MSFEM_TRY(batch_assemble_enqueue(V, h.xyz.p, h.lame.p, h.n_mat));
        break;
    case 1: {
        MSFEM_CK(cudaMemsetAsync(h.flag.p, 0, sizeof(int), st));
        MSFEM_CK(cudaMemsetAsync(h.prof.p, 0, sizeof(double) * 6 * h.n_nodes, st));
        const int n_edges = 12 * h.n_cells;
        k_edge_profiles<<<blocks_for(n_edges, 128), 128, 0, st>>>(n_edges, h.cap, h.edge_nodes.p, h.edge_len.p,
                                                                  h.seg_tri.p, F.emat.p, h.lame.p, h.n_mat, h.xyz.p,
                                                                  h.prof.p, h.flag.p);
        k_face_dirichlet<<<blocks_for(F.n_nodes), 256, 0, st>>>(F.n_nodes, h.fcell_node.p, F.fixed.p, F.node_off.p,
                                                                F.n_sys, h.mask.p, h.vert.p, h.node_off.p, h.n_cells,
                                                                h.prof.p, h.fx.p);
        MSFEM_CK(cudaGetLastError());
        break;
    }
    case 2:
        MSFEM_TRY(batch_solve(F, h.fx.p, precision, tol, maxiter, tf));
        break;
    default:
        k_volume_dirichlet<<<blocks_for(h.n_nodes), 256, 0, st>>>(h.n_nodes, h.mask.p, h.fidx.p, h.fx.p, h.bx.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_TRY(batch_solve(V, h.bx.p, precision, tol, maxiter, tv));
    }
    return 0;
}

int cells_build(CellsHandle& h, int precision, double tol, int maxiter, int threads)
{
    cudaStream_t st = h.stream;
    BatchSys& F = h.faces;
    BatchSys& V = h.vols;
    h.vols_assembled = true;
    const int tf = batch_threads(F, precision, threads), tv = batch_threads(V, precision, threads);
    const double key[5] = {(double)precision, tol, (double)maxiter, (double)tf, (double)tv};
    const bool have_graph = h.build_graph[0] && std::memcmp(key, h.build_key, sizeof(key)) == 0;
    // capture only a build whose launches have run once with this key: every buffer is then
    // allocated and the CTA sizes tuned, so the capture holds launches and copies only
    const bool can_capture = tf > 0 && tv > 0 && std::memcmp(key, h.eager_key, sizeof(key)) == 0;
    if (have_graph || can_capture) {
        if (!have_graph) {
            for (auto& g : h.build_graph)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
            for (int k = 0; k < 4; k++) {
                cudaGraph_t g;
                MSFEM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                const int rc = cells_stage(h, k, precision, tol, maxiter, tf, tv);
                const cudaError_t e = cudaStreamEndCapture(st, &g);
                if (rc < 0) return rc;
                if (e != cudaSuccess) {
                    set_error("msfem_cells_build_bases: graph capture failed: %s", cudaGetErrorString(e));
                    return MSFEM_ERR_CUDA;
                }
                const cudaError_t ei = cudaGraphInstantiate(&h.build_graph[k], g, 0);
                cudaGraphDestroy(g);
                if (ei != cudaSuccess) {
                    h.build_graph[k] = nullptr;
                    set_error("msfem_cells_build_bases: graph instantiate failed: %s", cudaGetErrorString(ei));
                    return MSFEM_ERR_CUDA;
                }
            }
            std::memcpy(h.build_key, key, sizeof(key));
        }
        for (int k = 0; k < 4; k++) {
            MSFEM_CK(cudaEventRecord(h.ev[k], st));
            MSFEM_CK(cudaGraphLaunch(h.build_graph[k], st));
        }
        MSFEM_CK(cudaEventRecord(h.ev[4], st));
        h.graph_builds++;
    } else {
        // launch by launch (the first build tunes the persistent launches' CTA sizes, which
        // synchronises); the next build with the same key is captured
        for (int k = 0; k < 4; k++) {
            MSFEM_CK(cudaEventRecord(h.ev[k], st));
            MSFEM_TRY(cells_stage(h, k, precision, tol, maxiter, tf, tv));
        }
        MSFEM_CK(cudaEventRecord(h.ev[4], st));
        const double k2[5] = {(double)precision, tol, (double)maxiter, (double)batch_threads(F, precision, threads),
                              (double)batch_threads(V, precision, threads)};
        std::memcpy(h.eager_key, k2, sizeof(k2));
    }
    MSFEM_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; k++) MSFEM_CK(cudaEventElapsedTime(&h.ms[k], h.ev[k], h.ev[k + 1]));
    int bad = 0, bad_f = 0, bad_v = 0;
    MSFEM_TRY(read_flag(st, h.flag, &bad));
    MSFEM_TRY(read_flag(st, F.aflag, &bad_f));
    MSFEM_TRY(read_flag(st, V.aflag, &bad_v));
    if (bad_f || bad_v) {
        set_error("msfem_cells_build_bases: a material id is out of range");
        return MSFEM_ERR_ARGUMENT;
    }
    if (bad) {
        set_error("msfem_cells_build_bases: an edge segment has a material with zero shear modulus");
        return MSFEM_ERR_ARGUMENT;
    }
    int nf = 0, nv = 0;
    MSFEM_TRY(batch_finish(F, &nf, tol, nullptr));
    MSFEM_TRY(batch_finish(V, &nv, tol, nullptr));
    if (nf || nv) {
        set_error("msfem_cells_build_bases: %d face and %d volume problems missed the tolerance", nf, nv);
        return MSFEM_NOT_CONVERGED;
    }
    return 0;
}

// ---- MsFEM Order2 bases (Grid_forMech::CreateFunctionalSpaces, MsFEM_Grid.h:1001-3080): 27 per
// cell, ordered vertex (8, the cell's vertex order) -> edge (12, ascending global edge id) ->
// face (6, x0 x1 y0 y1 z0 z1) -> cell (1), :3045-3054.
//   edges: every edge segment is material 0 (the reference reads the edge meshes out of its
//     Salome face files, whose ReadFromSalomeDat leaves every material id 0, Library/Math.h:91-147),
//     so the two linear edge problems are linear in arc length and the bubble problem (source of
//     phi = 4 xi (1 - xi) (1,1,1), :1378-1400) is phi (1,1,1) at the nodes: P1 is nodally exact
//     for a constant coefficient and load in 1-D;
//   faces: 4 linear + 4 edge-bubble problems per face on material 0, no load (FEM_2D adds element
//     loads only when it logs, FEM/FEM.h:4479-4490), one batch with R = 8; the face bubble is 0;
//   volume: 8 linear problems without load and 19 bubble problems whose loads are the integrals
//     of f . phi_I with the tetrahedron's 4-point rule (FEM/FEM_Grid.h:2521-2566), f the
//     operator -[(lambda + mu) H (1,1,1) + mu tr(H) (1,1,1)] of the bubble's Hessian H
//     (:2371-2480 edges, :2598-2700 faces, :2770-2830 cell) with the tetrahedron's own material,
//     solved as 4 passes of 8 right-hand sides on the cell matrices.
// For a box cell the reference's frames are the global axes up to sign, and every one of these
// sources is unchanged by those signs, so the bubbles are written in global coordinates.

// edge values at the interior edge nodes: eprof[node][0] = 1 - s (1 at the low end),
// [1] = s (1 at the high end), [2] = 4 s (1 - s), s = arc length from the low end / edge length
__global__ void k_o2_edges(int n_edges, int cap, const int32_t* __restrict__ edge_nodes,
                           const int32_t* __restrict__ edge_len, const double* __restrict__ xyz,
                           double* __restrict__ eprof)
{
    for (int eid = blockIdx.x * blockDim.x + threadIdx.x; eid < n_edges; eid += gridDim.x * blockDim.x) {
        const int n = edge_len[eid];
        if (n < 3) continue;
        const int32_t* nodes = edge_nodes + (int64_t)eid * cap;
        double total = 0.0;
        for (int k = 0; k + 1 < n; k++) {
            double L = 0.0;
            for (int q = 0; q < 3; q++) {
                const double u = xyz[3 * (int64_t)nodes[k + 1] + q] - xyz[3 * (int64_t)nodes[k] + q];
                L += u * u;
            }
            total += sqrt(L);
        }
        double acc = 0.0;
        for (int k = 1; k + 1 < n; k++) {
            double L = 0.0;
            for (int q = 0; q < 3; q++) {
                const double u = xyz[3 * (int64_t)nodes[k] + q] - xyz[3 * (int64_t)nodes[k - 1] + q];
                L += u * u;
            }
            acc += sqrt(L);
            const double s = acc / total;
            double* o = eprof + 3 * (int64_t)nodes[k];
            o[0] = 1.0 - s;
            o[1] = s;
            o[2] = 4.0 * s * (1.0 - s);
        }
    }
}

// index of edge e among the 4 edges of face f (ascending e), or -1
__host__ __device__ __forceinline__ int face_edge_index(int f, int e)
{
    int k = 0;
    for (int q = 0; q < 12; q++) {
        int axis, fa, fb, vl, vh;
        edge_info(q, axis, fa, fb, vl, vh);
        if (fa != f && fb != f) continue;
        if (q == e) return k;
        k++;
    }
    return -1;
}

// the edge of a non-corner boundary node that lies on face f (its other face g), or -1
__device__ __forceinline__ int node_edge(int m, int f)
{
    const int rest = m & ~(1 << f);
    if (__popc(m) != 2 || !rest) return -1;
    const int g = __ffs(rest) - 1;
    for (int e = 0; e < 12; e++) {
        int axis, fa, fb, vl, vh;
        edge_info(e, axis, fa, fb, vl, vh);
        if ((fa == f && fb == g) || (fa == g && fb == f)) return e;
    }
    return -1;
}

// Dirichlet data of the Order2 face problems: fx[face node][8][3]; slots 0-3 the linear problems
// of the face's vertices (increasing b), slots 4-7 the bubble problems of its edges (ascending e)
__global__ void k_o2_face_dirichlet(int64_t n_fnodes, const int32_t* __restrict__ fcell_node,
                                    const uint8_t* __restrict__ ffixed, const int64_t* __restrict__ fsys_node_off,
                                    int n_fsys, const int32_t* __restrict__ mask, const int32_t* __restrict__ vert,
                                    const double* __restrict__ eprof, double* __restrict__ fx)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_fnodes; k += (int64_t)gridDim.x * blockDim.x) {
        double* o = fx + 24 * k;
        for (int q = 0; q < 24; q++) o[q] = 0.0;
        if (!ffixed[k]) continue;
        int lo = 0, hi = n_fsys - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (fsys_node_off[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        const int c = lo / 6, f = lo % 6;
        const int64_t i = fcell_node[k];
        const int m = mask[i];
        const bool corner = __popc(m) == 3;
        const int e = corner ? -1 : node_edge(m, f);
        for (int j = 0; j < 4; j++) {
            const int v = face_vertex(f, j);
            double val = 0.0;
            if (corner) {
                val = (i == vert[8 * c + v]) ? 1.0 : 0.0;
            } else if (e >= 0) {
                int axis, fa, fb, vl, vh;
                edge_info(e, axis, fa, fb, vl, vh);
                if (v == vl) val = eprof[3 * i];
                else if (v == vh) val = eprof[3 * i + 1];
            }
            for (int q = 0; q < 3; q++) o[3 * j + q] = val;
        }
        if (e >= 0) {
            const int j = 4 + face_edge_index(f, e);
            for (int q = 0; q < 3; q++) o[3 * j + q] = eprof[3 * i + 2];
        }
    }
}

__device__ __forceinline__ int cell_of_node(const int64_t* __restrict__ node_off, int n_cells, int64_t i)
{
    int lo = 0, hi = n_cells - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (node_off[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct O2Slots {
    int dof[8];  // the basis each right-hand side of a volume pass solves for
};

// Dirichlet data of an Order2 volume pass: x[node][8][3] (boundary nodes; the rest 0)
__global__ void k_o2_volume_dirichlet(int64_t n_nodes, const int64_t* __restrict__ node_off, int n_cells,
                                     const int32_t* __restrict__ mask, const int32_t* __restrict__ fidx_all,
                                     const int32_t* __restrict__ perm, const double* __restrict__ fx, O2Slots sl,
                                     double* __restrict__ x)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const int m = mask[i];
        double* o = x + 24 * i;
        for (int q = 0; q < 24; q++) o[q] = 0.0;
        if (!m) continue;
        const int c = cell_of_node(node_off, n_cells, i);
        for (int s = 0; s < 8; s++) {
            const int d = sl.dof[s];
            int common = 0, j = -1;
            if (d < 8) {
                common = m & vertex_face_mask(d);
            } else if (d < 20) {
                int axis, fa, fb, vl, vh;
                edge_info(perm[12 * c + d - 8], axis, fa, fb, vl, vh);
                common = m & ((1 << fa) | (1 << fb));
            }
            if (!common) continue;
            const int f = __ffs(common) - 1;  // the lowest face through both
            j = d < 8 ? face_vertex_index(f, d) : 4 + face_edge_index(f, perm[12 * c + d - 8]);
            const int64_t k = fidx_all[(int64_t)f * n_nodes + i];
            for (int q = 0; q < 3; q++) o[3 * s + q] = fx[24 * k + 3 * j + q];
        }
    }
}

// (phi, phi', phi'') of one axis factor at xi: the bubble 4 xi (1 - xi), or the linear function
// that is 1 on side `side` (0: xi = 0) and 0 on the other
__device__ __forceinline__ void o2_factor(bool bubble, int side, double xi, double h, double out[3])
{
    if (bubble) {
        out[0] = -4.0 * xi * xi + 4.0 * xi;
        out[1] = -8.0 / h * xi + 4.0 / h;
        out[2] = -8.0 / (h * h);
    } else if (side == 0) {
        out[0] = 1.0 - xi;
        out[1] = -1.0 / h;
        out[2] = 0.0;
    } else {
        out[0] = xi;
        out[1] = 1.0 / h;
        out[2] = 0.0;
    }
}

// the source of bubble d (8..26) at x: -[(lambda + mu) H (1,1,1) + mu tr(H) (1,1,1)]
__device__ void o2_source(int d, int e, const double* bx, const double x[3], double lam, double mu, double f[3])
{
    bool bub[3] = {true, true, true};
    int side[3] = {0, 0, 0};
    if (d < 20) {
        int axis, fa, fb, vl, vh;
        edge_info(e, axis, fa, fb, vl, vh);
        bub[fa >> 1] = false;
        side[fa >> 1] = fa & 1;
        bub[fb >> 1] = false;
        side[fb >> 1] = fb & 1;
    } else if (d < 26) {
        const int face = d - 20;
        bub[face >> 1] = false;
        side[face >> 1] = face & 1;
    }
    double F[3][3];
    for (int a = 0; a < 3; a++) {
        const double h = bx[2 * a + 1] - bx[2 * a];
        o2_factor(bub[a], side[a], (x[a] - bx[2 * a]) / h, h, F[a]);
    }
    double H[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double v = 1.0;
            for (int k = 0; k < 3; k++) v *= (a == b) ? (k == a ? F[k][2] : F[k][0]) : (k == a || k == b ? F[k][1] : F[k][0]);
            H[a][b] = v;
        }
    const double tr = H[0][0] + H[1][1] + H[2][2];
    for (int a = 0; a < 3; a++) f[a] = -((lam + mu) * (H[a][0] + H[a][1] + H[a][2]) + mu * tr);
}

// loads of an Order2 volume pass at every node, gathered over the node's tetrahedra in element
// order (the contributions of its diagonal block): rhs[node][8][3]
__global__ void k_o2_loads(int64_t n_nodes, const int64_t* __restrict__ node_off, int n_cells,
                           const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                           const int64_t* __restrict__ cstart, const uint32_t* __restrict__ contrib,
                           const int32_t* __restrict__ elems, const int32_t* __restrict__ emat,
                           const double* __restrict__ lame, int n_mat, const double* __restrict__ xyz,
                           const double* __restrict__ box, const int32_t* __restrict__ perm, O2Slots sl,
                           double* __restrict__ rhs)
{
    const double u = (5.0 - sqrt(5.0)) / 20.0, vv = 1.0 - 3.0 * u;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        double acc[8][3];
        for (int s = 0; s < 8; s++)
            for (int q = 0; q < 3; q++) acc[s][q] = 0.0;
        const int c = cell_of_node(node_off, n_cells, i);
        const double* bx = box + 6 * c;
        int64_t kd = -1;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++)
            if (col[k] == i) kd = k;
        if (kd >= 0)
            for (int64_t t = cstart[kd]; t < cstart[kd + 1]; t++) {
                const uint32_t tag = contrib[t];
                const int64_t e = tag >> 4;
                const int a = (tag >> 2) & 3;
                int v[4];
                for (int k = 0; k < 4; k++) v[k] = elems[4 * e + k];
                TetGeom G;
                tet_geometry(xyz, v, G);
                const int mt = emat[e];
                if (mt < 0 || mt >= n_mat) continue;  // rejected when the cell matrices were assembled
                const double lam = lame[2 * mt], mu = lame[2 * mt + 1];
                for (int q = 0; q < 4; q++) {
                    double bar[4];
                    for (int k = 0; k < 4; k++) bar[k] = (k == q) ? vv : u;
                    double x[3] = {0, 0, 0};
                    for (int k = 0; k < 4; k++)
                        for (int r = 0; r < 3; r++) x[r] += bar[k] * xyz[3 * (int64_t)v[k] + r];
                    const double w = 0.25 * G.vol * bar[a];
                    for (int s = 0; s < 8; s++) {
                        const int d = sl.dof[s];
                        if (d < 8) continue;
                        double f[3];
                        o2_source(d, d < 20 ? perm[12 * c + d - 8] : -1, bx, x, lam, mu, f);
                        for (int r = 0; r < 3; r++) acc[s][r] += w * f[r];
                    }
                }
            }
        double* o = rhs + 24 * i;
        for (int s = 0; s < 8; s++)
            for (int r = 0; r < 3; r++) o[3 * s + r] = acc[s][r];
    }
}

__global__ void k_o2_scatter(int64_t n_nodes, const double* __restrict__ x, O2Slots sl, int n_real,
                             double* __restrict__ bases)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x)
        for (int s = 0; s < n_real; s++)
            for (int q = 0; q < 3; q++) bases[81 * i + 3 * sl.dof[s] + q] = x[24 * i + 3 * s + q];
}

}  // namespace

// host: the local edge (edge_info numbering) of each Order2 edge-bubble slot, per cell
int order2_edge_order(int n_cells, const int32_t* cell_vertex, int32_t* perm)
{
    for (int c = 0; c < n_cells; c++) {
        const int32_t* g = cell_vertex + 8 * (size_t)c;
        for (int a = 0; a < 8; a++)
            for (int b = a + 1; b < 8; b++)
                if (g[a] == g[b]) {
                    set_error("Order2 cells: cell %d repeats the global vertex %d", c, g[a]);
                    return MSFEM_ERR_ARGUMENT;
                }
        int idx[12];
        for (int e = 0; e < 12; e++) idx[e] = e;
        auto key = [&](int e) {
            int axis, fa, fb, vl, vh;
            edge_info(e, axis, fa, fb, vl, vh);
            return std::make_pair(std::min(g[vl], g[vh]), std::max(g[vl], g[vh]));
        };
        std::sort(idx, idx + 12, [&](int p, int q) { return key(p) < key(q); });
        for (int k = 0; k < 12; k++) perm[12 * (size_t)c + k] = idx[k];
    }
    return MSFEM_OK;
}

namespace {

int cells_build_order2(CellsHandle& h, const int32_t* cell_vertex, int precision, double tol, int maxiter, int threads)
{
    cudaStream_t st = h.stream;
    BatchSys& F = h.faces;
    BatchSys& F2 = h.faces2;
    BatchSys& V = h.vols;
    // DOF slot k of the edge bubbles -> local edge: ascending (lower, higher) global vertex pair
    {
        std::vector<int32_t> gv(8 * (size_t)h.n_cells), perm(12 * (size_t)h.n_cells);
        MSFEM_CK(cudaMemcpyAsync(gv.data(), cell_vertex, sizeof(int32_t) * gv.size(), cudaMemcpyDefault, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        MSFEM_TRY(order2_edge_order(h.n_cells, gv.data(), perm.data()));
        MSFEM_TRY(copy_in(st, h.edge_perm, perm.data(), perm.size()));
    }
    if (!h.faces2_ready) {
        F2.dim = 2;
        F2.k1 = 3;
        F2.R = 8;
        F2.n_sys = F.n_sys;
        F2.stream = st;
        F2.h_node_off = F.h_node_off;
        F2.h_elem_off = F.h_elem_off;
        F2.n_nodes = F.n_nodes;
        F2.n_elems = F.n_elems;
        MSFEM_TRY(copy_in(st, F2.node_off, F.h_node_off.data(), F.n_sys + 1));
        MSFEM_TRY(copy_in(st, F2.elem_off, F.h_elem_off.data(), F.n_sys + 1));
        MSFEM_TRY(F2.elems.alloc(3 * F.n_elems));
        MSFEM_CK(cudaMemcpyAsync(F2.elems.p, F.elems.p, sizeof(int32_t) * 3 * F.n_elems, cudaMemcpyDeviceToDevice, st));
        MSFEM_TRY(F2.fixed.alloc(F.n_nodes));
        MSFEM_CK(cudaMemcpyAsync(F2.fixed.p, F.fixed.p, F.n_nodes, cudaMemcpyDeviceToDevice, st));
        MSFEM_TRY(F2.emat.alloc(F.n_elems));
        MSFEM_CK(cudaMemsetAsync(F2.emat.p, 0, sizeof(int32_t) * F.n_elems, st));
        MSFEM_TRY(batch_build_pattern(F2, h.fxyz.p));
        h.faces2_ready = true;
    }
    MSFEM_CK(cudaEventRecord(h.ev[0], st));
    MSFEM_TRY(batch_assemble(F2, h.fxyz.p, h.lame.p, h.n_mat));
    if (!h.vols_assembled) {
        MSFEM_TRY(batch_assemble(V, h.xyz.p, h.lame.p, h.n_mat));
        h.vols_assembled = true;
    }
    MSFEM_CK(cudaEventRecord(h.ev[1], st));
    MSFEM_TRY(h.eprof2.alloc(3 * (size_t)h.n_nodes));
    MSFEM_CK(cudaMemsetAsync(h.eprof2.p, 0, sizeof(double) * 3 * h.n_nodes, st));
    const int n_edges = 12 * h.n_cells;
    k_o2_edges<<<blocks_for(n_edges, 128), 128, 0, st>>>(n_edges, h.cap, h.edge_nodes.p, h.edge_len.p, h.xyz.p,
                                                         h.eprof2.p);
    MSFEM_TRY(h.fx2.alloc(24 * (size_t)F2.n_nodes));
    k_o2_face_dirichlet<<<blocks_for(F2.n_nodes), 256, 0, st>>>(F2.n_nodes, h.fcell_node.p, F2.fixed.p, F2.node_off.p,
                                                                F2.n_sys, h.mask.p, h.vert.p, h.eprof2.p, h.fx2.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaEventRecord(h.ev[2], st));
    MSFEM_TRY(batch_solve(F2, h.fx2.p, precision, tol, maxiter, threads));
    int nf = 0;
    MSFEM_TRY(batch_finish(F2, &nf, tol, nullptr));
    MSFEM_CK(cudaEventRecord(h.ev[3], st));
    MSFEM_TRY(h.x2.alloc(24 * (size_t)h.n_nodes));
    MSFEM_TRY(h.rhs2.alloc(24 * (size_t)h.n_nodes));
    MSFEM_TRY(h.bases2.alloc(81 * (size_t)h.n_nodes));
    // four passes of 8 right-hand sides: vertices; edges 0-7; edges 8-11 + faces 0-3; faces 4-5 +
    // the cell bubble (repeated to fill the pass)
    const O2Slots pass[4] = {{{0, 1, 2, 3, 4, 5, 6, 7}},
                             {{8, 9, 10, 11, 12, 13, 14, 15}},
                             {{16, 17, 18, 19, 20, 21, 22, 23}},
                             {{24, 25, 26, 26, 26, 26, 26, 26}}};
    const int n_real[4] = {8, 8, 8, 3};
    int nv = 0;
    for (int p = 0; p < 4; p++) {
        k_o2_volume_dirichlet<<<blocks_for(h.n_nodes), 256, 0, st>>>(h.n_nodes, h.node_off.p, h.n_cells, h.mask.p,
                                                                     h.fidx.p, h.edge_perm.p, h.fx2.p, pass[p], h.x2.p);
        MSFEM_CK(cudaGetLastError());
        if (p > 0) {
            k_o2_loads<<<blocks_for(h.n_nodes, 128), 128, 0, st>>>(h.n_nodes, h.node_off.p, h.n_cells, V.row_ptr.p,
                                                                  V.col.p, V.cstart.p, V.contrib.p, V.elems.p, V.emat.p,
                                                                  h.lame.p, h.n_mat, h.xyz.p, h.box.p, h.edge_perm.p, pass[p],
                                                                  h.rhs2.p);
            MSFEM_CK(cudaGetLastError());
            V.rhs = h.rhs2.p;
        }
        const int rc = batch_solve(V, h.x2.p, precision, tol, maxiter, threads);
        V.rhs = nullptr;
        MSFEM_TRY(rc);
        int bad = 0;
        MSFEM_TRY(batch_finish(V, &bad, tol, nullptr));
        nv += bad;
        k_o2_scatter<<<blocks_for(h.n_nodes), 256, 0, st>>>(h.n_nodes, h.x2.p, pass[p], n_real[p], h.bases2.p);
        MSFEM_CK(cudaGetLastError());
    }
    MSFEM_CK(cudaEventRecord(h.ev[4], st));
    MSFEM_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; k++) MSFEM_CK(cudaEventElapsedTime(&h.ms2[k], h.ev[k], h.ev[k + 1]));
    h.order2_built = true;
    if (nf || nv) {
        set_error("msfem_cells_build_order2: %d face and %d volume problems missed the tolerance", nf, nv);
        return MSFEM_NOT_CONVERGED;
    }
    return 0;
}

}  // namespace
}  // namespace msfem

using msfem::BatchHandle;
using msfem::CellsHandle;

struct msfem_batch : BatchHandle {};

extern "C" {

int msfem_batch_create(int dim, int n_systems, const int64_t* node_off, const double* xyz, const int64_t* elem_off,
                       const int32_t* elems, const int32_t* material, int n_materials, const double* E, const double* nu,
                       const uint8_t* fixed, int n_rhs, int on_device, msfem_batch_t* out)
{
    using namespace msfem;
    (void)on_device;
    if (!out || (dim != 2 && dim != 3) || n_systems <= 0 || !node_off || !xyz || !elem_off || !elems || !fixed ||
        n_materials <= 0 || !E || !nu || (n_rhs != 1 && n_rhs != 4 && n_rhs != 8)) {
        set_error("msfem_batch_create: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    std::unique_ptr<msfem_batch> h(new (std::nothrow) msfem_batch());
    if (!h) {
        set_error("out of host memory");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaGetDevice(&h->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    MSFEM_CK(cudaEventCreate(&h->e0));
    MSFEM_CK(cudaEventCreate(&h->e1));
    cudaStream_t st = h->stream;
    BatchSys& b = h->b;
    b.dim = dim;
    b.k1 = dim + 1;
    b.n_sys = n_systems;
    b.R = n_rhs;
    b.stream = st;
    b.h_node_off.resize(n_systems + 1);
    b.h_elem_off.resize(n_systems + 1);
    MSFEM_CK(cudaMemcpyAsync(b.h_node_off.data(), node_off, sizeof(int64_t) * (n_systems + 1), cudaMemcpyDefault, st));
    MSFEM_CK(cudaMemcpyAsync(b.h_elem_off.data(), elem_off, sizeof(int64_t) * (n_systems + 1), cudaMemcpyDefault, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (b.h_node_off[0] != 0 || b.h_elem_off[0] != 0) {
        set_error("msfem_batch_create: offsets must start at 0");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int s = 0; s < n_systems; s++)
        if (b.h_node_off[s + 1] <= b.h_node_off[s] || b.h_elem_off[s + 1] < b.h_elem_off[s]) {
            set_error("msfem_batch_create: offsets of system %d are not increasing", s);
            return MSFEM_ERR_ARGUMENT;
        }
    b.n_nodes = b.h_node_off[n_systems];
    b.n_elems = b.h_elem_off[n_systems];
    h->n_mat = n_materials;
    MSFEM_TRY(copy_in(st, b.node_off, b.h_node_off.data(), n_systems + 1));
    MSFEM_TRY(copy_in(st, b.elem_off, b.h_elem_off.data(), n_systems + 1));
    MSFEM_TRY(copy_in(st, h->xyz, xyz, 3 * (size_t)b.n_nodes));
    MSFEM_TRY(copy_in(st, b.elems, elems, (size_t)b.k1 * b.n_elems));
    if (material) {
        MSFEM_TRY(copy_in(st, b.emat, material, (size_t)b.n_elems));
    } else {
        MSFEM_TRY(b.emat.alloc(std::max<int64_t>(1, b.n_elems)));
        MSFEM_CK(cudaMemsetAsync(b.emat.p, 0, sizeof(int32_t) * std::max<int64_t>(1, b.n_elems), st));
    }
    MSFEM_TRY(copy_in(st, b.fixed, fixed, (size_t)b.n_nodes));
    MSFEM_TRY(lame_to_device(st, h->lame, E, nu, n_materials));
    MSFEM_TRY(batch_build_pattern(b, h->xyz.p));
    MSFEM_TRY(batch_assemble(b, h->xyz.p, h->lame.p, n_materials));
    *out = h.release();
    return MSFEM_OK;
}

int msfem_batch_solve(msfem_batch_t h, double* x, int precision, double tol, int maxiter, int threads, int on_device)
{
    using namespace msfem;
    if (!h || !x || maxiter <= 0 || !(tol > 0.0) || (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("msfem_batch_solve: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    BatchSys& b = h->b;
    cudaStream_t st = h->stream;
    const size_t n = (size_t)b.n_nodes * b.R * 3;
    double* dx = x;
    if (!on_device) {
        MSFEM_TRY(h->x.alloc(n));
        MSFEM_CK(cudaMemcpyAsync(h->x.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        dx = h->x.p;
    }
    MSFEM_CK(cudaEventRecord(h->e0, st));
    MSFEM_TRY(batch_solve(b, dx, precision, tol, maxiter, threads));
    MSFEM_CK(cudaEventRecord(h->e1, st));
    if (!on_device) MSFEM_CK(cudaMemcpyAsync(x, h->x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    MSFEM_CK(cudaEventElapsedTime(&h->ms, h->e0, h->e1));
    int nbad = 0;
    MSFEM_TRY(batch_finish(b, &nbad, tol, nullptr));
    if (nbad) {
        set_error("msfem_batch_solve: %d of %d systems missed the tolerance", nbad, b.n_sys);
        return MSFEM_NOT_CONVERGED;
    }
    return MSFEM_OK;
}

int msfem_batch_report(msfem_batch_t h, int32_t* inner, int32_t* outer, double* rel, double* ms)
{
    using namespace msfem;
    if (!h) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    BatchSys& b = h->b;
    cudaStream_t st = h->stream;
    if (inner) MSFEM_CK(cudaMemcpyAsync(inner, b.iters.p, sizeof(int32_t) * b.n_sys, cudaMemcpyDeviceToHost, st));
    if (outer) MSFEM_CK(cudaMemcpyAsync(outer, b.outers.p, sizeof(int32_t) * b.n_sys, cudaMemcpyDeviceToHost, st));
    if (rel) MSFEM_CK(cudaMemcpyAsync(rel, b.rel.p, sizeof(double) * b.n_sys, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (ms) *ms = h->ms;
    return MSFEM_OK;
}

void msfem_batch_destroy(msfem_batch_t h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
}

int msfem_cells_create(int n_cells, const int64_t* node_off, const double* xyz, const int64_t* tet_off,
                       const int32_t* tets, const int32_t* material, const double* box, int n_materials,
                       const double* E, const double* nu, int on_device, msfem_cells_t* out)
{
    using namespace msfem;
    (void)on_device;
    if (!out || n_cells <= 0 || !node_off || !xyz || !tet_off || !tets || !box || n_materials <= 0 || !E || !nu) {
        set_error("msfem_cells_create: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    std::unique_ptr<msfem_cells> h(new (std::nothrow) msfem_cells());
    if (!h) {
        set_error("out of host memory");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaGetDevice(&h->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    MSFEM_TRY(cells_create(n_cells, node_off, xyz, tet_off, tets, material, box, n_materials, E, nu, *h));
    // the reference's convention: material 0 on the face and edge problems
    MSFEM_TRY(set_face_materials(*h, 1));
    *out = h.release();
    return MSFEM_OK;
}

int msfem_cells_set_face_material(msfem_cells_t h, int mode)
{
    using namespace msfem;
    if (!h || (mode != 0 && mode != 1)) {
        set_error("msfem_cells_set_face_material: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    return set_face_materials(*h, mode);
}

int msfem_cells_build_bases(msfem_cells_t h, int precision, double tol, int maxiter, int threads)
{
    using namespace msfem;
    if (!h || maxiter <= 0 || !(tol > 0.0) || (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("msfem_cells_build_bases: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    return cells_build(*h, precision, tol, maxiter, threads);
}

int msfem_cells_get_bases(msfem_cells_t h, double* bases, int on_device)
{
    using namespace msfem;
    if (!h || !bases) {
        set_error("msfem_cells_get_bases: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    MSFEM_CK(cudaMemcpyAsync(bases, h->bx.p, sizeof(double) * 24 * h->n_nodes,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_order2_edge_order(int n_cells, const int32_t* cell_vertex, int32_t* order)
{
    if (n_cells < 0 || (n_cells > 0 && (!cell_vertex || !order))) {
        msfem::set_error("msfem_order2_edge_order: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    return msfem::order2_edge_order(n_cells, cell_vertex, order);
}

int msfem_cells_build_order2(msfem_cells_t h, const int32_t* cell_vertex, int precision, double tol, int maxiter,
                             int threads)
{
    using namespace msfem;
    if (!h || !cell_vertex || maxiter <= 0 || !(tol > 0.0) ||
        (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("msfem_cells_build_order2: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    return cells_build_order2(*h, cell_vertex, precision, tol, maxiter, threads);
}

int msfem_cells_get_order2_bases(msfem_cells_t h, double* bases, int on_device)
{
    using namespace msfem;
    if (!h || !bases || !h->order2_built) {
        set_error("msfem_cells_get_order2_bases: bad arguments or no Order2 bases built");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    MSFEM_CK(cudaMemcpyAsync(bases, h->bases2.p, sizeof(double) * 81 * h->n_nodes,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_cells_set_bases(msfem_cells_t h, const double* bases, int on_device)
{
    using namespace msfem;
    if (!h || !bases) {
        set_error("msfem_cells_set_bases: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    MSFEM_CK(cudaMemcpyAsync(h->bx.p, bases, sizeof(double) * 24 * h->n_nodes,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_cells_copy_bases(msfem_cells_t dst, msfem_cells_t src, int n, const int32_t* dst_cells)
{
    using namespace msfem;
    if (!dst || !src || n < 0 || n > src->n_cells || (n > 0 && !dst_cells)) {
        set_error("msfem_cells_copy_bases: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int k = 0; k < n; k++) {
        const int c = dst_cells[k];
        if (c < 0 || c >= dst->n_cells ||
            dst->h_node_off[c + 1] - dst->h_node_off[c] != src->h_node_off[k + 1] - src->h_node_off[k]) {
            set_error("msfem_cells_copy_bases: cell %d of the source does not fit cell %d of the target", k, c);
            return MSFEM_ERR_ARGUMENT;
        }
    }
    MSFEM_CK(cudaSetDevice(dst->device));
    MSFEM_CK(cudaStreamSynchronize(src->stream));
    for (int k = 0; k < n; k++) {
        const int c = dst_cells[k];
        const int64_t nn = src->h_node_off[k + 1] - src->h_node_off[k];
        MSFEM_CK(cudaMemcpyAsync(dst->bx.p + 24 * dst->h_node_off[c], src->bx.p + 24 * src->h_node_off[k],
                                 sizeof(double) * 24 * nn, cudaMemcpyDeviceToDevice, dst->stream));
    }
    MSFEM_CK(cudaStreamSynchronize(dst->stream));
    return MSFEM_OK;
}

int msfem_cells_basis_residual(msfem_cells_t h, double* rel)
{
    using namespace msfem;
    if (!h || !rel) {
        set_error("msfem_cells_basis_residual: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    BatchSys& V = h->vols;
    if (!h->vols_assembled) {
        MSFEM_TRY(batch_assemble(V, h->xyz.p, h->lame.p, h->n_mat));
        h->vols_assembled = true;
    }
    DBuf<double> d;
    MSFEM_TRY(d.alloc(h->n_cells));
    k_basis_residual<<<h->n_cells, 256, 0, h->stream>>>(V.node_off.p, V.row_ptr.p, V.col.p, V.val64.p, V.fixed.p, h->bx.p, d.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(rel, d.p, sizeof(double) * h->n_cells, cudaMemcpyDeviceToHost, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_cells_report(msfem_cells_t h, int32_t* inner, int32_t* outer, double* rel, double* face_rel, double* ms,
                       int32_t* threads)
{
    using namespace msfem;
    if (!h) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    cudaStream_t st = h->stream;
    const int n = h->n_cells;
    if (inner) MSFEM_CK(cudaMemcpyAsync(inner, h->vols.iters.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    if (outer) MSFEM_CK(cudaMemcpyAsync(outer, h->vols.outers.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    if (rel) MSFEM_CK(cudaMemcpyAsync(rel, h->vols.rel.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    std::vector<double> fr(6 * (size_t)n);
    if (face_rel) MSFEM_CK(cudaMemcpyAsync(fr.data(), h->faces.rel.p, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (face_rel)
        for (int c = 0; c < n; c++) {
            double w = 0.0;
            for (int f = 0; f < 6; f++) w = std::max(w, fr[6 * c + f]);
            face_rel[c] = w;
        }
    if (ms)
        for (int k = 0; k < 4; k++) ms[k] = h->ms[k];
    if (threads) {
        threads[0] = h->faces.threads;
        threads[1] = h->vols.threads;
    }
    return MSFEM_OK;
}

int msfem_cells_macro_matrices(msfem_cells_t h, double* K, int on_device)
{
    using namespace msfem;
    if (!h || !K) {
        set_error("msfem_cells_macro_matrices: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    DBuf<double> dK;
    double* out = K;
    if (!on_device) {
        MSFEM_TRY(dK.alloc(576 * (size_t)h->n_cells));
        out = dK.p;
    }
    const size_t smem = sizeof(double) * (96 * 72 + 96 * 3 + 96) + sizeof(int) * 96;
    MSFEM_CK(cudaFuncSetAttribute(k_macro_cells<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MSFEM_CK(cudaMemsetAsync(h->flag.p, 0, sizeof(int), st));
    k_macro_cells<8, false><<<h->n_cells, 256, smem, st>>>(h->tet_off.p, h->vols.elems.p, h->xyz.p, h->box.p, h->bx.p,
                                                           h->lame.p, out, h->flag.p);
    MSFEM_CK(cudaGetLastError());
    if (!on_device)
        MSFEM_CK(cudaMemcpyAsync(K, dK.p, sizeof(double) * 576 * h->n_cells, cudaMemcpyDeviceToHost, st));
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, h->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_cells_macro_matrices: a quadrature point lies in no tetrahedron of its cell");
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

int msfem_cells_order2_macro_matrices(msfem_cells_t h, double* K, int on_device)
{
    using namespace msfem;
    if (!h || !K || !h->order2_built) {
        set_error("msfem_cells_order2_macro_matrices: bad arguments or no Order2 bases built");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    constexpr size_t per = 27 * 27 * 9;
    DBuf<double> dK;
    double* out = K;
    if (!on_device) {
        MSFEM_TRY(dK.alloc(per * (size_t)h->n_cells));
        out = dK.p;
    }
    const size_t smem = sizeof(double) * (96 * 27 * 9 + 96 * 3 + 96) + sizeof(int) * 96;
    MSFEM_CK(cudaFuncSetAttribute(k_macro_cells<27, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MSFEM_CK(cudaMemsetAsync(h->flag.p, 0, sizeof(int), st));
    k_macro_cells<27, true><<<h->n_cells, 256, smem, st>>>(h->tet_off.p, h->vols.elems.p, h->xyz.p, h->box.p,
                                                           h->bases2.p, h->lame.p, out, h->flag.p);
    MSFEM_CK(cudaGetLastError());
    if (!on_device)
        MSFEM_CK(cudaMemcpyAsync(K, dK.p, sizeof(double) * per * h->n_cells, cudaMemcpyDeviceToHost, st));
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, h->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_cells_order2_macro_matrices: a quadrature point lies in no tetrahedron of its cell");
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

int msfem_cells_face_loads(msfem_cells_t h, int n_items, const int32_t* items, const double* traction, double* loads)
{
    using namespace msfem;
    if (!h || n_items < 0 || (n_items > 0 && (!items || !traction || !loads))) {
        set_error("msfem_cells_face_loads: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    if (n_items == 0) return MSFEM_OK;
    for (int i = 0; i < n_items; i++)
        if (items[2 * i] < 0 || items[2 * i] >= h->n_cells || items[2 * i + 1] < 0 || items[2 * i + 1] > 5) {
            set_error("msfem_cells_face_loads: item %d names cell %d face %d", i, items[2 * i], items[2 * i + 1]);
            return MSFEM_ERR_ARGUMENT;
        }
    MSFEM_CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    DBuf<int32_t> di;
    DBuf<double> dt, dout;
    MSFEM_TRY(di.alloc(2 * (size_t)n_items));
    MSFEM_TRY(dt.alloc(3 * (size_t)n_items));
    MSFEM_TRY(dout.alloc(24 * (size_t)n_items));
    MSFEM_CK(cudaMemcpyAsync(di.p, items, sizeof(int32_t) * 2 * n_items, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemcpyAsync(dt.p, traction, sizeof(double) * 3 * n_items, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemsetAsync(h->flag.p, 0, sizeof(int), st));
    k_face_loads<<<n_items, 128, 0, st>>>(n_items, di.p, dt.p, h->tet_off.p, h->vols.elems.p, h->xyz.p, h->box.p, h->bx.p,
                                          dout.p, h->flag.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(loads, dout.p, sizeof(double) * 24 * n_items, cudaMemcpyDeviceToHost, st));
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, h->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_cells_face_loads: a quadrature point lies in no tetrahedron of its cell");
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

int msfem_cells_reconstruct(msfem_cells_t h, int n_vertices, const int32_t* cell_vertex, const double* U, double* u)
{
    using namespace msfem;
    if (!h || n_vertices <= 0 || !cell_vertex || !U || !u) {
        set_error("msfem_cells_reconstruct: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int k = 0; k < 8 * h->n_cells; k++)
        if (cell_vertex[k] < 0 || cell_vertex[k] >= n_vertices) {
            set_error("msfem_cells_reconstruct: coarse vertex id %d out of range", cell_vertex[k]);
            return MSFEM_ERR_ARGUMENT;
        }
    MSFEM_CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    DBuf<int32_t> dv;
    DBuf<double> dU, du;
    MSFEM_TRY(dv.alloc(8 * (size_t)h->n_cells));
    MSFEM_TRY(dU.alloc(3 * (size_t)n_vertices));
    MSFEM_TRY(du.alloc(3 * (size_t)h->n_nodes));
    MSFEM_CK(cudaMemcpyAsync(dv.p, cell_vertex, sizeof(int32_t) * 8 * h->n_cells, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemcpyAsync(dU.p, U, sizeof(double) * 3 * n_vertices, cudaMemcpyHostToDevice, st));
    k_reconstruct<<<h->n_cells, 256, 0, st>>>(h->n_cells, h->node_off.p, dv.p, dU.p, h->bx.p, du.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(u, du.p, sizeof(double) * 3 * h->n_nodes, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return MSFEM_OK;
}

int msfem_cells_order1_macro_solve(msfem_cells_t h, int n_vertices, const int32_t* cell_vertex, int n_items,
                                   const int32_t* items, const double* traction, int n_fixed,
                                   const int32_t* fixed_vertices, const double* fixed_values, int precision, double tol,
                                   int maxiter, double* U, double* u, double* K_out, double* F_out, int32_t* iterations,
                                   double* rel_residual)
{
    using namespace msfem;
    if (!h || n_vertices <= 0 || !cell_vertex || n_items < 0 || (n_items > 0 && (!items || !traction)) || !U) {
        set_error("msfem_cells_order1_macro_solve: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int k = 0; k < 8 * h->n_cells; k++)
        if (cell_vertex[k] < 0 || cell_vertex[k] >= n_vertices) {
            set_error("msfem_cells_order1_macro_solve: coarse vertex id %d out of range", cell_vertex[k]);
            return MSFEM_ERR_ARGUMENT;
        }
    for (int i = 0; i < n_items; i++)
        if (items[2 * i] < 0 || items[2 * i] >= h->n_cells || items[2 * i + 1] < 0 || items[2 * i + 1] > 5) {
            set_error("msfem_cells_order1_macro_solve: item %d names cell %d face %d", i, items[2 * i], items[2 * i + 1]);
            return MSFEM_ERR_ARGUMENT;
        }
    MSFEM_CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int nc = h->n_cells;
    DBuf<int32_t> dv, di;
    DBuf<double> dK, dt, dl, dF, dU, du;
    MSFEM_TRY(dv.alloc(8 * (size_t)nc));
    MSFEM_TRY(dK.alloc(576 * (size_t)nc));
    MSFEM_TRY(dF.alloc(3 * (size_t)n_vertices));
    MSFEM_TRY(dU.alloc(3 * (size_t)n_vertices));
    MSFEM_CK(cudaMemcpyAsync(dv.p, cell_vertex, sizeof(int32_t) * 8 * nc, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemsetAsync(dF.p, 0, sizeof(double) * 3 * n_vertices, st));
    MSFEM_CK(cudaMemsetAsync(h->flag.p, 0, sizeof(int), st));
    // macro element matrices (SolveLocalMatrix), on the device
    const size_t smem = sizeof(double) * (96 * 72 + 96 * 3 + 96) + sizeof(int) * 96;
    MSFEM_CK(cudaFuncSetAttribute(k_macro_cells<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_macro_cells<8, false><<<nc, 256, smem, st>>>(h->tet_off.p, h->vols.elems.p, h->xyz.p, h->box.p, h->bx.p,
                                                   h->lame.p, dK.p, h->flag.p);
    // boundary loads and their sum over the macro vertices, item by item (SummPartOfVector)
    if (n_items > 0) {
        MSFEM_TRY(di.alloc(2 * (size_t)n_items));
        MSFEM_TRY(dt.alloc(3 * (size_t)n_items));
        MSFEM_TRY(dl.alloc(24 * (size_t)n_items));
        MSFEM_CK(cudaMemcpyAsync(di.p, items, sizeof(int32_t) * 2 * n_items, cudaMemcpyHostToDevice, st));
        MSFEM_CK(cudaMemcpyAsync(dt.p, traction, sizeof(double) * 3 * n_items, cudaMemcpyHostToDevice, st));
        k_face_loads<<<n_items, 128, 0, st>>>(n_items, di.p, dt.p, h->tet_off.p, h->vols.elems.p, h->xyz.p, h->box.p,
                                              h->bx.p, dl.p, h->flag.p);
        k_macro_load_sum<<<1, 32, 0, st>>>(n_items, di.p, dv.p, dl.p, dF.p);
    }
    MSFEM_CK(cudaGetLastError());
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, h->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_cells_order1_macro_solve: a quadrature point lies in no tetrahedron of its cell");
        return MSFEM_ERR_ARGUMENT;
    }
    // the macro solve on those device arrays, then the fine reconstruction
    const int rc = macro_solve_device(n_vertices, nc, cell_vertex, dK.p, dF.p, n_fixed, fixed_vertices, fixed_values,
                                      precision, tol, maxiter, dU.p, iterations, rel_residual, st);
    if (rc < 0) return rc;
    MSFEM_CK(cudaMemcpyAsync(U, dU.p, sizeof(double) * 3 * n_vertices, cudaMemcpyDeviceToHost, st));
    if (u) {
        MSFEM_TRY(du.alloc(3 * (size_t)h->n_nodes));
        k_reconstruct<<<nc, 256, 0, st>>>(nc, h->node_off.p, dv.p, dU.p, h->bx.p, du.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_CK(cudaMemcpyAsync(u, du.p, sizeof(double) * 3 * h->n_nodes, cudaMemcpyDeviceToHost, st));
    }
    if (K_out) MSFEM_CK(cudaMemcpyAsync(K_out, dK.p, sizeof(double) * 576 * nc, cudaMemcpyDeviceToHost, st));
    if (F_out) MSFEM_CK(cudaMemcpyAsync(F_out, dF.p, sizeof(double) * 3 * n_vertices, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return rc;
}

void msfem_cells_destroy(msfem_cells_t h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
}

}  // extern "C"
