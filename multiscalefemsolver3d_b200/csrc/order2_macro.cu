// The MsFEM Order2 macro phase on the device (MsFEM::MsFEM_forElasticDeformation_OrderBF2_forPoly,
// MsFEM/MsFEM.h:14-569), after the cells' 27 bases are built (cells.cu, cells_build_order2):
//   * the macro system: the cells' 27-DOF element matrices (msfem_cells_order2_macro_matrices)
//     summed by the cells' DOF lists into the DOF-level portrait (Grid_forMech::CreationPortrait +
//     CSSD_Matrix::SummPartOfMatrix, MsFEM.h:53-131) and written as the scalar system of
//     MakeCopyMatrix_A_into_B (DOF 3 d + c, every 3x3 block of the portrait kept whole, structural
//     zeros included).  The portrait and the block sums come from the batched assembler
//     (batch.cu: one stable sort of the (row, column) pairs, each block summed over its
//     contributions in (cell, I, J) order), so the values do not depend on threads;
//   * the Dirichlet values (Grid_forMech::CreateBoundaryConditions, MsFEM_Grid.h:3303-3470): per
//     group, the L2 projection of its constant value onto its DOFs over its faces -- per face the
//     9 x 9 mass matrix and load of the face's DOFs (4 vertices, 4 edges, the face) with the polygon
//     rule 3 (GeometryShape.h:2625-2640, the fan of centroid triangles with the triangle rule of
//     :1482-1540 as written there: its third point repeats the second), the bases' z components
//     interpolated in the lowest-numbered micro tetrahedron holding each point; the faces' sums
//     in face order, (I, J) order; then the group's dense system solved by Cholesky on its rows
//     that carry mass (a face bubble vanishes on its own face, so its row is empty and its value 0,
//     as the least-squares solve of the restatement and the reference's Gauss give);
//   * the elimination of the Dirichlet rows and columns (MsFEM.h:300-365) and the solve.
#include <algorithm>
#include <cfloat>
#include <memory>
#include <new>
#include <vector>

#include "cells.cuh"
#include "element.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

// face table row: the cell, then the face's 9 DOF ids -- its 4 cycle vertices (a vertex's DOF id is
// its vertex id), the edges between cycle nodes k and k + 1, the face
constexpr int kFaceInts = 10;
// a group's projection is one CTA's dense Cholesky (n^3 / 6 FMA): 4096 DOFs is a face of about
// 32 x 32 macro cells and a few seconds
constexpr int kMaxGroupDofs = 4096;

// scalar CSR (row 3 d + a) from the block CSR of the DOF portrait: the blocks of DOF row d, each
// as its three columns 3 e + b
__global__ void k_o2_expand(int n_dofs, const int64_t* __restrict__ brp, const int32_t* __restrict__ bcol,
                            const double* __restrict__ bval, int32_t* __restrict__ rp, int32_t* __restrict__ col,
                            double* __restrict__ val)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < 3 * n_dofs; r += gridDim.x * blockDim.x) {
        const int d = r / 3, a = r % 3;
        const int64_t b0 = brp[d], len = brp[d + 1] - b0;
        int64_t out = 9 * b0 + 3 * a * len;
        rp[r] = (int32_t)out;
        for (int64_t k = 0; k < len; k++) {
            const int j = bcol[b0 + k];
            for (int b = 0; b < 3; b++) {
                col[out] = 3 * j + b;
                val[out] = bval[9 * (b0 + k) + 3 * a + b];
                out++;
            }
        }
        if (r == 3 * n_dofs - 1) rp[3 * n_dofs] = (int32_t)(9 * brp[n_dofs]);
    }
}

// per Dirichlet face: Ml[I][J] = sum_q w_q psi_I(x_q) psi_J(x_q), wl[I] = sum_q w_q psi_I(x_q) over
// the 12 points of the polygon rule 3 on the face's vertex cycle, psi the z component of the basis
// of face DOF I in the face's cell
__global__ void __launch_bounds__(128) k_o2_face_mass(int n_faces, const int32_t* __restrict__ faces,
                                                      const double* __restrict__ vxyz, const int32_t* __restrict__ cell_dofs,
                                                      const int64_t* __restrict__ tet_off, const int32_t* __restrict__ tets,
                                                      const double* __restrict__ xyz, const double* __restrict__ bases,
                                                      double* __restrict__ Ml, double* __restrict__ wl, int* bad)
{
    __shared__ double sP[12][3], sW[12], sPsi[12][9];
    __shared__ int sT[12], sSlot[9];
    const int f = blockIdx.x, tid = threadIdx.x;
    if (f >= n_faces) return;
    const int32_t* row = faces + (int64_t)kFaceInts * f;
    const int c = row[0];
    if (tid < 12) {
        const int i = tid / 3, j = tid % 3;
        double C[3] = {0, 0, 0};
        for (int k = 0; k < 4; k++)
            for (int d = 0; d < 3; d++) C[d] += vxyz[3 * (int64_t)row[1 + k] + d];
        double e1[3], e2[3];
        for (int d = 0; d < 3; d++) {
            C[d] *= 0.25;
            e1[d] = vxyz[3 * (int64_t)row[1 + i] + d] - C[d];
            e2[d] = vxyz[3 * (int64_t)row[1 + (i + 1) % 4] + d] - C[d];
        }
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double a = j == 0 ? 1.0 / 6.0 : 2.0 / 3.0, b = 1.0 / 6.0;
        for (int d = 0; d < 3; d++) sP[tid][d] = C[d] + a * e1[d] + b * e2[d];
        sW[tid] = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) / 6.0;
        sT[tid] = 0x7fffffff;
    } else if (tid < 21) {
        const int I = tid - 12, d = row[1 + I];
        int s = -1;
        for (int k = 0; k < 27; k++)
            if (cell_dofs[27 * (int64_t)c + k] == d) s = k;
        if (s < 0) atomicExch(bad, 2);
        sSlot[I] = s < 0 ? 0 : s;
    }
    __syncthreads();
    const int64_t t0 = tet_off[c], t1 = tet_off[c + 1];
    for (int64_t e = t0 + tid; e < t1; e += blockDim.x) {
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        const double* p0 = xyz + 3 * (int64_t)v[0];
        for (int q = 0; q < 12; q++) {
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
    if (tid < 108) {
        const int q = tid / 9, I = tid % 9;
        double psi = 0.0;
        if (sT[q] == 0x7fffffff) {
            atomicExch(bad, 1);
        } else {
            const int64_t e = t0 + sT[q];
            int v[4];
            for (int k = 0; k < 4; k++) v[k] = tets[4 * e + k];
            TetGeom G;
            tet_geometry(xyz, v, G);
            const double* p0 = xyz + 3 * (int64_t)v[0];
            const double dx[3] = {sP[q][0] - p0[0], sP[q][1] - p0[1], sP[q][2] - p0[2]};
            for (int k = 0; k < 4; k++) {
                const double lam = (k == 0 ? 1.0 : 0.0) + G.g[k][0] * dx[0] + G.g[k][1] * dx[1] + G.g[k][2] * dx[2];
                psi += lam * bases[(27 * (int64_t)v[k] + sSlot[I]) * 3 + 2];
            }
        }
        sPsi[q][I] = psi;
    }
    __syncthreads();
    if (tid < 81) {
        const int I = tid / 9, J = tid % 9;
        double acc = 0.0;
        for (int q = 0; q < 12; q++) acc += sW[q] * sPsi[q][I] * sPsi[q][J];
        Ml[81 * (int64_t)f + tid] = acc;
    } else if (tid < 90) {
        const int I = tid - 81;
        double acc = 0.0;
        for (int q = 0; q < 12; q++) acc += sW[q] * sPsi[q][I];
        wl[9 * (int64_t)f + I] = acc;
    }
}

__device__ __forceinline__ int find_sorted(const int32_t* a, int n, int key)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && a[lo] == key) ? lo : -1;
}

// one CTA per Dirichlet group: its mass matrix and loads summed over its faces in order, then the
// projection solved by Cholesky on the rows that carry mass (rows whose diagonal is at most
// n eps max diag hold 0); vals [n][3] of the group's sorted DOFs
__global__ void __launch_bounds__(256) k_o2_group_project(const int32_t* __restrict__ dof_off,
                                                          const int32_t* __restrict__ dofs,
                                                          const int32_t* __restrict__ face_off,
                                                          const int32_t* __restrict__ faces,
                                                          const double* __restrict__ values,
                                                          const double* __restrict__ Ml, const double* __restrict__ wl,
                                                          const int64_t* __restrict__ m_off, double* __restrict__ Mscr,
                                                          unsigned char* __restrict__ active_scr,
                                                          double* __restrict__ vals, int* bad)
{
    const int g = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int n = dof_off[g + 1] - dof_off[g];
    const int32_t* gd = dofs + dof_off[g];
    double* M = Mscr + m_off[g];
    unsigned char* act = active_scr + dof_off[g];
    double* X = vals + 3 * (int64_t)dof_off[g];
    const double val[3] = {values[3 * g], values[3 * g + 1], values[3 * g + 2]};
    for (int64_t k = tid; k < (int64_t)n * n; k += nt) M[k] = 0.0;
    for (int k = tid; k < 3 * n; k += nt) X[k] = 0.0;
    __syncthreads();
    for (int f = face_off[g]; f < face_off[g + 1]; f++) {
        const int32_t* fd = faces + (int64_t)kFaceInts * f + 1;
        if (tid < 81) {
            const int pi = find_sorted(gd, n, fd[tid / 9]), pj = find_sorted(gd, n, fd[tid % 9]);
            if (pi >= 0 && pj >= 0) M[(int64_t)pi * n + pj] += Ml[81 * (int64_t)f + tid];
        } else if (tid < 90) {
            const int I = tid - 81, pi = find_sorted(gd, n, fd[I]);
            if (pi >= 0)
                for (int a = 0; a < 3; a++) X[3 * pi + a] += wl[9 * (int64_t)f + I] * val[a];
        }
        __syncthreads();
    }
    // rows with mass
    __shared__ double s_max[256];
    double mx = 0.0;
    for (int i = tid; i < n; i += nt) mx = fmax(mx, fabs(M[(int64_t)i * n + i]));
    s_max[tid] = mx;
    __syncthreads();
    for (int w = nt / 2; w > 0; w >>= 1) {
        if (tid < w) s_max[tid] = fmax(s_max[tid], s_max[tid + w]);
        __syncthreads();
    }
    const double thr = (double)n * DBL_EPSILON * s_max[0];
    for (int i = tid; i < n; i += nt) act[i] = M[(int64_t)i * n + i] > thr ? 1 : 0;
    __syncthreads();
    // Cholesky of the rows with mass, lower triangle in place
    __shared__ int s_fail;
    if (tid == 0) s_fail = 0;
    __syncthreads();
    for (int k = 0; k < n; k++) {
        if (!act[k]) continue;
        const double piv = M[(int64_t)k * n + k];
        if (!(piv > 0.0)) {
            if (tid == 0) s_fail = 1;
            break;
        }
        const double l = sqrt(piv);
        __syncthreads();
        for (int i = k + 1 + tid; i < n; i += nt)
            if (act[i]) M[(int64_t)i * n + k] /= l;
        if (tid == 0) M[(int64_t)k * n + k] = l;
        __syncthreads();
        // the lower trailing triangle: a warp per row, its lanes along the row
        const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
        for (int i = k + 1 + warp; i < n; i += nwarp) {
            if (!act[i]) continue;
            const double lik = M[(int64_t)i * n + k];
            for (int j = k + 1 + lane; j <= i; j += 32)
                if (act[j]) M[(int64_t)i * n + j] -= lik * M[(int64_t)j * n + k];
        }
        __syncthreads();
    }
    __syncthreads();
    if (s_fail) {
        if (tid == 0) atomicExch(bad, 3);
        for (int k = tid; k < 3 * n; k += nt) X[k] = 0.0;
        return;
    }
    // L y = b, then L^T x = y, three columns at once; rows without mass hold 0
    for (int k = 0; k < n; k++) {
        if (!act[k]) continue;
        if (tid < 3) X[3 * k + tid] /= M[(int64_t)k * n + k];
        __syncthreads();
        for (int t = tid; t < 3 * (n - k - 1); t += nt) {
            const int i = k + 1 + t / 3, a = t % 3;
            if (act[i]) X[3 * i + a] -= M[(int64_t)i * n + k] * X[3 * k + a];
        }
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; k--) {
        if (!act[k]) continue;
        if (tid < 3) X[3 * k + tid] /= M[(int64_t)k * n + k];
        __syncthreads();
        for (int t = tid; t < 3 * k; t += nt) {
            const int i = t / 3, a = t % 3;
            if (act[i]) X[3 * i + a] -= M[(int64_t)k * n + i] * X[3 * k + a];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += nt)
        if (!act[i])
            for (int a = 0; a < 3; a++) X[3 * i + a] = 0.0;
}

__global__ void k_o2_gather(int n, const int32_t* __restrict__ src, const double* __restrict__ proj, double* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = proj[src[i]];
}

template <class T>
int upload(cudaStream_t st, DBuf<T>& dst, const T* src, size_t n)
{
    MSFEM_TRY(dst.alloc(std::max<size_t>(1, n)));
    if (n) MSFEM_CK(cudaMemcpyAsync(dst.p, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return 0;
}

int check_cell_dofs(const msfem_cells& h, int n_dofs, const int32_t* cell_dofs, const char* who)
{
    if (n_dofs <= 0 || !cell_dofs || (int64_t)3 * n_dofs >= ((int64_t)1 << 31)) {
        set_error("%s: bad DOF count or DOF list", who);
        return MSFEM_ERR_ARGUMENT;
    }
    std::vector<unsigned char> used(n_dofs, 0);
    for (int64_t q = 0; q < 27 * (int64_t)h.n_cells; q++) {
        if (cell_dofs[q] < 0 || cell_dofs[q] >= n_dofs) {
            set_error("%s: cell %lld names DOF %d outside [0, %d)", who, (long long)(q / 27), cell_dofs[q], n_dofs);
            return MSFEM_ERR_ARGUMENT;
        }
        used[cell_dofs[q]] = 1;
    }
    for (int d = 0; d < n_dofs; d++)
        if (!used[d]) {
            set_error("%s: DOF %d belongs to no cell", who, d);
            return MSFEM_ERR_ARGUMENT;
        }
    return MSFEM_OK;
}

// the macro system as a scalar System on the device
int order2_macro_system(msfem_cells& h, int n_dofs, const int32_t* cell_dofs, msfem_system_t* out)
{
    const char* who = "msfem_cells_order2_macro_system";
    MSFEM_TRY(check_cell_dofs(h, n_dofs, cell_dofs, who));
    cudaStream_t st = h.stream;
    const int nc = h.n_cells;
    DBuf<double> dK;
    MSFEM_TRY(dK.alloc((size_t)27 * 27 * 9 * nc));
    MSFEM_TRY(msfem_cells_order2_macro_matrices(&h, dK.p, 1));
    BatchSys b;
    b.dim = 3;
    b.k1 = 27;
    b.n_sys = 1;
    b.R = 1;
    b.stream = st;
    b.h_node_off = {0, n_dofs};
    b.h_elem_off = {0, nc};
    b.n_nodes = n_dofs;
    b.n_elems = nc;
    MSFEM_TRY(upload(st, b.node_off, b.h_node_off.data(), 2));
    MSFEM_TRY(upload(st, b.elem_off, b.h_elem_off.data(), 2));
    MSFEM_TRY(upload(st, b.elems, cell_dofs, 27 * (size_t)nc));
    MSFEM_TRY(batch_build_pattern(b, nullptr));
    if (9 * b.nnzb >= ((int64_t)1 << 31)) {
        set_error("%s: %lld scalar entries exceed the int32 range", who, (long long)(9 * b.nnzb));
        return MSFEM_ERR_LIMIT;
    }
    MSFEM_TRY(batch_assemble_given(b, dK.p, false));
    DBuf<int32_t> rp, col;
    DBuf<double> val;
    MSFEM_TRY(rp.alloc(3 * (size_t)n_dofs + 1));
    MSFEM_TRY(col.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
    MSFEM_TRY(val.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
    k_o2_expand<<<(3 * n_dofs + 255) / 256, 256, 0, st>>>(n_dofs, b.row_ptr.p, b.col.p, b.val64.p, rp.p, col.p, val.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaStreamSynchronize(st));
    return system_adopt_csr(3 * n_dofs, rp, col, val, 9 * b.nnzb, out);
}

struct O2Groups {
    int n_faces = 0, n_groups = 0, n_group_dofs = 0;
    DBuf<int32_t> faces, dof_off, dofs, face_off, cell_dofs;
    DBuf<double> vxyz, values, Ml, wl, M, proj;
    DBuf<int64_t> m_off;
    DBuf<unsigned char> act;
};

// the projected Dirichlet values of every group on the device: g.proj [n_group_dofs][3]
int order2_project(msfem_cells& h, int n_dofs, const int32_t* cell_dofs, int n_vertices, const double* vertex_xyz,
                   int n_faces, const int32_t* faces, int n_groups, const int32_t* group_dof_off,
                   const int32_t* group_dofs, const int32_t* group_face_off, const double* group_values, O2Groups& g)
{
    const char* who = "msfem_cells_order2_dirichlet";
    MSFEM_TRY(check_cell_dofs(h, n_dofs, cell_dofs, who));
    if (n_vertices <= 0 || !vertex_xyz || n_faces < 0 || n_groups < 0 ||
        (n_groups > 0 && (!group_dof_off || !group_face_off || !group_values)) || (n_faces > 0 && !faces)) {
        set_error("%s: bad arguments", who);
        return MSFEM_ERR_ARGUMENT;
    }
    if (n_groups > 0 && (group_dof_off[0] != 0 || group_face_off[0] != 0 || group_face_off[n_groups] != n_faces ||
                         (group_dof_off[n_groups] > 0 && !group_dofs))) {
        set_error("%s: group offsets must start at 0 and cover the %d faces", who, n_faces);
        return MSFEM_ERR_ARGUMENT;
    }
    std::vector<int64_t> m_off(n_groups + 1, 0);
    for (int k = 0; k < n_groups; k++) {
        const int n = group_dof_off[k + 1] - group_dof_off[k];
        if (n < 0 || n > kMaxGroupDofs || group_face_off[k + 1] < group_face_off[k]) {
            set_error("%s: group %d has %d DOFs (at most %d) or decreasing face offsets", who, k, n, kMaxGroupDofs);
            return MSFEM_ERR_ARGUMENT;
        }
        const int32_t* gd = group_dofs + group_dof_off[k];
        for (int i = 0; i < n; i++)
            if (gd[i] < 0 || gd[i] >= n_dofs || (i > 0 && gd[i] <= gd[i - 1])) {
                set_error("%s: group %d's DOF list is not ascending inside [0, %d)", who, k, n_dofs);
                return MSFEM_ERR_ARGUMENT;
            }
        m_off[k + 1] = m_off[k] + (int64_t)n * n;
    }
    for (int f = 0; f < n_faces; f++) {
        const int32_t* r = faces + (int64_t)kFaceInts * f;
        bool ok = r[0] >= 0 && r[0] < h.n_cells;
        for (int k = 1; k < 5; k++) ok = ok && r[k] >= 0 && r[k] < n_vertices;
        for (int k = 5; k < kFaceInts; k++) ok = ok && r[k] >= n_vertices && r[k] < n_dofs;
        if (!ok) {
            set_error("%s: face %d names a cell, vertex or DOF out of range", who, f);
            return MSFEM_ERR_ARGUMENT;
        }
    }
    g.n_faces = n_faces;
    g.n_groups = n_groups;
    g.n_group_dofs = n_groups > 0 ? group_dof_off[n_groups] : 0;
    cudaStream_t st = h.stream;
    MSFEM_TRY(upload(st, g.faces, faces, (size_t)kFaceInts * n_faces));
    MSFEM_TRY(upload(st, g.dof_off, group_dof_off, n_groups > 0 ? (size_t)n_groups + 1 : 0));
    MSFEM_TRY(upload(st, g.dofs, group_dofs, (size_t)g.n_group_dofs));
    MSFEM_TRY(upload(st, g.face_off, group_face_off, n_groups > 0 ? (size_t)n_groups + 1 : 0));
    MSFEM_TRY(upload(st, g.cell_dofs, cell_dofs, 27 * (size_t)h.n_cells));
    MSFEM_TRY(upload(st, g.vxyz, vertex_xyz, 3 * (size_t)n_vertices));
    MSFEM_TRY(upload(st, g.values, group_values, 3 * (size_t)n_groups));
    MSFEM_TRY(upload(st, g.m_off, m_off.data(), m_off.size()));
    MSFEM_TRY(g.Ml.alloc(std::max<size_t>(1, 81 * (size_t)n_faces)));
    MSFEM_TRY(g.wl.alloc(std::max<size_t>(1, 9 * (size_t)n_faces)));
    MSFEM_TRY(g.M.alloc(std::max<int64_t>(1, m_off[n_groups])));
    MSFEM_TRY(g.act.alloc(std::max(1, g.n_group_dofs)));
    MSFEM_TRY(g.proj.alloc(std::max<size_t>(1, 3 * (size_t)g.n_group_dofs)));
    MSFEM_CK(cudaMemsetAsync(h.flag.p, 0, sizeof(int), st));
    if (n_faces > 0)
        k_o2_face_mass<<<n_faces, 128, 0, st>>>(n_faces, g.faces.p, g.vxyz.p, g.cell_dofs.p, h.tet_off.p, h.vols.elems.p,
                                                h.xyz.p, h.bases2.p, g.Ml.p, g.wl.p, h.flag.p);
    if (n_groups > 0)
        k_o2_group_project<<<n_groups, 256, 0, st>>>(g.dof_off.p, g.dofs.p, g.face_off.p, g.faces.p, g.values.p, g.Ml.p,
                                                     g.wl.p, g.m_off.p, g.M.p, g.act.p, g.proj.p, h.flag.p);
    MSFEM_CK(cudaGetLastError());
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, h.flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error(bad == 1   ? "%s: a face quadrature point lies in no tetrahedron of its cell"
                  : bad == 2 ? "%s: a face DOF is not one of its cell's 27 DOFs"
                             : "%s: a group's projection matrix is not positive definite on its rows with mass",
                  who);
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

struct SystemGuard {
    msfem_system_t s = nullptr;
    ~SystemGuard()
    {
        if (s) msfem_system_destroy(s);
    }
};

}  // namespace
}  // namespace msfem

extern "C" {

int msfem_cells_order2_macro_system(msfem_cells_t h, int n_dofs, const int32_t* cell_dofs, msfem_system_t* out)
{
    using namespace msfem;
    if (!h || !out || !h->order2_built) {
        set_error("msfem_cells_order2_macro_system: bad arguments or no Order2 bases built");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    MSFEM_CK(cudaSetDevice(h->device));
    return order2_macro_system(*h, n_dofs, cell_dofs, out);
}

int msfem_cells_order2_dirichlet(msfem_cells_t h, int n_dofs, const int32_t* cell_dofs, int n_vertices,
                                 const double* vertex_xyz, int n_faces, const int32_t* faces, int n_groups,
                                 const int32_t* group_dof_off, const int32_t* group_dofs, const int32_t* group_face_off,
                                 const double* group_values, double* values)
{
    using namespace msfem;
    if (!h || !h->order2_built || (n_groups > 0 && !values)) {
        set_error("msfem_cells_order2_dirichlet: bad arguments or no Order2 bases built");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    O2Groups g;
    MSFEM_TRY(order2_project(*h, n_dofs, cell_dofs, n_vertices, vertex_xyz, n_faces, faces, n_groups, group_dof_off,
                             group_dofs, group_face_off, group_values, g));
    if (g.n_group_dofs > 0) {
        MSFEM_CK(cudaMemcpyAsync(values, g.proj.p, sizeof(double) * 3 * g.n_group_dofs, cudaMemcpyDeviceToHost, h->stream));
        MSFEM_CK(cudaStreamSynchronize(h->stream));
    }
    return MSFEM_OK;
}

int msfem_cells_order2_macro_solve(msfem_cells_t h, int n_dofs, const int32_t* cell_dofs, int n_vertices,
                                   const double* vertex_xyz, int n_faces, const int32_t* faces, int n_groups,
                                   const int32_t* group_dof_off, const int32_t* group_dofs,
                                   const int32_t* group_face_off, const double* group_values, int n_fixed,
                                   const int32_t* fixed_dofs, const int32_t* fixed_src, int precision, double tol,
                                   int maxiter, double* U, int32_t* iterations, double* rel_residual)
{
    using namespace msfem;
    const char* who = "msfem_cells_order2_macro_solve";
    if (!h || !h->order2_built || !U || n_fixed < 0 || (n_fixed > 0 && (!fixed_dofs || !fixed_src)) || !(tol > 0.0) ||
        maxiter <= 0 || (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("%s: bad arguments or no Order2 bases built", who);
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(h->device));
    O2Groups g;
    MSFEM_TRY(order2_project(*h, n_dofs, cell_dofs, n_vertices, vertex_xyz, n_faces, faces, n_groups, group_dof_off,
                             group_dofs, group_face_off, group_values, g));
    for (int i = 0; i < n_fixed; i++)
        if (fixed_dofs[i] < 0 || fixed_dofs[i] >= 3 * n_dofs || fixed_src[i] < 0 || fixed_src[i] >= 3 * g.n_group_dofs) {
            set_error("%s: fixed entry %d names row %d / projected value %d out of range", who, i, fixed_dofs[i],
                      fixed_src[i]);
            return MSFEM_ERR_ARGUMENT;
        }
    SystemGuard sg;
    MSFEM_TRY(order2_macro_system(*h, n_dofs, cell_dofs, &sg.s));
    System& s = *reinterpret_cast<System*>(sg.s);
    // the cells' stream produced the projection; the system's stream takes over after this wait
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    DBuf<int32_t> dd, dsrc;
    DBuf<double> dv;
    if (n_fixed > 0) {
        MSFEM_TRY(upload(s.stream, dd, fixed_dofs, (size_t)n_fixed));
        MSFEM_TRY(upload(s.stream, dsrc, fixed_src, (size_t)n_fixed));
        MSFEM_TRY(dv.alloc((size_t)n_fixed));
        k_o2_gather<<<(n_fixed + 255) / 256, 256, 0, s.stream>>>(n_fixed, dsrc.p, g.proj.p, dv.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_TRY(apply_dirichlet(s, n_fixed, dd.p, dv.p, MSFEM_ROW_AND_COLUMN));
    }
    MSFEM_TRY(msfem_copy_f_to_x(sg.s));
    double rel = 0.0;
    int it = 0;
    const int rc = solve(s, MSFEM_MINRES, precision, 30, maxiter, tol, &rel, &it);
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = rel;
    if (rc < 0) return rc;
    MSFEM_CK(cudaMemcpyAsync(U, s.X.p, sizeof(double) * 3 * (size_t)n_dofs, cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return rc;
}

}  // extern "C"
