// Cracked conduction (scalar Heaviside XFEM) assembled on the GPU into a matrix-only system.
//
// The reference's XFEM is for elasticity only (MultiXFEM/MultiXFEM_Grid.h:1090-2980); this is its
// scalar counterpart (multiscalefemsolver3d_b200/xfem.py states the method).  One thread per
// tetrahedron emits its entries as (row, column, value) triplets: the 16 standard entries
// sigma V grad(phi_i) . grad(phi_j), and on a cut tetrahedron the 48 enriched ones weighted by the
// exact side volumes of the crack plane.  A stable radix sort of the 64-bit keys row * n + col and
// a reduction by key (both CUB, deterministic for a given input) give the CSR matrix, diagonal
// included in every row, which becomes a scalar System without a mesh: Dirichlet rows and every
// solver (GMRES(m) with FP32 Krylov vectors in FP64 refinement included) then apply unchanged.
#include <cub/cub.cuh>

#include <algorithm>
#include <memory>
#include <new>
#include <vector>

#include "element.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

// fraction of the tetrahedron where the linear function with vertex values d is >= 0
__device__ double side_fraction(const double d[4])
{
    int P[4], M[4], np = 0, nm = 0;
    for (int v = 0; v < 4; v++) {
        if (d[v] >= 0.0) P[np++] = v;
        else M[nm++] = v;
    }
    if (np == 0) return 0.0;
    if (np == 4) return 1.0;
    if (np == 1) {
        const int a = P[0];
        double den = 1.0;
        for (int j = 0; j < 3; j++) den *= d[a] - d[M[j]];
        return d[a] * d[a] * d[a] / den;
    }
    if (np == 3) {
        const int b = M[0];
        double den = 1.0;
        for (int j = 0; j < 3; j++) den *= d[P[j]] - d[b];
        return 1.0 - (-d[b]) * (-d[b]) * (-d[b]) / den;
    }
    const double da = d[P[0]], db = d[P[1]], dc = d[M[0]], de = d[M[1]];
    const double p = dc + de, q = dc * de;
    const double num = da * da * db * db - p * da * db * (da + db) + q * (da * da + da * db + db * db);
    return num / ((da - dc) * (da - de) * (db - dc) * (db - de));
}

__global__ void k_xfem_emit(int n_tets, const double* __restrict__ xyz, const int32_t* __restrict__ tets,
                            const double* __restrict__ sigma, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ crack_of, const int32_t* __restrict__ enr,
                            const double* __restrict__ centre, const double* __restrict__ normal, int64_t n_dofs,
                            uint64_t* __restrict__ keys, double* __restrict__ vals)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_tets; e += gridDim.x * blockDim.x) {
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * (int64_t)e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        double Kc[4][4];  // per unit volume
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) Kc[i][j] = sigma[e] * (G.g[i][0] * G.g[j][0] + G.g[i][1] * G.g[j][1] + G.g[i][2] * G.g[j][2]);
        int64_t o = off[e];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++, o++) {
                keys[o] = (uint64_t)v[i] * (uint64_t)n_dofs + (uint64_t)v[j];
                vals[o] = G.vol * Kc[i][j];
            }
        const int k = crack_of[e];
        if (k < 0) continue;
        double d[4], H[4];
        for (int a = 0; a < 4; a++) {
            double s = 0.0;
            for (int c = 0; c < 3; c++) s += (xyz[3 * (int64_t)v[a] + c] - centre[3 * k + c]) * normal[3 * k + c];
            d[a] = s;
            H[a] = s >= 0.0 ? 1.0 : -1.0;
        }
        const double fp = side_fraction(d);
        const double Vp = fp * G.vol, Vm = (1.0 - fp) * G.vol;
        int r[4];
        for (int a = 0; a < 4; a++) r[a] = enr[4 * (int64_t)e + a];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                const double wse = Vp * (1.0 - H[j]) + Vm * (-1.0 - H[j]);
                const double wee = Vp * (1.0 - H[i]) * (1.0 - H[j]) + Vm * (-1.0 - H[i]) * (-1.0 - H[j]);
                keys[o] = (uint64_t)v[i] * (uint64_t)n_dofs + (uint64_t)r[j];      // std(i)-enr(j)
                vals[o++] = wse * Kc[i][j];
                keys[o] = (uint64_t)r[j] * (uint64_t)n_dofs + (uint64_t)v[i];      // enr(j)-std(i)
                vals[o++] = wse * Kc[i][j];
                keys[o] = (uint64_t)r[i] * (uint64_t)n_dofs + (uint64_t)r[j];      // enr(i)-enr(j)
                vals[o++] = wee * Kc[i][j];
            }
    }
}

__global__ void k_xfem_csr(int64_t nnz, int64_t n_dofs, const uint64_t* __restrict__ keys, int32_t* __restrict__ col,
                           int32_t* __restrict__ row_count)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t key = keys[q];
        col[q] = (int32_t)(key % (uint64_t)n_dofs);
        atomicAdd(&row_count[key / (uint64_t)n_dofs], 1);
    }
}

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

}  // namespace
}  // namespace msfem

extern "C" int msfem_xfem_system(int n_nodes, const double* xyz, int n_tets, const int32_t* tets, const double* sigma,
                                 int n_cracks, const double* centre, const double* normal, const int32_t* crack_of_tet,
                                 const int32_t* enr_dof, int n_dofs, msfem_system_t* out)
{
    using namespace msfem;
    if (!out || n_nodes <= 0 || n_tets <= 0 || !xyz || !tets || !sigma || !crack_of_tet || !enr_dof ||
        n_dofs < n_nodes || n_cracks < 0 || (n_cracks > 0 && (!centre || !normal))) {
        set_error("msfem_xfem_system: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    // host checks of every index the kernels use, and the triplet offsets
    std::vector<int64_t> off(n_tets + 1, 0);
    for (int e = 0; e < n_tets; e++) {
        for (int k = 0; k < 4; k++)
            if (tets[4 * (int64_t)e + k] < 0 || tets[4 * (int64_t)e + k] >= n_nodes) {
                set_error("msfem_xfem_system: tetrahedron %d names node %d", e, tets[4 * (int64_t)e + k]);
                return MSFEM_ERR_ARGUMENT;
            }
        const int k = crack_of_tet[e];
        if (k >= n_cracks || k < -1) {
            set_error("msfem_xfem_system: tetrahedron %d names crack %d", e, k);
            return MSFEM_ERR_ARGUMENT;
        }
        if (k >= 0)
            for (int a = 0; a < 4; a++) {
                const int r = enr_dof[4 * (int64_t)e + a];
                if (r < n_nodes || r >= n_dofs) {
                    set_error("msfem_xfem_system: tetrahedron %d has enriched DOF %d outside %d..%d", e, r, n_nodes, n_dofs - 1);
                    return MSFEM_ERR_ARGUMENT;
                }
            }
        off[e + 1] = off[e] + 16 + (k >= 0 ? 48 : 0);
    }
    const int64_t m = off[n_tets];
    if (m >= INT32_MAX || (int64_t)n_dofs * n_dofs < 0) {
        set_error("msfem_xfem_system: %lld triplets exceed the sort's int32 range", (long long)m);
        return MSFEM_ERR_LIMIT;
    }
    std::unique_ptr<System> s(new (std::nothrow) System());
    if (!s) {
        set_error("out of host memory");
        return MSFEM_ERR_LIMIT;
    }
    s->kind = MSFEM_SCALAR;
    s->bs = 1;
    s->n_nodes = n_dofs;
    s->n_tets = 0;
    s->n_rows = n_dofs;
    s->color_off = {0};
    MSFEM_CK(cudaGetDevice(&s->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    MSFEM_CK(cudaEventCreate(&s->ev0));
    MSFEM_CK(cudaEventCreate(&s->ev1));
    cudaStream_t st = s->stream;
    DBuf<double> dxyz, dsig, dcen, dnor;
    DBuf<int32_t> dtets, dcrack, denr;
    DBuf<int64_t> doff;
    auto up = [&](auto& dst, const auto* src, size_t n) -> int {
        MSFEM_TRY(dst.alloc(std::max<size_t>(1, n)));
        if (n) MSFEM_CK(cudaMemcpyAsync(dst.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st));
        return 0;
    };
    MSFEM_TRY(up(dxyz, xyz, 3 * (size_t)n_nodes));
    MSFEM_TRY(up(dtets, tets, 4 * (size_t)n_tets));
    MSFEM_TRY(up(dsig, sigma, (size_t)n_tets));
    MSFEM_TRY(up(dcen, centre, 3 * (size_t)n_cracks));
    MSFEM_TRY(up(dnor, normal, 3 * (size_t)n_cracks));
    MSFEM_TRY(up(dcrack, crack_of_tet, (size_t)n_tets));
    MSFEM_TRY(up(denr, enr_dof, 4 * (size_t)n_tets));
    MSFEM_TRY(up(doff, off.data(), off.size()));
    DBuf<uint64_t> k0, k1;
    DBuf<double> v0, v1;
    MSFEM_TRY(k0.alloc(m));
    MSFEM_TRY(k1.alloc(m));
    MSFEM_TRY(v0.alloc(m));
    MSFEM_TRY(v1.alloc(m));
    k_xfem_emit<<<grid_of(n_tets), 256, 0, st>>>(n_tets, dxyz.p, dtets.p, dsig.p, doff.p, dcrack.p, denr.p, dcen.p, dnor.p,
                                                 (int64_t)n_dofs, k0.p, v0.p);
    MSFEM_CK(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 64 && ((uint64_t)1 << end_bit) < (uint64_t)n_dofs * (uint64_t)n_dofs) end_bit++;
    {
        cub::DoubleBuffer<uint64_t> dk(k0.p, k1.p);
        cub::DoubleBuffer<double> dv(v0.p, v1.p);
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)m, 0, end_bit, st);
        DBuf<unsigned char> tmp;
        MSFEM_TRY(tmp.alloc(tb + 1));
        MSFEM_CK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, dk, dv, (int)m, 0, end_bit, st));
        // reduce by key into the other halves of the double buffers
        uint64_t* ukeys = dk.Alternate();
        double* uvals = dv.Alternate();
        DBuf<int64_t> nruns;
        MSFEM_TRY(nruns.alloc(1));
        size_t tr = 0;
        cub::DeviceReduce::ReduceByKey(nullptr, tr, dk.Current(), ukeys, dv.Current(), uvals, nruns.p, cub::Sum(), (int)m, st);
        DBuf<unsigned char> tmp2;
        MSFEM_TRY(tmp2.alloc(tr + 1));
        MSFEM_CK(cub::DeviceReduce::ReduceByKey(tmp2.p, tr, dk.Current(), ukeys, dv.Current(), uvals, nruns.p, cub::Sum(), (int)m, st));
        int64_t nnz = 0;
        MSFEM_CK(cudaMemcpyAsync(&nnz, nruns.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        if (nnz > INT32_MAX) {
            set_error("msfem_xfem_system: %lld entries exceed the int32 range", (long long)nnz);
            return MSFEM_ERR_LIMIT;
        }
        s->nnzb = nnz;
        MSFEM_TRY(s->ncol.alloc((size_t)nnz));
        MSFEM_TRY(s->val.alloc((size_t)nnz));
        MSFEM_TRY(s->nrp.alloc((size_t)n_dofs + 1));
        DBuf<int32_t> counts;
        MSFEM_TRY(counts.alloc((size_t)n_dofs + 1));
        MSFEM_CK(cudaMemsetAsync(counts.p, 0, sizeof(int32_t) * ((size_t)n_dofs + 1), st));
        k_xfem_csr<<<grid_of(nnz), 256, 0, st>>>(nnz, (int64_t)n_dofs, ukeys, s->ncol.p, counts.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_CK(cudaMemcpyAsync(s->val.p, uvals, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, st));
        size_t ts = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, ts, counts.p, s->nrp.p, n_dofs + 1, st);
        DBuf<unsigned char> tmp3;
        MSFEM_TRY(tmp3.alloc(ts + 1));
        MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp3.p, ts, counts.p, s->nrp.p, n_dofs + 1, st));
    }
    MSFEM_TRY(s->F.alloc((size_t)n_dofs));
    MSFEM_TRY(s->X.alloc((size_t)n_dofs));
    MSFEM_CK(cudaMemsetAsync(s->F.p, 0, sizeof(double) * n_dofs, st));
    MSFEM_CK(cudaMemsetAsync(s->X.p, 0, sizeof(double) * n_dofs, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    *out = reinterpret_cast<msfem_system_t>(s.release());
    return MSFEM_OK;
}
