// Dirichlet conditions with the reference's semantics.
//
// Rows (FEM/FEM.h:1697-1714 elasticity, :506-530 scalar): X = F = value, the
// diagonal becomes 1 and every off-diagonal entry of the row 0; when a DOF is
// listed twice the later value wins, as in the reference's sequential loop.
//
// Columns (FEM/FEM.h:1757-1812, :565-607): for every row the reference walks the
// row's A_up columns ascending with ONE pointer into the boundary list that only
// moves forward: for column c it advances while the entry is smaller than c and
// stops at the first entry >= c (a hit when equal: F_row -= a * F_c, a = 0).  The
// pointer is reset once for the A_down columns.  For a sorted list this is a
// plain membership test; for an unsorted list (e.g. two boundary "types" listed
// one after the other) some columns are never reached and stay in the matrix.
// The GPU reproduces the walk exactly: "first index >= p whose entry is >= c" is
// answered in O(log L) from a range-maximum sparse table over the list, so each
// row costs O(row length * log L) instead of the reference's O(L).
#include <cub/cub.cuh>

#include "devutil.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

__global__ void k_check_dofs(int L, const int32_t* __restrict__ dofs, int n_rows, int* bad)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    int d = dofs[i];
    if (d < 0 || d >= n_rows) atomicExch(bad, 1);
}

__global__ void k_iota(int n, int32_t* a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// sorted (dof, original position) pairs: the last occurrence of each DOF applies the row
__global__ void k_dirichlet_rows(int L, const int32_t* __restrict__ sdof, const int32_t* __restrict__ spos,
                                 const double* __restrict__ values, int bs, const int32_t* __restrict__ nrp,
                                 const int32_t* __restrict__ ncol, double* __restrict__ val, double* __restrict__ F,
                                 double* __restrict__ X, const int* bad)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L || *bad) return;
    const int d = sdof[i];
    if (i + 1 < L && sdof[i + 1] == d) return;
    const double v = values[spos[i]];
    X[d] = v;
    F[d] = v;
    if (bs == 1) {
        for (int p = nrp[d]; p < nrp[d + 1]; p++) val[p] = (ncol[p] == d) ? 1.0 : 0.0;
    } else {
        const int node = d / 3, a = d - 3 * node;
        for (int p = nrp[node]; p < nrp[node + 1]; p++) {
            const bool own = ncol[p] == node;
            double* blk = val + 9 * (int64_t)p + 3 * a;
            blk[0] = (own && a == 0) ? 1.0 : 0.0;
            blk[1] = (own && a == 1) ? 1.0 : 0.0;
            blk[2] = (own && a == 2) ? 1.0 : 0.0;
        }
    }
}

// per node Dirichlet bits for the matrix-free operators (kuhn.cu): bit a row, bit 3+a column
__global__ void k_dirichlet_mask(int L, const int32_t* __restrict__ dofs, int bs, int columns, uint32_t* __restrict__ mask,
                                 const int* bad)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L || *bad) return;
    const int d = dofs[i];
    const int node = d / bs, a = d - bs * node;
    atomicOr(mask + node, (1u << a) | (columns ? (1u << (3 + a)) : 0u));
}

__global__ void k_sparse_level(int L, int half, const int32_t* __restrict__ prev, int32_t* __restrict__ cur)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    int a = prev[i];
    int b = (i + half < L) ? prev[i + half] : a;
    cur[i] = a > b ? a : b;
}

// first index >= p whose list entry is >= c (L when there is none)
__device__ __forceinline__ int first_geq(const int32_t* __restrict__ st, int L, int T, int p, int c)
{
    if (p >= L) return L;
    for (int t = T; t >= 0; t--) {
        const int len = 1 << t;
        if (p + len <= L && __ldg(st + (int64_t)t * L + p) < c) p += len;
    }
    return p;
}

struct Walk {
    const int32_t* st;
    const int32_t* u;
    int L, T, p;
    __device__ __forceinline__ bool hit(int c)
    {
        p = first_geq(st, L, T, p, c);
        return p < L && __ldg(u + p) == c;
    }
};

__device__ __forceinline__ void eliminate(double* __restrict__ a, double& f, const double* __restrict__ F, int c)
{
    const double v = *a;
    if (v != 0.0) f = __dsub_rn(f, __dmul_rn(v, F[c]));
    *a = 0.0;
}

__global__ void k_column_sweep(int n_rows, int bs, const int32_t* __restrict__ nrp, const int32_t* __restrict__ ncol,
                               double* __restrict__ val, double* __restrict__ F, const int32_t* __restrict__ u,
                               const int32_t* __restrict__ st, int L, int T, const int* bad)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows || *bad) return;
    double f = F[r];
    const double f0 = f;
    Walk w{st, u, L, T, 0};
    if (bs == 1) {
        const int rb = nrp[r], re = nrp[r + 1];
        int pd = rb;
        while (pd < re && ncol[pd] < r) pd++;
        for (int k = pd + 1; k < re; k++) {  // A_up, ascending
            const int c = ncol[k];
            if (w.hit(c)) eliminate(val + k, f, F, c);
        }
        w.p = 0;
        for (int k = rb; k < pd; k++) {  // A_down, ascending
            const int c = ncol[k];
            if (w.hit(c)) eliminate(val + k, f, F, c);
        }
    } else {
        const int node = r / 3, a = r - 3 * node;
        const int rb = nrp[node], re = nrp[node + 1];
        for (int k = rb; k < re; k++) {  // A_up: expanded columns > r, ascending
            const int j = ncol[k];
            for (int b = 0; b < 3; b++) {
                const int c = 3 * j + b;
                if (c <= r) continue;
                if (w.hit(c)) eliminate(val + 9 * (int64_t)k + 3 * a + b, f, F, c);
            }
        }
        w.p = 0;
        for (int k = rb; k < re; k++) {  // A_down: expanded columns < r, ascending
            const int j = ncol[k];
            for (int b = 0; b < 3; b++) {
                const int c = 3 * j + b;
                if (c >= r) continue;
                if (w.hit(c)) eliminate(val + 9 * (int64_t)k + 3 * a + b, f, F, c);
            }
        }
    }
    if (f != f0) F[r] = f;
}

}  // namespace

int apply_dirichlet(System& s, int L, const int32_t* d_dofs, const double* d_values, int mode)
{
    if (L <= 0) return MSFEM_OK;
    if (mode != MSFEM_ROW_ONLY && mode != MSFEM_ROW_AND_COLUMN) {
        set_error("apply_dirichlet: unknown mode %d", mode);
        return MSFEM_ERR_ARGUMENT;
    }
    cudaStream_t st = s.stream;
    // scratch: sc_i32[0] may hold the caller's DOF list, so [1..4] are used here
    DBuf<int>& bad = s.flag;
    DBuf<int32_t>&pos = s.sc_i32[1], &sdof = s.sc_i32[2], &spos = s.sc_i32[3], &table = s.sc_i32[4];
    MSFEM_TRY(bad.alloc(8));
    MSFEM_TRY(pos.alloc(L));
    MSFEM_TRY(sdof.alloc(L));
    MSFEM_TRY(spos.alloc(L));
    int T = 0;
    while ((2 << T) <= L) T++;  // sparse-table levels 0..T, 2^T <= L
    if (mode == MSFEM_ROW_AND_COLUMN) MSFEM_TRY(table.alloc((size_t)(T + 1) * L));
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_dofs, sdof.p, pos.p, spos.p, L, 0, 32, st);
    MSFEM_TRY(s.sc_tmp.alloc(tmp_bytes + 1));

    MSFEM_CK(cudaEventRecord(s.ev0, st));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    // every kernel below that indexes by a DOF first reads this flag and does nothing if it is set
    k_check_dofs<<<grid_for(L, 256), 256, 0, st>>>(L, d_dofs, s.n_rows, bad.p);
    k_iota<<<grid_for(L, 256), 256, 0, st>>>(L, pos.p);
    MSFEM_CK(cub::DeviceRadixSort::SortPairs(s.sc_tmp.p, tmp_bytes, d_dofs, sdof.p, pos.p, spos.p, L, 0, 32, st));
    k_dirichlet_rows<<<grid_for(L, 128), 128, 0, st>>>(L, sdof.p, spos.p, d_values, s.bs, s.nrp.p, s.ncol.p, s.val.p,
                                                       s.F.p, s.X.p, bad.p);
    if (!s.dmask.p) {
        MSFEM_TRY(s.dmask.alloc((size_t)s.n_nodes + 4));  // 4 words of slack: staging copies
        MSFEM_CK(cudaMemsetAsync(s.dmask.p, 0, sizeof(uint32_t) * s.dmask.n, st));
    }
    k_dirichlet_mask<<<grid_for(L, 256), 256, 0, st>>>(L, d_dofs, s.bs, mode == MSFEM_ROW_AND_COLUMN, s.dmask.p,
                                                       bad.p);
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 4;  // check, iota, rows, mask (the radix sort's own kernels are not counted)
    if (mode == MSFEM_ROW_AND_COLUMN) {
        MSFEM_CK(cudaMemcpyAsync(table.p, d_dofs, sizeof(int32_t) * L, cudaMemcpyDeviceToDevice, st));
        for (int t = 1; t <= T; t++)
            k_sparse_level<<<grid_for(L, 256), 256, 0, st>>>(L, 1 << (t - 1), table.p + (size_t)(t - 1) * L,
                                                             table.p + (size_t)t * L);
        k_column_sweep<<<grid_for(s.n_rows, 128), 128, 0, st>>>(s.n_rows, s.bs, s.nrp.p, s.ncol.p, s.val.p, s.F.p,
                                                                d_dofs, table.p, L, T, bad.p);
        MSFEM_CK(cudaGetLastError());
        s.total_launches += T + 1;
    }
    int h_bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaEventRecord(s.ev1, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (h_bad) {
        set_error("a Dirichlet DOF is outside [0, %d); the system is unchanged", s.n_rows);
        return MSFEM_ERR_ARGUMENT;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, s.ev0, s.ev1);
    s.stats.ms_dirichlet = ms;
    s.invalidate_values();
    return MSFEM_OK;
}

}  // namespace msfem
