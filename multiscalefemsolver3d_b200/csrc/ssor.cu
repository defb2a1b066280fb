// The reference's SSOR preconditioner and its PCG on the GPU (CSSD_Matrix::PrecondorSSOR +
// SolvePrecondorSSOR_SLAE, Library/CSSD_Matrix.h:458-547; MSG_PreconditioningSSOR, :1302-1398),
// and the FEM drivers' restart loop around it (FEM/FEM.h:627-695, :1853-1939).
//
// The reference keeps -w*A_up / -w*A_down and 1/(A_ii w (2-w)) and applies, with z overwritten in
// place,
//   backward:  z_I = (r_I - sum_{j>I} z_j (-w a_Ij)) / a_II          for I = n-1 .. 0
//   scale:     z_I = z_I / ((1 / a_II / w) / (2 - w))
//   forward:   z_I = (z_I - sum_{j<I} z_j (-w a_Ij)) / a_II          for I = 0 .. n-1
// i.e. M = (D - wL) D^-1 (D - wU) / (w (2 - w)): SSOR with the signs of the off-diagonal parts
// flipped.  Each row's sum runs over its columns in ascending order.
//
// On the GPU the two triangular sweeps are level scheduled: a row's level is one more than the
// highest level among the rows it reads (upper neighbours for the backward sweep, lower ones for
// the forward sweep), so all rows of a level run in parallel, one launch per level.  Each row
// repeats the reference's operations in the reference's order, with every product and difference
// rounded separately (no fused multiply-add), so one application gives the reference's bits.
// Elasticity rows are handled per node: DOF 3v + a reads 3v + b (b > a backward, b < a forward)
// from the same thread, so the levels of the node portrait order the 3x3-block matrix too.
//
// The backward sweep keeps its own output (later backward rows read the unscaled z) and writes
// the scaled value into the forward sweep's vector, which the forward sweep then updates in place.
#include <algorithm>
#include <cmath>
#include <vector>

#include "devutil.cuh"
#include "internal.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

constexpr int kSweepThreads = 128;

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// x - z * ((-1 * w) * a), each operation rounded on its own as the reference's C++ computes it
__device__ __forceinline__ double sweep_term(double x, double z, double mw, double a)
{
    return __dsub_rn(x, __dmul_rn(z, __dmul_rn(mw, a)));
}

// z / ((1.0 / diag / w) / (2 - w))
__device__ __forceinline__ double ssor_scale(double z, double diag, double w)
{
    return __ddiv_rn(z, __ddiv_rn(__ddiv_rn(__ddiv_rn(1.0, diag), w), __dsub_rn(2.0, w)));
}

template <int BS>
__global__ void __launch_bounds__(kSweepThreads)
    k_ssor_backward(int count, const int32_t* __restrict__ rows, const int32_t* __restrict__ nrp,
                    const int32_t* __restrict__ ncol, const double* __restrict__ val, double w,
                    const double* __restrict__ r, double* zb, double* __restrict__ zs, const KState* S)
{
    if (S && S->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int v = rows[t];
    const int b = nrp[v], e = nrp[v + 1];
    const double mw = -1.0 * w;
    if (BS == 1) {
        double x = r[v], diag = 0.0;
        for (int p = b; p < e; p++) {
            const int c = ncol[p];
            if (c > v) x = sweep_term(x, zb[c], mw, val[p]);
            else if (c == v) diag = val[p];
        }
        const double z = __ddiv_rn(x, diag);
        zb[v] = z;
        zs[v] = ssor_scale(z, diag, w);
    } else {
        for (int a = 2; a >= 0; a--) {
            const int64_t I = 3 * (int64_t)v + a;
            double x = r[I], diag = 0.0;
            for (int p = b; p < e; p++) {
                const int u = ncol[p];
                if (u < v) continue;
                const double* blk = val + 9 * (int64_t)p + 3 * a;
                for (int c = 0; c < 3; c++) {
                    const int64_t J = 3 * (int64_t)u + c;
                    if (J > I) x = sweep_term(x, zb[J], mw, blk[c]);
                    else if (J == I) diag = blk[c];
                }
            }
            const double z = __ddiv_rn(x, diag);
            zb[I] = z;
            zs[I] = ssor_scale(z, diag, w);
        }
    }
}

template <int BS>
__global__ void __launch_bounds__(kSweepThreads)
    k_ssor_forward(int count, const int32_t* __restrict__ rows, const int32_t* __restrict__ nrp,
                   const int32_t* __restrict__ ncol, const double* __restrict__ val, double w, double* zs,
                   const KState* S)
{
    if (S && S->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int v = rows[t];
    const int b = nrp[v], e = nrp[v + 1];
    const double mw = -1.0 * w;
    if (BS == 1) {
        double x = zs[v], diag = 0.0;
        for (int p = b; p < e; p++) {
            const int c = ncol[p];
            if (c < v) x = sweep_term(x, zs[c], mw, val[p]);
            else if (c == v) diag = val[p];
        }
        zs[v] = __ddiv_rn(x, diag);
    } else {
        for (int a = 0; a < 3; a++) {
            const int64_t I = 3 * (int64_t)v + a;
            double x = zs[I], diag = 0.0;
            for (int p = b; p < e; p++) {
                const int u = ncol[p];
                if (u > v) break;  // columns ascending: nothing further is below the diagonal
                const double* blk = val + 9 * (int64_t)p + 3 * a;
                for (int c = 0; c < 3; c++) {
                    const int64_t J = 3 * (int64_t)u + c;
                    if (J < I) x = sweep_term(x, zs[J], mw, blk[c]);
                    else if (J == I) diag = blk[c];
                }
            }
            zs[I] = __ddiv_rn(x, diag);
        }
    }
}

// ------------------------------------------------------------------ PCG kernels
// The loop of MSG_PreconditioningSSOR (CSSD_Matrix.h:1336-1362): q = A p, alpha = (r, z) / (q, p);
// x += alpha p, r -= alpha q; z = M^-1 r; beta = (r, z)_new / (r, z); p = z + beta p.  The test
// sqrt((r, r) / (F, F)) > E at the loop head becomes "done" right after r is updated; the kernels
// that follow in the same iteration then return at once (x is already final).

__global__ void __launch_bounds__(kVecThreads) k_ss_dot_ff(int n, const double* __restrict__ f, KState* S,
                                                           double* __restrict__ partial)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] += f[i] * f[i];
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[1])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->ff = t[0];
            S->ticket[1] = 0;
        }
    }
}

__global__ void k_ss_limits(KState* S, double tol, int maxiter)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        S->tol2 = tol * tol * S->ff;
        S->maxiter = maxiter;
        S->done = 0;
        S->breakdown = 0;
        S->iter = 0;
    }
}

// p = z, (r, z), (r, r)
__global__ void __launch_bounds__(kVecThreads) k_ss_init(int n, const double* __restrict__ r,
                                                         const double* __restrict__ z, double* __restrict__ p,
                                                         KState* S, double* __restrict__ partial)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double rv = r[i], zv = z[i];
        p[i] = zv;
        acc[0] += rv * zv;
        acc[1] += rv * rv;
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = acc[0];
        partial[gridDim.x + blockIdx.x] = acc[1];
    }
    if (arrive_last(&S->ticket[0])) {
        double t[2];
        reduce_partials<2>(partial, gridDim.x, gridDim.x, t, sh);
        if (threadIdx.x == 0) {
            S->rz = t[0];
            S->rr = t[1];
            S->done = (t[1] <= S->tol2) ? 1 : (S->maxiter <= 0 ? 2 : 0);
            S->ticket[0] = 0;
        }
    }
}

// q = A p, (p, q) -> alpha = (r, z) / (q, p)
template <int BS>
__global__ void __launch_bounds__(256) k_ss_spmv(SellView<double> A, const double* __restrict__ p,
                                                 double* __restrict__ q, KState* S, double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[1] = {0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (BS == 1) {
            const double v = sell_row_scalar<double>(A, warp, lane, p);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                q[row] = v;
                acc[0] += p[row] * v;
            }
        } else {
            double v[3];
            sell_row_block<double>(A, warp, lane, p, v);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    q[3 * (int64_t)brow + c] = v[c];
                    acc[0] += p[3 * (int64_t)brow + c] * v[c];
                }
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->pq = t[0];
            if (t[0] == 0.0 || t[0] != t[0]) {
                S->breakdown = 1;
                S->done = 3;
            }
            S->alpha = S->rz / t[0];
            S->ticket[0] = 0;
        }
    }
}

// x += alpha p, r -= alpha q, (r, r) -> the stopping test
__global__ void __launch_bounds__(kVecThreads) k_ss_xr(int n, double* __restrict__ x, double* __restrict__ r,
                                                       const double* __restrict__ p, const double* __restrict__ q,
                                                       KState* S, double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const double alpha = S->alpha;
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double rv = r[i] - alpha * q[i];
        r[i] = rv;
        acc[0] += rv * rv;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->rr = t[0];
            S->iter += 1;
            if (t[0] <= S->tol2) S->done = 1;
            else if (S->iter >= S->maxiter) S->done = 2;
            else if (t[0] != t[0]) {
                S->breakdown = 1;
                S->done = 3;
            }
            S->ticket[0] = 0;
        }
    }
}

// (r, z) -> beta = (r, z) / rz, rz = (r, z)
__global__ void __launch_bounds__(kVecThreads) k_ss_rz(int n, const double* __restrict__ r,
                                                       const double* __restrict__ z, KState* S,
                                                       double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] += r[i] * z[i];
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->beta = t[0] / S->rz;
            S->rz = t[0];
            S->ticket[0] = 0;
        }
    }
}

__global__ void __launch_bounds__(kVecThreads) k_ss_p(int n, const double* __restrict__ z, double* __restrict__ p,
                                                      const KState* S)
{
    if (S->done) return;
    const double beta = S->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// ------------------------------------------------------------------ reference operation order
// With System::reference_order set, MSFEM_PCG_SSOR repeats the reference's arithmetic operation for
// operation: A x row by row as CSSD_Matrix::MultiplicationMatrixVector (CSSD_Matrix.h:395-423)
// sums it -- the upper entries in ascending column order, then the lower ones, then the diagonal --
// the inner products as math::MakeInnerProduct (Library/Math.h:1633-1654), a serial sum in index
// order, and the vector updates of MSG_PreconditioningSSOR unfused.  The products of an inner
// product are formed in parallel and one thread adds them in order, so its speed is that of a
// serial sum (about 0.1 ms per 30,000 entries): a parity mode, not a production one.

// y = A x in the reference's row order (BS = 3: the expanded scalar rows 3v + a of
// Library/Math.h:1963-2054, whole 3x3 blocks, the in-node entries first among the upper ones and
// last among the lower ones)
template <int BS>
__global__ void __launch_bounds__(kSweepThreads)
    k_ref_spmv(int n_nodes, const int32_t* __restrict__ nrp, const int32_t* __restrict__ ncol,
               const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
               const KState* S)
{
    if (S && S->done) return;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_nodes) return;
    const int b = nrp[v], e = nrp[v + 1];
    int d = b;
    while (d < e && ncol[d] != v) d++;
    if (d == e) {
        // no diagonal slot (the SSOR level build rejects such matrices before this runs)
        if (BS == 1) y[v] = 0.0;
        else for (int a = 0; a < 3; a++) y[3 * (int64_t)v + a] = 0.0;
        return;
    }
    if (BS == 1) {
        double t = 0.0;
        for (int p = d + 1; p < e; p++) t = __dadd_rn(t, __dmul_rn(val[p], x[ncol[p]]));
        for (int p = b; p < d; p++) t = __dadd_rn(t, __dmul_rn(val[p], x[ncol[p]]));
        y[v] = __dadd_rn(t, __dmul_rn(val[d], x[v]));
    } else {
        for (int a = 0; a < 3; a++) {
            const int64_t I = 3 * (int64_t)v + a;
            double t = 0.0;
            const double* dblk = val + 9 * (int64_t)d + 3 * a;
            for (int c = a + 1; c < 3; c++) t = __dadd_rn(t, __dmul_rn(dblk[c], x[3 * (int64_t)v + c]));
            for (int p = d + 1; p < e; p++) {
                const double* blk = val + 9 * (int64_t)p + 3 * a;
                const int64_t J = 3 * (int64_t)ncol[p];
                for (int c = 0; c < 3; c++) t = __dadd_rn(t, __dmul_rn(blk[c], x[J + c]));
            }
            for (int p = b; p < d; p++) {
                const double* blk = val + 9 * (int64_t)p + 3 * a;
                const int64_t J = 3 * (int64_t)ncol[p];
                for (int c = 0; c < 3; c++) t = __dadd_rn(t, __dmul_rn(blk[c], x[J + c]));
            }
            for (int c = 0; c < a; c++) t = __dadd_rn(t, __dmul_rn(dblk[c], x[3 * (int64_t)v + c]));
            y[I] = __dadd_rn(t, __dmul_rn(dblk[a], x[I]));
        }
    }
}

// DOT_FF .. DOT_OUT run whatever the state; DOT_PQ .. DOT_RZ are steps of an iteration
enum RefDot { DOT_FF = 0, DOT_INIT_RZ, DOT_INIT_RR, DOT_RES, DOT_OUT, DOT_PQ, DOT_RR, DOT_RZ };

constexpr int kDotThreads = 256;

// sum_i a_i b_i in index order (one product rounded, then one addition rounded, per entry), then
// the step of the PCG that consumes it; DOT_RES sums (a_i - b_i)^2 (the true residual's numerator),
// DOT_OUT only stores the sum
__global__ void __launch_bounds__(kDotThreads) k_ref_dot(int n, const double* __restrict__ a,
                                                         const double* __restrict__ b, int what, KState* S,
                                                         double* __restrict__ out)
{
    if (S->done && what >= DOT_PQ) return;
    __shared__ double prod[kDotThreads];
    double acc = 0.0;
    for (int base = 0; base < n; base += kDotThreads) {
        const int i = base + threadIdx.x;
        double t = 0.0;
        if (i < n) {
            if (what == DOT_RES) {
                const double dv = __dsub_rn(a[i], b[i]);
                t = __dmul_rn(dv, dv);
            } else {
                t = __dmul_rn(a[i], b[i]);
            }
        }
        prod[threadIdx.x] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            const int m = min(kDotThreads, n - base);
            for (int k = 0; k < m; k++) acc = __dadd_rn(acc, prod[k]);
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    switch (what) {
    case DOT_FF: S->ff = acc; break;
    case DOT_INIT_RZ: S->rz = acc; break;
    case DOT_INIT_RR:
        // the loop head of the first iteration: for (k = 1; k < maxiter && sqrt((r,r)/(F,F)) > E; ...)
        S->rr = acc;
        S->iter = 0;
        S->done = !(sqrt(acc / S->ff) > S->tol2) ? 1 : (S->maxiter <= 0 ? 2 : 0);
        break;
    case DOT_PQ:
        S->pq = acc;
        S->alpha = S->rz / acc;
        break;
    case DOT_RR:
        S->rr = acc;
        S->iter += 1;
        if (!(sqrt(acc / S->ff) > S->tol2)) S->done = 1;
        else if (S->iter >= S->maxiter) S->done = 2;
        break;
    case DOT_RZ:
        S->beta = acc / S->rz;
        S->rz = acc;
        break;
    case DOT_RES:
    case DOT_OUT: *out = acc; break;
    }
}

// x += alpha p, r -= alpha q (each product and sum rounded on its own)
__global__ void __launch_bounds__(kVecThreads) k_ref_xr(int n, double* __restrict__ x, double* __restrict__ r,
                                                        const double* __restrict__ p, const double* __restrict__ q,
                                                        const KState* S)
{
    if (S->done) return;
    const double alpha = S->alpha;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
        r[i] = __dsub_rn(r[i], __dmul_rn(alpha, q[i]));
    }
}

// p = z + beta p
__global__ void __launch_bounds__(kVecThreads) k_ref_p(int n, const double* __restrict__ z, double* __restrict__ p,
                                                       const KState* S)
{
    if (S->done) return;
    const double beta = S->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = __dadd_rn(z[i], __dmul_rn(beta, p[i]));
}

// r = F - t, p = copy later; the initial residual of MSG_PreconditioningSSOR
__global__ void __launch_bounds__(kVecThreads) k_ref_sub(int n, const double* __restrict__ f,
                                                         const double* __restrict__ t, double* __restrict__ r)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = __dsub_rn(f[i], t[i]);
}

__global__ void __launch_bounds__(kVecThreads) k_ref_copy(int n, const double* __restrict__ a, double* __restrict__ b)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void k_ref_limits(KState* S, double tol, int maxiter)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        S->tol2 = tol;  // the reference-order test compares sqrt((r,r)/(F,F)) with E itself
        S->maxiter = maxiter;
        S->done = 0;
        S->iter = 0;
        S->breakdown = 0;
    }
}

// Levels of the two sweeps from the node portrait (host, once per portrait).  Backward: a node's
// level is 1 + the highest level of its higher-numbered neighbours (0 without any); forward: of its
// lower-numbered ones.  Nodes are listed level by level, ascending within a level.
int build_levels(System& s)
{
    if (s.ssor_nnzb == s.nnzb && s.ssor_rows.p) return MSFEM_OK;
    const int nn = s.n_nodes;
    std::vector<int32_t> rp(nn + 1), col((size_t)s.nnzb);
    MSFEM_CK(cudaMemcpyAsync(rp.data(), s.nrp.p, sizeof(int32_t) * (nn + 1), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaMemcpyAsync(col.data(), s.ncol.p, sizeof(int32_t) * s.nnzb, cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    std::vector<int> lb(nn, 0), lf(nn, 0);
    int nb = 0, nf = 0;
    for (int v = nn - 1; v >= 0; v--) {
        int l = -1;
        bool has_diag = false;
        for (int p = rp[v]; p < rp[v + 1]; p++) {
            if (col[p] > v) l = std::max(l, lb[col[p]]);
            if (col[p] == v) has_diag = true;
        }
        if (!has_diag) {
            set_error("SSOR: row %d has no diagonal entry in the portrait", v);
            return MSFEM_ERR_NUMERIC;
        }
        lb[v] = l + 1;
        nb = std::max(nb, lb[v] + 1);
    }
    for (int v = 0; v < nn; v++) {
        int l = -1;
        for (int p = rp[v]; p < rp[v + 1]; p++)
            if (col[p] < v) l = std::max(l, lf[col[p]]);
        lf[v] = l + 1;
        nf = std::max(nf, lf[v] + 1);
    }
    auto group = [&](const std::vector<int>& lev, int nl, std::vector<int>& off, int32_t* out) {
        off.assign(nl + 1, 0);
        for (int v = 0; v < nn; v++) off[lev[v] + 1]++;
        for (int l = 0; l < nl; l++) off[l + 1] += off[l];
        std::vector<int> pos(off.begin(), off.end() - 1);
        for (int v = 0; v < nn; v++) out[pos[lev[v]]++] = v;
    };
    std::vector<int32_t> rows(2 * (size_t)nn);
    group(lb, nb, s.ssor_off_b, rows.data());
    group(lf, nf, s.ssor_off_f, rows.data() + nn);
    MSFEM_TRY(s.ssor_rows.alloc(2 * (size_t)nn));
    MSFEM_CK(cudaMemcpyAsync(s.ssor_rows.p, rows.data(), sizeof(int32_t) * 2 * nn, cudaMemcpyHostToDevice, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    s.ssor_nnzb = s.nnzb;
    return MSFEM_OK;
}

}  // namespace

// z = M^-1 r with the reference's SSOR(w); zb: scratch of n_rows doubles.  With S given, every
// launch returns at once when S->done is set.
int ssor_apply(System& s, const double* r, double* z, double* zb, const KState* S)
{
    MSFEM_TRY(build_levels(s));
    const int nn = s.n_nodes;
    const int32_t* rb = s.ssor_rows.p;
    const int32_t* rf = s.ssor_rows.p + nn;
    const double w = s.ssor_omega;
    for (size_t l = 0; l + 1 < s.ssor_off_b.size(); l++) {
        const int cnt = s.ssor_off_b[l + 1] - s.ssor_off_b[l];
        if (s.bs == 1)
            k_ssor_backward<1><<<grid_for(cnt, kSweepThreads), kSweepThreads, 0, s.stream>>>(
                cnt, rb + s.ssor_off_b[l], s.nrp.p, s.ncol.p, s.val.p, w, r, zb, z, S);
        else
            k_ssor_backward<3><<<grid_for(cnt, kSweepThreads), kSweepThreads, 0, s.stream>>>(
                cnt, rb + s.ssor_off_b[l], s.nrp.p, s.ncol.p, s.val.p, w, r, zb, z, S);
    }
    for (size_t l = 0; l + 1 < s.ssor_off_f.size(); l++) {
        const int cnt = s.ssor_off_f[l + 1] - s.ssor_off_f[l];
        if (s.bs == 1)
            k_ssor_forward<1><<<grid_for(cnt, kSweepThreads), kSweepThreads, 0, s.stream>>>(
                cnt, rf + s.ssor_off_f[l], s.nrp.p, s.ncol.p, s.val.p, w, z, S);
        else
            k_ssor_forward<3><<<grid_for(cnt, kSweepThreads), kSweepThreads, 0, s.stream>>>(
                cnt, rf + s.ssor_off_f[l], s.nrp.p, s.ncol.p, s.val.p, w, z, S);
    }
    MSFEM_CK(cudaGetLastError());
    s.launches += (int)(s.ssor_off_b.size() + s.ssor_off_f.size() - 2);
    return MSFEM_OK;
}

// MSG_PreconditioningSSOR (CSSD_Matrix.h:1302-1398) from the current X: at most maxiter iterations,
// stop when sqrt((r, r) / (F, F)) <= tol on the recurrence residual.  One iteration (SpMV, the two
// sweeps' levels, four vector kernels) is captured once into a CUDA graph and replayed; the host
// reads the state every few iterations (kernels of iterations past the stop return at once).
namespace {
int solve_pcg_ssor_reference(System& s, int maxiter, double tol, int* iters);
}  // namespace

int solve_pcg_ssor(System& s, int maxiter, double tol, int* iters)
{
    if (s.reference_order) return solve_pcg_ssor_reference(s, maxiter, tol, iters);
    MSFEM_TRY(build_levels(s));
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(5 * (size_t)n));
    double* r = s.work64.p;
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    double* zb = q + n;
    double* x = s.X.p;
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    k_ss_dot_ff<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.F.p, S, part);
    MSFEM_TRY(residual64(s, x, s.F.p, r, &S->rr));
    k_ss_limits<<<1, 32, 0, s.stream>>>(S, tol, maxiter);
    MSFEM_CK(cudaGetLastError());
    s.launches += 3;
    MSFEM_TRY(ssor_apply(s, r, z, zb, nullptr));
    k_ss_init<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, z, p, S, part);
    MSFEM_CK(cudaGetLastError());
    s.launches += 1;
    const SellView<double> A = sell_view<double>(s);
    const unsigned g = s.bs == 1 ? spmv_grid_of((const void*)k_ss_spmv<1>, s) : spmv_grid_of((const void*)k_ss_spmv<3>, s);
    const int per_iter = 4 + (int)(s.ssor_off_b.size() + s.ssor_off_f.size() - 2);
    auto iteration = [&]() -> int {
        if (s.bs == 1) k_ss_spmv<1><<<g, 256, 0, s.stream>>>(A, p, q, S, part);
        else k_ss_spmv<3><<<g, 256, 0, s.stream>>>(A, p, q, S, part);
        k_ss_xr<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, x, r, p, q, S, part);
        MSFEM_TRY(ssor_apply(s, r, z, zb, S));
        k_ss_rz<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, z, S, part);
        k_ss_p<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, z, p, S);
        return MSFEM_OK;
    };
    // one graph per iteration shape (vectors, matrix, levels)
    char key[160];
    std::snprintf(key, sizeof(key), "pcg_ssor:%p:%p:%p:%lld:%d", (const void*)x, (const void*)s.val.p,
                  (const void*)A.val, (long long)s.ssor_nnzb, n);
    auto it = s.graphs.find(key);
    if (it == s.graphs.end()) {
        std::array<cudaGraphExec_t, 8> empty{};
        it = s.graphs.emplace(key, empty).first;
    }
    cudaGraphExec_t& exec = it->second[0];
    if (!exec) {
        const int launches_before = s.launches;
        cudaGraph_t graph;
        MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
        const int rc = iteration();
        const cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
        s.launches = launches_before;  // captured, not launched
        if (rc < 0) return rc;
        if (e != cudaSuccess) {
            set_error("SSOR-PCG graph capture failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            set_error("SSOR-PCG graph instantiate failed: %s", cudaGetErrorString(ei));
            return MSFEM_ERR_CUDA;
        }
    }
    int k = 0;
    while (true) {
        MSFEM_TRY(read_state(s));
        if (s.h_kstate->done) break;
        for (int i = 0; i < 4; i++) MSFEM_CK(cudaGraphLaunch(exec, s.stream));
        s.launches += 4 * per_iter;
        k += 4;
        if (k > maxiter + 8) break;  // host-side bound; the device state stops at maxiter
    }
    MSFEM_TRY(read_state(s));
    *iters = s.h_kstate->iter;
    if (s.h_kstate->breakdown) {
        set_error("SSOR-PCG broke down after %d iterations ((p, Ap) = 0 or NaN)", s.h_kstate->iter);
        return MSFEM_ERR_NUMERIC;
    }
    return s.h_kstate->done == 1 ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

namespace {

int ref_spmv(System& s, const double* x, double* y, const KState* S)
{
    if (s.bs == 1)
        k_ref_spmv<1><<<grid_for(s.n_nodes, kSweepThreads), kSweepThreads, 0, s.stream>>>(s.n_nodes, s.nrp.p, s.ncol.p,
                                                                                       s.val.p, x, y, S);
    else
        k_ref_spmv<3><<<grid_for(s.n_nodes, kSweepThreads), kSweepThreads, 0, s.stream>>>(s.n_nodes, s.nrp.p, s.ncol.p,
                                                                                       s.val.p, x, y, S);
    MSFEM_CK(cudaGetLastError());
    s.launches += 1;
    return MSFEM_OK;
}

// MSG_PreconditioningSSOR in the reference's operation order: the iterates are the reference's bits
int solve_pcg_ssor_reference(System& s, int maxiter, double tol, int* iters)
{
    MSFEM_TRY(build_levels(s));
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(5 * (size_t)n));
    double* r = s.work64.p;
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    double* zb = q + n;
    double* x = s.X.p;
    KState* S = s.kstate.p;
    const unsigned gv = kReduceBlocks;
    k_ref_limits<<<1, 32, 0, s.stream>>>(S, tol, maxiter);
    k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, s.F.p, s.F.p, DOT_FF, S, nullptr);
    MSFEM_TRY(ref_spmv(s, x, q, nullptr));
    k_ref_sub<<<gv, kVecThreads, 0, s.stream>>>(n, s.F.p, q, r);
    MSFEM_CK(cudaGetLastError());
    MSFEM_TRY(ssor_apply(s, r, z, zb, nullptr));
    k_ref_copy<<<gv, kVecThreads, 0, s.stream>>>(n, z, p);
    k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, r, z, DOT_INIT_RZ, S, nullptr);
    k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, r, r, DOT_INIT_RR, S, nullptr);
    MSFEM_CK(cudaGetLastError());
    s.launches += 6;
    auto iteration = [&]() -> int {
        MSFEM_TRY(ref_spmv(s, p, q, S));
        k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, q, p, DOT_PQ, S, nullptr);
        k_ref_xr<<<gv, kVecThreads, 0, s.stream>>>(n, x, r, p, q, S);
        k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, r, r, DOT_RR, S, nullptr);
        MSFEM_TRY(ssor_apply(s, r, z, zb, S));
        k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, r, z, DOT_RZ, S, nullptr);
        k_ref_p<<<gv, kVecThreads, 0, s.stream>>>(n, z, p, S);
        return MSFEM_OK;
    };
    const int per_iter = 6 + (int)(s.ssor_off_b.size() + s.ssor_off_f.size() - 2);
    char key[160];
    std::snprintf(key, sizeof(key), "pcg_ssor_ref:%p:%p:%lld:%d", (const void*)x, (const void*)s.val.p,
                  (long long)s.ssor_nnzb, n);
    auto it = s.graphs.find(key);
    if (it == s.graphs.end()) {
        std::array<cudaGraphExec_t, 8> empty{};
        it = s.graphs.emplace(key, empty).first;
    }
    cudaGraphExec_t& exec = it->second[0];
    if (!exec) {
        const int launches_before = s.launches;
        cudaGraph_t graph;
        MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
        const int rc = iteration();
        const cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
        s.launches = launches_before;
        if (rc < 0) return rc;
        if (e != cudaSuccess) {
            set_error("reference-order SSOR-PCG graph capture failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            set_error("reference-order SSOR-PCG graph instantiate failed: %s", cudaGetErrorString(ei));
            return MSFEM_ERR_CUDA;
        }
    }
    int k = 0;
    while (true) {
        MSFEM_TRY(read_state(s));
        if (s.h_kstate->done) break;
        for (int i = 0; i < 4; i++) MSFEM_CK(cudaGraphLaunch(exec, s.stream));
        s.launches += 4 * per_iter;
        k += 4;
        if (k > maxiter + 8) break;
    }
    MSFEM_TRY(read_state(s));
    *iters = s.h_kstate->iter;
    return s.h_kstate->done == 1 ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

}  // namespace

int true_residual_reference(System& s, double* relres)
{
    MSFEM_TRY(build_levels(s));  // also checks that every row has its diagonal slot
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(5 * (size_t)n));
    double* t = s.work64.p + 3 * (size_t)n;
    KState* S = s.kstate.p;
    DBuf<double>& out = s.sc_f64[1];
    MSFEM_TRY(out.alloc(2));
    MSFEM_TRY(ref_spmv(s, s.X.p, t, nullptr));
    // tmp1 += (AX_i - F_i)^2, tmp2 += F_i^2 (CSSD_Matrix.h:1384-1397)
    k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, t, s.F.p, DOT_RES, S, out.p);
    k_ref_dot<<<1, kDotThreads, 0, s.stream>>>(n, s.F.p, s.F.p, DOT_OUT, S, out.p + 1);
    MSFEM_CK(cudaGetLastError());
    s.launches += 2;
    double h[2];
    MSFEM_CK(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    *relres = std::sqrt(h[0] / h[1]);
    return MSFEM_OK;
}

// The drivers' restart loops around a Krylov solve (loop 0: FEM_forBaseEliptic, FEM/FEM.h:627-695;
// loop 1: FEM_forElasticDeformation, FEM/FEM.h:1853-1939), step for step:
//   best_solution = X  [loop 0: then X = F];  current = 1, best = 1e25
//   for (i = 0; i <= MAX_STEPS; i++):                          MAX_STEPS = 5 | 4
//       needed = 10^-(ii + 1)                                  ii starts at 0 | 1
//       [loop 0: only if current > needed] current = |solve(X, maxiter = n, needed)|
//       if current < needed: i = 0, ii++  [loop 0: and stop if current > best + 1e-10]
//       if current <= MIN_RESIDUAL: best = current, stop      (X is NOT copied: that solve is dropped)
//       if current < best: best = current, best_solution = X
//   X = best_solution
int driver_loop(System& s, int loop, int method, int precision, double min_residual, double* best_residual,
                int* n_solves, int* iterations)
{
    if (loop != 0 && loop != 1) {
        set_error("driver loop: loop must be 0 (FEM_forBaseEliptic) or 1 (FEM_forElasticDeformation)");
        return MSFEM_ERR_ARGUMENT;
    }
    const int n = s.n_rows;
    MSFEM_TRY(s.loop_best.alloc((size_t)n));
    double* best = s.loop_best.p;
    MSFEM_CK(cudaMemcpyAsync(best, s.X.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s.stream));
    if (loop == 0) MSFEM_CK(cudaMemcpyAsync(s.X.p, s.F.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s.stream));
    double current = 1.0, best_res = 1e25;
    const int max_steps = loop == 0 ? 5 : 4;
    int ii = loop == 0 ? 0 : 1;
    int solves = 0, its = 0;
    const int maxiter = std::max(1, n - 1);  // for (k = 1; k < maxiter; k++): at most n - 1 iterations
    for (int i = 0; i <= max_steps; i++) {
        const double needed = std::pow(10., -1 * (ii + 1));
        if (loop == 1 || current > needed) {
            double rel = 0.0;
            int it = 0;
            const int rc = solve(s, method, precision, 30, maxiter, needed, &rel, &it);
            if (rc < 0) return rc;
            solves++;
            its += it;
            current = std::fabs(rel);
        }
        if (current < needed) {
            i = 0;
            ii++;
            if (loop == 0 && current > best_res + 1e-10) break;
        }
        if (current <= min_residual) {
            best_res = current;
            break;
        }
        if (current < best_res) {
            best_res = current;
            MSFEM_CK(cudaMemcpyAsync(best, s.X.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s.stream));
        }
    }
    MSFEM_CK(cudaMemcpyAsync(s.X.p, best, sizeof(double) * n, cudaMemcpyDeviceToDevice, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    if (best_residual) *best_residual = best_res;
    if (n_solves) *n_solves = solves;
    if (iterations) *iterations = its;
    return MSFEM_OK;
}

}  // namespace msfem
