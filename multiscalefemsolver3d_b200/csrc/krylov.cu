// Krylov solvers on the SELL-32 matrix with device-resident scalars.
//
// Every iteration is a short fixed sequence of kernels; the reductions inside
// them are two-stage and deterministic (each block writes its partial sum, the
// last block to arrive adds the partials in index order and derives the next
// scalar, e.g. alpha = (r,z)/(p,Ap)), so the host never waits inside an
// iteration.  A chunk of iterations is captured once into a CUDA graph and
// replayed; the host reads the solver state only between chunks.  When the
// stopping test fires, the remaining kernels of the chunk return at once.
//
// Stopping test: sqrt((r,r)/(F,F)) <= tol on the recurrence residual, as in
// CSSD_Matrix::MSG / MSG_PreconditioningSSOR (CSSD_Matrix.h:1336, :1524); the
// reported residual is recomputed as ||F - A X|| / ||F|| in FP64 at exit.
#include <cmath>
#include <cstdlib>

#include "devutil.cuh"
#include "internal.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

constexpr int kMaxOuter = 60;

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// ------------------------------------------------------------------ vector kernels

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_dot_self(int n, const VT* __restrict__ a, double* __restrict__ partial,
                                                          unsigned int* ticket, double* out)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)a[i];
        acc[0] += v * v;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(ticket)) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            *out = t[0];
            *ticket = 0;
        }
    }
}

// PCG as in CSSD_Matrix::MSG_PreconditioningSSOR (CSSD_Matrix.h:1336-1362), with M = diag(A)
// (or M = I): three kernels per iteration -- q = A p with (p, q) -> alpha; the x/r/z update with
// (r, z), (r, r) -> beta and the stopping test; p = z + beta p.  Without a preconditioner, and for
// the FP32 solves on the Jacobi-scaled matrix, z is r itself and is never stored.
// z = M^{-1} r, p = z, (r,z), (r,r); sets rz, rr and the initial stopping test
template <class VT, bool JAC>
__global__ void __launch_bounds__(kVecThreads) k_pcg_init(int n, const VT* r, const VT* __restrict__ dinv, VT* z,
                                                          VT* __restrict__ p, KState* S,
                                                          double* __restrict__ partial)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT rv = r[i];
        const VT zv = JAC ? rv * dinv[i] : rv;
        if (JAC) z[i] = zv;  // without a preconditioner z is r itself and is never stored
        p[i] = zv;
        acc[0] += (double)rv * (double)zv;
        acc[1] += (double)rv * (double)rv;
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
            S->rr_min = t[1];
            S->stall = 0;
            S->iter = 0;
            S->breakdown = 0;
            S->done = (t[1] <= S->tol2) ? 1 : 0;
            S->ticket[0] = 0;
        }
    }
}

// q = A p, (p, q) -> alpha = rz / (p, q)
template <class VT>
__global__ void __launch_bounds__(256) k_pcg_spmv(SellView<VT> A, const VT* __restrict__ p, VT* __restrict__ q,
                                                  KState* S, double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[1] = {0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (A.bs == 1) {
            const VT v = sell_row_scalar<VT>(A, warp, lane, p);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                q[row] = v;
                acc[0] += (double)p[row] * (double)v;
            }
        } else {
            VT v[3];
            sell_row_block<VT>(A, warp, lane, p, v);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    q[3 * (int64_t)brow + c] = v[c];
                    acc[0] += (double)p[3 * (int64_t)brow + c] * (double)v[c];
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
                S->done = 1;
            }
            S->alpha = S->rz / t[0];
            S->ticket[0] = 0;
        }
    }
}

// x += alpha p, r -= alpha q, z = M^{-1} r, (r,z), (r,r) -> beta, stopping test
template <class VT, bool JAC>
__global__ void __launch_bounds__(kVecThreads) k_pcg_update(int n, VT* __restrict__ x, VT* r, VT* z,
                                                            const VT* __restrict__ p,
                                                            const VT* __restrict__ q, const VT* __restrict__ dinv,
                                                            KState* S, double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[64];
    const VT alpha = (VT)S->alpha;
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const VT rv = r[i] - alpha * q[i];
        r[i] = rv;
        const VT zv = JAC ? rv * dinv[i] : rv;
        if (JAC) z[i] = zv;
        acc[0] += (double)rv * (double)zv;
        acc[1] += (double)rv * (double)rv;
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
            S->beta = t[0] / S->rz;
            S->rz = t[0];
            S->rr = t[1];
            S->iter += 1;
            if (t[1] < 0.98 * S->rr_min) {
                S->rr_min = t[1];
                S->stall = 0;
            } else {
                S->stall += 1;
            }
            if (t[1] <= S->tol2) S->done = 1;
            else if (S->iter >= S->maxiter) S->done = 2;
            else if (t[1] != t[1]) {
                S->breakdown = 1;
                S->done = 3;
            } else if (S->stall >= S->stall_limit) {
                S->done = 4;  // stagnated at the precision's attainable accuracy
            }
            S->ticket[0] = 0;
        }
    }
}

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_pcg_p(int n, const VT* z, VT* __restrict__ p,
                                                       const KState* S)
{
    if (S->done) return;
    const VT beta = (VT)S->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// ------------------------------------------------------------------ FP32 CG in two kernels
// The FP32 inner solve of the refinement runs CG in the Chronopoulos-Gear arrangement, which needs
// one reduction phase per iteration instead of two:
//   w = A r,  gamma = (r, r),  delta = (w, r)                      (k_cg2_spmv)
//   beta = gamma / gamma_old,  alpha = gamma / (delta - beta gamma / alpha_old)
//   p = r + beta p,  s = w + beta s,  x += alpha p,  r -= alpha s   (k_cg2_update)
// k_cg2_spmv writes per-block partial sums and its last block adds them in a fixed order into
// S->cg2_gd; every block of k_cg2_update forms the step's scalars from those two numbers (so all
// blocks hold the same scalars, bit for bit) and block 0 records the state.  The scalars of the previous iteration live in one of two slots (parity passed by the
// host), so no block reads a value that block 0 overwrites in the same launch.
// Slot layout in KState::mr: [5 * slot + 0] gamma, +1 alpha, +2 iterations, +3 lowest (r, r),
// +4 iterations since (r, r) last set a 2 % low.

__global__ void __launch_bounds__(256) k_cg2_spmv(SellView<float> A, const float* __restrict__ r,
                                                  float* __restrict__ w, const KState* S,
                                                  double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[64];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[2] = {0.0, 0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (A.bs == 1) {
            const float v = sell_row_scalar<float>(A, warp, lane, r);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                w[row] = v;
                const double rv = (double)r[row];
                acc[0] += rv * rv;
                acc[1] += (double)v * rv;
            }
        } else {
            float v[3];
            sell_row_block<float>(A, warp, lane, r, v);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    const int64_t i = 3 * (int64_t)brow + c;
                    w[i] = v[c];
                    const double rv = (double)r[i];
                    acc[0] += rv * rv;
                    acc[1] += (double)v[c] * rv;
                }
        }
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = acc[0];
        partial[gridDim.x + blockIdx.x] = acc[1];
    }
    KState* Sw = const_cast<KState*>(S);
    if (arrive_last(&Sw->ticket[2])) {
        double t[2];
        reduce_partials<2>(partial, gridDim.x, gridDim.x, t, sh);
        if (threadIdx.x == 0) {
            Sw->cg2_gd[0] = t[0];
            Sw->cg2_gd[1] = t[1];
            Sw->ticket[2] = 0;
        }
    }
}

// first = 1: the start (beta = 0, p = r, s = w); slot: the parity of the previous scalars
__global__ void __launch_bounds__(kVecThreads) k_cg2_update(int n, float* __restrict__ x, float* __restrict__ r,
                                                            const float* __restrict__ w, float* __restrict__ p,
                                                            float* __restrict__ s, KState* S,
                                                            const double* __restrict__ partial, int g_spmv, int slot,
                                                            int first)
{
    if (S->done) return;
    __shared__ double sc[4];  // alpha, beta, done
    (void)partial;
    (void)g_spmv;
    if (threadIdx.x == 0) {
        const double gamma = S->cg2_gd[0], delta = S->cg2_gd[1];
        const double* old = S->mr + 5 * slot;
        const int iter = first ? 0 : (int)old[2];
        double rr_min = first ? gamma : old[3];
        int stall = first ? 0 : (int)old[4];
        if (!first) {
            if (gamma < 0.98 * rr_min) {
                rr_min = gamma;
                stall = 0;
            } else {
                stall += 1;
            }
        }
        double beta = first ? 0.0 : gamma / old[0];
        const double den = first ? delta : delta - beta * gamma / old[1];
        const double alpha = gamma / den;
        int done = 0;
        if (gamma <= S->tol2) done = 1;
        else if (iter >= S->maxiter) done = 2;
        else if (!(den != 0.0) || den != den || gamma != gamma) done = 3;  // breakdown
        else if (stall >= S->stall_limit) done = 4;  // FP32 attainable accuracy reached
        sc[0] = alpha;
        sc[1] = beta;
        sc[2] = done;
        if (blockIdx.x == 0) {
            double* nw = S->mr + 5 * (1 - slot);
            nw[0] = gamma;
            nw[1] = alpha;
            nw[2] = done ? iter : iter + 1;
            nw[3] = rr_min;
            nw[4] = stall;
            S->rr = gamma;
            S->iter = done ? iter : iter + 1;
            if (done == 3) S->breakdown = 1;
            if (done) S->done = done;
        }
    }
    __syncthreads();
    if (sc[2] != 0.0) return;
    const float alpha = (float)sc[0], beta = (float)sc[1];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float ri = r[i], wi = w[i];
        const float pi = first ? ri : ri + beta * p[i];
        const float si = first ? wi : wi + beta * s[i];
        p[i] = pi;
        s[i] = si;
        x[i] += alpha * pi;
        r[i] = ri - alpha * si;
    }
}

// generic residual in VT: r = b - A x  (used by the FP32 inner solve with x = 0 -> r = b)
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_copy(int n, const VT* __restrict__ a, VT* __restrict__ b)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

// FP32-IR helpers
// r32 = D^-1/2 r / ||r||  (the scaled system's right-hand side), d32 = 0
__global__ void __launch_bounds__(kVecThreads) k_scale_to32(int n, const double* __restrict__ r, const double* rr,
                                                            const double* __restrict__ dscale, float* __restrict__ r32,
                                                            float* __restrict__ d32)
{
    const double s = 1.0 / sqrt(*rr);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        r32[i] = (float)(r[i] * dscale[i] * s);
        d32[i] = 0.0f;
    }
}

// x += ||r|| D^-1/2 d32  (back from the scaled unknowns)
__global__ void __launch_bounds__(kVecThreads) k_correct(int n, double* __restrict__ x, const float* __restrict__ d32,
                                                         const double* __restrict__ dscale, const double* rr)
{
    const double s = sqrt(*rr);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += s * dscale[i] * (double)d32[i];
}

// ------------------------------------------------------------------ BiCGStab kernels
// Preconditioned BiCGStab (van der Vorst) with M = diag(A):
//   p = r + beta (p - omega v);  y = M^-1 p;  v = A y;  alpha = rho / (rhat, v)
//   s = r - alpha v;  zz = M^-1 s;  t = A zz;  omega = (t, s) / (t, t)
//   x += alpha y + omega zz;  r = s - omega t;  rho' = (rhat, r);  beta = rho'/rho * alpha/omega

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_bcg_p(int n, const VT* __restrict__ r, VT* __restrict__ p,
                                                       const VT* __restrict__ v, VT* __restrict__ y,
                                                       const VT* __restrict__ dinv, const KState* S)
{
    if (S->done) return;
    const VT beta = (VT)S->beta, omega = (VT)S->omega;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT pv = r[i] + beta * (p[i] - omega * v[i]);
        p[i] = pv;
        y[i] = pv * dinv[i];
    }
}

// v = A y, (rhat, v) -> alpha
template <class VT>
__global__ void __launch_bounds__(256) k_bcg_spmv_alpha(SellView<VT> A, const VT* __restrict__ y, VT* __restrict__ v,
                                                        const VT* __restrict__ rhat, KState* S,
                                                        double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double acc[1] = {0.0};
    if (warp < A.n_slices) {
        if (A.bs == 1) {
            const VT t = sell_row_scalar<VT>(A, warp, lane, y);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                v[row] = t;
                acc[0] = (double)rhat[row] * (double)t;
            }
        } else {
            VT t[3];
            sell_row_block<VT>(A, warp, lane, y, t);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    v[3 * (int64_t)brow + c] = t[c];
                    acc[0] += (double)rhat[3 * (int64_t)brow + c] * (double)t[c];
                }
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            if (t[0] == 0.0 || t[0] != t[0]) {
                S->breakdown = 1;
                S->done = 3;
            }
            S->alpha = S->rho_old / t[0];
            S->ticket[0] = 0;
        }
    }
}

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_bcg_s(int n, const VT* __restrict__ r, const VT* __restrict__ v,
                                                       VT* __restrict__ s, VT* __restrict__ zz,
                                                       const VT* __restrict__ dinv, const KState* S)
{
    if (S->done) return;
    const VT alpha = (VT)S->alpha;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT sv = r[i] - alpha * v[i];
        s[i] = sv;
        zz[i] = sv * dinv[i];
    }
}

// t = A zz, (t, s), (t, t) -> omega
template <class VT>
__global__ void __launch_bounds__(256) k_bcg_spmv_omega(SellView<VT> A, const VT* __restrict__ zz, VT* __restrict__ t,
                                                        const VT* __restrict__ s, KState* S,
                                                        double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[64];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double acc[2] = {0.0, 0.0};
    if (warp < A.n_slices) {
        if (A.bs == 1) {
            const VT tv = sell_row_scalar<VT>(A, warp, lane, zz);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                t[row] = tv;
                acc[0] = (double)tv * (double)s[row];
                acc[1] = (double)tv * (double)tv;
            }
        } else {
            VT tv[3];
            sell_row_block<VT>(A, warp, lane, zz, tv);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    t[3 * (int64_t)brow + c] = tv[c];
                    acc[0] += (double)tv[c] * (double)s[3 * (int64_t)brow + c];
                    acc[1] += (double)tv[c] * (double)tv[c];
                }
        }
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = acc[0];
        partial[gridDim.x + blockIdx.x] = acc[1];
    }
    if (arrive_last(&S->ticket[0])) {
        double tt[2];
        reduce_partials<2>(partial, gridDim.x, gridDim.x, tt, sh);
        if (threadIdx.x == 0) {
            S->ts = tt[0];
            S->tt = tt[1];
            S->omega = (tt[1] > 0.0) ? tt[0] / tt[1] : 0.0;
            S->ticket[0] = 0;
        }
    }
}

// x += alpha y + omega zz, r = s - omega t, (rhat, r), (r, r) -> beta, stopping test
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_bcg_update(int n, VT* __restrict__ x, VT* __restrict__ r,
                                                            const VT* __restrict__ y, const VT* __restrict__ zz,
                                                            const VT* __restrict__ s, const VT* __restrict__ t,
                                                            const VT* __restrict__ rhat, KState* S,
                                                            double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[64];
    const VT alpha = (VT)S->alpha, omega = (VT)S->omega;
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * y[i] + omega * zz[i];
        const VT rv = s[i] - omega * t[i];
        r[i] = rv;
        acc[0] += (double)rhat[i] * (double)rv;
        acc[1] += (double)rv * (double)rv;
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = acc[0];
        partial[gridDim.x + blockIdx.x] = acc[1];
    }
    if (arrive_last(&S->ticket[0])) {
        double tt[2];
        reduce_partials<2>(partial, gridDim.x, gridDim.x, tt, sh);
        if (threadIdx.x == 0) {
            const double rho = tt[0];
            S->rr = tt[1];
            S->iter += 1;
            if (S->omega == 0.0 || S->rho_old == 0.0) {
                S->breakdown = 1;
                S->done = 3;
            } else {
                S->beta = (rho / S->rho_old) * (S->alpha / S->omega);
            }
            S->rho_old = rho;
            if (tt[1] <= S->tol2) S->done = 1;
            else if (S->iter >= S->maxiter && !S->done) S->done = 2;
            S->ticket[0] = 0;
        }
    }
}

// r = b - A x (VT) with rhat = r, p = v = 0, (r, r) -> rho_old, rr
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_bcg_init(int n, const VT* __restrict__ r, VT* __restrict__ rhat,
                                                          VT* __restrict__ p, VT* __restrict__ v, KState* S,
                                                          double* __restrict__ partial)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT rv = r[i];
        rhat[i] = rv;
        p[i] = 0;
        v[i] = 0;
        acc[0] += (double)rv * (double)rv;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->rho_old = t[0];
            S->rr = t[0];
            S->beta = 0.0;
            S->omega = 1.0;
            S->alpha = 1.0;
            S->iter = 0;
            S->breakdown = 0;
            S->done = (t[0] <= S->tol2) ? 1 : 0;
            S->ticket[0] = 0;
        }
    }
}

// ------------------------------------------------------------------ host side

struct Timer {
    System& s;
    explicit Timer(System& sys) : s(sys) { cudaEventRecord(s.ev0, s.stream); }
    float stop()
    {
        cudaEventRecord(s.ev1, s.stream);
        cudaEventSynchronize(s.ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, s.ev0, s.ev1);
        return ms;
    }
};

}  // namespace

int ensure_state(System& s)
{
    MSFEM_TRY(ensure_kstate(s));
    if (!s.h_kstate) MSFEM_CK(cudaMallocHost(&s.h_kstate, sizeof(KState)));
    const unsigned g = spmv_grid(s);
    MSFEM_TRY(s.partial.alloc(std::max<size_t>(3 * (size_t)g, 3 * (size_t)kReduceBlocks) + 64));
    return MSFEM_OK;
}

int read_state(System& s)
{
    MSFEM_CK(cudaMemcpyAsync(s.h_kstate, s.kstate.p, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

namespace {

// sets S->ff, S->tol2 (= tol^2 * ff), S->maxiter and the stagnation window on the device
__global__ void k_set_limits(KState* S, double tol, int maxiter, int use_rr_as_ff, int stall_limit)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        if (use_rr_as_ff) S->ff = S->rr;
        S->tol2 = tol * tol * S->ff;
        S->maxiter = maxiter;
        S->stall_limit = stall_limit;
        S->done = 0;
    }
}

// FP32 inner solves stop when (r, r) has not set a new 2 % low for this many iterations: FP32
// CG cannot go below about cond * eps32, and iterating on past that point only adds noise
constexpr int kInnerStall = 200;
constexpr int kNoStall = 0x7fffffff;

// Runs a captured chunk of `per_iter` launches per iteration until the state says done.
template <class F>
int run_chunks(System& s, const std::string& key, F&& enqueue_iteration, int per_iter, int maxiter)
{
    int chunk = 4;
    auto it = s.graphs.find(key);
    if (it == s.graphs.end()) {
        std::array<cudaGraphExec_t, 8> empty{};
        it = s.graphs.emplace(key, empty).first;
    }
    cudaGraphExec_t* exec = it->second.data();
    MSFEM_TRY(read_state(s));
    if (s.h_kstate->done) return MSFEM_OK;
    if (!s.h_ahead) {
        MSFEM_CK(cudaMallocHost(&s.h_ahead, 2 * sizeof(KState)));
        for (auto& e : s.ev_chunk) MSFEM_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int k = 0;
    // one chunk of iterations (4, 8, 16, then 32), then a snapshot of the state behind it
    auto launch = [&](int slot) -> int {
        int ci = 0;
        while ((4 << ci) < chunk) ci++;
        if (!exec[ci]) {
            cudaGraph_t g;
            MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < chunk; i++) enqueue_iteration();
            cudaError_t e = cudaStreamEndCapture(s.stream, &g);
            if (e != cudaSuccess) {
                set_error("graph capture failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
            e = cudaGraphInstantiate(&exec[ci], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                set_error("graph instantiate failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
        }
        MSFEM_CK(cudaGraphLaunch(exec[ci], s.stream));
        MSFEM_CK(cudaMemcpyAsync(s.h_ahead + slot, s.kstate.p, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaEventRecord(s.ev_chunk[slot], s.stream));
        s.launches += chunk * per_iter;
        k += chunk;
        if (chunk < 32) chunk *= 2;
        return MSFEM_OK;
    };
    // the next chunk is always queued before the host waits for the previous one's snapshot, so
    // the GPU does not idle while the host polls; iterations queued past the stop exit at once (every
    // iteration kernel checks the device flag), exactly as the rest of the stopping chunk does
    MSFEM_TRY(launch(0));
    int cur = 0;
    for (;;) {
        const bool more = k <= maxiter + 64;  // the device state also stops at maxiter; a host-side bound
        if (more) MSFEM_TRY(launch(cur ^ 1));
        MSFEM_CK(cudaEventSynchronize(s.ev_chunk[cur]));
        if (s.h_ahead[cur].done || !more) break;
        cur ^= 1;
    }
    return read_state(s);
}

std::string graph_key(const char* tag, std::initializer_list<const void*> ptrs, int n)
{
    std::string k(tag);
    char buf[32];
    for (const void* p : ptrs) {
        std::snprintf(buf, sizeof(buf), ":%p", p);
        k += buf;
    }
    std::snprintf(buf, sizeof(buf), ":%d", n);
    return k + buf;
}

template <class VT>
struct PcgVectors {
    VT *x, *r, *z, *p, *q;  // z == r without a preconditioner
    const VT* dinv;
};

// r holds the initial residual on entry; x is updated in place
template <class VT, bool JAC>
int pcg_run(System& s, PcgVectors<VT> v, int maxiter)
{
    const int n = s.n_rows;
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    k_pcg_init<VT, JAC><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, v.r, v.dinv, v.z, v.p, S, part);
    MSFEM_CK(cudaGetLastError());
    s.launches += 1;
    const SellView<VT> A = sell_view<VT>(s);
    const unsigned g = spmv_grid_of((const void*)k_pcg_spmv<VT>, s);
    auto iteration = [&]() {
        k_pcg_spmv<VT><<<g, 256, 0, s.stream>>>(A, v.p, v.q, S, part);
        k_pcg_update<VT, JAC><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, v.x, v.r, v.z, v.p, v.q, v.dinv, S, part);
        k_pcg_p<VT><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, v.z, v.p, S);
    };
    const std::string key = graph_key(sizeof(VT) == 8 ? (JAC ? "pcg64j" : "pcg64") : (JAC ? "pcg32j" : "pcg32"),
                                      {v.x, v.r, v.z, v.p, v.q, v.dinv, A.val, A.col, (const void*)S, part}, n);
    return run_chunks(s, key, iteration, 3, maxiter);
}

// FP32 CG (Chronopoulos-Gear, two kernels per iteration) on the Jacobi-scaled FP32 matrix from
// x = 0: r holds the right-hand side on entry; S->tol2 / maxiter / stall_limit set by the caller.
// Vectors: x, r, w, p, s (n floats each).
int cg2_run(System& s, float* x, float* r, float* w, float* p, float* sv, int maxiter)
{
    const int n = s.n_rows;
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    const SellView<float> A = sell_view<float>(s);
    const unsigned g = spmv_grid_of((const void*)k_cg2_spmv, s);
    MSFEM_CK(cudaMemsetAsync(x, 0, sizeof(float) * n, s.stream));
    k_cg2_spmv<<<g, 256, 0, s.stream>>>(A, r, w, S, part);
    k_cg2_update<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, x, r, w, p, sv, S, part, (int)g, 1, 1);
    MSFEM_CK(cudaGetLastError());
    s.launches += 2;
    int parity = 0;  // slot of the scalars the next update reads: the first update wrote slot 0
    auto iteration = [&]() {
        k_cg2_spmv<<<g, 256, 0, s.stream>>>(A, r, w, S, part);
        k_cg2_update<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, x, r, w, p, sv, S, part, (int)g, parity, 0);
        parity ^= 1;
    };
    // every captured chunk holds an even number of iterations, so each replay starts on slot 0
    const std::string key = graph_key("cg2_32", {x, r, w, p, sv, A.val, A.col, (const void*)S, part}, n);
    return run_chunks(s, key, iteration, 2, maxiter);
}

int true_residual(System& s, double* relres)
{
    double* r = s.work64.p;
    MSFEM_TRY(residual64(s, s.X.p, s.F.p, r, &s.kstate.p->rr));
    MSFEM_TRY(read_state(s));
    const double rr = s.h_kstate->rr;
    const double ff = s.h_kstate->ff;
    *relres = ff > 0 ? std::sqrt(rr / ff) : std::sqrt(rr);
    return MSFEM_OK;
}

int solve_pcg64(System& s, bool jacobi, int maxiter, double tol, int* iters)
{
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(4 * (size_t)n));
    double* r = s.work64.p;
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    KState* S = s.kstate.p;
    // ff = (F, F); r = F - A X
    k_dot_self<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.F.p, s.partial.p, &S->ticket[1], &S->ff);
    MSFEM_TRY(residual64(s, s.X.p, s.F.p, r, &S->rr));
    k_set_limits<<<1, 32, 0, s.stream>>>(S, tol, maxiter, 0, kNoStall);
    s.launches += 3;
    PcgVectors<double> v{s.X.p, r, jacobi ? z : r, p, q, s.dinv64.p};  // no preconditioner: z is r
    MSFEM_TRY((jacobi ? pcg_run<double, true>(s, v, maxiter) : pcg_run<double, false>(s, v, maxiter)));
    MSFEM_TRY(read_state(s));
    *iters = s.h_kstate->iter;
    return s.h_kstate->done == 1 ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

enum Inner { INNER_CG32 = 0, INNER_MINRES32 = 1, INNER_MINRES64 = 2, INNER_GMRES32 = 3 };

// Iterative refinement around an inner Krylov solve:
//   r = F - A x in FP64;  inner solve of the Jacobi-scaled system (S A S) y = S r to a relative
//   tolerance;  x += S y in FP64.
// INNER_CG32 / INNER_MINRES32: the inner solve runs in FP32 on the FP32 copy of S A S (the right-
// hand side S r / ||r|| is rounded to FP32 and the correction scaled back by ||r||); CG for SPD
// matrices, MINRES for symmetric indefinite ones, GMRES(m) (gmres32_inner) for nonsymmetric ones.
// INNER_MINRES64: FP64 MINRES, whose stopping test
// is on the scaled residual, refined until the true ||F - A x|| / ||F|| meets tol.
int solve_refined(System& s, Inner inner, int maxiter, double tol, int* iters, int* outer, int restart_m = 30)
{
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(4 * (size_t)n));
    double* r64 = s.work64.p;
    float *d32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
    if (inner == INNER_GMRES32 && (restart_m < 1 || restart_m > 1000)) {
        set_error("GMRES restart depth must be in [1, 1000]");
        return MSFEM_ERR_ARGUMENT;
    }
    if (inner != INNER_MINRES64) {
        // GMRES: d, r, then the (m+1) basis vectors and w
        MSFEM_TRY(s.work32.alloc((inner == INNER_GMRES32 ? (size_t)restart_m + 4 : 5) * (size_t)n));
        d32 = s.work32.p;
        r32 = d32 + n;
        p32 = r32 + n;
        q32 = p32 + n;
    }
    KState* S = s.kstate.p;
    DBuf<double>& rr_dev = s.sc_f64[1];
    MSFEM_TRY(rr_dev.alloc(2));
    k_dot_self<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.F.p, s.partial.p, &S->ticket[1], &S->ff);
    s.launches += 1;
    MSFEM_TRY(read_state(s));
    const double ff = s.h_kstate->ff;
    int total_inner = 0;
    int k = 0;
    double prev_rr = -1.0;
    int stalls = 0;
    for (k = 0; k < kMaxOuter; k++) {
        MSFEM_TRY(residual64(s, s.X.p, s.F.p, r64, rr_dev.p));
        s.launches += 1;
        double rr = 0;
        MSFEM_CK(cudaMemcpyAsync(&rr, rr_dev.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        if (!(rr == rr)) {
            set_error("refinement: the residual became NaN");
            return MSFEM_ERR_NUMERIC;
        }
        if (rr <= tol * tol * ff || rr == 0.0) break;
        if (total_inner >= maxiter) break;
        if (prev_rr >= 0 && rr > 0.25 * prev_rr) {
            if (++stalls >= 3) break;  // refinement no longer contracts
        }
        prev_rr = rr;
        const double need = tol * std::sqrt(ff / rr);  // the reduction still missing
        int it = 0, rc = MSFEM_OK;
        double tau;
        if (inner == INNER_MINRES64) {
            tau = std::max(1e-14, std::min(0.5, 0.5 * need));
            rc = minres_run<double, true>(s, s.X.p, r64, maxiter - total_inner, tau, 0, &it);
            s.launches += 0;
        } else {
            // inner tolerance: what FP32 reaches comfortably (CG, whose stall test stops it at FP32's
            // attainable accuracy: 1e-5, a deeper first pass saving a restart of the Krylov space;
            // GMRES 1e-4), or just what is still missing
            tau = std::max(inner == INNER_CG32 ? 1e-5 : 1e-4, std::min(0.5, 0.3 * need));
            k_scale_to32<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r64, rr_dev.p, s.dscale.p, r32, d32);
            s.launches += 1;
            if (inner == INNER_CG32) {
                k_dot_self<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r32, s.partial.p, &S->ticket[1], &S->rr);
                k_set_limits<<<1, 32, 0, s.stream>>>(S, tau, maxiter - total_inner, 1, kInnerStall);
                s.launches += 2;
                // d = x (from 0), r32 = the scaled right-hand side, then w, p, s
                MSFEM_TRY(cg2_run(s, d32, r32, p32, q32, q32 + n, maxiter - total_inner));
                MSFEM_TRY(read_state(s));
                it = s.h_kstate->iter;
                if (s.h_kstate->breakdown) rc = MSFEM_ERR_NUMERIC;
            } else if (inner == INNER_GMRES32) {
                float* V = r32 + n;
                rc = gmres32_inner(s, restart_m, d32, r32, V, V + (size_t)(restart_m + 1) * n, maxiter - total_inner, tau,
                                   &it);
            } else {
                rc = minres_run<float, false>(s, d32, r32, maxiter - total_inner, tau, 0, &it);
            }
        }
        total_inner += it;
        if (std::getenv("MSFEM_TRACE")) {
            read_state(s);
            std::fprintf(stderr, "[msfem] refine %d (inner %d): rel %.3e tau %.1e inner iters %d rc %d (done %d rr %.3e)\n",
                         k, (int)inner, std::sqrt(rr / ff), tau, it, rc, s.h_kstate->done, s.h_kstate->rr);
        }
        if (rc == MSFEM_ERR_NUMERIC) {
            // the inner solve broke down: keep x as it is and stop
            set_error("refinement: inner solve broke down after %d iterations", it);
            break;
        }
        if (rc < 0) return rc;
        if (inner != INNER_MINRES64) {
            k_correct<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.X.p, d32, s.dscale.p, rr_dev.p);
            s.launches += 1;
        }
    }
    // the final residual report uses (F, F)
    k_dot_self<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.F.p, s.partial.p, &S->ticket[1], &S->ff);
    s.launches += 1;
    *iters = total_inner;
    *outer = k;
    return MSFEM_OK;
}

int solve_bicgstab64(System& s, int maxiter, double tol, int* iters)
{
    const int n = s.n_rows;
    MSFEM_TRY(s.work64.alloc(9 * (size_t)n));
    double* r = s.work64.p;
    double* rhat = r + n;
    double* p = rhat + n;
    double* v = p + n;
    double* y = v + n;
    double* sv = y + n;
    double* zz = sv + n;
    double* t = zz + n;
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    k_dot_self<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.F.p, part, &S->ticket[1], &S->ff);
    MSFEM_TRY(residual64(s, s.X.p, s.F.p, r, &S->rr));
    k_set_limits<<<1, 32, 0, s.stream>>>(S, tol, maxiter, 0, kNoStall);
    k_bcg_init<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, rhat, p, v, S, part);
    MSFEM_CK(cudaGetLastError());
    s.launches += 4;
    const SellView<double> A = sell_view<double>(s);
    const unsigned g = spmv_grid(s);
    const double* dinv = s.dinv64.p;
    double* x = s.X.p;
    auto iteration = [&]() {
        k_bcg_p<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, p, v, y, dinv, S);
        k_bcg_spmv_alpha<double><<<g, 256, 0, s.stream>>>(A, y, v, rhat, S, part);
        k_bcg_s<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, v, sv, zz, dinv, S);
        k_bcg_spmv_omega<double><<<g, 256, 0, s.stream>>>(A, zz, t, sv, S, part);
        k_bcg_update<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, x, r, y, zz, sv, t, rhat, S, part);
    };
    const std::string key = graph_key("bicgstab64", {x, r, rhat, p, v, y, sv, zz, t, dinv, A.val, (const void*)S, part}, n);
    MSFEM_TRY(run_chunks(s, key, iteration, 5, maxiter));
    MSFEM_TRY(read_state(s));
    *iters = s.h_kstate->iter;
    return s.h_kstate->done == 1 ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

}  // namespace

int solve_gmres64(System& s, int m, int maxiter, double tol, int* iters, int* restarts);  // gmres.cu

int solve(System& s, int method, int precision, int restart_m, int maxiter, double tol, double* relres, int* iters)
{
    if (maxiter <= 0 || !(tol >= 0)) {
        set_error("solve: maxiter must be > 0 and tol >= 0");
        return MSFEM_ERR_ARGUMENT;
    }
    if (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR &&
        !(precision == MSFEM_FP64_REFERENCE && method == MSFEM_PCG_SSOR)) {
        set_error("solve: precision %d is not available for method %d (MSFEM_FP64_REFERENCE is for MSFEM_PCG_SSOR)",
                  precision, method);
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(prepare_sell(s));
    MSFEM_TRY(ensure_state(s));
    s.launches = 0;
    Timer timer(s);
    int it = 0, outer = 0;
    int rc = MSFEM_OK;
    const bool jac = method != MSFEM_CG;
    if (method != MSFEM_CG && s.zero_diag) {
        set_error("solve: the matrix has a zero diagonal entry; Jacobi preconditioning is undefined (use MSFEM_CG)");
        return MSFEM_ERR_NUMERIC;
    }
    switch (method) {
    case MSFEM_CG:
    case MSFEM_PCG_JACOBI:
        if (precision == MSFEM_FP64) {
            rc = solve_pcg64(s, jac, maxiter, tol, &it);
        } else if (precision == MSFEM_FP32_IR && jac) {
            rc = solve_refined(s, INNER_CG32, maxiter, tol, &it, &outer);
        } else {
            set_error("solve: FP32 iterative refinement uses a Jacobi-preconditioned inner solver; "
                      "use MSFEM_PCG_JACOBI or MSFEM_MINRES (precision %d)", precision);
            return MSFEM_ERR_ARGUMENT;
        }
        break;
    case MSFEM_MINRES:
        if (s.zero_diag) {
            set_error("solve: MINRES runs on the Jacobi-scaled matrix; a zero diagonal entry makes it undefined");
            return MSFEM_ERR_NUMERIC;
        }
        rc = solve_refined(s, precision == MSFEM_FP32_IR ? INNER_MINRES32 : INNER_MINRES64, maxiter, tol, &it, &outer);
        break;
    case MSFEM_BICGSTAB:
        rc = solve_bicgstab64(s, maxiter, tol, &it);
        break;
    case MSFEM_PCG_SSOR:
        if (precision != MSFEM_FP64 && precision != MSFEM_FP64_REFERENCE) {
            set_error("solve: the reference's SSOR-PCG runs in FP64 (precision %d)", precision);
            return MSFEM_ERR_ARGUMENT;
        }
        s.reference_order = precision == MSFEM_FP64_REFERENCE;
        rc = solve_pcg_ssor(s, maxiter, tol, &it);
        break;
    case MSFEM_GMRES:
        if (precision == MSFEM_FP32_IR)
            rc = solve_refined(s, INNER_GMRES32, maxiter, tol, &it, &outer, restart_m > 0 ? restart_m : 30);
        else
            rc = solve_gmres64(s, restart_m > 0 ? restart_m : 30, maxiter, tol, &it, &outer);
        break;
    default:
        rc = MSFEM_ERR_ARGUMENT;
    }
    if (rc == MSFEM_ERR_ARGUMENT) set_error("solve: unknown method %d / precision %d", method, precision);
    if (rc < 0) return rc;
    double rel = 0;
    if (method == MSFEM_PCG_SSOR && precision == MSFEM_FP64_REFERENCE) MSFEM_TRY(true_residual_reference(s, &rel));
    else MSFEM_TRY(true_residual(s, &rel));
    s.launches += 1;
    s.stats.ms_solve = timer.stop();
    s.stats.iterations = it;
    s.stats.outer_iterations = outer;
    s.stats.rel_residual = rel;
    s.stats.kernel_launches = s.launches;
    s.total_launches += s.launches;
    if (relres) *relres = rel;
    if (iters) *iters = it;
    if ((precision == MSFEM_FP32_IR || method == MSFEM_MINRES) && rc == MSFEM_OK && !(rel <= tol * (1.0 + 1e-6)))
        rc = MSFEM_NOT_CONVERGED;
    return rc;
}

}  // namespace msfem
