// Restarted GMRES(m) on the GPU, right-preconditioned by diag(A).
//
// The reference's compiled GMRES (CSSD_Matrix.h:1774-1989) has no caller and a
// fixed depth of 5; its legacy GMRS (Library/GMRES/7_gmres.for:95-222) is a
// restarted GMRES(M) with Givens rotations and a back substitution.  This is
// that method laid out for the GPU:
//   * Arnoldi with classical Gram-Schmidt applied twice (CGS2): the j+1
//     projections of a step are computed together by one multi-dot kernel and
//     removed by one update kernel, instead of 2(j+1) dependent passes;
//   * the Hessenberg column, its Givens rotations and the residual estimate
//     |g_{j+1}| are updated on the device by a one-thread kernel, so a whole
//     restart cycle (m steps) is one captured CUDA graph with no host wait;
//   * x += M^-1 V y is one fused pass after the cycle.
// Stopping test: |g_{j+1}| <= tol * ||F|| (the true residual norm in exact
// arithmetic for right preconditioning).
#include <cmath>

#include "devutil.cuh"
#include "internal.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

// layout of the small dense GMRES data in System::gm (doubles)
struct GmLayout {
    int m;
    __host__ __device__ size_t H() const { return 0; }                           // (m+1) x m, row-major H[i*m + j]
    __host__ __device__ size_t cs() const { return (size_t)(m + 1) * m; }        // m
    __host__ __device__ size_t sn() const { return cs() + m; }                   // m
    __host__ __device__ size_t g() const { return sn() + m; }                    // m+1
    __host__ __device__ size_t y() const { return g() + m + 1; }                 // m
    __host__ __device__ size_t h1() const { return y() + m; }                    // m+1 (first projection)
    __host__ __device__ size_t h2() const { return h1() + m + 1; }               // m+1 (second projection)
    __host__ __device__ size_t misc() const { return h2() + m + 1; }             // [0] steps done this cycle, [1] converged, [2] |g|
    __host__ __device__ size_t total() const { return misc() + 8; }
};

// V0 = r / ||r|| (r and V0 may be the same vector), g = (||r||, 0, ...)
template <class VT>
__global__ void k_gm_start(int n, const VT* r, VT* V0, double* gm, GmLayout L,
                           const KState* S)
{
    const double beta = sqrt(S->rr);
    const double inv = beta > 0 ? 1.0 / beta : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        V0[i] = (VT)((double)r[i] * inv);
    if (blockIdx.x == 0) {
        for (int i = threadIdx.x; i < L.m + 1; i += blockDim.x) gm[L.g() + i] = (i == 0) ? beta : 0.0;
        if (threadIdx.x == 0) {
            gm[L.misc()] = 0.0;
            gm[L.misc() + 1] = 0.0;
            gm[L.misc() + 2] = beta;
        }
    }
}

// z = M^-1 v (dinv == nullptr: the matrix is already Jacobi-scaled, z = v)
template <class VT>
__global__ void k_gm_prec(int n, const VT* __restrict__ v, const double* __restrict__ dinv, VT* __restrict__ z,
                          const double* gm, GmLayout L)
{
    if (gm[L.misc() + 1] != 0.0) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = dinv ? (VT)((double)v[i] * dinv[i]) : v[i];
}

template <class VT>
__global__ void __launch_bounds__(256) k_gm_spmv(SellView<VT> A, const VT* __restrict__ z, VT* __restrict__ w,
                                                 const double* gm, GmLayout L)
{
    if (gm[L.misc() + 1] != 0.0) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= A.n_slices) return;
    if (A.bs == 1) {
        const VT v = sell_row_scalar<VT>(A, warp, lane, z);
        const int row = warp * kSlice + lane;
        if (row < A.n_rows) w[row] = v;
    } else {
        VT v[3];
        sell_row_block<VT>(A, warp, lane, z, v);
        const int brow = warp * kSlice + lane;
        if (brow < A.n_brows)
            for (int c = 0; c < 3; c++) w[3 * (int64_t)brow + c] = v[c];
    }
}

// h[i] = (V_i, w), i = 0..j (FP64 accumulation for either vector type)
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_gm_multidot(int n, const VT* __restrict__ V, int j,
                                                             const VT* __restrict__ w, double* __restrict__ partial,
                                                             unsigned int* ticket, double* gm, GmLayout L, size_t hoff)
{
    if (gm[L.misc() + 1] != 0.0) return;
    __shared__ double sh[32];
    for (int i = 0; i <= j; i++) {
        const VT* vi = V + (size_t)i * n;
        double acc[1] = {0.0};
        for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
            acc[0] += (double)vi[r] * (double)w[r];
        block_sum<1>(acc, sh);
        if (threadIdx.x == 0) partial[(size_t)i * gridDim.x + blockIdx.x] = acc[0];
    }
    if (arrive_last(ticket)) {
        for (int i = 0; i <= j; i++) {
            double t[1];
            reduce_partials<1>(partial + (size_t)i * gridDim.x, gridDim.x, 0, t, sh);
            if (threadIdx.x == 0) gm[hoff + i] = t[0];
        }
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// w -= sum_i h[i] V_i ; with LAST, also (w, w) -> the new subdiagonal entry, and H[:, j] = h1 + h2
template <class VT, bool LAST>
__global__ void __launch_bounds__(kVecThreads) k_gm_orth(int n, const VT* __restrict__ V, int j,
                                                         VT* __restrict__ w, double* __restrict__ partial,
                                                         unsigned int* ticket, double* gm, GmLayout L, size_t hoff)
{
    if (gm[L.misc() + 1] != 0.0) return;
    __shared__ double sh[32];
    __shared__ double hs[1024];
    for (int i = threadIdx.x; i <= j; i += blockDim.x) hs[i] = gm[hoff + i];
    __syncthreads();
    double acc[1] = {0.0};
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double t = (double)w[r];
        for (int i = 0; i <= j; i++) t -= hs[i] * (double)V[(size_t)i * n + r];
        w[r] = (VT)t;
        const double tv = (double)w[r];
        acc[0] += tv * tv;
    }
    if (!LAST) return;
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(ticket)) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            const int m = L.m;
            for (int i = 0; i <= j; i++) gm[L.H() + (size_t)i * m + j] = gm[L.h1() + i] + gm[L.h2() + i];
            gm[L.H() + (size_t)(j + 1) * m + j] = sqrt(t[0]);
            *ticket = 0;
        }
    }
}

// Givens update of column j, residual estimate and stopping test (one thread).
__global__ void k_gm_givens(int j, double* gm, GmLayout L, KState* S)
{
    if (gm[L.misc() + 1] != 0.0) return;
    const int m = L.m;
    double* H = gm + L.H();
    double* cs = gm + L.cs();
    double* sn = gm + L.sn();
    double* g = gm + L.g();
    const double hn = H[(size_t)(j + 1) * m + j];
    for (int i = 0; i < j; i++) {
        const double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
    }
    const double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
    const double d = sqrt(a * a + b * b);
    const double c = d > 0 ? a / d : 1.0, s = d > 0 ? b / d : 0.0;
    cs[j] = c;
    sn[j] = s;
    H[(size_t)j * m + j] = d;
    H[(size_t)(j + 1) * m + j] = 0.0;
    g[j + 1] = -s * g[j];
    g[j] = c * g[j];
    const double res = fabs(g[j + 1]);
    gm[L.misc()] = j + 1;
    gm[L.misc() + 2] = res;
    S->iter += 1;
    S->rr = res * res;
    if (res * res <= S->tol2 || !(res == res)) {
        gm[L.misc() + 1] = 1.0;
        S->done = 1;
    } else if (hn == 0.0 || d == 0.0) {
        gm[L.misc() + 1] = 2.0;  // happy breakdown: the cycle's space holds the solution
    } else if (S->iter >= S->maxiter) {
        gm[L.misc() + 1] = 3.0;
        S->done = 2;
    }
}

// V_{j+1} = w / ||w||
template <class VT>
__global__ void k_gm_normalize(int n, const VT* __restrict__ w, VT* __restrict__ vnext, int j, const double* gm,
                               GmLayout L)
{
    if (gm[L.misc() + 1] != 0.0) return;
    // ||w|| was saved before the Givens step rotated H[j+1][j] to zero
    const double norm = gm[L.misc() + 3];
    const double inv = norm > 0 ? 1.0 / norm : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vnext[i] = (VT)((double)w[i] * inv);
}

// save ||w|| before the rotation overwrites H[j+1][j]
__global__ void k_gm_save_norm(int j, double* gm, GmLayout L)
{
    if (gm[L.misc() + 1] != 0.0) return;
    gm[L.misc() + 3] = gm[L.H() + (size_t)(j + 1) * L.m + j];
}

// y = R^{-1} g over the completed steps (one thread), then x += M^{-1} V y
__global__ void k_gm_backsolve(double* gm, GmLayout L)
{
    const int m = L.m;
    const int k = (int)gm[L.misc()];
    const double* H = gm + L.H();
    const double* g = gm + L.g();
    double* y = gm + L.y();
    for (int i = k - 1; i >= 0; i--) {
        double s = g[i];
        for (int l = i + 1; l < k; l++) s -= H[(size_t)i * m + l] * y[l];
        const double d = H[(size_t)i * m + i];
        y[i] = d != 0.0 ? s / d : 0.0;
    }
}

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_gm_update(int n, VT* __restrict__ x, const VT* __restrict__ V,
                                                           const double* __restrict__ dinv, const double* gm, GmLayout L)
{
    __shared__ double ys[1024];
    const int k = (int)gm[L.misc()];
    for (int i = threadIdx.x; i < k; i += blockDim.x) ys[i] = gm[L.y() + i];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int i = 0; i < k; i++) t += ys[i] * (double)V[(size_t)i * n + r];
        x[r] = (VT)((double)x[r] + (dinv ? dinv[r] : 1.0) * t);
    }
}

// FP32 residual of the inner solve: V0 = b - w (w = A d), (V0, V0) into S->rr (last block)
__global__ void __launch_bounds__(kVecThreads) k_gm_res32(int n, const float* __restrict__ b, const float* __restrict__ w,
                                                          float* __restrict__ V0, double* __restrict__ partial,
                                                          unsigned int* ticket, KState* S)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const float t = b[r] - w[r];
        V0[r] = t;
        acc[0] += (double)t * (double)t;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(ticket)) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->rr = t[0];
            *ticket = 0;
        }
    }
}

}  // namespace

int solve_gmres64(System& s, int m, int maxiter, double tol, int* iters, int* restarts)
{
    if (m < 1 || m > 1000) {
        set_error("GMRES restart depth must be in [1, 1000]");
        return MSFEM_ERR_ARGUMENT;
    }
    const int n = s.n_rows;
    // V: (m+1) vectors, plus z (preconditioned v) and w; the first work vector doubles as r
    MSFEM_TRY(s.work64.alloc((size_t)(m + 3) * n));
    double* V = s.work64.p;
    double* z = V + (size_t)(m + 1) * n;
    double* w = z + n;
    GmLayout L{m};
    MSFEM_TRY(s.gm.alloc(L.total()));
    MSFEM_TRY(s.partial.alloc((size_t)(m + 2) * kReduceBlocks + 64));
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    MSFEM_CK(cudaMemsetAsync(s.gm.p, 0, sizeof(double) * L.total(), s.stream));

    const SellView<double> A = sell_view<double>(s);
    const unsigned g = spmv_grid(s);
    int total = 0, cycles = 0;
    cudaGraphExec_t exec = nullptr;
    int rc = MSFEM_OK;
    // (F, F): the residual kernel on x = 0 gives r = F
    MSFEM_CK(cudaMemsetAsync(z, 0, sizeof(double) * n, s.stream));
    MSFEM_TRY(residual64(s, z, s.F.p, w, &S->ff));
    s.launches += 1;
    // tol2, maxiter, counters
    KState init{};
    MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    init = *s.h_kstate;
    init.tol2 = tol * tol * init.ff;
    init.maxiter = maxiter;
    init.iter = 0;
    init.done = 0;
    init.breakdown = 0;
    for (auto& t : init.ticket) t = 0;
    *s.h_kstate = init;
    MSFEM_CK(cudaMemcpyAsync(S, s.h_kstate, sizeof(KState), cudaMemcpyHostToDevice, s.stream));

    while (true) {
        // r = F - A x into V_0's slot, then V_0 = r / ||r||
        MSFEM_TRY(residual64(s, s.X.p, s.F.p, V, &S->rr));
        MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        s.launches += 1;
        if (s.h_kstate->rr <= s.h_kstate->tol2 || s.h_kstate->done || total >= maxiter) break;
        k_gm_start<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, V, s.gm.p, L, S);
        s.launches += 1;
        if (!exec) {
            cudaGraph_t graph;
            MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
            for (int j = 0; j < m; j++) {
                double* vj = V + (size_t)j * n;
                k_gm_prec<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, vj, s.dinv64.p, z, s.gm.p, L);
                k_gm_spmv<double><<<g, 256, 0, s.stream>>>(A, z, w, s.gm.p, L);
                k_gm_multidot<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0], s.gm.p,
                                                                                   L, L.h1());
                k_gm_orth<double, false><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0],
                                                                                      s.gm.p, L, L.h1());
                k_gm_multidot<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0], s.gm.p,
                                                                                   L, L.h2());
                k_gm_orth<double, true><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0],
                                                                                     s.gm.p, L, L.h2());
                k_gm_save_norm<<<1, 1, 0, s.stream>>>(j, s.gm.p, L);
                k_gm_givens<<<1, 1, 0, s.stream>>>(j, s.gm.p, L, S);
                k_gm_normalize<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, w, V + (size_t)(j + 1) * n, j,
                                                                                    s.gm.p, L);
            }
            k_gm_backsolve<<<1, 1, 0, s.stream>>>(s.gm.p, L);
            k_gm_update<double><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, s.X.p, V, s.dinv64.p, s.gm.p, L);
            cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
            if (e != cudaSuccess) {
                set_error("GMRES graph capture failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
            e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                set_error("GMRES graph instantiate failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
        }
        cudaError_t e = cudaGraphLaunch(exec, s.stream);
        if (e != cudaSuccess) {
            set_error("GMRES graph launch failed: %s", cudaGetErrorString(e));
            rc = MSFEM_ERR_CUDA;
            break;
        }
        s.launches += 9 * m + 2;
        cycles++;
        MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        total = s.h_kstate->iter;
        if (s.h_kstate->done) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (rc < 0) return rc;
    *iters = s.h_kstate->iter;
    *restarts = cycles;
    return (s.h_kstate->rr <= s.h_kstate->tol2) ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

// Inner solve of FP32 iterative refinement: GMRES(m) on the FP32 copy of the Jacobi-scaled matrix
// (unit diagonal, so no preconditioner), A d = b from d = 0, to ||b - A d|| <= tau ||b||.  The
// Krylov basis is FP32 (half the bytes of the FP64 solver per Arnoldi pass); the Hessenberg
// matrix, the rotations and every inner product are FP64.  V is (m+1) n floats, w one more n.
int gmres32_inner(System& s, int m, float* d, const float* b, float* V, float* w, int maxiter, double tau, int* iters)
{
    const int n = s.n_rows;
    GmLayout L{m};
    MSFEM_TRY(s.gm.alloc(L.total()));
    MSFEM_TRY(s.partial.alloc((size_t)(m + 2) * kReduceBlocks + 64));
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    MSFEM_CK(cudaMemsetAsync(s.gm.p, 0, sizeof(double) * L.total(), s.stream));
    const SellView<float> A = sell_view<float>(s);
    const unsigned g = spmv_grid(s);
    // (b, b) -> ff via the residual kernel with w = 0
    MSFEM_CK(cudaMemsetAsync(w, 0, sizeof(float) * n, s.stream));
    k_gm_res32<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, b, w, V, part, &S->ticket[0], S);
    s.launches += 1;
    MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    KState init = *s.h_kstate;
    init.ff = init.rr;
    init.tol2 = tau * tau * init.ff;
    init.maxiter = maxiter;
    init.iter = 0;
    init.done = 0;
    init.breakdown = 0;
    for (auto& t : init.ticket) t = 0;
    *s.h_kstate = init;
    MSFEM_CK(cudaMemcpyAsync(S, s.h_kstate, sizeof(KState), cudaMemcpyHostToDevice, s.stream));
    cudaGraphExec_t exec = nullptr;
    int rc = MSFEM_OK;
    bool first = true;
    while (true) {
        if (!first) {
            // V_0 = b - A d
            MSFEM_TRY(spmv32(s, d, w));
            k_gm_res32<<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, b, w, V, part, &S->ticket[0], S);
            s.launches += 2;
            MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
            MSFEM_CK(cudaStreamSynchronize(s.stream));
        }
        first = false;  // on entry d = 0 and V_0 already holds b
        if (s.h_kstate->rr <= s.h_kstate->tol2 || s.h_kstate->done || s.h_kstate->iter >= maxiter) break;
        k_gm_start<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, V, s.gm.p, L, S);
        s.launches += 1;
        if (!exec) {
            cudaGraph_t graph;
            MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
            for (int j = 0; j < m; j++) {
                const float* vj = V + (size_t)j * n;
                k_gm_spmv<float><<<g, 256, 0, s.stream>>>(A, vj, w, s.gm.p, L);
                k_gm_multidot<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0], s.gm.p,
                                                                                  L, L.h1());
                k_gm_orth<float, false><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0],
                                                                                     s.gm.p, L, L.h1());
                k_gm_multidot<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0], s.gm.p,
                                                                                  L, L.h2());
                k_gm_orth<float, true><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V, j, w, part, &S->ticket[0],
                                                                                    s.gm.p, L, L.h2());
                k_gm_save_norm<<<1, 1, 0, s.stream>>>(j, s.gm.p, L);
                k_gm_givens<<<1, 1, 0, s.stream>>>(j, s.gm.p, L, S);
                k_gm_normalize<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, w, V + (size_t)(j + 1) * n, j,
                                                                                   s.gm.p, L);
            }
            k_gm_backsolve<<<1, 1, 0, s.stream>>>(s.gm.p, L);
            k_gm_update<float><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, d, V, nullptr, s.gm.p, L);
            cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
            if (e != cudaSuccess) {
                set_error("GMRES graph capture failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
            e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                set_error("GMRES graph instantiate failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
        }
        cudaError_t e = cudaGraphLaunch(exec, s.stream);
        if (e != cudaSuccess) {
            set_error("GMRES graph launch failed: %s", cudaGetErrorString(e));
            rc = MSFEM_ERR_CUDA;
            break;
        }
        s.launches += 8 * m + 2;
        MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        if (s.h_kstate->done) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (rc < 0) return rc;
    *iters = s.h_kstate->iter;
    return MSFEM_OK;
}

}  // namespace msfem
