// MINRES (Paige-Saunders) on the GPU, for the symmetric but indefinite systems
// the reference's elasticity assembly produces.
//
// The reference stores the element block B_J^T D B_I at A[I][J] (FEM/FEM_Grid.h:
// 2147-2191), the transpose of the textbook orientation.  The global matrix is
// still symmetric, but the difference from the textbook operator (a null
// Lagrangian that survives on couplings between free-boundary nodes) makes it
// indefinite: the Jacobi-scaled matrix of a homogeneous 8^3 cube already has
// eigenvalues down to -0.0065, and -0.48 with an E contrast of 100.  CG
// (the reference's MSG / MSG_PreconditioningSSOR) usually still converges in
// FP64, but has no guarantee, and in FP32 it meets negative curvature
// ((p, Ap) < 0) and diverges.  MINRES minimises ||r|| over the same Krylov
// space and only needs A = A^T, so it is the inner solver of the elasticity
// FP32 refinement and an FP64 method of its own.
//
// The operator is the Jacobi-scaled S A S (S = D^-1/2): for FP32 the values
// are stored scaled; for FP64 the scaling is applied on the fly (the input
// vector t = S v is written by the previous update pass, and each output row is
// multiplied by s_i).  One iteration is three kernels:
//   k_mr_spmv     q = S A S v, alpha = (v, q)
//   k_mr_lanczos  q -= alpha v + beta v_old, beta' = ||q||; the last block
//                 applies the two previous Givens rotations to the new column of
//                 the tridiagonal matrix, forms the new rotation and the
//                 residual norm |eta|, and decides to stop
//   k_mr_update   w = (v - eps w'' - delta w') / gamma (into w''), x += tau w
//                 (times s_i for FP64), v_next = q / beta'  (in place)
// The Lanczos and w vectors rotate through fixed buffers with period 6, so a
// chunk of 6 iterations is captured once as a CUDA graph and replayed.
#include <cmath>
#include <cstdlib>
#include <string>

#include "devutil.cuh"
#include "internal.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

struct MrScalars {
    double alpha, beta, beta_next, eta, c0, s0, c1, s1, eps, delta, gamma, tau, res0;
};

template <class VT>
struct MrVectors {
    VT* x;           // solution (true space for FP64, scaled space for the FP32 inner solve)
    VT* buf[3];      // Lanczos vectors v_old, v, q (roles rotate with period 3)
    VT* wb[2];       // w'' and w' (roles swap every iteration)
    VT* t;           // S v (FP64 only)
    const double* s; // S = D^-1/2 (FP64 only)
};

// v = S r / ||S r|| (or r / ||r||), t = S v, w = v_old = 0, eta = ||.||
template <class VT, bool SCALE>
__global__ void __launch_bounds__(kVecThreads) k_mr_init_norm(int n, const VT* __restrict__ r, const double* __restrict__ s,
                                                              VT* __restrict__ v, KState* S, double* __restrict__ partial)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT vi = SCALE ? (VT)(s[i] * (double)r[i]) : r[i];
        v[i] = vi;
        acc[0] += (double)vi * (double)vi;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            MrScalars* m = reinterpret_cast<MrScalars*>(S->mr);
            *m = MrScalars{};
            const double b1 = sqrt(t[0]);
            m->eta = b1;
            m->res0 = b1;
            m->beta = 0.0;
            m->c0 = m->c1 = 1.0;
            m->s0 = m->s1 = 0.0;
            S->rr = t[0];
            S->ff = t[0];
            S->tol2 = S->tol2_rel * t[0];
            S->iter = 0;
            S->breakdown = 0;
            S->done = (b1 == 0.0) ? 1 : 0;
            S->mr_applied = (b1 == 0.0) ? 0 : -1;  // nothing to apply for a zero right-hand side
            S->ticket[0] = 0;
        }
    }
}

template <class VT, bool SCALE>
__global__ void __launch_bounds__(kVecThreads) k_mr_init_vectors(int n, VT* __restrict__ v, VT* __restrict__ vold,
                                                                 VT* __restrict__ w0, VT* __restrict__ w1,
                                                                 VT* __restrict__ t, const double* __restrict__ s,
                                                                 const KState* S)
{
    const MrScalars* m = reinterpret_cast<const MrScalars*>(S->mr);
    const double inv = m->eta > 0 ? 1.0 / m->eta : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT vi = (VT)((double)v[i] * inv);
        v[i] = vi;
        vold[i] = 0;
        w0[i] = 0;
        w1[i] = 0;
        if (SCALE) t[i] = (VT)(s[i] * (double)vi);
    }
}

// q = S A S v (x = t = S v for FP64, or the pre-scaled FP32 matrix on v); alpha = (v, q)
template <class VT, bool SCALE>
__global__ void __launch_bounds__(256) k_mr_spmv(SellView<VT> A, const VT* __restrict__ in, const VT* __restrict__ v,
                                                 VT* __restrict__ q, const double* __restrict__ s, KState* S,
                                                 double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[1] = {0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (A.bs == 1) {
            VT y = sell_row_scalar<VT>(A, warp, lane, in);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                if (SCALE) y = (VT)(s[row] * (double)y);
                q[row] = y;
                acc[0] += (double)v[row] * (double)y;
            }
        } else {
            VT y[3];
            sell_row_block<VT>(A, warp, lane, in, y);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    const int64_t i = 3 * (int64_t)brow + c;
                    VT yi = y[c];
                    if (SCALE) yi = (VT)(s[i] * (double)yi);
                    q[i] = yi;
                    acc[0] += (double)v[i] * (double)yi;
                }
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            reinterpret_cast<MrScalars*>(S->mr)->alpha = t[0];
            S->ticket[0] = 0;
        }
    }
}

// q -= alpha v + beta v_old; beta' = ||q||; Givens update and stopping test
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_mr_lanczos(int n, VT* __restrict__ q, const VT* __restrict__ v,
                                                            const VT* __restrict__ vold, KState* S,
                                                            double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const MrScalars* mc = reinterpret_cast<const MrScalars*>(S->mr);
    const VT a = (VT)mc->alpha, b = (VT)mc->beta;
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT qi = q[i] - a * v[i] - b * vold[i];
        q[i] = qi;
        acc[0] += (double)qi * (double)qi;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            MrScalars* m = reinterpret_cast<MrScalars*>(S->mr);
            const double bn = sqrt(t[0]);
            // previous rotations on the column (beta, alpha, beta') of the tridiagonal matrix
            const double eps = m->s0 * m->beta;
            const double d1 = m->c0 * m->beta;
            const double delta = m->c1 * d1 + m->s1 * m->alpha;
            const double g1 = -m->s1 * d1 + m->c1 * m->alpha;
            const double gamma = sqrt(g1 * g1 + bn * bn);
            const double c = gamma > 0 ? g1 / gamma : 1.0, sn = gamma > 0 ? bn / gamma : 0.0;
            m->eps = eps;
            m->delta = delta;
            m->gamma = gamma;
            m->tau = c * m->eta;
            m->eta = -sn * m->eta;
            m->c0 = m->c1;
            m->s0 = m->s1;
            m->c1 = c;
            m->s1 = sn;
            m->beta_next = bn;
            S->iter += 1;
            S->rr = m->eta * m->eta;
            if (gamma == 0.0 || !(gamma == gamma)) {
                S->breakdown = 1;
                m->tau = 0.0;
                S->done = 3;
            } else if (S->rr <= S->tol2) {
                S->done = 1;
            } else if (S->iter >= S->maxiter) {
                S->done = 2;
            }
            S->ticket[0] = 0;
        }
    }
}

// w = (v - eps w'' - delta w') / gamma  (stored over w''); x += tau w (x += tau S w for FP64);
// v_next = q / beta'  (in place); t = S v_next.  Runs on the step that set the stopping flag
// too (the last solution update), but not after.
template <class VT, bool SCALE>
__global__ void __launch_bounds__(kVecThreads) k_mr_update(int n, VT* __restrict__ x, VT* __restrict__ q,
                                                           const VT* __restrict__ v, VT* __restrict__ w2,
                                                           const VT* __restrict__ w1, VT* __restrict__ t,
                                                           const double* __restrict__ s, KState* S)
{
    const int last = S->iter;
    if (S->done && S->mr_applied == last) return;
    const MrScalars* m = reinterpret_cast<const MrScalars*>(S->mr);
    const double ig = m->gamma > 0 ? 1.0 / m->gamma : 0.0;
    const VT eps = (VT)m->eps, delta = (VT)m->delta, tau = (VT)m->tau;
    const VT ib = (VT)(m->beta_next > 0 ? 1.0 / m->beta_next : 0.0);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT wi = (VT)((double)(v[i] - eps * w2[i] - delta * w1[i]) * ig);
        w2[i] = wi;
        if (SCALE) x[i] += tau * (VT)(s[i] * (double)wi);
        else x[i] += tau * wi;
        const VT vn = q[i] * ib;
        q[i] = vn;
        if (SCALE) t[i] = (VT)(s[i] * (double)vn);
    }
}

// after k_mr_update: beta <- beta' for the next step, and mark the update of a finished solve as applied
__global__ void k_mr_advance(KState* S)
{
    MrScalars* m = reinterpret_cast<MrScalars*>(S->mr);
    if (S->done) {
        S->mr_applied = S->iter;
        return;
    }
    m->beta = m->beta_next;
}

inline std::string key_of(const char* tag, const void* const* p, int np, int n)
{
    std::string k(tag);
    char b[32];
    for (int i = 0; i < np; i++) {
        std::snprintf(b, sizeof(b), ":%p", p[i]);
        k += b;
    }
    std::snprintf(b, sizeof(b), ":%d", n);
    return k + b;
}

}  // namespace

// MINRES on S A S from x = 0 with right-hand side S r (or r for the pre-scaled FP32 matrix).
// FP64 (SCALE): x (true space) += S y.  FP32: x holds y.  Stops on |eta| <= tol * ||S r||.
template <class VT, bool SCALE>
int minres_run(System& s, VT* x, const VT* r, int maxiter, double tol, int stall_unused, int* iters)
{
    (void)stall_unused;
    const int n = s.n_rows;
    KState* S = s.kstate.p;
    double* part = s.partial.p;
    VT* base = nullptr;
    if constexpr (sizeof(VT) == 8) {
        MSFEM_TRY(s.mr64.alloc((size_t)(SCALE ? 6 : 5) * n));
        base = reinterpret_cast<VT*>(s.mr64.p);
    } else {
        MSFEM_TRY(s.mr32.alloc((size_t)(SCALE ? 6 : 5) * n));
        base = reinterpret_cast<VT*>(s.mr32.p);
    }
    struct {
        VT* p;
    } work{base};
    MrVectors<VT> V;
    V.x = x;
    V.buf[0] = work.p;          // v_old
    V.buf[1] = work.p + n;      // v
    V.buf[2] = work.p + 2 * (size_t)n;  // q
    V.wb[0] = work.p + 3 * (size_t)n;   // w''
    V.wb[1] = work.p + 4 * (size_t)n;   // w'
    V.t = SCALE ? work.p + 5 * (size_t)n : nullptr;
    V.s = SCALE ? s.dscale.p : nullptr;
    // limits: tol relative to the initial (scaled) residual norm
    {
        KState h = {};
        MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        h = *s.h_kstate;
        h.tol2_rel = tol * tol;
        h.maxiter = maxiter;
        h.done = 0;
        h.mr_applied = -1;
        for (auto& tk : h.ticket) tk = 0;
        *s.h_kstate = h;
        MSFEM_CK(cudaMemcpyAsync(S, s.h_kstate, sizeof(KState), cudaMemcpyHostToDevice, s.stream));
    }
    k_mr_init_norm<VT, SCALE><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, r, V.s, V.buf[1], S, part);
    k_mr_init_vectors<VT, SCALE><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V.buf[1], V.buf[0], V.wb[0], V.wb[1],
                                                                             V.t, V.s, S);
    MSFEM_CK(cudaGetLastError());
    s.launches += 2;
    const SellView<VT> A = sell_view<VT>(s);
    const unsigned g = spmv_grid_of((const void*)k_mr_spmv<VT, SCALE>, s);
    // one period of 6 iterations: Lanczos roles (v_old, v, q) rotate by one, w roles swap
    auto period = [&]() {
        for (int k = 0; k < 6; k++) {
            VT* vold = V.buf[k % 3];
            VT* v = V.buf[(k + 1) % 3];
            VT* q = V.buf[(k + 2) % 3];
            VT* w2 = V.wb[k % 2];
            VT* w1 = V.wb[(k + 1) % 2];
            const VT* in = SCALE ? V.t : v;
            k_mr_spmv<VT, SCALE><<<g, 256, 0, s.stream>>>(A, in, v, q, V.s, S, part);
            k_mr_lanczos<VT><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, q, v, vold, S, part);
            k_mr_update<VT, SCALE><<<kReduceBlocks, kVecThreads, 0, s.stream>>>(n, V.x, q, v, w2, w1, V.t, V.s, S);
            k_mr_advance<<<1, 1, 0, s.stream>>>(S);
        }
    };
    const void* keyp[] = {V.x, V.buf[0], V.wb[0], V.t, V.s, A.val, A.col, (const void*)S, part};
    const std::string key = key_of(sizeof(VT) == 8 ? "minres64" : "minres32", keyp, 9, n);
    auto it = s.graphs.find(key);
    if (it == s.graphs.end()) {
        std::array<cudaGraphExec_t, 8> empty{};
        it = s.graphs.emplace(key, empty).first;
    }
    cudaGraphExec_t& exec = it->second[0];
    int rounds = 0;
    for (;;) {
        MSFEM_CK(cudaMemcpyAsync(s.h_kstate, S, sizeof(KState), cudaMemcpyDeviceToHost, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
        if (s.h_kstate->done) break;
        if (6 * rounds > maxiter + 12) break;
        if (!exec) {
            cudaGraph_t gr;
            MSFEM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
            for (int c = 0; c < 4; c++) period();  // 24 iterations per replay
            cudaError_t e = cudaStreamEndCapture(s.stream, &gr);
            if (e != cudaSuccess) {
                set_error("MINRES graph capture failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
            e = cudaGraphInstantiate(&exec, gr, 0);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) {
                set_error("MINRES graph instantiate failed: %s", cudaGetErrorString(e));
                return MSFEM_ERR_CUDA;
            }
        }
        MSFEM_CK(cudaGraphLaunch(exec, s.stream));
        s.launches += 24 * 4;
        rounds += 4;
    }
    *iters = s.h_kstate->iter;
    if (s.h_kstate->breakdown) return MSFEM_ERR_NUMERIC;
    return s.h_kstate->done == 1 ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

template int minres_run<double, true>(System&, double*, const double*, int, double, int, int*);
template int minres_run<float, false>(System&, float*, const float*, int, double, int, int*);

}  // namespace msfem
