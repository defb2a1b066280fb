// Batched cell systems: sort-based deterministic portrait + assembly, and a
// persistent MINRES solver with one CTA per system.
//
// Portrait and assembly.  The reference builds each cell problem's portrait
// (Grid_forMech::CreationPortrait, FEM/FEM_Grid.h:3236-3287) and adds the element
// matrices serially in element order (CSSD_Matrix::SummPartOfMatrix,
// Library/CSSD_Matrix.h:307-363), one cell at a time in an OpenMP loop over cells
// (MsFEM/MsFEM_Grid.h:4800-4802).  Here every element of every system emits its
// (k+1)^2 (row, column) node pairs, tagged element << 2b | I << b | J (b = 2 bits for up to 4
// nodes per element, 3 for 8); one stable
// radix sort by (row, column) groups equal pairs (a block of the matrix) with
// their contributions in element order.  The unique keys are the portrait (rows
// sorted, diagonal included); the sorted tags are kept, so assembling a block is
// a gather-sum of its contributions in the same order as the reference's serial
// scatter -- no colouring, no atomics, the same bits on every run.
//
// Solve.  A cell problem has Dirichlet data on its whole boundary and zero
// source; its matrix is symmetric but, with stiff inclusions, indefinite (the
// reference's transposed element blocks leave interface terms; a few negative
// eigenvalues appear), so the inner solver is MINRES on the Jacobi-scaled free
// block S A_II S.  One persistent launch covers every system: each CTA takes the
// next system from an atomic queue (largest first), runs the FP64 outer
// refinement (true residual r = -A x with the Dirichlet values in x) and the
// inner MINRES for all R right-hand sides at once (one recurrence per
// right-hand side, one shared sparse product), with CTA barriers only.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "batch.cuh"
#include "devutil.cuh"
#include "element.cuh"

namespace msfem {
namespace {

constexpr unsigned kFull = 0xffffffffu;

int bits_for(int64_t n)
{
    int b = 1;
    while (((int64_t)1 << b) < n) b++;
    return b;
}

__global__ void k_check_elements(int n_sys, const int64_t* __restrict__ node_off, const int64_t* __restrict__ elem_off,
                                 const int32_t* __restrict__ elems, int k1, int* bad)
{
    const int s = blockIdx.x;
    if (s >= n_sys) return;
    const int64_t n0 = node_off[s], n1 = node_off[s + 1];
    for (int64_t e = elem_off[s] + threadIdx.x; e < elem_off[s + 1]; e += blockDim.x)
        for (int a = 0; a < k1; a++) {
            const int64_t v = elems[e * k1 + a];
            if (v < n0 || v >= n1) atomicExch(bad, 1);
        }
}

// bits of each element-local index in a contribution tag (element << 2 tb | I << tb | J)
__host__ __device__ __forceinline__ int tag_bits(int k1) { return k1 > 8 ? 5 : (k1 > 4 ? 3 : 2); }

__global__ void k_emit_pairs(int64_t e0, int64_t e1, int64_t n0, int nb, const int32_t* __restrict__ elems, int k1,
                             uint64_t* __restrict__ key, uint32_t* __restrict__ tag)
{
    const int64_t kk = (int64_t)k1 * k1;
    const int64_t count = (e1 - e0) * kk;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = e0 + t / kk;
        const int ab = (int)(t % kk);
        const int a = ab / k1, b = ab % k1;
        const uint64_t row = (uint64_t)(elems[e * k1 + a] - n0);
        const uint64_t col = (uint64_t)(elems[e * k1 + b] - n0);
        key[t] = (row << nb) | col;
        const int tb = tag_bits(k1);
        tag[t] = ((uint32_t)e << (2 * tb)) | (uint32_t)(a << tb) | (uint32_t)b;
    }
}

__global__ void k_heads(int64_t count, const uint64_t* __restrict__ key, int32_t* __restrict__ head)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// one thread per sorted pair that starts a block: its column, first contribution, row count
__global__ void k_slots(int64_t count, const uint64_t* __restrict__ key, const int32_t* __restrict__ head,
                        const int32_t* __restrict__ slot, int64_t n0, int nb, int64_t pair_base,
                        int32_t* __restrict__ col, int64_t* __restrict__ cstart, int32_t* __restrict__ row_cnt)
{
    const uint64_t mask = ((uint64_t)1 << nb) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        const int s = slot[i];
        const uint64_t k = key[i];
        col[s] = (int32_t)(n0 + (int64_t)(k & mask));
        cstart[s] = pair_base + i;
        atomicAdd(&row_cnt[n0 + (int64_t)(k >> nb)], 1);
    }
}

template <int K1>
__device__ __forceinline__ void element_block_of(const int32_t* __restrict__ elems, const double* __restrict__ xyz,
                                                 int64_t e, int I, int J, double lam, double mu, double out[9])
{
    if (K1 == 4) {
        int v[4];
#pragma unroll
        for (int a = 0; a < 4; a++) v[a] = elems[e * 4 + a];
        TetGeom G;
        tet_geometry(xyz, v, G);
        elastic_block(G.g[I], G.g[J], G.vol, lam, mu, out);
    } else {
        int v[3];
#pragma unroll
        for (int a = 0; a < 3; a++) v[a] = elems[e * 3 + a];
        double g[3][3], area;
        tri_geometry(xyz, v, g, area);
        elastic_block(g[I], g[J], area, lam, mu, out);
    }
}

// each block = sum of its element contributions in element order
template <int K1>
__global__ void k_assemble_blocks(int64_t nnzb, const int64_t* __restrict__ cstart, const uint32_t* __restrict__ contrib,
                                  const int32_t* __restrict__ elems, const int32_t* __restrict__ emat,
                                  const double* __restrict__ xyz, const double* __restrict__ lame, int n_mat,
                                  double* __restrict__ val, int* bad)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nnzb; s += (int64_t)gridDim.x * blockDim.x) {
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t c = cstart[s]; c < cstart[s + 1]; c++) {
            const uint32_t t = contrib[c];
            const int64_t e = t >> 4;
            const int I = (t >> 2) & 3, J = t & 3;
            const int m = emat ? emat[e] : 0;
            if (m < 0 || m >= n_mat) {
                atomicExch(bad, 1);
                continue;
            }
            const double lam = lame[2 * m], mu = lame[2 * m + 1];
            if (lam == 0.0 && mu == 0.0) continue;  // E <= 0: no contribution (FEM/FEM.h:1355-1363)
            double blk[9];
            element_block_of<K1>(elems, xyz, e, I, J, lam, mu, blk);
#pragma unroll
            for (int q = 0; q < 9; q++) acc[q] += blk[q];
        }
#pragma unroll
        for (int q = 0; q < 9; q++) val[9 * s + q] = acc[q];
    }
}

// each block = sum of the caller's element blocks eb[e][I][J][9] in element order (8-node
// elements: the MsFEM macro cells)
__global__ void k_assemble_given(int64_t nnzb, const int64_t* __restrict__ cstart, const uint32_t* __restrict__ contrib,
                                 int k1, const double* __restrict__ eb, double* __restrict__ val)
{
    const int tb = tag_bits(k1);
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nnzb; s += (int64_t)gridDim.x * blockDim.x) {
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t c = cstart[s]; c < cstart[s + 1]; c++) {
            const uint32_t t = contrib[c];
            const int64_t e = t >> (2 * tb);
            const int I = (t >> tb) & ((1 << tb) - 1), J = t & ((1 << tb) - 1);
            const double* blk = eb + 9 * (((int64_t)e * k1 + I) * k1 + J);
#pragma unroll
            for (int q = 0; q < 9; q++) acc[q] += blk[q];
        }
#pragma unroll
        for (int q = 0; q < 9; q++) val[9 * s + q] = acc[q];
    }
}

// s = 1/sqrt(A_ii[a][a]) (1 when not positive), then the scaled FP32 copy, row by row
__global__ void k_batch_scale(int64_t n_nodes, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                              const double* __restrict__ val, double* __restrict__ dscale)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        double d[3] = {0, 0, 0};
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++)
            if (col[k] == i) {
                d[0] = val[9 * k];
                d[1] = val[9 * k + 4];
                d[2] = val[9 * k + 8];
            }
        for (int a = 0; a < 3; a++) dscale[3 * i + a] = d[a] > 0.0 ? 1.0 / sqrt(d[a]) : 1.0;
    }
}

__global__ void k_batch_val32(int64_t n_nodes, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                              const double* __restrict__ val, const double* __restrict__ dscale, float* __restrict__ v32)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const double si[3] = {dscale[3 * i], dscale[3 * i + 1], dscale[3 * i + 2]};
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
            const int64_t j = col[k];
            const double sj[3] = {dscale[3 * j], dscale[3 * j + 1], dscale[3 * j + 2]};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) v32[9 * k + 3 * a + b] = (float)(si[a] * val[9 * k + 3 * a + b] * sj[b]);
        }
    }
}

// ------------------------------------------------------------------ persistent solver

struct BatchArgs {
    int n_sys;
    const int32_t* order;
    const int64_t* node_off;
    const int64_t* row_ptr;
    const int32_t* col;
    const double* val64;
    const float* val32;
    const double* dscale;
    const uint8_t* fixed;
    double* x;
    const double* rhs;  // [n_nodes][R][3] source term, or null (zero source)
    void* work;
    int64_t work_stride;  // elements of VT per vector
    int* queue;
    int32_t* iters;
    int32_t* outers;
    double* rel;
    double tol;
    int maxiter;
    int max_outer;
};

struct MrRhs {
    double alpha, beta, eta, c0, s0, c1, s1, eps, delta, gamma, tau, bnext, b1, target, fnorm2;
    int active, upd;
};

// per right-hand-side block reduction: thread t holds a partial of rhs t % R
template <int R>
__device__ __forceinline__ void rhs_sum(double v, double* red, double* out)
{
#pragma unroll
    for (int o = 16; o >= R; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane < R) red[warp * R + lane] = v;
    __syncthreads();
    if (threadIdx.x < R) {
        double t = 0.0;
        for (int w = 0; w < nw; w++) t += red[w * R + threadIdx.x];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

// y = S A S v on the free rows of one system (VT float: pre-scaled FP32 values;
// VT double: FP64 values scaled on the fly); rows of Dirichlet nodes give 0.
template <int R, class VT>
__device__ __forceinline__ void row_product(const BatchArgs& A, int64_t n0, int i, int r, const VT* __restrict__ v,
                                            VT y[3])
{
    const int64_t gi = n0 + i;
    VT acc[3] = {0, 0, 0};
    for (int64_t k = A.row_ptr[gi]; k < A.row_ptr[gi + 1]; k++) {
        const int64_t c = A.col[k] - n0;
        const VT* xv = v + (c * R + r) * 3;
        if (sizeof(VT) == 4) {
            const float* a = A.val32 + 9 * k;
            const VT x0 = xv[0], x1 = xv[1], x2 = xv[2];
            acc[0] += (VT)a[0] * x0 + (VT)a[1] * x1 + (VT)a[2] * x2;
            acc[1] += (VT)a[3] * x0 + (VT)a[4] * x1 + (VT)a[5] * x2;
            acc[2] += (VT)a[6] * x0 + (VT)a[7] * x1 + (VT)a[8] * x2;
        } else {
            const double* a = A.val64 + 9 * k;
            const double* sj = A.dscale + 3 * (n0 + c);
            const double x0 = (double)xv[0] * sj[0], x1 = (double)xv[1] * sj[1], x2 = (double)xv[2] * sj[2];
            acc[0] += a[0] * x0 + a[1] * x1 + a[2] * x2;
            acc[1] += a[3] * x0 + a[4] * x1 + a[5] * x2;
            acc[2] += a[6] * x0 + a[7] * x1 + a[8] * x2;
        }
    }
    if (sizeof(VT) == 4) {
#pragma unroll
        for (int a = 0; a < 3; a++) y[a] = acc[a];
    } else {
        const double* si = A.dscale + 3 * gi;
#pragma unroll
        for (int a = 0; a < 3; a++) y[a] = (VT)(si[a] * (double)acc[a]);
    }
}

// Shared state of one CTA's solve (one system at a time).
template <int R>
struct CtaShared {
    double red[32 * R];
    double s1[R], s2[R];
    MrRhs mr[R];
    double rr_prev[R];
    int q, active, conv, bad;
};

// FP64 residual r = -A x on the free rows of the CTA's system (x holds the Dirichlet
// values), written scaled (v = S r) into V; sums ||r||^2 -> s1, ||v||^2 -> s2 per rhs.
template <int R, class VT>
__device__ void residual_pass(const BatchArgs& A, int64_t n0, int np, const uint8_t* fx, const double* X, VT* V,
                              CtaShared<R>& sh)
{
    const int tid = threadIdx.x, T = blockDim.x, r = tid % R;
    double arr = 0.0, avv = 0.0;
    for (int p = tid; p < np; p += T) {
        const int i = p / R;
        if (fx[i]) {
#pragma unroll
            for (int c = 0; c < 3; c++) V[3 * (int64_t)p + c] = 0;
            continue;
        }
        const int64_t gi = n0 + i;
        double y[3] = {0, 0, 0};
        if (A.rhs)
#pragma unroll
            for (int c = 0; c < 3; c++) y[c] = A.rhs[(n0 * R + p) * 3 + c];
        for (int64_t k = A.row_ptr[gi]; k < A.row_ptr[gi + 1]; k++) {
            const int64_t cc = A.col[k] - n0;
            const double* a = A.val64 + 9 * k;
            const double* xv = X + (cc * R + r) * 3;
            y[0] -= a[0] * xv[0] + a[1] * xv[1] + a[2] * xv[2];
            y[1] -= a[3] * xv[0] + a[4] * xv[1] + a[5] * xv[2];
            y[2] -= a[6] * xv[0] + a[7] * xv[1] + a[8] * xv[2];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            arr += y[c] * y[c];
            const VT vs = (VT)(A.dscale[3 * gi + c] * y[c]);
            V[3 * (int64_t)p + c] = vs;
            avv += (double)vs * (double)vs;
        }
    }
    rhs_sum<R>(arr, sh.red, sh.s1);
    rhs_sum<R>(avv, sh.red, sh.s2);
}

// x += sign * S y on the free rows, for the rhs with want[r] set (all when want is null)
template <int R, class VT>
__device__ void apply_correction(const BatchArgs& A, int64_t n0, int np, const uint8_t* fx, double* X, const VT* Y,
                                 double sign, const int* want)
{
    const int tid = threadIdx.x, T = blockDim.x;
    if (want && !want[tid % R]) return;
    for (int p = tid; p < np; p += T) {
        const int i = p / R;
        if (fx[i]) continue;
        const int64_t gi = n0 + i;
#pragma unroll
        for (int c = 0; c < 3; c++)
            X[3 * (int64_t)p + c] += sign * A.dscale[3 * gi + c] * (double)Y[3 * (int64_t)p + c];
    }
}

// MINRES on S A_II S y = v (v = Vb[1] on entry, ||v|| = mr[r].b1), for all R rhs at once;
// returns the iterations.  The solution is left in Y.
template <int R, class VT>
__device__ int inner_minres(const BatchArgs& A, int64_t n0, int np, const uint8_t* fx, VT* base, CtaShared<R>& sh)
{
    const int tid = threadIdx.x, T = blockDim.x;
    const int rr_ = tid % R;
    const int64_t S = A.work_stride;
    VT* Vb[3] = {base, base + S, base + 2 * S};
    VT* Wb[2] = {base + 3 * S, base + 4 * S};
    VT* Y = base + 5 * S;
    {
        const double b1 = sh.mr[rr_].b1;
        const VT inv = (VT)(b1 > 0.0 ? 1.0 / b1 : 0.0);
        for (int p = tid; p < np; p += T)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int64_t o = 3 * (int64_t)p + c;
                Vb[1][o] *= inv;
                Vb[0][o] = 0;
                Wb[0][o] = 0;
                Wb[1][o] = 0;
                Y[o] = 0;
            }
    }
    __syncthreads();
    int iv_old = 0, iv = 1, iq = 2, iw2 = 0, iw1 = 1;
    int k = 0;
    for (; k < A.maxiter; k++) {
        VT* vo = Vb[iv_old];
        VT* v = Vb[iv];
        VT* qv = Vb[iq];
        // q = S A S v, alpha = (v, q)
        double a1 = 0.0;
        for (int p = tid; p < np; p += T) {
            const int i = p / R;
            VT y[3] = {0, 0, 0};
            if (!fx[i]) row_product<R, VT>(A, n0, i, rr_, v, y);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                qv[3 * (int64_t)p + c] = y[c];
                a1 += (double)v[3 * (int64_t)p + c] * (double)y[c];
            }
        }
        rhs_sum<R>(a1, sh.red, sh.s1);
        // q -= alpha v + beta v_old, ||q||^2
        const VT al = (VT)sh.s1[rr_], be = (VT)sh.mr[rr_].beta;
        double a2 = 0.0;
        for (int p = tid; p < np; p += T)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int64_t o = 3 * (int64_t)p + c;
                const VT t = qv[o] - al * v[o] - be * vo[o];
                qv[o] = t;
                a2 += (double)t * (double)t;
            }
        rhs_sum<R>(a2, sh.red, sh.s2);
        if (tid < R) {
            MrRhs& m = sh.mr[tid];
            m.upd = m.active;
            if (m.active) {
                m.alpha = sh.s1[tid];
                const double bn = sqrt(sh.s2[tid]);
                const double eps = m.s0 * m.beta;
                const double d1 = m.c0 * m.beta;
                const double delta = m.c1 * d1 + m.s1 * m.alpha;
                const double g1 = -m.s1 * d1 + m.c1 * m.alpha;
                const double gamma = sqrt(g1 * g1 + bn * bn);
                const double c = gamma > 0.0 ? g1 / gamma : 1.0, sn = gamma > 0.0 ? bn / gamma : 0.0;
                m.eps = eps;
                m.delta = delta;
                m.gamma = gamma;
                m.tau = gamma > 0.0 ? c * m.eta : 0.0;
                m.eta = -sn * m.eta;
                m.c0 = m.c1;
                m.s0 = m.s1;
                m.c1 = c;
                m.s1 = sn;
                m.bnext = bn;
                if (!(gamma > 0.0) || !(bn > 0.0) || fabs(m.eta) <= m.target * m.b1) m.active = 0;
                if (!(gamma > 0.0)) m.upd = 0;
            }
        }
        __syncthreads();
        if (tid == 0) {
            int na = 0;
            for (int r = 0; r < R; r++) na += sh.mr[r].active;
            sh.active = na;
        }
        // w = (v - eps w'' - delta w') / gamma into w''; y += tau w; v_next = q / beta'
        {
            const MrRhs& m = sh.mr[rr_];
            VT* w2 = Wb[iw2];
            const VT* w1 = Wb[iw1];
            if (m.upd) {
                const VT ig = (VT)(1.0 / m.gamma), ep = (VT)m.eps, de = (VT)m.delta, ta = (VT)m.tau;
                const VT ib = (VT)(m.bnext > 0.0 ? 1.0 / m.bnext : 0.0);
                for (int p = tid; p < np; p += T)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const int64_t o = 3 * (int64_t)p + c;
                        const VT w = (v[o] - ep * w2[o] - de * w1[o]) * ig;
                        w2[o] = w;
                        Y[o] += ta * w;
                        qv[o] *= ib;
                    }
            } else {
                // a finished right-hand side keeps its vectors: the rotation below
                // then leaves v_old = v = the last Lanczos vector (finite, unused)
                for (int p = tid; p < np; p += T)
#pragma unroll
                    for (int c = 0; c < 3; c++) qv[3 * (int64_t)p + c] = v[3 * (int64_t)p + c];
            }
        }
        __syncthreads();
        if (tid < R && sh.mr[tid].upd) sh.mr[tid].beta = sh.mr[tid].bnext;
        const int t0 = iv_old;
        iv_old = iv;
        iv = iq;
        iq = t0;
        const int t1 = iw2;
        iw2 = iw1;
        iw1 = t1;
        const int na = sh.active;
        __syncthreads();
        if (na == 0) {
            k++;
            break;
        }
    }
    return k;
}

// One CTA per system, taken from an atomic queue.  FP64 outer refinement; the inner
// solves start in FP32 (precision MSFEM_FP32_IR) and a system whose FP32 step fails to
// halve a right-hand side's residual has that step undone and continues with FP64
// inner solves (ill-conditioned cells: FP32 Lanczos vectors lose orthogonality).
template <int R>
__global__ void __launch_bounds__(512) k_batch_minres(BatchArgs A, int start64)
{
    __shared__ CtaShared<R> sh;
    __shared__ int s_bad[R];
    const int tid = threadIdx.x, T = blockDim.x;
    char* cta_base = reinterpret_cast<char*>(A.work) + (int64_t)blockIdx.x * 6 * A.work_stride * sizeof(double);
    float* base32 = reinterpret_cast<float*>(cta_base);
    double* base64 = reinterpret_cast<double*>(cta_base);

    for (;;) {
        if (tid == 0) sh.q = atomicAdd(A.queue, 1);
        __syncthreads();
        const int q = sh.q;
        __syncthreads();
        if (q >= A.n_sys) break;
        const int sys = A.order[q];
        const int64_t n0 = A.node_off[sys];
        const int n = (int)(A.node_off[sys + 1] - n0);
        const int np = n * R;
        double* X = A.x + n0 * R * 3;
        const uint8_t* fx = A.fixed + n0;
        if (tid < R) {
            sh.mr[tid].fnorm2 = 0.0;
            sh.rr_prev[tid] = 0.0;
            s_bad[tid] = 0;
        }
        int use64 = start64, last64 = start64;
        int inner_total = 0, outer = 0;
        double relmax = 0.0;
        for (outer = 0;; outer++) {
            if (use64) residual_pass<R, double>(A, n0, np, fx, X, base64 + A.work_stride, sh);
            else residual_pass<R, float>(A, n0, np, fx, X, base32 + A.work_stride, sh);
            if (tid == 0) {
                // a right-hand side whose last FP32 step did not halve its residual
                int bad = 0;
                if (outer > 0 && !last64)
                    for (int r = 0; r < R; r++) {
                        s_bad[r] = (sh.s1[r] > 0.25 * sh.rr_prev[r] && sh.rr_prev[r] > 0.0) ? 1 : 0;
                        bad |= s_bad[r];
                    }
                sh.bad = bad;
            }
            __syncthreads();
            if (sh.bad) {
                // undo those steps (their corrections are still in Y) and recompute in FP64
                apply_correction<R, float>(A, n0, np, fx, X, base32 + 5 * A.work_stride, -1.0, s_bad);
                __syncthreads();
                use64 = 1;
                last64 = 1;
                if (tid < R) s_bad[tid] = 0;
                residual_pass<R, double>(A, n0, np, fx, X, base64 + A.work_stride, sh);
            }
            if (tid == 0) {
                int conv = 1;
                double rm = 0.0;
                for (int r = 0; r < R; r++) {
                    if (outer == 0) sh.mr[r].fnorm2 = sh.s1[r];
                    const double rel = sh.mr[r].fnorm2 > 0.0 ? sqrt(sh.s1[r] / sh.mr[r].fnorm2) : 0.0;
                    rm = fmax(rm, rel);
                    const bool ok = rel <= A.tol;
                    conv &= ok ? 1 : 0;
                    sh.rr_prev[r] = sh.s1[r];
                    MrRhs& m = sh.mr[r];
                    m.b1 = sqrt(sh.s2[r]);
                    m.eta = m.b1;
                    m.beta = 0.0;
                    m.c0 = m.c1 = 1.0;
                    m.s0 = m.s1 = 0.0;
                    // inner target: FP32 stops near its own precision, FP64 aims past the goal
                    const double need = rel > 0.0 ? A.tol / rel : 1.0;
                    m.target = use64 ? fmax(1e-15, 0.1 * need) : fmax(1e-5, fmin(0.5, 0.3 * need));
                    m.active = (!ok && m.b1 > 0.0) ? 1 : 0;
                    m.upd = 0;
                }
                relmax = rm;
                sh.s1[0] = rm;
                sh.conv = conv || outer >= A.max_outer;
            }
            __syncthreads();
            relmax = sh.s1[0];
            if (sh.conv) break;
            if (use64) inner_total += inner_minres<R, double>(A, n0, np, fx, base64, sh);
            else inner_total += inner_minres<R, float>(A, n0, np, fx, base32, sh);
            last64 = use64;
            if (use64) apply_correction<R, double>(A, n0, np, fx, X, base64 + 5 * A.work_stride, 1.0, nullptr);
            else apply_correction<R, float>(A, n0, np, fx, X, base32 + 5 * A.work_stride, 1.0, nullptr);
            __syncthreads();
        }
        if (tid == 0) {
            A.iters[sys] = inner_total;
            A.outers[sys] = outer;
            A.rel[sys] = relmax;
        }
        __syncthreads();
    }
}

// one persistent launch over the first n_limit systems of the queue (largest first)
template <int R>
int launch_minres(BatchSys& b, double* d_x, int start64, double tol, int maxiter, int threads, int n_limit)
{
    auto kern = k_batch_minres<R>;
    int dev = 0, sms = 0, per_sm = 0;
    MSFEM_CK(cudaGetDevice(&dev));
    MSFEM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MSFEM_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
    if (per_sm < 1) per_sm = 1;
    const int grid = std::min<int64_t>((int64_t)sms * per_sm, std::max(1, n_limit));
    const int64_t stride = (((int64_t)b.max_nodes * R * 3) + 31) / 32 * 32;
    const size_t need = (size_t)grid * 6 * stride * sizeof(double);  // room for FP64 vectors
    if (b.work.n < need) MSFEM_TRY(b.work.alloc(need));
    MSFEM_TRY(b.queue.alloc(1));
    MSFEM_CK(cudaMemsetAsync(b.queue.p, 0, sizeof(int), b.stream));
    BatchArgs a{};
    a.n_sys = n_limit;
    a.order = b.order.p;
    a.node_off = b.node_off.p;
    a.row_ptr = b.row_ptr.p;
    a.col = b.col.p;
    a.val64 = b.val64.p;
    a.val32 = b.val32.p;
    a.dscale = b.dscale.p;
    a.fixed = b.fixed.p;
    a.x = d_x;
    a.work = b.work.p;
    a.work_stride = stride;
    a.queue = b.queue.p;
    a.iters = b.iters.p;
    a.outers = b.outers.p;
    a.rel = b.rel.p;
    a.rhs = b.rhs;
    a.tol = tol;
    a.maxiter = maxiter;
    a.max_outer = 30;
    b.grid = grid;
    b.threads = threads;
    b.work_stride = stride;
    kern<<<grid, threads, 0, b.stream>>>(a, start64);
    MSFEM_CK(cudaGetLastError());
    return 0;
}

}  // namespace

int batch_build_pattern(BatchSys& b, const double* d_xyz)
{
    (void)d_xyz;
    cudaStream_t st = b.stream;
    if (b.k1 > 32 || b.n_elems >= ((int64_t)1 << (32 - 2 * tag_bits(b.k1)))) {
        set_error("batched systems: %lld elements of %d nodes exceed the contribution tags", (long long)b.n_elems, b.k1);
        return MSFEM_ERR_LIMIT;
    }
    if (b.n_nodes >= ((int64_t)1 << 31)) {
        set_error("batched systems: node count exceeds the int32 range");
        return MSFEM_ERR_LIMIT;
    }
    // element nodes inside their own system
    DBuf<int> flag;
    MSFEM_TRY(flag.alloc(1));
    MSFEM_CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    if (b.n_sys > 0) k_check_elements<<<b.n_sys, 128, 0, st>>>(b.n_sys, b.node_off.p, b.elem_off.p, b.elems.p, b.k1, flag.p);
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("batched systems: an element references a node outside its system");
        return MSFEM_ERR_ARGUMENT;
    }
    b.max_nodes = 0;
    for (int s = 0; s < b.n_sys; s++) b.max_nodes = std::max<int>(b.max_nodes, (int)(b.h_node_off[s + 1] - b.h_node_off[s]));
    const int kk = b.k1 * b.k1;
    b.n_pairs = b.n_elems * kk;
    MSFEM_TRY(b.contrib.alloc(std::max<int64_t>(1, b.n_pairs)));
    DBuf<int32_t> row_cnt;
    MSFEM_TRY(row_cnt.alloc(b.n_nodes + 1));
    MSFEM_CK(cudaMemsetAsync(row_cnt.p, 0, sizeof(int32_t) * (b.n_nodes + 1), st));

    // chunks of whole systems, at most kChunkPairs pairs each
    const int64_t kChunkPairs = (int64_t)1 << 28;
    struct Chunk {
        int64_t nslots;
        DBuf<int32_t> col;
        DBuf<int64_t> cstart;
    };
    std::vector<Chunk*> chunks;
    DBuf<uint64_t> keys[2];
    DBuf<uint32_t> tags[2];
    DBuf<int32_t> head, slot;
    DBuf<unsigned char> tmp;
    int s0 = 0;
    int rc = 0;
    while (s0 < b.n_sys && rc == 0) {
        int s1 = s0 + 1;
        while (s1 < b.n_sys && (b.h_elem_off[s1 + 1] - b.h_elem_off[s0]) * kk <= kChunkPairs) s1++;
        const int64_t e0 = b.h_elem_off[s0], e1 = b.h_elem_off[s1];
        const int64_t n0 = b.h_node_off[s0], n1 = b.h_node_off[s1];
        const int64_t P = (e1 - e0) * kk;
        if (P >= ((int64_t)1 << 31)) {
            set_error("batched systems: one system has more than 2^31 element pairs");
            rc = MSFEM_ERR_LIMIT;
            break;
        }
        auto* ch = new Chunk();
        chunks.push_back(ch);
        if (P == 0) {
            ch->nslots = 0;
            s0 = s1;
            continue;
        }
        const int nb = bits_for(n1 - n0);
        if ((rc = keys[0].alloc(P)) || (rc = keys[1].alloc(P)) || (rc = tags[0].alloc(P)) || (rc = tags[1].alloc(P)) ||
            (rc = head.alloc(P)) || (rc = slot.alloc(P)))
            break;
        const int blocks = (int)std::min<int64_t>((P + 255) / 256, 148 * 16);
        k_emit_pairs<<<blocks, 256, 0, st>>>(e0, e1, n0, nb, b.elems.p, b.k1, keys[0].p, tags[0].p);
        cub::DoubleBuffer<uint64_t> dk(keys[0].p, keys[1].p);
        cub::DoubleBuffer<uint32_t> dv(tags[0].p, tags[1].p);
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)P, 0, 2 * nb, st);
        if ((rc = tmp.alloc(std::max(tb, (size_t)1)))) break;
        MSFEM_CK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, dk, dv, (int)P, 0, 2 * nb, st));
        k_heads<<<blocks, 256, 0, st>>>(P, dk.Current(), head.p);
        size_t ts = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, ts, head.p, slot.p, (int)P, st);
        if ((rc = tmp.alloc(std::max(ts, tb)))) break;
        MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp.p, ts, head.p, slot.p, (int)P, st));
        int last_slot = 0, last_head = 0;
        MSFEM_CK(cudaMemcpyAsync(&last_slot, slot.p + P - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaMemcpyAsync(&last_head, head.p + P - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        ch->nslots = (int64_t)last_slot + last_head;
        if ((rc = ch->col.alloc(ch->nslots)) || (rc = ch->cstart.alloc(ch->nslots))) break;
        const int64_t pair_base = e0 * kk;
        k_slots<<<blocks, 256, 0, st>>>(P, dk.Current(), head.p, slot.p, n0, nb, pair_base, ch->col.p, ch->cstart.p,
                                        row_cnt.p);
        MSFEM_CK(cudaMemcpyAsync(b.contrib.p + pair_base, dv.Current(), sizeof(uint32_t) * P, cudaMemcpyDeviceToDevice, st));
        MSFEM_CK(cudaGetLastError());
        s0 = s1;
    }
    if (rc == 0) {
        int64_t total = 0;
        for (auto* ch : chunks) total += ch->nslots;
        b.nnzb = total;
        if (!(rc = b.col.alloc(std::max<int64_t>(1, total))) && !(rc = b.cstart.alloc(total + 1)) &&
            !(rc = b.row_ptr.alloc(b.n_nodes + 1))) {
            int64_t off = 0;
            for (auto* ch : chunks) {
                if (ch->nslots) {
                    cudaMemcpyAsync(b.col.p + off, ch->col.p, sizeof(int32_t) * ch->nslots, cudaMemcpyDeviceToDevice, st);
                    cudaMemcpyAsync(b.cstart.p + off, ch->cstart.p, sizeof(int64_t) * ch->nslots, cudaMemcpyDeviceToDevice, st);
                }
                off += ch->nslots;
            }
            const int64_t np = b.n_pairs;
            MSFEM_CK(cudaMemcpyAsync(b.cstart.p + total, &np, sizeof(int64_t), cudaMemcpyHostToDevice, st));
            // row_ptr = exclusive scan of the per-row block counts (64-bit)
            DBuf<int64_t> cnt64;
            if (!(rc = cnt64.alloc(b.n_nodes + 1))) {
                std::vector<int32_t> h(b.n_nodes);
                MSFEM_CK(cudaMemcpyAsync(h.data(), row_cnt.p, sizeof(int32_t) * b.n_nodes, cudaMemcpyDeviceToHost, st));
                MSFEM_CK(cudaStreamSynchronize(st));
                std::vector<int64_t> rp(b.n_nodes + 1, 0);
                for (int64_t i = 0; i < b.n_nodes; i++) rp[i + 1] = rp[i] + h[i];
                if (rp[b.n_nodes] != total) {
                    set_error("batched systems: row counts (%lld) disagree with the block count (%lld)",
                              (long long)rp[b.n_nodes], (long long)total);
                    rc = MSFEM_ERR_STATE;
                } else {
                    MSFEM_CK(cudaMemcpyAsync(b.row_ptr.p, rp.data(), sizeof(int64_t) * (b.n_nodes + 1),
                                             cudaMemcpyHostToDevice, st));
                    MSFEM_CK(cudaStreamSynchronize(st));
                }
            }
        }
    }
    MSFEM_CK(cudaStreamSynchronize(st));
    for (auto* ch : chunks) delete ch;
    if (rc) return rc;
    // largest systems first
    std::vector<int32_t> ord(b.n_sys);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) {
        return b.h_node_off[a + 1] - b.h_node_off[a] > b.h_node_off[c + 1] - b.h_node_off[c];
    });
    MSFEM_TRY(b.order.alloc(std::max(1, b.n_sys)));
    if (b.n_sys) MSFEM_CK(cudaMemcpyAsync(b.order.p, ord.data(), sizeof(int32_t) * b.n_sys, cudaMemcpyHostToDevice, st));
    MSFEM_TRY(b.iters.alloc(std::max(1, b.n_sys)));
    MSFEM_TRY(b.outers.alloc(std::max(1, b.n_sys)));
    MSFEM_TRY(b.rel.alloc(std::max(1, b.n_sys)));
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

int batch_assemble_enqueue(BatchSys& b, const double* d_xyz, const double* d_lame, int n_mat)
{
    cudaStream_t st = b.stream;
    MSFEM_TRY(b.val64.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
    MSFEM_TRY(b.val32.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
    MSFEM_TRY(b.dscale.alloc(std::max<int64_t>(1, 3 * b.n_nodes)));
    DBuf<int>& flag = b.aflag;
    MSFEM_TRY(flag.alloc(1));
    MSFEM_CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    const int blocks = (int)std::min<int64_t>((b.nnzb + 255) / 256, 148 * 16);
    if (b.nnzb) {
        if (b.k1 == 4)
            k_assemble_blocks<4><<<blocks, 256, 0, st>>>(b.nnzb, b.cstart.p, b.contrib.p, b.elems.p, b.emat.p, d_xyz,
                                                         d_lame, n_mat, b.val64.p, flag.p);
        else
            k_assemble_blocks<3><<<blocks, 256, 0, st>>>(b.nnzb, b.cstart.p, b.contrib.p, b.elems.p, b.emat.p, d_xyz,
                                                         d_lame, n_mat, b.val64.p, flag.p);
    }
    const int nblk = (int)std::min<int64_t>((b.n_nodes + 255) / 256, 148 * 16);
    if (b.n_nodes) {
        k_batch_scale<<<nblk, 256, 0, st>>>(b.n_nodes, b.row_ptr.p, b.col.p, b.val64.p, b.dscale.p);
        k_batch_val32<<<nblk, 256, 0, st>>>(b.n_nodes, b.row_ptr.p, b.col.p, b.val64.p, b.dscale.p, b.val32.p);
    }
    MSFEM_CK(cudaGetLastError());
    return 0;
}

int batch_assemble(BatchSys& b, const double* d_xyz, const double* d_lame, int n_mat)
{
    MSFEM_TRY(batch_assemble_enqueue(b, d_xyz, d_lame, n_mat));
    cudaStream_t st = b.stream;
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, b.aflag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("batched systems: material id out of range");
        return MSFEM_ERR_ARGUMENT;
    }
    return 0;
}

int batch_assemble_given(BatchSys& b, const double* d_eblocks, bool scaled)
{
    cudaStream_t st = b.stream;
    MSFEM_TRY(b.val64.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
    if (scaled) {
        MSFEM_TRY(b.val32.alloc(std::max<int64_t>(1, 9 * b.nnzb)));
        MSFEM_TRY(b.dscale.alloc(std::max<int64_t>(1, 3 * b.n_nodes)));
    }
    const int blocks = (int)std::min<int64_t>((b.nnzb + 255) / 256, 148 * 16);
    if (b.nnzb)
        k_assemble_given<<<blocks, 256, 0, st>>>(b.nnzb, b.cstart.p, b.contrib.p, b.k1, d_eblocks, b.val64.p);
    const int nblk = (int)std::min<int64_t>((b.n_nodes + 255) / 256, 148 * 16);
    if (scaled && b.n_nodes) {
        k_batch_scale<<<nblk, 256, 0, st>>>(b.n_nodes, b.row_ptr.p, b.col.p, b.val64.p, b.dscale.p);
        k_batch_val32<<<nblk, 256, 0, st>>>(b.n_nodes, b.row_ptr.p, b.col.p, b.val64.p, b.dscale.p, b.val32.p);
    }
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

namespace {

int launch_any(BatchSys& b, double* d_x, int start64, double tol, int maxiter, int threads, int n_limit)
{
    switch (b.R) {
    case 4: return launch_minres<4>(b, d_x, start64, tol, maxiter, threads, n_limit);
    case 8: return launch_minres<8>(b, d_x, start64, tol, maxiter, threads, n_limit);
    case 1: return launch_minres<1>(b, d_x, start64, tol, maxiter, threads, n_limit);
    default:
        set_error("batched solve: %d right-hand sides per system (1, 4 or 8 supported)", b.R);
        return MSFEM_ERR_ARGUMENT;
    }
}

// Autotuner of the persistent launch: the CTA size (threads per system) decides how many
// row-rhs pairs a pass covers and how many CTAs fit per SM.  Each candidate solves the same
// sample -- the 2 x #SM largest systems, which dominate the batch's time -- from the same start
// (x is saved and restored around each trial), timed with CUDA events; the fastest is kept for
// this batch.  Batches smaller than the sample are not timed (the choice hardly matters there).
int autotune(BatchSys& b, double* d_x, int start64, double tol, int maxiter)
{
    int dev = 0, sms = 0;
    MSFEM_CK(cudaGetDevice(&dev));
    MSFEM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int sample = 2 * sms;
    b.tune_ms.clear();
    if (b.n_sys < 2 * sample) {
        b.tuned_threads = 256;
        return 0;
    }
    const size_t nx = (size_t)b.n_nodes * b.R * 3;
    DBuf<double> save;
    MSFEM_TRY(save.alloc(nx));
    MSFEM_CK(cudaMemcpyAsync(save.p, d_x, sizeof(double) * nx, cudaMemcpyDeviceToDevice, b.stream));
    cudaEvent_t e0, e1;
    MSFEM_CK(cudaEventCreate(&e0));
    MSFEM_CK(cudaEventCreate(&e1));
    const int cand[] = {128, 256, 384, 512};
    float best = 0.f;
    int best_t = 256;
    for (int t : cand) {
        MSFEM_CK(cudaMemcpyAsync(d_x, save.p, sizeof(double) * nx, cudaMemcpyDeviceToDevice, b.stream));
        MSFEM_CK(cudaEventRecord(e0, b.stream));
        MSFEM_TRY(launch_any(b, d_x, start64, tol, maxiter, t, sample));
        MSFEM_CK(cudaEventRecord(e1, b.stream));
        MSFEM_CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        MSFEM_CK(cudaEventElapsedTime(&ms, e0, e1));
        b.tune_ms.push_back(ms);
        if (b.tune_ms.size() == 1 || ms < best) {
            best = ms;
            best_t = t;
        }
    }
    MSFEM_CK(cudaMemcpyAsync(d_x, save.p, sizeof(double) * nx, cudaMemcpyDeviceToDevice, b.stream));
    MSFEM_CK(cudaStreamSynchronize(b.stream));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b.tuned_threads = best_t;
    return 0;
}

}  // namespace

int batch_threads(const BatchSys& b, int precision, int threads)
{
    if (b.n_sys == 0) return 256;
    if (threads > 0) return threads;
    return (b.tuned_threads != 0 && b.tuned_precision == precision) ? b.tuned_threads : 0;
}

int batch_solve(BatchSys& b, double* d_x, int precision, double tol, int maxiter, int threads)
{
    if (b.n_sys == 0) return 0;
    const int start64 = precision == MSFEM_FP32_IR ? 0 : 1;
    if (threads <= 0) {
        if (b.tuned_threads == 0 || b.tuned_precision != precision) {
            MSFEM_TRY(autotune(b, d_x, start64, tol, maxiter));
            b.tuned_precision = precision;
        }
        threads = b.tuned_threads;
    }
    if (threads % 32 != 0 || threads > 512) {
        set_error("batched solve: threads per system must be a multiple of 32, at most 512");
        return MSFEM_ERR_ARGUMENT;
    }
    return launch_any(b, d_x, start64, tol, maxiter, threads, b.n_sys);
}

}  // namespace msfem
