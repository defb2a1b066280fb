// Two-level preconditioner with the MsFEM coarse space, and the preconditioned
// MINRES around it (FP32 inner solves inside FP64 iterative refinement).
//
// Coarse space.  The Order1 bases of the macro cells (cells.cu; MsFEM/MsFEM_Grid.h:
// 4795-5759) give the prolongation P: coarse DOF (vertex V, component a) -> fine
// DOF (node g, a) with value psi_V^a(g), the a-component of the cell basis of V
// (the reference uses the components this way in FiniteElement_forMech_Poly_Order1::
// SolveLocalMatrix, MsFEM_Grid.h:3837-3975).  A fine node on a face, edge or corner
// shared by several cells takes the mean of the cells' values; P is zero on the
// Dirichlet DOFs of the fine problem, and coarse DOFs whose vertex carries a fine
// Dirichlet DOF are dropped.
//
// Coarse operator.  The reference's element blocks make the fine matrix A
// symmetric but indefinite; a Galerkin operator P^T A P is indefinite too and
// cannot define an SPD preconditioner (MINRES needs one).  The coarse operator is
// therefore the Galerkin product of the textbook (SPD) orientation of the same
// element blocks, A_c = P^T K P with K[I][J][a][b] = V (lambda gI_a gJ_b +
// mu gJ_a gI_b + mu delta_ab gI.gJ) -- the reference's blocks transposed --
// assembled cell by cell from the fine tetrahedra (24 x 24 per cell, summed in
// element order), then into a dense matrix colour by colour (cells of one colour
// share no vertex, so every entry receives its cell terms in a fixed order).
// A_c is inverted in FP64 by the block sweep operator with Cholesky-factored
// 64 x 64 pivots, and applied in FP32 as a dense matrix-vector product.
//
// Preconditioner (on the Jacobi-scaled system S A S, S = D^-1/2):
//   M^-1 = I + P^ A_c^-1 P^^T,  P^ = S^-1 P,
// i.e. diag(A)^-1 + P A_c^-1 P^T in the original unknowns: SPD.
//
// Preconditioned MINRES (Paige & Saunders 1975, in the form of their SYMMLQ/MINRES
// report with a preconditioner): per iteration one SpMV, one preconditioner
// application (restriction per cell -> coarse gather -> dense GEMV -> prolongation)
// and two inner products, in six kernels captured as a CUDA graph.
#include <cub/cub.cuh>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <new>
#include <numeric>

#include "cells.cuh"
#include "devutil.cuh"
#include "element.cuh"
#include "internal.cuh"
#include "kuhn_op.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

constexpr int kSB = 64;            // sweep pivot block
constexpr int kCoarseThreads = 576;  // one thread per entry of a 24 x 24 cell matrix
constexpr int kTetBatch = 8;

struct TlState {
    double alfa, beta, oldb, dbar, epsln, oldeps, phibar, cs, sn, phi, delta, gamma, denom, beta1, tol, bb;
    int iter, maxiter, done, applied;
    unsigned int ticket[4];
};

inline unsigned gridn(int64_t n, int t = 256)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + t - 1) / t, 148 * 32));
}

// ---- setup kernels

__global__ void k_batch_cell(int n_cells, const int64_t* __restrict__ node_off, int32_t* __restrict__ bcell)
{
    const int c = blockIdx.x;
    for (int64_t b = node_off[c] + threadIdx.x; b < node_off[c + 1]; b += blockDim.x) bcell[b] = c;
}

__global__ void k_inc_heads(int64_t n, const int32_t* __restrict__ key, int32_t* __restrict__ inc_ptr, int n_fine, int* bad)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = key[i];
        if (k < 0 || k >= n_fine) {
            atomicExch(bad, 1);
            continue;
        }
        if (i == 0 || key[i - 1] != k) inc_ptr[k] = (int32_t)i;
        if (i == n - 1) inc_ptr[n_fine] = (int32_t)n;
    }
}

// every fine node must appear: inc_ptr[g] was preset to -1
__global__ void k_inc_fill(int n_fine, int32_t* __restrict__ inc_ptr, int* bad)
{
    // a node that no cell holds is an error; fill from the right so that gaps would be visible
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n_fine; g += gridDim.x * blockDim.x)
        if (inc_ptr[g] < 0) atomicExch(bad, 2);
}

// cells whose bases leave [-kWildBasis, kWildBasis]: the reference's cell operator is indefinite,
// and a nearly singular cell problem returns bases in the thousands, which would wreck the
// conditioning of the coarse matrix (and the SPD-ness of its FP32 inverse)
constexpr double kWildBasis = 3.0;
__global__ void k_wild_cells(const int64_t* __restrict__ node_off, const double* __restrict__ bases, uint8_t* __restrict__ wild)
{
    const int c = blockIdx.x;
    int bad = 0;
    for (int64_t q = 24 * node_off[c] + threadIdx.x; q < 24 * node_off[c + 1]; q += blockDim.x) {
        const double b = bases[q];
        bad |= !(fabs(b) <= kWildBasis);
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) wild[c] = (uint8_t)(bad != 0);
}

// psi_cell[b][v][a]: mean over the cells holding the fine node of b of their basis of the
// coarse vertex cell_vertex[c][v]; zero on fine Dirichlet DOFs and dropped coarse DOFs
__global__ void k_psi_cell(int64_t n_batch, const int32_t* __restrict__ bcell, const int32_t* __restrict__ cng,
                           const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc_b,
                           const int32_t* __restrict__ cell_vertex, const int32_t* __restrict__ cdof,
                           const uint8_t* __restrict__ fixed3, const double* __restrict__ bases,
                           const uint8_t* __restrict__ wild, const double* __restrict__ box,
                           const double* __restrict__ cxyz, double* __restrict__ psi)
{
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < n_batch; b += (int64_t)gridDim.x * blockDim.x) {
        const int c = bcell[b];
        const int g = cng[b];
        const int e0 = inc_ptr[g], e1 = inc_ptr[g + 1];
        const double inv = 1.0 / (double)(e1 - e0);
        for (int v = 0; v < 8; v++) {
            const int V = cell_vertex[8 * c + v];
            double acc[3] = {0, 0, 0};
            for (int e = e0; e < e1; e++) {
                const int b2 = inc_b[e];
                const int c2 = bcell[b2];
                for (int v2 = 0; v2 < 8; v2++)
                    if (cell_vertex[8 * c2 + v2] == V) {
                        if (wild[c2]) {
                            // trilinear function of the cell box in place of wild bases
                            double q = 1.0;
                            for (int d = 0; d < 3; d++) {
                                const double lo = box[6 * c2 + 2 * d], hi = box[6 * c2 + 2 * d + 1];
                                const double t = (cxyz[3 * (int64_t)b2 + d] - lo) / (hi - lo);
                                q *= ((v2 >> d) & 1) ? t : 1.0 - t;
                            }
                            for (int a = 0; a < 3; a++) acc[a] += q;
                        } else {
                            for (int a = 0; a < 3; a++) acc[a] += bases[24 * (int64_t)b2 + 3 * v2 + a];
                        }
                        break;
                    }
            }
            for (int a = 0; a < 3; a++) {
                const bool keep = !fixed3[3 * (int64_t)g + a] && cdof[24 * c + 3 * v + a] >= 0;
                psi[24 * b + 3 * v + a] = keep ? acc[a] * inv : 0.0;
            }
        }
    }
}

// per fine node: owner cell (the cell of its first incidence) and the scaled prolongation row
__global__ void k_psi_hat(int n_fine, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc_b,
                          const int32_t* __restrict__ bcell, const double* __restrict__ psi,
                          const double* __restrict__ dscale, int32_t* __restrict__ owner, float* __restrict__ psi_hat)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n_fine; g += gridDim.x * blockDim.x) {
        const int b = inc_b[inc_ptr[g]];
        owner[g] = bcell[b];
        for (int j = 0; j < 24; j++) {
            const int a = j % 3;
            psi_hat[24 * (int64_t)g + j] = (float)(psi[24 * (int64_t)b + j] / dscale[3 * (int64_t)g + a]);
        }
    }
}

// cell coarse matrices K_c = sum_e P_e^T K_e P_e (textbook element blocks), 576 threads per cell
__global__ void __launch_bounds__(kCoarseThreads) k_coarse_cells(const int64_t* __restrict__ elem_off,
                                                                  const int32_t* __restrict__ elems,
                                                                  const int32_t* __restrict__ emat,
                                                                  const double* __restrict__ xyz,
                                                                  const double* __restrict__ lame, int n_mat,
                                                                  const double* __restrict__ psi, double* __restrict__ Kc,
                                                                  int* bad)
{
    __shared__ double s_g[kTetBatch][4][3];
    __shared__ double s_c[kTetBatch][3];  // meas, lambda, mu
    __shared__ double s_psi[kTetBatch][4][24];
    __shared__ double s_T[kTetBatch][12][24];
    const int c = blockIdx.x, tid = threadIdx.x;
    const int p = tid / 24, q = tid % 24;  // entry (v a) x (w b)
    const int pa = p % 3;
    double acc = 0.0;
    const int64_t t0 = elem_off[c], t1 = elem_off[c + 1];
    for (int64_t base = t0; base < t1; base += kTetBatch) {
        const int nb = (int)min((int64_t)kTetBatch, t1 - base);
        __syncthreads();
        if (tid < nb) {
            const int64_t e = base + tid;
            int v[4];
            for (int k = 0; k < 4; k++) v[k] = elems[4 * e + k];
            TetGeom G;
            tet_geometry(xyz, v, G);
            for (int k = 0; k < 4; k++)
                for (int a = 0; a < 3; a++) s_g[tid][k][a] = G.g[k][a];
            const int m = emat ? emat[e] : 0;
            if (m < 0 || m >= n_mat) atomicExch(bad, 1);
            const int mm = (m < 0 || m >= n_mat) ? 0 : m;
            s_c[tid][0] = G.vol;
            s_c[tid][1] = lame[2 * mm];
            s_c[tid][2] = lame[2 * mm + 1];
        }
        for (int i = tid; i < nb * 96; i += blockDim.x) {
            const int t = i / 96, r = i % 96, k = r / 24, j = r % 24;
            const int64_t node = elems[4 * (base + t) + k];
            s_psi[t][k][j] = psi[24 * node + j];
        }
        __syncthreads();
        // T[t][I a][w b] = sum_J K_e[I][J][a][b] psi[J][w b]
        for (int i = tid; i < nb * 288; i += blockDim.x) {
            const int t = i / 288, r = i % 288, Ia = r / 24, wb = r % 24;
            const int I = Ia / 3, a = Ia % 3, b = wb % 3;
            const double meas = s_c[t][0], lam = s_c[t][1], mu = s_c[t][2];
            double sum = 0.0;
            for (int J = 0; J < 4; J++) {
                const double* gi = s_g[t][I];
                const double* gj = s_g[t][J];
                double k = lam * gi[a] * gj[b] + mu * gj[a] * gi[b];
                if (a == b) k += mu * (gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]);
                sum += meas * k * s_psi[t][J][wb];
            }
            s_T[t][Ia][wb] = sum;
        }
        __syncthreads();
        for (int t = 0; t < nb; t++)
            for (int I = 0; I < 4; I++) acc += s_psi[t][I][p] * s_T[t][3 * I + pa][q];
    }
    Kc[576 * (int64_t)c + tid] = acc;
}

// add the cell matrices of one colour into the dense coarse matrix
__global__ void k_coarse_scatter(int n_sel, const int32_t* __restrict__ cells, const double* __restrict__ Kc,
                                 const int32_t* __restrict__ cdof, double* __restrict__ A, int64_t ld)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)n_sel * 576;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int c = cells[t / 576];
        const int e = (int)(t % 576), p = e / 24, q = e % 24;
        const int dp = cdof[24 * c + p], dq = cdof[24 * c + q];
        if (dp >= 0 && dq >= 0) A[dp * ld + dq] += Kc[576 * (int64_t)c + e];
    }
}

__global__ void k_sym_pad(double* __restrict__ A, int64_t ld, int n, int n_pad)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)n_pad * n_pad;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / n_pad), j = (int)(t % n_pad);
        if (i >= n || j >= n) {
            A[i * ld + j] = (i == j) ? 1.0 : 0.0;
        } else if (i < j) {
            const double m = 0.5 * (A[i * ld + j] + A[j * ld + i]);
            A[i * ld + j] = m;
            A[j * ld + i] = m;
        }
    }
}

// ---- block sweep: A <- A with pivot block K swept; after all blocks A = -A0^-1

// Pinv = A[K][K]^-1 via Cholesky in shared memory (one CTA)
__global__ void __launch_bounds__(256) k_sweep_pivot(const double* __restrict__ A, int64_t ld, int k0,
                                                     double* __restrict__ Pinv, int* bad)
{
    extern __shared__ double psm[];
    double(*L)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(psm);
    double(*W)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(psm + kSB * (kSB + 1));
    const int tid = threadIdx.x;
    for (int i = tid; i < kSB * kSB; i += blockDim.x) L[i / kSB][i % kSB] = A[(int64_t)(k0 + i / kSB) * ld + k0 + i % kSB];
    __syncthreads();
    // right-looking Cholesky, lower triangle
    for (int j = 0; j < kSB; j++) {
        if (tid == 0) {
            const double d = L[j][j];
            if (!(d > 0.0)) atomicExch(bad, 1);
            L[j][j] = d > 0.0 ? sqrt(d) : 1.0;
        }
        __syncthreads();
        const double djj = L[j][j];
        for (int i = j + 1 + tid; i < kSB; i += blockDim.x) L[i][j] /= djj;
        __syncthreads();
        for (int t = tid; t < (kSB - j - 1) * (kSB - j - 1); t += blockDim.x) {
            const int i = j + 1 + t / (kSB - j - 1), c = j + 1 + t % (kSB - j - 1);
            if (c <= i) L[i][c] -= L[i][j] * L[c][j];
        }
        __syncthreads();
    }
    // W = L^-1 (lower), column by column: one thread per column
    if (tid < kSB) {
        const int c = tid;
        for (int i = 0; i < kSB; i++) {
            if (i < c) {
                W[i][c] = 0.0;
                continue;
            }
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = c; k < i; k++) s -= L[i][k] * W[k][c];
            W[i][c] = s / L[i][i];
        }
    }
    __syncthreads();
    // Pinv = W^T W
    for (int t = tid; t < kSB * kSB; t += blockDim.x) {
        const int i = t / kSB, j = t % kSB;
        double s = 0.0;
        for (int k = max(i, j); k < kSB; k++) s += W[k][i] * W[k][j];
        Pinv[t] = s;
    }
}

// Bp = A[:, K] (old panel), Cp = Bp * Pinv.  Only the upper block triangle of A is kept up to date
// (the swept matrix stays symmetric): rows below the pivot block read the panel from its mirror,
// A[i][K] = A[K][i].
__global__ void __launch_bounds__(256) k_sweep_panel(const double* __restrict__ A, int64_t ld, int n, int k0,
                                                     const double* __restrict__ Pinv, double* __restrict__ Bp,
                                                     double* __restrict__ Cp)
{
    __shared__ double P[kSB][kSB];
    __shared__ double a[4][kSB];
    for (int t = threadIdx.x; t < kSB * kSB; t += blockDim.x) P[t / kSB][t % kSB] = Pinv[t];
    const int r = threadIdx.x / 64, j = threadIdx.x % 64;
    const int row = blockIdx.x * 4 + r;  // 4 rows per CTA, 64 threads per row
    if (row < n) a[r][j] = row < k0 + kSB ? A[(int64_t)row * ld + k0 + j] : A[(int64_t)(k0 + j) * ld + row];
    __syncthreads();
    if (row >= n) return;
    Bp[(int64_t)row * kSB + j] = a[r][j];
    double s = 0.0;
    for (int k = 0; k < kSB; k++) s += a[r][k] * P[k][j];
    Cp[(int64_t)row * kSB + j] = s;
}

// upper tile (I, J), I <= J, of 64 x 64 (one CTA per entry of `tiles`): A_IJ -= C_I B_J^T off the
// pivot block row/column; the pivot row/column take C, the pivot block -Pinv
__global__ void __launch_bounds__(256) k_sweep_update(double* __restrict__ A, int64_t ld, int kb,
                                                      const int2* __restrict__ tiles,
                                                      const double* __restrict__ Pinv, const double* __restrict__ Bp,
                                                      const double* __restrict__ Cp)
{
    extern __shared__ double sm[];
    double* Cs = sm;                 // [64][65]
    double* Bs = sm + kSB * (kSB + 1);  // [64][65]
    const int I = tiles[blockIdx.x].x, J = tiles[blockIdx.x].y;
    const int tid = threadIdx.x;
    const int64_t i0 = (int64_t)I * kSB, j0 = (int64_t)J * kSB;
    if (I == kb && J == kb) {
        for (int t = tid; t < kSB * kSB; t += blockDim.x) A[(i0 + t / kSB) * ld + j0 + t % kSB] = -Pinv[t];
        return;
    }
    if (J == kb) {  // column panel: C_I
        for (int t = tid; t < kSB * kSB; t += blockDim.x) A[(i0 + t / kSB) * ld + j0 + t % kSB] = Cp[(i0 + t / kSB) * kSB + t % kSB];
        return;
    }
    if (I == kb) {  // row panel: C_J^T
        for (int t = tid; t < kSB * kSB; t += blockDim.x) A[(i0 + t / kSB) * ld + j0 + t % kSB] = Cp[(j0 + t % kSB) * kSB + t / kSB];
        return;
    }
    for (int t = tid; t < kSB * kSB; t += blockDim.x) {
        const int r = t / kSB, k = t % kSB;
        Cs[r * (kSB + 1) + k] = Cp[(i0 + r) * kSB + k];
        Bs[r * (kSB + 1) + k] = Bp[(j0 + r) * kSB + k];
    }
    __syncthreads();
    const int tr = tid / 16, tc = tid % 16;  // 4 x 4 outputs per thread
    double acc[4][4] = {};
    for (int k = 0; k < kSB; k++) {
        double cr[4], bc[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            cr[u] = Cs[(tr + 16 * u) * (kSB + 1) + k];
            bc[u] = Bs[(tc + 16 * u) * (kSB + 1) + k];
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int w = 0; w < 4; w++) acc[u][w] += cr[u] * bc[w];
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int w = 0; w < 4; w++) A[(i0 + tr + 16 * u) * ld + j0 + tc + 16 * w] -= acc[u][w];
}

// The coarse inverse is symmetric: only its upper 64 x 64 blocks (I <= J) are stored, packed row by
// row of blocks, each block row-major, FP32 (half the bytes of the dense matrix).  ec = Cinv rc is
// one CTA per stored block -- the block times rc_J gives block row I's share, its transpose times
// rc_I (I < J) block row J's share -- into a partial per (block row, block column), then a fixed-
// order sum over the block columns.
constexpr int kSymB = 64;

// pack -A (the swept matrix, FP64, leading dimension ld) into the upper blocks; zero past n
__global__ void k_pack_sym(const double* __restrict__ A, int64_t ld, int n, const int2* __restrict__ blocks,
                           int n_blocks, float* __restrict__ P)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)n_blocks * kSymB * kSymB;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / (kSymB * kSymB);
        const int e = (int)(t - b * kSymB * kSymB), r = e / kSymB, c = e % kSymB;
        const int i = blocks[b].x * kSymB + r, j = blocks[b].y * kSymB + c;
        P[t] = (i < n && j < n) ? (float)(-A[(int64_t)i * ld + j]) : 0.0f;
    }
}

// per stored block (I, J): part[I][J] = C_IJ x_J and, for I < J, part[J][I] = C_IJ^T x_I.  The
// block's 1024 float4 chunks are read by consecutive threads (warp loads of 512 contiguous bytes):
// thread t holds rows t/16 + 16k (k = 0..3), columns 4 (t%16) .. +3.  Row sums reduce over the 16
// lanes of a row, column sums over the lane pair (l, l+16) and then the 8 warps in shared memory,
// in fixed orders.  Persistent: CTA c takes blocks c, c + grid, ...
__global__ void __launch_bounds__(256) k_tl_symv(int nb, int n_blocks, const int2* __restrict__ blocks,
                                                 const float* __restrict__ P, const float* __restrict__ x,
                                                 float* __restrict__ part, const TlState* S)
{
    if (S->done) return;
    __shared__ float colp[8][kSymB];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int cq = t & 15, r0 = t >> 4;
    // the next block's chunks are loaded while this one is reduced: two blocks in flight per thread
    float4 a[4], an[4];
    if (blockIdx.x < n_blocks) {
        const float4* blk = reinterpret_cast<const float4*>(P + (int64_t)blockIdx.x * kSymB * kSymB);
#pragma unroll
        for (int k = 0; k < 4; k++) an[k] = __ldcs(blk + t + 256 * k);
    }
    for (int b = blockIdx.x; b < n_blocks; b += gridDim.x) {
        const int I = blocks[b].x, J = blocks[b].y;
#pragma unroll
        for (int k = 0; k < 4; k++) a[k] = an[k];
        if (b + (int)gridDim.x < n_blocks) {
            const float4* nxt = reinterpret_cast<const float4*>(P + (int64_t)(b + gridDim.x) * kSymB * kSymB);
#pragma unroll
            for (int k = 0; k < 4; k++) an[k] = __ldcs(nxt + t + 256 * k);
        }
        const float4 xq = __ldg(reinterpret_cast<const float4*>(x + J * kSymB) + cq);
        float xi[4];
#pragma unroll
        for (int k = 0; k < 4; k++) xi[k] = x[I * kSymB + r0 + 16 * k];
        float rs[4], cs[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            rs[k] = a[k].x * xq.x + a[k].y * xq.y + a[k].z * xq.z + a[k].w * xq.w;
            cs[0] += a[k].x * xi[k];
            cs[1] += a[k].y * xi[k];
            cs[2] += a[k].z * xi[k];
            cs[3] += a[k].w * xi[k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) rs[k] += __shfl_xor_sync(0xffffffffu, rs[k], o);
        }
        if (cq == 0)
#pragma unroll
            for (int k = 0; k < 4; k++) part[((int64_t)I * nb + J) * kSymB + r0 + 16 * k] = rs[k];
        if (I == J) continue;  // uniform across the CTA
#pragma unroll
        for (int c = 0; c < 4; c++) cs[c] += __shfl_xor_sync(0xffffffffu, cs[c], 16);
        if (lane < 16)
#pragma unroll
            for (int c = 0; c < 4; c++) colp[warp][4 * cq + c] = cs[c];
        __syncthreads();
        if (t < kSymB) {
            float w = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; k++) w += colp[k][t];
            part[((int64_t)J * nb + I) * kSymB + t] = w;
        }
        __syncthreads();
    }
}

// y[i] = sum over block columns K of part[i / 64][K][i % 64], K ascending
__global__ void k_tl_symv_sum(int n_pad, int nb, const float* __restrict__ part, float* __restrict__ y,
                              const TlState* S)
{
    if (S->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const int I = i / kSymB, r = i % kSymB;
    const float* p = part + (int64_t)I * nb * kSymB + r;
    float v = 0.0f;
    for (int K = 0; K < nb; K++) v += p[(int64_t)K * kSymB];
    y[i] = v;
}

// ---- preconditioner application kernels (FP32)

// per cell: restriction partials over its owned nodes, cpart[c][v a] = sum psi_hat[g][v a] q[g a],
// q = r (scaled FP32 system) or s r (FP64 in the original unknowns, s = D^-1/2);
// with `lanczos`, r is first formed as r_new = z - (alfa / beta) r2 and written over `out`
template <class VT>
__global__ void __launch_bounds__(128) k_tl_restrict(const int32_t* __restrict__ own_ptr, const int32_t* __restrict__ own,
                                                     const float* __restrict__ psi_hat, const VT* __restrict__ z,
                                                     const VT* __restrict__ r2, VT* __restrict__ out,
                                                     float* __restrict__ cpart, const double* __restrict__ s,
                                                     const TlState* S, int lanczos)
{
    if (S->done) return;
    __shared__ VT red[4][24];
    const int c = blockIdx.x;
    const VT coef = lanczos ? (VT)(S->alfa / S->beta) : (VT)0;
    VT acc[24];
#pragma unroll
    for (int j = 0; j < 24; j++) acc[j] = 0;
    for (int k = own_ptr[c] + threadIdx.x; k < own_ptr[c + 1]; k += blockDim.x) {
        const int64_t g = own[k];
        VT rv[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            VT r = z[3 * g + a];
            if (lanczos) {
                r -= coef * r2[3 * g + a];
                out[3 * g + a] = r;
            }
            rv[a] = s ? (VT)(s[3 * g + a] * (double)r) : r;
        }
        float ph[24];  // 96 bytes per node, 16-byte aligned: six float4 loads
        const float4* p4 = reinterpret_cast<const float4*>(psi_hat + 24 * g);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const float4 t = __ldg(p4 + q);
            ph[4 * q] = t.x;
            ph[4 * q + 1] = t.y;
            ph[4 * q + 2] = t.z;
            ph[4 * q + 3] = t.w;
        }
#pragma unroll
        for (int j = 0; j < 24; j++) acc[j] += (VT)ph[j] * rv[j % 3];
    }
    // block reduction of 24 values (fixed order)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 24; j++) {
        VT v = acc[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < 24) {
        VT v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
        cpart[24 * c + threadIdx.x] = (float)v;
    }
}

// coarse residual: rc[d] = sum of the cell partials of coarse DOF d (fixed order)
__global__ void k_tl_gather(int n_cf, const int32_t* __restrict__ dptr, const int32_t* __restrict__ dent,
                            const float* __restrict__ cpart, float* __restrict__ rc, const TlState* S)
{
    if (S->done) return;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n_cf; d += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int e = dptr[d]; e < dptr[d + 1]; e++) s += cpart[dent[e]];
        rc[d] = s;
    }
}


// bb = (r, M^-1 r) of the new Lanczos vector: beta' = sqrt(bb) and the MINRES Givens step;
// init: the first application (beta1).  One thread.
__device__ void givens_step(TlState* S, double bb, int init)
{
    if (init) {
        const double b1 = bb > 0.0 ? sqrt(bb) : 0.0;
        S->beta1 = b1;
        S->beta = b1;
        S->oldb = 0.0;
        S->phibar = b1;
        S->dbar = 0.0;
        S->epsln = 0.0;
        S->cs = -1.0;
        S->sn = 0.0;
        S->iter = 0;
        S->applied = -1;
        S->done = (b1 > 0.0) ? 0 : 1;
        return;
    }
    const double beta = bb > 0.0 ? sqrt(bb) : 0.0;
    S->oldb = S->beta;
    S->beta = beta;
    S->oldeps = S->epsln;
    const double delta = S->cs * S->dbar + S->sn * S->alfa;
    const double gbar = S->sn * S->dbar - S->cs * S->alfa;
    S->epsln = S->sn * beta;
    S->dbar = -S->cs * beta;
    double gamma = sqrt(gbar * gbar + beta * beta);
    if (!(gamma > 1e-300)) gamma = 1e-300;
    S->cs = gbar / gamma;
    S->sn = beta / gamma;
    S->phi = S->cs * S->phibar;
    S->phibar = S->sn * S->phibar;
    S->delta = delta;
    S->gamma = gamma;
    S->denom = 1.0 / gamma;
    S->iter += 1;
    if (!(bb == bb)) S->done = 3;
    else if (fabs(S->phibar) <= S->tol * S->beta1 || !(beta > 0.0)) S->done = 1;
    else if (S->iter >= S->maxiter) S->done = 2;
}

// y = r + P^ ec (scaled FP32 system) or y = s^2 r + s P^ ec (FP64, original unknowns); bb = (r, y);
// the last block updates the Givens recurrence.  init: first application (beta1 = sqrt(bb)).
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_tl_prolong(int n_fine, const int32_t* __restrict__ owner,
                                                           const int32_t* __restrict__ cdof,
                                                           const float* __restrict__ psi_hat,
                                                           const float* __restrict__ ec, const VT* __restrict__ r,
                                                           VT* __restrict__ y, const double* __restrict__ s, TlState* S,
                                                           double* __restrict__ partial, int init)
{
    if (S->done) return;
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_fine; g += (int64_t)gridDim.x * blockDim.x) {
        const int c = owner[g];
        const int32_t* cd = cdof + 24 * c;
        const float* ph = psi_hat + 24 * g;
        float z[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int j = 0; j < 24; j++) {
            const int d = cd[j];
            if (d >= 0) z[j % 3] += ph[j] * ec[d];
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const VT ra = r[3 * g + a];
            VT ya;
            if (s) {
                const double sa = s[3 * g + a];
                ya = (VT)(sa * sa * (double)ra + sa * (double)z[a]);
            } else {
                ya = ra + (VT)z[a];
            }
            y[3 * g + a] = ya;
            acc[0] += (double)ra * (double)ya;
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            givens_step(S, t[0], init);
            S->ticket[0] = 0;
        }
    }
}

// v = y / beta; z = (S A S) y / beta - (beta / oldb) r1 (after the first step); alfa = (v, z)
template <class VT>
__global__ void __launch_bounds__(256) k_tl_spmv(SellView<VT> A, const VT* __restrict__ y, VT* __restrict__ v,
                                                 VT* __restrict__ z, const VT* __restrict__ r1, TlState* S,
                                                 double* __restrict__ partial)
{
    if (S->done) return;
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const VT inv = (VT)(1.0 / S->beta);
    const VT coef = S->iter > 0 ? (VT)(S->beta / S->oldb) : (VT)0;
    double acc[1] = {0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        VT yv[3];
        sell_row_block<VT>(A, warp, lane, y, yv);
        const int brow = warp * kSlice + lane;
        if (brow < A.n_brows)
            for (int c = 0; c < 3; c++) {
                const int64_t i = 3 * (int64_t)brow + c;
                const VT vi = y[i] * inv;
                const VT zi = yv[c] * inv - coef * r1[i];
                v[i] = vi;
                z[i] = zi;
                acc[0] += (double)vi * (double)zi;
            }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[1])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->alfa = t[0];
            S->ticket[1] = 0;
        }
    }
}

// w_new = (v - oldeps w1 - delta w2) / gamma (over w1); x += phi w_new.  Runs on the step that
// set the stopping flag (its update), not after.
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_tl_update(int n, const VT* __restrict__ v, VT* __restrict__ w1,
                                                          const VT* __restrict__ w2, VT* __restrict__ x,
                                                          const TlState* S)
{
    if (S->done && S->applied == S->iter) return;
    if (S->done == 3) return;
    const VT oe = (VT)S->oldeps, de = (VT)S->delta, dn = (VT)S->denom, ph = (VT)S->phi;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT w = (v[i] - oe * w1[i] - de * w2[i]) * dn;
        w1[i] = w;
        x[i] += ph * w;
    }
}

__global__ void k_tl_applied(TlState* S)
{
    if (S->done) S->applied = S->iter;
}

// rhs of the inner solve: b = S r / ||S r|| (scaled FP32 system) or r / ||r|| (FP64), and the
// copies r1 = r2 = b, x = w1 = w2 = 0
__global__ void __launch_bounds__(kVecThreads) k_tl_norm(int n, const double* __restrict__ r, const double* __restrict__ s,
                                                        TlState* S, double* __restrict__ partial)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double t = s ? s[i] * r[i] : r[i];
        acc[0] += t * t;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[2])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            S->bb = t[0];
            S->ticket[2] = 0;
        }
    }
}

template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_tl_rhs(int n, const double* __restrict__ r, const double* __restrict__ s,
                                                       const TlState* S, VT* __restrict__ r1, VT* __restrict__ r2,
                                                       VT* __restrict__ x, VT* __restrict__ w1, VT* __restrict__ w2)
{
    const double inv = S->bb > 0.0 ? 1.0 / sqrt(S->bb) : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT b = (VT)((s ? s[i] * r[i] : r[i]) * inv);
        r1[i] = b;
        r2[i] = b;
        x[i] = 0.0f;
        w1[i] = 0.0f;
        w2[i] = 0.0f;
    }
}

// X += ||S r|| S x (scaled FP32 system) or ||r|| x (FP64)
template <class VT>
__global__ void __launch_bounds__(kVecThreads) k_tl_correct(int n, double* __restrict__ X, const VT* __restrict__ x,
                                                           const double* __restrict__ s, const TlState* S)
{
    const double sc = sqrt(S->bb);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        X[i] += sc * (s ? s[i] : 1.0) * (double)x[i];
}

// the outer system's true residual after the inner correction so far: ||r - sqrt(bb) A x||^2 (the
// inner MINRES solves for r / ||r||, r = the refinement step's residual) into *out
__global__ void __launch_bounds__(kVecThreads) k_tl_true_norm(int n, const double* __restrict__ r,
                                                             const double* __restrict__ ax, const TlState* S,
                                                             double* __restrict__ partial, unsigned int* ticket,
                                                             double* out)
{
    __shared__ double sh[32];
    const double sc = sqrt(S->bb);
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = r[i] - sc * ax[i];
        acc[0] += d * d;
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

// ---- symmetric multiplicative two-level cycle on the textbook operator (FP32, its
// Jacobi-scaled space K^ = S_t K_t S_t): pre-smoothing by k Chebyshev steps, coarse correction
// with P^_t = S_t^-1 P, post-smoothing by the same k steps.  M^-1 r = S_t cycle(S_t r).

// 3x3-block SELL row times x with the values stored in FP32 or, when v16 is set, in FP16.  The
// FP16 values of block column k of a slice sit as 5 half2 words per lane, word p at
// 5 * blk + 32 p + lane (blk = the slice's first block of the column; word 4 = (v8, 0)): each of
// the 5 loads is one 128-byte line per warp.
// c16, when set, holds each stored block's column as a 16-bit delta from its block row (the last
// row for the padding lanes past the end), 2 instead of 4 bytes per block.
__device__ __forceinline__ void sell_row_block_mixed(const SellView<float>& A, const __half2* __restrict__ v16,
                                                     const int16_t* __restrict__ c16, int warp, int lane,
                                                     const float* __restrict__ x, float (&acc)[3])
{
    if (!v16) {
        sell_row_block<float>(A, warp, lane, x, acc);
        return;
    }
    const int64_t base = A.sp[warp];
    const int w = (int)((A.sp[warp + 1] - base) >> 5);
    const int row0 = min(warp * kSlice + lane, A.n_brows - 1);
    acc[0] = acc[1] = acc[2] = 0.0f;
#pragma unroll 2
    for (int k = 0; k < w; k++) {
        const int64_t blk = base + (int64_t)k * kSlice;
        const int c = c16 ? row0 + (int)__ldcs(c16 + blk + lane) : __ldcs(A.col + blk + lane);
        const unsigned int* vb = reinterpret_cast<const unsigned int*>(v16) + 5 * blk + lane;
        const float x0 = __ldg(x + 3 * (int64_t)c), x1 = __ldg(x + 3 * (int64_t)c + 1), x2 = __ldg(x + 3 * (int64_t)c + 2);
        float v[10];
#pragma unroll
        for (int p = 0; p < 5; p++) {
            const unsigned int u = __ldcs(vb + p * kSlice);
            const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&u));
            v[2 * p] = f.x;
            v[2 * p + 1] = f.y;
        }
        acc[0] += v[0] * x0 + v[1] * x1 + v[2] * x2;
        acc[1] += v[3] * x0 + v[4] * x1 + v[5] * x2;
        acc[2] += v[6] * x0 + v[7] * x1 + v[8] * x2;
    }
}

// FP32 SELL values (9 per block: 9 blk + 32 e + lane) -> the paired FP16 layout above
__global__ void k_to_half(int64_t stored, const float* __restrict__ a, __half2* __restrict__ h)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < stored; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t blk = q & ~(int64_t)31;
        const int l = (int)(q & 31);
        float v[10];
        for (int e = 0; e < 9; e++) v[e] = a[9 * blk + 32 * e + l];
        v[9] = 0.0f;
        for (int p = 0; p < 5; p++) h[5 * blk + 32 * p + l] = __floats2half2_rn(v[2 * p], v[2 * p + 1]);
    }
}

// block columns of the SELL copy as 16-bit deltas from the block row (overflow -> flag)
// (grid-stride over the rows: the launch helper caps the grid)
__global__ void k_block_delta16(int n_brows, int n_slices, const int64_t* __restrict__ sp,
                                const int32_t* __restrict__ col, int16_t* __restrict__ c16, int* overflow)
{
    const int64_t n_lanes = (int64_t)n_slices * kSlice;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_lanes; t += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)t;
        const int slice = row / kSlice, lane = row % kSlice;
        const int64_t base = sp[slice];
        const int w = (int)((sp[slice + 1] - base) / kSlice);
        const int row0 = min(row, n_brows - 1);
        for (int k = 0; k < w; k++) {
            const int64_t pos = base + (int64_t)k * kSlice + lane;
            // lanes past the last row hold zero blocks: any valid column will do, so point them at row0
            const int d = (row < n_brows ? col[pos] : row0) - row0;
            if (d < -32768 || d > 32767) atomicExch(overflow, 1);
            c16[pos] = (int16_t)d;
        }
    }
}

struct ChebCoef {
    float inv_theta;   // first step: d = res / theta
    float a[8], b[8];  // step i >= 1: d_i = a_i d_{i-1} + b_i res_i
};

// entry of the cycle: r_new = z - (alfa / beta) r2 (lanczos; else r_new = z), written over `out`;
// rhat = S_t r_new; res = rhat; d = rhat / theta; x = d; and, for the matrix-free smoother (dh
// non-null), dh = s d with the eliminated columns zero (s32: the operator's FP32 Jacobi scale,
// fixw: its Dirichlet words, bit 3 + c of node i / 3 for component c)
__global__ void __launch_bounds__(kVecThreads) k_mg_in(int n, const double* __restrict__ z, const double* __restrict__ r2,
                                                      double* __restrict__ out, const double* __restrict__ st,
                                                      float* __restrict__ rhat, float* __restrict__ res,
                                                      float* __restrict__ d, float* __restrict__ x, ChebCoef cc,
                                                      const TlState* S, int lanczos, const float* __restrict__ s32,
                                                      const uint32_t* __restrict__ fixw, float* __restrict__ dh)
{
    if (S->done) return;
    const double coef = lanczos ? S->alfa / S->beta : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double r = z[i];
        if (lanczos) {
            r -= coef * r2[i];
            out[i] = r;
        }
        const float rh = (float)(st[i] * r);
        rhat[i] = rh;
        res[i] = rh;
        const float di = rh * cc.inv_theta;
        d[i] = di;
        x[i] = di;
        if (dh) dh[i] = ((fixw[i / 3] >> (3 + i % 3)) & 1u) ? 0.0f : s32[i] * di;
    }
}

// one Chebyshev step: res -= K^ d_prev; d = a d_prev + b res; x += d
__global__ void __launch_bounds__(256) k_mg_cheb(SellView<float> A, const __half2* __restrict__ v16,
                                                 const int16_t* __restrict__ c16, const float* __restrict__ dprev,
                                                 float* __restrict__ d, float* __restrict__ res, float* __restrict__ x,
                                                 float a, float b, const TlState* S)
{
    if (S->done) return;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        float kd[3];
        sell_row_block_mixed(A, v16, c16, warp, lane, dprev, kd);
        const int brow = warp * kSlice + lane;
        if (brow < A.n_brows)
            for (int c = 0; c < 3; c++) {
                const int64_t i = 3 * (int64_t)brow + c;
                const float ri = res[i] - kd[c];
                res[i] = ri;
                const float di = a * dprev[i] + b * ri;
                d[i] = di;
                x[i] += di;
            }
    }
}

// res = rhat - K^ x; with `start`: also the first post-smoothing step d = res / theta,
// x2 = x + d (into a second buffer: x is being gathered)
__global__ void __launch_bounds__(256) k_mg_resid(SellView<float> A, const __half2* __restrict__ v16,
                                                  const int16_t* __restrict__ c16, const float* __restrict__ rhat,
                                                  const float* __restrict__ x, float* __restrict__ res,
                                                  float* __restrict__ d, float* __restrict__ x2, float inv_theta,
                                                  const TlState* S, int start)
{
    if (S->done) return;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        float kx[3];
        sell_row_block_mixed(A, v16, c16, warp, lane, x, kx);
        const int brow = warp * kSlice + lane;
        if (brow < A.n_brows)
            for (int c = 0; c < 3; c++) {
                const int64_t i = 3 * (int64_t)brow + c;
                const float ri = rhat[i] - kx[c];
                res[i] = ri;
                if (start) {
                    const float di = ri * inv_theta;
                    d[i] = di;
                    x2[i] = x[i] + di;
                }
            }
    }
}

// v = y / beta; z = A y / beta - (beta / oldb) r1; alfa = (v, z) (k_tl_spmv<double>) as the epilogue
// of the z-marching matrix-free product (kuhn25.cuh): y = the product's input at the node
struct EpiMinresZ {
    static constexpr int NE = 1;  // r1
    double* __restrict__ v;
    double* __restrict__ z;
    const double* __restrict__ r1;
    TlState* S;
    double* __restrict__ partial;
    double acc;
    __device__ __forceinline__ bool skip() const { return S->done; }
    __host__ __device__ __forceinline__ void sources(const double** ev) const { ev[0] = r1; }
    __device__ __forceinline__ void operator()(int64_t g, const double* ay, const double* y, const double (*e)[3])
    {
        const double inv = 1.0 / S->beta;
        const double coef = S->iter > 0 ? S->beta / S->oldb : 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int64_t i = 3 * g + c;
            const double vi = y[c] * inv;
            const double zi = ay[c] * inv - coef * e[0][c];
            v[i] = vi;
            z[i] = zi;
            acc += vi * zi;
        }
    }
    __device__ __forceinline__ void finish()
    {
        __shared__ double sh[32];
        double t[1] = {acc};
        block_sum<1>(t, sh);
        if (threadIdx.x == 0) partial[blockIdx.x] = t[0];
        if (arrive_last(&S->ticket[1])) {
            double r[1];
            reduce_partials<1>(partial, gridDim.x, 0, r, sh);
            if (threadIdx.x == 0) {
                S->alfa = r[0];
                S->ticket[1] = 0;
            }
        }
    }
};

// the smoothing kernels' epilogues on the z-marching kernel (kuhn25.cuh), whose per-node inputs
// arrive staged: xin = the product's input at the node, e[q] = the staged vectors of sources()
// one Chebyshev step on the pre-scaled z-marching kernel (k_kuhn_zp), whose input is dh = s d with
// the eliminated columns zero: y = K dh at the node; the Dirichlet rows take d itself, the others
// s y; then res -= y, d = a d + b res, x += d, and dh = s d (masked) for the next step
struct EpiChebP {
    static constexpr int NE = 4;  // res, x, the previous d, the Jacobi scale
    float* __restrict__ d;
    float* __restrict__ dh;
    float* __restrict__ res;
    float* __restrict__ x;
    const float* __restrict__ dprev;
    const float* __restrict__ scale;
    float a, b;
    const TlState* S;
    float* __restrict__ xh;  // non-null (the last step before a residual): also s x, masked
    __device__ __forceinline__ bool skip() const { return S->done; }
    __host__ __device__ __forceinline__ void sources(const float** ev) const
    {
        ev[0] = res;
        ev[1] = x;
        ev[2] = dprev;
        ev[3] = scale;
    }
    __device__ __forceinline__ void operator()(int64_t g, const float* y, uint32_t fx, const float (*e)[3])
    {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int64_t i = 3 * g + c;
            const float dp = e[2][c], sc = e[3][c];
            const float yc = ((fx >> c) & 1u) ? dp : y[c] * sc;
            const float ri = e[0][c] - yc;
            res[i] = ri;
            const float di = a * dp + b * ri;
            d[i] = di;
            const float xi = e[1][c] + di;
            x[i] = xi;
            const bool col = (fx >> (3 + c)) & 1u;
            dh[i] = col ? 0.0f : sc * di;
            if (xh) xh[i] = col ? 0.0f : sc * xi;
        }
    }
    __device__ __forceinline__ void finish() {}
};

// the cycle's residual on the pre-scaled kernel: y = K xh at the node with xh = s x (masked);
// res = rhat - (x on the Dirichlet rows, s y elsewhere); start (after the coarse correction): also
// d = res / theta, dh = s d (masked, the next step's input) and x2 = x + d
struct EpiResidP {
    static constexpr int NE = 3;  // rhat, x, the Jacobi scale
    const float* __restrict__ rhat;
    float* __restrict__ res;
    float* __restrict__ d;
    float* __restrict__ dh;
    float* __restrict__ x2;
    const float* __restrict__ x;
    const float* __restrict__ scale;
    float inv_theta;
    const TlState* S;
    int start;
    __device__ __forceinline__ bool skip() const { return S->done; }
    __host__ __device__ __forceinline__ void sources(const float** ev) const
    {
        ev[0] = rhat;
        ev[1] = x;
        ev[2] = scale;
    }
    __device__ __forceinline__ void operator()(int64_t g, const float* y, uint32_t fx, const float (*e)[3])
    {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int64_t i = 3 * g + c;
            const float xc = e[1][c], sc = e[2][c];
            const float ri = e[0][c] - (((fx >> c) & 1u) ? xc : y[c] * sc);
            res[i] = ri;
            if (start) {
                const float di = ri * inv_theta;
                d[i] = di;
                dh[i] = ((fx >> (3 + c)) & 1u) ? 0.0f : sc * di;
                x2[i] = xc + di;
            }
        }
    }
    __device__ __forceinline__ void finish() {}
};

using KChebP = KzpKernel<2, float, kKzTX, kKzTY, kKzMinB, EpiChebP>;
using KResidP = KzpKernel<2, float, kKzTX, kKzTY, kKzMinB, EpiResidP>;
using KMinres = KzKernel<1, false, double, kKzTX, kKzTY, kKzMinB64, EpiMinresZ>;

// x += P^_t ec; with xh non-null also xh = s x with the eliminated columns zero (the next product's
// input: s32 the operator's FP32 Jacobi scale, fixw its Dirichlet words)
__global__ void __launch_bounds__(kVecThreads) k_mg_prolong(int n_fine, const int32_t* __restrict__ owner,
                                                           const int32_t* __restrict__ cdof,
                                                           const float* __restrict__ psi, const float* __restrict__ ec,
                                                           float* __restrict__ x, const TlState* S,
                                                           const float* __restrict__ s32,
                                                           const uint32_t* __restrict__ fixw, float* __restrict__ xh)
{
    if (S->done) return;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_fine; g += (int64_t)gridDim.x * blockDim.x) {
        // 24 coarse DOFs of the owner cell and the node's 24 prolongation weights: six 16-byte loads each
        const int4* c4 = reinterpret_cast<const int4*>(cdof + 24 * (int64_t)owner[g]);
        const float4* p4 = reinterpret_cast<const float4*>(psi + 24 * g);
        float z[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int4 cq = __ldg(c4 + q);
            const float4 pq = __ldg(p4 + q);
            const int dd[4] = {cq.x, cq.y, cq.z, cq.w};
            const float pp[4] = {pq.x, pq.y, pq.z, pq.w};
#pragma unroll
            for (int t = 0; t < 4; t++)
                if (dd[t] >= 0) z[(4 * q + t) % 3] += pp[t] * ec[dd[t]];
        }
        const uint32_t fw = xh ? fixw[g] : 0u;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float xa = x[3 * g + a] + z[a];
            x[3 * g + a] = xa;
            if (xh) xh[3 * g + a] = ((fw >> (3 + a)) & 1u) ? 0.0f : s32[3 * g + a] * xa;
        }
    }
}

// exit of the cycle: y = S_t x (FP64), bb = (r, y) and the Givens step
__global__ void __launch_bounds__(kVecThreads) k_mg_out(int n, const float* __restrict__ x, const double* __restrict__ st,
                                                       const double* __restrict__ r, double* __restrict__ y, TlState* S,
                                                       double* __restrict__ partial, int init)
{
    if (S->done) return;
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double yi = st[i] * (double)x[i];
        y[i] = yi;
        acc[0] += r[i] * yi;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
    if (arrive_last(&S->ticket[0])) {
        double t[1];
        reduce_partials<1>(partial, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            givens_step(S, t[0], init);
            S->ticket[0] = 0;
        }
    }
}

// psi_t = psi_hat * s_ref / s_t (the prolongation rescaled to the textbook system's Jacobi scaling)
__global__ void k_mg_psi(int n_fine, const float* __restrict__ psi_hat, const double* __restrict__ s_ref,
                         const double* __restrict__ s_t, float* __restrict__ psi_t)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 24 * (int64_t)n_fine;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = t / 24;
        const int a = (int)(t % 24) % 3;
        psi_t[t] = (float)((double)psi_hat[t] * s_ref[3 * g + a] / s_t[3 * g + a]);
    }
}

// ||y||^2 into *out (power iteration of the smoother set-up)
__global__ void __launch_bounds__(kVecThreads) k_mg_norm2(int n, const float* __restrict__ y, double* __restrict__ partial,
                                                         unsigned int* ticket, double* out)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] += (double)y[i] * (double)y[i];
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

__global__ void __launch_bounds__(kVecThreads) k_mg_scale(int n, float* __restrict__ v, const double* norm2)
{
    const float inv = (float)(*norm2 > 0.0 ? 1.0 / sqrt(*norm2) : 0.0);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] *= inv;
}

}  // namespace

struct CoarseHandle {
    System* fine = nullptr;
    CellsHandle* cells = nullptr;
    int n_cells = 0, n_cv = 0, n_cf = 0, n_pad = 0;
    int n_fine = 0;
    DBuf<int32_t> cdof;              // [n_cells][8][3] free coarse DOF or -1
    DBuf<int32_t> owner;             // [n_fine] owner cell
    DBuf<int32_t> own_ptr, own;      // owned fine nodes per cell
    DBuf<float> psi_hat;             // [n_fine][24]
    DBuf<int32_t> dptr, dent;        // coarse DOF -> cell partial entries
    DBuf<float> Csym;                // upper 64 x 64 blocks of the FP32 coarse inverse, packed
    DBuf<int2> sym_blocks;           // (block row, block column) of each stored block
    DBuf<float> sym_part;            // [nb][nb][64] partial products
    int sym_nb = 0, sym_n = 0;
    DBuf<double> Ac;                 // dense coarse matrix (kept for inspection), n_cf x n_cf
    DBuf<float> cpart, rc, ec;
    DBuf<double> vec;                // 8 fine vectors (FP64 room; the FP32 solve uses the front half)
    int64_t ldv64 = 0;               // their stride
    DBuf<double> r64, partial;
    DBuf<TlState> st;
    TlState* h_st = nullptr;
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // FP32, FP64, multiplicative iteration graphs
    float ms_setup = 0.f;
    // multiplicative cycle (msfem_coarse_set_smoother): the textbook-orientation system, the
    // Chebyshev degree and coefficients, the prolongation in its scaling, cycle vectors
    System* text = nullptr;
    int cheb_deg = 0;
    double lmax = 0.0, lmin = 0.0, ratio = 30.0;
    int widened = 0;            // times the solve widened lmax after a step that raised the residual
    int n_trilinear = 0;        // cells whose wild bases were replaced by trilinear functions
    ChebCoef cc{};
    DBuf<double> xkeep;         // X before the current refinement step (restored when the step fails)
    DBuf<double> rtmp, rr_true;  // the inner solve's true-residual check: A x, ||r - A x||^2
    DBuf<unsigned int> tk;       // its reduction ticket
    DBuf<float> psi_t, mgv;
    int64_t ldv = 0;            // stride of the cycle's nine FP32 vectors in mgv (16-byte aligned, with slack)
    DBuf<__half2> val16;  // FP16 copy of the textbook system's scaled SELL values, paired (when requested)
    DBuf<int16_t> col16;  // its block columns as 16-bit deltas (empty when some delta does not fit)
    bool half_matrix = false;
    // the smoother's operator: 0 FP32 SELL, 1 FP16 SELL (half_matrix), 2 matrix-free on the Kuhn grid
    int storage = 0;
    KuhnOperator kt;      // matrix-free textbook operator (storage 2)
    KuhnOperator ka;      // matrix-free reference operator for MINRES's products (msfem_coarse_set_matrix_free)
    bool mf_fine = false;
    ~CoarseHandle()
    {
        for (auto g : graph)
            if (g) cudaGraphExecDestroy(g);
        if (h_st) cudaFreeHost(h_st);
    }
};

namespace {

int coarse_build(CoarseHandle& C, System& F, CellsHandle& Ce, const int32_t* h_cng, int n_cv, const int32_t* h_cvert,
                 const int32_t* h_color, int n_fixed, const int32_t* h_fixed)
{
    cudaStream_t st = F.stream;
    MSFEM_TRY(prepare_sell(F));
    C.fine = &F;
    C.cells = &Ce;
    C.n_cells = Ce.n_cells;
    C.n_cv = n_cv;
    C.n_fine = F.n_nodes;
    const int64_t nb = Ce.n_nodes;  // batch (cell-local) nodes
    cudaEvent_t e0, e1;
    MSFEM_CK(cudaEventCreate(&e0));
    MSFEM_CK(cudaEventCreate(&e1));
    MSFEM_CK(cudaEventRecord(e0, st));
    // fine Dirichlet flags
    std::vector<uint8_t> fixed3(3 * (size_t)F.n_nodes, 0);
    for (int i = 0; i < n_fixed; i++) {
        if (h_fixed[i] < 0 || h_fixed[i] >= 3 * F.n_nodes) {
            set_error("msfem_coarse_create: Dirichlet DOF %d out of range", h_fixed[i]);
            return MSFEM_ERR_ARGUMENT;
        }
        fixed3[h_fixed[i]] = 1;
    }
    for (int64_t b = 0; b < nb; b++)
        if (h_cng[b] < 0 || h_cng[b] >= F.n_nodes) {
            set_error("msfem_coarse_create: cell node %lld maps to fine node %d (out of range)", (long long)b, h_cng[b]);
            return MSFEM_ERR_ARGUMENT;
        }
    // coarse DOFs: (V, a) is dropped when the fine node at the vertex has a Dirichlet a-component
    std::vector<int32_t> vert(8 * (size_t)C.n_cells);
    MSFEM_CK(cudaMemcpyAsync(vert.data(), Ce.vert.p, sizeof(int32_t) * vert.size(), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    std::vector<int8_t> vfix(3 * (size_t)n_cv, -1);
    for (int c = 0; c < C.n_cells; c++)
        for (int v = 0; v < 8; v++) {
            const int V = h_cvert[8 * c + v];
            if (V < 0 || V >= n_cv) {
                set_error("msfem_coarse_create: coarse vertex id %d out of range", V);
                return MSFEM_ERR_ARGUMENT;
            }
            const int g = h_cng[vert[8 * c + v]];
            for (int a = 0; a < 3; a++) vfix[3 * V + a] = fixed3[3 * (size_t)g + a] ? 1 : 0;
        }
    std::vector<int32_t> dof_of(3 * (size_t)n_cv, -1);
    int n_cf = 0;
    for (int d = 0; d < 3 * n_cv; d++)
        if (vfix[d] == 0) dof_of[d] = n_cf++;
    C.n_cf = n_cf;
    C.n_pad = (n_cf + kSB - 1) / kSB * kSB;
    std::vector<int32_t> cdof(24 * (size_t)C.n_cells);
    for (int c = 0; c < C.n_cells; c++)
        for (int v = 0; v < 8; v++)
            for (int a = 0; a < 3; a++) cdof[24 * c + 3 * v + a] = dof_of[3 * h_cvert[8 * c + v] + a];
    // coarse DOF -> (cell, slot) entries in cell order
    std::vector<int32_t> dcnt(n_cf + 1, 0);
    for (size_t k = 0; k < cdof.size(); k++)
        if (cdof[k] >= 0) dcnt[cdof[k] + 1]++;
    for (int d = 0; d < n_cf; d++) dcnt[d + 1] += dcnt[d];
    std::vector<int32_t> dent(dcnt[n_cf]);
    {
        std::vector<int32_t> fill(dcnt.begin(), dcnt.end() - 1);
        for (size_t k = 0; k < cdof.size(); k++)
            if (cdof[k] >= 0) dent[fill[cdof[k]]++] = (int32_t)k;
    }
    MSFEM_TRY(C.cdof.alloc(cdof.size()));
    MSFEM_CK(cudaMemcpyAsync(C.cdof.p, cdof.data(), sizeof(int32_t) * cdof.size(), cudaMemcpyHostToDevice, st));
    MSFEM_TRY(C.dptr.alloc(n_cf + 1));
    MSFEM_TRY(C.dent.alloc(std::max<size_t>(1, dent.size())));
    MSFEM_CK(cudaMemcpyAsync(C.dptr.p, dcnt.data(), sizeof(int32_t) * (n_cf + 1), cudaMemcpyHostToDevice, st));
    if (!dent.empty()) MSFEM_CK(cudaMemcpyAsync(C.dent.p, dent.data(), sizeof(int32_t) * dent.size(), cudaMemcpyHostToDevice, st));

    // device copies of the maps
    DBuf<int32_t> cng, cvert, bcell, inc_ptr, keys2, vals, vals2;
    DBuf<uint8_t> dfix;
    MSFEM_TRY(cng.alloc(nb));
    MSFEM_TRY(cvert.alloc(8 * (size_t)C.n_cells));
    MSFEM_TRY(dfix.alloc(fixed3.size()));
    MSFEM_CK(cudaMemcpyAsync(cng.p, h_cng, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemcpyAsync(cvert.p, h_cvert, sizeof(int32_t) * 8 * C.n_cells, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemcpyAsync(dfix.p, fixed3.data(), fixed3.size(), cudaMemcpyHostToDevice, st));
    MSFEM_TRY(bcell.alloc(nb));
    k_batch_cell<<<C.n_cells, 256, 0, st>>>(C.n_cells, Ce.node_off.p, bcell.p);
    // incidence fine node -> batch nodes (stable: batch order)
    MSFEM_TRY(vals.alloc(nb));
    MSFEM_TRY(keys2.alloc(nb));
    MSFEM_TRY(vals2.alloc(nb));
    {
        std::vector<int32_t> iota(nb);
        std::iota(iota.begin(), iota.end(), 0);
        MSFEM_CK(cudaMemcpyAsync(vals.p, iota.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice, st));
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, cng.p, keys2.p, vals.p, vals2.p, (int)nb, 0, 32, st);
        DBuf<unsigned char> tmp;
        MSFEM_TRY(tmp.alloc(std::max<size_t>(tb, 1)));
        MSFEM_CK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, cng.p, keys2.p, vals.p, vals2.p, (int)nb, 0, 32, st));
        MSFEM_CK(cudaStreamSynchronize(st));
    }
    DBuf<int> flag;
    MSFEM_TRY(flag.alloc(1));
    MSFEM_CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    MSFEM_TRY(inc_ptr.alloc((size_t)F.n_nodes + 1));
    MSFEM_CK(cudaMemsetAsync(inc_ptr.p, 0xff, sizeof(int32_t) * ((size_t)F.n_nodes + 1), st));
    k_inc_heads<<<gridn(nb), 256, 0, st>>>(nb, keys2.p, inc_ptr.p, F.n_nodes, flag.p);
    k_inc_fill<<<gridn(F.n_nodes), 256, 0, st>>>(F.n_nodes, inc_ptr.p, flag.p);
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_coarse_create: %s", bad == 2 ? "a fine node belongs to no cell" : "bad cell node map");
        return MSFEM_ERR_ARGUMENT;
    }
    // prolongation values
    DBuf<double> psi;
    MSFEM_TRY(psi.alloc(24 * (size_t)nb));
    DBuf<uint8_t> wild;
    MSFEM_TRY(wild.alloc(C.n_cells));
    k_wild_cells<<<C.n_cells, 256, 0, st>>>(Ce.node_off.p, Ce.bx.p, wild.p);
    {
        std::vector<uint8_t> hw(C.n_cells);
        MSFEM_CK(cudaMemcpyAsync(hw.data(), wild.p, C.n_cells, cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        C.n_trilinear = 0;
        for (uint8_t w : hw) C.n_trilinear += w;
    }
    k_psi_cell<<<gridn(nb), 256, 0, st>>>(nb, bcell.p, cng.p, inc_ptr.p, vals2.p, cvert.p, C.cdof.p, dfix.p, Ce.bx.p, wild.p,
                                          Ce.box.p, Ce.xyz.p, psi.p);
    MSFEM_TRY(C.owner.alloc(F.n_nodes));
    MSFEM_TRY(C.psi_hat.alloc(24 * (size_t)F.n_nodes));
    k_psi_hat<<<gridn(F.n_nodes), 256, 0, st>>>(F.n_nodes, inc_ptr.p, vals2.p, bcell.p, psi.p, F.dscale.p, C.owner.p,
                                                 C.psi_hat.p);
    MSFEM_CK(cudaGetLastError());
    // owned fine nodes per cell (sorted by owner, then node)
    {
        std::vector<int32_t> own(F.n_nodes);
        MSFEM_CK(cudaMemcpyAsync(own.data(), C.owner.p, sizeof(int32_t) * F.n_nodes, cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        std::vector<int32_t> ptr(C.n_cells + 1, 0), lst(F.n_nodes);
        for (int g = 0; g < F.n_nodes; g++) ptr[own[g] + 1]++;
        for (int c = 0; c < C.n_cells; c++) ptr[c + 1] += ptr[c];
        std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
        for (int g = 0; g < F.n_nodes; g++) lst[fill[own[g]]++] = g;
        MSFEM_TRY(C.own_ptr.alloc(C.n_cells + 1));
        MSFEM_TRY(C.own.alloc(F.n_nodes));
        MSFEM_CK(cudaMemcpyAsync(C.own_ptr.p, ptr.data(), sizeof(int32_t) * (C.n_cells + 1), cudaMemcpyHostToDevice, st));
        MSFEM_CK(cudaMemcpyAsync(C.own.p, lst.data(), sizeof(int32_t) * F.n_nodes, cudaMemcpyHostToDevice, st));
    }
    // cell coarse matrices and the dense coarse matrix, colour by colour
    DBuf<double> Kc;
    MSFEM_TRY(Kc.alloc(576 * (size_t)C.n_cells));
    MSFEM_CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    k_coarse_cells<<<C.n_cells, kCoarseThreads, 0, st>>>(Ce.vols.elem_off.p, Ce.vols.elems.p, Ce.mat.p, Ce.xyz.p,
                                                         Ce.lame.p, Ce.n_mat, psi.p, Kc.p, flag.p);
    const int64_t ld = C.n_pad;
    MSFEM_TRY(C.Ac.alloc((size_t)ld * ld));
    MSFEM_CK(cudaMemsetAsync(C.Ac.p, 0, sizeof(double) * ld * ld, st));
    {
        int max_col = 0;
        for (int c = 0; c < C.n_cells; c++) max_col = std::max(max_col, h_color[c]);
        std::vector<int32_t> sel;
        DBuf<int32_t> dsel;
        MSFEM_TRY(dsel.alloc(C.n_cells));
        for (int col = 0; col <= max_col; col++) {
            sel.clear();
            for (int c = 0; c < C.n_cells; c++)
                if (h_color[c] == col) sel.push_back(c);
            if (sel.empty()) continue;
            MSFEM_CK(cudaMemcpyAsync(dsel.p, sel.data(), sizeof(int32_t) * sel.size(), cudaMemcpyHostToDevice, st));
            k_coarse_scatter<<<gridn((int64_t)sel.size() * 576), 256, 0, st>>>((int)sel.size(), dsel.p, Kc.p, C.cdof.p,
                                                                               C.Ac.p, ld);
            MSFEM_CK(cudaStreamSynchronize(st));  // dsel is reused by the next colour
        }
    }
    k_sym_pad<<<gridn((int64_t)ld * ld), 256, 0, st>>>(C.Ac.p, ld, C.n_cf, C.n_pad);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_coarse_create: material id out of range");
        return MSFEM_ERR_ARGUMENT;
    }
    // invert: sweep every 64-block pivot (A becomes -A^-1), working on a copy
    DBuf<double> W, Pinv, Bp, Cp;
    MSFEM_TRY(W.alloc((size_t)ld * ld));
    MSFEM_CK(cudaMemcpyAsync(W.p, C.Ac.p, sizeof(double) * ld * ld, cudaMemcpyDeviceToDevice, st));
    MSFEM_TRY(Pinv.alloc(kSB * kSB));
    MSFEM_TRY(Bp.alloc((size_t)ld * kSB));
    MSFEM_TRY(Cp.alloc((size_t)ld * kSB));
    const int nblk = C.n_pad / kSB;
    const size_t smem = 2 * kSB * (kSB + 1) * sizeof(double);
    MSFEM_CK(cudaFuncSetAttribute(k_sweep_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MSFEM_CK(cudaFuncSetAttribute(k_sweep_pivot, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MSFEM_CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    // the swept matrix stays symmetric: only its upper block triangle is updated
    std::vector<int2> up;
    up.reserve((size_t)nblk * (nblk + 1) / 2);
    for (int I = 0; I < nblk; I++)
        for (int J = I; J < nblk; J++) up.push_back(make_int2(I, J));
    DBuf<int2> d_up;
    MSFEM_TRY(d_up.alloc(up.size()));
    MSFEM_CK(cudaMemcpyAsync(d_up.p, up.data(), sizeof(int2) * up.size(), cudaMemcpyHostToDevice, st));
    for (int kb = 0; kb < nblk; kb++) {
        k_sweep_pivot<<<1, 256, smem, st>>>(W.p, ld, kb * kSB, Pinv.p, flag.p);
        k_sweep_panel<<<(C.n_pad + 3) / 4, 256, 0, st>>>(W.p, ld, C.n_pad, kb * kSB, Pinv.p, Bp.p, Cp.p);
        k_sweep_update<<<(unsigned)up.size(), 256, smem, st>>>(W.p, ld, kb, d_up.p, Pinv.p, Bp.p, Cp.p);
    }
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (bad) {
        set_error("msfem_coarse_create: the coarse matrix is not positive definite");
        return MSFEM_ERR_NUMERIC;
    }
    {
        const int nb = (int)(ld / kSymB);
        std::vector<int2> hb;
        hb.reserve((size_t)nb * (nb + 1) / 2);
        for (int I = 0; I < nb; I++)
            for (int J = I; J < nb; J++) hb.push_back(make_int2(I, J));
        C.sym_nb = nb;
        C.sym_n = (int)hb.size();
        MSFEM_TRY(C.sym_blocks.alloc(hb.size()));
        MSFEM_CK(cudaMemcpyAsync(C.sym_blocks.p, hb.data(), sizeof(int2) * hb.size(), cudaMemcpyHostToDevice, st));
        MSFEM_TRY(C.Csym.alloc(hb.size() * kSymB * kSymB));
        MSFEM_TRY(C.sym_part.alloc((size_t)nb * nb * kSymB));
        k_pack_sym<<<gridn((int64_t)C.sym_n * kSymB * kSymB), 256, 0, st>>>(W.p, ld, C.n_cf, C.sym_blocks.p, C.sym_n,
                                                                               C.Csym.p);
        MSFEM_CK(cudaStreamSynchronize(st));  // the host block list is released here
    }
    // solver storage
    const int n = F.n_rows;
    MSFEM_TRY(C.cpart.alloc(24 * (size_t)C.n_cells));
    MSFEM_TRY(C.rc.alloc(C.n_pad));
    MSFEM_TRY(C.ec.alloc(C.n_pad));
    MSFEM_CK(cudaMemsetAsync(C.rc.p, 0, sizeof(float) * C.n_pad, st));  // the GEMV reads the zero tail
    // eight vectors of doubles (room for the FP64 solve) at a 16-byte-aligned stride with slack,
    // as the z-marching kernel's staging copies need
    C.ldv64 = (n + 16 + 7) / 8 * 8;
    MSFEM_TRY(C.vec.alloc(8 * (size_t)C.ldv64));
    MSFEM_TRY(C.r64.alloc(n));
    MSFEM_TRY(C.partial.alloc(4096));
    MSFEM_TRY(C.st.alloc(1));
    MSFEM_CK(cudaMemsetAsync(C.st.p, 0, sizeof(TlState), st));
    MSFEM_CK(cudaMallocHost(&C.h_st, sizeof(TlState)));
    MSFEM_CK(cudaEventRecord(e1, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    MSFEM_CK(cudaEventElapsedTime(&C.ms_setup, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MSFEM_OK;
}

// ec = Cinv rc (symmetric packed blocks)
void coarse_solve(CoarseHandle& C, const TlState* S, cudaStream_t st)
{
    k_tl_symv<<<std::min(C.sym_n, 148 * 4), 256, 0, st>>>(C.sym_nb, C.sym_n, C.sym_blocks.p, C.Csym.p, C.rc.p,
                                                          C.sym_part.p, S);
    k_tl_symv_sum<<<(C.n_pad + 255) / 256, 256, 0, st>>>(C.n_pad, C.sym_nb, C.sym_part.p, C.ec.p, S);
}

// y = M^-1 r into y (FP32: scaled system; FP64: original unknowns with s = D^-1/2);
// init: also sets beta1 etc.
template <class VT>
void precondition(CoarseHandle& C, const VT* r, VT* y, int init, cudaStream_t st, unsigned gprol, const double* s)
{
    k_tl_restrict<VT><<<C.n_cells, 128, 0, st>>>(C.own_ptr.p, C.own.p, C.psi_hat.p, r, nullptr, nullptr, C.cpart.p, s,
                                                 C.st.p, 0);
    k_tl_gather<<<gridn(C.n_cf), 256, 0, st>>>(C.n_cf, C.dptr.p, C.dent.p, C.cpart.p, C.rc.p, C.st.p);
    coarse_solve(C, C.st.p, st);
    k_tl_prolong<VT><<<gprol, kVecThreads, 0, st>>>(C.n_fine, C.owner.p, C.cdof.p, C.psi_hat.p, C.ec.p, r, y, s, C.st.p,
                                                    C.partial.p, init);
}

int read_st(CoarseHandle& C, cudaStream_t st)
{
    MSFEM_CK(cudaMemcpyAsync(C.h_st, C.st.p, sizeof(TlState), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return 0;
}

// preconditioned MINRES from 0 on b = S r / ||S r|| (FP32, Jacobi-scaled matrix) or b = r / ||r||
// (FP64, original matrix), to |phibar| <= tau beta1
template <class VT>
int inner_solve(CoarseHandle& C, int maxiter, double tau, int* iters)
{
    System& F = *C.fine;
    cudaStream_t st = F.stream;
    const int n = F.n_rows;
    constexpr bool f32 = sizeof(VT) == 4;
    const double* s = f32 ? nullptr : F.dscale.p;  // FP64 works in the original unknowns
    const int64_t ld = C.ldv64;
    VT* X = reinterpret_cast<VT*>(C.vec.p);
    VT* V = X + ld;
    VT* Z = V + ld;
    VT* Y = Z + ld;
    VT* R[2] = {Y + ld, Y + 2 * ld};
    VT* Wb[2] = {Y + 3 * ld, Y + 4 * ld};
    TlState* S = C.st.p;
    const unsigned gvec = kReduceBlocks;
    k_tl_norm<<<gvec, kVecThreads, 0, st>>>(n, C.r64.p, f32 ? F.dscale.p : nullptr, S, C.partial.p);
    k_tl_rhs<VT><<<gvec, kVecThreads, 0, st>>>(n, C.r64.p, f32 ? F.dscale.p : nullptr, S, R[0], R[1], X, Wb[0], Wb[1]);
    MSFEM_TRY(read_st(C, st));
    TlState h = *C.h_st;
    h.tol = tau;
    h.maxiter = maxiter;
    h.done = 0;
    h.applied = -1;
    h.iter = 0;
    for (auto& t : h.ticket) t = 0;
    *C.h_st = h;
    MSFEM_CK(cudaMemcpyAsync(S, C.h_st, sizeof(TlState), cudaMemcpyHostToDevice, st));
    const unsigned gprol = kReduceBlocks;
    precondition<VT>(C, R[1], Y, 1, st, gprol, s);
    const SellView<VT> A = sell_view<VT>(F);
    const unsigned gsp = spmv_grid_of((const void*)k_tl_spmv<VT>, F);
    // two iterations: r1/r2 and w1/w2 swap each step
    auto two = [&]() {
        for (int p = 0; p < 2; p++) {
            VT* r1 = R[p];
            VT* r2 = R[1 - p];
            VT* w1 = Wb[p];
            VT* w2 = Wb[1 - p];
            k_tl_spmv<VT><<<gsp, 256, 0, st>>>(A, Y, V, Z, r1, S, C.partial.p + 2048);
            // r2_new = z - (alfa/beta) r2 over r1's buffer, and its restriction partials
            k_tl_restrict<VT><<<C.n_cells, 128, 0, st>>>(C.own_ptr.p, C.own.p, C.psi_hat.p, Z, r2, r1, C.cpart.p, s, S, 1);
            k_tl_gather<<<gridn(C.n_cf), 256, 0, st>>>(C.n_cf, C.dptr.p, C.dent.p, C.cpart.p, C.rc.p, S);
            coarse_solve(C, S, st);
            k_tl_prolong<VT><<<gprol, kVecThreads, 0, st>>>(C.n_fine, C.owner.p, C.cdof.p, C.psi_hat.p, C.ec.p, r1, Y, s,
                                                            S, C.partial.p, 0);
            k_tl_update<VT><<<gvec, kVecThreads, 0, st>>>(n, V, w1, w2, X, S);
            k_tl_applied<<<1, 1, 0, st>>>(S);
        }
    };
    cudaGraphExec_t& graph = C.graph[f32 ? 0 : 1];
    if (!graph) {
        cudaGraph_t gr;
        MSFEM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < 8; k++) two();  // 16 iterations per replay
        cudaError_t e = cudaStreamEndCapture(st, &gr);
        if (e != cudaSuccess) {
            set_error("two-level MINRES graph capture failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            set_error("two-level MINRES graph instantiate failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
    }
    int rounds = 0;
    for (;;) {
        MSFEM_TRY(read_st(C, st));
        if (C.h_st->done) break;
        if (16 * rounds > maxiter + 32) break;
        for (int k = 0; k < 4; k++) MSFEM_CK(cudaGraphLaunch(graph, st));
        rounds += 4;
        F.total_launches += 4 * 16 * 7;
    }
    *iters = C.h_st->iter;
    return C.h_st->done == 3 ? MSFEM_ERR_NUMERIC : MSFEM_OK;
}

// The multiplicative cycle M^-1 r into y (FP64), with bb = (r, y) and the Givens step.
// r_in: z (lanczos) or the right-hand side (first application); r_out: where r_new goes.
void mg_cycle(CoarseHandle& C, const double* z, const double* r2, double* r_out, double* y, int lanczos, int init,
              cudaStream_t st)
{
    System& T = *C.text;
    const int n = T.n_rows;
    const int64_t ld = C.ldv;
    float* rhat = C.mgv.p;
    float* res = rhat + ld;
    float* dA = res + ld;
    float* dB = dA + ld;
    float* x = dB + ld;
    float* x2 = x + ld;
    float* dhA = x2 + ld;  // matrix-free: s d with the eliminated columns zero, the next step's input
    float* dhB = dhA + ld;
    float* xh = dhB + ld;  // matrix-free: s x (masked), the residual products' input
    TlState* S = C.st.p;
    const SellView<float> At = sell_view<float>(T);
    const unsigned gsp = spmv_grid_of((const void*)k_mg_cheb, T);
    const unsigned gvec = kReduceBlocks;
    const double* s_t = T.dscale.p;
    const __half2* v16 = C.half_matrix ? C.val16.p : nullptr;
    const int16_t* c16 = C.half_matrix ? C.col16.p : nullptr;
    const bool mf = C.storage == 2;
    const KuhnView<float>& Kv = C.kt.v32;
    const int sms = C.kt.sms;
    int* kerr = C.kt.err.p;
    float* d[2] = {dA, dB};
    float* dh[2] = {dhA, dhB};
    // the pre-smoothing's last step also writes xh (with degree 1, xh is d_0's own scaled copy)
    auto cheb = [&](int i, float* xx, float* xhout) {
        float *dprev = d[(i - 1) & 1], *dnew = d[i & 1];
        if (mf)
            KChebP::launch(Kv, dh[(i - 1) & 1],
                           EpiChebP{dnew, dh[i & 1], res, xx, dprev, Kv.scale, C.cc.a[i], C.cc.b[i], S, xhout}, sms,
                           kerr, st);
        else
            k_mg_cheb<<<gsp, 256, 0, st>>>(At, v16, c16, dprev, dnew, res, xx, C.cc.a[i], C.cc.b[i], S);
    };
    auto resid = [&](const float* xin_h, float* d0, float* x2, float inv_theta, int start) {
        if (mf)
            KResidP::launch(Kv, xin_h, EpiResidP{rhat, res, d0, dhA, x2, x, Kv.scale, inv_theta, S, start}, sms, kerr,
                            st);
        else
            k_mg_resid<<<gsp, 256, 0, st>>>(At, v16, c16, rhat, x, res, d0, x2, inv_theta, S, start);
    };
    k_mg_in<<<gvec, kVecThreads, 0, st>>>(n, z, r2, r_out, s_t, rhat, res, dA, x, C.cc, S, lanczos, Kv.scale, Kv.fix,
                                          mf ? dhA : nullptr);
    for (int i = 1; i < C.cheb_deg; i++) cheb(i, x, i == C.cheb_deg - 1 ? xh : nullptr);
    resid(C.cheb_deg > 1 ? xh : dhA, nullptr, nullptr, 0.0f, 0);
    k_tl_restrict<float><<<C.n_cells, 128, 0, st>>>(C.own_ptr.p, C.own.p, C.psi_t.p, res, nullptr, nullptr, C.cpart.p,
                                                    nullptr, S, 0);
    k_tl_gather<<<gridn(C.n_cf), 256, 0, st>>>(C.n_cf, C.dptr.p, C.dent.p, C.cpart.p, C.rc.p, S);
    coarse_solve(C, S, st);
    k_mg_prolong<<<gvec, kVecThreads, 0, st>>>(C.n_fine, C.owner.p, C.cdof.p, C.psi_t.p, C.ec.p, x, S, Kv.scale, Kv.fix,
                                               mf ? xh : nullptr);
    resid(xh, dA, x2, C.cc.inv_theta, 1);
    for (int i = 1; i < C.cheb_deg; i++) cheb(i, x2, nullptr);
    k_mg_out<<<gvec, kVecThreads, 0, st>>>(n, x2, s_t, lanczos ? r_out : z, y, S, C.partial.p, init);
}

// FP64 MINRES on the original matrix with the multiplicative cycle as preconditioner
// stop2 > 0: also stop once the outer system's true residual, checked every 64 iterations (one
// FP64 product), has fallen to stop2 (squared 2-norm) -- the preconditioned residual MINRES
// tracks is in the cycle's norm, whose distance to the 2-norm depends on the smoother
int inner_solve_mg(CoarseHandle& C, int maxiter, double tau, double stop2, int* iters)
{
    System& F = *C.fine;
    cudaStream_t st = F.stream;
    const int n = F.n_rows;
    const int64_t ld = C.ldv64;
    double* X = C.vec.p;
    double* V = X + ld;
    double* Z = V + ld;
    double* Y = Z + ld;
    double* R[2] = {Y + ld, Y + 2 * ld};
    double* Wb[2] = {Y + 3 * ld, Y + 4 * ld};
    TlState* S = C.st.p;
    const unsigned gvec = kReduceBlocks;
    k_tl_norm<<<gvec, kVecThreads, 0, st>>>(n, C.r64.p, nullptr, S, C.partial.p);
    k_tl_rhs<double><<<gvec, kVecThreads, 0, st>>>(n, C.r64.p, nullptr, S, R[0], R[1], X, Wb[0], Wb[1]);
    MSFEM_TRY(read_st(C, st));
    TlState h = *C.h_st;
    h.tol = tau;
    h.maxiter = maxiter;
    h.done = 0;
    h.applied = -1;
    h.iter = 0;
    for (auto& t : h.ticket) t = 0;
    *C.h_st = h;
    MSFEM_CK(cudaMemcpyAsync(S, C.h_st, sizeof(TlState), cudaMemcpyHostToDevice, st));
    mg_cycle(C, R[1], nullptr, nullptr, Y, 0, 1, st);
    const SellView<double> A = sell_view<double>(F);
    const unsigned gsp = spmv_grid_of((const void*)k_tl_spmv<double>, F);
    auto two = [&]() {
        for (int p = 0; p < 2; p++) {
            double* r1 = R[p];
            double* r2 = R[1 - p];
            double* w1 = Wb[p];
            double* w2 = Wb[1 - p];
            if (C.mf_fine)
                KMinres::launch(C.ka.v64, Y, EpiMinresZ{V, Z, r1, S, C.partial.p + 2048, 0.0}, C.ka.sms, C.ka.err.p,
                                st);
            else
                k_tl_spmv<double><<<gsp, 256, 0, st>>>(A, Y, V, Z, r1, S, C.partial.p + 2048);
            mg_cycle(C, Z, r2, r1, Y, 1, 0, st);  // r2_new over r1's buffer, then y = M^-1 r2_new
            k_tl_update<double><<<gvec, kVecThreads, 0, st>>>(n, V, w1, w2, X, S);
            k_tl_applied<<<1, 1, 0, st>>>(S);
        }
    };
    cudaGraphExec_t& graph = C.graph[2];
    if (!graph) {
        cudaGraph_t gr;
        MSFEM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < 8; k++) two();  // 16 iterations per replay
        cudaError_t e = cudaStreamEndCapture(st, &gr);
        if (e != cudaSuccess) {
            set_error("two-level MINRES graph capture failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            set_error("two-level MINRES graph instantiate failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
    }
    if (stop2 > 0.0) {
        MSFEM_TRY(C.rtmp.alloc(n));
        if (!C.tk.p) {
            MSFEM_TRY(C.tk.alloc(1));
            MSFEM_CK(cudaMemsetAsync(C.tk.p, 0, sizeof(unsigned int), st));
        }
        MSFEM_TRY(C.rr_true.alloc(1));
    }
    int rounds = 0;
    for (;;) {
        MSFEM_TRY(read_st(C, st));
        if (C.h_st->done) break;
        if (16 * rounds > maxiter + 32) break;
        if (stop2 > 0.0 && rounds > 0) {
            if (C.mf_fine)
                MSFEM_TRY(kuhn_spmv64(C.ka, X, C.rtmp.p, st));
            else
                MSFEM_TRY(spmv64(F, X, C.rtmp.p));
            k_tl_true_norm<<<gvec, kVecThreads, 0, st>>>(n, C.r64.p, C.rtmp.p, S, C.partial.p + 1024, C.tk.p,
                                                         C.rr_true.p);
            double r2 = 0.0;
            MSFEM_CK(cudaMemcpyAsync(&r2, C.rr_true.p, sizeof(double), cudaMemcpyDeviceToHost, st));
            MSFEM_CK(cudaStreamSynchronize(st));
            F.total_launches += 2;
            if (r2 <= stop2) {  // converged for the outer system: stop the inner solve here
                C.h_st->done = 1;
                MSFEM_CK(cudaMemcpyAsync(&S->done, &C.h_st->done, sizeof(int), cudaMemcpyHostToDevice, st));
                MSFEM_CK(cudaStreamSynchronize(st));
                break;
            }
        }
        for (int k = 0; k < 4; k++) MSFEM_CK(cudaGraphLaunch(graph, st));
        rounds += 4;
        F.total_launches += 4 * 16 * (11 + 2 * (C.cheb_deg - 1));
    }
    *iters = C.h_st->iter;
    return C.h_st->done == 3 ? MSFEM_ERR_NUMERIC : MSFEM_OK;
}

// Chebyshev step coefficients of the Jacobi-scaled textbook operator; drops the captured cycle (it
// holds the old coefficients).  ratio > 1: the first-kind polynomial for the spectrum bound
// [lmax / ratio, lmax]; ratio 0: the fourth-kind polynomial on [0, lmax] (J. Lottes, "Optimal
// polynomial smoothers for multigrid V-cycles", 2023: d_0 = 4 / (3 lmax) r_0,
// d_k = (2k - 1) / (2k + 3) d_k-1 + (8k + 4) / ((2k + 3) lmax) r_k), which needs no lower bound
void cheb_coefs(CoarseHandle& C, double lmax, double ratio, int degree)
{
    C.lmax = lmax;
    C.ratio = ratio;
    C.cc = ChebCoef{};
    if (ratio == 0.0) {
        C.lmin = 0.0;
        C.cc.inv_theta = (float)(4.0 / (3.0 * lmax));
        for (int k = 1; k < degree; k++) {
            C.cc.a[k] = (float)((2.0 * k - 1.0) / (2.0 * k + 3.0));
            C.cc.b[k] = (float)((8.0 * k + 4.0) / ((2.0 * k + 3.0) * lmax));
        }
    } else {
        C.lmin = C.lmax / ratio;
        const double theta = 0.5 * (C.lmax + C.lmin), delta = 0.5 * (C.lmax - C.lmin), sigma = theta / delta;
        double rho = 1.0 / sigma;
        C.cc.inv_theta = (float)(1.0 / theta);
        for (int i = 1; i < degree; i++) {
            const double rn = 1.0 / (2.0 * sigma - rho);
            C.cc.a[i] = (float)(rn * rho);
            C.cc.b[i] = (float)(2.0 * rn / delta);
            rho = rn;
        }
    }
    C.cheb_deg = degree;
    if (C.graph[2]) {
        cudaGraphExecDestroy(C.graph[2]);
        C.graph[2] = nullptr;
    }
}

// Chebyshev smoothing on the textbook system: lambda_max of its Jacobi-scaled FP32 operator by
// 50 power steps (times 1.1), lambda_min = lambda_max / ratio.  The smoother -- and with it the
// symmetric cycle -- is SPD only while lambda_max really bounds the spectrum; the power estimate
// approaches it from below, so solve_twolevel widens the bound if a step ever raises the residual.
int set_smoother(CoarseHandle& C, System& T, int degree, double ratio, int storage)
{
    System& F = *C.fine;
    if (T.kind != MSFEM_ELASTIC || T.n_rows != F.n_rows || T.device != F.device) {
        set_error("msfem_coarse_set_smoother: the textbook system must be an elasticity system on the fine mesh");
        return MSFEM_ERR_ARGUMENT;
    }
    if (storage < 0 || storage > 2) {
        set_error("msfem_coarse_set_smoother: storage must be 0 (FP32), 1 (FP16) or 2 (matrix-free)");
        return MSFEM_ERR_ARGUMENT;
    }
    if (degree < 1 || degree > 8 || !(ratio > 1.0 || ratio == 0.0)) {
        set_error("msfem_coarse_set_smoother: degree must be 1..8 and ratio > 1 (or 0: fourth kind)");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(prepare_sell(T));
    cudaStream_t st = F.stream;
    MSFEM_CK(cudaStreamSynchronize(T.stream));
    const int n = T.n_rows;
    MSFEM_TRY(C.psi_t.alloc(24 * (size_t)C.n_fine));
    k_mg_psi<<<gridn(24 * (int64_t)C.n_fine), 256, 0, st>>>(C.n_fine, C.psi_hat.p, F.dscale.p, T.dscale.p, C.psi_t.p);
    C.ldv = (n + 16 + 63) / 64 * 64;  // 16-byte aligned sub-vectors with 16 elements of slack
    MSFEM_TRY(C.mgv.alloc(9 * (size_t)C.ldv));
    // power iteration from a fixed pseudo-random start
    std::vector<float> h0(n);
    for (int i = 0; i < n; i++) h0[i] = (float)((hash32((unsigned)i) & 0xffff) / 65536.0 - 0.5);
    float* v = C.mgv.p;
    float* w = v + C.ldv;
    MSFEM_CK(cudaMemcpyAsync(v, h0.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
    DBuf<double> nb;
    MSFEM_TRY(nb.alloc(2));
    DBuf<unsigned int> tk;
    MSFEM_TRY(tk.alloc(1));
    MSFEM_CK(cudaMemsetAsync(tk.p, 0, sizeof(unsigned int), st));
    k_mg_norm2<<<kReduceBlocks, kVecThreads, 0, st>>>(n, v, C.partial.p, tk.p, nb.p);
    k_mg_scale<<<kReduceBlocks, kVecThreads, 0, st>>>(n, v, nb.p);
    MSFEM_CK(cudaStreamSynchronize(st));
    // the 50 steps run back to back on the device (the norm stays there); the host reads the last
    for (int it = 0; it < 50; it++) {
        cudaStream_t ts = T.stream;
        T.stream = st;  // run the textbook system's SpMV on the solve stream
        const int rc = spmv32(T, v, w);
        T.stream = ts;
        MSFEM_TRY(rc);
        k_mg_norm2<<<kReduceBlocks, kVecThreads, 0, st>>>(n, w, C.partial.p, tk.p, nb.p);
        k_mg_scale<<<kReduceBlocks, kVecThreads, 0, st>>>(n, w, nb.p);
        std::swap(v, w);
    }
    double nrm2 = 0.0;
    MSFEM_CK(cudaMemcpyAsync(&nrm2, nb.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    const double lam = std::sqrt(nrm2);
    cheb_coefs(C, 1.1 * lam, ratio, degree);
    C.widened = 0;
    C.text = &T;
    C.storage = storage;
    C.half_matrix = storage == 1;
    C.col16.release();
    C.val16.release();
    if (storage == 2) {
        C.text = nullptr;  // usable only once the matrix-free operator passed its check
        MSFEM_TRY(kuhn_operator_build(T, 2, false, true, C.kt));
        MSFEM_CK(KChebP::prepare());
        MSFEM_CK(KResidP::prepare());
        C.text = &T;
    }
    if (C.half_matrix) {
        MSFEM_TRY(C.val16.alloc(5 * (size_t)T.sell.stored));
        k_to_half<<<gridn(T.sell.stored), 256, 0, st>>>(T.sell.stored, T.sell.val32.p, C.val16.p);
        DBuf<int> ovf;
        MSFEM_TRY(ovf.alloc(1));
        MSFEM_TRY(C.col16.alloc((size_t)T.sell.stored));
        MSFEM_CK(cudaMemsetAsync(ovf.p, 0, sizeof(int), st));
        k_block_delta16<<<gridn((int64_t)T.sell.n_slices * kSlice), 256, 0, st>>>(T.n_nodes, T.sell.n_slices,
                                                                                  T.sell.slice_ptr.p, T.sell.col.p,
                                                                                  C.col16.p, ovf.p);
        int h_ovf = 0;
        MSFEM_CK(cudaMemcpyAsync(&h_ovf, ovf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        if (h_ovf) C.col16.release();
    }
    MSFEM_CK(cudaGetLastError());
    return MSFEM_OK;
}

int solve_twolevel(CoarseHandle& C, int precision, int maxiter, double tol, double* rel, int* iters, int* outer)
{
    System& F = *C.fine;
    cudaStream_t st = F.stream;
    MSFEM_TRY(prepare_sell(F));
    MSFEM_TRY(ensure_kstate(F));
    const int n = F.n_rows;
    const bool f32 = precision == MSFEM_FP32_IR;
    DBuf<double>& rr = F.sc_f64[1];
    MSFEM_TRY(rr.alloc(2));
    cudaEvent_t e0, e1;
    MSFEM_CK(cudaEventCreate(&e0));
    MSFEM_CK(cudaEventCreate(&e1));
    MSFEM_CK(cudaEventRecord(e0, st));
    double ff = 0.0;
    {
        // (F, F) as the residual of a zero vector
        DBuf<double> zero;
        MSFEM_TRY(zero.alloc(n));
        MSFEM_CK(cudaMemsetAsync(zero.p, 0, sizeof(double) * n, st));
        MSFEM_TRY(residual64(F, zero.p, F.F.p, C.r64.p, rr.p + 1));
        MSFEM_CK(cudaMemcpyAsync(&ff, rr.p + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
    }
    int total = 0, k = 0, rc = MSFEM_OK;
    double r2 = 0.0, prev = -1.0;
    const bool mg = C.text && !f32;
    if (mg && C.storage == 2) MSFEM_TRY(kuhn_operator_current(C.kt));
    if (mg && C.mf_fine) MSFEM_TRY(kuhn_operator_current(C.ka));
    if (mg) MSFEM_TRY(C.xkeep.alloc(n));
    for (k = 0; k < 40; k++) {
        MSFEM_TRY(residual64(F, F.X.p, F.F.p, C.r64.p, rr.p));
        MSFEM_CK(cudaMemcpyAsync(&r2, rr.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        const bool failed = rc == MSFEM_ERR_NUMERIC || !(r2 == r2) || (prev >= 0.0 && r2 > prev);
        if (mg && failed && C.widened < 4) {
            // the step broke down or raised the residual: the cycle was not SPD, so lambda_max
            // was underestimated.  Undo the step, widen the bound and take it again.
            MSFEM_CK(cudaMemcpyAsync(F.X.p, C.xkeep.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            cheb_coefs(C, 1.5 * C.lmax, C.ratio, C.cheb_deg);
            C.widened++;
            if (std::getenv("MSFEM_TRACE"))
                std::fprintf(stderr, "[msfem] two-level: step failed, lambda_max widened to %.4f\n", C.lmax);
            r2 = prev;
            rc = MSFEM_OK;
        } else {
            if (!(r2 == r2)) {
                set_error("two-level solve: the residual became NaN");
                return MSFEM_ERR_NUMERIC;
            }
            if (rc == MSFEM_ERR_NUMERIC) break;
            if (r2 <= tol * tol * ff || r2 == 0.0 || total >= maxiter) break;
            if (prev >= 0.0 && r2 > 0.25 * prev) break;  // refinement no longer contracts
        }
        prev = r2;
        if (mg) MSFEM_CK(cudaMemcpyAsync(C.xkeep.p, F.X.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        const double need = tol * std::sqrt(ff / r2);
        // FP32 stops near its own precision; FP64 aims a little past what is missing
        // (the multiplicative cycle's M-norm is further from the 2-norm: aim lower, one pass)
        const double tau = f32 ? std::max(1e-5, std::min(0.5, 0.3 * need))
                               : std::max(1e-14, (C.text ? 0.02 : 0.1) * need);
        int it = 0;
        if (mg) rc = inner_solve_mg(C, maxiter - total, tau, 0.81 * tol * tol * ff, &it);
        else rc = f32 ? inner_solve<float>(C, maxiter - total, tau, &it) : inner_solve<double>(C, maxiter - total, tau, &it);
        total += it;
        if (std::getenv("MSFEM_TRACE"))
            std::fprintf(stderr, "[msfem] two-level refine %d (%s): rel %.3e tau %.1e inner %d\n", k, f32 ? "fp32" : "fp64",
                         std::sqrt(r2 / ff), tau, it);
        if (rc == MSFEM_ERR_NUMERIC && !mg) break;
        if (mg && C.mf_fine) MSFEM_TRY(kuhn_check_err(C.ka, st));
        if (rc != MSFEM_ERR_NUMERIC) {
            if (f32)
                k_tl_correct<float><<<kReduceBlocks, kVecThreads, 0, st>>>(n, F.X.p, reinterpret_cast<float*>(C.vec.p),
                                                                           F.dscale.p, C.st.p);
            else
                k_tl_correct<double><<<kReduceBlocks, kVecThreads, 0, st>>>(n, F.X.p, C.vec.p, nullptr, C.st.p);
        }
    }
    MSFEM_CK(cudaEventRecord(e1, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    MSFEM_CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    F.stats.ms_solve = ms;
    F.stats.iterations = total;
    F.stats.outer_iterations = k;
    *rel = ff > 0 ? std::sqrt(r2 / ff) : std::sqrt(r2);
    F.stats.rel_residual = *rel;
    *iters = total;
    *outer = k;
    if (mg && C.storage == 2) MSFEM_TRY(kuhn_check_err(C.kt, st));
    if (rc == MSFEM_ERR_NUMERIC) {
        set_error("two-level solve: the inner MINRES broke down");
        return MSFEM_ERR_NUMERIC;
    }
    return *rel <= tol * (1.0 + 1e-6) ? MSFEM_OK : MSFEM_NOT_CONVERGED;
}

}  // namespace
}  // namespace msfem

struct msfem_coarse : msfem::CoarseHandle {};
struct msfem_cells;
struct msfem_system;

extern "C" {

int msfem_coarse_create(msfem_system_t fine, msfem_cells_t cells, const int32_t* cell_node_global,
                        int n_coarse_vertices, const int32_t* cell_vertex, const int32_t* cell_color, int n_fixed,
                        const int32_t* fixed_dofs, msfem_coarse_t* out)
{
    using namespace msfem;
    if (!out || !fine || !cells || !cell_node_global || n_coarse_vertices <= 0 || !cell_vertex || !cell_color ||
        n_fixed < 0 || (n_fixed > 0 && !fixed_dofs)) {
        set_error("msfem_coarse_create: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    System& F = *reinterpret_cast<System*>(fine);
    CellsHandle& Ce = *reinterpret_cast<CellsHandle*>(cells);
    if (F.kind != MSFEM_ELASTIC) {
        set_error("msfem_coarse_create: the fine system must be an elasticity system");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(F.device));
    *out = nullptr;
    std::unique_ptr<msfem_coarse> h(new (std::nothrow) msfem_coarse());
    if (!h) {
        set_error("out of host memory");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(coarse_build(*h, F, Ce, cell_node_global, n_coarse_vertices, cell_vertex, cell_color, n_fixed, fixed_dofs));
    *out = h.release();
    return MSFEM_OK;
}

int msfem_coarse_info(msfem_coarse_t c, int* n_coarse_dofs, double* ms_setup)
{
    using namespace msfem;
    if (!c) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    if (n_coarse_dofs) *n_coarse_dofs = c->n_cf;
    if (ms_setup) *ms_setup = c->ms_setup;
    return MSFEM_OK;
}

int msfem_coarse_stats(msfem_coarse_t c, int* trilinear_cells, double* lambda_max, int* widened)
{
    using namespace msfem;
    if (!c) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    if (trilinear_cells) *trilinear_cells = c->n_trilinear;
    if (lambda_max) *lambda_max = c->lmax;
    if (widened) *widened = c->widened;
    return MSFEM_OK;
}

int msfem_coarse_matrix(msfem_coarse_t c, double* A, int32_t* coarse_dof)
{
    using namespace msfem;
    if (!c) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    cudaStream_t st = c->fine->stream;
    if (A)
        MSFEM_CK(cudaMemcpy2DAsync(A, sizeof(double) * c->n_cf, c->Ac.p, sizeof(double) * c->n_pad,
                                   sizeof(double) * c->n_cf, c->n_cf, cudaMemcpyDeviceToHost, st));
    if (coarse_dof)
        MSFEM_CK(cudaMemcpyAsync(coarse_dof, c->cdof.p, sizeof(int32_t) * 24 * c->n_cells, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return MSFEM_OK;
}

int msfem_coarse_apply(msfem_coarse_t c, const float* r, float* y)
{
    using namespace msfem;
    if (!c || !r || !y) {
        set_error("msfem_coarse_apply: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    System& F = *c->fine;
    cudaStream_t st = F.stream;
    const int n = F.n_rows;
    float* dr = reinterpret_cast<float*>(c->vec.p) + 5 * (size_t)n;  // inner-solve work vectors
    float* dy = reinterpret_cast<float*>(c->vec.p) + 6 * (size_t)n;
    MSFEM_CK(cudaMemcpyAsync(dr, r, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemsetAsync(c->st.p, 0, sizeof(TlState), st));
    precondition<float>(*c, dr, dy, 1, st, kReduceBlocks, nullptr);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return MSFEM_OK;
}

int msfem_solve_twolevel(msfem_system_t fine, msfem_coarse_t c, int precision, int maxiter, double tol,
                         double* rel_residual, int* iterations, int* outer)
{
    using namespace msfem;
    if (!fine || !c || maxiter <= 0 || !(tol > 0.0) || reinterpret_cast<System*>(fine) != c->fine ||
        (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("msfem_solve_twolevel: bad arguments (the coarse handle must belong to this system)");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(c->fine->device));
    double rel = 0.0;
    int it = 0, out = 0;
    const int rc = solve_twolevel(*c, precision, maxiter, tol, &rel, &it, &out);
    if (rel_residual) *rel_residual = rel;
    if (iterations) *iterations = it;
    if (outer) *outer = out;
    return rc;
}

int msfem_coarse_set_smoother(msfem_coarse_t c, msfem_system_t textbook, int degree, double ratio, int storage)
{
    using namespace msfem;
    if (!c || !textbook) {
        set_error("msfem_coarse_set_smoother: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaSetDevice(c->fine->device));
    return set_smoother(*c, *reinterpret_cast<System*>(textbook), degree, ratio, storage);
}

int msfem_coarse_set_matrix_free(msfem_coarse_t c, int on)
{
    using namespace msfem;
    if (!c) {
        set_error("msfem_coarse_set_matrix_free: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    CoarseHandle& C = *c;
    MSFEM_CK(cudaSetDevice(C.fine->device));
    C.mf_fine = false;
    if (C.graph[2]) {
        cudaGraphExecDestroy(C.graph[2]);
        C.graph[2] = nullptr;
    }
    if (!on) return MSFEM_OK;
    MSFEM_TRY(kuhn_operator_build(*C.fine, 1, true, false, C.ka));
    MSFEM_CK(KMinres::prepare());
    C.mf_fine = true;
    return MSFEM_OK;
}

int msfem_coarse_bench_smoother(msfem_coarse_t c, int reps, double* ms_per_step, int64_t* bytes_per_step)
{
    using namespace msfem;
    if (!c || !c->text || reps <= 0 || !ms_per_step || !bytes_per_step) {
        set_error("msfem_coarse_bench_smoother: bad arguments (set the smoother first)");
        return MSFEM_ERR_ARGUMENT;
    }
    CoarseHandle& C = *c;
    System& T = *C.text;
    MSFEM_CK(cudaSetDevice(C.fine->device));
    cudaStream_t st = C.fine->stream;
    const int n = T.n_rows;
    const int64_t ld = C.ldv;
    float* res = C.mgv.p + ld;
    float* dA = res + ld;
    float* dB = dA + ld;
    float* x = dB + ld;
    float* dhA = x + 2 * ld;
    float* dhB = dhA + ld;
    MSFEM_CK(cudaMemsetAsync(C.mgv.p, 0, sizeof(float) * 9 * (size_t)ld, st));
    DBuf<TlState> run;  // a state that is not done, so the kernel does its work
    MSFEM_TRY(run.alloc(1));
    MSFEM_CK(cudaMemsetAsync(run.p, 0, sizeof(TlState), st));
    const SellView<float> At = sell_view<float>(T);
    const unsigned gsp = spmv_grid_of((const void*)k_mg_cheb, T);
    const __half2* v16 = C.half_matrix ? C.val16.p : nullptr;
    const int16_t* c16 = C.half_matrix ? C.col16.p : nullptr;
    const bool mf = C.storage == 2;
    if (mf) MSFEM_TRY(kuhn_operator_current(C.kt));
    auto step = [&](int i) {
        float* dp = (i & 1) ? dB : dA;
        float* dn = (i & 1) ? dA : dB;
        if (mf)
            KChebP::launch(C.kt.v32, (i & 1) ? dhB : dhA,
                           EpiChebP{dn, (i & 1) ? dhA : dhB, res, x, dp, C.kt.v32.scale, C.cc.a[1], C.cc.b[1], run.p,
                                    nullptr},
                           C.kt.sms, C.kt.err.p, st);
        else
            k_mg_cheb<<<gsp, 256, 0, st>>>(At, v16, c16, dp, dn, res, x, C.cc.a[1], C.cc.b[1], run.p);
    };
    for (int i = 0; i < 3; i++) step(i);
    cudaEvent_t e0, e1;
    MSFEM_CK(cudaEventCreate(&e0));
    MSFEM_CK(cudaEventCreate(&e1));
    MSFEM_CK(cudaEventRecord(e0, st));
    for (int i = 0; i < reps; i++) step(i);
    MSFEM_CK(cudaEventRecord(e1, st));
    MSFEM_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    MSFEM_CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MSFEM_CK(cudaGetLastError());
    *ms_per_step = ms / reps;
    // matrix values (FP16 pairs: 5 x 4 B per block, FP32: 36 B) and block columns, each once;
    // slice pointers; per DOF the previous direction (4 B), res read and written (8 B), the new
    // direction (4 B), x read and written (8 B).  Matrix-free: instead of the matrix, per DOF the
    // Jacobi scale (4 B) and the scaled input read and the next one written (8 B), per node its
    // Dirichlet bits (4 B), per tetrahedron its material (1 B)
    if (mf) {
        *bytes_per_step = (int64_t)n * (24 + 12) + (int64_t)T.n_nodes * 4 + (int64_t)T.n_tets;
    } else {
        const int64_t vb = C.half_matrix ? 20 : 36;
        const int64_t cb = c16 ? 2 : 4;
        *bytes_per_step = T.sell.stored * (vb + cb) + (int64_t)(T.sell.n_slices + 1) * 8 + (int64_t)n * 24;
    }
    T.total_launches += 3 + reps;
    if (mf) MSFEM_TRY(kuhn_check_err(C.kt, st));
    return MSFEM_OK;
}

void msfem_coarse_destroy(msfem_coarse_t c)
{
    if (!c) return;
    cudaSetDevice(c->fine->device);
    cudaStreamSynchronize(c->fine->stream);
    delete c;
}

}  // extern "C"
