// Matrix-free elasticity operators on a structured Kuhn grid.
//
// A mesh of nx x ny x nz hexahedra, each cut into the six Kuhn tetrahedra that share its 0-7
// diagonal (corner b of hexahedron (i, j, k) at (i + (b & 1), j + (b >> 1 & 1), k + (b >> 2 & 1)),
// node id i + (nx+1) (j + (ny+1) k), tetrahedra 6c .. 6c+5 of hexahedron c = i + nx (j + ny k)
// with corners {0,1,3,7} {0,1,5,7} {0,2,3,7} {0,2,6,7} {0,4,5,7} {0,4,6,7}), has congruent
// elements: tetrahedron {0, p, q, 7} walks the axes a, b, c of its corner path 0 -> p -> q -> 7,
// its basis gradients are -e_a/h_a, e_a/h_a - e_b/h_b, e_b/h_b - e_c/h_c, e_c/h_c and its volume
// is hx hy hz / 6.  With the displacement gradient G (column s = du/dx_s, a difference of two
// corner values) the element force on vertex I is V sigma g_I, where
//   textbook orientation (symmetric, semi-definite):   sigma = lambda tr(G) I + mu (G + G^T)
//   the reference's assembly (FEM_Grid.h:2125-2192):   sigma = mu tr(G) I + mu G + lambda G^T
// -- the two block formulas of k_assemble_elastic, summed over the element's columns -- so the
// product of the assembled matrix with a vector needs only a material code per tetrahedron: about
// 100 bytes per node (vectors included) instead of ~430 bytes of FP16 blocks or ~1.2 KB of FP64.
//
// One CTA owns a brick of BX x BY x BZ nodes.  Phase 0 stages the input on the brick's nodes and a
// one-node halo in shared memory (scaled by the Jacobi scale, zero on eliminated Dirichlet
// columns); phase 1 has one thread per hexahedron touching the brick add its six tetrahedra's
// forces into its eight corner sums (fixed order); phase 2 gives each owned node the sum of the
// eight hexahedra around it, corner 0 .. 7 in order.  No atomics: the product is deterministic.
#pragma once

#include <cstdint>

namespace msfem {

constexpr int kKuhnMaxMat = 64;  // materials in the table a launch stages in shared memory

template <class T>
struct KuhnView {
    int nx, ny, nz;                     // hexahedra per axis
    int nbx, nby, nbz;                  // bricks per axis
    T ih[3];                            // 1 / h per axis
    T vh[3];                            // V / h per axis (V = hx hy hz / 6)
    const uint2* __restrict__ mat;      // per hexahedron the material codes of its six tetrahedra (bytes 0..5)
    const uint32_t* __restrict__ fix;   // per node: bit a = row 3n+a is a Dirichlet row; bit 3+a = column eliminated
    const T* __restrict__ scale;        // per DOF Jacobi scale of the operator S K S (nullptr: K itself)
    const T* __restrict__ lame;         // [n_mat][2] lambda, mu (iso: lambda V/h^2, mu V/h^2)
    int n_mat;
    int iso;                            // hx = hy = hz and the table folded (kuhn_tet_iso)
};

// the forces of one tetrahedron {0, P, Q, 7} with corner path axes (A, B, C) on its corners
// FORM 1: the reference's assembly; FORM 2: the textbook orientation
template <int FORM, int A, int B, int C, class T>
__device__ __forceinline__ void kuhn_tet(const T* u0, const T* up, const T* uq, const T* u7, T lam, T mu,
                                         const T* ih, const T* vh, T* f0, T* fp, T* fq, T* f7)
{
    T col[3][3];  // col[s][r] = G[r][s] = du_r / dx_s
#pragma unroll
    for (int r = 0; r < 3; r++) {
        col[A][r] = (up[r] - u0[r]) * ih[A];
        col[B][r] = (uq[r] - up[r]) * ih[B];
        col[C][r] = (u7[r] - uq[r]) * ih[C];
    }
    const T tr = col[0][0] + col[1][1] + col[2][2];
    T tau[3][3];  // tau[s] = V sigma[:, s] / h_s
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            T sg;
            if (FORM == 2)  // textbook: lambda tr delta + mu (G[r][s] + G[s][r])
                sg = mu * (col[s][r] + col[r][s]) + (r == s ? lam * tr : T(0));
            else            // reference: mu tr delta + mu G[r][s] + lambda G[s][r]
                sg = mu * col[s][r] + lam * col[r][s] + (r == s ? mu * tr : T(0));
            tau[s][r] = sg * vh[s];
        }
#pragma unroll
    for (int r = 0; r < 3; r++) {
        f0[r] -= tau[A][r];
        fp[r] += tau[A][r] - tau[B][r];
        fq[r] += tau[B][r] - tau[C][r];
        f7[r] += tau[C][r];
    }
}

// The same forces on an isotropic grid (hx = hy = hz = h) with the material table holding
// lambda V / h^2 and mu V / h^2: the gradient columns are the raw corner differences and the
// column scaling is folded into the table (18 multiplies fewer); the textbook stress is formed
// once per symmetric pair.
template <int FORM, int A, int B, int C, class T>
__device__ __forceinline__ void kuhn_tet_iso(const T* u0, const T* up, const T* uq, const T* u7, T lam, T mu, T* f0,
                                             T* fp, T* fq, T* f7)
{
    T col[3][3];  // col[s][r] = h du_r / dx_s
#pragma unroll
    for (int r = 0; r < 3; r++) {
        col[A][r] = up[r] - u0[r];
        col[B][r] = uq[r] - up[r];
        col[C][r] = u7[r] - uq[r];
    }
    const T tr = col[0][0] + col[1][1] + col[2][2];
    T sg[3][3];  // sg[s][r] = sigma[r][s], scaled
    if (FORM == 2) {
        const T lt = lam * tr, m2 = mu + mu;
#pragma unroll
        for (int r = 0; r < 3; r++) sg[r][r] = m2 * col[r][r] + lt;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int s = r + 1; s < 3; s++) sg[s][r] = sg[r][s] = mu * (col[s][r] + col[r][s]);
    } else {
        const T mt = mu * tr;
#pragma unroll
        for (int s = 0; s < 3; s++)
#pragma unroll
            for (int r = 0; r < 3; r++) sg[s][r] = mu * col[s][r] + lam * col[r][s] + (r == s ? mt : T(0));
    }
#pragma unroll
    for (int r = 0; r < 3; r++) {
        f0[r] -= sg[A][r];
        fp[r] += sg[A][r] - sg[B][r];
        fq[r] += sg[B][r] - sg[C][r];
        f7[r] += sg[C][r];
    }
}

// shared memory of one brick: staged input (3 components x halo nodes) + corner sums (24 x hexahedra)
template <class T, int BX, int BY, int BZ>
struct KuhnBrick {
    static constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2;  // staged nodes
    static constexpr int CX = BX + 1, CY = BY + 1, CZ = BZ + 1;  // hexahedra touching the brick
    static constexpr int NH = HX * HY * HZ;
    static constexpr int NC = CX * CY * CZ;
    static constexpr size_t smem = sizeof(T) * (3 * (size_t)NH + 24 * (size_t)NC + 2 * kKuhnMaxMat);
};

// y = (S K S) x on brick `brick` (rows of Dirichlet DOFs: y = x); epi(node, y[3]) per owned node
template <int FORM, int BX, int BY, int BZ, int THREADS, class T, class Epi>
__device__ __forceinline__ void kuhn_brick(const KuhnView<T>& K, const T* __restrict__ x, int brick, T* su, T* sc,
                                           const T* slame, Epi& epi)
{
    using L = KuhnBrick<T, BX, BY, BZ>;
    const int bx = brick % K.nbx;
    const int by = (brick / K.nbx) % K.nby;
    const int bz = brick / (K.nbx * K.nby);
    const int i0 = bx * BX, j0 = by * BY, k0 = bz * BZ;
    const int nnx = K.nx + 1, nny = K.ny + 1, nnz = K.nz + 1;
    // phase 0: staged u = s x on nodes i0-1 .. i0+BX (zero outside the grid and on eliminated
    // columns).  Every load of the phase is independent and issued before any is used (addresses
    // clamped into the arrays, results selected afterwards), and the material codes of this
    // thread's phase-1 hexahedra are fetched with them: one memory round trip per brick.
    constexpr int kE0 = 3 * L::NH, kPer0 = (kE0 + THREADS - 1) / THREADS;
    constexpr int kPer1 = (L::NC + THREADS - 1) / THREADS;
    T xv[kPer0], sv[kPer0];
    uint32_t fx[kPer0];
    bool in0[kPer0];
#pragma unroll
    for (int r = 0; r < kPer0; r++) {
        const int e = threadIdx.x + r * THREADS;
        const int row = e / (3 * L::HX);
        const int w = e - row * (3 * L::HX);
        const int hi = w / 3, a = w - 3 * hi;
        const int hj = row % L::HY, hk = row / L::HY;
        const int gi = i0 - 1 + hi, gj = j0 - 1 + hj, gk = k0 - 1 + hk;
        in0[r] = e < kE0 && gi >= 0 && gi < nnx && gj >= 0 && gj < nny && gk >= 0 && gk < nnz;
        const int64_t g = in0[r] ? gi + (int64_t)nnx * (gj + (int64_t)nny * gk) : 0;
        fx[r] = __ldg(K.fix + g);
        xv[r] = __ldg(x + 3 * g + (in0[r] ? a : 0));
        sv[r] = K.scale ? __ldg(K.scale + 3 * g + (in0[r] ? a : 0)) : T(1);
    }
    uint2 mc[kPer1];
    bool in1[kPer1];
#pragma unroll
    for (int r = 0; r < kPer1; r++) {
        const int c = threadIdx.x + r * THREADS;
        const int ci = c % L::CX, cj = (c / L::CX) % L::CY, ck = c / (L::CX * L::CY);
        const int gi = i0 - 1 + ci, gj = j0 - 1 + cj, gk = k0 - 1 + ck;
        in1[r] = c < L::NC && gi >= 0 && gi < K.nx && gj >= 0 && gj < K.ny && gk >= 0 && gk < K.nz;
        const int64_t cube = in1[r] ? gi + (int64_t)K.nx * (gj + (int64_t)K.ny * gk) : 0;
        mc[r] = __ldg(K.mat + cube);
    }
#pragma unroll
    for (int r = 0; r < kPer0; r++) {
        const int e = threadIdx.x + r * THREADS;
        if (e < kE0) {
            const int row = e / (3 * L::HX);
            const int w = e - row * (3 * L::HX);
            const int hi = w / 3, a = w - 3 * hi;
            const int hj = row % L::HY, hk = row / L::HY;
            const bool keep = in0[r] && !((fx[r] >> (3 + a)) & 1u);
            su[a * L::NH + hi + L::HX * (hj + L::HY * hk)] = keep ? xv[r] * sv[r] : T(0);
        }
    }
    __syncthreads();
    // phase 1: per hexahedron, the corner sums of its six tetrahedra
#pragma unroll
    for (int r = 0; r < kPer1; r++) {
        const int c = threadIdx.x + r * THREADS;
        if (c >= L::NC) break;
        const int ci = c % L::CX, cj = (c / L::CX) % L::CY, ck = c / (L::CX * L::CY);
        T f[8][3];
#pragma unroll
        for (int b = 0; b < 8; b++) f[b][0] = f[b][1] = f[b][2] = T(0);
        if (in1[r]) {
            T u[8][3];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int h = (ci + (b & 1)) + L::HX * ((cj + ((b >> 1) & 1)) + L::HY * (ck + ((b >> 2) & 1)));
#pragma unroll
                for (int a = 0; a < 3; a++) u[b][a] = su[a * L::NH + h];
            }
            T lam[6], mu[6];
#pragma unroll
            for (int t = 0; t < 6; t++) {
                const int m = ((t < 4 ? mc[r].x >> (8 * t) : mc[r].y >> (8 * (t - 4)))) & 0xff;
                lam[t] = slame[2 * m];
                mu[t] = slame[2 * m + 1];
            }
            // {0,1,3,7}: x y z   {0,1,5,7}: x z y   {0,2,3,7}: y x z
            // {0,2,6,7}: y z x   {0,4,5,7}: z x y   {0,4,6,7}: z y x
            kuhn_tet<FORM, 0, 1, 2>(u[0], u[1], u[3], u[7], lam[0], mu[0], K.ih, K.vh, f[0], f[1], f[3], f[7]);
            kuhn_tet<FORM, 0, 2, 1>(u[0], u[1], u[5], u[7], lam[1], mu[1], K.ih, K.vh, f[0], f[1], f[5], f[7]);
            kuhn_tet<FORM, 1, 0, 2>(u[0], u[2], u[3], u[7], lam[2], mu[2], K.ih, K.vh, f[0], f[2], f[3], f[7]);
            kuhn_tet<FORM, 1, 2, 0>(u[0], u[2], u[6], u[7], lam[3], mu[3], K.ih, K.vh, f[0], f[2], f[6], f[7]);
            kuhn_tet<FORM, 2, 0, 1>(u[0], u[4], u[5], u[7], lam[4], mu[4], K.ih, K.vh, f[0], f[4], f[5], f[7]);
            kuhn_tet<FORM, 2, 1, 0>(u[0], u[4], u[6], u[7], lam[5], mu[5], K.ih, K.vh, f[0], f[4], f[6], f[7]);
        }
#pragma unroll
        for (int b = 0; b < 8; b++)
#pragma unroll
            for (int a = 0; a < 3; a++) sc[(3 * b + a) * L::NC + c] = f[b][a];
    }
    __syncthreads();
    // phase 2: each owned node sums its eight hexahedra (corner b of hexahedron node - offset(b))
    for (int q = threadIdx.x; q < BX * BY * BZ; q += THREADS) {
        const int ni = q % BX, nj = (q / BX) % BY, nk = q / (BX * BY);
        const int gi = i0 + ni, gj = j0 + nj, gk = k0 + nk;
        if (gi >= nnx || gj >= nny || gk >= nnz) continue;
        const int64_t g = gi + (int64_t)nnx * (gj + (int64_t)nny * gk);
        T y[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int c = (ni + 1 - (b & 1)) + L::CX * ((nj + 1 - ((b >> 1) & 1)) + L::CY * (nk + 1 - ((b >> 2) & 1)));
#pragma unroll
            for (int a = 0; a < 3; a++) y[a] += sc[(3 * b + a) * L::NC + c];
        }
        const uint32_t fx = __ldg(K.fix + g);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if ((fx >> a) & 1u)
                y[a] = __ldg(x + 3 * g + a);
            else if (K.scale)
                y[a] *= __ldg(K.scale + 3 * g + a);
        }
        epi(g, y);
    }
}

// stages the material table in shared memory
template <class T>
__device__ __forceinline__ void kuhn_stage_lame(const KuhnView<T>& K, T* slame)
{
    for (int i = threadIdx.x; i < 2 * kKuhnMaxMat; i += blockDim.x) slame[i] = i < 2 * K.n_mat ? K.lame[i] : T(0);
}

}  // namespace msfem
