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
// The kernel that applies it is the z-marching one of kuhn25.cuh.
#pragma once

#include <cstdint>

namespace msfem {

constexpr int kKuhnMaxMat = 64;  // materials in the table a launch stages in shared memory

template <class T>
struct KuhnView {
    int nx, ny, nz;                     // hexahedra per axis
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

// stages the material table in shared memory
template <class T>
__device__ __forceinline__ void kuhn_stage_lame(const KuhnView<T>& K, T* slame)
{
    for (int i = threadIdx.x; i < 2 * kKuhnMaxMat; i += blockDim.x) slame[i] = i < 2 * K.n_mat ? K.lame[i] : T(0);
}

}  // namespace msfem
