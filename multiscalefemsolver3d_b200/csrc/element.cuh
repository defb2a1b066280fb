// P1 simplex geometry and the reference's elasticity element block, shared by
// the single-system assembly (assemble.cu) and the batched cell systems
// (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace msfem {

struct TetGeom {
    double g[4][3];  // gradients of the four P1 basis functions
    double vol;      // |det| / 6
};

// Gradients from edge vectors: for e_k = p_k - p_0, grad(l1) = (e2 x e3)/det,
// grad(l2) = (e3 x e1)/det, grad(l3) = (e1 x e2)/det, grad(l0) = -sum; these are
// the alpha[v][1..3] of Tetrahedron::SolveAlphaMatrix (GeometryShape.h:1960-2086)
// and vol = GetVolume (:1674-1705).
__device__ __forceinline__ void tet_geometry(const double* __restrict__ xyz, const int v[4], TetGeom& t)
{
    double p0[3], e1[3], e2[3], e3[3];
#pragma unroll
    for (int a = 0; a < 3; a++) p0[a] = xyz[3 * (int64_t)v[0] + a];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        e1[a] = xyz[3 * (int64_t)v[1] + a] - p0[a];
        e2[a] = xyz[3 * (int64_t)v[2] + a] - p0[a];
        e3[a] = xyz[3 * (int64_t)v[3] + a] - p0[a];
    }
    const double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
    const double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
    const double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
    const double inv = 1.0 / det;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        t.g[1][a] = c23[a] * inv;
        t.g[2][a] = c31[a] * inv;
        t.g[3][a] = c12[a] * inv;
        t.g[0][a] = -(t.g[1][a] + t.g[2][a] + t.g[3][a]);
    }
    t.vol = fabs(det) / 6.0;
}

// Triangle in 3-D (the face elements of FEM/FEM_Grid.h:4420-4530): with
// e1 = p1 - p0, e2 = p2 - p0 and n = e1 x e2, the in-plane gradients are
// grad(l1) = (e2 x n)/|n|^2, grad(l2) = (n x e1)/|n|^2, grad(l0) = -sum, and the
// area |n|/2.  The reference's local-frame derivatives (FEM_Grid.h:4888-4935)
// are these vectors written in the element's own orthonormal frame.
__device__ __forceinline__ void tri_geometry(const double* __restrict__ xyz, const int v[3], double g[3][3], double& area)
{
    double p0[3], e1[3], e2[3];
#pragma unroll
    for (int a = 0; a < 3; a++) p0[a] = xyz[3 * (int64_t)v[0] + a];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        e1[a] = xyz[3 * (int64_t)v[1] + a] - p0[a];
        e2[a] = xyz[3 * (int64_t)v[2] + a] - p0[a];
    }
    const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const double inv = 1.0 / nn;
    const double g1[3] = {e2[1] * n[2] - e2[2] * n[1], e2[2] * n[0] - e2[0] * n[2], e2[0] * n[1] - e2[1] * n[0]};
    const double g2[3] = {n[1] * e1[2] - n[2] * e1[1], n[2] * e1[0] - n[0] * e1[2], n[0] * e1[1] - n[1] * e1[0]};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        g[1][a] = g1[a] * inv;
        g[2][a] = g2[a] * inv;
        g[0][a] = -(g[1][a] + g[2][a]);
    }
    area = 0.5 * sqrt(nn);
}

// The element block of FEM_Grid.h:2147-2191 (tetrahedra), :4429-4500
// (triangles) and :3649-3720 (segments) for row node I and column node J:
//   A[I][J][a][b] = meas * (lambda gJ_a gI_b + mu gI_a gJ_b + mu delta_ab gI.gJ)
__device__ __forceinline__ void elastic_block(const double* gi, const double* gj, double meas, double lam, double mu,
                                              double out[9])
{
    const double dd = mu * (gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]);
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            double v = lam * gj[a] * gi[b] + mu * gi[a] * gj[b];
            if (a == b) v += dd;
            out[3 * a + b] = meas * v;
        }
}

}  // namespace msfem
