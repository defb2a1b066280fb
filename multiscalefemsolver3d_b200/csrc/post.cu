// Elasticity post-processing after the solve, one thread per tetrahedron: the reference grid's
// per-element fields at the centroid (FEM/FEM_Grid.h:3289-3365: GetSolutionInPoint,
// GetDerevativeFromSolutionInPoint, GetStressTensorFromSolutionInPoint through
// Domain::forMech::solve_SIGMA, Library/Domain.h:231-290, and GetVonMisesStress) and the fields
// the elasticity driver prints (FEM/FEM_Main.cpp:1018-1040: domain 0's material for every element,
// engineering shear strains, shear stresses k 2 b gamma, its own von Mises line).
#include <vector>

#include "element.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

constexpr int kPostFields = 23;

// out[e] = U(3), dU(9: row a = grad u_a), sigma (xx yy zz yz xz xy), von Mises,
//          driver sigma_xx, sigma_yy, sigma_zz, driver von Mises
__global__ void k_postprocess(int n_tets, const double* __restrict__ xyz, const int32_t* __restrict__ tets,
                              const int32_t* __restrict__ mat, int n_mat, const double* __restrict__ X,
                              const double* __restrict__ Dm, double k0, double a0, double b0,
                              double* __restrict__ out, int* bad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_tets; e += gridDim.x * blockDim.x) {
        int v[4];
        for (int k = 0; k < 4; k++) v[k] = tets[4 * (int64_t)e + k];
        TetGeom G;
        tet_geometry(xyz, v, G);
        double U[3] = {0, 0, 0}, dU[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int j = 0; j < 4; j++)
            for (int a = 0; a < 3; a++) {
                const double xa = X[3 * (int64_t)v[j] + a];
                U[a] += 0.25 * xa;
                for (int d = 0; d < 3; d++) dU[a][d] += xa * G.g[j][d];
            }
        double* o = out + (int64_t)kPostFields * e;
        for (int a = 0; a < 3; a++) {
            o[a] = U[a];
            for (int d = 0; d < 3; d++) o[3 + 3 * a + d] = dU[a][d];
        }
        const int m = mat ? mat[e] : 0;
        if (m < 0 || m >= n_mat) {
            atomicExch(bad, 1);
            for (int q = 12; q < kPostFields; q++) o[q] = 0.0;
            continue;
        }
        // strain (symmetric part) in Voigt order with engineering shears, sigma = D veps
        const double ve[6] = {dU[0][0], dU[1][1], dU[2][2], dU[1][2] + dU[2][1], dU[0][2] + dU[2][0], dU[0][1] + dU[1][0]};
        const double* D = Dm + 36 * (int64_t)m;
        double s[6];
        for (int i = 0; i < 6; i++) {
            double acc = 0.0;
            for (int j = 0; j < 6; j++) acc += D[6 * i + j] * ve[j];
            s[i] = acc;
        }
        for (int i = 0; i < 6; i++) o[12 + i] = s[i];
        // s: xx yy zz yz xz xy; the tensor's off-diagonal pairs are equal
        o[18] = sqrt((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) + (s[0] - s[2]) * (s[0] - s[2]) +
                     6.0 * (s[5] * s[5] + s[4] * s[4] + s[3] * s[3]) / 2.0);
        // the driver's printed fields: its strain order xx yy zz xy yz xz and domain 0's constants
        const double ed[6] = {dU[0][0], dU[1][1], dU[2][2], dU[0][1] + dU[1][0], dU[1][2] + dU[2][1], dU[0][2] + dU[2][0]};
        const double sd[6] = {k0 * (ed[0] + ed[1] * a0 + ed[2] * a0), k0 * (ed[0] * a0 + ed[1] + ed[2] * a0),
                              k0 * (ed[0] * a0 + ed[1] * a0 + ed[2]), k0 * (2 * ed[3] * b0), k0 * (2 * ed[4] * b0),
                              k0 * (2 * ed[5] * b0)};
        o[19] = sd[0];
        o[20] = sd[1];
        o[21] = sd[2];
        o[22] = sqrt((sd[0] - sd[1]) * (sd[0] - sd[1]) + (sd[1] - sd[2]) * (sd[1] - sd[2]) + (sd[0] - sd[2]) * (sd[0] - sd[2]) +
                     6.0 * (sd[3] * sd[3] + sd[4] * sd[4] + sd[5] * sd[5]) / 2.0);
    }
}

// Domain::forMech::SetIsotropic_D (Library/Domain.h:53-78): k (1, a, a | b shear diagonal)
void isotropic_D(double E, double nu, double* D)
{
    const double k = E * (1.0 - nu) / (1.0 + nu) / (1.0 - 2.0 * nu);
    const double b = (1.0 - 2.0 * nu) / (2.0 * (1.0 - nu));
    const double a = nu / (1.0 - nu);
    for (int i = 0; i < 36; i++) D[i] = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[6 * i + j] = k * (i == j ? 1.0 : a);
    for (int i = 3; i < 6; i++) D[6 * i + i] = k * b;
}

}  // namespace
}  // namespace msfem

extern "C" int msfem_postprocess_elastic(msfem_system_t h, int n_materials, const double* E, const double* nu,
                                         double* out, int on_device)
{
    using namespace msfem;
    System* S = reinterpret_cast<System*>(h);
    if (!S || S->kind != MSFEM_ELASTIC || n_materials <= 0 || !E || !nu || !out) {
        set_error("msfem_postprocess_elastic: bad arguments (an elasticity system, materials, output)");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int m = 0; m < n_materials; m++)
        if (!(E[m] > 0.0) || !(nu[m] > -1.0 && nu[m] < 0.5)) {
            set_error("msfem_postprocess_elastic: material %d has E = %g, nu = %g", m, E[m], nu[m]);
            return MSFEM_ERR_ARGUMENT;
        }
    MSFEM_CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    if (!S->X.p) {
        set_error("msfem_postprocess_elastic: the system has no solution vector");
        return MSFEM_ERR_ARGUMENT;
    }
    std::vector<double> hD(36 * (size_t)n_materials);
    for (int m = 0; m < n_materials; m++) isotropic_D(E[m], nu[m], hD.data() + 36 * m);
    const double v0 = nu[0];
    const double k0 = E[0] * (1.0 - v0) / (1.0 + v0) / (1.0 - 2.0 * v0);
    const double a0 = v0 / (1.0 - v0), b0 = (1.0 - 2.0 * v0) / (2.0 * (1.0 - v0));
    DBuf<double> dD, dout;
    DBuf<int> bad;
    MSFEM_TRY(dD.alloc(hD.size()));
    MSFEM_TRY(bad.alloc(1));
    double* o = out;
    if (!on_device) {
        MSFEM_TRY(dout.alloc((size_t)kPostFields * S->n_tets));
        o = dout.p;
    }
    MSFEM_CK(cudaMemcpyAsync(dD.p, hD.data(), sizeof(double) * hD.size(), cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    const int grid = (int)std::min<int64_t>(((int64_t)S->n_tets + 255) / 256, 148 * 32);
    if (S->n_tets > 0)
        k_postprocess<<<grid, 256, 0, st>>>(S->n_tets, S->xyz.p, S->tets.p, S->mat.p, n_materials, S->X.p, dD.p, k0, a0,
                                            b0, o, bad.p);
    MSFEM_CK(cudaGetLastError());
    if (!on_device)
        MSFEM_CK(cudaMemcpyAsync(out, dout.p, sizeof(double) * kPostFields * S->n_tets, cudaMemcpyDeviceToHost, st));
    int hb = 0;
    MSFEM_CK(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (hb) {
        set_error("msfem_postprocess_elastic: a tetrahedron has a material id outside 0..%d", n_materials - 1);
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}
