// Coloured, deterministic element assembly into the node-level portrait.
//
// The reference computes every element matrix in an OpenMP loop and then adds
// them into CSSD_Matrix serially, element by element, finding each target entry
// by a linear search of the row (FEM/FEM.h:1349-1384, CSSD_Matrix.h:307-363).
// Here one launch per element colour class computes the element matrices and
// adds them straight into the matrix through the precomputed element -> slot
// map: elements of one colour share no node, so no two threads touch the same
// entry, no atomics are needed and every entry receives its contributions in
// the same (colour) order on every run.
#include <cub/cub.cuh>

#include "devutil.cuh"
#include "element.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

__device__ __forceinline__ void load_tet(const int32_t* __restrict__ tets, int e, int v[4])
{
    const int4 q = __ldg(reinterpret_cast<const int4*>(tets) + e);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
}

__device__ __forceinline__ void load_slots(const int32_t* __restrict__ eslot, int e, int s[16])
{
    const int4* p = reinterpret_cast<const int4*>(eslot) + 4 * (int64_t)e;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int4 v = __ldg(p + q);
        s[4 * q] = v.x;
        s[4 * q + 1] = v.y;
        s[4 * q + 2] = v.z;
        s[4 * q + 3] = v.w;
    }
}

// FEM_Grid.h:103-152: K_IJ = sigma * grad(phi_I).grad(phi_J) * V (1-point rule, weight V)
__global__ void k_assemble_scalar(int count, const int32_t* __restrict__ elems, const int32_t* __restrict__ tets,
                                  const double* __restrict__ xyz, const int32_t* __restrict__ mat,
                                  const double* __restrict__ sigma, int n_mat, const int32_t* __restrict__ eslot,
                                  double* __restrict__ val, int* bad)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int e = elems[t];
    const int m = mat ? mat[e] : 0;
    if (m < 0 || m >= n_mat) {
        atomicExch(bad, 1);
        return;
    }
    int v[4], s[16];
    load_tet(tets, e, v);
    load_slots(eslot, e, s);
    TetGeom G;
    tet_geometry(xyz, v, G);
    const double sv = sigma[m];
#pragma unroll
    for (int I = 0; I < 4; I++)
#pragma unroll
        for (int J = 0; J < 4; J++) {
            double k = sv * (G.g[I][0] * G.g[J][0] + G.g[I][1] * G.g[J][1] + G.g[I][2] * G.g[J][2]) * G.vol;
            val[s[4 * I + J]] += k;
        }
}

// FEM_Grid.h:25-102, the three-coefficient element with the one-point rule (centroid, weight V):
// A_IJ = V (S g_I.g_J + M / 16), F_I += V f / 4, with the element's coefficients S, M, f (the
// reference's koef(elem, X) at the centroid).  Elements of one colour share no node, so the F
// updates do not race.
__global__ void k_assemble_scalar3(int count, const int32_t* __restrict__ elems, const int32_t* __restrict__ tets,
                                   const double* __restrict__ xyz, const double* __restrict__ S,
                                   const double* __restrict__ M, const double* __restrict__ f,
                                   const int32_t* __restrict__ eslot, double* __restrict__ val, double* __restrict__ F)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int e = elems[t];
    int v[4], sl[16];
    load_tet(tets, e, v);
    load_slots(eslot, e, sl);
    TetGeom G;
    tet_geometry(xyz, v, G);
    const double se = S[e], m16 = M[e] / 16.0;
#pragma unroll
    for (int I = 0; I < 4; I++)
#pragma unroll
        for (int J = 0; J < 4; J++) {
            const double k = se * (G.g[I][0] * G.g[J][0] + G.g[I][1] * G.g[J][1] + G.g[I][2] * G.g[J][2]) + m16;
            val[sl[4 * I + J]] += k * G.vol;
        }
    const double fe = f[e] * G.vol / 4.0;
#pragma unroll
    for (int I = 0; I < 4; I++) F[v[I]] += fe;
}

// FEM_Grid.h:2125-2192.  The reference forms B_J^T D B_I (3x6 * 6x6 * 6x3) at
// each of the 4 quadrature points; for the isotropic D of Domain.h:53-78 with
// lambda = k*a and mu = k*b that product is, entry by entry,
//   A[I][J][a][b] = V * (lambda * gJ_a * gI_b + mu * gI_a * gJ_b + mu * delta_ab * gI.gJ)
// (g = basis gradient), which also equals the reference's mirrored blocks
// A[J][I] = A[I][J]^T, so all 16 blocks come from this one expression.
// TEXTBOOK: the textbook orientation lambda gI_a gJ_b + mu gJ_a gI_b (the transpose of every
// block), symmetric positive semi-definite; used to build preconditioners, not by the reference.
template <bool TEXTBOOK>
__global__ void k_assemble_elastic(int count, const int32_t* __restrict__ elems, const int32_t* __restrict__ tets,
                                   const double* __restrict__ xyz, const int32_t* __restrict__ mat,
                                   const double* __restrict__ lame /* [n_mat][2] */, int n_mat,
                                   const int32_t* __restrict__ eslot, double* __restrict__ val, int* bad)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int e = elems[t];
    const int m = mat ? mat[e] : 0;
    if (m < 0 || m >= n_mat) {
        atomicExch(bad, 1);
        return;
    }
    const double lam = lame[2 * m], mu = lame[2 * m + 1];
    if (lam == 0.0 && mu == 0.0) return;  // E <= 0: the element contributes nothing (FEM/FEM.h:1355-1363)
    int v[4], s[16];
    load_tet(tets, e, v);
    load_slots(eslot, e, s);
    TetGeom G;
    tet_geometry(xyz, v, G);
    const double V = G.vol;
#pragma unroll
    for (int I = 0; I < 4; I++)
#pragma unroll
        for (int J = 0; J < 4; J++) {
            const double* gi = G.g[I];
            const double* gj = G.g[J];
            const double dd = mu * (gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]);
            double* out = val + 9 * (int64_t)s[4 * I + J];
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) {
                    double k = TEXTBOOK ? lam * gi[a] * gj[b] + mu * gj[a] * gi[b]
                                        : lam * gj[a] * gi[b] + mu * gi[a] * gj[b];
                    if (a == b) k += dd;
                    out[3 * a + b] += V * k;
                }
        }
}

// ---- traction: per (face, vertex) contribution, then a per-node sum in face order
__global__ void k_traction_contrib(int n_faces, const int32_t* __restrict__ faces, const double* __restrict__ tr,
                                   const double* __restrict__ xyz, int n_nodes, int32_t* key, int32_t* idx,
                                   double* contrib, int* bad)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    int a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
    if (a < 0 || a >= n_nodes || b < 0 || b >= n_nodes || c < 0 || c >= n_nodes) {
        atomicExch(bad, 1);
        key[3 * f] = key[3 * f + 1] = key[3 * f + 2] = 0;
        idx[3 * f] = 3 * f;
        idx[3 * f + 1] = 3 * f + 1;
        idx[3 * f + 2] = 3 * f + 2;
        for (int q = 0; q < 9; q++) contrib[9 * f + q] = 0.0;
        return;
    }
    double u[3], w[3];
    for (int d = 0; d < 3; d++) {
        u[d] = xyz[3 * (int64_t)b + d] - xyz[3 * (int64_t)a + d];
        w[d] = xyz[3 * (int64_t)c + d] - xyz[3 * (int64_t)a + d];
    }
    double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    int nodes[3] = {a, b, c};
    for (int vtx = 0; vtx < 3; vtx++) {
        key[3 * f + vtx] = nodes[vtx];
        idx[3 * f + vtx] = 3 * f + vtx;
        for (int d = 0; d < 3; d++) contrib[3 * (3 * f + vtx) + d] = tr[3 * f + d] * area / 3.0;
    }
}

__global__ void k_traction_sum(int m, const int32_t* __restrict__ key, const int32_t* __restrict__ idx,
                               const double* __restrict__ contrib, double* F)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (i > 0 && key[i - 1] == key[i]) return;  // the first entry of each node's run adds the run
    const int node = key[i];
    double f0 = F[3 * (int64_t)node], f1 = F[3 * (int64_t)node + 1], f2 = F[3 * (int64_t)node + 2];
    for (int j = i; j < m && key[j] == node; j++) {
        const double* c = contrib + 3 * (int64_t)idx[j];
        f0 += c[0];
        f1 += c[1];
        f2 += c[2];
    }
    F[3 * (int64_t)node] = f0;
    F[3 * (int64_t)node + 1] = f1;
    F[3 * (int64_t)node + 2] = f2;
}

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int finish_assembly(System& s, DBuf<int>& bad)
{
    int h_bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaEventRecord(s.ev1, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, s.ev0, s.ev1);
    s.stats.ms_assemble = ms;
    if (h_bad) {
        set_error("a material id is outside [0, n_materials)");
        return MSFEM_ERR_ARGUMENT;
    }
    s.invalidate_values();
    return MSFEM_OK;
}

}  // namespace

int assemble_scalar(System& s, const double* sigma, int n_mat)
{
    if (s.kind != MSFEM_SCALAR) {
        set_error("assemble_scalar on an elasticity system");
        return MSFEM_ERR_STATE;
    }
    if (n_mat <= 0 || !sigma) {
        set_error("assemble_scalar: no materials");
        return MSFEM_ERR_ARGUMENT;
    }
    DBuf<double>& d_sig = s.params;
    DBuf<int>& bad = s.flag;
    MSFEM_TRY(d_sig.alloc(n_mat));
    MSFEM_TRY(bad.alloc(8));
    MSFEM_CK(cudaEventRecord(s.ev0, s.stream));
    MSFEM_CK(cudaMemcpyAsync(d_sig.p, sigma, sizeof(double) * n_mat, cudaMemcpyHostToDevice, s.stream));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), s.stream));
    const int nc = (int)s.color_off.size() - 1;
    for (int c = 0; c < nc; c++) {
        int cnt = s.color_off[c + 1] - s.color_off[c];
        k_assemble_scalar<<<grid_for(cnt, 128), 128, 0, s.stream>>>(cnt, s.color_elems.p + s.color_off[c], s.tets.p,
                                                                    s.xyz.p, s.mat.p, d_sig.p, n_mat, s.eslot.p,
                                                                    s.val.p, bad.p);
    }
    MSFEM_CK(cudaGetLastError());
    s.total_launches += nc;
    return finish_assembly(s, bad);
}

int assemble_scalar3(System& s, const double* S, const double* M, const double* f, bool on_device)
{
    if (s.kind != MSFEM_SCALAR) {
        set_error("assemble_scalar3 on an elasticity system");
        return MSFEM_ERR_STATE;
    }
    if (!S || !M || !f) {
        set_error("assemble_scalar3: coefficient arrays missing");
        return MSFEM_ERR_ARGUMENT;
    }
    const size_t ne = (size_t)s.n_tets;
    DBuf<double> coef;
    DBuf<int>& bad = s.flag;
    MSFEM_TRY(coef.alloc(3 * ne));
    MSFEM_TRY(bad.alloc(8));
    MSFEM_CK(cudaEventRecord(s.ev0, s.stream));
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    MSFEM_CK(cudaMemcpyAsync(coef.p, S, sizeof(double) * ne, kind, s.stream));
    MSFEM_CK(cudaMemcpyAsync(coef.p + ne, M, sizeof(double) * ne, kind, s.stream));
    MSFEM_CK(cudaMemcpyAsync(coef.p + 2 * ne, f, sizeof(double) * ne, kind, s.stream));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), s.stream));
    const int nc = (int)s.color_off.size() - 1;
    for (int c = 0; c < nc; c++) {
        int cnt = s.color_off[c + 1] - s.color_off[c];
        k_assemble_scalar3<<<grid_for(cnt, 128), 128, 0, s.stream>>>(cnt, s.color_elems.p + s.color_off[c], s.tets.p,
                                                                     s.xyz.p, coef.p, coef.p + ne, coef.p + 2 * ne,
                                                                     s.eslot.p, s.val.p, s.F.p);
    }
    MSFEM_CK(cudaGetLastError());
    s.total_launches += nc;
    return finish_assembly(s, bad);
}

// Domain::forMech::SetIsotropic_D (Library/Domain.h:53-78): k = E(1-nu)/((1+nu)(1-2nu)),
// off-diagonal normal coupling a*k, shear b*k  ->  lambda = a*k, mu = b*k; E <= 0 gives a
// material that contributes nothing (FEM/FEM.h:1355-1363)
void lame_params(const double* E, const double* nu, int n_mat, double* lame)
{
    for (int m = 0; m < n_mat; m++) {
        if (E[m] <= 0) {
            lame[2 * m] = 0.0;
            lame[2 * m + 1] = 0.0;
            continue;
        }
        double k = E[m] * (1. - nu[m]) / (1. + nu[m]) / (1. - 2. * nu[m]);
        double b = (1. - 2. * nu[m]) / (2. * (1. - nu[m]));
        double a = nu[m] / (1. - nu[m]);
        lame[2 * m] = a * k;
        lame[2 * m + 1] = b * k;
    }
}

int assemble_elastic(System& s, const double* E, const double* nu, int n_mat, bool textbook)
{
    if (s.kind != MSFEM_ELASTIC) {
        set_error("assemble_elastic on a scalar system");
        return MSFEM_ERR_STATE;
    }
    if (n_mat <= 0 || !E || !nu) {
        set_error("assemble_elastic: no materials");
        return MSFEM_ERR_ARGUMENT;
    }
    std::vector<double> lame(2 * (size_t)n_mat);
    lame_params(E, nu, n_mat, lame.data());
    DBuf<double>& d_lame = s.params;
    DBuf<int>& bad = s.flag;
    MSFEM_TRY(d_lame.alloc(2 * (size_t)n_mat));
    MSFEM_TRY(bad.alloc(8));
    MSFEM_CK(cudaEventRecord(s.ev0, s.stream));
    MSFEM_CK(cudaMemcpyAsync(d_lame.p, lame.data(), sizeof(double) * 2 * n_mat, cudaMemcpyHostToDevice, s.stream));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), s.stream));
    const int nc = (int)s.color_off.size() - 1;
    for (int c = 0; c < nc; c++) {
        int cnt = s.color_off[c + 1] - s.color_off[c];
        auto kern = textbook ? k_assemble_elastic<true> : k_assemble_elastic<false>;
        kern<<<grid_for(cnt, 128), 128, 0, s.stream>>>(cnt, s.color_elems.p + s.color_off[c], s.tets.p,
                                                                     s.xyz.p, s.mat.p, d_lame.p, n_mat, s.eslot.p,
                                                                     s.val.p, bad.p);
    }
    MSFEM_CK(cudaGetLastError());
    s.total_launches += nc;
    // a matrix-free operator (kuhn.cu) can stand for the values only while they hold one assembly
    if (s.elastic_form == 0) {
        s.elastic_form = textbook ? 2 : 1;
        s.lame_host = lame;
    } else {
        s.elastic_form = -1;
    }
    return finish_assembly(s, bad);
}

int add_traction(System& s, int n_faces, const int32_t* d_faces, const double* d_traction)
{
    if (s.kind != MSFEM_ELASTIC) {
        set_error("add_traction needs an elasticity system");
        return MSFEM_ERR_STATE;
    }
    if (n_faces <= 0) return MSFEM_OK;
    const int m = 3 * n_faces;
    DBuf<int32_t>&key = s.sc_i32[1], &idx = s.sc_i32[2], &key2 = s.sc_i32[3], &idx2 = s.sc_i32[4];
    DBuf<double>& contrib = s.sc_f64[1];
    DBuf<int>& bad = s.flag;
    MSFEM_TRY(key.alloc(m));
    MSFEM_TRY(idx.alloc(m));
    MSFEM_TRY(key2.alloc(m));
    MSFEM_TRY(idx2.alloc(m));
    MSFEM_TRY(contrib.alloc(3 * (size_t)m));
    MSFEM_TRY(bad.alloc(8));
    MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), s.stream));
    k_traction_contrib<<<grid_for(n_faces, 128), 128, 0, s.stream>>>(n_faces, d_faces, d_traction, s.xyz.p, s.n_nodes,
                                                                     key.p, idx.p, contrib.p, bad.p);
    MSFEM_CK(cudaGetLastError());
    size_t tmp_bytes = 0;
    DBuf<unsigned char>& tmp = s.sc_tmp;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, key2.p, idx.p, idx2.p, m, 0, 32, s.stream);
    MSFEM_TRY(tmp.alloc(tmp_bytes + 1));
    MSFEM_CK(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.p, key2.p, idx.p, idx2.p, m, 0, 32, s.stream));
    k_traction_sum<<<grid_for(m, 128), 128, 0, s.stream>>>(m, key2.p, idx2.p, contrib.p, s.F.p);
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 2;
    int h_bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    if (h_bad) {
        set_error("a traction face references a node id outside [0, %d)", s.n_nodes);
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

}  // namespace msfem
