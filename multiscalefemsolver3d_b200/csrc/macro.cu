// The MsFEM macro problem (MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly, MsFEM/MsFEM.h:
// 572-1010): the macro element matrices of the cells (cells.cu, SolveLocalMatrix) assembled over
// the macro vertices (CreationPortrait + SummPartOfMatrix, :609-700), the boundary loads, the
// Dirichlet vertices, and the solve.  The macro system is one batched system of 8-node elements
// with caller-given blocks (batch.cu): a sort-built portrait, block sums in element order, and the
// persistent MINRES (the macro matrix keeps the reference's transposed blocks, so it is symmetric
// but need not be definite).
#include <memory>
#include <new>
#include <vector>

#include "batch.cuh"
#include "internal.cuh"

namespace msfem {

// The macro solve on device data: K [n_cells][8][8][3][3] and F [n_vertices][3] (or null) on the
// device, cell_vertex and the Dirichlet list on the host (checked here); U [n_vertices][3] device out.
int macro_solve_device(int n_vertices, int n_cells, const int32_t* cell_vertex, const double* dK, const double* dF,
                       int n_fixed, const int32_t* fixed_vertices, const double* fixed_values, int precision, double tol,
                       int maxiter, double* dU, int32_t* iterations, double* rel_residual, cudaStream_t st)
{
    if (n_vertices <= 0 || n_cells <= 0 || !cell_vertex || !dK || !dU || n_fixed < 0 ||
        (n_fixed > 0 && (!fixed_vertices || !fixed_values)) || !(tol > 0.0) || maxiter <= 0 ||
        (precision != MSFEM_FP64 && precision != MSFEM_FP32_IR)) {
        set_error("msfem_macro_solve: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int k = 0; k < 8 * n_cells; k++)
        if (cell_vertex[k] < 0 || cell_vertex[k] >= n_vertices) {
            set_error("msfem_macro_solve: cell %d names vertex %d (of %d)", k / 8, cell_vertex[k], n_vertices);
            return MSFEM_ERR_ARGUMENT;
        }
    std::vector<uint8_t> fixed(n_vertices, 0);
    std::vector<double> x0(3 * (size_t)n_vertices, 0.0);
    for (int i = 0; i < n_fixed; i++) {
        const int v = fixed_vertices[i];
        if (v < 0 || v >= n_vertices) {
            set_error("msfem_macro_solve: Dirichlet vertex %d out of range", v);
            return MSFEM_ERR_ARGUMENT;
        }
        fixed[v] = 1;  // a later duplicate overwrites the value, as in the reference
        for (int a = 0; a < 3; a++) x0[3 * (size_t)v + a] = fixed_values[3 * i + a];
    }
    BatchSys b;
    b.dim = 3;
    b.k1 = 8;
    b.n_sys = 1;
    b.R = 1;
    b.stream = st;
    b.h_node_off = {0, n_vertices};
    b.h_elem_off = {0, n_cells};
    b.n_nodes = n_vertices;
    b.n_elems = n_cells;
    auto up = [&](auto& dst, const auto* src, size_t n) -> int {
        MSFEM_TRY(dst.alloc(std::max<size_t>(1, n)));
        if (n) MSFEM_CK(cudaMemcpyAsync(dst.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st));
        return 0;
    };
    MSFEM_TRY(up(b.node_off, b.h_node_off.data(), 2));
    MSFEM_TRY(up(b.elem_off, b.h_elem_off.data(), 2));
    MSFEM_TRY(up(b.elems, cell_vertex, 8 * (size_t)n_cells));
    MSFEM_TRY(up(b.fixed, fixed.data(), (size_t)n_vertices));
    MSFEM_CK(cudaMemcpyAsync(dU, x0.data(), sizeof(double) * x0.size(), cudaMemcpyHostToDevice, st));
    b.rhs = const_cast<double*>(dF);
    MSFEM_TRY(batch_build_pattern(b, nullptr));
    MSFEM_TRY(batch_assemble_given(b, dK));
    MSFEM_TRY(batch_solve(b, dU, precision, tol, maxiter, 0));
    int32_t it = 0;
    double rel = 0.0;
    MSFEM_CK(cudaMemcpyAsync(&it, b.iters.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaMemcpyAsync(&rel, b.rel.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));  // the host vectors above are released here
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = rel;
    if (!(rel <= tol)) {
        set_error("msfem_macro_solve: stopped at relative residual %.3e", rel);
        return MSFEM_NOT_CONVERGED;
    }
    return MSFEM_OK;
}

}  // namespace msfem

extern "C" int msfem_macro_solve(int n_vertices, int n_cells, const int32_t* cell_vertex, const double* K,
                                 const double* F, int n_fixed, const int32_t* fixed_vertices,
                                 const double* fixed_values, int precision, double tol, int maxiter, double* U,
                                 int32_t* iterations, double* rel_residual)
{
    using namespace msfem;
    if (n_vertices <= 0 || n_cells <= 0 || !cell_vertex || !K || !U) {
        set_error("msfem_macro_solve: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    cudaStream_t st = nullptr;
    MSFEM_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamSynchronize(s), cudaStreamDestroy(s); }
    } guard{st};
    DBuf<double> dK, dF, dU;
    MSFEM_TRY(dK.alloc(576 * (size_t)n_cells));
    MSFEM_CK(cudaMemcpyAsync(dK.p, K, sizeof(double) * 576 * n_cells, cudaMemcpyHostToDevice, st));
    if (F) {
        MSFEM_TRY(dF.alloc(3 * (size_t)n_vertices));
        MSFEM_CK(cudaMemcpyAsync(dF.p, F, sizeof(double) * 3 * n_vertices, cudaMemcpyHostToDevice, st));
    }
    MSFEM_TRY(dU.alloc(3 * (size_t)n_vertices));
    const int rc = macro_solve_device(n_vertices, n_cells, cell_vertex, dK.p, F ? dF.p : nullptr, n_fixed,
                                      fixed_vertices, fixed_values, precision, tol, maxiter, dU.p, iterations,
                                      rel_residual, st);
    if (rc < 0) return rc;
    MSFEM_CK(cudaMemcpyAsync(U, dU.p, sizeof(double) * 3 * n_vertices, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return rc;
}
