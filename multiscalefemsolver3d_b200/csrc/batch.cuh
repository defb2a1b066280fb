// Batches of independent 3x3-block elasticity systems: the MsFEM cell
// sub-problems (faces and volumes of every macro cell) solved together.
#pragma once

#include <vector>

#include "internal.cuh"

namespace msfem {

// n_sys systems on one node numbering: system s owns nodes [node_off[s],
// node_off[s+1]) and elements [elem_off[s], elem_off[s+1]) whose node ids lie in
// its own range.  Matrix: node-level CSR of 3x3 blocks (global column ids), rows
// sorted, diagonal included, built by one stable sort of every element's
// (row, column) pairs; `contrib` keeps the sorted pairs so that each block is
// the sum of its element contributions in element order.
struct BatchSys {
    int dim = 3;  // 2: triangles, 3: tetrahedra
    int k1 = 4;   // nodes per element (at most 32)
    int n_sys = 0;
    int R = 1;    // right-hand sides per system
    int64_t n_nodes = 0, n_elems = 0, nnzb = 0, n_pairs = 0;
    int max_nodes = 0;
    cudaStream_t stream = nullptr;  // the owner's stream
    std::vector<int64_t> h_node_off, h_elem_off;

    DBuf<int64_t> node_off, elem_off;
    DBuf<int32_t> elems;     // [n_elems * k1] global node ids
    DBuf<int32_t> emat;      // [n_elems]
    DBuf<uint8_t> fixed;     // [n_nodes] 1 = Dirichlet node (all three components)
    DBuf<int64_t> row_ptr;   // [n_nodes + 1]
    DBuf<int64_t> cstart;    // [nnzb + 1] first contribution of each block
    DBuf<int32_t> col;       // [nnzb]
    DBuf<uint32_t> contrib;  // [n_pairs] element << 4 | I << 2 | J, grouped by block, element order
    DBuf<double> val64;      // [9 * nnzb] A[a][b] of each block, row-major
    DBuf<float> val32;       // [9 * nnzb] s_a A[a][b] s_b (Jacobi scaled)
    DBuf<double> dscale;     // [3 * n_nodes] 1 / sqrt(diagonal)
    DBuf<int32_t> order;     // systems, largest first (the persistent solver's queue)

    // solver scratch and per-system report
    DBuf<unsigned char> work;  // per-CTA Krylov vectors (bytes: room for FP64)
    DBuf<int> queue;
    DBuf<int32_t> iters, outers;
    DBuf<double> rel;
    const double* rhs = nullptr;  // optional source term [n_nodes][R][3] (device), used by batch_solve
    int grid = 0, threads = 0;
    int tuned_threads = 0, tuned_precision = -1;  // autotuned CTA size (0: not tuned yet)
    std::vector<float> tune_ms;                   // trial times of the candidates 128/256/384/512
    int64_t work_stride = 0;
    float last_ms = 0.f;
    DBuf<int> aflag;  // set by the assembly when an element's material id is out of range
};

// pattern: elems/emat/node_off/elem_off/fixed filled; builds row_ptr, col, cstart, contrib
int batch_build_pattern(BatchSys& b, const double* d_xyz);
// values from the current materials (lame: [n_mat][2] lambda, mu on the device)
int batch_assemble(BatchSys& b, const double* d_xyz, const double* d_lame, int n_mat);
// the same launches without waiting for them (no host synchronisation, no allocation once the
// buffers exist): capturable into a CUDA graph; a bad material id is left in b.aflag
int batch_assemble_enqueue(BatchSys& b, const double* d_xyz, const double* d_lame, int n_mat);
// values from caller-given element blocks [n_elems][k1][k1][9] (device), each block the sum of
// its element contributions in element order; scaled: also the Jacobi scale and the FP32 copy
// the batched solver reads
int batch_assemble_given(BatchSys& b, const double* d_eblocks, bool scaled = true);
// solves every system; x: [n_nodes][R][3] FP64, fixed entries hold the Dirichlet data on
// entry, free entries are overwritten.  precision: MSFEM_FP64 or MSFEM_FP32_IR.  threads <= 0:
// the CTA size is autotuned on the first call (cached per batch and precision).
int batch_solve(BatchSys& b, double* d_x, int precision, double tol, int maxiter, int threads);
// the CTA size batch_solve would use with `threads` (0 when the autotuner has not run yet)
int batch_threads(const BatchSys& b, int precision, int threads);

}  // namespace msfem
