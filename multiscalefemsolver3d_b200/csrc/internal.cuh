// Internal declarations shared by the CUDA translation units of libmsfem_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <array>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "msfem_b200.h"

namespace msfem {

void set_error(const char* fmt, ...);

// device memory through the library's caching allocator (devpool.cu)
void* dev_alloc(size_t bytes, cudaError_t* err);
void dev_free(void* p, size_t bytes);

#define MSFEM_CK(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            ::msfem::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));       \
            return MSFEM_ERR_CUDA;                                                                       \
        }                                                                                                \
    } while (0)

#define MSFEM_TRY(expr)               \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ < 0) return rc_;      \
    } while (0)

constexpr int kSlice = 32;        // rows (or block rows) per SELL slice = one warp
constexpr int kChunk = 4;         // scalar SELL: entries per lane per 128-bit load group
constexpr int kMaxCandidates = 256;  // portrait: candidates per row handled by one warp
constexpr int kReduceBlocks = 148 * 4;  // fixed grid of the vector kernels (deterministic reductions)
constexpr int kVecThreads = 256;

// device scratch that lives with a system and is allocated on first use
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    int alloc(size_t count) {
        if (count <= n && p) return 0;
        release();
        if (count == 0) return 0;
        cudaError_t e = cudaSuccess;
        p = static_cast<T*>(dev_alloc(count * sizeof(T), &e));
        if (e != cudaSuccess) {
            set_error("cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
            p = nullptr;
            return MSFEM_ERR_CUDA;
        }
        n = count;
        return 0;
    }
    void release() {
        if (p) dev_free(p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
};

// SELL-32 copy of the matrix used by the solvers (rebuilt when values change).
// scalar:  entry (slice s, position k, lane l) at slice_ptr[s] + (k/4)*128 + 4*l + k%4
// block3:  block (s, k, l) column at slice_ptr[s] + 32*k + l, its 9 values at
//          9*slice_ptr[s] + (9*k + e)*32 + l   (e = 3*a + b, row a / column b of the 3x3 block)
struct Sell {
    int n_slices = 0;
    int64_t stored = 0;  // stored entries (scalar) or blocks (block3), padding included
    DBuf<int64_t> slice_ptr;
    DBuf<int32_t> col;    // absolute column (3x3 blocks, or scalar when deltas do not fit 16 bits)
    DBuf<int16_t> col16;  // scalar: column - min(row, n-1), when every delta fits in 16 bits
    DBuf<double> val64;
    DBuf<float> val32;  // Jacobi-scaled copy, D^-1/2 A D^-1/2, for the FP32 inner solves
    bool pattern_ok = false;
    bool values_ok = false;
    // FP32 product on the 16-bit column deltas: -1 not yet tuned, 0 no, 1 yes (timed once per
    // portrait: the FP32 product is gather-latency bound, so fewer bytes need not be faster)
    int fp32_col16 = -1;
    float tune_ms[2] = {0.f, 0.f};  // FP32 product time with 32-bit columns / 16-bit deltas
};

// Device-resident scalars of a Krylov solve.  Written by the last block of the
// reduction kernels, read by the following kernels: no host round trip per iteration.
struct KState {
    double rz, rz_new, rr, ff, pq, alpha, beta, omega, tol2;
    double r0v, tt, ts, rho_old;  // BiCGStab
    double mr[16];              // MINRES: Lanczos / Givens scalars
    double tol2_rel;            // MINRES: tol^2, scaled by the initial residual norm on the device
    int mr_applied;             // MINRES: iteration whose solution update has been applied after stopping
    double rr_min;              // smallest (r, r) seen in this solve
    double cg2_gd[2];           // Chronopoulos-Gear CG: (r, r) and (A r, r) of the last product
    int stall, stall_limit;     // iterations since rr_min last fell by 2 %; stop when it reaches stall_limit
    int iter, maxiter, done, breakdown, primed;
    unsigned int ticket[4];
};

struct System {
    int kind = MSFEM_SCALAR;
    int bs = 1;  // 1 scalar, 3 elasticity
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_nodes = 0, n_tets = 0, n_rows = 0;

    DBuf<double> xyz;
    DBuf<int32_t> tets;
    DBuf<int32_t> mat;

    // node -> element incidence (CSR)
    DBuf<int32_t> inc_ptr, inc_elem;
    // node-level portrait, diagonal included, rows sorted
    DBuf<int32_t> nrp, ncol;
    int64_t nnzb = 0;
    // element (e, I, J) -> node-portrait slot, e*16 + 4*I + J
    DBuf<int32_t> eslot;
    // element colouring: elements listed colour by colour
    DBuf<int32_t> color_elems;
    std::vector<int> color_off;  // host copy, size n_colors + 1

    // values: scalar val[slot]; elasticity val[9*slot + 3*a + b]
    DBuf<double> val;
    DBuf<double> F, X;

    // solver data
    Sell sell;
    DBuf<double> diag64;  // diagonal of A (FP64)
    DBuf<float> dinv32;   // 1/diag (FP32)
    DBuf<double> dinv64;  // 1/diag (FP64)
    DBuf<double> dscale;  // 1/sqrt|diag|: the FP32 SELL values hold D^-1/2 A D^-1/2
    DBuf<double> work64;  // Krylov vectors (FP64)
    DBuf<float> work32;   // Krylov vectors (FP32)
    DBuf<double> partial; // reduction partials
    DBuf<KState> kstate;
    KState* h_kstate = nullptr;  // pinned mirror for polling
    KState* h_ahead = nullptr;   // two pinned snapshots taken after queued iteration chunks
    cudaEvent_t ev_chunk[2] = {nullptr, nullptr};
    DBuf<double> gm;      // GMRES: Hessenberg / rotations / y on the device
    DBuf<double> mr64;    // MINRES vectors (FP64)
    DBuf<float> mr32;     // MINRES vectors (FP32)

    // reusable scratch: once grown, the per-step calls (assembly, Dirichlet,
    // solve) allocate and free nothing, so they neither block nor serialise
    DBuf<int> flag;        // device flags (8 ints)
    DBuf<double> params;   // material parameters
    DBuf<int32_t> sc_i32[6];
    DBuf<double> sc_f64[2];
    DBuf<unsigned char> sc_tmp;

    // captured iteration graphs, keyed by solver variant and vector addresses;
    // index = log2(chunk / 4)
    std::map<std::string, std::array<cudaGraphExec_t, 8>> graphs;

    // the reference's SSOR (ssor.cu): node rows grouped by the level of the backward (upper) and
    // forward (lower) triangular sweeps -- rows of one level depend only on earlier levels
    double ssor_omega = 0.75;        // PrecondorSSOR(0.75, ...) in both FEM drivers
    DBuf<int32_t> ssor_rows;         // [backward levels | forward levels], node ids
    std::vector<int> ssor_off_b, ssor_off_f;  // host level offsets into ssor_rows
    int64_t ssor_nnzb = -1;          // portrait the levels were built for
    DBuf<double> loop_best;          // the drivers' restart loop: best solution so far
    bool reference_order = false;    // MSFEM_PCG_SSOR in the reference's operation order (ssor.cu)

    // structured Kuhn grid (kuhn.cu): hexahedra per axis and spacing, set by msfem_set_kuhn_grid
    // once the mesh is checked to be that grid; per hexahedron the material codes of its six
    // tetrahedra in bytes 0..5 of 8
    int kuhn_n[3] = {0, 0, 0};
    double kuhn_h[3] = {0.0, 0.0, 0.0};
    DBuf<uint8_t> kuhn_mat;
    // what the values hold since the last clear: 0 nothing, 1 the reference's elasticity assembly,
    // 2 the textbook orientation, -1 anything else (two assemblies, imported values); the lambda,
    // mu table of that assembly; per node the Dirichlet bits (bit a: row 3n+a is a Dirichlet row,
    // bit 3+a: its column was eliminated)
    int elastic_form = 0;
    std::vector<double> lame_host;
    DBuf<uint32_t> dmask;
    uint64_t values_version = 0;  // bumped whenever the values change

    bool zero_diag = false;
    bool force_col32 = false;  // keep 32-bit SELL columns even when 16-bit deltas fit
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    msfem_stats stats{};
    int launches = 0;          // kernels of the current solve
    int64_t total_launches = 0;  // kernels of this library launched on the handle

    void invalidate_values()
    {
        sell.values_ok = false;
        values_version++;
    }
};

// ---- mesh / portrait (portrait.cu)
int build_topology(System& s);
// a scalar system (no mesh) owning a device CSR with the diagonal in every row, F = X = 0; the
// buffers are moved into it (capi.cu)
int system_adopt_csr(int n, DBuf<int32_t>& row_ptr, DBuf<int32_t>& col, DBuf<double>& val, int64_t nnz,
                     msfem_system_t* out);
// ---- assembly (assemble.cu)
int assemble_scalar(System& s, const double* sigma, int n_mat);
int assemble_scalar3(System& s, const double* S, const double* M, const double* f, bool on_device);
int assemble_elastic(System& s, const double* E, const double* nu, int n_mat, bool textbook = false);
// lambda, mu per material from E, nu (host): lame[2m], lame[2m+1]
void lame_params(const double* E, const double* nu, int n_mat, double* lame);
int add_traction(System& s, int n_faces, const int32_t* d_faces, const double* d_traction);
// ---- boundary conditions (bc.cu)
int apply_dirichlet(System& s, int n, const int32_t* d_dofs, const double* d_values, int mode);
// ---- SpMV and SELL (spmv.cu)
int prepare_sell(System& s);
int spmv64(System& s, const double* x, double* y);
int spmv32(System& s, const float* x, float* y);
int residual64(System& s, const double* x, const double* f, double* r, double* rr_out);
// allocates the solver state (KState) zeroed on first use
int ensure_kstate(System& s);
// ---- Krylov (krylov.cu)
int solve(System& s, int method, int precision, int restart_m, int maxiter, double tol, double* relres, int* iters);
int ensure_state(System& s);
int read_state(System& s);
// ---- the MsFEM macro solve on device data (macro.cu)
int macro_solve_device(int n_vertices, int n_cells, const int32_t* cell_vertex, const double* dK, const double* dF,
                       int n_fixed, const int32_t* fixed_vertices, const double* fixed_values, int precision, double tol,
                       int maxiter, double* dU, int32_t* iterations, double* rel_residual, cudaStream_t st);
// ---- the reference's SSOR preconditioner and its PCG (ssor.cu)
int ssor_apply(System& s, const double* r, double* z, double* zb, const KState* S);
int solve_pcg_ssor(System& s, int maxiter, double tol, int* iters);
int driver_loop(System& s, int loop, int method, int precision, double min_residual, double* best_residual,
                int* n_solves, int* iterations);
// ||F - A X|| / ||F|| summed serially in index order, with A X in the reference's row order
int true_residual_reference(System& s, double* relres);
// ---- MINRES (minres.cu): on S A S from x = 0 with right-hand side S r (FP64: x += S y) or r (FP32)
template <class VT, bool SCALE>
int minres_run(System& s, VT* x, const VT* r, int maxiter, double tol, int stall_unused, int* iters);
// FP32 GMRES(m) inner solve on the Jacobi-scaled FP32 matrix (gmres.cu)
int gmres32_inner(System& s, int m, float* d, const float* b, float* V, float* w, int maxiter, double tau, int* iters);

}  // namespace msfem
