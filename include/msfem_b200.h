/*
 * msfem_b200.h -- C ABI of the B200 (sm_100a) implementation of the
 * MultiscaleFEMSolver3D hot path: P1 tetrahedral assembly into the CSSD_Matrix
 * layout and the Krylov solve on that matrix.
 *
 * The reference has no FFI; its "boundary" is a sequence of C++ member calls
 * made by the FEM drivers (FEM/FEM.h).  Each entry point below replaces one
 * step of that sequence; the comment on each names the reference code it
 * stands for (paths relative to the reference project).
 *
 * Conventions
 *  - Every function returns an int status: MSFEM_OK (0), a negative error code,
 *    or MSFEM_NOT_CONVERGED (1) from a solver that stopped at maxiter.  Nothing
 *    throws; msfem_last_error() returns the message of the calling thread's
 *    last failure.  (The reference prints and continues, CSSD_Matrix.h:359-362.)
 *  - Arrays are caller owned.  `on_device` = 0: host pointers (pinned or not),
 *    copied in or out on the handle's stream;  = 1: CUDA device pointers on the
 *    handle's device, used in place (no host round trip).
 *  - DOF numbering is the reference's: scalar DOF = mesh node id
 *    (FEM_Grid.h:509-574); elasticity DOF = 3*node + component
 *    (Library/Math.h:1963-2054).
 *  - Matrices export as CSR with the diagonal included and every row sorted
 *    ascending: the reference CSSD row [A_down | Diag | A_up] laid end to end
 *    (Library/CSSD_Matrix.h:11-15).  Structural zeros are kept.
 *  - One handle = one system on one device with its own CUDA stream.  Calls on
 *    different handles may run concurrently from different host threads; calls
 *    on the same handle must not.
 */
#ifndef MSFEM_B200_H
#define MSFEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSFEM_OK 0
#define MSFEM_NOT_CONVERGED 1
#define MSFEM_ERR_ARGUMENT (-1)
#define MSFEM_ERR_CUDA (-2)
#define MSFEM_ERR_STATE (-3)
#define MSFEM_ERR_LIMIT (-4)
#define MSFEM_ERR_NUMERIC (-5)

enum msfem_kind { MSFEM_SCALAR = 0, MSFEM_ELASTIC = 1 };

enum msfem_method {
    MSFEM_CG = 0,          /* plain CG, CSSD_Matrix::MSG (CSSD_Matrix.h:1496-1576)                 */
    MSFEM_PCG_JACOBI = 1,  /* the PCG loop of MSG_PreconditioningSSOR (:1302-1398), M = diag(A)    */
    MSFEM_BICGSTAB = 2,    /* Jacobi-preconditioned BiCGStab (the role of BiCG_Stab/BCG_Stab2)      */
    MSFEM_GMRES = 3,       /* restarted GMRES(m), Jacobi-preconditioned (CSSD_Matrix::GMRES role)  */
    MSFEM_MINRES = 4,      /* MINRES on the Jacobi-scaled matrix: for symmetric indefinite systems,
                              which the reference's elasticity assembly produces (its transposed
                              element blocks leave the global matrix symmetric but indefinite) */
    MSFEM_PCG_SSOR = 5     /* MSG_PreconditioningSSOR (:1302-1398) with the reference's own SSOR
                              (PrecondorSSOR + SolvePrecondorSSOR_SLAE, :458-547): the off-diagonal
                              signs flipped, M = (D - wL) D^-1 (D - wU) / (w (2 - w)), w from
                              msfem_set_ssor_omega (0.75, as both FEM drivers use).  The sweeps are
                              level scheduled, one launch per level, and give the reference's bits
                              for each application.  FP64 only.                                   */
};

enum msfem_precision {
    MSFEM_FP64 = 0,    /* everything in FP64                                                        */
    MSFEM_FP64_REFERENCE = 2,  /* MSFEM_PCG_SSOR only: FP64 in the reference's operation order -- A x
                          summed per row as MultiplicationMatrixVector does (CSSD_Matrix.h:395-423:
                          the upper entries in ascending column order, then the lower ones, then
                          the diagonal), inner products summed serially in index order
                          (math::MakeInnerProduct, Library/Math.h:1633-1654), the updates of
                          MSG_PreconditioningSSOR unfused, its loop test sqrt((r,r)/(F,F)) > E as
                          written, the returned residual summed as it sums it (:1384-1397) -- so
                          the iterates, iteration counts and residuals are the reference's bits
                          (for CSSD lists in ascending column order, as CreationPortrait builds
                          them).  The serial sums make it a parity mode: about 0.1 ms per inner
                          product of 30,000 entries.                                             */
    MSFEM_FP32_IR = 1  /* FP32 matrix + FP32 Krylov inner solves inside FP64 iterative refinement:
                          r = F - A x and x accumulate in FP64.  The inner solver is CG on the
                          Jacobi-scaled matrix for MSFEM_PCG_JACOBI, MINRES on it for
                          MSFEM_MINRES, GMRES(restart_m) on it for MSFEM_GMRES; BiCGStab is
                          FP64 only                                                               */
};

enum msfem_dirichlet_mode {
    MSFEM_ROW_ONLY = 0,       /* row := e_d, F = X = value (FEM/FEM.h:297-324, 3-coefficient driver) */
    MSFEM_ROW_AND_COLUMN = 1  /* rows as above, then the column sweep F -= A(:,d) F_d, A(:,d) = 0 with
                                 the reference's forward-only walk over the boundary list
                                 (FEM/FEM.h:506-619 scalar, :1676-1813 elasticity)                   */
};

typedef struct msfem_system* msfem_system_t;

typedef struct {
    int iterations;          /* Krylov iterations of the last solve (inner iterations for FP32_IR) */
    int outer_iterations;    /* refinement steps (FP32_IR), restarts (GMRES), else 0               */
    double rel_residual;     /* ||F - A X|| / ||F|| recomputed in FP64 at exit                       */
    double ms_portrait;      /* device time of the last portrait build                             */
    double ms_assemble;      /* device time of the last assembly (elements + scatter)              */
    double ms_dirichlet;     /* device time of the last Dirichlet application                       */
    double ms_solve;         /* device time of the last solve                                       */
    double ms_spmv;          /* mean device time of one SpMV of the solve's working precision       */
    int n_colors;            /* element colour classes used by the assembly                         */
    int kernel_launches;     /* kernels of this library launched by the last solve                  */
    int64_t total_launches;  /* kernels of this library launched on this handle since creation      */
} msfem_stats;

const char* msfem_last_error(void);
int msfem_version(void);

/* Grid_forScal / Grid_forMech::Initialization + CreationPortrait + CSSD_Matrix::Initialization
 * (FEM/FEM_Grid.h:575-663, :3017-3102; :665-716, :3236-3287; Library/CSSD_Matrix.h:79-99):
 * uploads the mesh (nvtr = tets[4*n_tets], nvkat = material[n_tets], xyz[3*n_nodes]),
 * builds the node-level portrait (every pair of nodes of an element couples), the
 * element -> matrix-slot map and the element colouring, and allocates the zeroed
 * matrix, F and X.  kind = MSFEM_SCALAR (n rows = n_nodes) or MSFEM_ELASTIC
 * (n rows = 3*n_nodes, 3x3 blocks).  material may be NULL (all zero). */
int msfem_system_create(int kind, int n_nodes, const double* xyz, int n_tets, const int32_t* tets,
                        const int32_t* material, int on_device, msfem_system_t* out);
int msfem_system_destroy(msfem_system_t h);

/* A scalar system from a matrix the caller already holds in the reference's CSSD_Matrix<double,
 * double> layout (Library/CSSD_Matrix.h:11-17): Diag[n]; row i's lower entries A_down[i] with
 * their columns id_column_for_A_down[i] (< i) and upper entries A_up[i] with
 * id_column_for_A_up[i] (> i), flattened with row offsets down_ptr / up_ptr [n + 1]; F and X
 * (either may be NULL: zeros).  Host arrays; lists may be unsorted (sorted here), a repeated
 * column is an error.  Every solver (msfem_solve, msfem_solve_gmres, FP32 refinement, Dirichlet
 * rows, export) then runs on the GPU copy: the drop-in for CSSD_Matrix::MSG /
 * MSG_PreconditioningSSOR / BiCG_Stab / GMRES on the reference's own matrix object.  The system
 * has no mesh (assembly calls return an error). */
int msfem_system_from_cssd(int n, const double* diag, const int64_t* down_ptr, const int32_t* down_col,
                           const double* down_val, const int64_t* up_ptr, const int32_t* up_col, const double* up_val,
                           const double* F, const double* X, msfem_system_t* out);
/* Cracked conduction with Heaviside enrichment (no reference counterpart: the reference's XFEM,
 * MultiXFEM/MultiXFEM_Grid.h:1090-2980, is for elasticity): a scalar system of n_dofs unknowns
 * (the mesh nodes, then the enriched DOFs) assembled on the GPU from the mesh, the conductivity
 * of each tetrahedron, the cracks (disc centre and unit normal, [n_cracks][3] each), the crack
 * cutting each tetrahedron (-1: none) and its vertices' enriched DOFs (enr_dof [n_tets][4],
 * n_nodes..n_dofs-1 where cut) -- the cut detection and numbering of
 * multiscalefemsolver3d_b200/xfem.py.  Entries: sigma V grad(phi_i).grad(phi_j) on every
 * tetrahedron; on a cut one, std-enr sum_s V_s (H_s - H_j) K_ij and enr-enr
 * sum_s V_s (H_s - H_i)(H_s - H_j) K_ij with the exact side volumes V_s of the crack plane.
 * F = X = 0; Dirichlet rows and solvers as for any system.  Host arrays. */
int msfem_xfem_system(int n_nodes, const double* xyz, int n_tets, const int32_t* tets, const double* sigma,
                      int n_cracks, const double* centre, const double* normal, const int32_t* crack_of_tet,
                      const int32_t* enr_dof, int n_dofs, msfem_system_t* out);
/* n_rows, scalar nnz of the CSR export (diagonal included), element colour count */
int msfem_system_info(msfem_system_t h, int* n_rows, int64_t* nnz, int* n_colors);
int msfem_get_stats(msfem_system_t h, msfem_stats* out);
/* the handle's CUDA stream (cudaStream_t) */
void* msfem_get_stream(msfem_system_t h);

/* Zeroes the matrix values, F and X, keeping the portrait (CSSD_Matrix::ClearVariables, :172). */
int msfem_clear(msfem_system_t h);

/* Scalar stiffness assembly: element loop + SummPartOfMatrix (FEM/FEM.h:474-482,
 * FEM_Grid.h:103-152 with the 1-point rule, CSSD_Matrix.h:307-363).
 * sigma[material] is the element coefficient. */
int msfem_assemble_scalar(msfem_system_t h, const double* sigma, int n_materials);
/* The three-coefficient scalar element (FiniteElement_forScal::SolveLocalMatrix with stiffness,
 * mass and source coefficients, FEM/FEM_Grid.h:25-102, as FEM_forBaseEliptic at FEM/FEM.h:206-397
 * calls it): per tetrahedron e, with the one-point rule, A += V (S[e] grad(phi_I).grad(phi_J) +
 * M[e] / 16) and F += V f[e] / 4; S, M, f: the coefficients at each element's centroid, n_tets
 * each (host or device).  The driver then sets Dirichlet rows only (MSFEM_ROW_ONLY) and runs
 * BiCG_Stab. */
int msfem_assemble_scalar3(msfem_system_t h, const double* S, const double* M, const double* f, int on_device);

/* Linear elasticity assembly (FEM/FEM.h:1349-1384, FEM_Grid.h:2125-2192): block
 * A[I][J] = V * B_J^T D(E, nu) B_I for J >= I and A[J][I] = A[I][J]^T (the
 * reference's orientation), D from Domain::forMech::SetIsotropic_D
 * (Library/Domain.h:53-78).  Materials with E <= 0 contribute nothing. */
int msfem_assemble_elastic(msfem_system_t h, const double* E, const double* nu, int n_materials);

/* No counterpart in the reference: the same assembly with every block transposed, i.e. the
 * textbook orientation A[I][J] = V * B_I^T D B_J, which is symmetric positive semi-definite
 * (the reference's orientation is symmetric but indefinite).  Used as the operator of the
 * smoothing and coarse levels of msfem_coarse_set_smoother. */
int msfem_assemble_elastic_textbook(msfem_system_t h, const double* E, const double* nu, int n_materials);

/* Traction load (FEM/FEM.h:1338-1343, BoundaryFace_forMech::SolveLocalBoundaryVector
 * FEM_Grid.h:2622-2661): F[3*v+c] += traction[3*f+c] * area_f / 3 for the three
 * nodes v of face f.  ELASTIC only. */
int msfem_add_traction(msfem_system_t h, int n_faces, const int32_t* face_nodes, const double* traction,
                       int on_device);

/* Adds a caller vector to F (CSSD_Matrix::SummPartOfVector, :364-379, for a whole vector). */
int msfem_add_rhs(msfem_system_t h, const double* f, int on_device);

/* Dirichlet conditions on `n` DOFs in the caller's boundary-list order
 * (the order of the reference's boundary_vertexes), see enum msfem_dirichlet_mode. */
int msfem_apply_dirichlet(msfem_system_t h, int n, const int32_t* dofs, const double* values, int mode,
                          int on_device);

int msfem_set_x(msfem_system_t h, const double* x, int on_device);
int msfem_get_x(msfem_system_t h, double* x, int on_device);
int msfem_get_f(msfem_system_t h, double* f, int on_device);
/* X := F (FEM/FEM.h:635, the scalar driver's initial guess) */
int msfem_copy_f_to_x(msfem_system_t h);

/* Solves A X = F from the current X (CSSD_Matrix::MSG / MSG_PreconditioningSSOR /
 * BiCG_Stab / GMRES, CSSD_Matrix.h:1302-1989).  Stops when ||r||/||F|| <= tol
 * (the reference's test) or after maxiter iterations (MSFEM_NOT_CONVERGED).
 * restart_m: GMRES restart depth (ignored otherwise).  rel_residual / iterations
 * may be NULL. */
int msfem_solve(msfem_system_t h, int method, int precision, int restart_m, int maxiter, double tol,
                double* rel_residual, int* iterations);

/* The SSOR relaxation factor w of MSFEM_PCG_SSOR (PrecondorSSOR(w, ...), CSSD_Matrix.h:458);
 * 0 < w < 2, default 0.75. */
int msfem_set_ssor_omega(msfem_system_t h, double omega);
/* z = M^-1 r with the reference's SSOR (SolvePrecondorSSOR_SLAE, CSSD_Matrix.h:514-547) on the
 * current matrix: the same bits as the reference's sweeps.  r, z: n_rows doubles. */
int msfem_ssor_apply(msfem_system_t h, const double* r, double* z, int on_device);

/* The FEM drivers' solve as the reference runs it: a restart loop around `method` with the needed
 * residual tightened tenfold after each success, a best-solution copy, and X rolled back to the
 * best solution at the end (loop 0: FEM_forBaseEliptic, FEM/FEM.h:627-695 -- X = F first, targets
 * 1e-1, 1e-2, ..., up to 6 tries per target, stop when a success does not improve on the best by
 * 1e-10; loop 1: FEM_forElasticDeformation, FEM/FEM.h:1853-1939 -- targets 1e-2, 1e-3, ..., up to
 * 5 tries per target).  Each solve runs from the current X with at most n_rows - 1 iterations, as
 * MSG_PreconditioningSSOR(GetMatrixSize(), ...) does.  The loop ends at min_residual; as in the
 * reference, a solve that reaches it is not copied into the best solution, so X is the best
 * solution of the earlier solves.  best_residual: the loop's best true relative residual;
 * n_solves / iterations: solves run and their iterations in total (any may be NULL). */
int msfem_solve_driver_loop(msfem_system_t h, int loop, int method, int precision, double min_residual,
                            double* best_residual, int* n_solves, int* iterations);

/* y = A x in FP64 (CSSD_Matrix::MultiplicationMatrixVector, :395-423) */
int msfem_spmv(msfem_system_t h, const double* x, double* y, int on_device);

/* y = (D^-1/2 A D^-1/2) x in FP32, D = diag(A): the Jacobi-scaled operator that the FP32
 * inner solves of MSFEM_FP32_IR apply (no counterpart in the reference; exposed so that the
 * FP32 path can be checked on its own).  x, y: n_rows floats. */
int msfem_spmv_scaled32(msfem_system_t h, const float* x, float* y, int on_device);
/* Structured Kuhn grid (no reference counterpart; the mesh of the reference's generated cubes):
 * checks on the device that the system's mesh is nx x ny x nz hexahedra, each cut into the six
 * Kuhn tetrahedra of its 0-7 diagonal -- tetrahedra 6c .. 6c+5 of hexahedron c = i + nx (j + ny k)
 * with corners {0,1,3,7} {0,1,5,7} {0,2,3,7} {0,2,6,7} {0,4,5,7} {0,4,6,7} in that vertex order,
 * corner b at node (i + (b&1)) + (nx+1) ((j + (b>>1&1)) + (ny+1) (k + (b>>2&1))), nodes on a
 * regular grid -- with material ids in [0, 64).  MSFEM_ERR_ARGUMENT (first offending tetrahedron or
 * node in the message) otherwise.  Elasticity systems only. */
int msfem_set_kuhn_grid(msfem_system_t h, int nx, int ny, int nz);
/* The library's device buffers come from a caching allocator: a released buffer's memory stays
 * with the library (per device, by size class, at most 48 GiB) for the next buffer of that class,
 * so handles built and destroyed step after step do not pay cudaMalloc / cudaFree each time; a
 * release synchronises the device first, as cudaFree does.  This returns every cached block to the
 * driver (no reference counterpart). */
void msfem_release_cached_memory(void);
/* y = A x formed matrix-free on the Kuhn grid (FP64): A is the system's values -- one
 * msfem_assemble_elastic or msfem_assemble_elastic_textbook since the last msfem_clear, plus its
 * Dirichlet rows -- applied from the tetrahedra's materials; checked against the assembled product
 * on a probe vector first (MSFEM_ERR_STATE if the relative distance exceeds 1e-12). */
int msfem_kuhn_spmv(msfem_system_t h, const double* x, double* y, int on_device);
/* y = S A S x in FP32 formed matrix-free on the Kuhn grid (S = diag(1/sqrt|A_ii|), the scaling of
 * msfem_spmv_scaled32) by the kernel the two-level cycle's smoother runs: the input is first scaled
 * to s x with the eliminated columns zero, then staged as it is.  At set-up the product is checked
 * against the assembled FP32 product (relative 1e-5) and against the staged-scale matrix-free
 * kernel bit for bit (MSFEM_ERR_STATE otherwise).  No reference counterpart. */
int msfem_kuhn_spmv_scaled32(msfem_system_t h, const float* x, float* y, int on_device);

/* CSR export of the assembled matrix (sizes from msfem_system_info), host or device buffers. */
int msfem_export_csr(msfem_system_t h, int32_t* row_ptr, int32_t* col, double* val, int on_device);

/* Measurement helper (no counterpart in the reference): times `reps` back-to-back
 * FP64 (precision MSFEM_FP64) or FP32 (MSFEM_FP32_IR) SpMV launches with CUDA
 * events on the handle's stream after 3 warm-up launches, and reports the mean
 * device time per product and the algorithmic bytes of one product
 * (values + column indices in the stored width + row structure + x + y, each
 * counted once). */
int msfem_bench_spmv(msfem_system_t h, int precision, int reps, double* ms_per_product, int64_t* bytes_per_product);

/* No counterpart in the reference.  r = f - A x and *rr = ||r||^2 for a caller-owned
 * CSR matrix (device pointers: row_ptr[n_rows+1], col, val, x, f, r, and rr a single
 * device double), launched on `stream` (a cudaStream_t, NULL = legacy default stream)
 * and NOT synchronised.  This entry point allocates no device memory: it is meant for
 * callers that cannot let a library call cudaMalloc (applications that give the whole
 * device heap to their own arena, or loops that cannot absorb cudaFree's device-wide
 * synchronisation).  Its reduction scratch is a fixed 128 KiB device array inside the
 * library, held by every GPU that loads it until the process exits, which limits
 * n_rows to 4,194,304 (larger sizes return MSFEM_ERR_LIMIT).  All calls share that
 * array: calls whose kernels overlap on one GPU race and must be serialised.  The
 * first call on each device looks the array's address up (cudaGetSymbolAddress) with
 * that device current; make it before any stream capture on the calling thread.  Later
 * calls check the kept address (cudaPointerGetAttributes) and look it up again when it no
 * longer names device memory of the current device -- after cudaDeviceReset, or with a
 * different context current -- so such a call is a first call too. */
int msfem_residual_noalloc(int n_rows, const int32_t* row_ptr, const int32_t* col, const double* val,
                           const double* x, const double* f, double* r, double* rr, void* stream);

/* One-call drivers: the reference driver sequence on the GPU, host buffers in and out.
 * With method MSFEM_PCG_SSOR the solve is the reference's own: its SSOR(0.75)-PCG inside its restart
 * loop (msfem_solve_driver_loop; maxiter is then unused); any other method runs one solve to
 * min_residual.
 *
 * FEM::FEM_forBaseEliptic, stiffness-only overload (FEM/FEM.h:398-717):
 * create -> assemble (sigma per material) -> Dirichlet rows + column sweep ->
 * X = F -> solve to min_residual.  solution: n_nodes doubles. */
int msfem_fem_scalar_driver(int n_nodes, const double* xyz, int n_tets, const int32_t* tets,
                            const int32_t* material, int n_materials, const double* sigma,
                            int n_bc, const int32_t* bc_nodes, const double* bc_values,
                            int method, int precision, double min_residual, int maxiter,
                            double* solution, msfem_stats* stats);

/* FEM::FEM_forElasticDeformation (FEM/FEM.h:1286-1961): create -> traction ->
 * assemble -> Dirichlet (mask bit c = component c fixed, values[3*i+c]) with the
 * column sweep -> solve to min_residual from X = Dirichlet values, 0 elsewhere.
 * solution: 3*n_nodes doubles, node-major. */
int msfem_fem_elastic_driver(int n_nodes, const double* xyz, int n_tets, const int32_t* tets,
                             const int32_t* material, int n_materials, const double* E, const double* nu,
                             int n_bc, const int32_t* bc_nodes, const int32_t* bc_mask, const double* bc_values,
                             int n_faces, const int32_t* face_nodes, const double* face_traction,
                             int method, int precision, double min_residual, int maxiter,
                             double* solution, msfem_stats* stats);


/* ---------------------------------------------------------------------------------------
 * Batched MsFEM cell problems.
 *
 * The reference builds the MsFEM Order1 basis one macro cell at a time inside an OpenMP
 * loop over cells (Grid_forMech_Poly_Order1::CreateFunctionalSpaces,
 * MsFEM/MsFEM_Grid.h:4795-5759): per cell 24 edge problems (FEM::FEM_1D_forElasticDeformation,
 * FEM/FEM.h:3796), 24 face problems (FEM_2D_forElasticDeformation, :4367) and 8 volume
 * problems (FEM_3D_forElasticDeformation, :2970), each assembled and solved by its own
 * SSOR-PCG restart loop.  Here every problem of every cell is solved in one persistent
 * launch per problem kind.
 * ------------------------------------------------------------------------------------- */

/* Post-processing of an elasticity system's current solution X, per tetrahedron at its centroid
 * (FEM/FEM_Grid.h:3289-3365 and the fields FEM/FEM_Main.cpp:1018-1040 prints).  out:
 * [n_tets][23] doubles = U (3), grad U (9, row a = grad u_a), sigma (xx yy zz yz xz xy) of the
 * element's own material (Domain::forMech::solve_SIGMA), von Mises as GetVonMisesStress computes
 * it, then the driver's printed sigma_xx, sigma_yy, sigma_zz and von Mises (domain 0's E and nu
 * for every element, as the reference driver does).  Host or device output. */
int msfem_postprocess_elastic(msfem_system_t h, int n_materials, const double* E, const double* nu, double* out,
                              int on_device);

typedef struct msfem_batch* msfem_batch_t;

/* n_systems independent FEM_2D (dim 2: triangles) or FEM_3D (dim 3: tetrahedra)
 * elasticity problems with zero source, as the cell drivers pose them.  System s owns the
 * nodes [node_off[s], node_off[s+1]) of xyz and the elements [elem_off[s], elem_off[s+1])
 * of elems (dim+1 node ids each, GLOBAL ids inside the system's own node range).
 * fixed[node] = 1 marks a Dirichlet node (all three components).  n_rhs right-hand sides
 * per system (1, 4 or 8).  The portrait is built and the matrices assembled here. */
int msfem_batch_create(int dim, int n_systems, const int64_t* node_off, const double* xyz, const int64_t* elem_off,
                       const int32_t* elems, const int32_t* material, int n_materials, const double* E,
                       const double* nu, const uint8_t* fixed, int n_rhs, int on_device, msfem_batch_t* out);

/* Solves every system.  x: [n_nodes][n_rhs][3] doubles; on entry the Dirichlet values at
 * fixed nodes, on return the solution (free entries overwritten).  precision MSFEM_FP64 or
 * MSFEM_FP32_IR (FP32 inner MINRES on the Jacobi-scaled free block, FP64 residual and
 * accumulation).  Stops when ||F_I - A_II x_I|| <= tol ||F_I|| for every right-hand side, with
 * F_I = -A_IB g the right-hand side of the free rows after the Dirichlet elimination (the
 * reference's cell drivers also count the Dirichlet values g in ||F||, a measure up to ~1/h
 * looser, and compensate with MIN_RESIDUAL = 5e-15).  maxiter bounds each inner solve,
 * threads = CTA size (multiple of 32, <= 512; 0 = autotune: the first call times 128, 256, 384
 * and 512 threads on the largest systems and keeps the fastest).
 * Returns MSFEM_NOT_CONVERGED when some system missed tol. */
int msfem_batch_solve(msfem_batch_t b, double* x, int precision, double tol, int maxiter, int threads, int on_device);

/* Per-system report of the last solve (host arrays of n_systems, any may be NULL) and its
 * device time in ms. */
int msfem_batch_report(msfem_batch_t b, int32_t* inner_iterations, int32_t* outer_iterations, double* rel_residual,
                       double* ms);
void msfem_batch_destroy(msfem_batch_t b);

typedef struct msfem_cells* msfem_cells_t;

/* n_cells MsFEM Order1 macro cells.  Cell c is the axis-aligned box
 * box[6c..6c+5] = (x0, x1, y0, y1, z0, z1) carrying its own fine tetrahedral mesh: nodes
 * [node_off[c], node_off[c+1]) of xyz and tets [tet_off[c], tet_off[c+1]) whose four node ids
 * are CELL-LOCAL (0-based within the cell, as in the reference's per-cell NVTR files,
 * MsFEM_Grid.h:4837).  Vertex v of a cell is its box corner (x_{v&1}, y_{(v>>1)&1},
 * z_{(v>>2)&1}); a fine node must sit on each corner.  Builds the cell topology (faces,
 * edges, face triangles) and the portraits of all face and volume problems. */
int msfem_cells_create(int n_cells, const int64_t* node_off, const double* xyz, const int64_t* tet_off,
                       const int32_t* tets, const int32_t* material, const double* box, int n_materials,
                       const double* E, const double* nu, int on_device, msfem_cells_t* out);

/* The Order1 basis of every cell: edge profiles (the exact FEM_1D solutions), the 4 face
 * problems of each of the 6 faces and the 8 volume problems, in that order, on the GPU.
 * precision / tol / maxiter / threads as for msfem_batch_solve. */
int msfem_cells_build_bases(msfem_cells_t c, int precision, double tol, int maxiter, int threads);

/* Materials of the Order1 face and edge problems: mode 1 (the default) -- material 0 everywhere,
 * which is what the reference computes: its face meshes come from Salome files whose
 * ReadFromSalomeDat leaves every material id 0 (Library/Math.h:91-147; MsFEM_Grid.h:4848, the edge
 * segments copy the face ids, :4905); mode 0 -- each face triangle and edge segment takes the
 * material of the tetrahedra it bounds.  Takes effect at the next msfem_cells_build_bases. */
int msfem_cells_set_face_material(msfem_cells_t c, int mode);

/* bases: [n_nodes][8][3] doubles, node-major (the reference's self_basis_functions[v][node]
 * as Points, MsFEM_Grid.h:5510-5530, transposed to node-major). */
int msfem_cells_get_bases(msfem_cells_t c, double* bases, int on_device);

/* The MsFEM Order2 basis of every cell (Grid_forMech::CreateFunctionalSpaces,
 * MsFEM/MsFEM_Grid.h:1001-3080): 27 per cell, in the reference's order (:3045-3054) -- the 8
 * vertices, the 12 edges in ascending global edge id (the edge's (lower, higher) global vertex
 * pair), the 6 faces x0 x1 y0 y1 z0 z1, the cell bubble.  cell_vertex: [n_cells][8] global
 * macro vertex ids of each cell's corners (host or device).  The edge problems are exact (every
 * edge segment is material 0 in the reference), the face problems (4 linear + 4 edge bubbles per
 * face, material 0, no load as FEM_2D leaves them) and the 27 volume problems with their bubble
 * loads run on the GPU; precision / tol / maxiter / threads as for msfem_batch_solve. */
int msfem_cells_build_order2(msfem_cells_t c, const int32_t* cell_vertex, int precision, double tol, int maxiter,
                             int threads);

/* Host only (no device work): the Order2 edge-bubble order of every cell -- order[c][k] = the
 * cell-local edge (0..11: edge e runs along axis e / 4, at side (e >> 1) & 1 of the lower other
 * axis and e & 1 of the higher one) of edge basis k, i.e. the cell's edges sorted by their
 * (lower, higher) global vertex pair as the reference numbers its macro edges
 * (MsFEM_Grid.h:597-760). */
int msfem_order2_edge_order(int n_cells, const int32_t* cell_vertex, int32_t* order);


/* bases: [n_nodes][27][3] doubles, node-major (self_basis_functions[i][node] of
 * MsFEM_Grid.h:2926-2937 transposed). */
int msfem_cells_get_order2_bases(msfem_cells_t c, double* bases, int on_device);

/* The Order2 macro element matrices (FiniteElement_forMech_Poly::SolveLocalMatrix,
 * MsFEM/MsFEM_Grid.h:34-171) from the cells' Order2 bases, each basis taken as its z component in
 * all three components as the reference's macro basis functions return it (:2978-2979, :3038-3040);
 * quadrature, micro-element lookup and D as msfem_cells_macro_matrices.
 * K: [n_cells][27][27][3][3] doubles. */
int msfem_cells_order2_macro_matrices(msfem_cells_t c, double* K, int on_device);

/* The MsFEM Order2 macro system on the device (MsFEM::MsFEM_forElasticDeformation_OrderBF2_forPoly,
 * MsFEM/MsFEM.h:53-131: Grid_forMech::CreationPortrait + CSSD_Matrix::SummPartOfMatrix, then
 * math::MakeCopyMatrix_A_into_B): the cells' element matrices (msfem_cells_order2_macro_matrices)
 * summed by the cells' DOF lists cell_dofs [n_cells][27] (host; the reference's numbering:
 * vertices, NV + edge, NV + NE + face, NV + NE + NF + cell; every DOF in some cell) into the
 * scalar system of DOF 3 d + c, whole 3x3 blocks of the DOF portrait, diagonal in place, each
 * block summed in (cell, I, J) order.  *out: a new scalar system (no mesh) with F = X = 0; the
 * caller destroys it.  Replaces the host assembly loop of MsFEM.h:61-131. */
int msfem_cells_order2_macro_system(msfem_cells_t c, int n_dofs, const int32_t* cell_dofs, msfem_system_t* out);

/* The Order2 Dirichlet values on the device (Grid_forMech::CreateBoundaryConditions,
 * MsFEM/MsFEM_Grid.h:3303-3470): per group, the L2 projection of its constant value over its faces
 * onto its DOFs.  Host arrays:
 *   vertex_xyz [n_vertices][3]: the macro vertices;
 *   faces [n_faces][10]: per group face (grouped by group, in the group's face order): its cell
 *     and its 9 DOF ids -- its 4 cycle vertices (a vertex's DOF id is its vertex id; the
 *     quadrature runs over this cycle), the edges between cycle nodes k and k+1, the face;
 *   group_dof_off [n_groups + 1], group_dofs: each group's DOF list, ascending;
 *   group_face_off [n_groups + 1]: each group's faces in `faces`;
 *   group_values [n_groups][3]: each group's value.
 * Per face: the mass matrix and load of its 9 DOFs with the polygon rule 3 (GeometryShape.h:
 * 2625-2640 with the triangle rule of :1482-1540 as written there), the bases' z components from
 * the lowest-numbered micro tetrahedron holding each point; summed per group in face order and
 * solved by Cholesky on the rows that carry mass (rows whose diagonal is at most n eps times the
 * largest diagonal -- the face bubbles, DOFs on no group face -- hold 0).  At most 4096 DOFs
 * per group (one CTA's dense Cholesky).  values: host [group_dof_off[n_groups]][3] out, the projected value of each group
 * DOF. */
int msfem_cells_order2_dirichlet(msfem_cells_t c, int n_dofs, const int32_t* cell_dofs, int n_vertices,
                                 const double* vertex_xyz, int n_faces, const int32_t* faces, int n_groups,
                                 const int32_t* group_dof_off, const int32_t* group_dofs, const int32_t* group_face_off,
                                 const double* group_values, double* values);

/* The Order2 macro phase in one call, on the device: msfem_cells_order2_macro_system, the
 * projected values of msfem_cells_order2_dirichlet, the elimination of the rows fixed_dofs
 * [n_fixed] (scalar rows 3 d + c, in elimination order) with values projected[fixed_src[i]]
 * (index 3 k + c into the projection's [group DOF k][c] output) by rows and columns
 * (MsFEM/MsFEM.h:300-365; MSFEM_ROW_AND_COLUMN of msfem_apply_dirichlet), X = F, and MINRES
 * (precision MSFEM_FP64 or MSFEM_FP32_IR) to ||F - A X|| <= tol ||F||.  The reference runs plain
 * CG restarts on the same system (MsFEM.h:445-478).  U: host [n_dofs][3] out. */
int msfem_cells_order2_macro_solve(msfem_cells_t c, int n_dofs, const int32_t* cell_dofs, int n_vertices,
                                   const double* vertex_xyz, int n_faces, const int32_t* faces, int n_groups,
                                   const int32_t* group_dof_off, const int32_t* group_dofs,
                                   const int32_t* group_face_off, const double* group_values, int n_fixed,
                                   const int32_t* fixed_dofs, const int32_t* fixed_src, int precision, double tol,
                                   int maxiter, double* U, int32_t* iterations, double* rel_residual);

/* Per-cell report of the last build (host arrays of n_cells, any may be NULL):
 * inner iterations, outer refinement steps and final relative residual of the volume
 * problems, and the worst relative residual of the cell's face problems.
 * ms[0..3] = device ms of assembly, edges, faces, volumes; threads[0..1] = CTA size the face
 * and volume launches used (autotuned when build_bases got threads <= 0). */
int msfem_cells_report(msfem_cells_t c, int32_t* inner_iterations, int32_t* outer_iterations, double* rel_residual,
                       double* face_rel_residual, double* ms, int32_t* threads);
/* The MsFEM macro element matrices of every cell from its current bases
 * (FiniteElement_forMech_Poly_Order1::SolveLocalMatrix, MsFEM/MsFEM_Grid.h:3837-3975):
 * the polyhedron quadrature of Library/GeometryShape.h:2708-2760 (for each face cycle of the
 * box (x0: 0 2 6 4, x1: 1 3 7 5, y0: 0 1 5 4, y1: 2 3 7 6, z0: 0 1 3 2, z1: 4 5 7 6) and each
 * face edge, the sub-tetrahedron centroid / face centroid / edge with the 4-point rule), the
 * basis gradients of the micro tetrahedron holding each point (the lowest index on ties), and the
 * material of domain 0 for every cell (MsFEM/MsFEM.h:644-647).
 * K: [n_cells][8][8][3][3] doubles, K[c][I][J] = sum_q w_q B_J^T D B_I as the reference stores
 * A[I][J]. */
int msfem_cells_macro_matrices(msfem_cells_t c, double* K, int on_device);
/* Macro boundary loads (BoundaryFace_forMech_Poly_Order1::SolveLocalBoundaryVector,
 * MsFEM/MsFEM_Grid.h:4104-4135): for item i = (cell, face) with a constant traction t_i,
 * loads[i][v][a] = sum_q w_q t_a psi_v^a(x_q) over the face, with the polygon rule of
 * Library/GeometryShape.h:2563-2600 (sub-triangles centroid / face edge, the triangle 4-point
 * rule of :1482-1540) and the bases interpolated in the micro tetrahedron holding each point.
 * items: [n][2] host ints, traction: [n][3], loads: [n][8][3] host doubles. */
int msfem_cells_face_loads(msfem_cells_t c, int n_items, const int32_t* items, const double* traction, double* loads);

/* The fine solution of every cell from the macro one (the MsFEM solution on the micro meshes):
 * u[b] = sum_v U[cell_vertex[8c+v]] (.) psi_v(b), component by component.  U: [n_vertices][3],
 * u: [cell nodes][3] (concatenated cell numbering), host arrays. */
int msfem_cells_reconstruct(msfem_cells_t c, int n_vertices, const int32_t* cell_vertex, const double* U, double* u);
/* The whole Order1 macro phase of MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly (MsFEM/
 * MsFEM.h:572-1010) on the device after the bases are built: the macro element matrices
 * (msfem_cells_macro_matrices), the boundary loads of the items (msfem_cells_face_loads) summed
 * over the macro vertices item by item (SummPartOfVector, the reference's order), the Dirichlet
 * vertices and the macro solve (msfem_macro_solve), and the fine reconstruction
 * (msfem_cells_reconstruct), without the matrices or loads leaving the GPU.  Host arrays: items
 * [n_items][2], traction [n_items][3], U [n_vertices][3] out; u [cell nodes][3], K_out
 * [n_cells][8][8][3][3] and F_out [n_vertices][3] are optional outputs (NULL: not copied). */
int msfem_cells_order1_macro_solve(msfem_cells_t c, int n_vertices, const int32_t* cell_vertex, int n_items,
                                   const int32_t* items, const double* traction, int n_fixed,
                                   const int32_t* fixed_vertices, const double* fixed_values, int precision, double tol,
                                   int maxiter, double* U, double* u, double* K_out, double* F_out, int32_t* iterations,
                                   double* rel_residual);
/* Replace the bases of every cell ([n_nodes][8][3] doubles, as msfem_cells_get_bases returns
 * them), e.g. with predicted ones.  No reference counterpart. */
int msfem_cells_set_bases(msfem_cells_t c, const double* bases, int on_device);
/* Per cell, how far its current bases are from solving the cell's volume problems: over the
 * interior nodes, rel[c] = ||A_II psi_I + A_IB psi_B|| / ||A_IB psi_B|| (all 8 bases, the matrices
 * of the volume problems, FEM_3D_forElasticDeformation's system for each basis); 0 up to the
 * solver tolerance for the exact bases.  rel: host [n_cells].  No reference counterpart: the
 * learned coarse space's fallback test. */
int msfem_cells_basis_residual(msfem_cells_t c, double* rel);
/* Copies the bases of cell k of src into cell dst_cells[k] of dst (k < n; same node count, same
 * cell-local numbering): the exact bases of re-solved cells back into the full set. */
int msfem_cells_copy_bases(msfem_cells_t dst, msfem_cells_t src, int n, const int32_t* dst_cells);
void msfem_cells_destroy(msfem_cells_t c);

/* The MsFEM macro problem (MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly, MsFEM/MsFEM.h:
 * 572-1010): element matrices K [n_cells][8][8][3][3] over the vertices cell_vertex[8c+v]
 * (SummPartOfMatrix in cell order), loads F [n_vertices][3] (or NULL), every component of the
 * listed Dirichlet vertices fixed (values [n_fixed][3]; a later duplicate wins), then MINRES
 * (the macro matrix is symmetric, not necessarily definite) on the free vertices to
 * ||F_I - A_II U_I|| <= tol ||F_I||.  U: [n_vertices][3] out.  Host arrays. */
int msfem_macro_solve(int n_vertices, int n_cells, const int32_t* cell_vertex, const double* K, const double* F,
                      int n_fixed, const int32_t* fixed_vertices, const double* fixed_values, int precision, double tol,
                      int maxiter, double* U, int32_t* iterations, double* rel_residual);


/* ---------------------------------------------------------------------------------------
 * Two-level preconditioner with the MsFEM coarse space (no counterpart in the reference, which
 * solves the MsFEM macro problem instead, MsFEM/MsFEM.h:572-1010): the Order1 cell bases of a
 * decomposition of the fine mesh into macro cells define the prolongation P (coarse DOF
 * (vertex V, component a) -> the a-component of the cell bases of V; nodes shared by several
 * cells take the mean); the coarse operator is P^T K P with K the textbook (SPD) orientation of
 * the fine element blocks, inverted densely in FP64; M^-1 = diag(A)^-1 + P A_c^-1 P^T.
 * ------------------------------------------------------------------------------------- */

typedef struct msfem_coarse* msfem_coarse_t;

/* fine: an assembled elasticity system with its Dirichlet rows applied; cells: the macro cells
 * (msfem_cells_create + msfem_cells_build_bases) whose fine meshes together are the fine mesh,
 * cell_node_global[b] = fine node of cell node b (concatenated cell numbering);
 * cell_vertex[8c+v] = coarse vertex id (0..n_coarse_vertices-1) of vertex v of cell c;
 * cell_color[c]: cells of one colour share no coarse vertex (fixes the summation order);
 * fixed_dofs: the fine Dirichlet DOFs (3*node + component).  Host arrays. */
int msfem_coarse_create(msfem_system_t fine, msfem_cells_t cells, const int32_t* cell_node_global,
                        int n_coarse_vertices, const int32_t* cell_vertex, const int32_t* cell_color, int n_fixed,
                        const int32_t* fixed_dofs, msfem_coarse_t* out);

/* n_coarse_dofs: free coarse DOFs; ms_setup: device ms of the setup (prolongation, coarse
 * Galerkin matrix, FP64 inverse). */
int msfem_coarse_info(msfem_coarse_t c, int* n_coarse_dofs, double* ms_setup);

/* Inspection: the dense coarse matrix (n_coarse_dofs^2, row-major, before inversion) and the
 * coarse DOF of each (cell, vertex, component), -1 when dropped ([n_cells][8][3]). */
int msfem_coarse_matrix(msfem_coarse_t c, double* A, int32_t* coarse_dof);

/* y = M^-1 r on the Jacobi-scaled system (FP32 host arrays of n_rows): y = r + P^ A_c^-1 P^^T r
 * with P^ = D^1/2 P. */
int msfem_coarse_apply(msfem_coarse_t c, const float* r, float* y);

/* Solves the fine system from its current X: FP64 iterative refinement (r = F - A X, X += d)
 * around preconditioned MINRES with M^-1 above, to ||F - A X|| <= tol ||F||.  precision
 * MSFEM_FP32_IR: FP32 MINRES on the Jacobi-scaled matrix; MSFEM_FP64: FP64 MINRES on the
 * original matrix (the coarse correction stays FP32 in both).  iterations: inner MINRES steps in
 * total; outer: refinement steps. */
int msfem_solve_twolevel(msfem_system_t fine, msfem_coarse_t c, int precision, int maxiter, double tol,
                         double* rel_residual, int* iterations, int* outer);
/* Switches msfem_solve_twolevel (precision MSFEM_FP64) to the symmetric multiplicative cycle
 * on the textbook operator: `textbook` is a second system on the same mesh assembled with
 * msfem_assemble_elastic_textbook and given the same Dirichlet rows.  One application of M^-1:
 * `degree` Chebyshev steps on its Jacobi-scaled FP32 matrix (ratio > 1: the first-kind polynomial
 * for the spectrum bound [lmax/ratio, lmax]; ratio 0: the fourth-kind polynomial on [0, lmax],
 * which needs no lower bound; lmax from 50 power steps x 1.1, widened by the solve if a step
 * fails), the coarse correction,
 * the same Chebyshev steps again; SPD, so
 * MINRES on the reference's matrix keeps its guarantees.  storage: 0 the FP32 SELL matrix; 1 its
 * values in FP16 (arithmetic stays FP32; rounding each entry keeps the matrix symmetric, so the
 * cycle stays SPD; it halves the bytes of the 2*degree SpMVs per cycle); 2 matrix-free on the
 * structured Kuhn grid (msfem_set_kuhn_grid on `textbook`, whose values must be one textbook
 * assembly plus Dirichlet rows since the last msfem_clear): the product is formed from each
 * tetrahedron's material code, FP32, and is checked here against the assembled matrix on a probe
 * vector (relative 1e-5); MSFEM_ERR_STATE if it differs.  The textbook system must outlive c. */
int msfem_coarse_set_smoother(msfem_coarse_t c, msfem_system_t textbook, int degree, double ratio, int storage);
/* on = 1: msfem_solve_twolevel's FP64 MINRES products with the fine (reference) matrix are formed
 * matrix-free on its Kuhn grid (msfem_set_kuhn_grid on the fine system, whose values must be one
 * msfem_assemble_elastic plus Dirichlet rows since the last msfem_clear), checked here against the
 * assembled matrix on a probe vector (relative 1e-12; MSFEM_ERR_STATE if it differs).  The
 * solve's true residuals stay on the assembled matrix.  on = 0: the assembled SELL product. */
int msfem_coarse_set_matrix_free(msfem_coarse_t c, int on);
/* Robustness record of the two-level preconditioner: cells whose bases left [-3, 3] and were
 * replaced by the trilinear functions of their box in the prolongation (the reference's cell
 * operator is indefinite; a nearly singular cell problem returns bases in the thousands, which
 * would make the coarse matrix unusable), the smoother's current lambda_max bound, and how often
 * msfem_solve_twolevel widened it (x1.5, after a refinement step that raised the residual or
 * broke down; the step is undone and repeated).  Any argument may be NULL. */
int msfem_coarse_stats(msfem_coarse_t c, int* trilinear_cells, double* lambda_max, int* widened);
/* Measurement helper (no counterpart in the reference): times `reps` back-to-back launches of one
 * Chebyshev smoothing step of the multiplicative cycle (the smoother's SpMV with its vector update,
 * the dominant kernel of msfem_solve_twolevel) with CUDA events on the solve stream after 3 warm-up
 * launches; reports the mean device time per step and its algorithmic bytes (matrix values in the
 * stored width and block columns as stored, slice pointers, and 24 bytes of vector traffic per
 * row), each counted once.  msfem_coarse_set_smoother must have been called. */
int msfem_coarse_bench_smoother(msfem_coarse_t c, int reps, double* ms_per_step, int64_t* bytes_per_step);
void msfem_coarse_destroy(msfem_coarse_t c);

/* ---------------------------------------------------------------------------------------
 * Learned coarse space (no reference counterpart: the reference's Order1 bases always come
 * from its cell problems).  A 3D convolutional operator reads a macro cell's voxelised
 * Young's-modulus field (16^3 voxels, s ln(E / E_ref) averaged over each voxel, plus the voxel
 * centre) and predicts the cell's 8 vector bases on its 9^3 nodes as a correction to the
 * trilinear functions; it is trained on bases made by msfem_cells_build_bases.  Four 3x3x3
 * layers (4 -> 32 FP32, 32 -> 32, 32 -> 32, 32 -> 24 on BF16 tensor cores with FP32
 * accumulation), ReLU between them; Adam on FP32 master parameters.  Cells must be 8x8x8
 * hexahedra of six Kuhn tetrahedra in Kuhn-cube node and tetrahedron order (checked).
 * Predicted bases only feed the two-level preconditioner's coarse space; with
 * msfem_cells_basis_residual the caller re-solves cells whose prediction is poor. */
typedef struct msfem_net* msfem_net_t;
/* Number of FP32 parameters (the layout of msfem_net_get_params / set_params). */
int msfem_net_param_count(void);
/* New network with seeded He-uniform weights (last layer x 0.1), zero biases. */
int msfem_net_create(uint64_t seed, double E_ref, double in_scale, msfem_net_t* out);
int msfem_net_get_params(msfem_net_t n, float* params);
/* Sets the parameters (host array of msfem_net_param_count() floats) and resets Adam. */
int msfem_net_set_params(msfem_net_t n, const float* params);
/* The network input of every cell of c: vox [n_cells][16][16][16] (host). */
int msfem_net_voxelise(msfem_net_t n, msfem_cells_t c, float* vox);
/* Appends every cell of c (voxels, and its current bases as the target) to the training set; a
 * cell whose bases leave [-3, 3] gets the trilinear functions as its target, as the two-level
 * coarse build would use it. */
int msfem_net_add_cells(msfem_net_t n, msfem_cells_t c, int* n_total);
/* `steps` Adam steps (lr, betas 0.9 / 0.999) on minibatches of `batch` cells drawn from seeded
 * permutations of the training set; losses: [steps] host floats (or NULL). */
int msfem_net_train(msfem_net_t n, int steps, int batch, float lr, uint64_t seed, float* losses);
/* One forward and backward pass on host data without an update: vox [cells][4096], target
 * [cells][729][24] (psi_exact - Q1, channel 3 v + a); loss (mean square) and grad
 * [msfem_net_param_count()] on the host. */
int msfem_net_loss_grad(msfem_net_t n, int cells, const float* vox, const float* target, float* loss, float* grad);
/* The last layer's output: out [cells][4096][32] (channels 24..31 zero). */
int msfem_net_forward(msfem_net_t n, int cells, const float* vox, float* out);
/* Predicts the bases of every cell of c into c (as msfem_cells_set_bases would); ms: device time. */
int msfem_net_predict(msfem_net_t n, msfem_cells_t c, float* ms);
/* Tensor-core path of layers 1-3 (forward and data gradient): 0 = warp-level mma.sync, 1 =
 * tcgen05 with TMEM accumulators and M = 64 voxel tiles (N = 32 channels), 2 = tcgen05 on the
 * transposed product (M = 64 channel rows, N = 256 voxels of a plane), 3 = the M = 64 tcgen05
 * tiles in a persistent warp-specialised kernel (a producer warp fills a ring of plane slots, one
 * thread issues the MMAs into two TMEM accumulators, four epilogue warps drain them).  All compute
 * the same function (FP32 accumulation order may differ). */
int msfem_net_set_tensor_path(msfem_net_t n, int tcgen05);
int msfem_net_destroy(msfem_net_t n);

#ifdef __cplusplus
}
#endif
#endif /* MSFEM_B200_H */
