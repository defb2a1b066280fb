/* Test infrastructure only: the CPU oracle, a plain-C restatement of the
 * reference's hot path (element matrices, portrait, assembly into CSSD,
 * boundary conditions, Krylov solvers).  Used by tests/ and bench.py's CPU
 * baseline as the checker; never linked into the product.
 *
 * Matrices are CSR with the diagonal included and every row sorted ascending,
 * which is the reference CSSD row [A_down asc | Diag | A_up asc]
 * (Library/CSSD_Matrix.h:11-15) laid end to end.
 */
#ifndef FEMORACLE_H
#define FEMORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;
    long long nnz;
    int* row_ptr;
    int* col;
    double* val;
    double* F;
    double* X;
} fo_csr;

void fo_free_csr(fo_csr* A);

/* FEM/FEM_Grid.h:2125-2192 : K[((I*4+J)*3+a)*3+b] = A[I][J].val[a][b] */
void fo_elastic_local(const double* xyz4, double E, double nu, double* K144);
/* FEM/FEM_Grid.h:103-152 : K[I*4+J] */
void fo_scalar_local(const double* xyz4, double sigma, double* K16);

/* FEM/FEM_Grid.h:665-716 (scalar) / :3236-3287 (mech): node-level portrait as CSR with diagonal */
int fo_portrait(int n_nodes, int n_tets, const int* tets, int** row_ptr, int** col);

/* FEM/FEM.h:1286-1813 : FEM_forElasticDeformation up to the solve (stage 0: before BCs) */
int fo_elastic_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                      int n_mat, const double* E, const double* nu,
                      int n_bc, const int* bc_node, const int* bc_mask, const double* bc_val,
                      int n_faces, const int* face_nodes, const int* face_elem, const double* face_traction,
                      int stage, fo_csr* out);

/* FEM/FEM.h:398-619 (+ X = F, FEM.h:635): stiffness-only FEM_forBaseEliptic up to the solve */
int fo_scalar_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                     int n_mat, const double* sigma, int n_bc, const int* bc_node, const double* bc_val,
                     int stage, fo_csr* out);

/* Library/CSSD_Matrix.h:395-423 */
void fo_spmv(int n, const int* row_ptr, const int* col, const double* val, const double* x, double* y);

/* Solvers.  X: initial guess in, solution out.  Return the true relative residual
 * ||F-AX||/||F|| computed at exit; *iters = iterations performed. */
double fo_cg(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
             int maxiter, double tol, int* iters);                                   /* CSSD_Matrix.h:1496-1576 */
double fo_pcg_ssor(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                   int maxiter, double tol, double w, int* iters);                   /* CSSD_Matrix.h:1302-1398, :458-547 */
double fo_pcg_jacobi(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                     int maxiter, double tol, int* iters);                           /* the PCG loop above, M = diag(A) */
double fo_bicgstab(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                   int maxiter, double tol, int* iters);                             /* CSSD_Matrix.h:730-853 */
double fo_gmres(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                int m, int maxiter, double tol, int* iters);                         /* restarted GMRES(m), Givens; Library/GMRES/7_gmres.for:95-222 */
double fo_gmres_ref(int n, const int* rp, const int* ci, double* v, double* F, double* X,
                    int maxiter, double tol, int* iters);                            /* CSSD_Matrix.h:1774-1989, quirks included */
void fo_ssor_apply(int n, const int* rp, const int* ci, const double* v, double w, const double* r, double* z);
/* Not in the reference (test infrastructure and the CPU baseline of the elasticity benchmark):
 * MINRES (Paige-Saunders) on the Jacobi-scaled matrix inside FP64 iterative refinement, OpenMP
 * products; stops when ||F - A X|| <= tol ||F||.  Returns that relative residual. */
double fo_minres(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                 int maxiter, double tol, int* iters);

#ifdef __cplusplus
}
#endif
#endif
