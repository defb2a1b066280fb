/* Test infrastructure only: the CPU oracle (plain C restatement of the
 * reference's hot path).  See femoracle.h.  Compiled with -O2
 * -ffp-contract=off so that, like the reference built by g++ for x86-64, no
 * multiply-add is fused: the solvers below evaluate every sum in the
 * reference's order and reproduce its iterates bit for bit on the same matrix.
 */
#include "femoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void fo_free_csr(fo_csr* A)
{
    if (!A) return;
    free(A->row_ptr); free(A->col); free(A->val); free(A->F); free(A->X);
    memset(A, 0, sizeof(*A));
}

/* ---------------------------------------------------------------- geometry */

/* Gradients of the four P1 basis functions and the volume of a tetrahedron.
 * Same quantities as Tetrahedron::SolveAlphaMatrix (alpha[v][1..3],
 * Library/GeometryShape.h:1960-2086) and GetVolume (:1674-1705), written with
 * edge vectors: for e_k = p_k - p_0, grad(lambda_1) = (e2 x e3)/det,
 * grad(lambda_2) = (e3 x e1)/det, grad(lambda_3) = (e1 x e2)/det, and
 * grad(lambda_0) = -(sum of the other three); det = e1 . (e2 x e3) = +-6V. */
static void tet_gradients(const double* p, double g[4][3], double* vol)
{
    double e1[3], e2[3], e3[3];
    for (int a = 0; a < 3; a++) {
        e1[a] = p[3 + a] - p[a];
        e2[a] = p[6 + a] - p[a];
        e3[a] = p[9 + a] - p[a];
    }
    double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
    double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
    double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
    for (int a = 0; a < 3; a++) {
        g[1][a] = c23[a] / det;
        g[2][a] = c31[a] / det;
        g[3][a] = c12[a] / det;
        g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
    }
    *vol = fabs(det) / 6.0;
}

/* Isotropic Voigt D in the order xx, yy, zz, xy, yz, xz
 * (Domain::forMech::SetIsotropic_D, Library/Domain.h:53-78). */
static void isotropic_d(double E, double nu, double D[6][6])
{
    double k = E * (1. - nu) / (1. + nu) / (1. - 2. * nu);
    double b = (1. - 2. * nu) / (2. * (1. - nu));
    double a = nu / (1. - nu);
    memset(D, 0, sizeof(double) * 36);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = (i == j ? 1. : a) * k;
    for (int i = 3; i < 6; i++) D[i][i] = b * k;
}

/* Strain-displacement matrix of one basis function with gradient g (6x3),
 * rows xx, yy, zz, xy, yz, xz (FEM/FEM_Grid.h:2158-2166). */
static void b_matrix(const double* g, double B[6][3])
{
    memset(B, 0, sizeof(double) * 18);
    B[0][0] = g[0];
    B[1][1] = g[1];
    B[2][2] = g[2];
    B[3][0] = g[1]; B[3][1] = g[0];
    B[4][1] = g[2]; B[4][2] = g[1];
    B[5][0] = g[2]; B[5][2] = g[0];
}

/* FEM/FEM_Grid.h:2125-2192.  For J >= I the block A[I][J] = V * B_J^T D B_I
 * (the 4-point rule of a constant integrand sums the weights to V), and
 * A[J][I] = A[I][J]^T.  Note the orientation: the trial function I sits on the
 * right, which is the transpose of the textbook K_IJ. */
void fo_elastic_local(const double* xyz4, double E, double nu, double* K)
{
    double g[4][3], V, D[6][6], B[4][6][3];
    tet_gradients(xyz4, g, &V);
    isotropic_d(E, nu, D);
    for (int v = 0; v < 4; v++) b_matrix(g[v], B[v]);
    for (int I = 0; I < 4; I++)
        for (int J = I; J < 4; J++) {
            double blk[3][3];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    double s = 0;
                    for (int k = 0; k < 6; k++) {
                        double t = 0;
                        for (int l = 0; l < 6; l++) t += B[J][l][a] * D[l][k];
                        s += t * B[I][k][b];
                    }
                    blk[a][b] = s * V;
                }
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    K[((I * 4 + J) * 3 + a) * 3 + b] = blk[a][b];
                    K[((J * 4 + I) * 3 + b) * 3 + a] = blk[a][b];
                }
        }
}

/* FEM/FEM_Grid.h:103-152: K_IJ = sigma * grad(phi_I) . grad(phi_J) * V (1-point rule). */
void fo_scalar_local(const double* xyz4, double sigma, double* K)
{
    double g[4][3], V;
    tet_gradients(xyz4, g, &V);
    for (int I = 0; I < 4; I++)
        for (int J = 0; J < 4; J++)
            K[I * 4 + J] = sigma * (g[I][0] * g[J][0] + g[I][1] * g[J][1] + g[I][2] * g[J][2]) * V;
}

/* ---------------------------------------------------------------- portrait */

static int cmp_int(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* CreationPortrait (FEM/FEM_Grid.h:665-716, :3236-3287): every pair of distinct
 * nodes of an element couples; rows sorted and de-duplicated; the diagonal is
 * stored separately by the reference and appears here at its sorted place. */
int fo_portrait(int n, int n_tets, const int* tets, int** row_ptr_out, int** col_out)
{
    int* cnt = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int e = 0; e < n_tets; e++)
        for (int a = 0; a < 4; a++) cnt[tets[4 * e + a]] += 3;
    long long* start = (long long*)malloc(sizeof(long long) * ((size_t)n + 1));
    start[0] = 0;
    for (int i = 0; i < n; i++) start[i + 1] = start[i] + cnt[i] + 1;
    int* tmp = (int*)malloc(sizeof(int) * (size_t)start[n]);
    long long* fill = (long long*)malloc(sizeof(long long) * (size_t)n);
    for (int i = 0; i < n; i++) { tmp[start[i]] = i; fill[i] = start[i] + 1; }
    for (int e = 0; e < n_tets; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++)
                if (a != b) {
                    int i = tets[4 * e + a];
                    tmp[fill[i]++] = tets[4 * e + b];
                }
    int* rp = (int*)malloc(sizeof(int) * ((size_t)n + 1));
    long long total = 0;
    for (int i = 0; i < n; i++) {
        int len = (int)(fill[i] - start[i]);
        int* r = tmp + start[i];
        qsort(r, (size_t)len, sizeof(int), cmp_int);
        int u = 0;
        for (int k = 0; k < len; k++)
            if (k == 0 || r[k] != r[u - 1]) r[u++] = r[k];
        cnt[i] = u;
        rp[i] = (int)total;
        total += u;
    }
    rp[n] = (int)total;
    int* col = (int*)malloc(sizeof(int) * (size_t)total);
    for (int i = 0; i < n; i++) memcpy(col + rp[i], tmp + start[i], sizeof(int) * (size_t)cnt[i]);
    free(cnt); free(start); free(tmp); free(fill);
    *row_ptr_out = rp;
    *col_out = col;
    return 0;
}

static int find_col(const int* rp, const int* col, int row, int c)
{
    int lo = rp[row], hi = rp[row + 1] - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (col[mid] == c) return mid;
        if (col[mid] < c) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

/* ---------------------------------------------------------------- boundary conditions */

/* The reference's column sweep (FEM/FEM.h:1757-1812 and :565-607): for every
 * row, walk its A_up columns ascending with a pointer into the boundary list
 * that only moves forward and stops at the first entry >= the column; a hit
 * moves A*F[col] to the right-hand side and zeroes the entry.  The pointer is
 * reset for the A_down walk.  With an unsorted boundary list some columns are
 * therefore never reached, exactly as in the reference. */
static void column_sweep(int n, const int* rp, const int* col, double* val, double* F, const int* use_id, int L)
{
    for (int row = 0; row < n; row++) {
        int pd = rp[row];
        while (pd < rp[row + 1] && col[pd] < row) pd++;
        /* A_up part: entries after the diagonal */
        int it = 0;
        for (int p = pd + 1; p < rp[row + 1]; p++) {
            int c = col[p];
            for (; it < L; it++) {
                if (use_id[it] == c) { F[row] -= val[p] * F[c]; val[p] = 0; break; }
                if (use_id[it] > c) break;
            }
        }
        it = 0;
        for (int p = rp[row]; p < pd; p++) {
            int c = col[p];
            for (; it < L; it++) {
                if (use_id[it] == c) { F[row] -= val[p] * F[c]; val[p] = 0; break; }
                if (use_id[it] > c) break;
            }
        }
    }
}

static void dirichlet_row(const int* rp, const int* col, double* val, double* F, double* X, int d, double value)
{
    X[d] = value;
    F[d] = value;
    for (int p = rp[d]; p < rp[d + 1]; p++) val[p] = (col[p] == d) ? 1.0 : 0.0;
}

/* ---------------------------------------------------------------- systems */

int fo_elastic_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                      int n_mat, const double* E, const double* nu,
                      int n_bc, const int* bc_node, const int* bc_mask, const double* bc_val,
                      int n_faces, const int* face_nodes, const int* face_elem, const double* face_traction,
                      int stage, fo_csr* out)
{
    (void)face_elem;
    int *brp, *bcol;
    fo_portrait(n_nodes, n_tets, tets, &brp, &bcol);
    long long nb = brp[n_nodes];
    double* bval = (double*)calloc((size_t)nb * 9, sizeof(double));
    double* bF = (double*)calloc((size_t)n_nodes * 3, sizeof(double));
    /* traction (FEM/FEM.h:1338-1343; FEM_Grid.h:2622-2661): the 4-point triangle
     * rule on a linear integrand gives each face vertex area/3 of the traction */
    for (int f = 0; f < n_faces; f++) {
        const double* a = xyz + 3 * face_nodes[3 * f];
        const double* b = xyz + 3 * face_nodes[3 * f + 1];
        const double* c = xyz + 3 * face_nodes[3 * f + 2];
        double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        for (int v = 0; v < 3; v++)
            for (int d = 0; d < 3; d++) bF[3 * face_nodes[3 * f + v] + d] += face_traction[3 * f + d] * area / 3.0;
    }
    /* element loop + SummPartOfMatrix in element order (FEM/FEM.h:1349-1384) */
    for (int e = 0; e < n_tets; e++) {
        int m = mat ? mat[e] : 0;
        if (m < 0 || m >= n_mat || E[m] <= 0) continue;
        double p[12], K[144];
        for (int v = 0; v < 4; v++)
            for (int d = 0; d < 3; d++) p[3 * v + d] = xyz[3 * tets[4 * e + v] + d];
        fo_elastic_local(p, E[m], nu[m], K);
        for (int I = 0; I < 4; I++) {
            int row = tets[4 * e + I];
            for (int J = 0; J < 4; J++) {
                int slot = find_col(brp, bcol, row, tets[4 * e + J]);
                for (int q = 0; q < 9; q++) bval[(size_t)slot * 9 + q] += K[(I * 4 + J) * 9 + q];
            }
        }
    }
    /* block -> scalar expansion, DOF = 3*node + component (Library/Math.h:1963-2054) */
    int n = 3 * n_nodes;
    out->n = n;
    out->nnz = nb * 9;
    out->row_ptr = (int*)malloc(sizeof(int) * ((size_t)n + 1));
    out->col = (int*)malloc(sizeof(int) * (size_t)out->nnz);
    out->val = (double*)malloc(sizeof(double) * (size_t)out->nnz);
    out->F = bF;
    out->X = (double*)calloc((size_t)n, sizeof(double));
    long long p = 0;
    for (int i = 0; i < n_nodes; i++)
        for (int c = 0; c < 3; c++) {
            out->row_ptr[3 * i + c] = (int)p;
            for (int s = brp[i]; s < brp[i + 1]; s++)
                for (int d = 0; d < 3; d++) {
                    out->col[p] = 3 * bcol[s] + d;
                    out->val[p++] = bval[(size_t)s * 9 + c * 3 + d];
                }
        }
    out->row_ptr[n] = (int)p;
    free(brp); free(bcol); free(bval);
    if (stage >= 1) {
        /* Dirichlet rows in boundary-list order, then the column sweep (FEM/FEM.h:1676-1813) */
        int* use_id = (int*)malloc(sizeof(int) * (size_t)(3 * n_bc + 1));
        int L = 0;
        for (int b = 0; b < n_bc; b++)
            for (int c = 0; c < 3; c++)
                if (bc_mask[b] & (1 << c)) {
                    int d = 3 * bc_node[b] + c;
                    use_id[L++] = d;
                    dirichlet_row(out->row_ptr, out->col, out->val, out->F, out->X, d, bc_val[3 * b + c]);
                }
        column_sweep(n, out->row_ptr, out->col, out->val, out->F, use_id, L);
        free(use_id);
    }
    return 0;
}

int fo_scalar_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                     int n_mat, const double* sigma, int n_bc, const int* bc_node, const double* bc_val,
                     int stage, fo_csr* out)
{
    int *rp, *col;
    fo_portrait(n_nodes, n_tets, tets, &rp, &col);
    out->n = n_nodes;
    out->nnz = rp[n_nodes];
    out->row_ptr = rp;
    out->col = col;
    out->val = (double*)calloc((size_t)out->nnz, sizeof(double));
    out->F = (double*)calloc((size_t)n_nodes, sizeof(double));
    out->X = (double*)calloc((size_t)n_nodes, sizeof(double));
    for (int e = 0; e < n_tets; e++) {
        int m = mat ? mat[e] : 0;
        if (m < 0 || m >= n_mat) continue;
        double p[12], K[16];
        for (int v = 0; v < 4; v++)
            for (int d = 0; d < 3; d++) p[3 * v + d] = xyz[3 * tets[4 * e + v] + d];
        fo_scalar_local(p, sigma[m], K);
        for (int I = 0; I < 4; I++)
            for (int J = 0; J < 4; J++) out->val[find_col(rp, col, tets[4 * e + I], tets[4 * e + J])] += K[I * 4 + J];
    }
    if (stage >= 1) {
        for (int b = 0; b < n_bc; b++) dirichlet_row(rp, col, out->val, out->F, out->X, bc_node[b], bc_val[b]);
        column_sweep(n_nodes, rp, col, out->val, out->F, bc_node, n_bc);
        memcpy(out->X, out->F, sizeof(double) * (size_t)n_nodes); /* X = F before the solve, FEM/FEM.h:635 */
    }
    return 0;
}

/* ---------------------------------------------------------------- solvers */

/* CSSD_Matrix::MultiplicationMatrixVector (Library/CSSD_Matrix.h:395-423):
 * per row, A_up terms ascending, then A_down ascending, then the diagonal. */
void fo_spmv(int n, const int* rp, const int* col, const double* v, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        int pd = rp[i];
        while (pd < rp[i + 1] && col[pd] < i) pd++;
        double t = 0.0;
        for (int p = pd + 1; p < rp[i + 1]; p++) t += v[p] * x[col[p]];
        for (int p = rp[i]; p < pd; p++) t += v[p] * x[col[p]];
        if (pd < rp[i + 1] && col[pd] == i) t += v[pd] * x[i];
        y[i] = t;
    }
}

/* math::MakeInnerProduct (Library/Math.h:1633-1654): serial FP64 sum */
static double dot(int n, const double* a, const double* b)
{
    double r = 0.0;
    for (int i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}

static double true_residual(int n, const int* rp, const int* ci, const double* v, const double* F, const double* X)
{
    double* t = (double*)malloc(sizeof(double) * (size_t)n);
    fo_spmv(n, rp, ci, v, X, t);
    double a = 0, b = 0;
    for (int i = 0; i < n; i++) { a += (t[i] - F[i]) * (t[i] - F[i]); b += F[i] * F[i]; }
    free(t);
    return sqrt(a / b);
}

/* MSG (Library/CSSD_Matrix.h:1496-1576) */
double fo_cg(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
             int maxiter, double tol, int* iters)
{
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    fo_spmv(n, rp, ci, v, X, q);
    for (int i = 0; i < n; i++) { r[i] = F[i] - q[i]; z[i] = r[i]; }
    int k;
    for (k = 1; k <= maxiter && sqrt(dot(n, r, r) / dot(n, F, F)) > tol; k++) {
        double rs = dot(n, r, r);
        fo_spmv(n, rp, ci, v, z, q);
        double a = rs / dot(n, q, z);
        for (int i = 0; i < n; i++) { X[i] += a * z[i]; r[i] -= a * q[i]; }
        double b = dot(n, r, r) / rs;
        for (int i = 0; i < n; i++) z[i] = r[i] + b * z[i];
    }
    if (iters) *iters = k - 1;
    free(r); free(z); free(q);
    return true_residual(n, rp, ci, v, F, X);
}

/* PrecondorSSOR(w) + SolvePrecondorSSOR_SLAE (Library/CSSD_Matrix.h:458-547):
 * the stored off-diagonals are -w*A and the sweeps subtract them, so
 * z = (D - wL)^{-1} [w(2-w) D] (D - wU)^{-1} r, backward sweep first. */
void fo_ssor_apply(int n, const int* rp, const int* ci, const double* v, double w, const double* r, double* z)
{
    for (int I = n - 1; I >= 0; I--) {
        double diag = 0;
        double x = r[I];
        for (int p = rp[I]; p < rp[I + 1]; p++) {
            if (ci[p] > I) x -= z[ci[p]] * (-1 * w * v[p]);
            else if (ci[p] == I) diag = v[p];
        }
        z[I] = x / diag;
    }
    for (int I = 0; I < n; I++) {
        double diag = 0;
        for (int p = rp[I]; p < rp[I + 1]; p++)
            if (ci[p] == I) diag = v[p];
        z[I] = z[I] / (1.0 / diag / w / (2 - w));
    }
    for (int I = 0; I < n; I++) {
        double diag = 0;
        double x = z[I];
        for (int p = rp[I]; p < rp[I + 1]; p++) {
            if (ci[p] < I) x -= z[ci[p]] * (-1 * w * v[p]);
            else if (ci[p] == I) diag = v[p];
        }
        z[I] = x / diag;
    }
}

/* the PCG loop of MSG_PreconditioningSSOR (Library/CSSD_Matrix.h:1302-1398) with a
 * pluggable preconditioner: kind 0 = reference SSOR(w), kind 1 = Jacobi */
static double pcg(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                  int maxiter, double tol, int kind, double w, int* iters)
{
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    double* dg = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        dg[i] = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i) dg[i] = v[k];
    }
#define PRECOND()                                                    \
    do {                                                             \
        if (kind == 0) fo_ssor_apply(n, rp, ci, v, w, r, z);         \
        else for (int i_ = 0; i_ < n; i_++) z[i_] = r[i_] / dg[i_];  \
    } while (0)
    fo_spmv(n, rp, ci, v, X, q);
    for (int i = 0; i < n; i++) r[i] = F[i] - q[i];
    PRECOND();
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = dot(n, r, z);
    int k;
    for (k = 1; k < maxiter && sqrt(dot(n, r, r) / dot(n, F, F)) > tol; k++) {
        fo_spmv(n, rp, ci, v, p, q);
        double alpha = rz / dot(n, q, p);
        for (int i = 0; i < n; i++) { X[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        PRECOND();
        double beta = dot(n, r, z) / rz;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = dot(n, r, z);
    }
#undef PRECOND
    if (iters) *iters = k - 1;
    free(r); free(z); free(p); free(q); free(dg);
    return true_residual(n, rp, ci, v, F, X);
}

double fo_pcg_ssor(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                   int maxiter, double tol, double w, int* iters)
{
    return pcg(n, rp, ci, v, F, X, maxiter, tol, 0, w, iters);
}

double fo_pcg_jacobi(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                     int maxiter, double tol, int* iters)
{
    return pcg(n, rp, ci, v, F, X, maxiter, tol, 1, 0.0, iters);
}

/* BiCG_Stab (Library/CSSD_Matrix.h:730-853): the residual is recomputed as F - AX
 * every step, and the loop stops as soon as (r, r) grows. */
double fo_bicgstab(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                   int maxiter, double tol, int* iters)
{
    size_t sz = sizeof(double) * (size_t)n;
    double *res = malloc(sz), *mult = malloc(sz), *P = malloc(sz), *V = malloc(sz), *S = malloc(sz), *T = malloc(sz),
           *radd = malloc(sz);
    fo_spmv(n, rp, ci, v, X, mult);
    for (int i = 0; i < n; i++) res[i] = F[i] * 1.0 + mult[i] * -1.0;
    double nrc = dot(n, res, res), nF = dot(n, F, F), nrp = 0;
    double alpha = 1, omega = 1, betta;
    memcpy(radd, res, sz);
    memcpy(P, res, sz);
    double real_prev = nrc, real;
    int k;
    for (k = 1; k < maxiter && sqrt(nrc / nF) > tol && nrc == nrc; k++) {
        fo_spmv(n, rp, ci, v, P, V);
        nrp = dot(n, res, radd);
        alpha = nrp / dot(n, radd, V);
        for (int i = 0; i < n; i++) S[i] = res[i] * 1.0 + V[i] * -alpha;
        fo_spmv(n, rp, ci, v, S, T);
        omega = dot(n, T, S) / dot(n, T, T);
        for (int i = 0; i < n; i++) mult[i] = S[i] * omega + P[i] * alpha;
        for (int i = 0; i < n; i++) X[i] = X[i] * 1.0 + mult[i] * 1.0;
        fo_spmv(n, rp, ci, v, X, mult);
        for (int i = 0; i < n; i++) res[i] = F[i] * 1.0 + mult[i] * -1.0;
        nrc = dot(n, res, radd);
        betta = (nrc / nrp) * (alpha / omega);
        for (int i = 0; i < n; i++) mult[i] = P[i] * betta + V[i] * (-betta * omega);
        for (int i = 0; i < n; i++) P[i] = res[i] * 1 + mult[i] * 1;
        real = dot(n, res, res);
        if (real > real_prev) break;
        real_prev = real;
    }
    if (iters) *iters = k - 1;
    free(res); free(mult); free(P); free(V); free(S); free(T); free(radd);
    double result = true_residual(n, rp, ci, v, F, X);
    return (k == 1) ? -result : result;
}

/* Restarted GMRES(m) with modified Gram-Schmidt and Givens rotations, x0 from X;
 * stops when the relative residual estimate drops below tol.  Follows the
 * restart loop, rotations and back substitution of the reference's legacy
 * GMRS (Library/GMRES/7_gmres.for:95-222) with its preconditioner disabled
 * (intik = 0 there).  The reference ships no compiled GMRES(m>5). */
double fo_gmres(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                int m, int maxiter, double tol, int* iters)
{
    size_t sz = sizeof(double) * (size_t)n;
    double* Vb = (double*)malloc(sz * (size_t)(m + 1));
    double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
    double *cs = calloc(m, sizeof(double)), *sn = calloc(m, sizeof(double)), *g = calloc(m + 1, sizeof(double));
    double* w = (double*)malloc(sz);
    double nF = sqrt(dot(n, F, F));
    int total = 0;
    double rel = 1.0;
    while (total < maxiter) {
        fo_spmv(n, rp, ci, v, X, w);
        for (int i = 0; i < n; i++) Vb[i] = F[i] - w[i];
        double beta = sqrt(dot(n, Vb, Vb));
        rel = beta / nF;
        if (rel <= tol) break;
        for (int i = 0; i < n; i++) Vb[i] /= beta;
        memset(g, 0, sizeof(double) * (m + 1));
        g[0] = beta;
        int j;
        for (j = 0; j < m && total < maxiter; j++, total++) {
            double* vj = Vb + (size_t)j * n;
            double* vn = Vb + (size_t)(j + 1) * n;
            fo_spmv(n, rp, ci, v, vj, vn);
            for (int i = 0; i <= j; i++) {
                double h = dot(n, vn, Vb + (size_t)i * n);
                H[i * m + j] = h;
                for (int l = 0; l < n; l++) vn[l] -= h * Vb[(size_t)i * n + l];
            }
            double hn = sqrt(dot(n, vn, vn));
            H[(j + 1) * m + j] = hn;
            if (hn != 0) for (int l = 0; l < n; l++) vn[l] /= hn;
            for (int i = 0; i < j; i++) {
                double a = H[i * m + j], b = H[(i + 1) * m + j];
                H[i * m + j] = cs[i] * a + sn[i] * b;
                H[(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
            }
            double a = H[j * m + j], b = H[(j + 1) * m + j];
            double d = sqrt(a * a + b * b);
            cs[j] = a / d;
            sn[j] = b / d;
            H[j * m + j] = d;
            H[(j + 1) * m + j] = 0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            rel = fabs(g[j + 1]) / nF;
            if (rel <= tol) { j++; total++; break; }
        }
        /* back substitution and update */
        double* y = (double*)calloc((size_t)j + 1, sizeof(double));
        for (int i = j - 1; i >= 0; i--) {
            double s = g[i];
            for (int l = i + 1; l < j; l++) s -= H[i * m + l] * y[l];
            y[i] = s / H[i * m + i];
        }
        for (int i = 0; i < j; i++)
            for (int l = 0; l < n; l++) X[l] += y[i] * Vb[(size_t)i * n + l];
        free(y);
        if (rel <= tol) break;
    }
    if (iters) *iters = total;
    free(Vb); free(H); free(cs); free(sn); free(g); free(w);
    return true_residual(n, rp, ci, v, F, X);
}

/* CSSD_Matrix::GMRES (Library/CSSD_Matrix.h:1774-1989), restated with its
 * behaviour intact: depth 5, every row (and F, X) divided in place by its
 * Euclidean norm, an absolute stopping test on the least-squares residual, the
 * orthogonalisation vector reset to A*v_j before each projection (so only the
 * last projection is subtracted), Givens rotations applied across all 5 columns
 * (Minimization_Problem, :1727-1773), and the update V^T y accumulated on top of
 * A*X (left there by the progress print) with the residual coefficient
 * included.  v, F and X are
 * modified in place like the reference's own members.  *iters = restarts. */
double fo_gmres_ref(int n, const int* rp, const int* ci, double* v, double* F, double* X,
                    int maxiter, double tol, int* iters)
{
    const int M0 = 5;
    int M = M0;
    for (int i = 0; i < n; i++) {
        double koef = 0.0;
        int pd = rp[i];
        while (pd < rp[i + 1] && ci[pd] < i) pd++;
        koef += v[pd] * v[pd];
        for (int p = pd + 1; p < rp[i + 1]; p++) koef += v[p] * v[p];
        for (int p = rp[i]; p < pd; p++) koef += v[p] * v[p];
        koef = sqrt(koef);
        X[i] /= koef;
        F[i] /= koef;
        for (int p = rp[i]; p < rp[i + 1]; p++) v[p] /= koef;
    }
    double H[6][5], V_dummy = 0;
    (void)V_dummy;
    double* V = (double*)calloc((size_t)(M0 + 1) * n, sizeof(double));
    double* W = (double*)calloc((size_t)M0 * n, sizeof(double));
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* Help = (double*)malloc(sizeof(double) * (size_t)n);
    double f[6];
    int fsize = M0 + 1;
    fo_spmv(n, rp, ci, v, X, Help);
    for (int i = 0; i < n; i++) r[i] = F[i] * 1.0 + Help[i] * -1.0;
    double Norma_r = sqrt(dot(n, r, r));
    double Norma_F = sqrt(dot(n, F, F));
    int Flag = 0, Iter = 0;
    while (Flag == 0 && Iter < maxiter) {
        M = M0;
        int flag_m = 0;
        memset(H, 0, sizeof(H));
        memset(V, 0, sizeof(double) * (size_t)(M0 + 1) * n);
        memset(W, 0, sizeof(double) * (size_t)M0 * n);
        for (int i = 0; i < n; i++) V[i] = r[i] / Norma_r;
        for (int j = 0; j < M && flag_m == 0; j++) {
            fo_spmv(n, rp, ci, v, V + (size_t)j * n, Help);
            for (int i = 0; i <= j; i++) {
                H[i][j] = 0.0;
                for (int l = 0; l < n; l++) {
                    W[(size_t)j * n + l] = Help[l];
                    H[i][j] += W[(size_t)j * n + l] * V[(size_t)i * n + l];
                }
                for (int l = 0; l < n; l++) W[(size_t)j * n + l] -= H[i][j] * V[(size_t)i * n + l];
            }
            H[j + 1][j] = sqrt(dot(n, W + (size_t)j * n, W + (size_t)j * n));
            if (fabs(H[j + 1][j]) < tol) {
                M = j;
                flag_m = 1;
            } else {
                for (int l = 0; l < n; l++) V[(size_t)(j + 1) * n + l] = W[(size_t)j * n + l] / H[j + 1][j];
            }
        }
        /* Minimization_Problem(M, Norma_r, f, H) */
        int m = M;
        fsize = m + 1;
        for (int i = 1; i < m + 1; i++) f[i] = 0.0;
        f[0] = Norma_r;
        for (int i = 0; i < m; i++) {
            double t = H[i + 1][i] / H[i][i];
            double c = 1.0 / sqrt(1 + t * t);
            double s = t * c;
            for (int k = i; k < M0; k++) {
                double h1 = c * H[i][k] + s * H[i + 1][k];
                double h2 = c * H[i + 1][k] - s * H[i][k];
                H[i][k] = h1;
                H[i + 1][k] = h2;
            }
            double h1 = c * f[i] + s * f[i + 1];
            double h2 = c * f[i + 1] - s * f[i];
            f[i] = h1;
            f[i + 1] = h2;
        }
        for (int i = m - 1; i >= 0; i--) {
            f[i] /= H[i][i];
            for (int j = i - 1; j >= 0; j--) f[j] -= H[j][i] * f[i];
        }
        double Norma_Residual = fabs(f[m]);
        /* the per-cycle progress print (CSSD_Matrix.h:1919-1926) leaves Help = A*X */
        fo_spmv(n, rp, ci, v, X, Help);
        if (Norma_Residual < tol) {
            Flag = 1;
        } else {
            /* MultiplicationTMatrixVector(V, f, Help): Help keeps its contents and accumulates */
            for (int i = 0; i < fsize; i++)
                for (int l = 0; l < n; l++) Help[l] += V[(size_t)i * n + l] * f[i];
            for (int l = 0; l < n; l++) X[l] += Help[l];
            fo_spmv(n, rp, ci, v, X, Help);
            for (int l = 0; l < n; l++) r[l] = F[l] * 1.0 + Help[l] * -1.0;
            Norma_r = sqrt(dot(n, r, r));
            Iter++;
        }
    }
    fo_spmv(n, rp, ci, v, X, Help);
    double temp = 0;
    for (int i = 0; i < n; i++) temp += (F[i] - Help[i]) * (F[i] - Help[i]);
    if (iters) *iters = Iter;
    free(V); free(W); free(r); free(Help);
    return sqrt(temp) / Norma_F;
}

/* ---------------------------------------------------------------------------------------------
 * MINRES on S A S (S = |diag A|^-1/2) inside FP64 iterative refinement -- not a reference
 * routine: the CPU counterpart of the GPU's Jacobi MINRES, for matrices that are symmetric but
 * indefinite (the reference's elasticity assembly), where CG need not converge.  Recurrences as in
 * Elman, Silvester and Wathen, "Finite Elements and Fast Iterative Solvers", Algorithm 2.4.
 * ------------------------------------------------------------------------------------------- */
static double pdot(int n, const double* a, const double* b)
{
    double r = 0.0;
#pragma omp parallel for reduction(+ : r) schedule(static)
    for (int i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}

/* y = S A S x */
static void scaled_spmv(int n, const int* rp, const int* ci, const double* v, const double* s, const double* x,
                        double* t, double* y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) t[i] = s[i] * x[i];
    fo_spmv(n, rp, ci, v, t, y);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) y[i] *= s[i];
}

/* y += solution of (S A S) y = b to ||b - S A S y|| <= tau ||b||, from y = 0; returns iterations */
static int minres_scaled(int n, const int* rp, const int* ci, const double* v, const double* s, const double* b,
                         double* y, int maxiter, double tau)
{
    double* vp = (double*)calloc((size_t)n, sizeof(double));
    double* vc = (double*)malloc(sizeof(double) * (size_t)n);
    double* vn = (double*)malloc(sizeof(double) * (size_t)n);
    double* wp = (double*)calloc((size_t)n, sizeof(double));
    double* wc = (double*)calloc((size_t)n, sizeof(double));
    double* t = (double*)malloc(sizeof(double) * (size_t)n);
    double g1 = sqrt(pdot(n, b, b));
    int it = 0;
    if (g1 == 0.0) goto done;
    for (int i = 0; i < n; i++) vc[i] = b[i] / g1;
    double gam = g1, eta = g1, c0 = 1.0, c1 = 1.0, s0 = 0.0, s1 = 0.0;
    for (it = 0; it < maxiter && fabs(eta) > tau * g1; it++) {
        scaled_spmv(n, rp, ci, v, s, vc, t, vn);
        const double del = pdot(n, vn, vc);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) vn[i] -= del * vc[i] + gam * vp[i];
        const double gn = sqrt(pdot(n, vn, vn));
        const double a0 = c1 * del - c0 * s1 * gam;
        const double a1 = sqrt(a0 * a0 + gn * gn);
        const double a2 = s1 * del + c0 * c1 * gam;
        const double a3 = s0 * gam;
        const double cn = a0 / a1, sn = gn / a1;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            const double wn = (vc[i] - a3 * wp[i] - a2 * wc[i]) / a1;
            wp[i] = wc[i];
            wc[i] = wn;
            y[i] += cn * eta * wn;
            vp[i] = vc[i];
            vc[i] = gn > 0.0 ? vn[i] / gn : 0.0;
        }
        eta = -sn * eta;
        gam = gn;
        c0 = c1;
        c1 = cn;
        s0 = s1;
        s1 = sn;
        if (gn == 0.0) {
            it++;
            break;
        }
    }
done:
    free(vp); free(vc); free(vn); free(wp); free(wc); free(t);
    return it;
}

double fo_minres(int n, const int* rp, const int* ci, const double* v, const double* F, double* X,
                 int maxiter, double tol, int* iters)
{
    double* s = (double*)malloc(sizeof(double) * (size_t)n);
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* b = (double*)malloc(sizeof(double) * (size_t)n);
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        double d = 0.0;
        for (int p = rp[i]; p < rp[i + 1]; p++)
            if (ci[p] == i) d = v[p];
        s[i] = d != 0.0 ? 1.0 / sqrt(fabs(d)) : 1.0;
    }
    const double ff = pdot(n, F, F);
    int total = 0;
    double rel = 1.0;
    for (int outer = 0; outer < 30; outer++) {
        fo_spmv(n, rp, ci, v, X, r);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) r[i] = F[i] - r[i];
        const double rr = pdot(n, r, r);
        rel = ff > 0.0 ? sqrt(rr / ff) : sqrt(rr);
        if (rel <= tol || total >= maxiter) break;
        /* the reduction still missing, with some margin; at least 1e-14 */
        double tau = 0.5 * tol / rel;
        if (tau < 1e-14) tau = 1e-14;
        if (tau > 0.5) tau = 0.5;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            b[i] = s[i] * r[i];
            y[i] = 0.0;
        }
        total += minres_scaled(n, rp, ci, v, s, b, y, maxiter - total, tau);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) X[i] += s[i] * y[i];
    }
    if (iters) *iters = total;
    free(s); free(r); free(b); free(y);
    return rel;
}

