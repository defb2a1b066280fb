/* Test infrastructure only: a C-ABI harness around the reference's own C++ code,
 * compiled from the reference sources in place (see oracle/Makefile).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * load the library built from this file; the product path never does.
 *
 * Every function below calls the reference's own member functions in the same
 * order as the reference driver it names, so its outputs ARE the reference's
 * outputs for the given in-memory mesh:
 *   ref_elastic_system  -> FEM/FEM.h:1286-1813 (FEM_forElasticDeformation up to the solve)
 *   ref_elastic_driver  -> FEM/FEM.h:1286-1961 (the whole driver, restart loop included)
 *   ref_scalar_system   -> FEM/FEM.h:398-619  (stiffness-only FEM_forBaseEliptic up to the solve)
 *   ref_scalar_driver   -> FEM/FEM.h:398-717  (the whole driver)
 *   ref_cssd_solve      -> Library/CSSD_Matrix.h solvers on a caller-given CSSD matrix
 *   ref_elastic_local / ref_scalar_local -> FEM/FEM_Grid.h:2125-2192 / :103-152 for one element
 *
 * Matrices are returned as CSR with the diagonal included, each row ordered
 * [A_down columns ascending, diagonal, A_up columns ascending], i.e. exactly the
 * reference's CSSD row split (Library/CSSD_Matrix.h:11-15) laid end to end.
 */
#include "FEM/FEM.h"

#include <cstring>
#include <fcntl.h>
#include <sys/stat.h>

namespace {

struct DirichletMech {
    std::vector<int> id_vertexes;
    std::function<Point<double>(Point<bool>&, int)> value;
};
struct DirichletMech1D { /* edge problems: one constant Point per group (FEM/FEM_Grid.h:3798) */
    std::vector<int> id_vertexes;
    std::function<Point<double>(Point<bool>&)> value;
};
struct NeumannMech {
    std::function<Point<double>(Point<double>)> value;
    std::vector<std::function<Point<double>(Point<double>)>> values;
    std::vector<std::vector<int>> id_vertexes_as_triangle;
    std::vector<int> id_base_element;
};
struct DirichletScal {
    std::vector<int> id_vertexes;
    std::function<double(Point<double>)> value;
};
struct NeumannScal {
    std::function<Point<double>(Point<double>)> value;
    std::vector<std::vector<int>> id_vertexes_as_triangle;
    std::vector<int> id_base_element;
};

int g_quiet = 1;

/* Redirects fd 1 to /dev/null for the lifetime of the object when quiet, and fd 0 from
 * /dev/null always: the reference's drivers wait on scanf_s when a solve reports trouble
 * (FEM/FEM.h:1933-1937, :3782-3786), which must return at once instead of blocking on a
 * caller's open stdin. */
struct StdoutSilencer {
    int saved = -1;
    int saved_in = -1;
    StdoutSilencer() {
        saved_in = dup(0);
        int nin = open("/dev/null", O_RDONLY);
        if (nin >= 0) { dup2(nin, 0); close(nin); }
        if (!g_quiet) return;
        fflush(stdout);
        saved = dup(1);
        int nul = open("/dev/null", O_WRONLY);
        if (nul >= 0) { dup2(nul, 1); close(nul); }
    }
    ~StdoutSilencer() {
        if (saved_in >= 0) { dup2(saved_in, 0); close(saved_in); }
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

double wall_now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* math::SimpleGrid (Library/Math.h:26-33) from arrays; k nodes per element. */
void make_simple_grid_k(math::SimpleGrid& g, int n_nodes, const double* xyz, int n_elems, int k, const int* elems,
                        const int* mat)
{
    g.xyz.resize(n_nodes);
    for (int i = 0; i < n_nodes; i++) g.xyz[i] = Point<double>(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    g.nvtr.resize(n_elems);
    g.nvkat.resize(n_elems);
    for (int e = 0; e < n_elems; e++) {
        g.nvtr[e].assign(elems + (size_t)k * e, elems + (size_t)k * (e + 1));
        g.nvkat[e] = mat ? mat[e] : 0;
    }
}

void make_simple_grid(math::SimpleGrid& g, int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat)
{
    make_simple_grid_k(g, n_nodes, xyz, n_tets, 4, tets, mat);
}

struct CsrOut {
    int n;
    long long nnz;
    int* row_ptr;
    int* col;
    double* val;
    double* F;
    double* X;
};

void cssd_to_csr(CSSD_Matrix<double, double>& A, CsrOut* out)
{
    int n = A.GetMatrixSize();
    long long nnz = 0;
    for (int i = 0; i < n; i++) nnz += 1 + (long long)A.A_up[i].size() + (long long)A.A_down[i].size();
    out->n = n;
    out->nnz = nnz;
    out->row_ptr = (int*)malloc(sizeof(int) * (n + 1));
    out->col = (int*)malloc(sizeof(int) * nnz);
    out->val = (double*)malloc(sizeof(double) * nnz);
    out->F = (double*)malloc(sizeof(double) * n);
    out->X = (double*)malloc(sizeof(double) * n);
    long long p = 0;
    for (int i = 0; i < n; i++) {
        out->row_ptr[i] = (int)p;
        for (size_t j = 0; j < A.A_down[i].size(); j++) { out->col[p] = A.id_column_for_A_down[i][j]; out->val[p++] = A.A_down[i][j]; }
        out->col[p] = i; out->val[p++] = A.Diag[i];
        for (size_t j = 0; j < A.A_up[i].size(); j++) { out->col[p] = A.id_column_for_A_up[i][j]; out->val[p++] = A.A_up[i][j]; }
        out->F[i] = A.F[i];
        out->X[i] = A.X[i];
    }
    out->row_ptr[n] = (int)p;
}

/* Loads a CSR laid out as above back into a CSSD matrix. */
void csr_to_cssd(int n, const int* row_ptr, const int* col, const double* val, const double* F, const double* X,
                 CSSD_Matrix<double, double>& A)
{
    std::vector<std::vector<int>> up(n), down(n);
    for (int i = 0; i < n; i++)
        for (int p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
            if (col[p] < i) down[i].push_back(col[p]);
            else if (col[p] > i) up[i].push_back(col[p]);
        }
    A.Initialization(up, down);
    for (int i = 0; i < n; i++) {
        int pu = 0, pd = 0;
        A.Diag[i] = 0;
        for (int p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
            if (col[p] < i) A.A_down[i][pd++] = val[p];
            else if (col[p] > i) A.A_up[i][pu++] = val[p];
            else A.Diag[i] = val[p];
        }
        A.F[i] = F[i];
        A.X[i] = X[i];
    }
    A.print_logs = false;
    A.log_out = NULL;
}

/* Builds the mech boundary structures the way Solve_ElasticDeformationProblem
 * does (FEM/FEM_Main.cpp:605-900): one Dirichlet type whose value lambda is
 * looked up by node id, and one Neumann type with an individual traction per
 * face and the face's base element. */
void make_mech_boundaries(int n_bc, const int* bc_node, const int* bc_mask, const double* bc_val,
                          int n_faces, const int* face_nodes, const int* face_elem, const double* face_traction,
                          std::vector<DirichletMech>& dir, std::vector<NeumannMech>& neu)
{
    dir.clear();
    neu.clear();
    if (n_bc > 0) {
        typedef std::map<int, std::pair<int, Point<double> > > BcTable;
        BcTable* table = new BcTable(); /* lives as long as the lambda; never freed */
        dir.resize(1);
        for (int i = 0; i < n_bc; i++) {
            dir[0].id_vertexes.push_back(bc_node[i]);
            (*table)[bc_node[i]] = {bc_mask[i], Point<double>(bc_val[3 * i], bc_val[3 * i + 1], bc_val[3 * i + 2])};
        }
        dir[0].value = [table](Point<bool>& take, int id) -> Point<double> {
            auto it = table->find(id);
            take = Point<bool>();
            if (it == table->end()) { take.x = take.y = take.z = false; return Point<double>(0, 0, 0); }
            take.x = (it->second.first & 1) != 0;
            take.y = (it->second.first & 2) != 0;
            take.z = (it->second.first & 4) != 0;
            return it->second.second;
        };
    }
    if (n_faces > 0) {
        neu.resize(1);
        neu[0].value = [](Point<double>) { return Point<double>(0, 0, 0); };
        for (int f = 0; f < n_faces; f++) {
            neu[0].id_vertexes_as_triangle.push_back({face_nodes[3 * f], face_nodes[3 * f + 1], face_nodes[3 * f + 2]});
            neu[0].id_base_element.push_back(face_elem[f]);
            Point<double> t(face_traction[3 * f], face_traction[3 * f + 1], face_traction[3 * f + 2]);
            neu[0].values.push_back([t](Point<double>) { return t; });
        }
    }
}

/* Groups Dirichlet nodes by value (one reference "type" per distinct value, in
 * order of first appearance), the way the reference's param files group them. */
void make_scal_boundaries(int n_bc, const int* bc_node, const double* bc_val, std::vector<DirichletScal>& dir)
{
    dir.clear();
    std::vector<double> values;
    for (int i = 0; i < n_bc; i++) {
        size_t t = 0;
        while (t < values.size() && values[t] != bc_val[i]) t++;
        if (t == values.size()) {
            values.push_back(bc_val[i]);
            dir.emplace_back();
            double v = bc_val[i];
            dir.back().value = [v](Point<double>) { return v; };
        }
        dir[t].id_vertexes.push_back(bc_node[i]);
    }
}

template <class Grid>
void set_materials_mech(Grid& grid, int n_mat, const double* E, const double* nu)
{
    for (int m = 0; m < n_mat; m++) {
        grid.AddDomain();
        grid.GetDomain(m)->forMech.SetE(E[m]);
        grid.GetDomain(m)->forMech.SetV(nu[m]);
    }
}

char* make_tmpdir()
{
    char* tmpl = strdup("/tmp/msfem_ref_XXXXXX");
    if (!mkdtemp(tmpl)) { free(tmpl); return nullptr; }
    return tmpl;
}

}  // namespace

extern "C" {

typedef CsrOut ref_csr;

void ref_set_quiet(int q) { g_quiet = q; }
void ref_free(void* p) { free(p); }
void ref_free_csr(ref_csr* c)
{
    if (!c) return;
    free(c->row_ptr); free(c->col); free(c->val); free(c->F); free(c->X);
    c->row_ptr = nullptr; c->col = nullptr; c->val = nullptr; c->F = nullptr; c->X = nullptr;
}

/* One element's 4x4 blocks of 3x3, FEM/FEM_Grid.h:2125-2192 through the
 * reference's own Grid_forMech on a one-tet mesh.  K[((I*4+J)*3+a)*3+b] = A[I][J].val[a][b]. */
int ref_elastic_local(const double* xyz4, double E, double nu, double* K)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    int tet[4] = {0, 1, 2, 3};
    make_simple_grid(g, 4, xyz4, 1, tet, nullptr);
    std::vector<DirichletMech> d;
    std::vector<NeumannMech> nb;
    auto* grid = new FEM::Grid_forMech();
    set_materials_mech(*grid, 1, &E, &nu);
    grid->Initialization(g, d, nb);
    DenseMatrix<Tensor2Rank3D, Point<double>> local;
    std::function<std::vector<std::vector<double>>(Point<double>)> kD = [&](Point<double>) {
        return grid->GetDomain(0)->forMech.GetD(3);
    };
    grid->GetElement(0)->SolveLocalMatrix(local, kD);
    for (int I = 0; I < 4; I++)
        for (int J = 0; J < 4; J++)
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) K[((I * 4 + J) * 3 + a) * 3 + b] = local.A[I][J].val[a][b];
    return 0; /* grid intentionally leaked: the reference's destructor chain is not exercised */
}

/* One element's 4x4 scalar stiffness, FEM/FEM_Grid.h:103-152 (1-point rule). */
int ref_scalar_local(const double* xyz4, double sigma, double* K)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    int tet[4] = {0, 1, 2, 3};
    make_simple_grid(g, 4, xyz4, 1, tet, nullptr);
    std::vector<DirichletScal> d;
    std::vector<NeumannScal> nb;
    auto* grid = new FEM::Grid_forScal();
    grid->Initialization(g, d, nb);
    DenseMatrix<double, double> local;
    std::function<double(int, Point<double>)> k = [sigma](int, Point<double>) { return sigma; };
    grid->GetElement(0)->SolveLocalMatrix(local, k);
    for (int I = 0; I < 4; I++)
        for (int J = 0; J < 4; J++) K[I * 4 + J] = local.A[I][J];
    return 0;
}

/* FiniteElement_forScal::SolveLocalMatrix with stiffness, mass and source coefficients
 * (FEM/FEM_Grid.h:25-102, the one-point rule): K[16] = K + M of the element, F[4] its load, for the
 * constant coefficients S, Mc, f. */
int ref_scalar3_local(const double* xyz4, double S, double Mc, double f, double* K, double* F)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    int tet[4] = {0, 1, 2, 3};
    make_simple_grid(g, 4, xyz4, 1, tet, nullptr);
    std::vector<DirichletScal> d;
    std::vector<NeumannScal> nb;
    auto* grid = new FEM::Grid_forScal();
    grid->Initialization(g, d, nb);
    DenseMatrix<double, double> local;
    std::function<double(int, Point<double>)> ks = [S](int, Point<double>) { return S; };
    std::function<double(int, Point<double>)> km = [Mc](int, Point<double>) { return Mc; };
    std::function<double(int, Point<double>)> kf = [f](int, Point<double>) { return f; };
    grid->GetElement(0)->SolveLocalMatrix(local, ks, km, kf);
    for (int I = 0; I < 4; I++) {
        F[I] = local.F[I];
        for (int J = 0; J < 4; J++) K[I * 4 + J] = local.A[I][J];
    }
    return 0;
}

/* The three-coefficient scalar driver FEM_forBaseEliptic (FEM/FEM.h:206-397): K + M + F per element
 * with per-element coefficients S[e], Mc[e], f[e], Dirichlet rows only, BiCG_Stab restarts to
 * min_residual; solution: n_nodes doubles. */
int ref_scalar3_driver(int n_nodes, const double* xyz, int n_tets, const int* tets, const double* S,
                       const double* Mc, const double* f, int n_bc, const int* bc_node, const double* bc_val,
                       double min_residual, double* solution)
{
    StdoutSilencer s;
    math::NUM_THREADS = 1;
    auto* g = new math::SimpleGrid();
    make_simple_grid(*g, n_nodes, xyz, n_tets, tets, nullptr);
    auto* dir = new std::vector<DirichletScal>();
    auto* neu = new std::vector<NeumannScal>();
    make_scal_boundaries(n_bc, bc_node, bc_val, *dir);
    auto* vs = new std::vector<double>(S, S + n_tets);
    auto* vm = new std::vector<double>(Mc, Mc + n_tets);
    auto* vf = new std::vector<double>(f, f + n_tets);
    auto* ks = new std::function<double(int, Point<double>)>([vs](int e, Point<double>) { return (*vs)[e]; });
    auto* km = new std::function<double(int, Point<double>)>([vm](int e, Point<double>) { return (*vm)[e]; });
    auto* kf = new std::function<double(int, Point<double>)>([vf](int e, Point<double>) { return (*vf)[e]; });
    auto* grid = new FEM::Grid_forScal();
    auto* sol = new std::vector<double>();
    char* dirname = make_tmpdir();
    if (!dirname) return -1;
    FEM::FEM_forBaseEliptic(false, min_residual, *g, *dir, *neu, *ks, *km, *kf, dirname, *grid, *sol);
    if ((int)sol->size() != n_nodes) return -3;
    for (int i = 0; i < n_nodes; i++) solution[i] = (*sol)[i];
    std::string cmd = std::string("rm -rf ") + dirname;
    if (system(cmd.c_str()) != 0) { }
    free(dirname);
    return 0;
}

/* FEM_forElasticDeformation (FEM/FEM.h:1286-1813) up to the solve.
 * stage 0: the expanded scalar matrix before any boundary condition (FEM.h:1673-1674);
 * stage 1: after the Dirichlet rows and the column sweep (FEM.h:1676-1813).
 * t_out[0] = wall seconds of init+portrait+traction+elements+scatter, t_out[1] = expand+BCs. */
int ref_elastic_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                       int n_mat, const double* E, const double* nu,
                       int n_bc, const int* bc_node, const int* bc_mask, const double* bc_val,
                       int n_faces, const int* face_nodes, const int* face_elem, const double* face_traction,
                       int nthreads, int stage, ref_csr* out, double* t_out)
{
    StdoutSilencer s;
    math::NUM_THREADS = nthreads > 0 ? nthreads : 1;
    math::SimpleGrid g;
    make_simple_grid(g, n_nodes, xyz, n_tets, tets, mat);
    std::vector<DirichletMech> dir;
    std::vector<NeumannMech> neu;
    make_mech_boundaries(n_bc, bc_node, bc_mask, bc_val, n_faces, face_nodes, face_elem, face_traction, dir, neu);

    double t0 = wall_now();
    auto* gridp = new FEM::Grid_forMech();
    FEM::Grid_forMech& solver_grid = *gridp;
    set_materials_mech(solver_grid, n_mat, E, nu);
    solver_grid.Initialization(g, dir, neu);

    auto* gsp = new CSSD_Matrix<Tensor2Rank3D, Point<double>>();
    auto& global_SLAE = *gsp;
    solver_grid.CreationPortrait(global_SLAE);
    for (size_t f = 0; f < solver_grid.boundary_faces.size(); f++) {
        std::vector<Point<double>> lv;
        solver_grid.boundary_faces[f].SolveLocalBoundaryVector(lv, solver_grid.boundary_faces[f].boundary_value);
        global_SLAE.SummPartOfVector(lv, *solver_grid.boundary_faces[f].GetElementDOFs());
    }
    {
        std::vector<DenseMatrix<Tensor2Rank3D, Point<double>>> local_SLAE(solver_grid.GetElementsCount());
        omp_set_num_threads(math::NUM_THREADS);
#pragma omp parallel for schedule(dynamic)
        for (int id_elem = 0; id_elem < solver_grid.GetElementsCount(); id_elem++) {
            auto element = solver_grid.GetElement(id_elem);
            if (solver_grid.GetDomain(element->GetIdDomain())->forMech.GetE(0) <= 0) {
                local_SLAE[id_elem].SetSize(element->GetDOFsCount());
            } else {
                std::function<std::vector<std::vector<double>>(Point<double>)> koefD = [&](Point<double>) {
                    return (solver_grid.GetDomain(element->GetIdDomain()))->forMech.GetD(3);
                };
                element->SolveLocalMatrix(local_SLAE[id_elem], koefD);
            }
        }
        for (int id_elem = 0; id_elem < solver_grid.GetElementsCount(); id_elem++)
            global_SLAE.SummPartOfMatrix(local_SLAE[id_elem], *solver_grid.GetElementDOFs(id_elem));
    }
    double t1 = wall_now();
    auto* nsp = new CSSD_Matrix<double, double>();
    auto& newSLAE = *nsp;
    math::MakeCopyMatrix_A_into_B(global_SLAE, newSLAE);
    if (stage >= 1) {
        std::vector<int> use_id;
        for (size_t id_vertex = 0; id_vertex < solver_grid.boundary_vertexes.size(); id_vertex++) {
            auto boundary = &(solver_grid.boundary_vertexes[id_vertex]);
            Point<bool> is_take;
            Point<double> bv = boundary->boundary_value(is_take, solver_grid.boundary_vertexes[id_vertex].GetIdNode(0));
            int global_id = boundary->GetDOFInLocalID(0);
            if (global_id < global_SLAE.GetMatrixSize()) {
                auto enter_value = [&newSLAE, &use_id](int value_id, double value) {
                    use_id.push_back(value_id);
                    newSLAE.X[value_id] = value;
                    newSLAE.F[value_id] = value;
                    newSLAE.Diag[value_id] = 1;
                    for (size_t i = 0; i < newSLAE.A_down[value_id].size(); i++) newSLAE.A_down[value_id][i] = 0;
                    for (size_t i = 0; i < newSLAE.A_up[value_id].size(); i++) newSLAE.A_up[value_id][i] = 0;
                };
                if (is_take.x) enter_value(global_id * 3 + 0, bv.x);
                if (is_take.y) enter_value(global_id * 3 + 1, bv.y);
                if (is_take.z) enter_value(global_id * 3 + 2, bv.z);
            }
        }
        /* column sweep, FEM/FEM.h:1757-1812 (same shared-iterator walk) */
#pragma omp parallel for schedule(dynamic)
        for (int id_row = 0; id_row < newSLAE.GetMatrixSize(); id_row++) {
            size_t it = 0;
            for (size_t jj = 0; jj < newSLAE.id_column_for_A_up[id_row].size(); jj++) {
                int c = newSLAE.id_column_for_A_up[id_row][jj];
                for (; it < use_id.size(); it++) {
                    if (use_id[it] == c) { newSLAE.F[id_row] -= newSLAE.A_up[id_row][jj] * newSLAE.F[c]; newSLAE.A_up[id_row][jj] = 0; break; }
                    if (use_id[it] > c) break;
                }
            }
            it = 0;
            for (size_t jj = 0; jj < newSLAE.id_column_for_A_down[id_row].size(); jj++) {
                int c = newSLAE.id_column_for_A_down[id_row][jj];
                for (; it < use_id.size(); it++) {
                    if (use_id[it] == c) { newSLAE.F[id_row] -= newSLAE.A_down[id_row][jj] * newSLAE.F[c]; newSLAE.A_down[id_row][jj] = 0; break; }
                    if (use_id[it] > c) break;
                }
            }
        }
    }
    double t2 = wall_now();
    cssd_to_csr(newSLAE, out);
    if (t_out) { t_out[0] = t1 - t0; t_out[1] = t2 - t1; }
    return 0; /* objects leaked on purpose: see ref_elastic_driver */
}

/* The whole FEM_forElasticDeformation driver (FEM/FEM.h:1286-1961), restart loop
 * and SSOR(0.75)-PCG included.  solution: 3*n_nodes doubles (node-major).
 * The driver writes Solution_residual_*.txt into a fresh temp directory, which
 * is removed afterwards.  The grid is leaked because the reference's destructor
 * chain aborts after the solution exists. */
int ref_elastic_driver(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                       int n_mat, const double* E, const double* nu,
                       int n_bc, const int* bc_node, const int* bc_mask, const double* bc_val,
                       int n_faces, const int* face_nodes, const int* face_elem, const double* face_traction,
                       int nthreads, double min_residual, double* solution, double* wall_seconds)
{
    StdoutSilencer s;
    math::NUM_THREADS = nthreads > 0 ? nthreads : 1;
    math::SimpleGrid* g = new math::SimpleGrid();
    make_simple_grid(*g, n_nodes, xyz, n_tets, tets, mat);
    auto* dir = new std::vector<DirichletMech>();
    auto* neu = new std::vector<NeumannMech>();
    make_mech_boundaries(n_bc, bc_node, bc_mask, bc_val, n_faces, face_nodes, face_elem, face_traction, *dir, *neu);
    auto* grid = new FEM::Grid_forMech();
    set_materials_mech(*grid, n_mat, E, nu);
    auto* sol = new std::vector<Point<double>>();
    char* dirname = make_tmpdir();
    if (!dirname) return -1;
    double t0 = wall_now();
    FEM::FEM_forElasticDeformation(false, min_residual, *g, *dir, *neu, dirname, *grid, *sol);
    double t1 = wall_now();
    /* the driver copies the scalar newSLAE.X (3n doubles) into n Points (Library/Math.h:1741) */
    if ((int)sol->size() != n_nodes) return -3;
    for (int i = 0; i < n_nodes; i++) { solution[3 * i] = (*sol)[i].x; solution[3 * i + 1] = (*sol)[i].y; solution[3 * i + 2] = (*sol)[i].z; }
    if (wall_seconds) *wall_seconds = t1 - t0;
    std::string cmd = std::string("rm -rf ") + dirname;
    if (system(cmd.c_str()) != 0) { /* best effort */ }
    free(dirname);
    return 0;
}

/* Stiffness-only FEM_forBaseEliptic (FEM/FEM.h:398-619) up to the solve.
 * stage 0: assembled matrix, no BCs; stage 1: after Dirichlet rows + column sweep,
 * with X = F as the driver sets it before the solve (FEM.h:635). */
int ref_scalar_system(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                      int n_mat, const double* sigma, int n_bc, const int* bc_node, const double* bc_val,
                      int nthreads, int stage, ref_csr* out, double* t_out)
{
    StdoutSilencer s;
    math::NUM_THREADS = nthreads > 0 ? nthreads : 1;
    math::SimpleGrid g;
    make_simple_grid(g, n_nodes, xyz, n_tets, tets, mat);
    std::vector<DirichletScal> dir;
    std::vector<NeumannScal> neu;
    make_scal_boundaries(n_bc, bc_node, bc_val, dir);
    std::vector<double> sig(sigma, sigma + n_mat);

    double t0 = wall_now();
    auto* gridp = new FEM::Grid_forScal();
    FEM::Grid_forScal& solver_grid = *gridp;
    solver_grid.Initialization(g, dir, neu);
    std::function<double(int, Point<double>)> koef = [&](int elem, Point<double>) {
        return sig[solver_grid.GetElement(elem)->GetIdDomain()];
    };
    auto* gsp = new CSSD_Matrix<double, double>();
    auto& global_SLAE = *gsp;
    solver_grid.CreationPortrait(global_SLAE);
    {
        std::vector<DenseMatrix<double, double>> local_SLAE(solver_grid.GetElementsCount());
        omp_set_num_threads(math::NUM_THREADS);
#pragma omp parallel for schedule(dynamic)
        for (int id_elem = 0; id_elem < solver_grid.GetElementsCount(); id_elem++)
            solver_grid.GetElement(id_elem)->SolveLocalMatrix(local_SLAE[id_elem], koef);
        for (int id_elem = 0; id_elem < solver_grid.GetElementsCount(); id_elem++)
            global_SLAE.SummPartOfMatrix(local_SLAE[id_elem], *solver_grid.GetElementDOFs(id_elem));
    }
    double t1 = wall_now();
    if (stage >= 1) {
        for (size_t id_vertex = 0; id_vertex < solver_grid.boundary_vertexes.size(); id_vertex++) {
            auto boundary = &(solver_grid.boundary_vertexes[id_vertex]);
            int global_id = boundary->GetDOFInLocalID(0);
            Point<double> x = solver_grid.GetCoordinateViaID(global_id);
            double bv = boundary->boundary_value(x);
            global_SLAE.X[global_id] = bv;
            global_SLAE.F[global_id] = bv;
            global_SLAE.Diag[global_id] = 1.0;
            for (size_t j = 0; j < global_SLAE.A_down[global_id].size(); j++) global_SLAE.A_down[global_id][j] = 0.0;
            for (size_t j = 0; j < global_SLAE.A_up[global_id].size(); j++) global_SLAE.A_up[global_id][j] = 0.0;
        }
        auto& bvs = solver_grid.boundary_vertexes;
#pragma omp parallel for
        for (int id_row = 0; id_row < global_SLAE.GetMatrixSize(); id_row++) {
            size_t it = 0;
            for (size_t jj = 0; jj < global_SLAE.id_column_for_A_up[id_row].size(); jj++) {
                int c = global_SLAE.id_column_for_A_up[id_row][jj];
                for (; it < bvs.size(); it++) {
                    if (bvs[it].GetDOFInLocalID(0) == c) { global_SLAE.F[id_row] -= global_SLAE.A_up[id_row][jj] * global_SLAE.F[c]; global_SLAE.A_up[id_row][jj] = 0; break; }
                    if (bvs[it].GetDOFInLocalID(0) > c) break;
                }
            }
            it = 0;
            for (size_t jj = 0; jj < global_SLAE.id_column_for_A_down[id_row].size(); jj++) {
                int c = global_SLAE.id_column_for_A_down[id_row][jj];
                for (; it < bvs.size(); it++) {
                    if (bvs[it].GetDOFInLocalID(0) == c) { global_SLAE.F[id_row] -= global_SLAE.A_down[id_row][jj] * global_SLAE.F[c]; global_SLAE.A_down[id_row][jj] = 0; break; }
                    if (bvs[it].GetDOFInLocalID(0) > c) break;
                }
            }
        }
        math::MakeCopyVector_A_into_B(global_SLAE.F, global_SLAE.X);
    }
    double t2 = wall_now();
    cssd_to_csr(global_SLAE, out);
    if (t_out) { t_out[0] = t1 - t0; t_out[1] = t2 - t1; }
    return 0;
}

/* The whole stiffness-only FEM_forBaseEliptic driver (FEM/FEM.h:398-717). */
int ref_scalar_driver(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat,
                      int n_mat, const double* sigma, int n_bc, const int* bc_node, const double* bc_val,
                      int nthreads, double min_residual, double* solution, double* wall_seconds)
{
    StdoutSilencer s;
    math::NUM_THREADS = nthreads > 0 ? nthreads : 1;
    auto* g = new math::SimpleGrid();
    make_simple_grid(*g, n_nodes, xyz, n_tets, tets, mat);
    auto* dir = new std::vector<DirichletScal>();
    auto* neu = new std::vector<NeumannScal>();
    make_scal_boundaries(n_bc, bc_node, bc_val, *dir);
    auto* sig = new std::vector<double>(sigma, sigma + n_mat);
    auto* grid = new FEM::Grid_forScal();
    auto* koef = new std::function<double(int, Point<double>)>([grid, sig](int elem, Point<double>) {
        return (*sig)[grid->GetElement(elem)->GetIdDomain()];
    });
    auto* sol = new std::vector<double>();
    char* dirname = make_tmpdir();
    if (!dirname) return -1;
    double t0 = wall_now();
    FEM::FEM_forBaseEliptic(false, min_residual, *g, *dir, *neu, *koef, dirname, *grid, *sol);
    double t1 = wall_now();
    if ((int)sol->size() != n_nodes) return -3;
    for (int i = 0; i < n_nodes; i++) solution[i] = (*sol)[i];
    if (wall_seconds) *wall_seconds = t1 - t0;
    std::string cmd = std::string("rm -rf ") + dirname;
    if (system(cmd.c_str()) != 0) { }
    free(dirname);
    return 0;
}

/* Runs one of the reference's CSSD solvers on a caller-given matrix.
 * method 0: MSG (plain CG, CSSD_Matrix.h:1496)          maxiter as given
 * method 1: MSG_PreconditioningSSOR with PrecondorSSOR(0.75) (CSSD_Matrix.h:1302, :458)
 * method 2: BiCG_Stab (CSSD_Matrix.h:730)
 * method 3: BCG_Stab2 (CSSD_Matrix.h:634)
 * method 4: GMRES (CSSD_Matrix.h:1774; GMRES(5), rows normalised in place)
 * X holds the initial guess on entry and the result on exit; the solver's
 * return value (true relative residual, sign as the reference returns it) goes
 * to *residual. */
int ref_cssd_solve(int method, int n, const int* row_ptr, const int* col, const double* val, const double* F,
                   double* X, int maxiter, double tol, int nthreads, double* residual, double* wall_seconds)
{
    StdoutSilencer s;
    math::NUM_THREADS = nthreads > 0 ? nthreads : 1;
    auto* A = new CSSD_Matrix<double, double>();
    csr_to_cssd(n, row_ptr, col, val, F, X, *A);
    double t0 = wall_now();
    double r = 0;
    switch (method) {
    case 0: r = A->MSG(maxiter, tol); break;
    case 1: {
        auto* P = new CSSD_Matrix<double, double>();
        P->PrecondorSSOR(0.75, *A);
        r = A->MSG_PreconditioningSSOR(maxiter, tol, *P);
        break;
    }
    case 2: r = A->BiCG_Stab(maxiter, tol); break;
    case 3: r = A->BCG_Stab2(maxiter, tol); break;
    case 4: r = A->GMRES(maxiter, tol); break;
    default: return -1;
    }
    double t1 = wall_now();
    for (int i = 0; i < n; i++) X[i] = A->X[i];
    if (residual) *residual = r;
    if (wall_seconds) *wall_seconds = t1 - t0;
    return 0;
}

/* SSOR preconditioner application z = M^{-1} r with the reference's
 * PrecondorSSOR(w)/SolvePrecondorSSOR_SLAE (CSSD_Matrix.h:458-547). */
int ref_ssor_apply(int n, const int* row_ptr, const int* col, const double* val, double w, const double* r, double* z)
{
    StdoutSilencer s;
    std::vector<double> F(n, 0.0), X(n, 0.0);
    auto* A = new CSSD_Matrix<double, double>();
    csr_to_cssd(n, row_ptr, col, val, F.data(), X.data(), *A);
    auto* P = new CSSD_Matrix<double, double>();
    P->PrecondorSSOR(w, *A);
    std::vector<double> rr(r, r + n), zz;
    P->SolvePrecondorSSOR_SLAE(A->Diag, zz, rr);
    for (int i = 0; i < n; i++) z[i] = zz[i];
    return 0;
}


/* One MsFEM cell sub-problem through the reference's own drivers, the calls
 * MsFEM/MsFEM_Grid.h:5119-5176 (edges), :5312 (faces) and :5495 (volume) make:
 *   dim 1 -> FEM::FEM_1D_forElasticDeformation (FEM/FEM.h:3796), segments
 *   dim 2 -> FEM::FEM_2D_forElasticDeformation (FEM/FEM.h:4367), triangles
 *   dim 3 -> FEM::FEM_3D_forElasticDeformation (FEM/FEM.h:2970), tetrahedra
 * elems: (dim+1) node ids per element; Dirichlet: all three components of every
 * listed node take bc_val[3i..3i+2] (the cell drivers fix whole Points); zero
 * source, no traction.  solution: 3*n_nodes doubles, node-major. */
int ref_cell_problem(int dim, int n_nodes, const double* xyz, int n_elems, const int* elems, const int* mat,
                     int n_mat, const double* E, const double* nu, int n_bc, const int* bc_node, const double* bc_val,
                     double min_residual, double* solution)
{
    StdoutSilencer s;
    math::NUM_THREADS = 1;
    auto* g = new math::SimpleGrid();
    make_simple_grid_k(*g, n_nodes, xyz, n_elems, dim + 1, elems, mat);
    auto* dir = new std::vector<DirichletMech>();
    auto* neu = new std::vector<NeumannMech>();
    std::vector<int> mask(n_bc, 7);
    make_mech_boundaries(n_bc, bc_node, mask.data(), bc_val, 0, nullptr, nullptr, nullptr, *dir, *neu);
    std::function<Point<double>(bool&, int, Point<double>)> source = [](bool& is_solve, int, Point<double>) {
        is_solve = false;
        return Point<double>(0, 0, 0);
    };
    auto* sol = new std::vector<Point<double>>();
    auto* K = new CSSD_Matrix<Tensor2Rank3D, Point<double>>();
    char* dirname = make_tmpdir();
    if (!dirname) return -1;
    if (dim == 1) {
        /* one group per node, as MsFEM_Grid.h:5061-5100 builds the two edge ends */
        auto* dir1 = new std::vector<DirichletMech1D>(n_bc);
        for (int i = 0; i < n_bc; i++) {
            (*dir1)[i].id_vertexes.push_back(bc_node[i]);
            Point<double> v(bc_val[3 * i], bc_val[3 * i + 1], bc_val[3 * i + 2]);
            (*dir1)[i].value = [v](Point<bool>& take) {
                take.x = take.y = take.z = true;
                return v;
            };
        }
        auto* grid = new FEM::Grid_1D_forMech();
        set_materials_mech(*grid, n_mat, E, nu);
        FEM::FEM_1D_forElasticDeformation(false, min_residual, *g, *dir1, *neu, source, dirname, *grid, *sol, *K);
    } else if (dim == 2) {
        auto* grid = new FEM::Grid_2D_forMech();
        set_materials_mech(*grid, n_mat, E, nu);
        FEM::FEM_2D_forElasticDeformation(false, min_residual, *g, *dir, *neu, source, dirname, *grid, *sol, *K);
    } else if (dim == 3) {
        auto* grid = new FEM::Grid_forMech();
        set_materials_mech(*grid, n_mat, E, nu);
        FEM::FEM_3D_forElasticDeformation(false, min_residual, *g, *dir, *neu, source, dirname, *grid, *sol, *K);
    } else {
        return -2;
    }
    std::string cmd = std::string("rm -rf ") + dirname;
    if (system(cmd.c_str()) != 0) { /* best effort */ }
    free(dirname);
    if ((int)sol->size() != n_nodes) return -3;
    for (int i = 0; i < n_nodes; i++) {
        solution[3 * i] = (*sol)[i].x;
        solution[3 * i + 1] = (*sol)[i].y;
        solution[3 * i + 2] = (*sol)[i].z;
    }
    return 0; /* objects leaked on purpose, as in ref_elastic_driver */
}


/* The quadrature of an MsFEM macro element (geometry::Polyhedron::CreateSubMeshInSelf and
 * SetIntegrationLaw, Library/GeometryShape.h:2708-2760, :2820-2836): the sub-tetrahedra
 * (centroid, face centroid, edge of the face) over every face, each with the tetrahedron's
 * 4-point rule (:1754-1851).  xyz8: the 8 vertices; faces: 6 cycles of 4 local vertex ids.
 * points: 3 * 96 doubles, weights: 96 doubles (faces in order, edges in order, rule points in
 * order). */
int ref_poly_quadrature(const double* xyz8, const int* faces, double* points, double* weights)
{
    StdoutSilencer s;
    auto* P = new std::vector<Point<double>>(8);
    std::vector<Point<double>*> ptr(8);
    for (int i = 0; i < 8; i++) {
        (*P)[i] = Point<double>(xyz8[3 * i], xyz8[3 * i + 1], xyz8[3 * i + 2]);
        ptr[i] = &(*P)[i];
    }
    std::vector<int> ids(8);
    for (int i = 0; i < 8; i++) ids[i] = i;
    std::vector<std::vector<int>> fc(6, std::vector<int>(4));
    for (int f = 0; f < 6; f++)
        for (int k = 0; k < 4; k++) fc[f][k] = faces[4 * f + k];
    auto* poly = new geometry::Polyhedron();
    poly->SetGeometry(ids, fc, ptr);
    poly->SetIntegrationLaw(4);
    const int n = (int)poly->GetIntegrationPointsCount();
    if (n != 96) return -2;
    for (int q = 0; q < n; q++) {
        Point<double> x = poly->GetIntegrationPoint(q);
        points[3 * q] = x.x;
        points[3 * q + 1] = x.y;
        points[3 * q + 2] = x.z;
        weights[q] = poly->GetIntegrationWeight(q);
    }
    return 0; /* objects leaked on purpose (the nodes must outlive the polyhedron) */
}

/* geometry::Polygon over the 4 given vertices (GeometryShape.h:2541-2640: centroid fan of
   triangles, SetIntegrationLaw(4)): the 16 points and weights of the macro face loads. */
int ref_polygon_quadrature(const double* xyz4, double* points, double* weights)
{
    StdoutSilencer s;
    auto* P = new std::vector<Point<double>>(4);
    std::vector<Point<double>*> ptr(4);
    for (int i = 0; i < 4; i++) {
        (*P)[i] = Point<double>(xyz4[3 * i], xyz4[3 * i + 1], xyz4[3 * i + 2]);
        ptr[i] = &(*P)[i];
    }
    std::vector<int> ids = {0, 1, 2, 3};
    auto* poly = new geometry::Polygon();
    poly->SetGeometry(ids, ptr);
    poly->SetIntegrationLaw(4);
    const int n = (int)poly->GetIntegrationPointsCount();
    if (n != 16) return -2;
    for (int q = 0; q < n; q++) {
        Point<double> x = poly->GetIntegrationPoint(q);
        points[3 * q] = x.x;
        points[3 * q + 1] = x.y;
        points[3 * q + 2] = x.z;
        weights[q] = poly->GetIntegrationWeight(q);
    }
    return 0; /* objects leaked on purpose, as above */
}

/* math::SimpleGrid::ReadFromNVTR (Library/Math.h:150-291) on a directory: the reference's own
   reader.  k = nodes per element (4) or -1 (polyhedra, flattened as the file holds them).
   Outputs are truncated to the given capacities; counts and read_from_zero are always set. */
int ref_read_nvtr(const char* dir, int k, int cap_v, int cap_e, int cap_idx, int* n_vert, int* n_elem, int* n_idx,
                  double* xyz, int* idx, int* elem_len, int* nvkat, int* read_from_zero)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    std::vector<char> d(dir, dir + std::strlen(dir) + 1);
    if (!g.ReadFromNVTR(d.data(), k)) return -2;
    *n_vert = (int)g.xyz.size();
    *n_elem = (int)g.nvtr.size();
    *read_from_zero = g.read_from_zero ? 1 : 0;
    for (int i = 0; i < *n_vert && i < cap_v; i++) {
        xyz[3 * i] = g.xyz[i].x;
        xyz[3 * i + 1] = g.xyz[i].y;
        xyz[3 * i + 2] = g.xyz[i].z;
    }
    int t = 0;
    for (int e = 0; e < *n_elem; e++) {
        if (e < cap_e) {
            elem_len[e] = (int)g.nvtr[e].size();
            nvkat[e] = g.nvkat[e];
        }
        for (int v : g.nvtr[e]) {
            if (t < cap_idx) idx[t] = v;
            t++;
        }
    }
    *n_idx = t;
    return 0;
}

/* math::SimpleGrid::ReadFromSalomeDat (Library/Math.h:35-149), the map_size variant when
   map_size >= 0: vertex_map[i] = id - 1. */
int ref_read_salome(const char* file, int dim, int map_size, int cap_v, int cap_e, int* n_vert, int* n_elem, double* xyz,
                    int* elems, int* vmap)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    std::vector<char> f(file, file + std::strlen(file) + 1);
    const bool ok = map_size >= 0 ? g.ReadFromSalomeDat(f.data(), dim, map_size) : g.ReadFromSalomeDat(f.data(), dim);
    if (!ok) return -2;
    *n_vert = (int)g.xyz.size();
    *n_elem = (int)g.nvtr.size();
    for (int i = 0; i < *n_vert && i < cap_v; i++) {
        xyz[3 * i] = g.xyz[i].x;
        xyz[3 * i + 1] = g.xyz[i].y;
        xyz[3 * i + 2] = g.xyz[i].z;
        if (map_size >= 0) vmap[i] = g.vertex_map[i];
    }
    for (int e = 0; e < *n_elem && e < cap_e; e++)
        for (int j = 0; j <= dim; j++) elems[(dim + 1) * e + j] = g.nvtr[e][j];
    return 0;
}

/* The reference grid's post-processing at each element's centroid (FEM/FEM_Grid.h:3289-3365):
   GetSolutionInPoint, GetDerevativeFromSolutionInPoint, GetStressTensorFromSolutionInPoint (the
   element's own material through Domain::forMech::solve_SIGMA) and GetVonMisesStress.
   solution: [n_nodes][3]; out: [n_tets][19] = U(3), dU(9: row a = grad u_a), sigma (xx yy zz yz
   xz xy), von Mises. */
int ref_postprocess(int n_nodes, const double* xyz, int n_tets, const int* tets, const int* mat, int n_mat,
                    const double* E, const double* nu, const double* solution, double* out)
{
    StdoutSilencer s;
    math::SimpleGrid g;
    make_simple_grid(g, n_nodes, xyz, n_tets, tets, mat);
    std::vector<DirichletMech> dir;
    std::vector<NeumannMech> neu;
    auto* gridp = new FEM::Grid_forMech();
    FEM::Grid_forMech& grid = *gridp;
    set_materials_mech(grid, n_mat, E, nu);
    grid.Initialization(g, dir, neu);
    std::vector<Point<double>> sol(n_nodes);
    for (int i = 0; i < n_nodes; i++) sol[i] = Point<double>(solution[3 * i], solution[3 * i + 1], solution[3 * i + 2]);
    for (int e = 0; e < grid.GetElementsCount(); e++) {
        auto element = grid.GetElement(e);
        Point<double> X = element->GetWeightCentr();
        Point<double> U = grid.GetSolutionInPoint(e, X, sol);
        Point<Point<double>> dU = grid.GetDerevativeFromSolutionInPoint(e, X, sol);
        Tensor2Rank3D S = grid.GetStressTensorFromSolutionInPoint(e, X, dU);
        double* o = out + 19 * (size_t)e;
        o[0] = U.x; o[1] = U.y; o[2] = U.z;
        const Point<double> rows[3] = {dU.x, dU.y, dU.z};
        for (int a = 0; a < 3; a++) {
            o[3 + 3 * a] = rows[a].x;
            o[4 + 3 * a] = rows[a].y;
            o[5 + 3 * a] = rows[a].z;
        }
        o[12] = S.val[0][0]; o[13] = S.val[1][1]; o[14] = S.val[2][2];
        o[15] = S.val[1][2]; o[16] = S.val[0][2]; o[17] = S.val[0][1];
        o[18] = grid.GetVonMisesStress(S);
    }
    return 0; /* grid leaked on purpose, as the other entry points do */
}

/* Domain::forMech::GetD(3) (Library/Domain.h:170-175, isotropic D of :53-78) as 36 doubles. */
int ref_mech_D(double E, double nu, double* D)
{
    StdoutSilencer s;
    auto* d = new Domain();
    d->forMech.SetE(E);
    d->forMech.SetV(nu);
    auto m = d->forMech.GetD(3);
    if (m.size() != 6) return -2;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) D[6 * i + j] = m[i][j];
    return 0;
}

}  // extern "C"
