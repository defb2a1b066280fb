// C++ host drivers: the reference's FEM driver sequences, step for step, with
// every step handed to the C ABI (include/msfem_b200.h).  Only the public ABI
// is used here, exactly as a caller inside the reference would use it.
#include <cstring>
#include <vector>

#include "msfem_b200.h"

namespace {

struct Handle {
    msfem_system_t h = nullptr;
    ~Handle() { msfem_system_destroy(h); }
};

void fill_stats(msfem_system_t h, msfem_stats* stats)
{
    if (stats) msfem_get_stats(h, stats);
}

}  // namespace

extern "C" {

// FEM::FEM_forBaseEliptic, stiffness-only overload (FEM/FEM.h:398-717)
int msfem_fem_scalar_driver(int n_nodes, const double* xyz, int n_tets, const int32_t* tets, const int32_t* material,
                            int n_materials, const double* sigma, int n_bc, const int32_t* bc_nodes,
                            const double* bc_values, int method, int precision, double min_residual, int maxiter,
                            double* solution, msfem_stats* stats)
{
    Handle H;
    int rc;
    // Grid_forScal::Initialization + CreationPortrait (FEM.h:427-448)
    if ((rc = msfem_system_create(MSFEM_SCALAR, n_nodes, xyz, n_tets, tets, material, 0, &H.h)) < 0) return rc;
    // element loop + SummPartOfMatrix (FEM.h:469-492)
    if ((rc = msfem_assemble_scalar(H.h, sigma, n_materials)) < 0) return rc;
    // first boundary condition: rows, then the column sweep (FEM.h:506-619)
    if ((rc = msfem_apply_dirichlet(H.h, n_bc, bc_nodes, bc_values, MSFEM_ROW_AND_COLUMN, 0)) < 0) return rc;
    int solve_rc;
    if (method == MSFEM_PCG_SSOR) {
        // the reference's own solve: X = F, then SSOR(0.75)-PCG in its restart loop (FEM.h:627-695)
        solve_rc = msfem_solve_driver_loop(H.h, 0, method, precision, min_residual, nullptr, nullptr, nullptr);
    } else {
        // X = F (FEM.h:635), then one solve to MIN_RESIDUAL
        if ((rc = msfem_copy_f_to_x(H.h)) < 0) return rc;
        solve_rc = msfem_solve(H.h, method, precision, 30, maxiter, min_residual, nullptr, nullptr);
    }
    if (solve_rc < 0) return solve_rc;
    if ((rc = msfem_get_x(H.h, solution, 0)) < 0) return rc;
    fill_stats(H.h, stats);
    return solve_rc;
}

// FEM::FEM_forElasticDeformation (FEM/FEM.h:1286-1961)
int msfem_fem_elastic_driver(int n_nodes, const double* xyz, int n_tets, const int32_t* tets, const int32_t* material,
                             int n_materials, const double* E, const double* nu, int n_bc, const int32_t* bc_nodes,
                             const int32_t* bc_mask, const double* bc_values, int n_faces, const int32_t* face_nodes,
                             const double* face_traction, int method, int precision, double min_residual, int maxiter,
                             double* solution, msfem_stats* stats)
{
    Handle H;
    int rc;
    // Grid_forMech::Initialization + CreationPortrait (FEM.h:1310-1335)
    if ((rc = msfem_system_create(MSFEM_ELASTIC, n_nodes, xyz, n_tets, tets, material, 0, &H.h)) < 0) return rc;
    // second boundary condition (traction) into F (FEM.h:1338-1343)
    if ((rc = msfem_add_traction(H.h, n_faces, face_nodes, face_traction, 0)) < 0) return rc;
    // element loop + SummPartOfMatrix (FEM.h:1346-1384)
    if ((rc = msfem_assemble_elastic(H.h, E, nu, n_materials)) < 0) return rc;
    // first boundary condition on the expanded scalar system: DOF 3*node + component in
    // boundary-list order (FEM.h:1676-1723), then the column sweep (FEM.h:1757-1812)
    std::vector<int32_t> dofs;
    std::vector<double> vals;
    dofs.reserve(3 * (size_t)n_bc);
    vals.reserve(3 * (size_t)n_bc);
    for (int i = 0; i < n_bc; i++)
        for (int c = 0; c < 3; c++)
            if (bc_mask[i] & (1 << c)) {
                dofs.push_back(3 * bc_nodes[i] + c);
                vals.push_back(bc_values[3 * i + c]);
            }
    if ((rc = msfem_apply_dirichlet(H.h, (int)dofs.size(), dofs.data(), vals.data(), MSFEM_ROW_AND_COLUMN, 0)) < 0)
        return rc;
    // X holds the Dirichlet values and 0 elsewhere, as the reference's newSLAE.X; MSFEM_PCG_SSOR runs
    // the reference's own solve, SSOR(0.75)-PCG in its restart loop (FEM.h:1853-1939)
    const int solve_rc = method == MSFEM_PCG_SSOR
                             ? msfem_solve_driver_loop(H.h, 1, method, precision, min_residual, nullptr, nullptr, nullptr)
                             : msfem_solve(H.h, method, precision, 30, maxiter, min_residual, nullptr, nullptr);
    if (solve_rc < 0) return solve_rc;
    if ((rc = msfem_get_x(H.h, solution, 0)) < 0) return rc;
    fill_stats(H.h, stats);
    return solve_rc;
}

}  // extern "C"
