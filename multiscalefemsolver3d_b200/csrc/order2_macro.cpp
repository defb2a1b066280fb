// The MsFEM Order2 macro system on the host: the 27-DOF element matrices of the cells (built on the
// GPU by msfem_cells_order2_macro_matrices) summed by the cells' DOF lists into the DOF-level
// portrait (Grid_forMech::CreationPortrait + CSSD_Matrix::SummPartOfMatrix, MsFEM/MsFEM.h:48-131)
// and written as the scalar system of MakeCopyMatrix_A_into_B (DOF 3 d + c, every 3x3 block of the
// portrait kept whole, structural zeros included), CSR with the diagonal in place -- the input of
// msfem_system_from_cssd.  The macro system is small (27 DOFs per macro cell); the sums run in cell
// order, then (I, J) order, so the result does not depend on threads.
#include <algorithm>
#include <cstring>
#include <vector>

#include "msfem_b200.h"

namespace msfem {
void set_error(const char* fmt, ...);
}

int msfem_order2_macro_csr(int n_cells, int n_dofs, const int32_t* cell_dofs, const double* K, int64_t* row_ptr,
                           int32_t* col, double* val, int64_t* nnz)
{
    using namespace msfem;
    if (n_cells < 0 || n_dofs <= 0 || (n_cells > 0 && !cell_dofs) || !nnz || (int64_t)3 * n_dofs >= ((int64_t)1 << 31)) {
        set_error("msfem_order2_macro_csr: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    for (int64_t q = 0; q < 27 * (int64_t)n_cells; q++)
        if (cell_dofs[q] < 0 || cell_dofs[q] >= n_dofs) {
            set_error("msfem_order2_macro_csr: cell %lld names DOF %d outside [0, %d)", (long long)(q / 27), cell_dofs[q],
                      n_dofs);
            return MSFEM_ERR_ARGUMENT;
        }
    // DOF-level portrait: the DOFs sharing a cell, sorted
    std::vector<std::vector<int32_t>> adj(n_dofs);
    for (int c = 0; c < n_cells; c++) {
        const int32_t* d = cell_dofs + 27 * (int64_t)c;
        for (int I = 0; I < 27; I++)
            for (int J = 0; J < 27; J++) adj[d[I]].push_back(d[J]);
    }
    for (int i = 0; i < n_dofs; i++) {
        adj[i].push_back(i);  // the diagonal is in every row
        std::sort(adj[i].begin(), adj[i].end());
        adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
    }
    int64_t total = 0;
    for (int i = 0; i < n_dofs; i++) total += 9 * (int64_t)adj[i].size();
    *nnz = total;
    if (!row_ptr || !col || !val) return MSFEM_OK;  // size query
    if (n_cells > 0 && !K) {
        set_error("msfem_order2_macro_csr: K missing");
        return MSFEM_ERR_ARGUMENT;
    }
    // scalar row 3 d + a holds the blocks of DOF row d, each as its three columns 3 e + b
    int64_t pos = 0;
    for (int d = 0; d < n_dofs; d++)
        for (int a = 0; a < 3; a++) {
            row_ptr[3 * (int64_t)d + a] = pos;
            for (int32_t e : adj[d])
                for (int b = 0; b < 3; b++) col[pos++] = 3 * e + b;
        }
    row_ptr[3 * (int64_t)n_dofs] = pos;
    std::memset(val, 0, sizeof(double) * total);
    for (int c = 0; c < n_cells; c++) {
        const int32_t* d = cell_dofs + 27 * (int64_t)c;
        const double* Kc = K + (int64_t)c * 27 * 27 * 9;
        for (int I = 0; I < 27; I++) {
            const std::vector<int32_t>& row = adj[d[I]];
            for (int J = 0; J < 27; J++) {
                const int64_t k = std::lower_bound(row.begin(), row.end(), d[J]) - row.begin();
                const double* blk = Kc + ((int64_t)I * 27 + J) * 9;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        val[row_ptr[3 * (int64_t)d[I] + a] + 3 * k + b] += blk[3 * a + b];
            }
        }
    }
    return MSFEM_OK;
}
