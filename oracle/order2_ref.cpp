/* Test infrastructure only: runs the reference's own MsFEM Order2 construction
 * (MsFEM::Grid_forMech::Initialization, MsFEM/MsFEM_Grid.h:3525-3576: topology,
 * CreateFunctionalSpaces :1001-3080) and, on request, its macro element matrices
 * (FiniteElement_forMech_Poly::SolveLocalMatrix, :34-171, with domain 0's D as the
 * Order2 driver passes it, MsFEM/MsFEM.h:75-78) on a macro mesh and cell directories
 * written by multiscalefemsolver3d_b200/meshio.py, and dumps what the tests compare.
 *
 * A standalone program, not a library: the reference's grids copy their members
 * shallowly and free them twice when the per-face solver grids go out of scope
 * (MsFEM_Grid.h:2939), which aborts under glibc.  This program replaces the global
 * operator delete with a no-op, so the process only leaks; it exits right after
 * writing its output.
 *
 *   order2_ref <macro_dir> <fine_dir> <out_file> <n_mat> E0 nu0 [E1 nu1 ...] [--matrices]
 *
 * The bases themselves are the reference's BasisFunction_<i>.txt files in each
 * Elem_<c>/SubElem_0 directory (written by CreateFunctionalSpaces, :2926-2937).
 * out_file: a sequence of records, each `int32 tag, int32 count, payload` with
 *   tag 1: [n_elements, n_vertices, n_edges, n_faces, n_dofs]
 *   tag 2: edges, 2 vertex ids each (the edge's lower vertices 0 and 1)
 *   tag 3: per face (first-reached order): its id, n_edges, its edges in order
 *   tag 4: per element: n_dofs, its DOF global ids in local order, then its 6 faces
 *   tag 5: (--matrices) per element: the (3 n_dofs)^2 doubles of its local matrix,
 *          row 3I+i, column 3J+j = A[I][J].val[i][j]
 */
#include "MsFEM/MsFEM_Grid.h"

#include <cstdio>
#include <cstring>
#include <new>
#include <unistd.h>

void operator delete(void*) noexcept {}
void operator delete(void*, std::size_t) noexcept {}
void operator delete[](void*) noexcept {}
void operator delete[](void*, std::size_t) noexcept {}

namespace {

struct Dirichlet {
    std::vector<int> id_vertexes;
    std::function<Point<double>(Point<bool>&)> value;
};
struct Neumann {
    std::function<Point<double>(Point<double>)> value;
    std::vector<std::function<Point<double>(Point<double>)>> values;
    std::vector<std::vector<int>> id_vertexes_as_triangle;
    std::vector<int> id_base_element;
};

void put(FILE* f, int tag, const std::vector<int>& v)
{
    int h[2] = {tag, (int)v.size()};
    fwrite(h, sizeof(int), 2, f);
    if (!v.empty()) fwrite(v.data(), sizeof(int), v.size(), f);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 7) {
        fprintf(stderr, "usage: order2_ref macro_dir fine_dir out_file n_mat E0 nu0 ... [--matrices]\n");
        return 2;
    }
    const int n_mat = atoi(argv[4]);
    if (argc < 5 + 2 * n_mat) return 2;
    const bool matrices = argc > 5 + 2 * n_mat && strcmp(argv[5 + 2 * n_mat], "--matrices") == 0;

    math::SimpleGrid geo;
    geo.ReadFromNVTR(argv[1], -1);
    auto* grid = new MsFEM::Grid_forMech();
    grid->is_print_logFile = false;
    for (int m = 0; m < n_mat; m++) {
        grid->AddDomain();
        grid->GetDomain(m)->forMech.SetE(atof(argv[5 + 2 * m]));
        grid->GetDomain(m)->forMech.SetV(atof(argv[6 + 2 * m]));
    }
    std::vector<Dirichlet> first;
    std::vector<Neumann> second;
    grid->Initialization(geo, first, second, argv[2]);

    FILE* f = fopen(argv[3], "wb");
    if (!f) return 3;
    const int ne = grid->GetElementsCount();
    std::vector<int> edges, faces, elems;
    int n_edges = 0, n_faces = 0;
    // the grid keeps its edges and faces private; the elements reach all of them
    std::vector<int> seen_face;
    for (int e = 0; e < ne; e++) {
        auto* el = grid->GetElement(e);
        elems.push_back(el->GetDOFsCount());
        for (int d = 0; d < el->GetDOFsCount(); d++) elems.push_back(el->GetDOFInLocalID(d));
        for (int fl = 0; fl < el->GetLowerElementCount(); fl++) {
            auto* fc = el->GetLowerElement(fl);
            const int fid = fc->GetSelfGlobalId();
            elems.push_back(fid);
            if (fid >= (int)seen_face.size()) seen_face.resize(fid + 1, 0);
            if (seen_face[fid]) continue;
            seen_face[fid] = 1;
            if (fid + 1 > n_faces) n_faces = fid + 1;
            std::vector<int> rec{fid, fc->GetLowerElementCount()};
            for (int k = 0; k < fc->GetLowerElementCount(); k++) {
                auto* ed = fc->GetLowerElement(k);
                const int eid = ed->GetSelfGlobalId();
                rec.push_back(eid);
                if (2 * eid + 1 >= (int)edges.size()) edges.resize(2 * eid + 2, -1);
                edges[2 * eid] = ed->GetLowerElement(0)->GetSelfGlobalId();
                edges[2 * eid + 1] = ed->GetLowerElement(1)->GetSelfGlobalId();
                if (eid + 1 > n_edges) n_edges = eid + 1;
            }
            faces.insert(faces.end(), rec.begin(), rec.end());
        }
    }
    put(f, 1, {ne, grid->GetVertexCount(), n_edges, n_faces, grid->GetDOFsCount()});
    put(f, 2, edges);
    put(f, 3, faces);
    put(f, 4, elems);
    if (matrices) {
        std::function<std::vector<std::vector<double>>(Point<double>)> koefD = [grid](Point<double>) {
            return grid->GetDomain(0)->forMech.GetD(3);
        };
        for (int e = 0; e < ne; e++) {
            DenseMatrix<Tensor2Rank3D, Point<double>> A;
            grid->GetElement(e)->SolveLocalMatrix(A, koefD);
            const int n = grid->GetElement(e)->GetDOFsCount();
            std::vector<double> M((size_t)9 * n * n);
            for (int I = 0; I < n; I++)
                for (int i = 0; i < 3; i++)
                    for (int J = 0; J < n; J++)
                        for (int j = 0; j < 3; j++)
                            M[(size_t)(3 * I + i) * 3 * n + 3 * J + j] = A.A[I][J].val[i][j];
            int h[2] = {5, (int)M.size()};
            fwrite(h, sizeof(int), 2, f);
            fwrite(M.data(), sizeof(double), M.size(), f);
        }
    }
    fclose(f);
    fflush(stdout);
    _exit(0);
}
