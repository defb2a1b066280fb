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
 *              [--driver <bc_file> <min_residual>]
 *
 * --driver runs the whole Order2 driver instead (MsFEM::MsFEM_forElasticDeformation_OrderBF2_forPoly,
 * MsFEM/MsFEM.h:14-569) with the Dirichlet groups of bc_file (text: n_groups, then per group
 * `take_x take_y take_z  vx vy vz  n  v_0 .. v_{n-1}`, the vertex lists and masked constant
 * values MsFEM/MsFEM_Main.cpp:187-300 reads from its kraev1 file) and no Neumann data, and adds
 *   tag 6: the solution, 3 doubles per macro DOF;
 *   tag 7: the driver system's block portrait (per DOF row: n_down, its columns, n_up, its columns).
 * --order1 (with --driver) runs the Order1 driver instead (MsFEM_forElasticDeformation_OrderBF1_forPoly,
 * MsFEM/MsFEM.h:571-1062, on Grid_forMech_Poly_Order1): tag 6 holds 3 doubles per macro vertex,
 * and only tag 6 is written.
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
#include "MsFEM/MsFEM.h"

#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <new>
#include <set>
#include <unistd.h>

// The Order1 construction closes each TecPlot stream twice (printTecPlot3D_DiffDomains closes it,
// then MsFEM_Grid.h:5607 again): streams closed once here ignore a second close until fopen hands
// their address out again.
namespace {
struct ClosedStreams {
    std::mutex mu;
    std::set<FILE*> closed;
};
ClosedStreams& closed_streams()
{
    static ClosedStreams* c = new ClosedStreams();
    return *c;
}
}  // namespace

extern "C" int fclose(FILE* f)
{
    static int (*real_close)(FILE*) = reinterpret_cast<int (*)(FILE*)>(dlsym(RTLD_NEXT, "fclose"));
    if (!f) return EOF;
    ClosedStreams& c = closed_streams();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (!c.closed.insert(f).second) return 0;
    }
    return real_close(f);
}

extern "C" FILE* fopen(const char* path, const char* mode)
{
    static FILE* (*real_open)(const char*, const char*) =
        reinterpret_cast<FILE* (*)(const char*, const char*)>(dlsym(RTLD_NEXT, "fopen"));
    FILE* f = real_open(path, mode);
    if (f) {
        ClosedStreams& c = closed_streams();
        std::lock_guard<std::mutex> lock(c.mu);
        c.closed.erase(f);
    }
    return f;
}

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
    bool matrices = false, order1 = false;
    const char* bc_file = nullptr;
    double min_residual = 1e-12;
    for (int a = 5 + 2 * n_mat; a < argc; a++) {
        if (strcmp(argv[a], "--matrices") == 0) matrices = true;
        if (strcmp(argv[a], "--order1") == 0) order1 = true;
        if (strcmp(argv[a], "--driver") == 0 && a + 2 < argc) {
            bc_file = argv[a + 1];
            min_residual = atof(argv[a + 2]);
            a += 2;
        }
    }

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
    std::vector<Point<double>> solution;
    CSSD_Matrix<Tensor2Rank3D, Point<double>> order2_slae;
    if (bc_file) {
        FILE* fb = fopen(bc_file, "r");
        if (!fb) return 4;
        int ng = 0;
        if (fscanf(fb, "%d", &ng) != 1) return 4;
        first.resize(ng);
        for (int g = 0; g < ng; g++) {
            int tx, ty, tz, n;
            double vx, vy, vz;
            if (fscanf(fb, "%d %d %d %lf %lf %lf %d", &tx, &ty, &tz, &vx, &vy, &vz, &n) != 7) return 4;
            for (int k = 0; k < n; k++) {
                int v;
                if (fscanf(fb, "%d", &v) != 1) return 4;
                first[g].id_vertexes.push_back(v);
            }
            const Point<bool> take(tx != 0, ty != 0, tz != 0);
            const Point<double> val(vx, vy, vz);
            first[g].value = [take, val](Point<bool>& is_take) {
                is_take = take;
                return val;
            };
        }
        fclose(fb);
        CSSD_Matrix<Tensor2Rank3D, Point<double>>& slae = order2_slae;
        if (order1) {
            auto* g1 = new MsFEM::Grid_forMech_Poly_Order1();
            g1->is_print_logFile = false;
            for (int m = 0; m < n_mat; m++) {
                g1->AddDomain();
                g1->GetDomain(m)->forMech.SetE(atof(argv[5 + 2 * m]));
                g1->GetDomain(m)->forMech.SetV(atof(argv[6 + 2 * m]));
            }
            MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly(false, min_residual, argv[2], geo, first, second,
                                                               argv[2], *g1, solution, slae);
            FILE* f1 = fopen(argv[3], "wb");
            if (!f1) return 3;
            std::vector<double> sol;
            for (auto& p : solution) {
                sol.push_back(p.x);
                sol.push_back(p.y);
                sol.push_back(p.z);
            }
            int h[2] = {6, (int)sol.size()};
            fwrite(h, sizeof(int), 2, f1);
            fwrite(sol.data(), sizeof(double), sol.size(), f1);
            fclose(f1);
            fflush(stdout);
            _exit(0);
        }
        MsFEM::MsFEM_forElasticDeformation_OrderBF2_forPoly(false, min_residual, argv[2], geo, first, second, argv[2],
                                                           *grid, solution, slae);
    } else {
        grid->Initialization(geo, first, second, argv[2]);
    }

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
    if (bc_file) {
        // tag 7: the block portrait of the driver's system, per DOF row: n_down, its columns, n_up,
        // its columns (CSSD_Matrix id_column_for_A_down / id_column_for_A_up)
        std::vector<int> port;
        for (int i = 0; i < (int)order2_slae.id_column_for_A_down.size(); i++) {
            port.push_back((int)order2_slae.id_column_for_A_down[i].size());
            for (int c : order2_slae.id_column_for_A_down[i]) port.push_back(c);
            port.push_back((int)order2_slae.id_column_for_A_up[i].size());
            for (int c : order2_slae.id_column_for_A_up[i]) port.push_back(c);
        }
        put(f, 7, port);
        std::vector<double> sol;
        for (auto& p : solution) {
            sol.push_back(p.x);
            sol.push_back(p.y);
            sol.push_back(p.z);
        }
        int h[2] = {6, (int)sol.size()};
        fwrite(h, sizeof(int), 2, f);
        fwrite(sol.data(), sizeof(double), sol.size(), f);
    }
    fclose(f);
    fflush(stdout);
    _exit(0);
}
