// Handles of the batched cell problems (cells.cu), shared with the two-level
// preconditioner (twolevel.cu), which reads the cells' meshes and bases.
#pragma once

#include <vector>

#include "batch.cuh"

namespace msfem {

struct BatchHandle {
    int device = 0;
    cudaStream_t stream = nullptr;
    BatchSys b;
    DBuf<double> xyz, lame, x;
    int n_mat = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.f;
    ~BatchHandle()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct CellsHandle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_cells = 0, n_mat = 0;
    int64_t n_nodes = 0, n_tets = 0;
    std::vector<int64_t> h_node_off, h_tet_off;
    DBuf<int64_t> node_off, tet_off;
    DBuf<double> xyz, box, lame;
    DBuf<int32_t> mat, mask, vert, fidx, fcell_node;
    BatchSys faces, vols;
    DBuf<double> fxyz, prof, fx, bx;
    int cap = 0;
    bool vols_assembled = false;  // volume problem matrices hold the current materials
    // materials of the face triangles and edge segments: 0 = those of the tetrahedra they bound,
    // 1 = material 0 everywhere (the reference's Salome face meshes carry no materials).  The
    // face batch is built in mode 0; msfem_cells_create then switches to mode 1, the default.
    int face_material = 0;
    DBuf<int32_t> face_emat_cells;  // the cells' face-triangle materials, kept while mode 1 is on
    DBuf<int32_t> edge_nodes, edge_len, seg_tri;
    DBuf<int> flag;
    // Order2 (27 bases per cell): face problems on material 0 with 8 right-hand sides, the edge
    // values, the per-cell edge order (DOF slot -> local edge) and the bases [node][27][3]
    BatchSys faces2;
    bool faces2_ready = false;
    DBuf<double> eprof2, fx2, x2, rhs2, bases2;
    DBuf<int32_t> edge_perm;
    bool order2_built = false;
    float ms2[4] = {0, 0, 0, 0};
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    float ms[4] = {0, 0, 0, 0};
    // the Order1 build's four stages (assemblies, edges, face batch, volume batch) captured into
    // CUDA graphs once the persistent launches' CTA sizes are tuned; replayed by later builds with
    // the same key (precision, tolerance, iteration limit, CTA sizes), with the timing events
    // recorded between the graphs
    cudaGraphExec_t build_graph[4] = {nullptr, nullptr, nullptr, nullptr};  // one per stage
    double build_key[5] = {0, 0, 0, 0, 0};
    double eager_key[5] = {-1, 0, 0, 0, 0};  // key of the last build run launch by launch
    int graph_builds = 0;  // builds run by replaying the graph
    ~CellsHandle()
    {
        for (auto g : build_graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};


}  // namespace msfem

// the C ABI's opaque cells handle (msfem_cells_t)
struct msfem_cells : msfem::CellsHandle {};
