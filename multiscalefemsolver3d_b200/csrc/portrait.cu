// Mesh topology on the GPU: node -> element incidence, the node-level portrait
// (the reference's CreationPortrait, FEM/FEM_Grid.h:665-716 and :3236-3287),
// the element -> matrix-slot map used by the scatter, and the element colouring
// that makes the scatter race-free and deterministic.
#include <cub/cub.cuh>

#include <climits>

#include "devutil.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

__global__ void k_count_incidence(int n_tets, const int32_t* __restrict__ tets, int n_nodes, int32_t* cnt,
                                  int* bad)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n_tets * 4) return;
    int v = tets[t];
    if (v < 0 || v >= n_nodes) {
        atomicExch(bad, 1);
        return;
    }
    atomicAdd(&cnt[v], 1);
}

__global__ void k_fill_incidence(int n_tets, const int32_t* __restrict__ tets, const int32_t* __restrict__ ptr,
                                 int32_t* cursor, int32_t* inc)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n_tets * 4) return;
    int v = tets[t];
    int pos = atomicAdd(&cursor[v], 1);
    inc[ptr[v] + pos] = (int32_t)(t >> 2);
}

// Sort each node's element list ascending (lists are short: 24 for an interior Kuhn node).
__global__ void k_sort_incidence(int n_nodes, const int32_t* __restrict__ ptr, int32_t* inc)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_nodes) return;
    int b = ptr[v], e = ptr[v + 1];
    for (int i = b + 1; i < e; i++) {
        int x = inc[i], j = i - 1;
        while (j >= b && inc[j] > x) {
            inc[j + 1] = inc[j];
            j--;
        }
        inc[j + 1] = x;
    }
}

// One warp per node row: gather the nodes of all incident elements (self
// included) into shared memory, bitonic-sort them, drop duplicates.  Pass 0
// stores the unique count, pass 1 writes the sorted columns.
template <int PASS>
__global__ void k_portrait_rows(int n_nodes, const int32_t* __restrict__ tets, const int32_t* __restrict__ inc_ptr,
                                const int32_t* __restrict__ inc, int32_t* count, const int32_t* __restrict__ rp,
                                int32_t* col, int* overflow)
{
    constexpr int WPB = 4;
    __shared__ int buf[WPB][kMaxCandidates];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int row = blockIdx.x * WPB + w;
    if (row >= n_nodes) return;
    int* s = buf[w];
    const int b = inc_ptr[row], deg = inc_ptr[row + 1] - b;
    const int nc = 4 * deg;
    if (nc > kMaxCandidates) {
        if (lane == 0) atomicMax(overflow, nc);
        return;
    }
    int size = 32;
    while (size < nc) size <<= 1;
    for (int i = lane; i < size; i += 32) {
        int v = INT_MAX;
        if (i < nc) v = tets[4 * (int64_t)inc[b + (i >> 2)] + (i & 3)];
        s[i] = v;
    }
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < size; i += 32) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool asc = (i & k) == 0;
                    int a = s[i], c = s[ixj];
                    if ((a > c) == asc) {
                        s[i] = c;
                        s[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
    int total = 0;
    const int out0 = PASS ? rp[row] : 0;
    for (int base = 0; base < size; base += 32) {
        int i = base + lane;
        int v = s[i];
        bool keep = (v != INT_MAX) && (i == 0 || s[i - 1] != v);
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (PASS && keep) col[out0 + total + __popc(m & ((1u << lane) - 1u))] = v;
        total += __popc(m);
    }
    if (!PASS && lane == 0) count[row] = total;
}

__device__ __forceinline__ int find_slot(const int32_t* __restrict__ col, int lo, int hi, int c)
{
    hi -= 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = col[mid];
        if (v == c) return mid;
        if (v < c) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

__global__ void k_element_slots(int n_tets, const int32_t* __restrict__ tets, const int32_t* __restrict__ rp,
                                const int32_t* __restrict__ col, int32_t* eslot, int* bad)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    int v[4];
#pragma unroll
    for (int a = 0; a < 4; a++) v[a] = tets[4 * (int64_t)e + a];
#pragma unroll
    for (int I = 0; I < 4; I++)
#pragma unroll
        for (int J = 0; J < 4; J++) {
            int s = find_slot(col, rp[v[I]], rp[v[I] + 1], v[J]);
            if (s < 0) atomicExch(bad, 1);
            eslot[16 * (int64_t)e + 4 * I + J] = s;
        }
}

// Speculative greedy colouring of the element conflict graph (elements
// conflict when they share a node), deterministic by construction:
//  1. every uncoloured element proposes the smallest colour that none of its
//     already-coloured neighbours holds (reads only colours committed in
//     earlier rounds);
//  2. among neighbours that proposed the same colour in this round, the one
//     with the highest priority (hash of the id, ties by id) keeps it;
//  3. winners are committed, losers try again in the next round.
// Each kernel only reads arrays that no thread of the same kernel writes, so
// the colouring -- and with it the order in which the assembly adds element
// contributions -- is identical on every run.
constexpr int kMaxColors = 256;

__global__ void k_color_propose(int n_tets, const int32_t* __restrict__ tets, const int32_t* __restrict__ inc_ptr,
                                const int32_t* __restrict__ inc, const int32_t* __restrict__ color,
                                int32_t* __restrict__ tent, int* overflow)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    if (color[e] >= 0) {
        tent[e] = -1;
        return;
    }
    unsigned used[kMaxColors / 32];
#pragma unroll
    for (int w = 0; w < kMaxColors / 32; w++) used[w] = 0u;
    for (int a = 0; a < 4; a++) {
        const int v = tets[4 * (int64_t)e + a];
        for (int k = inc_ptr[v]; k < inc_ptr[v + 1]; k++) {
            const int c = color[inc[k]];
            if (c >= 0) used[c >> 5] |= 1u << (c & 31);
        }
    }
    int pick = -1;
#pragma unroll
    for (int w = 0; w < kMaxColors / 32; w++)
        if (pick < 0 && used[w] != 0xffffffffu) pick = 32 * w + __ffs(~used[w]) - 1;
    if (pick < 0) atomicExch(overflow, 1);
    tent[e] = pick;
}

__global__ void k_color_resolve(int n_tets, const int32_t* __restrict__ tets, const int32_t* __restrict__ inc_ptr,
                                const int32_t* __restrict__ inc, const int32_t* __restrict__ tent,
                                int32_t* __restrict__ win)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    const int c = tent[e];
    if (c < 0) {
        win[e] = 0;
        return;
    }
    const unsigned pe = hash32((unsigned)e);
    bool best = true;
    for (int a = 0; a < 4 && best; a++) {
        const int v = tets[4 * (int64_t)e + a];
        for (int k = inc_ptr[v]; k < inc_ptr[v + 1]; k++) {
            const int f = inc[k];
            if (f == e || tent[f] != c) continue;
            const unsigned pf = hash32((unsigned)f);
            if (pf > pe || (pf == pe && f > e)) {
                best = false;
                break;
            }
        }
    }
    win[e] = best ? 1 : 0;
}

__global__ void k_color_commit(int n_tets, const int32_t* __restrict__ tent, const int32_t* __restrict__ win,
                               int32_t* __restrict__ color, unsigned int* remaining)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    if (win[e]) color[e] = tent[e];
    else if (color[e] < 0) atomicAdd(remaining, 1u);
}

// off[c] = first position of colour c in the sorted key array
__global__ void k_color_starts(int n, const int32_t* __restrict__ keys, int32_t* off)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0 || keys[i] != keys[i - 1]) off[keys[i]] = i;
}

__global__ void k_max(int n, const int32_t* __restrict__ a, int32_t* mx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicMax(mx, a[i]);
}

__global__ void k_iota(int n, int32_t* a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int build_topology(System& s)
{
    cudaStream_t st = s.stream;
    const int N = s.n_nodes, E = s.n_tets;
    DBuf<int> flags;  // [0] bad node id, [1] overflow, [2] bad slot, [3] uncoloured count, [4] max colour
    MSFEM_TRY(flags.alloc(8));
    MSFEM_CK(cudaMemsetAsync(flags.p, 0, 8 * sizeof(int), st));

    // ---- incidence
    MSFEM_TRY(s.inc_ptr.alloc((size_t)N + 1));
    MSFEM_TRY(s.inc_elem.alloc((size_t)E * 4));
    DBuf<int32_t> cnt;
    MSFEM_TRY(cnt.alloc((size_t)N + 1));
    MSFEM_CK(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * ((size_t)N + 1), st));
    k_count_incidence<<<grid_for((int64_t)E * 4, 256), 256, 0, st>>>(E, s.tets.p, N, cnt.p, flags.p);
    MSFEM_CK(cudaGetLastError());
    int h_flags[4];
    MSFEM_CK(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (h_flags[0]) {  // checked before any kernel indexes by node id
        set_error("tets reference a node id outside [0, %d)", N);
        return MSFEM_ERR_ARGUMENT;
    }

    size_t tmp_bytes = 0;
    DBuf<unsigned char> tmp;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.p, s.inc_ptr.p, N + 1, st);
    MSFEM_TRY(tmp.alloc(tmp_bytes + 1));
    MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, cnt.p, s.inc_ptr.p, N + 1, st));
    MSFEM_CK(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * ((size_t)N + 1), st));
    k_fill_incidence<<<grid_for((int64_t)E * 4, 256), 256, 0, st>>>(E, s.tets.p, s.inc_ptr.p, cnt.p, s.inc_elem.p);
    k_sort_incidence<<<grid_for(N, 128), 128, 0, st>>>(N, s.inc_ptr.p, s.inc_elem.p);
    MSFEM_CK(cudaGetLastError());

    // ---- node-level portrait
    MSFEM_TRY(s.nrp.alloc((size_t)N + 1));
    k_portrait_rows<0><<<grid_for(N, 4), 128, 0, st>>>(N, s.tets.p, s.inc_ptr.p, s.inc_elem.p, cnt.p, nullptr,
                                                       nullptr, flags.p + 1);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemsetAsync(cnt.p + N, 0, sizeof(int32_t), st));
    tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.p, s.nrp.p, N + 1, st);
    MSFEM_TRY(tmp.alloc(tmp_bytes + 1));
    MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, cnt.p, s.nrp.p, N + 1, st));
    int32_t nnzb = 0;
    MSFEM_CK(cudaMemcpyAsync(&nnzb, s.nrp.p + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (h_flags[1]) {
        set_error("a node belongs to %d element-vertex slots; the portrait builder handles at most %d (node degree <= %d)",
                  h_flags[1], kMaxCandidates, kMaxCandidates / 4);
        return MSFEM_ERR_LIMIT;
    }
    s.nnzb = nnzb;
    MSFEM_TRY(s.ncol.alloc((size_t)nnzb));
    k_portrait_rows<1><<<grid_for(N, 4), 128, 0, st>>>(N, s.tets.p, s.inc_ptr.p, s.inc_elem.p, nullptr, s.nrp.p,
                                                       s.ncol.p, flags.p + 1);
    MSFEM_CK(cudaGetLastError());

    // ---- element -> slot map
    MSFEM_TRY(s.eslot.alloc((size_t)E * 16));
    k_element_slots<<<grid_for(E, 128), 128, 0, st>>>(E, s.tets.p, s.nrp.p, s.ncol.p, s.eslot.p, flags.p + 2);
    MSFEM_CK(cudaGetLastError());

    // ---- colouring
    DBuf<int32_t> color, tent, win;
    MSFEM_TRY(color.alloc((size_t)E));
    MSFEM_TRY(tent.alloc((size_t)E));
    MSFEM_TRY(win.alloc((size_t)E));
    MSFEM_CK(cudaMemsetAsync(color.p, 0xff, sizeof(int32_t) * (size_t)E, st));
    unsigned int* remaining = reinterpret_cast<unsigned int*>(flags.p + 3);
    int rounds = 0;
    for (;;) {
        if (rounds >= 1024) {
            set_error("element colouring did not finish in 1024 rounds");
            return MSFEM_ERR_LIMIT;
        }
        MSFEM_CK(cudaMemsetAsync(remaining, 0, sizeof(unsigned int), st));
        k_color_propose<<<grid_for(E, 256), 256, 0, st>>>(E, s.tets.p, s.inc_ptr.p, s.inc_elem.p, color.p, tent.p,
                                                          flags.p + 1);
        k_color_resolve<<<grid_for(E, 256), 256, 0, st>>>(E, s.tets.p, s.inc_ptr.p, s.inc_elem.p, tent.p, win.p);
        k_color_commit<<<grid_for(E, 256), 256, 0, st>>>(E, tent.p, win.p, color.p, remaining);
        MSFEM_CK(cudaGetLastError());
        rounds++;
        unsigned int h_rem = 0;
        MSFEM_CK(cudaMemcpyAsync(&h_rem, remaining, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        if (h_flags[1]) {
            set_error("element colouring needs more than %d colours", kMaxColors);
            return MSFEM_ERR_LIMIT;
        }
        if (h_rem == 0) break;
    }
    int n_colors = 0;
    {
        // number of colours = 1 + max colour
        int32_t* mx = flags.p + 4;
        MSFEM_CK(cudaMemsetAsync(mx, 0, sizeof(int32_t), st));
        k_max<<<grid_for(E, 256), 256, 0, st>>>(E, color.p, mx);
        int32_t h_mx = 0;
        MSFEM_CK(cudaMemcpyAsync(&h_mx, mx, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        n_colors = h_mx + 1;
        MSFEM_CK(cudaMemsetAsync(mx, 0, sizeof(int32_t), st));
    }
    // elements grouped by colour, ascending element id inside a colour (stable radix sort)
    DBuf<int32_t> ids, keys_out;
    MSFEM_TRY(ids.alloc((size_t)E));
    MSFEM_TRY(keys_out.alloc((size_t)E));
    MSFEM_TRY(s.color_elems.alloc((size_t)E));
    k_iota<<<grid_for(E, 256), 256, 0, st>>>(E, ids.p);
    int end_bit = 1;
    while ((1 << end_bit) <= n_colors) end_bit++;
    tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, color.p, keys_out.p, ids.p, s.color_elems.p, E, 0, end_bit, st);
    MSFEM_TRY(tmp.alloc(tmp_bytes + 1));
    MSFEM_CK(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, color.p, keys_out.p, ids.p, s.color_elems.p, E, 0,
                                             end_bit, st));
    // greedy colours are dense: every colour below the maximum is used
    DBuf<int32_t> starts;
    MSFEM_TRY(starts.alloc((size_t)n_colors));
    k_color_starts<<<grid_for(E, 256), 256, 0, st>>>(E, keys_out.p, starts.p);
    MSFEM_CK(cudaGetLastError());
    s.color_off.assign(n_colors + 1, 0);
    MSFEM_CK(cudaMemcpyAsync(s.color_off.data(), starts.p, sizeof(int32_t) * n_colors, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    s.color_off[n_colors] = E;
    starts.release();
    if (h_flags[2]) {
        set_error("element slot lookup failed (inconsistent portrait)");
        return MSFEM_ERR_STATE;
    }
    s.stats.n_colors = n_colors;
    // incidence count/fill/sort, portrait count/fill, slots, max, iota, colour starts, 3 launches per round
    s.total_launches += 9 + 3 * rounds;

    cnt.release();
    tmp.release();
    flags.release();
    color.release();
    tent.release();
    win.release();
    ids.release();
    keys_out.release();
    return MSFEM_OK;
}

}  // namespace msfem
