// z-marching matrix-free Kuhn-grid product (the operator of kuhn.cuh), with TMA-staged layers.
//
// A CTA owns a column of (TX-1) x (TY-1) nodes and a range of node layers [k0, k1); its TX x TY
// threads each own one column of hexahedra (the owned nodes' columns plus one on the low side of
// each axis) and step up through the slabs kz = k0-1 .. k1-1.  Step kz computes the hexahedra of
// slab kz (one per thread: the six tetrahedra's forces summed into bottom and top corner sums, the
// same arithmetic and order as kuhn_brick) and completes node layer kz: bottom corners of slab kz
// plus top corners of slab kz-1, corner 0 .. 7 in order -- the brick kernel's sums in the brick
// kernel's order (bit-identical on anisotropic grids; on isotropic ones the 1/h and V/h factors are
// folded into the material table, kuhn_tet_iso).
//
// Staging.  Stage L holds node layer L (input values, Jacobi scale, Dirichlet bits, over the
// (TX+1) x (TY+1) window) and the material codes of slab L.  Its rows are copied by cp.async.bulk
// (the 16-byte-aligned superset of each contiguous row) onto one mbarrier per ring slot: every warp
// posts its share's byte count with arrive.expect_tx, then its lanes issue the copies.  Step kz
// waits for stage kz+1 (issued two steps earlier), converts it to the scaled, masked input of the
// next slab, and issues stage kz+3 into the slot stage kz-1 left, so three stages are in flight
// while a slab computes.  The epilogue's other per-node vectors are loaded into registers before
// the slab's arithmetic, which hides their latency.
// Every wait is bounded: on expiry the CTA raises *err, waits (bounded) for its copies in flight
// and stops; the host reads the flag.
#pragma once

#include <cstdint>

#include "kuhn.cuh"

namespace msfem {

__host__ __device__ constexpr int kz_round_up(int v, int m) { return (v + m - 1) / m * m; }

template <class T, int TX_, int TY_, int NE_, bool SC_>
struct KzLayout {
    static constexpr int TX = TX_, TY = TY_, NE = NE_;
    static constexpr bool SC = SC_;                 // a Jacobi scale is staged (S K S)
    static constexpr int THREADS = TX * TY;        // one thread per hexahedron column
    static constexpr int WX = TX + 1, WY = TY + 1;  // staged node window per layer
    static constexpr int OX = TX - 1, OY = TY - 1;  // owned nodes per layer
    static constexpr int RING = 4;
    static constexpr int EL = 16 / (int)sizeof(T);  // elements per 16 bytes
    static constexpr int XP = kz_round_up(3 * WX + 2 * (EL - 1), EL);  // window row pitch (elements)
    static constexpr int FP = kz_round_up(WX + 6, 4);                  // Dirichlet-bit row pitch (words)
    static constexpr int MP = kz_round_up(TX + 2, 2);                  // material row pitch (hexahedra)
    // one stage, bytes (every part a multiple of 16)
    static constexpr int X_OFF = 0;
    static constexpr int S_OFF = X_OFF + WY * XP * (int)sizeof(T);
    static constexpr int F_OFF = S_OFF + (SC ? WY * XP * (int)sizeof(T) : 0);
    static constexpr int M_OFF = F_OFF + WY * FP * 4;
    static constexpr int STAGE = M_OFF + TY * MP * 8;
    // after the ring: two converted layers, bottom corner sums, two sets of top corner sums, barriers.
    // A converted layer's rows have pitch UP = 16 (mod 32) words, so the two rows of hexahedron
    // columns a warp covers read disjoint bank halves.
    static constexpr int U_OFF = RING * STAGE;
    static constexpr int NU = 3 * WX * WY;  // converted elements
    static constexpr int UP = kz_round_up(WX - 16, 32) + 16;
    static constexpr int UPLANE = UP * WY;
    static constexpr int UL = 3 * UPLANE;  // one converted layer (elements)
    static constexpr int B_OFF = U_OFF + 2 * UL * (int)sizeof(T);
    static constexpr int T_OFF = B_OFF + 12 * THREADS * (int)sizeof(T);
    static constexpr int L_OFF = T_OFF + 2 * 12 * THREADS * (int)sizeof(T);
    static constexpr int BAR_OFF = kz_round_up(L_OFF + 2 * kKuhnMaxMat * (int)sizeof(T), 16);
    static constexpr size_t smem = BAR_OFF + 8 * RING;
    static_assert(STAGE % 16 == 0, "stage parts must stay 16-byte aligned");
};

__device__ __forceinline__ uint32_t kz_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void kz_bulk(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void kz_expect(uint32_t bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}

// bounded wait for phase `parity` of `bar`
__device__ __forceinline__ bool kz_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 24); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <class T>
struct KzArgs {
    KuhnView<T> K;         // grid, materials, Dirichlet bits, scale (may be null), lame
    const T* x;            // input
    int tiles_x, tiles_y;  // CTA columns per axis
    int seg_len, n_seg;    // node layers per CTA and segments along z
    int* err;              // raised when a staging wait expires
};

// One lane's row of a stage, fixed for the CTA except for the layer: kind 0 input values, 1 Jacobi
// scale, 2 Dirichlet bits (window rows of nodes), 3 material codes (rows of hexahedra), -1 none;
// first node (hexahedron) of the row at layer 0, its length, and the row's place in the stage.
struct KzCopy {
    int64_t lo0;
    int kind, cnt;
    uint32_t dst;
};

// the copy list [x rows WY][scale rows WY][fix rows WY][material rows TY], shared out over the
// CTA's warps: lane l of warp w takes entry w * CPW + l
template <class L, class T>
__device__ __forceinline__ KzCopy kz_copy_of(const KuhnView<T>& K, int i0, int j0)
{
    constexpr int NCOPY = 3 * L::WY + L::TY;
    constexpr int NWARPS = L::THREADS / 32;
    constexpr int CPW = (NCOPY + NWARPS - 1) / NWARPS;
    static_assert(CPW <= 32, "one copy per lane");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = warp * CPW + lane;
    const int nnx = K.nx + 1, nny = K.ny + 1;
    const int gi_lo = i0 - 1 < 0 ? 0 : i0 - 1;
    const int gi_hi = (i0 - 1 + L::WX - 1) > K.nx ? K.nx : (i0 - 1 + L::WX - 1);
    const int ci_hi = (i0 - 1 + L::TX - 1) > K.nx - 1 ? K.nx - 1 : (i0 - 1 + L::TX - 1);
    KzCopy c{0, -1, 0, 0u};
    if (lane >= CPW || q >= NCOPY) return c;
    if (q < 3 * L::WY) {
        const int part = q / L::WY, wj = q - part * L::WY;
        const int gj = j0 - 1 + wj;
        if (gj >= 0 && gj < nny && (part != 1 || L::SC)) {
            c.kind = part;
            c.lo0 = gi_lo + (int64_t)nnx * gj;
            c.cnt = gi_hi - gi_lo + 1;
            c.dst = part == 0 ? L::X_OFF + wj * L::XP * sizeof(T)
                              : (part == 1 ? L::S_OFF + wj * L::XP * sizeof(T) : L::F_OFF + wj * L::FP * 4);
        }
    } else {
        const int cj = q - 3 * L::WY, gcj = j0 - 1 + cj;
        if (gcj >= 0 && gcj < K.ny) {
            c.kind = 3;
            c.lo0 = gi_lo + (int64_t)K.nx * gcj;
            c.cnt = ci_hi - gi_lo + 1;
            c.dst = L::M_OFF + cj * L::MP * 8;
        }
    }
    return c;
}

// One stage's copies: each warp's lane 0 posts the warp's byte count (arrive.expect_tx: the barrier
// expects one arrival per warp), then its lanes issue their rows (16-byte-aligned supersets).
template <class L, class T>
__device__ __forceinline__ void kz_issue(const KzArgs<T>& A, const KzCopy& c, int64_t P, int64_t Q, int layer,
                                         unsigned char* stage, uint32_t bar)
{
    const KuhnView<T>& K = A.K;
    const int lane = threadIdx.x & 31;
    const void* src = nullptr;
    uint32_t bytes = 0;
    if (c.kind >= 0 && layer >= 0 && layer <= K.nz && (c.kind < 3 || layer < K.nz)) {
        const int64_t lo = c.lo0 + (c.kind < 3 ? P : Q) * layer;
        if (c.kind < 2) {
            const int64_t a0 = (3 * lo) & ~(int64_t)(L::EL - 1);
            const int64_t a1 = (3 * (lo + c.cnt) + L::EL - 1) & ~(int64_t)(L::EL - 1);
            src = (c.kind == 0 ? A.x : K.scale) + a0;
            bytes = (uint32_t)((a1 - a0) * sizeof(T));
        } else if (c.kind == 2) {
            const int64_t a0 = lo & ~(int64_t)3, a1 = (lo + c.cnt + 3) & ~(int64_t)3;
            src = K.fix + a0;
            bytes = (uint32_t)((a1 - a0) * 4);
        } else {
            const int64_t a0 = lo & ~(int64_t)1, a1 = (lo + c.cnt + 1) & ~(int64_t)1;
            src = K.mat + a0;
            bytes = (uint32_t)((a1 - a0) * 8);
        }
    }
    uint32_t total = bytes;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) kz_expect(bar, total);
    __syncwarp();
    if (bytes) kz_bulk(kz_smem_addr(stage + c.dst), src, bytes, bar);
}

// the z-marching product; Epi: NE per-node input vectors (sources(ev)), skip(), finish(),
// operator()(node, y[3], input x[3], e[NE][3] = those vectors at the node)
template <int FORM, bool ISO, bool SC, class T, int TX, int TY, int MINB, class Epi>
__global__ void __launch_bounds__(TX* TY, MINB) k_kuhn_z(KzArgs<T> A, Epi epi)
{
    using L = KzLayout<T, TX, TY, Epi::NE, SC>;
    if (epi.skip()) return;
    extern __shared__ __align__(128) unsigned char kz_smem[];
    const KuhnView<T>& K = A.K;
    T* U = reinterpret_cast<T*>(kz_smem + L::U_OFF);
    T* Bc = reinterpret_cast<T*>(kz_smem + L::B_OFF);
    T* Tc = reinterpret_cast<T*>(kz_smem + L::T_OFF);
    T* slame = reinterpret_cast<T*>(kz_smem + L::L_OFF);
    const uint32_t bar0 = kz_smem_addr(kz_smem + L::BAR_OFF);
    const int tid = threadIdx.x;
    kuhn_stage_lame(K, slame);
    if (tid == 0) {
        for (int s = 0; s < L::RING; s++)  // one arrival per warp and stage
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar0 + 8 * s), "r"(L::THREADS / 32));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
    }
    __syncthreads();
    const int nnx = K.nx + 1, nny = K.ny + 1, nnz = K.nz + 1;
    const int tile = blockIdx.x % (A.tiles_x * A.tiles_y);
    const int seg = blockIdx.x / (A.tiles_x * A.tiles_y);
    const int i0 = (tile % A.tiles_x) * L::OX, j0 = (tile / A.tiles_x) * L::OY;
    const int k0 = seg * A.seg_len;
    const int k1 = (k0 + A.seg_len) < nnz ? (k0 + A.seg_len) : nnz;
    if (k0 >= k1) return;  // whole-CTA exit before any copy
    const T* ev[Epi::NE > 0 ? Epi::NE : 1] = {};
    epi.sources(ev);
    const int first = k0 - 1;  // the first stage (and slab) of the march
    auto slot = [&](int layer) { return (layer - first) % L::RING; };
    auto parity = [&](int layer) { return (uint32_t)(((layer - first) / L::RING) & 1); };
    auto stage_of = [&](int layer) { return kz_smem + slot(layer) * L::STAGE; };
    const int gi_lo = i0 - 1 < 0 ? 0 : i0 - 1;
    // per-layer offsets in 32 bits: node g(i, j, L) = i + nnx j + P L, hexahedron c = i + nx j + Q L;
    // only their residues (mod 4, mod 2) enter the staged-row offsets
    const int64_t P = (int64_t)nnx * nny;
    const int Pm4 = (int)(P & 3), P3m = (int)((3 * P) & (L::EL - 1));
    const int Qm2 = (int)(((int64_t)K.nx * K.ny) & 1);
    // convert stage `layer` into its U buffer: u = s x on the window (0 outside the grid and on
    // eliminated columns)
    auto convert = [&](int layer) {
        const unsigned char* st = stage_of(layer);
        const T* xr = reinterpret_cast<const T*>(st + L::X_OFF);
        const T* sr = reinterpret_cast<const T*>(st + L::S_OFF);
        const uint32_t* fr = reinterpret_cast<const uint32_t*>(st + L::F_OFF);
        T* u = U + ((layer - first) & 1) * L::UL;
        const bool lay_ok = layer >= 0 && layer < nnz;
        // one node (three components) per thread and pass
        for (int w = tid; w < L::WX * L::WY; w += L::THREADS) {
            const int wj = w / L::WX, wi = w - wj * L::WX;
            const int gi = i0 - 1 + wi, gj = j0 - 1 + wj;
            T v[3] = {T(0), T(0), T(0)};
            if (lay_ok && gi >= 0 && gi < nnx && gj >= 0 && gj < nny) {
                const int r0 = gi_lo + nnx * gj;  // row start at layer 0
                const uint32_t fx = fr[wj * L::FP + ((r0 + Pm4 * layer) & 3) + (gi - gi_lo)];
                const int xo = wj * L::XP + ((3 * r0 + P3m * layer) & (L::EL - 1)) + 3 * (gi - gi_lo);
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    T t = xr[xo + a];
                    if (SC) t *= sr[xo + a];
                    v[a] = ((fx >> (3 + a)) & 1u) ? T(0) : t;
                }
            }
            const int uo = wj * L::UP + wi;
#pragma unroll
            for (int a = 0; a < 3; a++) u[a * L::UPLANE + uo] = v[a];
        }
    };
    // prologue: stages first .. first+2 in flight.  A wait's outcome is made block-wide at the
    // next barrier (__syncthreads_and), so every thread takes the same path.
    const KzCopy cp = kz_copy_of<L>(K, i0, j0);
    const int64_t Q = (int64_t)K.nx * K.ny;
    kz_issue<L>(A, cp, P, Q, first, stage_of(first), bar0 + 8 * slot(first));
    kz_issue<L>(A, cp, P, Q, first + 1, stage_of(first + 1), bar0 + 8 * slot(first + 1));
    if (first + 2 <= k1) kz_issue<L>(A, cp, P, Q, first + 2, stage_of(first + 2), bar0 + 8 * slot(first + 2));
    int issued = first + 2 <= k1 ? first + 2 : first + 1, landed = first - 1;
    bool ok = kz_wait(bar0 + 8 * slot(first), parity(first));
    convert(first);  // reads only this CTA's shared memory, whatever the wait's outcome
    const int ci = tid % TX, cj = tid / TX;
    const int gci = i0 - 1 + ci, gcj = j0 - 1 + cj;
    const bool col_ok = gci >= 0 && gci < K.nx && gcj >= 0 && gcj < K.ny;
    const int mrow = gi_lo + K.nx * gcj;  // hexahedron row start at layer 0 (when col_ok)
    // the node this thread completes: (ni, nj) = (ci, cj) when both are below the owned extent
    const int gi = i0 + ci, gj = j0 + cj;
    const bool own = ci < L::OX && cj < L::OY && gi < nnx && gj < nny;
    const int64_t g0 = gi + (int64_t)nnx * gj;
    const int wrow = gi_lo + nnx * gj;
    for (int kz = first; kz < k1; kz++) {
        // stage kz+1 (issued two steps ago): wait, convert; the barrier then also frees stage kz-1's
        // ring slot (every thread is past step kz-1) for stage kz+3
        ok = kz_wait(bar0 + 8 * slot(kz + 1), parity(kz + 1)) && ok;
        convert(kz + 1);
        ok = __syncthreads_and(ok);
        if (!ok) break;
        landed = kz + 1;
        if (kz + 3 <= k1) {
            kz_issue<L>(A, cp, P, Q, kz + 3, stage_of(kz + 3), bar0 + 8 * slot(kz + 3));
            issued = kz + 3;
        }
        // the epilogue's per-node vectors, loaded now so the loads overlap the hexahedron
        T e[Epi::NE > 0 ? Epi::NE : 1][3];
        const int64_t gk = g0 + P * kz;
        if (kz >= k0 && own) {
#pragma unroll
            for (int q = 0; q < Epi::NE; q++)
#pragma unroll
                for (int a = 0; a < 3; a++) e[q][a] = __ldg(ev[q] + 3 * gk + a);
        }
        // slab kz: this thread's hexahedron
        {
            const unsigned char* st = stage_of(kz);
            const uint2* mr = reinterpret_cast<const uint2*>(st + L::M_OFF);
            const T* ub = U + ((kz - first) & 1) * L::UL;
            const T* ut = U + ((kz + 1 - first) & 1) * L::UL;
            T f[8][3];
#pragma unroll
            for (int b = 0; b < 8; b++) f[b][0] = f[b][1] = f[b][2] = T(0);
            if (col_ok && kz >= 0 && kz < K.nz) {
                T u[8][3];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const T* src = (b & 4) ? ut : ub;
                    const int w = (cj + ((b >> 1) & 1)) * L::UP + ci + (b & 1);
#pragma unroll
                    for (int a = 0; a < 3; a++) u[b][a] = src[a * L::UPLANE + w];
                }
                const uint2 mc = mr[cj * L::MP + ((mrow + Qm2 * kz) & 1) + (gci - gi_lo)];
                T lam[6], mu[6];
#pragma unroll
                for (int t = 0; t < 6; t++) {
                    const int m = ((t < 4 ? mc.x >> (8 * t) : mc.y >> (8 * (t - 4)))) & 0xff;
                    lam[t] = slame[2 * m];
                    mu[t] = slame[2 * m + 1];
                }
                if (ISO) {
                    kuhn_tet_iso<FORM, 0, 1, 2>(u[0], u[1], u[3], u[7], lam[0], mu[0], f[0], f[1], f[3], f[7]);
                    kuhn_tet_iso<FORM, 0, 2, 1>(u[0], u[1], u[5], u[7], lam[1], mu[1], f[0], f[1], f[5], f[7]);
                    kuhn_tet_iso<FORM, 1, 0, 2>(u[0], u[2], u[3], u[7], lam[2], mu[2], f[0], f[2], f[3], f[7]);
                    kuhn_tet_iso<FORM, 1, 2, 0>(u[0], u[2], u[6], u[7], lam[3], mu[3], f[0], f[2], f[6], f[7]);
                    kuhn_tet_iso<FORM, 2, 0, 1>(u[0], u[4], u[5], u[7], lam[4], mu[4], f[0], f[4], f[5], f[7]);
                    kuhn_tet_iso<FORM, 2, 1, 0>(u[0], u[4], u[6], u[7], lam[5], mu[5], f[0], f[4], f[6], f[7]);
                } else {
                    kuhn_tet<FORM, 0, 1, 2>(u[0], u[1], u[3], u[7], lam[0], mu[0], K.ih, K.vh, f[0], f[1], f[3], f[7]);
                    kuhn_tet<FORM, 0, 2, 1>(u[0], u[1], u[5], u[7], lam[1], mu[1], K.ih, K.vh, f[0], f[1], f[5], f[7]);
                    kuhn_tet<FORM, 1, 0, 2>(u[0], u[2], u[3], u[7], lam[2], mu[2], K.ih, K.vh, f[0], f[2], f[3], f[7]);
                    kuhn_tet<FORM, 1, 2, 0>(u[0], u[2], u[6], u[7], lam[3], mu[3], K.ih, K.vh, f[0], f[2], f[6], f[7]);
                    kuhn_tet<FORM, 2, 0, 1>(u[0], u[4], u[5], u[7], lam[4], mu[4], K.ih, K.vh, f[0], f[4], f[5], f[7]);
                    kuhn_tet<FORM, 2, 1, 0>(u[0], u[4], u[6], u[7], lam[5], mu[5], K.ih, K.vh, f[0], f[4], f[6], f[7]);
                }
            }
            T* tc = Tc + ((kz - first) & 1) * 12 * L::THREADS;
#pragma unroll
            for (int b = 0; b < 4; b++)
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    Bc[(3 * b + a) * L::THREADS + tid] = f[b][a];
                    tc[(3 * b + a) * L::THREADS + tid] = f[b + 4][a];
                }
        }
        __syncthreads();
        // node layer kz: bottom corners of slab kz, then top corners of slab kz-1 (a warp reads 32
        // consecutive hexahedron columns: no bank conflicts)
        if (kz >= k0 && own) {
            const T* tp = Tc + ((kz - 1 - first) & 1) * 12 * L::THREADS;
            T y[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = tid + (1 - ((b >> 1) & 1)) * TX + 1 - (b & 1);
                const T* src = (b & 4) ? tp : Bc;
                const int k = 3 * (b & 3);
#pragma unroll
                for (int a = 0; a < 3; a++) y[a] += src[(k + a) * L::THREADS + c];
            }
            const unsigned char* st = stage_of(kz);
            const T* xr = reinterpret_cast<const T*>(st + L::X_OFF);
            const T* sr = reinterpret_cast<const T*>(st + L::S_OFF);
            const uint32_t* fr = reinterpret_cast<const uint32_t*>(st + L::F_OFF);
            const int wj = cj + 1;
            const int xo = ((3 * wrow + P3m * kz) & (L::EL - 1)) + 3 * (gi - gi_lo);
            const uint32_t fx = fr[wj * L::FP + ((wrow + Pm4 * kz) & 3) + (gi - gi_lo)];
            T xin[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                xin[a] = xr[wj * L::XP + xo + a];
                if ((fx >> a) & 1u)
                    y[a] = xin[a];
                else if (SC)
                    y[a] *= sr[wj * L::XP + xo + a];
            }
            epi(gk, y, xin, e);
        }
    }
    if (!ok) {
        if (tid == 0) atomicExch(A.err, 1);
        // the copies this CTA issued must land before it leaves: bounded waits on the stages issued
        // and not yet seen complete
        for (int layer = landed + 1; layer <= issued; layer++) kz_wait(bar0 + 8 * slot(layer), parity(layer));
        return;
    }
    epi.finish();
}

// ---- the pre-scaled variant: the input arrives as s x with the eliminated columns already zero
// (its producer writes that copy next to x), so a stage holds the input rows, the Dirichlet bits
// and the material codes only; the corners are read straight from the staged rows (each row at
// its own 16-byte misalignment) and no layer is converted.  With the conversion gone a step needs
// one barrier: the bottom corner sums are double- and the top ones triple-buffered, so a step's
// sums never overwrite those a slower thread still gathers, and a five-slot ring keeps four
// stages in flight.  The epilogue gets the raw sums y = K (s x) at its node and the node's
// Dirichlet word, and applies the scale and the Dirichlet rows itself: operator()(node, y, fix, e).
template <class T, int TX, int TY, int NE>
struct KzpLayout : KzLayout<T, TX, TY, NE, false> {
    using B = KzLayout<T, TX, TY, NE, false>;
    static constexpr int RING = 5;
    static constexpr int B_OFF = RING * B::STAGE;
    static constexpr int T_OFF = B_OFF + 2 * 12 * B::THREADS * (int)sizeof(T);
    static constexpr int L_OFF = T_OFF + 3 * 12 * B::THREADS * (int)sizeof(T);
    static constexpr int BAR_OFF = kz_round_up(L_OFF + 2 * kKuhnMaxMat * (int)sizeof(T), 16);
    static constexpr size_t smem = BAR_OFF + 8 * RING;
};

template <int FORM, bool ISO, class T, int TX, int TY, int MINB, class Epi>
__global__ void __launch_bounds__(TX* TY, MINB) k_kuhn_zp(KzArgs<T> A, Epi epi)
{
    using L = KzpLayout<T, TX, TY, Epi::NE>;
    if (epi.skip()) return;
    extern __shared__ __align__(128) unsigned char kz_smem[];
    const KuhnView<T>& K = A.K;
    T* Bc = reinterpret_cast<T*>(kz_smem + L::B_OFF);
    T* Tc = reinterpret_cast<T*>(kz_smem + L::T_OFF);
    T* slame = reinterpret_cast<T*>(kz_smem + L::L_OFF);
    const uint32_t bar0 = kz_smem_addr(kz_smem + L::BAR_OFF);
    const int tid = threadIdx.x;
    kuhn_stage_lame(K, slame);
    if (tid == 0) {
        for (int s = 0; s < L::RING; s++)  // one arrival per warp and stage
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar0 + 8 * s), "r"(L::THREADS / 32));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
    }
    __syncthreads();
    const int nnx = K.nx + 1, nny = K.ny + 1, nnz = K.nz + 1;
    const int tile = blockIdx.x % (A.tiles_x * A.tiles_y);
    const int seg = blockIdx.x / (A.tiles_x * A.tiles_y);
    const int i0 = (tile % A.tiles_x) * L::OX, j0 = (tile / A.tiles_x) * L::OY;
    const int k0 = seg * A.seg_len;
    const int k1 = (k0 + A.seg_len) < nnz ? (k0 + A.seg_len) : nnz;
    if (k0 >= k1) return;  // whole-CTA exit before any copy
    const T* ev[Epi::NE > 0 ? Epi::NE : 1] = {};
    epi.sources(ev);
    const int first = k0 - 1;  // the first stage (and slab) of the march
    auto slot = [&](int layer) { return (layer - first) % L::RING; };
    auto parity = [&](int layer) { return (uint32_t)(((layer - first) / L::RING) & 1); };
    auto stage_of = [&](int layer) { return kz_smem + slot(layer) * L::STAGE; };
    const int gi_lo = i0 - 1 < 0 ? 0 : i0 - 1;
    const int64_t P = (int64_t)nnx * nny;
    const int Pm4 = (int)(P & 3), P3m = (int)((3 * P) & (L::EL - 1));
    const int Qm2 = (int)(((int64_t)K.nx * K.ny) & 1);
    // prologue: stages first .. first+RING-2 in flight
    const KzCopy cp = kz_copy_of<L>(K, i0, j0);
    const int64_t Q = (int64_t)K.nx * K.ny;
    int issued = first - 1;
    for (int layer = first; layer <= first + L::RING - 2 && layer <= k1; layer++) {
        kz_issue<L>(A, cp, P, Q, layer, stage_of(layer), bar0 + 8 * slot(layer));
        issued = layer;
    }
    int landed = first - 1;
    bool ok = kz_wait(bar0 + 8 * slot(first), parity(first));
    const int ci = tid % TX, cj = tid / TX;
    const int gci = i0 - 1 + ci, gcj = j0 - 1 + cj;
    const bool col_ok = gci >= 0 && gci < K.nx && gcj >= 0 && gcj < K.ny;
    const int mrow = gi_lo + K.nx * gcj;  // hexahedron row start at layer 0 (when col_ok)
    // staged input rows cj, cj + 1 of this thread's hexahedron: row start at layer 0 and the
    // element of its first corner column
    const int r0b = gi_lo + nnx * gcj, r0t = r0b + nnx;
    const int cx = 3 * (gci - gi_lo);
    // the node this thread completes: (ni, nj) = (ci, cj) when both are below the owned extent
    const int gi = i0 + ci, gj = j0 + cj;
    const bool own = ci < L::OX && cj < L::OY && gi < nnx && gj < nny;
    const int64_t g0 = gi + (int64_t)nnx * gj;
    const int wrow = gi_lo + nnx * gj;
    for (int kz = first; kz < k1; kz++) {
        // stage kz+1 (the slab's top layer)
        ok = kz_wait(bar0 + 8 * slot(kz + 1), parity(kz + 1)) && ok;
        // the epilogue's per-node vectors, loaded now so the loads overlap the hexahedron
        T e[Epi::NE > 0 ? Epi::NE : 1][3];
        const int64_t gk = g0 + P * kz;
        if (kz >= k0 && own) {
#pragma unroll
            for (int q = 0; q < Epi::NE; q++)
#pragma unroll
                for (int a = 0; a < 3; a++) e[q][a] = __ldg(ev[q] + 3 * gk + a);
        }
        // slab kz: this thread's hexahedron
        {
            T f[8][3];
#pragma unroll
            for (int b = 0; b < 8; b++) f[b][0] = f[b][1] = f[b][2] = T(0);
            if (ok && col_ok && kz >= 0 && kz < K.nz) {
                const unsigned char* stb = stage_of(kz);
                const T* xb = reinterpret_cast<const T*>(stb + L::X_OFF);
                const T* xt = reinterpret_cast<const T*>(stage_of(kz + 1) + L::X_OFF);
                // corner b at row cj + ((b >> 1) & 1) of layer kz + (b >> 2)
                const int o[4] = {cj * L::XP + ((3 * r0b + P3m * kz) & (L::EL - 1)) + cx,
                                  (cj + 1) * L::XP + ((3 * r0t + P3m * kz) & (L::EL - 1)) + cx,
                                  cj * L::XP + ((3 * r0b + P3m * (kz + 1)) & (L::EL - 1)) + cx,
                                  (cj + 1) * L::XP + ((3 * r0t + P3m * (kz + 1)) & (L::EL - 1)) + cx};
                T u[8][3];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const T* src = (b & 4) ? xt : xb;
                    const int w = o[b >> 1] + 3 * (b & 1);
#pragma unroll
                    for (int a = 0; a < 3; a++) u[b][a] = src[w + a];
                }
                const uint2* mr = reinterpret_cast<const uint2*>(stb + L::M_OFF);
                const uint2 mc = mr[cj * L::MP + ((mrow + Qm2 * kz) & 1) + (gci - gi_lo)];
                T lam[6], mu[6];
#pragma unroll
                for (int t = 0; t < 6; t++) {
                    const int m = ((t < 4 ? mc.x >> (8 * t) : mc.y >> (8 * (t - 4)))) & 0xff;
                    lam[t] = slame[2 * m];
                    mu[t] = slame[2 * m + 1];
                }
                if (ISO) {
                    kuhn_tet_iso<FORM, 0, 1, 2>(u[0], u[1], u[3], u[7], lam[0], mu[0], f[0], f[1], f[3], f[7]);
                    kuhn_tet_iso<FORM, 0, 2, 1>(u[0], u[1], u[5], u[7], lam[1], mu[1], f[0], f[1], f[5], f[7]);
                    kuhn_tet_iso<FORM, 1, 0, 2>(u[0], u[2], u[3], u[7], lam[2], mu[2], f[0], f[2], f[3], f[7]);
                    kuhn_tet_iso<FORM, 1, 2, 0>(u[0], u[2], u[6], u[7], lam[3], mu[3], f[0], f[2], f[6], f[7]);
                    kuhn_tet_iso<FORM, 2, 0, 1>(u[0], u[4], u[5], u[7], lam[4], mu[4], f[0], f[4], f[5], f[7]);
                    kuhn_tet_iso<FORM, 2, 1, 0>(u[0], u[4], u[6], u[7], lam[5], mu[5], f[0], f[4], f[6], f[7]);
                } else {
                    kuhn_tet<FORM, 0, 1, 2>(u[0], u[1], u[3], u[7], lam[0], mu[0], K.ih, K.vh, f[0], f[1], f[3], f[7]);
                    kuhn_tet<FORM, 0, 2, 1>(u[0], u[1], u[5], u[7], lam[1], mu[1], K.ih, K.vh, f[0], f[1], f[5], f[7]);
                    kuhn_tet<FORM, 1, 0, 2>(u[0], u[2], u[3], u[7], lam[2], mu[2], K.ih, K.vh, f[0], f[2], f[3], f[7]);
                    kuhn_tet<FORM, 1, 2, 0>(u[0], u[2], u[6], u[7], lam[3], mu[3], K.ih, K.vh, f[0], f[2], f[6], f[7]);
                    kuhn_tet<FORM, 2, 0, 1>(u[0], u[4], u[5], u[7], lam[4], mu[4], K.ih, K.vh, f[0], f[4], f[5], f[7]);
                    kuhn_tet<FORM, 2, 1, 0>(u[0], u[4], u[6], u[7], lam[5], mu[5], K.ih, K.vh, f[0], f[4], f[6], f[7]);
                }
            }
            T* bc = Bc + ((kz - first) & 1) * 12 * L::THREADS;
            T* tc = Tc + ((kz - first) % 3) * 12 * L::THREADS;
#pragma unroll
            for (int b = 0; b < 4; b++)
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    bc[(3 * b + a) * L::THREADS + tid] = f[b][a];
                    tc[(3 * b + a) * L::THREADS + tid] = f[b + 4][a];
                }
        }
        // the sums are complete; every thread is past step kz-1, so stage kz-1's slot is free
        ok = __syncthreads_and(ok);
        if (!ok) break;
        landed = kz + 1;
        if (kz + L::RING - 1 <= k1) {
            kz_issue<L>(A, cp, P, Q, kz + L::RING - 1, stage_of(kz + L::RING - 1), bar0 + 8 * slot(kz + L::RING - 1));
            issued = kz + L::RING - 1;
        }
        // node layer kz: bottom corners of slab kz, then top corners of slab kz-1
        if (kz >= k0 && own) {
            const T* bp = Bc + ((kz - first) & 1) * 12 * L::THREADS;
            const T* tp = Tc + ((kz - 1 - first) % 3) * 12 * L::THREADS;
            T y[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = tid + (1 - ((b >> 1) & 1)) * TX + 1 - (b & 1);
                const T* src = (b & 4) ? tp : bp;
                const int k = 3 * (b & 3);
#pragma unroll
                for (int a = 0; a < 3; a++) y[a] += src[(k + a) * L::THREADS + c];
            }
            const uint32_t* fr = reinterpret_cast<const uint32_t*>(stage_of(kz) + L::F_OFF);
            const uint32_t fx = fr[(cj + 1) * L::FP + ((wrow + Pm4 * kz) & 3) + (gi - gi_lo)];
            epi(gk, y, fx, e);
        }
    }
    if (!ok) {
        if (tid == 0) atomicExch(A.err, 1);
        // the copies this CTA issued must land before it leaves: bounded waits on the stages issued
        // and not yet seen complete
        for (int layer = landed + 1; layer <= issued; layer++) kz_wait(bar0 + 8 * slot(layer), parity(layer));
        return;
    }
    epi.finish();
}

}  // namespace msfem
