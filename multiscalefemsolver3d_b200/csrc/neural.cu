// Learned MsFEM coarse space: a 3D convolutional operator that maps a macro cell's voxelised
// Young's-modulus field to the cell's 8 vector basis functions, trained on bases made by the
// batched cell solver (cells.cu) with this file's own forward and backward kernels.
//
// The reference has no learned component: its Order1 bases come from the cell problems
// (MsFEM_Grid.h, Grid_forMech_Poly_Order1::CreateFunctionalSpaces).  Here a predicted basis only
// feeds the two-level preconditioner's coarse space (twolevel.cu), so a poor prediction costs
// Krylov iterations, never accuracy; msfem_cells_basis_residual measures each cell's predicted
// bases against its own volume problem so that the caller can fall back to the exact solve.
//
// Cells: structured 8 x 8 x 8 hexahedra, six Kuhn tetrahedra each, in the node and tetrahedron
// order of a Kuhn cube (node i + 9 (j + 9 k), tetrahedron 6 * (hi + 8 (hj + 8 hk)) + t with t the
// corner sets {0,1,3,7} {0,1,5,7} {0,2,3,7} {0,2,6,7} {0,4,5,7} {0,4,6,7}); checked on the device.
//
// Network (parameters in one FP32 vector, layout below; BF16 copies for the tensor cores):
//   input  I[v][c], v in a 16^3 voxel grid (2 voxels per hexahedron edge), c = 0: the voxel
//          average of s ln(E / E_ref) (exact Kuhn-tetrahedron volume fractions per voxel),
//          c = 1..3: the voxel centre in [-1, 1]^3; zero outside the cell (zero padding)
//   L0     3x3x3 conv 4 -> 32, bias, ReLU           FP32 CUDA cores, output BF16
//   L1, L2 3x3x3 conv 32 -> 32, bias, ReLU          BF16 tensor cores (mma m16n8k16), FP32 accumulate
//   L3     3x3x3 conv 32 -> 24 (padded to 32), bias  same kernel, FP32 output
//   node   corr[n][3 v + a] = mean of L3 over the voxels touching node n (a partition: voxel x
//          belongs to node (x + 1) / 2 along each axis), zero at the 8 cell vertices
//   basis  psi_v^a(n) = Q1_v(n) + corr[n][3 v + a]   (Q1: trilinear in the node's grid position)
// Loss: mean over cells, nodes and the 24 channels of (corr - (psi_exact - Q1))^2; a training
// cell whose exact bases leave [-3, 3] (a nearly singular cell problem) has target corr = 0.
// Training: Adam on the FP32 master parameters; every gradient is deterministic (fixed-order
// partial sums, no atomics).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <new>
#include <vector>

#include "cells.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

constexpr int kV = 16;        // voxels per cell edge
constexpr int kVox = 4096;    // voxels per cell
constexpr int kN = 9;         // nodes per cell edge
constexpr int kNodes = 729;   // nodes per cell
constexpr int kTets = 3072;   // tetrahedra per cell
constexpr int kCh = 32;       // channels
constexpr int kOut = 24;      // output channels used (8 bases x 3 components)
constexpr int kTaps = 27;
constexpr int kCin0 = 4;
// parameter layout
constexpr int kW0 = 0;                                   // [27][32][4]
constexpr int kB0 = kTaps * kCh * kCin0;                 // [32]
constexpr int kL1 = kB0 + kCh;                           // layer l >= 1 at kL1 + (l - 1) * kLayer
constexpr int kLayerW = kTaps * kCh * kCh;               // [27][32 co][32 ci]
constexpr int kLayer = kLayerW + kCh;                    // weights + bias
constexpr int kParams = kL1 + 3 * kLayer;
constexpr int kPart0 = kL1;                              // first-layer weight-gradient partial
// conv kernel shared memory: a 4-plane halo of 18 x 18 voxel records (64 B) + the weights
constexpr int kHaloRec = 4 * 18 * 18;
constexpr int kConvSmem = kHaloRec * 64 + kTaps * kCh * 64;
constexpr int kWgradSmem = kHaloRec * 64 + 512 * 64;

__host__ __device__ constexpr int layer_base(int l) { return kL1 + (l - 1) * kLayer; }

// 16-byte chunk c of 64-byte record r: chunks XOR-swizzled by (r >> 1) & 3 so that eight
// consecutive records read at one chunk index hit eight different bank groups
__device__ __forceinline__ uint32_t swz(int rec, int chunk) { return rec * 64 + ((chunk ^ ((rec >> 1) & 3)) << 4); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], uint32_t addr)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], uint32_t addr)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g));
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// the halo of planes z0-1 .. z0+2 of one cell: 18 x 18 records per plane, zero outside the cell
__device__ __forceinline__ void load_halo(unsigned char* sm, const __nv_bfloat16* cell_base, int z0)
{
    for (int q = threadIdx.x; q < kHaloRec * 4; q += blockDim.x) {
        const int rec = q >> 2, c = q & 3;
        const int hz = rec / 324, rem = rec - hz * 324, hy = rem / 18, hx = rem - hy * 18;
        const int gz = z0 - 1 + hz, gy = hy - 1, gx = hx - 1;
        const uint32_t dst = smem_u32(sm) + swz(rec, c);
        if (gz >= 0 && gz < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV)
            cp_async16(dst, cell_base + ((size_t)((gz * kV + gy) * kV + gx) * kCh + c * 8));
        else
            *reinterpret_cast<uint4*>(sm + swz(rec, c)) = make_uint4(0, 0, 0, 0);
    }
}

// ------------------------------------------------------------------ layer 0 (4 -> 32, FP32)

__device__ __forceinline__ float coord_of(int i) { return (2.0f * i + 1.0f) / kV - 1.0f; }

__global__ void __launch_bounds__(256) k_first_fwd(const float* __restrict__ x, const float* __restrict__ p,
                                                   __nv_bfloat16* __restrict__ a0)
{
    __shared__ float xs[3][18][18];
    __shared__ float w[kTaps * kCh * kCin0 + kCh];
    const int z = blockIdx.x, cell = blockIdx.y, tid = threadIdx.x;
    const float* xc = x + (size_t)cell * kVox;
    for (int q = tid; q < 3 * 18 * 18; q += blockDim.x) {
        const int hz = q / 324, rem = q % 324, hy = rem / 18, hx = rem % 18;
        const int gz = z - 1 + hz, gy = hy - 1, gx = hx - 1;
        xs[hz][hy][hx] = (gz >= 0 && gz < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV) ? xc[(gz * kV + gy) * kV + gx] : 0.f;
    }
    for (int q = tid; q < kTaps * kCh * kCin0 + kCh; q += blockDim.x) w[q] = p[kW0 + q];
    __syncthreads();
    const int vx = tid & 15, vy = tid >> 4;
    float acc[kCh];
#pragma unroll
    for (int co = 0; co < kCh; co++) acc[co] = w[kB0 + co];
    for (int tap = 0; tap < kTaps; tap++) {
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
        const int gz = z + dz - 1, gy = vy + dy - 1, gx = vx + dx - 1;
        if (gz < 0 || gz >= kV || gy < 0 || gy >= kV || gx < 0 || gx >= kV) continue;
        const float in0 = xs[dz][vy + dy][vx + dx], in1 = coord_of(gx), in2 = coord_of(gy), in3 = coord_of(gz);
        const float* wt = w + tap * kCh * kCin0;
#pragma unroll
        for (int co = 0; co < kCh; co++)
            acc[co] += wt[4 * co] * in0 + wt[4 * co + 1] * in1 + wt[4 * co + 2] * in2 + wt[4 * co + 3] * in3;
    }
    __nv_bfloat162 o[kCh / 2];
#pragma unroll
    for (int k = 0; k < kCh / 2; k++) o[k] = __floats2bfloat162_rn(fmaxf(acc[2 * k], 0.f), fmaxf(acc[2 * k + 1], 0.f));
    uint4* dst = reinterpret_cast<uint4*>(a0 + ((size_t)cell * kVox + (z * kV + vy) * kV + vx) * kCh);
    const uint4* src = reinterpret_cast<const uint4*>(o);
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k] = src[k];
}

// dW0[tap][co][c] = sum_v dZ0[v][co] I[v + tap][c], db0[co] = sum_v dZ0[v][co]; one partial per CTA
__global__ void __launch_bounds__(256) k_first_wgrad(int n_cells, int cells_per_cta, const float* __restrict__ x,
                                                     const __nv_bfloat16* __restrict__ dz, float* __restrict__ part)
{
    __shared__ float xs[3][18][18];
    __shared__ float ds[256][kCh + 1];
    const int tid = threadIdx.x, co = tid & 31, tg = tid >> 5;
    float acc[4][kCin0];
    float accb = 0.f;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int c = 0; c < kCin0; c++) acc[i][c] = 0.f;
    const int c0 = blockIdx.x * cells_per_cta, c1 = min(n_cells, c0 + cells_per_cta);
    for (int cell = c0; cell < c1; cell++) {
        const float* xc = x + (size_t)cell * kVox;
        for (int z = 0; z < kV; z++) {
            __syncthreads();
            for (int q = tid; q < 3 * 18 * 18; q += blockDim.x) {
                const int hz = q / 324, rem = q % 324, hy = rem / 18, hx = rem % 18;
                const int gz = z - 1 + hz, gy = hy - 1, gx = hx - 1;
                xs[hz][hy][hx] =
                    (gz >= 0 && gz < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV) ? xc[(gz * kV + gy) * kV + gx] : 0.f;
            }
            const __nv_bfloat16* dzp = dz + ((size_t)cell * kVox + z * 256) * kCh;
            for (int q = tid; q < 256 * kCh; q += blockDim.x) ds[q >> 5][q & 31] = __bfloat162float(dzp[q]);
            __syncthreads();
            for (int v = 0; v < 256; v++) {
                const float d = ds[v][co];
                const int vx = v & 15, vy = v >> 4;
                accb += d;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int tap = tg + 8 * i;
                    if (tap >= kTaps) break;
                    const int dzt = tap / 9, dyt = (tap / 3) % 3, dxt = tap % 3;
                    const int gz = z + dzt - 1, gy = vy + dyt - 1, gx = vx + dxt - 1;
                    if (gz < 0 || gz >= kV || gy < 0 || gy >= kV || gx < 0 || gx >= kV) continue;
                    acc[i][0] += d * xs[dzt][vy + dyt][vx + dxt];
                    acc[i][1] += d * coord_of(gx);
                    acc[i][2] += d * coord_of(gy);
                    acc[i][3] += d * coord_of(gz);
                }
            }
        }
    }
    float* out = part + (size_t)blockIdx.x * kPart0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int tap = tg + 8 * i;
        if (tap >= kTaps) break;
#pragma unroll
        for (int c = 0; c < kCin0; c++) out[(tap * kCh + co) * kCin0 + c] = acc[i][c];
    }
    if (tg == 0) out[kB0 + co] = accb;
}

// ------------------------------------------------------------------ 32 -> 32 convolutions (tensor cores)

enum { kEpiRelu = 0, kEpiF32 = 1, kEpiMask = 2 };

// One CTA = two z-planes (512 voxels) of one cell; warp w owns the x-rows 4w .. 4w+3 (16 voxels
// each, one m16 tile) and all 32 output channels (four n8 tiles).  K = 27 taps x 32 input
// channels, walked as 54 k16 steps over the shared-memory halo (implicit GEMM).
//   kEpiRelu: out = bf16(relu(acc + bias))           (forward, hidden layers)
//   kEpiF32:  outf = acc + bias                      (forward, last layer)
//   kEpiMask: out = bf16(acc * (mask > 0))           (backward data: w holds the flipped,
//             transposed weights and mask the activations of the layer below)
template <int EPI>
__global__ void __launch_bounds__(256, 1) k_conv32(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                   const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
                                                   __nv_bfloat16* __restrict__ out, float* __restrict__ outf)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* halo = sm;
    unsigned char* ws = sm + kHaloRec * 64;
    const int slab = blockIdx.x, cell = blockIdx.y, tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    load_halo(halo, in + (size_t)cell * kVox * kCh, 2 * slab);
    for (int q = tid; q < kTaps * kCh * 4; q += blockDim.x) {
        const int row = q >> 2, c = q & 3;
        cp_async16(smem_u32(ws) + swz(row, c), w + (size_t)row * kCh + c * 8);
    }
    cp_async_wait_all();
    __syncthreads();

    float acc[4][4][4];
#pragma unroll
    for (int mt = 0; mt < 4; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[mt][nt][q] = 0.f;

    const uint32_t hb = smem_u32(halo), wb = smem_u32(ws);
    const int xa = (lane & 7) + 8 * ((lane >> 3) & 1), ka = lane >> 4;
    const int nb = lane & 7, ntoff = lane >> 4, kb = (lane >> 3) & 1;
    for (int tap = 0; tap < kTaps; tap++) {
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll
        for (int kc = 0; kc < 2; kc++) {
            uint32_t a[4][4];
#pragma unroll
            for (int mt = 0; mt < 4; mt++) {
                const int rr = 4 * warp + mt, zl = rr >> 4, y = rr & 15;
                const int rec = ((zl + dz) * 18 + (y + dy)) * 18 + (xa + dx);
                ldsm_x4(a[mt], hb + swz(rec, 2 * kc + ka));
            }
            uint32_t b[4][2];
#pragma unroll
            for (int pr = 0; pr < 2; pr++) {
                uint32_t r[4];
                const int row = tap * kCh + 8 * (2 * pr + ntoff) + nb;
                ldsm_x4(r, wb + swz(row, 2 * kc + kb));
                b[2 * pr][0] = r[0];
                b[2 * pr][1] = r[1];
                b[2 * pr + 1][0] = r[2];
                b[2 * pr + 1][1] = r[3];
            }
#pragma unroll
            for (int mt = 0; mt < 4; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++) mma16816(acc[mt][nt], a[mt], b[nt][0], b[nt][1]);
        }
    }

    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 4; mt++) {
        const int rr = 4 * warp + mt, z = 2 * slab + (rr >> 4), y = rr & 15;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int xv = g + 8 * h;
            const size_t vox = (size_t)cell * kVox + (z * kV + y) * kV + xv;
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                const int co = 8 * nt + 2 * t;
                float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
                if (EPI == kEpiF32) {
                    *reinterpret_cast<float2*>(outf + vox * kCh + co) = make_float2(v0 + bias[co], v1 + bias[co + 1]);
                } else {
                    if (EPI == kEpiRelu) {
                        v0 = fmaxf(v0 + bias[co], 0.f);
                        v1 = fmaxf(v1 + bias[co + 1], 0.f);
                    } else {
                        const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(mask + vox * kCh + co);
                        v0 = __bfloat162float(m.x) > 0.f ? v0 : 0.f;
                        v1 = __bfloat162float(m.y) > 0.f ? v1 : 0.f;
                    }
                    *reinterpret_cast<__nv_bfloat162*>(out + vox * kCh + co) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
    }
}

// ---- the same convolution on the 5th-generation tensor cores (tcgen05, accumulators in TMEM).
// One CTA (4 warps) per cell walks its 16 z-planes.  Per plane the GEMM is D[256 voxels][32] =
// sum over 27 taps x 2 k16 steps of A_tap[256][16] B_tap[16][32], issued by one thread as 4
// M = 64 tiles (8 y rows x 8 x of one x-half) x 54 tcgen05.mma (kind::f16, BF16 in, FP32
// accumulate, N = 32).  Operands come from shared memory through K-major, no-swizzle descriptors
// (8-row x 16-byte core matrices): a tile's core matrix g is y row g, 8 consecutive x records, so
// every tap is the same descriptor with its start moved by (dy, dx) records -- the halo is stored
// once per plane, [16-byte channel chunk][18 y][18 x] (x and y from -1 to 16, zero outside), in
// a ring of 4 plane slots; the weights as [chunk][tap][co].  The ring lets the loads of plane
// z + 2 overlap the MMAs and the epilogue of plane z.  TMEM: x-half h at lane offset 16 h (the
// M = 64 accumulator layout: row m in lane m % 16 + 32 (m / 16)), y block b at column 32 b.
// Completion is signalled on an mbarrier through tcgen05.commit; every wait on it is bounded (a
// timeout sets *err and skips the epilogue).  The epilogue reads one voxel's 32 channels per
// thread with tcgen05.ld and writes its 64 (BF16) or 128 (FP32) contiguous bytes.
constexpr int kTcRow = 18 * 16;                            // one y row of records (bytes)
constexpr int kTcChunk = 18 * kTcRow;                      // 5,184 B: one channel chunk of a plane
constexpr int kTcSlot = 4 * kTcChunk;                      // 20,736 B: one plane
constexpr int kTcA = 4 * kTcSlot;                          // 82,944 B: the ring
constexpr int kTcB = 4 * kTaps * kCh * 16;                 // 55,296 B
constexpr int kTcSmem = kTcA + kTcB + 16;                  // + mbarrier + TMEM address
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCh >> 3) << 17) | ((uint32_t)(64 >> 4) << 24);

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 22); i++) {
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

// plane gz of one cell into ring slot `slot`: [chunk][18 y][18 x] records, zero outside the cell
__device__ __forceinline__ void tc_load_plane(unsigned char* A, const __nv_bfloat16* cell_base, int gz, int slot)
{
    for (int q = threadIdx.x; q < 4 * 18 * 18; q += blockDim.x) {
        const int c = q / 324, hy = (q / 18) % 18, hx = q % 18;
        const int gy = hy - 1, gx = hx - 1;
        const uint32_t off = slot * kTcSlot + c * kTcChunk + (hy * 18 + hx) * 16;
        if (gz >= 0 && gz < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV)
            cp_async16(smem_u32(A) + off, cell_base + ((size_t)((gz * kV + gy) * kV + gx) * kCh + c * 8));
        else
            *reinterpret_cast<uint4*>(A + off) = make_uint4(0, 0, 0, 0);
    }
}

template <int EPI>
__global__ void __launch_bounds__(128, 1) k_conv32_tc(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                      const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
                                                      __nv_bfloat16* __restrict__ out, float* __restrict__ outf, int* err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* A = sm;
    unsigned char* B = sm + kTcA;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kTcA + kTcB);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTcA + kTcB + 8);
    const int cell = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const __nv_bfloat16* inc = in + (size_t)cell * kVox * kCh;
    const uint32_t bar = smem_u32(mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;\n" ::"r"(smem_u32(tslot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    // weights [chunk][tap][co] x 16 B from w[tap][co][ci]
    for (int q = tid; q < kTaps * kCh * 4; q += blockDim.x) {
        const int row = q >> 2, c = q & 3;
        cp_async16(smem_u32(B) + (c * kTaps * kCh + row) * 16, w + (size_t)row * kCh + c * 8);
    }
    // planes -1, 0, 1 in slots 0, 1, 2 (plane gz lives in slot (gz + 1) % 4)
    tc_load_plane(A, inc, -1, 0);
    tc_load_plane(A, inc, 0, 1);
    tc_load_plane(A, inc, 1, 2);
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tbase = *tslot;
    const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
    // this thread's accumulator row: x-half h = lane / 16, row m = 16 warp + lane % 16 of the tile
    const int h = lane >> 4, m = 16 * warp + (lane & 15);
    bool ok = true;
    for (int z = 0; z < kV; z++) {
        if (tid == 0 && ok) {
            for (int yb = 0; yb < 2; yb++)
                for (int hh = 0; hh < 2; hh++)
                    for (int tap = 0; tap < kTaps; tap++) {
                        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3, slot = (z + dz) & 3;
                        for (int kc = 0; kc < 2; kc++) {
                            const uint32_t aoff = slot * kTcSlot + 2 * kc * kTcChunk + ((8 * yb + dy) * 18 + 8 * hh + dx) * 16;
                            const uint32_t boff = (2 * kc * kTaps + tap) * kCh * 16;
                            tc_mma(tbase + ((uint32_t)(16 * hh) << 16) + 32 * yb, tc_desc(a0 + aoff, kTcChunk, kTcRow),
                                   tc_desc(b0 + boff, kTaps * kCh * 16, 128), (tap | kc) != 0);
                        }
                    }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
        }
        // plane z + 2 into the slot plane z - 2 used (its MMAs finished in the previous step)
        tc_load_plane(A, inc, z + 2, (z + 3) & 3);
        ok = ok && tc_wait(bar, z & 1);
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        if (ok) {
#pragma unroll
            for (int yb = 0; yb < 2; yb++) {
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                    "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                      "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                      "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(tbase + ((uint32_t)(32 * warp) << 16) + 32 * yb));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                const int y = 8 * yb + (m >> 3), xv = 8 * h + (m & 7);
                const size_t vox = (size_t)cell * kVox + (z * kV + y) * kV + xv;
                if (EPI == kEpiF32) {
                    float4* o = reinterpret_cast<float4*>(outf + vox * kCh);
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        o[k] = make_float4(__uint_as_float(v[4 * k]) + bias[4 * k], __uint_as_float(v[4 * k + 1]) + bias[4 * k + 1],
                                           __uint_as_float(v[4 * k + 2]) + bias[4 * k + 2], __uint_as_float(v[4 * k + 3]) + bias[4 * k + 3]);
                } else {
                    __nv_bfloat162 hv[16];
                    if (EPI == kEpiRelu) {
#pragma unroll
                        for (int k = 0; k < 16; k++)
                            hv[k] = __floats2bfloat162_rn(fmaxf(__uint_as_float(v[2 * k]) + bias[2 * k], 0.f),
                                                          fmaxf(__uint_as_float(v[2 * k + 1]) + bias[2 * k + 1], 0.f));
                    } else {
                        uint4 mm[4];
                        const uint4* mp = reinterpret_cast<const uint4*>(mask + vox * kCh);
#pragma unroll
                        for (int k = 0; k < 4; k++) mm[k] = mp[k];
                        const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(mm);
#pragma unroll
                        for (int k = 0; k < 16; k++)
                            hv[k] = __floats2bfloat162_rn(__bfloat162float(m2[k].x) > 0.f ? __uint_as_float(v[2 * k]) : 0.f,
                                                          __bfloat162float(m2[k].y) > 0.f ? __uint_as_float(v[2 * k + 1]) : 0.f);
                    }
                    uint4* o = reinterpret_cast<uint4*>(out + vox * kCh);
                    const uint4* hs = reinterpret_cast<const uint4*>(hv);
#pragma unroll
                    for (int k = 0; k < 4; k++) o[k] = hs[k];
                }
            }
        }
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;\n" ::"r"(tbase));
}

// ---- the transposed product on tcgen05: D^T[co][voxel] = sum_tap W_tap^T[co][ci] A_tap^T[ci][voxel].
// One instruction now covers a whole plane: M = 64 (the 32 output channels; rows 32-63 read the
// next tap's weights and are never used), N = 256 voxels, K = 16 -- 54 per plane instead of 216.
// The N operand must be 256 rows of 16 bytes at one stride for every tap, so the halo is kept as
// three x-shifted copies: a plane slot is [dx][chunk][18 y][16 x] x 16 B, three slots in a ring.
// The weights stay [chunk][tap][co] x 16 B (plus 1 KB of zero slack read by the unused rows of
// the last tap).  TMEM holds D^T as 64 lanes (row m in lane m % 16 + 32 (m / 16)) x 256 columns:
// the channels of warps 0 and 1, lanes 0-15.  The epilogue reads them with tcgen05.ld, stages the
// plane as [voxel][channel] in the ring slot that just went out of use, and copies it out with
// 16-byte stores.
constexpr int kTtPlane = 3 * 4 * 18 * 16 * 16;            // 55,296 B: one plane slot
constexpr int kTtDx = 4 * 18 * 16 * 16;                   // 18,432 B between x-shifted copies
constexpr int kTtChunk = 18 * 16 * 16;                    // 4,608 B between channel chunks
constexpr int kTtA = 3 * kTtPlane;                        // 165,888 B: the ring
constexpr int kTtW = kTaps * kCh * 4 * 16 + 1024;         // 56,320 B: weights + slack
constexpr int kTtSmem = kTtA + kTtW + 16;
constexpr uint32_t kTtIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(64 >> 4) << 24);

__device__ __forceinline__ void tt_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(kTtIdesc), "r"(accumulate));
}

// plane gz of one cell into ring slot `slot` as three x-shifted copies, zero outside the cell
__device__ __forceinline__ void tt_load_plane(unsigned char* A, const __nv_bfloat16* cell_base, int gz, int slot)
{
    for (int q = threadIdx.x; q < 3 * 4 * 18 * 16; q += blockDim.x) {
        const int x = q & 15, hy = (q >> 4) % 18, c = (q / (18 * 16)) & 3, dx = q / (4 * 18 * 16);
        const int gy = hy - 1, gx = x + dx - 1;
        const uint32_t off = slot * kTtPlane + dx * kTtDx + c * kTtChunk + (hy * 16 + x) * 16;
        if (gz >= 0 && gz < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV)
            cp_async16(smem_u32(A) + off, cell_base + ((size_t)((gz * kV + gy) * kV + gx) * kCh + c * 8));
        else
            *reinterpret_cast<uint4*>(A + off) = make_uint4(0, 0, 0, 0);
    }
}

template <int EPI>
__global__ void __launch_bounds__(128, 1) k_conv32_tt(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                      const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
                                                      __nv_bfloat16* __restrict__ out, float* __restrict__ outf, int* err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* A = sm;
    unsigned char* W = sm + kTtA;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kTtA + kTtW);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTtA + kTtW + 8);
    const int cell = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const __nv_bfloat16* inc = in + (size_t)cell * kVox * kCh;
    const uint32_t bar = smem_u32(mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;\n" ::"r"(smem_u32(tslot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    for (int q = tid; q < kTaps * kCh * 4; q += blockDim.x) {
        const int row = q >> 2, c = q & 3;
        cp_async16(smem_u32(W) + (c * kTaps * kCh + row) * 16, w + (size_t)row * kCh + c * 8);
    }
    for (int q = tid; q < 64; q += blockDim.x)
        *reinterpret_cast<uint4*>(W + kTaps * kCh * 4 * 16 + 16 * q) = make_uint4(0, 0, 0, 0);
    // planes -1, 0, 1 in slots 0, 1, 2 (plane gz in slot (gz + 1) % 3)
    tt_load_plane(A, inc, -1, 0);
    tt_load_plane(A, inc, 0, 1);
    tt_load_plane(A, inc, 1, 2);
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tbase = *tslot;
    const uint32_t a0 = smem_u32(A), w0 = smem_u32(W);
    bool ok = true;
    for (int z = 0; z < kV; z++) {
        if (tid == 0 && ok) {
            for (int tap = 0; tap < kTaps; tap++) {
                const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3, slot = (z + dz) % 3;
                for (int kc = 0; kc < 2; kc++) {
                    const uint32_t woff = (2 * kc * kTaps + tap) * kCh * 16;
                    const uint32_t aoff = slot * kTtPlane + dx * kTtDx + 2 * kc * kTtChunk + dy * 16 * 16;
                    tt_mma(tbase, tc_desc(w0 + woff, kTaps * kCh * 16, 128), tc_desc(a0 + aoff, kTtChunk, 128),
                           (tap | kc) != 0);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
        }
        ok = ok && tc_wait(bar, z & 1);
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        // stage the plane in the slot of plane z - 1 (no longer read): [voxel][channel]
        unsigned char* T = A + (z % 3) * kTtPlane;
        if (ok && warp < 2) {
            const int co = 16 * warp + (lane & 15);
#pragma unroll 1
            for (int cb = 0; cb < 8; cb++) {
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                    "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                      "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                      "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(tbase + ((uint32_t)(32 * warp) << 16) + 32 * cb));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (lane < 16) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const int vox = 32 * cb + j;
                        const float a = __uint_as_float(v[j]);
                        if (EPI == kEpiF32) {
                            reinterpret_cast<float*>(T)[vox * kCh + co] = a + bias[co];
                        } else {
                            const float r = EPI == kEpiRelu ? fmaxf(a + bias[co], 0.f) : a;
                            reinterpret_cast<__nv_bfloat16*>(T)[vox * kCh + co] = __float2bfloat16_rn(r);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (ok) {
            // copy out: 256 voxel records of 64 B (BF16) or 128 B (FP32), 16-byte stores
            const size_t vbase = (size_t)cell * kVox + (size_t)z * 256;
            if (EPI == kEpiF32) {
                for (int q = tid; q < 256 * 8; q += blockDim.x)
                    reinterpret_cast<uint4*>(outf + vbase * kCh)[q] = reinterpret_cast<const uint4*>(T)[q];
            } else {
                for (int q = tid; q < 256 * 4; q += blockDim.x) {
                    uint4 val = reinterpret_cast<const uint4*>(T)[q];
                    if (EPI == kEpiMask) {
                        const uint4 mm = reinterpret_cast<const uint4*>(mask + vbase * kCh)[q];
                        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&val);
                        const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(&mm);
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            const __nv_bfloat162 zero = __floats2bfloat162_rn(0.f, 0.f);
                            h[k].x = __bfloat162float(m2[k].x) > 0.f ? h[k].x : zero.x;
                            h[k].y = __bfloat162float(m2[k].y) > 0.f ? h[k].y : zero.y;
                        }
                    }
                    reinterpret_cast<uint4*>(out + vbase * kCh)[q] = val;
                }
            }
        }
        __syncthreads();
        // plane z + 2 into the slot just used for staging (plane z - 1's)
        tt_load_plane(A, inc, z + 2, z % 3);
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;\n" ::"r"(tbase));
}

// ---- the M = 64 tcgen05 convolution, warp-specialised and persistent.
// Operands and tiles as k_conv32_tc (planes stored once as [chunk][18 y][18 x] records, weights
// [chunk][tap][co], per plane 4 M = 64 tiles x 27 taps x 2 k16 steps into TMEM), but the three
// stages run in different warps and overlap:
//   warp 4       producer: copies planes -1 .. 16 of each cell into a ring of kWsSlots plane
//                slots (cp.async; zeros outside the cell), then arrives on the slot's `full`
//                barrier; it reuses a slot only after the MMAs that read it have completed
//                (`empty`, signalled by tcgen05.commit);
//   warp 5       one thread issues the plane's 216 tcgen05.mma into one of two TMEM accumulator
//                buffers (64 columns each), commits them to `accf[b]` and releases the plane slot
//                no later MMA reads;
//   warps 0-3    epilogue: each reads its quadrant of TMEM lanes (tcgen05.ld), hands the buffer
//                back (`acce[b]`), adds the bias / applies ReLU or the mask and stores the voxels.
// So the loads of the next planes and the epilogue of plane z overlap the MMAs of plane z + 1.
// One CTA per SM walks cells blockIdx.x, + gridDim.x, ... with the weights loaded once.  Every
// wait is bounded: a timeout sets *err, raises a shared abort flag that every role polls, and
// the CTA still waits (bounded) for its issued MMAs before it frees TMEM.
constexpr int kWsSlots = 6;
constexpr int kWsA = kWsSlots * kTcSlot;                   // 124,416 B
constexpr int kWsBar = kWsA + kTcB;                         // barriers after ring and weights
constexpr int kWsNBar = 2 * kWsSlots + 2 + 2 + 1;           // full, empty, accf, acce, fin
constexpr int kWsSmem = kWsBar + 8 * kWsNBar + 16;
constexpr int kWsThreads = 192;
constexpr int kWsTmemCols = 128;

__device__ __forceinline__ void mb_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mb_arrive(uint32_t bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

// bounded wait on phase `parity` of `bar`; gives up early when another role raised *abort
__device__ __forceinline__ bool ws_wait(uint32_t bar, uint32_t parity, volatile int* abort)
{
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255) == 255 && *abort) return false;
    }
    *abort = 1;
    return false;
}

template <int EPI>
__global__ void __launch_bounds__(kWsThreads, 1) k_conv32_ws(int n_cells, const __nv_bfloat16* __restrict__ in,
                                                             const __nv_bfloat16* __restrict__ w,
                                                             const float* __restrict__ bias,
                                                             const __nv_bfloat16* __restrict__ mask,
                                                             __nv_bfloat16* __restrict__ out, float* __restrict__ outf,
                                                             int* err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* A = sm;
    unsigned char* B = sm + kWsA;
    const uint32_t bar0 = smem_u32(sm + kWsBar);
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (kWsSlots + s); };
    auto accf = [&](int b) { return bar0 + 8u * (2 * kWsSlots + b); };
    auto acce = [&](int b) { return bar0 + 8u * (2 * kWsSlots + 2 + b); };
    const uint32_t fin = bar0 + 8u * (2 * kWsSlots + 4);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kWsBar + 8 * kWsNBar);
    volatile int* abort = reinterpret_cast<volatile int*>(sm + kWsBar + 8 * kWsNBar + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < kWsSlots; s++) {
            mb_init(full(s), 32);
            mb_init(empty(s), 1);
        }
        for (int b = 0; b < 2; b++) {
            mb_init(accf(b), 1);
            mb_init(acce(b), 128);
        }
        mb_init(fin, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(kWsTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    // weights [chunk][tap][co] x 16 B from w[tap][co][ci], once for all the CTA's cells
    for (int q = tid; q < kTaps * kCh * 4; q += blockDim.x) {
        const int row = q >> 2, c = q & 3;
        cp_async16(smem_u32(B) + (c * kTaps * kCh + row) * 16, w + (size_t)row * kCh + c * 8);
    }
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tbase = *tslot;
    const int my_cells = blockIdx.x < n_cells ? (n_cells - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == 4) {
        // ---- producer: planes -1 .. 16 of each cell, plane g of the CTA in slot g % kWsSlots
        for (int k = 0; k < my_cells && !*abort; k++) {
            const __nv_bfloat16* inc = in + (size_t)(blockIdx.x + (size_t)k * gridDim.x) * kVox * kCh;
            for (int p = -1; p <= kV; p++) {
                const int g = 18 * k + p + 1, s = g % kWsSlots, use = g / kWsSlots;
                if (use > 0 && !ws_wait(empty(s), (use - 1) & 1, abort)) break;
                for (int q = lane; q < 4 * 18 * 18; q += 32) {
                    const int c = q / 324, hy = (q / 18) % 18, hx = q % 18;
                    const int gy = hy - 1, gx = hx - 1;
                    const uint32_t off = s * kTcSlot + c * kTcChunk + (hy * 18 + hx) * 16;
                    if (p >= 0 && p < kV && gy >= 0 && gy < kV && gx >= 0 && gx < kV)
                        cp_async16(smem_u32(A) + off, inc + ((size_t)((p * kV + gy) * kV + gx) * kCh + c * 8));
                    else
                        *reinterpret_cast<uint4*>(A + off) = make_uint4(0, 0, 0, 0);
                }
                cp_async_wait_all();
                asm volatile("fence.proxy.async.shared::cta;\n" ::);
                mb_arrive(full(s));
            }
        }
    } else if (warp == 5) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
            int issued = 0;
            for (int k = 0; k < my_cells && !*abort; k++) {
                bool ok = true;
                for (int z = 0; z < kV && ok; z++) {
                    // planes z - 1, z, z + 1 of the cell: g = 18 k + z .. 18 k + z + 2
                    for (int g = 18 * k + (z == 0 ? 0 : z + 2); g <= 18 * k + z + 2 && ok; g++)
                        ok = ws_wait(full(g % kWsSlots), (g / kWsSlots) & 1, abort);
                    const int t = 16 * k + z, b = t & 1, use = t >> 1;
                    if (ok && use > 0) ok = ws_wait(acce(b), (use - 1) & 1, abort);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                    const uint32_t dcol = tbase + 64u * b;
                    for (int yb = 0; yb < 2; yb++)
                        for (int hh = 0; hh < 2; hh++)
                            for (int tap = 0; tap < kTaps; tap++) {
                                const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                                const int slot = (18 * k + z + dz) % kWsSlots;
                                for (int kc = 0; kc < 2; kc++) {
                                    const uint32_t aoff =
                                        slot * kTcSlot + 2 * kc * kTcChunk + ((8 * yb + dy) * 18 + 8 * hh + dx) * 16;
                                    const uint32_t boff = (2 * kc * kTaps + tap) * kCh * 16;
                                    tc_mma(dcol + ((uint32_t)(16 * hh) << 16) + 32 * yb,
                                           tc_desc(a0 + aoff, kTcChunk, kTcRow), tc_desc(b0 + boff, kTaps * kCh * 16, 128),
                                           (tap | kc) != 0);
                                }
                            }
                    issued = 1;
                    tc_commit(accf(b));
                    // plane z - 1 is read by no later MMA; after the last plane, neither are z, z + 1
                    tc_commit(empty((18 * k + z) % kWsSlots));
                    if (z == kV - 1) {
                        tc_commit(empty((18 * k + z + 1) % kWsSlots));
                        tc_commit(empty((18 * k + z + 2) % kWsSlots));
                    }
                }
            }
            // every issued MMA has completed before the CTA frees TMEM
            if (issued) {
                tc_commit(fin);
                if (!ws_wait(fin, 0, abort)) {
                    // the bounded wait gave up: wait once more without the abort shortcut
                    for (int i = 0; i < (1 << 22); i++) {
                        uint32_t done;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                            "selp.b32 %0, 1, 0, p;\n\t}\n"
                            : "=r"(done)
                            : "r"(fin)
                            : "memory");
                        if (done) break;
                    }
                }
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp q reads TMEM lanes 32 q .. 32 q + 31 (tile rows m = 16 q + lane % 16
        // of x-half lane / 16), both y blocks of one plane per accumulator buffer
        const int h = lane >> 4, m = 16 * warp + (lane & 15);
        for (int k = 0; k < my_cells && !*abort; k++) {
            const int cell = blockIdx.x + k * gridDim.x;
            for (int z = 0; z < kV; z++) {
                const int t = 16 * k + z, b = t & 1;
                if (!ws_wait(accf(b), (t >> 1) & 1, abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                uint32_t v[2][32];
#pragma unroll
                for (int yb = 0; yb < 2; yb++)
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                        : "=r"(v[yb][0]), "=r"(v[yb][1]), "=r"(v[yb][2]), "=r"(v[yb][3]), "=r"(v[yb][4]), "=r"(v[yb][5]),
                          "=r"(v[yb][6]), "=r"(v[yb][7]), "=r"(v[yb][8]), "=r"(v[yb][9]), "=r"(v[yb][10]), "=r"(v[yb][11]),
                          "=r"(v[yb][12]), "=r"(v[yb][13]), "=r"(v[yb][14]), "=r"(v[yb][15]), "=r"(v[yb][16]),
                          "=r"(v[yb][17]), "=r"(v[yb][18]), "=r"(v[yb][19]), "=r"(v[yb][20]), "=r"(v[yb][21]),
                          "=r"(v[yb][22]), "=r"(v[yb][23]), "=r"(v[yb][24]), "=r"(v[yb][25]), "=r"(v[yb][26]),
                          "=r"(v[yb][27]), "=r"(v[yb][28]), "=r"(v[yb][29]), "=r"(v[yb][30]), "=r"(v[yb][31])
                        : "r"(tbase + ((uint32_t)(32 * warp) << 16) + 64u * b + 32 * yb));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
                mb_arrive(acce(b));  // the buffer is free for the MMAs of plane z + 2
#pragma unroll
                for (int yb = 0; yb < 2; yb++) {
                    const int y = 8 * yb + (m >> 3), xv = 8 * h + (m & 7);
                    const size_t vox = (size_t)cell * kVox + (z * kV + y) * kV + xv;
                    if (EPI == kEpiF32) {
                        float4* o = reinterpret_cast<float4*>(outf + vox * kCh);
#pragma unroll
                        for (int q = 0; q < 8; q++)
                            o[q] = make_float4(__uint_as_float(v[yb][4 * q]) + bias[4 * q],
                                               __uint_as_float(v[yb][4 * q + 1]) + bias[4 * q + 1],
                                               __uint_as_float(v[yb][4 * q + 2]) + bias[4 * q + 2],
                                               __uint_as_float(v[yb][4 * q + 3]) + bias[4 * q + 3]);
                    } else {
                        __nv_bfloat162 hv[16];
                        if (EPI == kEpiRelu) {
#pragma unroll
                            for (int q = 0; q < 16; q++)
                                hv[q] = __floats2bfloat162_rn(fmaxf(__uint_as_float(v[yb][2 * q]) + bias[2 * q], 0.f),
                                                              fmaxf(__uint_as_float(v[yb][2 * q + 1]) + bias[2 * q + 1], 0.f));
                        } else {
                            uint4 mm[4];
                            const uint4* mp = reinterpret_cast<const uint4*>(mask + vox * kCh);
#pragma unroll
                            for (int q = 0; q < 4; q++) mm[q] = mp[q];
                            const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(mm);
#pragma unroll
                            for (int q = 0; q < 16; q++)
                                hv[q] = __floats2bfloat162_rn(
                                    __bfloat162float(m2[q].x) > 0.f ? __uint_as_float(v[yb][2 * q]) : 0.f,
                                    __bfloat162float(m2[q].y) > 0.f ? __uint_as_float(v[yb][2 * q + 1]) : 0.f);
                        }
                        uint4* o = reinterpret_cast<uint4*>(out + vox * kCh);
                        const uint4* hs = reinterpret_cast<const uint4*>(hv);
#pragma unroll
                        for (int q = 0; q < 4; q++) o[q] = hs[q];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (*abort && tid == 0) atomicExch(err, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(kWsTmemCols));
}

// dW[tap][co][ci] = sum_v dZ[v][co] A[v + tap][ci] and db[co] = sum_v dZ[v][co] over the cells of
// this CTA (one fixed-order partial per CTA).  M = co (two m16 tiles, A operand = dZ^T through
// ldmatrix.trans), N = ci (four n8 tiles, B operand = shifted activations through ldmatrix.trans),
// K = voxels (16 per step: one x-row).  Warp w owns the taps w, w + 8, w + 16, w + 24 (< 27).
__global__ void __launch_bounds__(256, 1) k_wgrad32(int n_cells, int cells_per_cta, const __nv_bfloat16* __restrict__ act,
                                                    const __nv_bfloat16* __restrict__ dz, float* __restrict__ part)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* halo = sm;
    unsigned char* ds = sm + kHaloRec * 64;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntap = warp < 3 ? 4 : 3;
    float acc[4][2][4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][mt][nt][q] = 0.f;
    float accb = 0.f;
    const uint32_t hb = smem_u32(halo), db = smem_u32(ds);
    const int lr = lane & 7, lj = lane >> 3;
    const int c0 = blockIdx.x * cells_per_cta, c1 = min(n_cells, c0 + cells_per_cta);
    for (int cell = c0; cell < c1; cell++) {
        for (int slab = 0; slab < 8; slab++) {
            __syncthreads();
            load_halo(halo, act + (size_t)cell * kVox * kCh, 2 * slab);
            const __nv_bfloat16* dzp = dz + ((size_t)cell * kVox + slab * 512) * kCh;
            for (int q = tid; q < 512 * 4; q += blockDim.x) cp_async16(db + swz(q >> 2, q & 3), dzp + (size_t)q * 8);
            cp_async_wait_all();
            __syncthreads();
            {   // bias: thread (co = lane, voxels warp, warp + 8, ...)
                for (int v = warp; v < 512; v += 8) {
                    const __nv_bfloat16* r = reinterpret_cast<const __nv_bfloat16*>(ds + swz(v, lane >> 3));
                    accb += __bfloat162float(r[lane & 7]);
                }
            }
            for (int rr = 0; rr < 32; rr++) {
                const int zl = rr >> 4, y = rr & 15;
                uint32_t a[2][4];
#pragma unroll
                for (int mt = 0; mt < 2; mt++) {
                    const int xv = lr + 8 * (lj >> 1);
                    ldsm_x4_t(a[mt], db + swz(rr * 16 + xv, 2 * mt + (lj & 1)));
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (i >= ntap) break;
                    const int tap = warp + 8 * i;
                    const int dzt = tap / 9, dyt = (tap / 3) % 3, dxt = tap % 3;
                    uint32_t b[4][2];
#pragma unroll
                    for (int pr = 0; pr < 2; pr++) {
                        uint32_t r[4];
                        const int xv = lr + 8 * (lj & 1);
                        const int rec = ((zl + dzt) * 18 + (y + dyt)) * 18 + (xv + dxt);
                        ldsm_x4_t(r, hb + swz(rec, 2 * pr + (lj >> 1)));
                        b[2 * pr][0] = r[0];
                        b[2 * pr][1] = r[1];
                        b[2 * pr + 1][0] = r[2];
                        b[2 * pr + 1][1] = r[3];
                    }
#pragma unroll
                    for (int mt = 0; mt < 2; mt++)
#pragma unroll
                        for (int nt = 0; nt < 4; nt++) mma16816(acc[i][mt][nt], a[mt], b[nt][0], b[nt][1]);
                }
            }
        }
    }
    float* out = part + (size_t)blockIdx.x * kLayer;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i >= ntap) break;
        const int tap = warp + 8 * i;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                const int ci = 8 * nt + 2 * t;
                const int co0 = 16 * mt + g, co1 = co0 + 8;
                *reinterpret_cast<float2*>(out + (tap * kCh + co0) * kCh + ci) = make_float2(acc[i][mt][nt][0], acc[i][mt][nt][1]);
                *reinterpret_cast<float2*>(out + (tap * kCh + co1) * kCh + ci) = make_float2(acc[i][mt][nt][2], acc[i][mt][nt][3]);
            }
    }
    // bias partials: 8 warps x 32 channels, summed in warp order
    __shared__ float sb[8][32];
    sb[warp][lane] = accb;
    __syncthreads();
    if (tid < 32) {
        float s = 0.f;
        for (int k = 0; k < 8; k++) s += sb[k][tid];
        out[kLayerW + tid] = s;
    }
}

// out[i] = sum_p part[p][i] in p order
__global__ void k_reduce_parts(int n_parts, int len, const float* __restrict__ part, float* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int p = 0; p < n_parts; p++) s += part[(size_t)p * len + i];
        out[i] = s;
    }
}

// ------------------------------------------------------------------ loss, nodes, bases

__device__ __forceinline__ int node_count(int i) { return (i == 0 || i == kN - 1) ? 1 : 2; }
__device__ __forceinline__ bool is_vertex(int i, int j, int k)
{
    return (i == 0 || i == kN - 1) && (j == 0 || j == kN - 1) && (k == 0 || k == kN - 1);
}

// corr of node (i, j, k), channel ch, from the voxel outputs of one cell
__device__ __forceinline__ float node_corr(const float* __restrict__ o, int i, int j, int k, int ch)
{
    if (is_vertex(i, j, k)) return 0.f;
    float s = 0.f;
    for (int c = max(0, 2 * k - 1); c <= min(kV - 1, 2 * k); c++)
        for (int b = max(0, 2 * j - 1); b <= min(kV - 1, 2 * j); b++)
            for (int a = max(0, 2 * i - 1); a <= min(kV - 1, 2 * i); a++) s += o[((c * kV + b) * kV + a) * kCh + ch];
    return s / (float)(node_count(i) * node_count(j) * node_count(k));
}

// per cell: sum of (corr - y)^2 into lossp[cell]; gnode = d loss / d corr (times the node mask)
__global__ void __launch_bounds__(256) k_loss_nodes(const float* __restrict__ o, const float* __restrict__ y,
                                                    float inv_norm, float* __restrict__ gnode, float* __restrict__ lossp)
{
    const int cell = blockIdx.x;
    const float* oc = o + (size_t)cell * kVox * kCh;
    float s = 0.f;
    for (int q = threadIdx.x; q < kNodes * kOut; q += blockDim.x) {
        const int n = q / kOut, ch = q - n * kOut;
        const int i = n % kN, j = (n / kN) % kN, k = n / (kN * kN);
        const float d = node_corr(oc, i, j, k, ch) - y[(size_t)cell * kNodes * kOut + q];
        s += d * d;
        gnode[(size_t)cell * kNodes * kOut + q] =
            is_vertex(i, j, k) ? 0.f : 2.f * d * inv_norm / (float)(node_count(i) * node_count(j) * node_count(k));
    }
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) lossp[cell] = red[0];
}

// d loss / d L3 output (BF16, channels >= 24 zero): each voxel belongs to one node
__global__ void k_dout(int n_cells, const float* __restrict__ gnode, __nv_bfloat16* __restrict__ d)
{
    const int64_t total = (int64_t)n_cells * kVox * kCh;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q & 31);
        const int64_t v = q >> 5;
        const int cell = (int)(v / kVox), vl = (int)(v % kVox);
        const int vx = vl & 15, vy = (vl >> 4) & 15, vz = vl >> 8;
        const int n = ((vx + 1) >> 1) + kN * (((vy + 1) >> 1) + kN * ((vz + 1) >> 1));
        d[q] = __float2bfloat16_rn(ch < kOut ? gnode[((size_t)cell * kNodes + n) * kOut + ch] : 0.f);
    }
}

__global__ void k_loss_sum(int n, const float* __restrict__ lossp, float inv_norm, float* __restrict__ out)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += lossp[i];
        *out = (float)(s * inv_norm);
    }
}

__device__ __forceinline__ float q1(int v, int i, int j, int k)
{
    const float tx = i / 8.0f, ty = j / 8.0f, tz = k / 8.0f;
    return ((v & 1) ? tx : 1.f - tx) * ((v & 2) ? ty : 1.f - ty) * ((v & 4) ? tz : 1.f - tz);
}

// cells whose bases leave [-3, 3] (the bound the two-level coarse build applies: a nearly
// singular cell problem of the reference's indefinite operator): their target is the trilinear
// space itself (zero correction), as the coarse space would use it
__global__ void k_wild_targets(int c_first, const int64_t* __restrict__ node_off, const double* __restrict__ bx,
                               uint8_t* __restrict__ wild)
{
    const int c = blockIdx.x;
    int bad = 0;
    for (int64_t q = 24 * node_off[c_first + c] + threadIdx.x; q < 24 * node_off[c_first + c + 1]; q += blockDim.x)
        bad |= !(fabs(bx[q]) <= 3.0);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) wild[c] = (uint8_t)(bad != 0);
}

// targets y[cell][node][3 v + a] = psi_exact - Q1 from the cells' current bases (0 for wild cells)
__global__ void k_targets(int n_cells, int c_first, const int64_t* __restrict__ node_off, const double* __restrict__ bx,
                          const uint8_t* __restrict__ wild, float* __restrict__ y)
{
    const int64_t total = (int64_t)n_cells * kNodes * kOut;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int cell = (int)(q / (kNodes * kOut)), r = (int)(q % (kNodes * kOut));
        const int n = r / kOut, ch = r % kOut, v = ch / 3;
        const int i = n % kN, j = (n / kN) % kN, k = n / (kN * kN);
        const double b = bx[(node_off[c_first + cell] + n) * 24 + ch];
        y[q] = wild[cell] ? 0.f : (float)(b - (double)q1(v, i, j, k));
    }
}

// bases of cells c_first .. c_first + n - 1 from the L3 output of this chunk
__global__ void k_predict(int n_cells, int c_first, const float* __restrict__ o, const int64_t* __restrict__ node_off,
                          double* __restrict__ bx)
{
    const int64_t total = (int64_t)n_cells * kNodes * kOut;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int cell = (int)(q / (kNodes * kOut)), r = (int)(q % (kNodes * kOut));
        const int n = r / kOut, ch = r % kOut, v = ch / 3;
        const int i = n % kN, j = (n / kN) % kN, k = n / (kN * kN);
        const float corr = node_corr(o + (size_t)cell * kVox * kCh, i, j, k, ch);
        bx[(node_off[c_first + cell] + n) * 24 + ch] = (double)q1(v, i, j, k) + (double)corr;
    }
}

// ------------------------------------------------------------------ voxels and cell checks

__constant__ int c_kuhn_order[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
__constant__ int c_kuhn_corners[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

// share of octant oct (bit a: upper half along axis a) of a hexahedron inside Kuhn tetrahedron t
// (coordinates ordered as c_kuhn_order[t], largest first): zero unless the octant's halves are
// non-increasing along that order; the consistent orders split the octant equally (coordinates
// in the same half are exchangeable)
__device__ float kuhn_share(int oct, int t)
{
    const int h[3] = {oct & 1, (oct >> 1) & 1, (oct >> 2) & 1};
    int n = 0, mine = 0;
    for (int u = 0; u < 6; u++) {
        const int* o = c_kuhn_order[u];
        const int ok = h[o[0]] >= h[o[1]] && h[o[1]] >= h[o[2]];
        n += ok;
        if (u == t) mine = ok;
    }
    return mine ? 1.f / (float)n : 0.f;
}

__global__ void k_voxelise(int n_cells, const int64_t* __restrict__ tet_off, const int32_t* __restrict__ mat,
                           const double* __restrict__ logE, int n_mat, float* __restrict__ vox)
{
    const int64_t total = (int64_t)n_cells * kVox;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int cell = (int)(q / kVox), v = (int)(q % kVox);
        const int vx = v & 15, vy = (v >> 4) & 15, vz = v >> 8;
        const int hex = (vx >> 1) + 8 * ((vy >> 1) + 8 * (vz >> 1));
        const int oct = (vx & 1) | ((vy & 1) << 1) | ((vz & 1) << 2);
        double s = 0.0;
        for (int t = 0; t < 6; t++) {
            const float f = kuhn_share(oct, t);
            if (f == 0.f) continue;
            int m = mat[tet_off[cell] + 6 * hex + t];
            m = min(max(m, 0), n_mat - 1);  // ids were range-checked when the cells were created
            s += (double)f * logE[m];
        }
        vox[q] = (float)s;
    }
}

__global__ void k_check_kuhn8(int n_cells, const int64_t* __restrict__ node_off, const int64_t* __restrict__ tet_off,
                              const int32_t* __restrict__ elems, int* bad)
{
    const int64_t total = (int64_t)n_cells * kTets;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int cell = (int)(q / kTets), e = (int)(q % kTets);
        if (node_off[cell + 1] - node_off[cell] != kNodes || tet_off[cell + 1] - tet_off[cell] != kTets) {
            atomicExch(bad, 1);
            continue;
        }
        const int hex = e / 6, t = e % 6;
        const int hi = hex % 8, hj = (hex / 8) % 8, hk = hex / 64;
        const int32_t* nd = elems + 4 * (tet_off[cell] + e);
        for (int c = 0; c < 4; c++) {
            const int b = c_kuhn_corners[t][c];
            const int want = (hi + (b & 1)) + kN * ((hj + ((b >> 1) & 1)) + kN * (hk + ((b >> 2) & 1)));
            if ((int64_t)nd[c] - node_off[cell] != want) atomicExch(bad, 1);
        }
    }
}

// ------------------------------------------------------------------ optimiser

__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// BF16 copies of layers 1..3: wf[l][tap][co][ci] (forward), wb[l][26 - tap][ci][co] (backward data)
__global__ void k_cast(const float* __restrict__ p, __nv_bfloat16* __restrict__ wf, __nv_bfloat16* __restrict__ wb)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 3 * kLayerW; q += gridDim.x * blockDim.x) {
        const int l = q / kLayerW, r = q % kLayerW;
        const int tap = r / (kCh * kCh), co = (r / kCh) % kCh, ci = r % kCh;
        const __nv_bfloat16 w = __float2bfloat16_rn(p[layer_base(l + 1) + r]);
        wf[q] = w;
        wb[(size_t)l * kLayerW + ((kTaps - 1 - tap) * kCh + ci) * kCh + co] = w;
    }
}

__global__ void k_gather(int n, const int32_t* __restrict__ idx, const float* __restrict__ dx, const float* __restrict__ dy,
                         float* __restrict__ x, float* __restrict__ y)
{
    const int64_t nx = (int64_t)n * kVox, ny = (int64_t)n * kNodes * kOut;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nx + ny; q += (int64_t)gridDim.x * blockDim.x) {
        if (q < nx) x[q] = dx[(int64_t)idx[q / kVox] * kVox + q % kVox];
        else {
            const int64_t r = q - nx;
            y[r] = dy[(int64_t)idx[r / (kNodes * kOut)] * kNodes * kOut + r % (kNodes * kOut)];
        }
    }
}

int grid_for(int64_t n, int threads = 256) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16)); }

}  // namespace

struct NetHandle {
    int device = 0;
    cudaStream_t stream = nullptr;
    double E_ref = 1.0, in_scale = 1.0;
    DBuf<float> p, g, m, v;
    DBuf<__nv_bfloat16> wf, wb;
    int64_t adam_t = 0;
    int n_data = 0;
    DBuf<float> data_x, data_y;
    int cap = 0;
    DBuf<float> x, y, o, gnode, lossp, part, loss_dev;
    DBuf<__nv_bfloat16> a0, a1, a2, d0, d1;
    DBuf<int32_t> idx;
    DBuf<int> flag;
    DBuf<int> err;       // set by a tcgen05 kernel whose completion wait timed out
    int tcgen05 = 0;     // layers 1-3: 0 mma.sync (k_conv32), 1 tcgen05 M=64 tiles (k_conv32_tc), 2 tcgen05 transposed
                         // (k_conv32_tt), 3 tcgen05 M=64 tiles warp-specialised and persistent (k_conv32_ws)
    int sms = 148;       // multiprocessors of the device (the persistent kernel's grid)
    ~NetHandle()
    {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int net_reserve(NetHandle& N, int cap)
{
    if (cap <= N.cap) return 0;
    const size_t c = (size_t)cap;
    MSFEM_TRY(N.x.alloc(c * kVox));
    MSFEM_TRY(N.y.alloc(c * kNodes * kOut));
    MSFEM_TRY(N.o.alloc(c * kVox * kCh));
    MSFEM_TRY(N.gnode.alloc(c * kNodes * kOut));
    MSFEM_TRY(N.lossp.alloc(c));
    MSFEM_TRY(N.a0.alloc(c * kVox * kCh));
    MSFEM_TRY(N.a1.alloc(c * kVox * kCh));
    MSFEM_TRY(N.a2.alloc(c * kVox * kCh));
    MSFEM_TRY(N.d0.alloc(c * kVox * kCh));
    MSFEM_TRY(N.d1.alloc(c * kVox * kCh));
    MSFEM_TRY(N.part.alloc(std::max<size_t>(c, 1) * kLayer));
    MSFEM_TRY(N.idx.alloc(c));
    N.cap = cap;
    return 0;
}

int conv_attrs()
{
    static bool done = false;
    if (done) return 0;
    MSFEM_CK(cudaFuncSetAttribute(k_conv32<kEpiRelu>, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32<kEpiF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32<kEpiMask>, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_wgrad32, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgradSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tc<kEpiRelu>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tc<kEpiF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tc<kEpiMask>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tt<kEpiRelu>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTtSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tt<kEpiF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTtSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_tt<kEpiMask>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTtSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_ws<kEpiRelu>, cudaFuncAttributeMaxDynamicSharedMemorySize, kWsSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_ws<kEpiF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kWsSmem));
    MSFEM_CK(cudaFuncSetAttribute(k_conv32_ws<kEpiMask>, cudaFuncAttributeMaxDynamicSharedMemorySize, kWsSmem));
    done = true;
    return 0;
}

// one 32 -> 32 convolution of n cells on the selected tensor-core path
template <int EPI>
void conv(NetHandle& N, int n, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias, const __nv_bfloat16* mask,
          __nv_bfloat16* out, float* outf)
{
    if (N.tcgen05 == 3)
        k_conv32_ws<EPI><<<std::min(n, N.sms), kWsThreads, kWsSmem, N.stream>>>(n, in, w, bias, mask, out, outf, N.err.p);
    else if (N.tcgen05 == 2)
        k_conv32_tt<EPI><<<n, 128, kTtSmem, N.stream>>>(in, w, bias, mask, out, outf, N.err.p);
    else if (N.tcgen05 == 1)
        k_conv32_tc<EPI><<<n, 128, kTcSmem, N.stream>>>(in, w, bias, mask, out, outf, N.err.p);
    else
        k_conv32<EPI><<<dim3(8, n), 256, kConvSmem, N.stream>>>(in, w, bias, mask, out, outf);
}

// forward of n cells held in N.x -> N.a0, N.a1, N.a2, N.o
int net_forward(NetHandle& N, int n)
{
    cudaStream_t st = N.stream;
    MSFEM_TRY(conv_attrs());
    const __nv_bfloat16* wf = N.wf.p;
    k_first_fwd<<<dim3(kV, n), 256, 0, st>>>(N.x.p, N.p.p, N.a0.p);
    conv<kEpiRelu>(N, n, N.a0.p, wf, N.p.p + layer_base(1) + kLayerW, nullptr, N.a1.p, nullptr);
    conv<kEpiRelu>(N, n, N.a1.p, wf + kLayerW, N.p.p + layer_base(2) + kLayerW, nullptr, N.a2.p, nullptr);
    conv<kEpiF32>(N, n, N.a2.p, wf + 2 * kLayerW, N.p.p + layer_base(3) + kLayerW, nullptr, nullptr, N.o.p);
    MSFEM_CK(cudaGetLastError());
    return 0;
}

// the tcgen05 kernels' timeout flag (read after the caller's synchronisation)
int check_err(NetHandle& N)
{
    int e = 0;
    MSFEM_CK(cudaMemcpyAsync(&e, N.err.p, sizeof(int), cudaMemcpyDeviceToHost, N.stream));
    MSFEM_CK(cudaStreamSynchronize(N.stream));
    if (e) {
        set_error("learned coarse space: a tensor-core completion wait timed out");
        return MSFEM_ERR_CUDA;
    }
    return 0;
}

int wgrad_layer(NetHandle& N, int n, const __nv_bfloat16* act, const __nv_bfloat16* dz, float* grad_out)
{
    cudaStream_t st = N.stream;
    const int n_parts = std::min(n, N.cap);
    const int per = (n + n_parts - 1) / n_parts;
    const int used = (n + per - 1) / per;
    k_wgrad32<<<used, 256, kWgradSmem, st>>>(n, per, act, dz, N.part.p);
    k_reduce_parts<<<grid_for(kLayer), 256, 0, st>>>(used, kLayer, N.part.p, grad_out);
    MSFEM_CK(cudaGetLastError());
    return 0;
}

// loss and gradients of n cells (inputs N.x, targets N.y) into N.g; loss into *d_loss (device)
int net_loss_backward(NetHandle& N, int n, float* d_loss)
{
    cudaStream_t st = N.stream;
    MSFEM_TRY(net_forward(N, n));
    const float inv_norm = 1.0f / ((float)n * kNodes * kOut);
    k_loss_nodes<<<n, 256, 0, st>>>(N.o.p, N.y.p, inv_norm, N.gnode.p, N.lossp.p);
    k_loss_sum<<<1, 32, 0, st>>>(n, N.lossp.p, inv_norm, d_loss);
    k_dout<<<grid_for((int64_t)n * kVox * kCh), 256, 0, st>>>(n, N.gnode.p, N.d0.p);
    const __nv_bfloat16* wb = N.wb.p;
    // layer 3
    MSFEM_TRY(wgrad_layer(N, n, N.a2.p, N.d0.p, N.g.p + layer_base(3)));
    conv<kEpiMask>(N, n, N.d0.p, wb + 2 * kLayerW, nullptr, N.a2.p, N.d1.p, nullptr);
    // layer 2
    MSFEM_TRY(wgrad_layer(N, n, N.a1.p, N.d1.p, N.g.p + layer_base(2)));
    conv<kEpiMask>(N, n, N.d1.p, wb + kLayerW, nullptr, N.a1.p, N.d0.p, nullptr);
    // layer 1
    MSFEM_TRY(wgrad_layer(N, n, N.a0.p, N.d0.p, N.g.p + layer_base(1)));
    conv<kEpiMask>(N, n, N.d0.p, wb, nullptr, N.a0.p, N.d1.p, nullptr);
    // layer 0
    const int n_parts = std::min(n, N.cap);
    const int per = (n + n_parts - 1) / n_parts;
    const int used = (n + per - 1) / per;
    k_first_wgrad<<<used, 256, 0, st>>>(n, per, N.x.p, N.d1.p, N.part.p);
    k_reduce_parts<<<grid_for(kPart0), 256, 0, st>>>(used, kPart0, N.part.p, N.g.p);
    MSFEM_CK(cudaGetLastError());
    return 0;
}

int upload_params(NetHandle& N)
{
    k_cast<<<grid_for(3 * kLayerW), 256, 0, N.stream>>>(N.p.p, N.wf.p, N.wb.p);
    MSFEM_CK(cudaGetLastError());
    return 0;
}

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

int check_cells(NetHandle& N, CellsHandle& C)
{
    if (C.n_cells <= 0) {
        set_error("learned coarse space: no cells");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(N.flag.alloc(1));
    MSFEM_CK(cudaMemsetAsync(N.flag.p, 0, sizeof(int), N.stream));
    MSFEM_CK(cudaStreamSynchronize(C.stream));
    k_check_kuhn8<<<grid_for((int64_t)C.n_cells * kTets), 256, 0, N.stream>>>(C.n_cells, C.node_off.p, C.tet_off.p,
                                                                              C.vols.elems.p, N.flag.p);
    MSFEM_CK(cudaGetLastError());
    int bad = 0;
    MSFEM_CK(cudaMemcpyAsync(&bad, N.flag.p, sizeof(int), cudaMemcpyDeviceToHost, N.stream));
    MSFEM_CK(cudaStreamSynchronize(N.stream));
    if (bad) {
        set_error("learned coarse space: every cell must be an 8 x 8 x 8 Kuhn cube (729 nodes, 3072 tetrahedra in cube order)");
        return MSFEM_ERR_ARGUMENT;
    }
    return 0;
}

// s ln(E_m / E_ref) per material, E from the cells' Lame parameters
int log_moduli(NetHandle& N, CellsHandle& C, DBuf<double>& out)
{
    std::vector<double> lame(2 * (size_t)C.n_mat), le(C.n_mat);
    MSFEM_CK(cudaMemcpyAsync(lame.data(), C.lame.p, sizeof(double) * lame.size(), cudaMemcpyDeviceToHost, C.stream));
    MSFEM_CK(cudaStreamSynchronize(C.stream));
    for (int m = 0; m < C.n_mat; m++) {
        const double l = lame[2 * m], mu = lame[2 * m + 1];
        const double E = mu * (3.0 * l + 2.0 * mu) / (l + mu);
        if (!(E > 0.0)) {
            set_error("learned coarse space: material %d has E = %g", m, E);
            return MSFEM_ERR_ARGUMENT;
        }
        le[m] = N.in_scale * std::log(E / N.E_ref);
    }
    MSFEM_TRY(out.alloc(C.n_mat));
    MSFEM_CK(cudaMemcpyAsync(out.p, le.data(), sizeof(double) * le.size(), cudaMemcpyHostToDevice, N.stream));
    return 0;
}

}  // namespace
}  // namespace msfem

struct msfem_net : msfem::NetHandle {};

extern "C" {

int msfem_net_param_count(void) { return msfem::kParams; }

int msfem_net_create(uint64_t seed, double E_ref, double in_scale, msfem_net_t* out)
{
    using namespace msfem;
    if (!out || !(E_ref > 0.0) || !(in_scale > 0.0)) {
        set_error("msfem_net_create: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    std::unique_ptr<msfem_net> h(new (std::nothrow) msfem_net());
    if (!h) {
        set_error("out of host memory");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaGetDevice(&h->device));
    MSFEM_CK(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->E_ref = E_ref;
    h->in_scale = in_scale;
    MSFEM_TRY(h->p.alloc(kParams));
    MSFEM_TRY(h->g.alloc(kParams));
    MSFEM_TRY(h->m.alloc(kParams));
    MSFEM_TRY(h->v.alloc(kParams));
    MSFEM_TRY(h->wf.alloc(3 * kLayerW));
    MSFEM_TRY(h->wb.alloc(3 * kLayerW));
    MSFEM_TRY(h->loss_dev.alloc(1));
    MSFEM_TRY(h->err.alloc(1));
    // uniform(-b, b) with b = sqrt(6 / fan_in) (He), the last layer scaled by 0.1 so that the
    // untrained network starts near the trilinear coarse space; biases zero; padded rows zero
    std::vector<float> p(kParams, 0.f);
    uint64_t s = seed;
    const double b0 = std::sqrt(6.0 / (kTaps * kCin0));
    for (int i = 0; i < kTaps * kCh * kCin0; i++) p[kW0 + i] = (float)((2.0 * uniform01(s) - 1.0) * b0);
    const double b1 = std::sqrt(6.0 / (kTaps * kCh));
    for (int l = 1; l <= 3; l++)
        for (int tap = 0; tap < kTaps; tap++)
            for (int co = 0; co < kCh; co++)
                for (int ci = 0; ci < kCh; ci++) {
                    const double u = (2.0 * uniform01(s) - 1.0) * b1 * (l == 3 ? 0.1 : 1.0);
                    p[layer_base(l) + (tap * kCh + co) * kCh + ci] = (l == 3 && co >= kOut) ? 0.f : (float)u;
                }
    cudaStream_t st = h->stream;
    MSFEM_CK(cudaMemcpyAsync(h->p.p, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemsetAsync(h->g.p, 0, sizeof(float) * kParams, st));
    MSFEM_CK(cudaMemsetAsync(h->m.p, 0, sizeof(float) * kParams, st));
    MSFEM_CK(cudaMemsetAsync(h->v.p, 0, sizeof(float) * kParams, st));
    MSFEM_CK(cudaMemsetAsync(h->err.p, 0, sizeof(int), st));
    MSFEM_TRY(upload_params(*h));
    MSFEM_CK(cudaStreamSynchronize(st));
    *out = h.release();
    return MSFEM_OK;
}

int msfem_net_get_params(msfem_net_t h, float* params)
{
    using namespace msfem;
    if (!h || !params) {
        set_error("msfem_net_get_params: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_CK(cudaMemcpyAsync(params, h->p.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_net_set_params(msfem_net_t h, const float* params)
{
    using namespace msfem;
    if (!h || !params) {
        set_error("msfem_net_set_params: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    std::vector<float> p(params, params + kParams);
    for (int tap = 0; tap < kTaps; tap++)
        for (int co = kOut; co < kCh; co++) {
            for (int ci = 0; ci < kCh; ci++) p[layer_base(3) + (tap * kCh + co) * kCh + ci] = 0.f;
        }
    for (int co = kOut; co < kCh; co++) p[layer_base(3) + kLayerW + co] = 0.f;
    MSFEM_CK(cudaMemcpyAsync(h->p.p, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, h->stream));
    MSFEM_CK(cudaMemsetAsync(h->m.p, 0, sizeof(float) * kParams, h->stream));
    MSFEM_CK(cudaMemsetAsync(h->v.p, 0, sizeof(float) * kParams, h->stream));
    h->adam_t = 0;
    MSFEM_TRY(upload_params(*h));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_net_voxelise(msfem_net_t h, msfem_cells_t cells, float* vox)
{
    using namespace msfem;
    if (!h || !cells || !vox) {
        set_error("msfem_net_voxelise: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    CellsHandle& C = *reinterpret_cast<CellsHandle*>(cells);
    MSFEM_TRY(check_cells(*h, C));
    DBuf<double> le;
    DBuf<float> dv;
    MSFEM_TRY(log_moduli(*h, C, le));
    MSFEM_TRY(dv.alloc((size_t)C.n_cells * kVox));
    k_voxelise<<<grid_for((int64_t)C.n_cells * kVox), 256, 0, h->stream>>>(C.n_cells, C.tet_off.p, C.mat.p, le.p, C.n_mat, dv.p);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaMemcpyAsync(vox, dv.p, sizeof(float) * C.n_cells * kVox, cudaMemcpyDeviceToHost, h->stream));
    MSFEM_CK(cudaStreamSynchronize(h->stream));
    return MSFEM_OK;
}

int msfem_net_add_cells(msfem_net_t h, msfem_cells_t cells, int* n_total)
{
    using namespace msfem;
    if (!h || !cells) {
        set_error("msfem_net_add_cells: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    CellsHandle& C = *reinterpret_cast<CellsHandle*>(cells);
    MSFEM_TRY(check_cells(*h, C));
    const size_t n_old = h->n_data, n_new = n_old + C.n_cells;
    DBuf<float> nx, ny;
    MSFEM_TRY(nx.alloc(n_new * kVox));
    MSFEM_TRY(ny.alloc(n_new * kNodes * kOut));
    cudaStream_t st = h->stream;
    if (n_old) {
        MSFEM_CK(cudaMemcpyAsync(nx.p, h->data_x.p, sizeof(float) * n_old * kVox, cudaMemcpyDeviceToDevice, st));
        MSFEM_CK(cudaMemcpyAsync(ny.p, h->data_y.p, sizeof(float) * n_old * kNodes * kOut, cudaMemcpyDeviceToDevice, st));
    }
    DBuf<double> le;
    MSFEM_TRY(log_moduli(*h, C, le));
    k_voxelise<<<grid_for((int64_t)C.n_cells * kVox), 256, 0, st>>>(C.n_cells, C.tet_off.p, C.mat.p, le.p, C.n_mat,
                                                                    nx.p + n_old * kVox);
    DBuf<uint8_t> wild;
    MSFEM_TRY(wild.alloc(C.n_cells));
    k_wild_targets<<<C.n_cells, 256, 0, st>>>(0, C.node_off.p, C.bx.p, wild.p);
    k_targets<<<grid_for((int64_t)C.n_cells * kNodes * kOut), 256, 0, st>>>(C.n_cells, 0, C.node_off.p, C.bx.p, wild.p,
                                                                            ny.p + n_old * kNodes * kOut);
    MSFEM_CK(cudaGetLastError());
    MSFEM_CK(cudaStreamSynchronize(st));
    std::swap(h->data_x.p, nx.p);
    std::swap(h->data_x.n, nx.n);
    std::swap(h->data_y.p, ny.p);
    std::swap(h->data_y.n, ny.n);
    h->n_data = (int)n_new;
    if (n_total) *n_total = h->n_data;
    return MSFEM_OK;
}

int msfem_net_train(msfem_net_t h, int steps, int batch, float lr, uint64_t seed, float* losses)
{
    using namespace msfem;
    if (!h || steps <= 0 || batch <= 0 || batch > 4096 || !(lr > 0.f) || h->n_data <= 0) {
        set_error("msfem_net_train: bad arguments (batch 1 to 4096, training cells present)");
        return MSFEM_ERR_ARGUMENT;
    }
    batch = std::min(batch, h->n_data);
    MSFEM_TRY(net_reserve(*h, batch));
    cudaStream_t st = h->stream;
    // minibatches: successive slices of seeded permutations of the training cells
    std::vector<int32_t> order(h->n_data), all((size_t)steps * batch);
    uint64_t s = seed;
    size_t pos = order.size();
    for (size_t k = 0; k < all.size(); k++) {
        if (pos == order.size()) {
            for (int i = 0; i < h->n_data; i++) order[i] = i;
            for (int i = h->n_data - 1; i > 0; i--) std::swap(order[i], order[splitmix(s) % (uint64_t)(i + 1)]);
            pos = 0;
        }
        all[k] = order[pos++];
    }
    DBuf<int32_t> didx;
    DBuf<float> dloss;
    MSFEM_TRY(didx.alloc(all.size()));
    MSFEM_TRY(dloss.alloc(steps));
    MSFEM_CK(cudaMemcpyAsync(didx.p, all.data(), sizeof(int32_t) * all.size(), cudaMemcpyHostToDevice, st));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int k = 0; k < steps; k++) {
        k_gather<<<grid_for((int64_t)batch * (kVox + kNodes * kOut)), 256, 0, st>>>(
            batch, didx.p + (size_t)k * batch, h->data_x.p, h->data_y.p, h->x.p, h->y.p);
        MSFEM_TRY(net_loss_backward(*h, batch, dloss.p + k));
        h->adam_t++;
        const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)h->adam_t)));
        const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)h->adam_t)));
        k_adam<<<grid_for(kParams), 256, 0, st>>>(kParams, h->p.p, h->g.p, h->m.p, h->v.p, lr, b1, b2, eps, c1, c2);
        MSFEM_TRY(upload_params(*h));
    }
    MSFEM_CK(cudaGetLastError());
    if (losses) MSFEM_CK(cudaMemcpyAsync(losses, dloss.p, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return check_err(*h);
}

int msfem_net_loss_grad(msfem_net_t h, int n, const float* vox, const float* target, float* loss, float* grad)
{
    using namespace msfem;
    if (!h || n <= 0 || n > 4096 || !vox || !target) {
        set_error("msfem_net_loss_grad: bad arguments (1 to 4096 cells)");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(net_reserve(*h, n));
    cudaStream_t st = h->stream;
    MSFEM_CK(cudaMemcpyAsync(h->x.p, vox, sizeof(float) * n * kVox, cudaMemcpyHostToDevice, st));
    MSFEM_CK(cudaMemcpyAsync(h->y.p, target, sizeof(float) * n * kNodes * kOut, cudaMemcpyHostToDevice, st));
    MSFEM_TRY(net_loss_backward(*h, n, h->loss_dev.p));
    if (loss) MSFEM_CK(cudaMemcpyAsync(loss, h->loss_dev.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    if (grad) MSFEM_CK(cudaMemcpyAsync(grad, h->g.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return check_err(*h);
}

int msfem_net_forward(msfem_net_t h, int n, const float* vox, float* out)
{
    using namespace msfem;
    if (!h || n <= 0 || n > 4096 || !vox || !out) {
        set_error("msfem_net_forward: bad arguments (1 to 4096 cells)");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(net_reserve(*h, n));
    cudaStream_t st = h->stream;
    MSFEM_CK(cudaMemcpyAsync(h->x.p, vox, sizeof(float) * n * kVox, cudaMemcpyHostToDevice, st));
    MSFEM_TRY(net_forward(*h, n));
    MSFEM_CK(cudaMemcpyAsync(out, h->o.p, sizeof(float) * n * kVox * kCh, cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    return check_err(*h);
}

int msfem_net_predict(msfem_net_t h, msfem_cells_t cells, float* ms)
{
    using namespace msfem;
    if (!h || !cells) {
        set_error("msfem_net_predict: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    CellsHandle& C = *reinterpret_cast<CellsHandle*>(cells);
    MSFEM_TRY(check_cells(*h, C));
    const int chunk = std::min(C.n_cells, 512);
    MSFEM_TRY(net_reserve(*h, chunk));
    DBuf<double> le;
    MSFEM_TRY(log_moduli(*h, C, le));
    cudaStream_t st = h->stream;
    cudaEvent_t e0, e1;
    MSFEM_CK(cudaEventCreate(&e0));
    MSFEM_CK(cudaEventCreate(&e1));
    MSFEM_CK(cudaEventRecord(e0, st));
    int rc = 0;
    for (int c0 = 0; c0 < C.n_cells && rc == 0; c0 += chunk) {
        const int n = std::min(chunk, C.n_cells - c0);
        k_voxelise<<<grid_for((int64_t)n * kVox), 256, 0, st>>>(n, C.tet_off.p + c0, C.mat.p, le.p, C.n_mat, h->x.p);
        rc = net_forward(*h, n);
        if (rc == 0)
            k_predict<<<grid_for((int64_t)n * kNodes * kOut), 256, 0, st>>>(n, c0, h->o.p, C.node_off.p, C.bx.p);
    }
    MSFEM_CK(cudaEventRecord(e1, st));
    MSFEM_CK(cudaEventSynchronize(e1));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MSFEM_CK(cudaGetLastError());
    if (rc) return rc;
    if (ms) *ms = t;
    return check_err(*h);
}

int msfem_net_set_tensor_path(msfem_net_t h, int tcgen05)
{
    using namespace msfem;
    if (!h || tcgen05 < 0 || tcgen05 > 3) {
        set_error("msfem_net_set_tensor_path: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    h->tcgen05 = tcgen05;
    return MSFEM_OK;
}

int msfem_net_destroy(msfem_net_t h)
{
    if (!h) return MSFEM_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
    return MSFEM_OK;
}

}  // extern "C"
