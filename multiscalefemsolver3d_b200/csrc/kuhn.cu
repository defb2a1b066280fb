// The structured Kuhn grid and its matrix-free elasticity operators (kuhn.cuh): the mesh check
// behind msfem_set_kuhn_grid, the operator set-up that checks a matrix-free product against the
// assembled matrix before anything uses it, and the plain products msfem_kuhn_spmv exposes.
#include <cmath>
#include <vector>

#include "devutil.cuh"
#include "internal.cuh"
#include "kuhn.cuh"
#include "kuhn_op.cuh"

namespace msfem {
namespace {

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// the mesh is the Kuhn grid: tetrahedron 6c+t has the corners of Kuhn tetrahedron t of hexahedron c
// in order, and node (i, j, k) sits at origin + (i hx, j hy, k hz); the first failure is recorded
__global__ void k_kuhn_check_tets(int nx, int ny, int nz, const int32_t* __restrict__ tets,
                                  const int32_t* __restrict__ mat, uint8_t* __restrict__ code, int* bad)
{
    const int64_t n_tets = 6 * (int64_t)nx * ny * nz;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_tets; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / 6;
        const int t = (int)(e - 6 * c);
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((int64_t)nx * ny));
        // corner paths 0 -> p -> q -> 7 of the six tetrahedra: p = 1 1 2 2 4 4, q = 3 5 3 6 5 6
        const int p = (0x442211 >> (4 * t)) & 0xf;
        const int q = (0x656353 >> (4 * t)) & 0xf;
        const int corner[4] = {0, p, q, 7};
        bool ok = true;
        for (int v = 0; v < 4; v++) {
            const int b = corner[v];
            const int64_t g = (i + (b & 1)) + (int64_t)(nx + 1) * ((j + ((b >> 1) & 1)) + (int64_t)(ny + 1) * (k + ((b >> 2) & 1)));
            if ((int64_t)tets[4 * e + v] != g) ok = false;
        }
        const int m = mat ? mat[e] : 0;
        if (m < 0 || m >= kKuhnMaxMat) ok = false;
        code[8 * c + t] = (uint8_t)(m < 0 || m >= kKuhnMaxMat ? 0 : m);
        if (t == 5) code[8 * c + 6] = code[8 * c + 7] = 0;
        if (!ok) atomicMin(bad, (int)(e < INT32_MAX ? e : INT32_MAX - 1));
    }
}

__global__ void k_kuhn_check_xyz(int nx, int ny, int nz, const double* __restrict__ xyz, double ox, double oy, double oz,
                                 double hx, double hy, double hz, double tol, int* bad)
{
    const int64_t n_nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_nodes; g += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(g % (nx + 1)), j = (int)((g / (nx + 1)) % (ny + 1)), k = (int)(g / ((int64_t)(nx + 1) * (ny + 1)));
        const double e = fabs(xyz[3 * g] - (ox + i * hx)) + fabs(xyz[3 * g + 1] - (oy + j * hy)) +
                         fabs(xyz[3 * g + 2] - (oz + k * hz));
        if (!(e <= tol)) atomicMin(bad, (int)(g < INT32_MAX ? g : INT32_MAX - 1));
    }
}

// a pseudo-random test vector in [-0.5, 0.5)
template <class T>
__global__ void k_kuhn_probe(int64_t n, T* __restrict__ x)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = (T)((hash32((unsigned)i ^ 0x9e3779b9u) & 0xffffff) / 16777216.0 - 0.5);
}

// per block: sum (a-b)^2, sum b^2, max |a-b|, max |b|
template <class T>
__global__ void __launch_bounds__(256) k_kuhn_compare(int64_t n, const T* __restrict__ a, const T* __restrict__ b,
                                                      double* __restrict__ out)
{
    __shared__ double sh[4][256];
    double s0 = 0.0, s1 = 0.0, m0 = 0.0, m1 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)a[i] - (double)b[i], r = (double)b[i];
        s0 += d * d;
        s1 += r * r;
        m0 = fmax(m0, fabs(d));
        m1 = fmax(m1, fabs(r));
        if (d != d) m0 = INFINITY;
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = s1;
    sh[2][threadIdx.x] = m0;
    sh[3][threadIdx.x] = m1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
            sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][threadIdx.x + w]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++) out[4 * blockIdx.x + q] = sh[q][0];
}

template <class T>
__global__ void k_to_t(int64_t n, const double* __restrict__ a, T* __restrict__ b)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (T)a[i];
}

// relative distance of the matrix-free and the assembled products of one probe vector
template <class T>
int compare(cudaStream_t st, int64_t n, const T* a, const T* b, double* rel_l2, double* rel_max)
{
    constexpr int kBlocks = 148;
    DBuf<double> part;
    MSFEM_TRY(part.alloc(4 * kBlocks));
    k_kuhn_compare<T><<<kBlocks, 256, 0, st>>>(n, a, b, part.p);
    std::vector<double> h(4 * kBlocks);
    MSFEM_CK(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    double s0 = 0.0, s1 = 0.0, m0 = 0.0, m1 = 0.0;
    for (int q = 0; q < kBlocks; q++) {
        s0 += h[4 * q];
        s1 += h[4 * q + 1];
        m0 = std::max(m0, h[4 * q + 2]);
        m1 = std::max(m1, h[4 * q + 3]);
    }
    *rel_l2 = s1 > 0.0 ? std::sqrt(s0 / s1) : (s0 > 0.0 ? INFINITY : 0.0);
    *rel_max = m1 > 0.0 ? m0 / m1 : (m0 > 0.0 ? INFINITY : 0.0);
    if (!(*rel_l2 == *rel_l2)) *rel_l2 = INFINITY;
    return MSFEM_OK;
}

}  // namespace

int kuhn_set_grid(System& s, int nx, int ny, int nz)
{
    if (s.kind != MSFEM_ELASTIC || !s.tets.p || !s.xyz.p) {
        set_error("msfem_set_kuhn_grid: needs an elasticity system with a mesh");
        return MSFEM_ERR_ARGUMENT;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0 || 6 * (int64_t)nx * ny * nz != s.n_tets ||
        (int64_t)(nx + 1) * (ny + 1) * (nz + 1) != s.n_nodes) {
        set_error("msfem_set_kuhn_grid: %d x %d x %d hexahedra do not give the mesh's %d nodes and %d tetrahedra", nx,
                  ny, nz, s.n_nodes, s.n_tets);
        return MSFEM_ERR_ARGUMENT;
    }
    cudaStream_t st = s.stream;
    // origin and spacing from nodes (0,0,0), (nx,0,0), (0,ny,0), (0,0,nz)
    const int64_t corner[4] = {0, nx, (int64_t)(nx + 1) * ny, (int64_t)(nx + 1) * (ny + 1) * nz};
    double c[4][3];
    for (int q = 0; q < 4; q++)
        MSFEM_CK(cudaMemcpyAsync(c[q], s.xyz.p + 3 * corner[q], 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    const double hx = (c[1][0] - c[0][0]) / nx, hy = (c[2][1] - c[0][1]) / ny, hz = (c[3][2] - c[0][2]) / nz;
    if (!(hx > 0.0 && hy > 0.0 && hz > 0.0)) {
        set_error("msfem_set_kuhn_grid: the corner nodes do not span a box with positive spacing");
        return MSFEM_ERR_ARGUMENT;
    }
    DBuf<int> bad;
    MSFEM_TRY(bad.alloc(2));
    const int big[2] = {INT32_MAX, INT32_MAX};
    MSFEM_CK(cudaMemcpyAsync(bad.p, big, sizeof(big), cudaMemcpyHostToDevice, st));
    // 8 bytes per hexahedron (six codes + padding), and two hexahedra of slack for the staging copies
    MSFEM_TRY(s.kuhn_mat.alloc(8 * (size_t)(s.n_tets / 6 + 2)));
    const unsigned g = std::min<unsigned>(grid_for(s.n_tets, 256), 148 * 16);
    k_kuhn_check_tets<<<g, 256, 0, st>>>(nx, ny, nz, s.tets.p, s.mat.p, s.kuhn_mat.p, bad.p);
    const double tol = 1e-9 * std::max(hx, std::max(hy, hz));
    k_kuhn_check_xyz<<<std::min<unsigned>(grid_for(s.n_nodes, 256), 148 * 16), 256, 0, st>>>(
        nx, ny, nz, s.xyz.p, c[0][0], c[0][1], c[0][2], hx, hy, hz, tol, bad.p + 1);
    MSFEM_CK(cudaGetLastError());
    int h_bad[2];
    MSFEM_CK(cudaMemcpyAsync(h_bad, bad.p, sizeof(h_bad), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    s.total_launches += 2;
    s.kuhn_n[0] = s.kuhn_n[1] = s.kuhn_n[2] = 0;
    if (h_bad[0] != INT32_MAX) {
        set_error("msfem_set_kuhn_grid: tetrahedron %d is not the Kuhn tetrahedron of the grid (or its material is "
                  "outside [0, %d))", h_bad[0], kKuhnMaxMat);
        return MSFEM_ERR_ARGUMENT;
    }
    if (h_bad[1] != INT32_MAX) {
        set_error("msfem_set_kuhn_grid: node %d is not at its grid position", h_bad[1]);
        return MSFEM_ERR_ARGUMENT;
    }
    s.kuhn_n[0] = nx;
    s.kuhn_n[1] = ny;
    s.kuhn_n[2] = nz;
    s.kuhn_h[0] = hx;
    s.kuhn_h[1] = hy;
    s.kuhn_h[2] = hz;
    return MSFEM_OK;
}

template <class T>
static void fill_view(const System& s, KuhnView<T>& v)
{
    v.nx = s.kuhn_n[0];
    v.ny = s.kuhn_n[1];
    v.nz = s.kuhn_n[2];
    const double V = s.kuhn_h[0] * s.kuhn_h[1] * s.kuhn_h[2] / 6.0;
    for (int a = 0; a < 3; a++) {
        v.ih[a] = (T)(1.0 / s.kuhn_h[a]);
        v.vh[a] = (T)(V / s.kuhn_h[a]);
    }
    v.mat = reinterpret_cast<const uint2*>(s.kuhn_mat.p);
    v.fix = s.dmask.p;
    v.n_mat = (int)(s.lame_host.size() / 2);
    v.iso = 0;
}

// hx = hy = hz to 1e-12: the z-marching kernel folds V / h^2 into the material table
static bool kuhn_isotropic(const System& s)
{
    const double h = s.kuhn_h[0];
    return std::fabs(s.kuhn_h[1] - h) <= 1e-12 * h && std::fabs(s.kuhn_h[2] - h) <= 1e-12 * h;
}

namespace {

// xh = s x with the eliminated columns zero: the input of the pre-scaled kernel (k_kuhn_zp)
__global__ void k_kuhn_prescale(int64_t n, const float* __restrict__ x, const float* __restrict__ scale,
                                const uint32_t* __restrict__ fix, float* __restrict__ xh)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        xh[i] = ((fix[i / 3] >> (3 + i % 3)) & 1u) ? 0.0f : scale[i] * x[i];
}

// y = S K S x through the pre-scaled kernel: y = x on the Dirichlet rows, s (K xh) elsewhere
struct EpiStoreP {
    static constexpr int NE = 2;  // x, the Jacobi scale
    float* y;
    const float* x;
    const float* scale;
    __device__ __forceinline__ bool skip() const { return false; }
    __host__ __device__ __forceinline__ void sources(const float** ev) const
    {
        ev[0] = x;
        ev[1] = scale;
    }
    __device__ __forceinline__ void operator()(int64_t g, const float* v, uint32_t fx, const float (*e)[3])
    {
#pragma unroll
        for (int c = 0; c < 3; c++) y[3 * g + c] = ((fx >> c) & 1u) ? e[0][c] : v[c] * e[1][c];
    }
    __device__ __forceinline__ void finish() {}
};

}  // namespace

int kuhn_operator_build(System& s, int form, bool fp64, bool scaled, KuhnOperator& op)
{
    op.sys = nullptr;
    if (!s.kuhn_n[0]) {
        set_error("matrix-free operator: the system's mesh was not checked as a Kuhn grid (msfem_set_kuhn_grid)");
        return MSFEM_ERR_STATE;
    }
    if ((form != 1 && form != 2) || s.elastic_form != form) {
        set_error("matrix-free operator: the system's values are not one %s elasticity assembly since the last clear",
                  form == 2 ? "textbook-orientation" : "reference");
        return MSFEM_ERR_STATE;
    }
    const int n_mat = (int)(s.lame_host.size() / 2);
    if (n_mat <= 0 || n_mat > kKuhnMaxMat) {
        set_error("matrix-free operator: %d materials (at most %d)", n_mat, kKuhnMaxMat);
        return MSFEM_ERR_LIMIT;
    }
    if (!s.dmask.p) {  // no Dirichlet rows yet: an all-zero mask
        MSFEM_TRY(s.dmask.alloc((size_t)s.n_nodes + 4));  // 4 words of slack: staging copies
        MSFEM_CK(cudaMemsetAsync(s.dmask.p, 0, sizeof(uint32_t) * s.dmask.n, s.stream));
    }
    MSFEM_TRY(prepare_sell(s));  // the assembled product the check compares with, and the Jacobi scale
    cudaStream_t st = s.stream;
    const int64_t n = s.n_rows;
    op.form = form;
    op.fp64 = fp64;
    op.scaled = scaled;
    MSFEM_TRY(op.err.alloc(1));
    MSFEM_CK(cudaMemsetAsync(op.err.p, 0, sizeof(int), st));
    int dev = 0, sms = 0;
    MSFEM_CK(cudaGetDevice(&dev));
    MSFEM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    op.sms = sms;
    if (fp64) {
        if (scaled) {
            set_error("matrix-free operator: the FP64 operator is unscaled");
            return MSFEM_ERR_ARGUMENT;
        }
        const bool iso = kuhn_isotropic(s);
        const double fold = iso ? s.kuhn_h[0] * s.kuhn_h[1] * s.kuhn_h[2] / 6.0 / (s.kuhn_h[0] * s.kuhn_h[0]) : 1.0;
        std::vector<double> l64(2 * (size_t)n_mat);
        for (int i = 0; i < 2 * n_mat; i++) l64[i] = s.lame_host[i] * fold;
        MSFEM_TRY(op.lame64.alloc(2 * (size_t)n_mat));
        MSFEM_CK(cudaMemcpyAsync(op.lame64.p, l64.data(), sizeof(double) * 2 * n_mat, cudaMemcpyHostToDevice, st));
        MSFEM_CK(cudaStreamSynchronize(st));  // l64 is released here
        fill_view(s, op.v64);
        op.v64.scale = nullptr;
        op.v64.lame = op.lame64.p;
        op.v64.iso = iso ? 1 : 0;
    } else {
        const bool iso = kuhn_isotropic(s);
        const double fold = iso ? s.kuhn_h[0] * s.kuhn_h[1] * s.kuhn_h[2] / 6.0 / (s.kuhn_h[0] * s.kuhn_h[0]) : 1.0;
        std::vector<float> l32(2 * (size_t)n_mat);
        for (int i = 0; i < 2 * n_mat; i++) l32[i] = (float)(s.lame_host[i] * fold);
        MSFEM_TRY(op.lame32.alloc(2 * (size_t)n_mat));
        MSFEM_CK(cudaMemcpyAsync(op.lame32.p, l32.data(), sizeof(float) * 2 * n_mat, cudaMemcpyHostToDevice, st));
        MSFEM_CK(cudaStreamSynchronize(st));  // l32 is released here
        if (scaled) {
            MSFEM_TRY(op.scale32.alloc((size_t)n + 16));  // 16 elements of slack for the staging copies
            k_to_t<float><<<grid_for(n, 256), 256, 0, st>>>(n, s.dscale.p, op.scale32.p);
        }
        fill_view(s, op.v32);
        op.v32.scale = scaled ? op.scale32.p : nullptr;
        op.v32.lame = op.lame32.p;
        op.v32.iso = iso ? 1 : 0;
    }
    // the check: one probe vector through both products
    double rl2 = 0.0, rmax = 0.0;
    if (fp64) {
        DBuf<double> x, y1, y2;
        MSFEM_TRY(x.alloc(n + 16));
        MSFEM_TRY(y1.alloc(n));
        MSFEM_TRY(y2.alloc(n));
        k_kuhn_probe<double><<<148 * 4, 256, 0, st>>>(n, x.p);
        MSFEM_TRY(kuhn_spmv64(op, x.p, y1.p, st));
        MSFEM_TRY(spmv64(s, x.p, y2.p));
        MSFEM_TRY(kuhn_check_err(op, st));
        MSFEM_TRY(compare<double>(st, n, y1.p, y2.p, &rl2, &rmax));
        if (!(rl2 <= 1e-12 && rmax <= 1e-11)) {
            set_error("matrix-free operator: its product differs from the assembled matrix's (relative %.3g in l2, "
                      "%.3g in max); the values are not the Kuhn grid's elasticity operator", rl2, rmax);
            return MSFEM_ERR_STATE;
        }
    } else {
        DBuf<float> x, y1, y2;
        MSFEM_TRY(x.alloc(n + 16));
        MSFEM_TRY(y1.alloc(n));
        MSFEM_TRY(y2.alloc(n));
        k_kuhn_probe<float><<<148 * 4, 256, 0, st>>>(n, x.p);
        MSFEM_TRY(kuhn_spmv32(op, x.p, y1.p, st));
        if (scaled) {
            MSFEM_TRY(spmv32(s, x.p, y2.p));
        } else {
            set_error("matrix-free operator: the FP32 operator is the Jacobi-scaled one");
            return MSFEM_ERR_ARGUMENT;
        }
        MSFEM_TRY(kuhn_check_err(op, st));
        MSFEM_TRY(compare<float>(st, n, y1.p, y2.p, &rl2, &rmax));
        if (!(rl2 <= 1e-5 && rmax <= 1e-4)) {
            set_error("matrix-free operator: its product differs from the assembled matrix's (relative %.3g in l2, "
                      "%.3g in max); the values are not the Kuhn grid's elasticity operator", rl2, rmax);
            return MSFEM_ERR_STATE;
        }
        // the pre-scaled kernel the smoother steps run: the same product, bit for bit
        DBuf<float> xh;
        MSFEM_TRY(xh.alloc(n + 16));
        op.sys = &s;  // for the pre-scaled product below; cleared again if the check fails
        const int rc = kuhn_spmv32_pre(op, x.p, xh.p, y2.p, st);
        op.sys = nullptr;
        MSFEM_TRY(rc);
        MSFEM_TRY(kuhn_check_err(op, st));
        double pl2 = 0.0, pmax = 0.0;
        MSFEM_TRY(compare<float>(st, n, y2.p, y1.p, &pl2, &pmax));
        if (pmax != 0.0) {
            set_error("matrix-free operator: the pre-scaled kernel's product differs from the staged-scale "
                      "kernel's (relative %.3g in max)", pmax);
            return MSFEM_ERR_STATE;
        }
    }
    op.check_l2 = rl2;
    op.check_max = rmax;
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 4;
    op.version = s.values_version;
    op.sys = &s;
    return MSFEM_OK;
}

int kuhn_operator_current(const KuhnOperator& op)
{
    if (!op.sys || op.version != op.sys->values_version) {
        set_error("matrix-free operator: the system's values changed after it was set up");
        return MSFEM_ERR_STATE;
    }
    return MSFEM_OK;
}

int kuhn_spmv64(KuhnOperator& op, const double* x, double* y, cudaStream_t st)
{
    EpiStoreZ<double> e{y};
    cudaError_t err = op.form == 2
                          ? KzKernel<2, false, double, kKzTX, kKzTY, kKzMinB64, EpiStoreZ<double>>::launch(
                                op.v64, x, e, op.sms, op.err.p, st)
                          : KzKernel<1, false, double, kKzTX, kKzTY, kKzMinB64, EpiStoreZ<double>>::launch(
                                op.v64, x, e, op.sms, op.err.p, st);
    if (err != cudaSuccess) {
        set_error("matrix-free FP64 product: %s", cudaGetErrorString(err));
        return MSFEM_ERR_CUDA;
    }
    return MSFEM_OK;
}

int kuhn_spmv32(KuhnOperator& op, const float* x, float* y, cudaStream_t st)
{
    EpiStoreZ<float> e{y};
    cudaError_t err = op.form == 2
                          ? KzKernel<2, true, float, kKzTX, kKzTY, kKzMinB, EpiStoreZ<float>>::launch(
                                op.v32, x, e, op.sms, op.err.p, st)
                          : KzKernel<1, true, float, kKzTX, kKzTY, kKzMinB, EpiStoreZ<float>>::launch(
                                op.v32, x, e, op.sms, op.err.p, st);
    if (err != cudaSuccess) {
        set_error("matrix-free FP32 product: %s", cudaGetErrorString(err));
        return MSFEM_ERR_CUDA;
    }
    return MSFEM_OK;
}

int kuhn_spmv32_pre(KuhnOperator& op, const float* x, float* xh, float* y, cudaStream_t st)
{
    if (!op.scaled || op.fp64) {
        set_error("matrix-free FP32 product (pre-scaled input): the operator is not the Jacobi-scaled FP32 one");
        return MSFEM_ERR_ARGUMENT;
    }
    const int64_t n = op.sys ? op.sys->n_rows : 0;
    k_kuhn_prescale<<<148 * 4, 256, 0, st>>>(n, x, op.scale32.p, op.v32.fix, xh);
    const EpiStoreP e{y, x, op.scale32.p};
    cudaError_t err = op.form == 2
                          ? KzpKernel<2, float, kKzTX, kKzTY, kKzMinB, EpiStoreP>::launch(op.v32, xh, e, op.sms,
                                                                                           op.err.p, st)
                          : KzpKernel<1, float, kKzTX, kKzTY, kKzMinB, EpiStoreP>::launch(op.v32, xh, e, op.sms,
                                                                                           op.err.p, st);
    if (err != cudaSuccess) {
        set_error("matrix-free FP32 product (pre-scaled input): %s", cudaGetErrorString(err));
        return MSFEM_ERR_CUDA;
    }
    if (op.sys) op.sys->total_launches += 2;
    return MSFEM_OK;
}

int kuhn_check_err(KuhnOperator& op, cudaStream_t st)
{
    int h = 0;
    MSFEM_CK(cudaMemcpyAsync(&h, op.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSFEM_CK(cudaStreamSynchronize(st));
    if (h) {
        MSFEM_CK(cudaMemsetAsync(op.err.p, 0, sizeof(int), st));
        set_error("matrix-free product: a staging wait expired (bulk copies did not complete)");
        return MSFEM_ERR_CUDA;
    }
    return MSFEM_OK;
}

}  // namespace msfem
