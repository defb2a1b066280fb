// The C ABI (include/msfem_b200.h): handle management, host/device transfers
// and argument checking around the kernels of the other translation units.
#include <cstdarg>
#include <cstring>
#include <algorithm>
#include <memory>
#include <new>
#include <string>

#include "devutil.cuh"
#include "internal.cuh"
#include "kuhn_op.cuh"
#include "spmv.cuh"

namespace msfem {

namespace {
thread_local char g_err[1024] = "";
}

void set_error(const char* fmt, ...)
{
    va_list v;
    va_start(v, fmt);
    std::vsnprintf(g_err, sizeof(g_err), fmt, v);
    va_end(v);
}

namespace {

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

__global__ void k_add(int n, const double* __restrict__ a, double* __restrict__ b)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] += a[i];
}

// expanded scalar CSR of a 3x3-block portrait, DOF = 3*node + component
// (Library/Math.h:1963-2054): row 3i+a holds the a-th rows of the blocks of block row i
__global__ void k_expand_rows(int n_nodes, const int32_t* __restrict__ nrp, int32_t* __restrict__ rp)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > 3 * n_nodes) return;
    if (r == 3 * n_nodes) {
        rp[r] = 9 * nrp[n_nodes];
        return;
    }
    const int i = r / 3, a = r - 3 * i;
    rp[r] = 9 * nrp[i] + 3 * a * (nrp[i + 1] - nrp[i]);
}

__global__ void k_expand_entries(int n_nodes, const int32_t* __restrict__ nrp, const int32_t* __restrict__ ncol,
                                 const double* __restrict__ bval, int32_t* __restrict__ col, double* __restrict__ val)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 3 * n_nodes) return;
    const int i = r / 3, a = r - 3 * i;
    const int b0 = nrp[i], len = nrp[i + 1] - b0;
    int64_t out = 9 * (int64_t)b0 + 3 * (int64_t)a * len;
    for (int k = 0; k < len; k++) {
        const int j = ncol[b0 + k];
        for (int b = 0; b < 3; b++) {
            col[out] = 3 * j + b;
            val[out] = bval[9 * (int64_t)(b0 + k) + 3 * a + b];
            out++;
        }
    }
}

template <class T>
int to_device(System& s, DBuf<T>& dst, const T* src, size_t n)
{
    MSFEM_TRY(dst.alloc(n));
    if (n) MSFEM_CK(cudaMemcpyAsync(dst.p, src, n * sizeof(T), cudaMemcpyDefault, s.stream));
    return MSFEM_OK;
}

System* as_sys(msfem_system_t h) { return reinterpret_cast<System*>(h); }

int check_handle(msfem_system_t h)
{
    if (!h) {
        set_error("null handle");
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

int use_device(System& s)
{
    MSFEM_CK(cudaSetDevice(s.device));
    return MSFEM_OK;
}

// systems imported as a matrix (msfem_system_from_cssd) have no mesh to assemble from
int need_mesh(System& s, const char* who)
{
    if (!s.tets.p) {
        set_error("%s: the system was imported as a matrix and has no mesh", who);
        return MSFEM_ERR_ARGUMENT;
    }
    return MSFEM_OK;
}

}  // namespace

template <class T>
static void take_buffer(DBuf<T>& dst, DBuf<T>& src)
{
    dst.release();
    dst.p = src.p;
    dst.n = src.n;
    src.p = nullptr;
    src.n = 0;
}

int system_adopt_csr(int n, DBuf<int32_t>& row_ptr, DBuf<int32_t>& col, DBuf<double>& val, int64_t nnz,
                     msfem_system_t* out)
{
    *out = nullptr;
    std::unique_ptr<System> s(new (std::nothrow) System());
    if (!s) {
        set_error("out of host memory");
        return MSFEM_ERR_LIMIT;
    }
    s->kind = MSFEM_SCALAR;
    s->bs = 1;
    s->n_nodes = n;
    s->n_tets = 0;
    s->n_rows = n;
    s->nnzb = nnz;
    s->color_off = {0};
    MSFEM_CK(cudaGetDevice(&s->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    MSFEM_CK(cudaEventCreate(&s->ev0));
    MSFEM_CK(cudaEventCreate(&s->ev1));
    take_buffer(s->nrp, row_ptr);
    take_buffer(s->ncol, col);
    take_buffer(s->val, val);
    MSFEM_TRY(s->F.alloc((size_t)n));
    MSFEM_TRY(s->X.alloc((size_t)n));
    MSFEM_CK(cudaMemsetAsync(s->F.p, 0, sizeof(double) * n, s->stream));
    MSFEM_CK(cudaMemsetAsync(s->X.p, 0, sizeof(double) * n, s->stream));
    MSFEM_CK(cudaStreamSynchronize(s->stream));
    *out = reinterpret_cast<msfem_system_t>(s.release());
    return MSFEM_OK;
}

}  // namespace msfem

using namespace msfem;

extern "C" {

const char* msfem_last_error(void) { return g_err; }
int msfem_version(void) { return 100; }

int msfem_system_create(int kind, int n_nodes, const double* xyz, int n_tets, const int32_t* tets,
                        const int32_t* material, int on_device, msfem_system_t* out)
{
    (void)on_device;  // cudaMemcpyDefault resolves host vs device pointers (unified addressing)
    if (!out || !xyz || !tets || n_nodes <= 0 || n_tets <= 0 || (kind != MSFEM_SCALAR && kind != MSFEM_ELASTIC)) {
        set_error("msfem_system_create: bad arguments (kind %d, n_nodes %d, n_tets %d)", kind, n_nodes, n_tets);
        return MSFEM_ERR_ARGUMENT;
    }
    if (kind == MSFEM_ELASTIC && (int64_t)n_nodes * 3 > INT32_MAX) {
        set_error("msfem_system_create: 3*n_nodes exceeds the int32 DOF range");
        return MSFEM_ERR_LIMIT;
    }
    *out = nullptr;
    std::unique_ptr<System> s(new (std::nothrow) System());
    if (!s) {
        set_error("out of host memory");
        return MSFEM_ERR_LIMIT;
    }
    s->kind = kind;
    s->bs = kind == MSFEM_SCALAR ? 1 : 3;
    s->n_nodes = n_nodes;
    s->n_tets = n_tets;
    s->n_rows = n_nodes * s->bs;
    MSFEM_CK(cudaGetDevice(&s->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    MSFEM_CK(cudaEventCreate(&s->ev0));
    MSFEM_CK(cudaEventCreate(&s->ev1));
    cudaEvent_t t0, t1;
    MSFEM_CK(cudaEventCreate(&t0));
    MSFEM_CK(cudaEventCreate(&t1));
    MSFEM_CK(cudaEventRecord(t0, s->stream));
    MSFEM_TRY(to_device(*s, s->xyz, xyz, 3 * (size_t)n_nodes));
    MSFEM_TRY(to_device(*s, s->tets, tets, 4 * (size_t)n_tets));
    if (material) {
        MSFEM_TRY(to_device(*s, s->mat, material, (size_t)n_tets));
    } else {
        MSFEM_TRY(s->mat.alloc((size_t)n_tets));
        MSFEM_CK(cudaMemsetAsync(s->mat.p, 0, sizeof(int32_t) * (size_t)n_tets, s->stream));
    }
    int rc = build_topology(*s);
    if (rc < 0) return rc;
    MSFEM_TRY(s->val.alloc((size_t)s->nnzb * s->bs * s->bs));
    MSFEM_TRY(s->F.alloc((size_t)s->n_rows));
    MSFEM_TRY(s->X.alloc((size_t)s->n_rows));
    MSFEM_CK(cudaMemsetAsync(s->val.p, 0, sizeof(double) * s->val.n, s->stream));
    MSFEM_CK(cudaMemsetAsync(s->F.p, 0, sizeof(double) * s->F.n, s->stream));
    MSFEM_CK(cudaMemsetAsync(s->X.p, 0, sizeof(double) * s->X.n, s->stream));
    MSFEM_CK(cudaEventRecord(t1, s->stream));
    MSFEM_CK(cudaStreamSynchronize(s->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    s->stats.ms_portrait = ms;
    *out = reinterpret_cast<msfem_system_t>(s.release());
    return MSFEM_OK;
}

int msfem_system_from_cssd(int n, const double* diag, const int64_t* down_ptr, const int32_t* down_col,
                           const double* down_val, const int64_t* up_ptr, const int32_t* up_col, const double* up_val,
                           const double* F, const double* X, msfem_system_t* out)
{
    if (!out || n <= 0 || !diag || !down_ptr || !up_ptr) {
        set_error("msfem_system_from_cssd: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    *out = nullptr;
    if (down_ptr[0] != 0 || up_ptr[0] != 0) {
        set_error("msfem_system_from_cssd: row offsets must start at 0");
        return MSFEM_ERR_ARGUMENT;
    }
    const int64_t n_down = down_ptr[n], n_up = up_ptr[n];
    if ((n_down > 0 && (!down_col || !down_val)) || (n_up > 0 && (!up_col || !up_val)) ||
        (int64_t)n + n_down + n_up > INT32_MAX) {
        set_error("msfem_system_from_cssd: bad entry arrays or more than 2^31 entries");
        return MSFEM_ERR_ARGUMENT;
    }
    // CSR rows [A_down (columns < i, ascending) | Diag | A_up (columns > i, ascending)]: the
    // reference's row layout; lists given unsorted are sorted here, repeated columns rejected
    std::vector<int32_t> rp(n + 1, 0), col;
    std::vector<double> val;
    col.reserve(n + n_down + n_up);
    val.reserve(n + n_down + n_up);
    std::vector<std::pair<int32_t, double>> tmp;
    for (int i = 0; i < n; i++) {
        for (int part = 0; part < 3; part++) {
            if (part == 1) {
                col.push_back(i);
                val.push_back(diag[i]);
                continue;
            }
            const int64_t* ptr = part == 0 ? down_ptr : up_ptr;
            const int32_t* c = part == 0 ? down_col : up_col;
            const double* v = part == 0 ? down_val : up_val;
            if (ptr[i + 1] < ptr[i]) {
                set_error("msfem_system_from_cssd: row %d has decreasing offsets", i);
                return MSFEM_ERR_ARGUMENT;
            }
            tmp.clear();
            for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) {
                const int32_t j = c[k];
                if ((part == 0 && (j < 0 || j >= i)) || (part == 2 && (j <= i || j >= n))) {
                    set_error("msfem_system_from_cssd: row %d lists column %d in its %s part", i, j,
                              part == 0 ? "lower" : "upper");
                    return MSFEM_ERR_ARGUMENT;
                }
                tmp.emplace_back(j, v[k]);
            }
            std::sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (size_t k = 0; k < tmp.size(); k++) {
                if (k && tmp[k].first == tmp[k - 1].first) {
                    set_error("msfem_system_from_cssd: row %d lists column %d twice", i, tmp[k].first);
                    return MSFEM_ERR_ARGUMENT;
                }
                col.push_back(tmp[k].first);
                val.push_back(tmp[k].second);
            }
        }
        rp[i + 1] = (int32_t)col.size();
    }
    std::unique_ptr<System> s(new (std::nothrow) System());
    if (!s) {
        set_error("out of host memory");
        return MSFEM_ERR_LIMIT;
    }
    s->kind = MSFEM_SCALAR;
    s->bs = 1;
    s->n_nodes = n;
    s->n_tets = 0;
    s->n_rows = n;
    s->nnzb = (int64_t)col.size();
    s->color_off = {0};
    MSFEM_CK(cudaGetDevice(&s->device));
    MSFEM_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    MSFEM_CK(cudaEventCreate(&s->ev0));
    MSFEM_CK(cudaEventCreate(&s->ev1));
    MSFEM_TRY(to_device(*s, s->nrp, rp.data(), rp.size()));
    MSFEM_TRY(to_device(*s, s->ncol, col.data(), col.size()));
    MSFEM_TRY(to_device(*s, s->val, val.data(), val.size()));
    MSFEM_TRY(s->F.alloc((size_t)n));
    MSFEM_TRY(s->X.alloc((size_t)n));
    if (F) MSFEM_CK(cudaMemcpyAsync(s->F.p, F, sizeof(double) * n, cudaMemcpyDefault, s->stream));
    else MSFEM_CK(cudaMemsetAsync(s->F.p, 0, sizeof(double) * n, s->stream));
    if (X) MSFEM_CK(cudaMemcpyAsync(s->X.p, X, sizeof(double) * n, cudaMemcpyDefault, s->stream));
    else MSFEM_CK(cudaMemsetAsync(s->X.p, 0, sizeof(double) * n, s->stream));
    MSFEM_CK(cudaStreamSynchronize(s->stream));
    *out = reinterpret_cast<msfem_system_t>(s.release());
    return MSFEM_OK;
}

int msfem_system_destroy(msfem_system_t h)
{
    if (!h) return MSFEM_OK;
    System* s = as_sys(h);
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    if (s->h_kstate) cudaFreeHost(s->h_kstate);
    if (s->h_ahead) cudaFreeHost(s->h_ahead);
    for (auto& e : s->ev_chunk)
        if (e) cudaEventDestroy(e);
    cudaStream_t st = s->stream;
    cudaEvent_t e0 = s->ev0, e1 = s->ev1;
    for (auto& kv : s->graphs)
        for (auto g : kv.second)
            if (g) cudaGraphExecDestroy(g);
    delete s;  // device buffers are released by their owners
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    return MSFEM_OK;
}

int msfem_system_info(msfem_system_t h, int* n_rows, int64_t* nnz, int* n_colors)
{
    MSFEM_TRY(check_handle(h));
    System* s = as_sys(h);
    if (n_rows) *n_rows = s->n_rows;
    if (nnz) *nnz = s->nnzb * s->bs * s->bs;
    if (n_colors) *n_colors = (int)s->color_off.size() - 1;
    return MSFEM_OK;
}

int msfem_get_stats(msfem_system_t h, msfem_stats* out)
{
    MSFEM_TRY(check_handle(h));
    as_sys(h)->stats.total_launches = as_sys(h)->total_launches;
    if (out) *out = as_sys(h)->stats;
    return MSFEM_OK;
}

void* msfem_get_stream(msfem_system_t h) { return h ? (void*)as_sys(h)->stream : nullptr; }

int msfem_clear(msfem_system_t h)
{
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    MSFEM_CK(cudaMemsetAsync(s.val.p, 0, sizeof(double) * s.val.n, s.stream));
    MSFEM_CK(cudaMemsetAsync(s.F.p, 0, sizeof(double) * s.F.n, s.stream));
    MSFEM_CK(cudaMemsetAsync(s.X.p, 0, sizeof(double) * s.X.n, s.stream));
    if (s.dmask.p) MSFEM_CK(cudaMemsetAsync(s.dmask.p, 0, sizeof(uint32_t) * s.dmask.n, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    s.elastic_form = 0;
    s.lame_host.clear();
    s.invalidate_values();
    return MSFEM_OK;
}

int msfem_assemble_scalar(msfem_system_t h, const double* sigma, int n_materials)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(need_mesh(*as_sys(h), "msfem_assemble_scalar"));
    MSFEM_TRY(use_device(*as_sys(h)));
    return assemble_scalar(*as_sys(h), sigma, n_materials);
}

int msfem_assemble_scalar3(msfem_system_t h, const double* S, const double* M, const double* f, int on_device)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(need_mesh(*as_sys(h), "msfem_assemble_scalar3"));
    MSFEM_TRY(use_device(*as_sys(h)));
    return assemble_scalar3(*as_sys(h), S, M, f, on_device != 0);
}

int msfem_assemble_elastic(msfem_system_t h, const double* E, const double* nu, int n_materials)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(need_mesh(*as_sys(h), "msfem_assemble_elastic"));
    MSFEM_TRY(use_device(*as_sys(h)));
    return assemble_elastic(*as_sys(h), E, nu, n_materials);
}

int msfem_assemble_elastic_textbook(msfem_system_t h, const double* E, const double* nu, int n_materials)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(need_mesh(*as_sys(h), "msfem_assemble_elastic_textbook"));
    MSFEM_TRY(use_device(*as_sys(h)));
    return assemble_elastic(*as_sys(h), E, nu, n_materials, true);
}

int msfem_add_traction(msfem_system_t h, int n_faces, const int32_t* face_nodes, const double* traction, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(need_mesh(s, "msfem_add_traction"));
    MSFEM_TRY(use_device(s));
    if (n_faces < 0 || (n_faces > 0 && (!face_nodes || !traction))) {
        set_error("msfem_add_traction: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    if (n_faces == 0) return MSFEM_OK;
    DBuf<int32_t>& f = s.sc_i32[0];
    DBuf<double>& t = s.sc_f64[0];
    MSFEM_TRY(to_device(s, f, face_nodes, 3 * (size_t)n_faces));
    MSFEM_TRY(to_device(s, t, traction, 3 * (size_t)n_faces));
    return add_traction(s, n_faces, f.p, t.p);
}

int msfem_add_rhs(msfem_system_t h, const double* f, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (!f) {
        set_error("msfem_add_rhs: null vector");
        return MSFEM_ERR_ARGUMENT;
    }
    DBuf<double>& d = s.sc_f64[0];
    MSFEM_TRY(to_device(s, d, f, (size_t)s.n_rows));
    k_add<<<grid_for(s.n_rows, 256), 256, 0, s.stream>>>(s.n_rows, d.p, s.F.p);
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 1;
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_apply_dirichlet(msfem_system_t h, int n, const int32_t* dofs, const double* values, int mode, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (n < 0 || (n > 0 && (!dofs || !values))) {
        set_error("msfem_apply_dirichlet: bad arguments");
        return MSFEM_ERR_ARGUMENT;
    }
    if (n == 0) return MSFEM_OK;
    DBuf<int32_t>& d = s.sc_i32[0];
    DBuf<double>& v = s.sc_f64[0];
    MSFEM_TRY(to_device(s, d, dofs, (size_t)n));
    MSFEM_TRY(to_device(s, v, values, (size_t)n));
    return apply_dirichlet(s, n, d.p, v.p, mode);
}

int msfem_set_x(msfem_system_t h, const double* x, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    MSFEM_CK(cudaMemcpyAsync(s.X.p, x, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_get_x(msfem_system_t h, double* x, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    MSFEM_CK(cudaMemcpyAsync(x, s.X.p, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_get_f(msfem_system_t h, double* f, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    MSFEM_CK(cudaMemcpyAsync(f, s.F.p, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_copy_f_to_x(msfem_system_t h)
{
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    MSFEM_CK(cudaMemcpyAsync(s.X.p, s.F.p, sizeof(double) * s.n_rows, cudaMemcpyDeviceToDevice, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_solve(msfem_system_t h, int method, int precision, int restart_m, int maxiter, double tol,
                double* rel_residual, int* iterations)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(use_device(*as_sys(h)));
    return solve(*as_sys(h), method, precision, restart_m, maxiter, tol, rel_residual, iterations);
}

int msfem_set_ssor_omega(msfem_system_t h, double omega)
{
    MSFEM_TRY(check_handle(h));
    if (!(omega > 0.0 && omega < 2.0)) {
        set_error("msfem_set_ssor_omega: omega must lie in (0, 2), got %g", omega);
        return MSFEM_ERR_ARGUMENT;
    }
    as_sys(h)->ssor_omega = omega;
    return MSFEM_OK;
}

int msfem_ssor_apply(msfem_system_t h, const double* r, double* z, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (!r || !z) {
        set_error("msfem_ssor_apply: null vector");
        return MSFEM_ERR_ARGUMENT;
    }
    DBuf<double> buf;
    MSFEM_TRY(buf.alloc(3 * (size_t)s.n_rows));
    MSFEM_CK(cudaMemcpyAsync(buf.p, r, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_TRY(ssor_apply(s, buf.p, buf.p + s.n_rows, buf.p + 2 * (size_t)s.n_rows, nullptr));
    MSFEM_CK(cudaMemcpyAsync(z, buf.p + s.n_rows, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_solve_driver_loop(msfem_system_t h, int loop, int method, int precision, double min_residual,
                            double* best_residual, int* n_solves, int* iterations)
{
    MSFEM_TRY(check_handle(h));
    MSFEM_TRY(use_device(*as_sys(h)));
    return driver_loop(*as_sys(h), loop, method, precision, min_residual, best_residual, n_solves, iterations);
}

int msfem_spmv(msfem_system_t h, const double* x, double* y, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    DBuf<double> dx, dy;
    MSFEM_TRY(to_device(s, dx, x, (size_t)s.n_rows));
    MSFEM_TRY(dy.alloc((size_t)s.n_rows));
    MSFEM_TRY(spmv64(s, dx.p, dy.p));
    MSFEM_CK(cudaMemcpyAsync(y, dy.p, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_spmv_scaled32(msfem_system_t h, const float* x, float* y, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    DBuf<float> dx, dy;
    MSFEM_TRY(dx.alloc((size_t)s.n_rows));
    MSFEM_TRY(dy.alloc((size_t)s.n_rows));
    MSFEM_CK(cudaMemcpyAsync(dx.p, x, sizeof(float) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_TRY(spmv32(s, dx.p, dy.p));
    MSFEM_CK(cudaMemcpyAsync(y, dy.p, sizeof(float) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_set_kuhn_grid(msfem_system_t h, int nx, int ny, int nz)
{
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    return kuhn_set_grid(s, nx, ny, nz);
}

int msfem_kuhn_spmv(msfem_system_t h, const double* x, double* y, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (!x || !y) {
        set_error("msfem_kuhn_spmv: null vector");
        return MSFEM_ERR_ARGUMENT;
    }
    KuhnOperator op;
    MSFEM_TRY(kuhn_operator_build(s, s.elastic_form, true, false, op));
    DBuf<double> dx, dy;
    MSFEM_TRY(dx.alloc((size_t)s.n_rows + 16));  // slack for the staging copies
    MSFEM_CK(cudaMemcpyAsync(dx.p, x, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_TRY(dy.alloc((size_t)s.n_rows));
    MSFEM_TRY(kuhn_spmv64(op, dx.p, dy.p, s.stream));
    MSFEM_CK(cudaMemcpyAsync(y, dy.p, sizeof(double) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    s.total_launches += 1;
    return MSFEM_OK;
}

int msfem_kuhn_spmv_scaled32(msfem_system_t h, const float* x, float* y, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (!x || !y) {
        set_error("msfem_kuhn_spmv_scaled32: null vector");
        return MSFEM_ERR_ARGUMENT;
    }
    KuhnOperator op;
    MSFEM_TRY(kuhn_operator_build(s, s.elastic_form, false, true, op));
    DBuf<float> dx, dxh, dy;
    MSFEM_TRY(dx.alloc((size_t)s.n_rows + 16));  // slack for the staging copies
    MSFEM_TRY(dxh.alloc((size_t)s.n_rows + 16));
    MSFEM_TRY(dy.alloc((size_t)s.n_rows));
    MSFEM_CK(cudaMemcpyAsync(dx.p, x, sizeof(float) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_TRY(kuhn_spmv32_pre(op, dx.p, dxh.p, dy.p, s.stream));
    MSFEM_TRY(kuhn_check_err(op, s.stream));
    MSFEM_CK(cudaMemcpyAsync(y, dy.p, sizeof(float) * s.n_rows, cudaMemcpyDefault, s.stream));
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_export_csr(msfem_system_t h, int32_t* row_ptr, int32_t* col, double* val, int on_device)
{
    (void)on_device;
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (!row_ptr || !col || !val) {
        set_error("msfem_export_csr: null output");
        return MSFEM_ERR_ARGUMENT;
    }
    if (s.bs == 1) {
        MSFEM_CK(cudaMemcpyAsync(row_ptr, s.nrp.p, sizeof(int32_t) * (s.n_nodes + 1), cudaMemcpyDefault, s.stream));
        MSFEM_CK(cudaMemcpyAsync(col, s.ncol.p, sizeof(int32_t) * s.nnzb, cudaMemcpyDefault, s.stream));
        MSFEM_CK(cudaMemcpyAsync(val, s.val.p, sizeof(double) * s.nnzb, cudaMemcpyDefault, s.stream));
    } else {
        const size_t nnz = 9 * (size_t)s.nnzb;
        DBuf<int32_t> rp, c;
        DBuf<double> v;
        MSFEM_TRY(rp.alloc((size_t)s.n_rows + 1));
        MSFEM_TRY(c.alloc(nnz));
        MSFEM_TRY(v.alloc(nnz));
        k_expand_rows<<<grid_for(s.n_rows + 1, 256), 256, 0, s.stream>>>(s.n_nodes, s.nrp.p, rp.p);
        k_expand_entries<<<grid_for(s.n_rows, 128), 128, 0, s.stream>>>(s.n_nodes, s.nrp.p, s.ncol.p, s.val.p, c.p, v.p);
        MSFEM_CK(cudaGetLastError());
        MSFEM_CK(cudaMemcpyAsync(row_ptr, rp.p, sizeof(int32_t) * (s.n_rows + 1), cudaMemcpyDefault, s.stream));
        MSFEM_CK(cudaMemcpyAsync(col, c.p, sizeof(int32_t) * nnz, cudaMemcpyDefault, s.stream));
        MSFEM_CK(cudaMemcpyAsync(val, v.p, sizeof(double) * nnz, cudaMemcpyDefault, s.stream));
        MSFEM_CK(cudaStreamSynchronize(s.stream));
    }
    MSFEM_CK(cudaStreamSynchronize(s.stream));
    return MSFEM_OK;
}

int msfem_bench_spmv(msfem_system_t h, int precision, int reps, double* ms_per_product, int64_t* bytes_per_product)
{
    MSFEM_TRY(check_handle(h));
    System& s = *as_sys(h);
    MSFEM_TRY(use_device(s));
    if (reps <= 0) {
        set_error("msfem_bench_spmv: reps must be > 0");
        return MSFEM_ERR_ARGUMENT;
    }
    MSFEM_TRY(prepare_sell(s));
    const int n = s.n_rows;
    const bool fp32 = precision == MSFEM_FP32_IR;
    const size_t w = fp32 ? 4 : 8;
    DBuf<unsigned char> xb, yb;
    MSFEM_TRY(xb.alloc(w * n));
    MSFEM_TRY(yb.alloc(w * n));
    MSFEM_CK(cudaMemsetAsync(xb.p, 0, w * n, s.stream));
    auto launch = [&]() -> int {
        if (fp32) return spmv32(s, reinterpret_cast<float*>(xb.p), reinterpret_cast<float*>(yb.p));
        return spmv64(s, reinterpret_cast<double*>(xb.p), reinterpret_cast<double*>(yb.p));
    };
    for (int i = 0; i < 3; i++) MSFEM_TRY(launch());
    MSFEM_CK(cudaEventRecord(s.ev0, s.stream));
    for (int i = 0; i < reps; i++) MSFEM_TRY(launch());
    MSFEM_CK(cudaEventRecord(s.ev1, s.stream));
    MSFEM_CK(cudaEventSynchronize(s.ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, s.ev0, s.ev1);
    if (ms_per_product) *ms_per_product = ms / reps;
    // algorithmic bytes: each nonzero's value and column index once (in the width the format
    // stores: 2 bytes for 16-bit column deltas, else 4), row structure once, x and y once
    if (bytes_per_product) {
        const int64_t nnz_alg = s.nnzb * s.bs * s.bs;
        const int64_t cw = (s.sell.col16.p && (!fp32 || s.sell.fp32_col16 == 1)) ? 2 : 4;
        if (s.bs == 1)
            *bytes_per_product = nnz_alg * (int64_t)(w + cw) + (int64_t)(n + 1) * 4 + 2 * (int64_t)n * w;
        else
            *bytes_per_product = s.nnzb * (int64_t)(9 * w + 4) + (int64_t)(s.n_nodes + 1) * 4 + 2 * (int64_t)n * w;
    }
    s.stats.ms_spmv = ms / reps;
    return MSFEM_OK;
}

}  // extern "C"
