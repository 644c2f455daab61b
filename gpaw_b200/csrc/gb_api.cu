// C ABI of gpaw_b200 (declared in include/gpaw_b200.h): object lifetimes,
// argument checks that mirror the reference's, and the host-side sequencing
// of the kernels in gb_fd.cu and gb_transform.cu.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gb_objects.cuh"
#include "gb_tma.cuh"

using namespace gb;

// ------------------------------------------------------------------- errors
static thread_local std::string g_err;

int gb::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}


extern "C" int gb_version(void) { return 100; }
extern "C" const char* gb_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------ tensor maps
namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    // through the runtime's driver entry point table: no link against libcuda
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return (EncodeTiledFn)f;
    }();
    return fn;
}
}  // namespace

int gb::make_plane_map16(CUtensorMap* map, const void* base, long long nb, int n0, int n1,
                         int n2, int box_rows, int box_cols, const char** why) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) {
        *why = "cuTensorMapEncodeTiled is not available";
        return -1;
    }
    // 8-byte words: a 16-byte element is two of them
    const cuuint64_t dims[4] = {(cuuint64_t)2 * n2, (cuuint64_t)n1, (cuuint64_t)n0,
                                (cuuint64_t)nb};
    const cuuint64_t strides[3] = {(cuuint64_t)n2 * 16, (cuuint64_t)n1 * n2 * 16,
                                   (cuuint64_t)n0 * n1 * n2 * 16};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * box_cols), (cuuint32_t)box_rows, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        *why = "cuTensorMapEncodeTiled refused the plane map";
        return -1;
    }
    return 0;
}

extern "C" int gb_device_fault(int* code) {
    if (!code) return fail(GB_EINVAL, "device_fault: NULL argument");
    *code = 0;
    int (*units[])(int*) = {take_fault_transform, take_fault_cfd, take_fault_mixed};
    for (auto take : units) {
        int c = 0;
        if (take(&c)) return fail(GB_ECUDA, "device_fault: cannot read the flag");
        if (c && !*code) *code = c;
    }
    return 0;
}

// ----------------------------------------------------------- kernel trace
// Profiling aid for composite entry points: while a trace is open, each
// kernel of gb_fd_precond is preceded by a CUDA event on the call's stream,
// and one more event follows the last kernel.
namespace {
struct Trace {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<const char*> label;
    int used = 0;
};
Trace g_trace;
}  // namespace

void gb::trace_mark(const char* label, cudaStream_t st) {
    if (!g_trace.on) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return;
    std::lock_guard<std::mutex> lock(g_trace.mu);
    if (!g_trace.on || g_trace.used >= (int)g_trace.ev.size()) return;
    if (cudaEventRecord(g_trace.ev[g_trace.used], st) != cudaSuccess) return;
    g_trace.label[g_trace.used++] = label;
}

extern "C" int gb_trace_begin(int capacity) {
    if (capacity < 2 || capacity > 1 << 16) return fail(GB_EINVAL, "trace: capacity 2..65536");
    std::lock_guard<std::mutex> lock(g_trace.mu);
    for (cudaEvent_t e : g_trace.ev) cudaEventDestroy(e);
    g_trace.ev.assign(capacity, nullptr);
    g_trace.label.assign(capacity, nullptr);
    for (int i = 0; i < capacity; i++)
        GB_CUDA_TRY(cudaEventCreate(&g_trace.ev[i]));
    g_trace.used = 0;
    g_trace.on = true;
    return 0;
}

extern "C" int gb_trace_end(int max, float* ms, const char** labels, int* count) {
    std::lock_guard<std::mutex> lock(g_trace.mu);
    g_trace.on = false;
    const int n = std::max(0, g_trace.used - 1);
    if (count) *count = n;
    if (g_trace.used > 0) GB_CUDA_TRY(cudaEventSynchronize(g_trace.ev[g_trace.used - 1]));
    for (int i = 0; i < n && i < max; i++) {
        float t = 0.f;
        GB_CUDA_TRY(cudaEventElapsedTime(&t, g_trace.ev[i], g_trace.ev[i + 1]));
        if (ms) ms[i] = t;
        if (labels) labels[i] = g_trace.label[i];
    }
    for (cudaEvent_t e : g_trace.ev) cudaEventDestroy(e);
    g_trace.ev.clear();
    g_trace.label.clear();
    g_trace.used = 0;
    return 0;
}

extern "C" int gb_operator_new(const double* coefs, const int64_t* offsets, int ncoefs,
                               const int64_t size[3], int range, const int64_t neighbors[6],
                               int real, int cfd, gb_operator** out) {
    if (!out || !coefs || !offsets || !size || !neighbors)
        return fail(GB_EINVAL, "Operator: NULL argument");
    *out = nullptr;
    if (ncoefs < 1 || ncoefs > GB_MAX_COEFS)
        return fail(GB_EINVAL, "Operator: %d coefficients (1..%d supported)", ncoefs, GB_MAX_COEFS);
    if (range < 0) return fail(GB_EINVAL, "Operator: negative range");
    for (int c = 0; c < 3; c++)
        if (size[c] < 1 || size[c] > (1 << 20)) return fail(GB_EINVAL, "Operator: bad size");
    if ((double)size[0] * size[1] * size[2] >= 2147483647.0)
        return fail(GB_EINVAL, "Operator: grid has 2^31 points or more");
    gb_operator* op = new gb_operator();
    memset(&op->st, 0, sizeof op->st);
    op->st.ncoefs = ncoefs;
    op->st.range = range;
    op->st.cfd = cfd ? 1 : 0;
    op->real = real ? 1 : 0;
    for (int c = 0; c < 3; c++) {
        op->g.n[c] = (int)size[c];
        const int64_t lo = neighbors[2 * c], hi = neighbors[2 * c + 1];
        if (lo > 0 || hi > 0) {
            delete op;
            return fail(GB_EINVAL, "Operator: neighbour ranks > 0 need domain decomposition");
        }
        // both sides periodic or both zero on a single domain
        op->g.periodic[c] = (lo == 0 && hi == 0) ? 1 : 0;
        if ((lo == 0) != (hi == 0)) {
            delete op;
            return fail(GB_EINVAL, "Operator: mixed periodic/zero on one axis");
        }
        if (op->g.periodic[c] && size[c] < range) {
            delete op;
            return fail(GB_EINVAL, "Stencil longer than domain");
        }
    }
    // Split each flat padded offset into (o0, o1, o2) with |o_c| <= range.
    op->diag = 0.0;
    for (int p = 0; p < ncoefs; p++) {
        const long long f = offsets[p];
        int o[3];
        if (!split_offset(f, size, range, o)) {
            delete op;
            return fail(GB_EINVAL, "Operator: offset %lld does not fit range %d", f, range);
        }
        op->st.coef[p] = coefs[p];
        op->st.off[p][0] = o[0];
        op->st.off[p][1] = o[1];
        op->st.off[p][2] = o[2];
        op->st.flat[p] = ((long long)o[0] * size[1] + o[1]) * size[2] + o[2];
        if (f == 0) op->diag = coefs[p];
    }
    const char* path = getenv("GPAW_B200_FD_PATH");
    const bool force_generic = path && strcmp(path, "generic") == 0;
    op->tiled = (!force_generic && to_cfd_stencil(op->st, op->cs, op->nn)) ? 1 : 0;
    *out = op;
    return 0;
}

extern "C" void gb_operator_free(gb_operator* op) { delete op; }

extern "C" double gb_operator_get_diagonal_element(const gb_operator* op) {
    return op ? op->diag : 0.0;
}

extern "C" int gb_operator_reserve(gb_operator* op, int64_t nin, int dtype) {
    if (!op) return fail(GB_EINVAL, "NULL operator");
    return op->scratch.ensure((size_t)(nin < 1 ? 1 : nin) * op->ng() * elem_size(dtype));
}

static int check_dtype(const gb_operator* op, int dtype) {
    if (dtype != GB_F64 && dtype != GB_C128) return fail(GB_EINVAL, "unsupported dtype %d", dtype);
    if ((dtype == GB_F64) != (op->real != 0))
        return fail(GB_EINVAL, "dtype does not match the operator (real=%d)", op->real);
    return 0;
}

extern "C" int gb_operator_apply(gb_operator* op, const void* in, void* out, int64_t nin,
                                 int dtype, const double* phases, void* stream) {
    if (!op || !in || !out) return fail(GB_EINVAL, "apply: NULL argument");
    if (int e = check_dtype(op, dtype)) return e;
    if (nin < 0) return fail(GB_EINVAL, "apply: negative batch");
    if (nin == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Phases P;
    read_phases(dtype, phases, P);
    const size_t bytes = (size_t)nin * op->ng() * elem_size(dtype);
    if (ranges_overlap(in, out, bytes)) {
        if (int e = op->scratch.ensure(bytes)) return e;
        GB_CUDA_TRY(cudaMemcpyAsync(op->scratch.ptr, in, bytes, cudaMemcpyDeviceToDevice, st));
        in = op->scratch.ptr;
    }
    if (int rc = op_sweep(op, EPI_APPLY, in, out, nullptr, (int)nin, dtype, P, 0, 0, 0, nullptr, st))
        return rc;
    GB_LAUNCH_CHECK();
    return 0;
}

extern "C" int gb_operator_apply_potential(gb_operator* op, const void* in, void* out,
                                           int64_t nin, int dtype, const double* phases,
                                           const double* v, void* stream) {
    if (!op || !in || !out || !v) return fail(GB_EINVAL, "apply_potential: NULL argument");
    if (int e = check_dtype(op, dtype)) return e;
    if (nin < 0) return fail(GB_EINVAL, "apply_potential: negative batch");
    if (nin == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Phases P;
    read_phases(dtype, phases, P);
    const size_t bytes = (size_t)nin * op->ng() * elem_size(dtype);
    const char* vb = (const char*)v;
    const char* ob = (const char*)out;
    if (vb < ob + bytes && ob < vb + (size_t)op->ng() * sizeof(double))
        return fail(GB_EINVAL, "apply_potential: v must not overlap out");
    if (ranges_overlap(in, out, bytes)) {
        if (int e = op->scratch.ensure(bytes)) return e;
        GB_CUDA_TRY(cudaMemcpyAsync(op->scratch.ptr, in, bytes, cudaMemcpyDeviceToDevice, st));
        in = op->scratch.ptr;
    }
    if (int rc = op_sweep(op, EPI_POT, in, out, v, (int)nin, dtype, P, 0, 0, 0, nullptr, st))
        return rc;
    GB_LAUNCH_CHECK();
    return 0;
}

extern "C" int gb_operator_set_chunk(gb_operator* op, int chunk) {
    if (!op) return fail(GB_EINVAL, "set_chunk: NULL operator");
    if (chunk < 0) return fail(GB_EINVAL, "set_chunk: chunk must be >= 0");
    op->chunk = chunk;
    return 0;
}

extern "C" int gb_transformer_set_chunk(gb_transformer* t, int chunk) {
    if (!t) return fail(GB_EINVAL, "set_chunk: NULL transformer");
    if (chunk < 0) return fail(GB_EINVAL, "set_chunk: chunk must be >= 0");
    t->G.chunk = chunk;
    return 0;
}

extern "C" int gb_operator_residual(gb_operator* op, const void* phi, const void* rho, void* r,
                                    int64_t nin, int dtype, const double* phases, double scale,
                                    double* norm2, void* stream) {
    if (!op || !phi || !rho) return fail(GB_EINVAL, "residual: NULL argument");
    if (int e = check_dtype(op, dtype)) return e;
    if (nin <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Phases P;
    read_phases(dtype, phases, P);
    const size_t bytes = (size_t)nin * op->ng() * elem_size(dtype);
    if (r && (ranges_overlap(phi, r, bytes)))
        return fail(GB_EINVAL, "residual: r must not overlap phi");
    double* partial = nullptr;
    const int nblk = op_resid_blocks(op, (int)nin, (int)elem_size(dtype));
    if (norm2) {
        if (int e = op->partial.ensure((size_t)nin * nblk * sizeof(double))) return e;
        partial = (double*)op->partial.ptr;
    }
    if (int rc = op_sweep(op, EPI_RESID, phi, r, rho, (int)nin, dtype, P, 0, 0, 0, partial, st))
        return rc;
    GB_LAUNCH_CHECK();
    if (norm2) {
        launch_reduce_partials(partial, nblk, (int)nin, scale, norm2, st);
        GB_LAUNCH_CHECK();
    }
    return 0;
}

// The relaxation itself, with its scratch grid X (op->ng() doubles) given by
// the caller: the operator's own buffer (gb_operator_relax) or the fixed
// device array of gb_operator_relax_noalloc.
static int relax_with_scratch(gb_operator* op, int method, double* f, const double* s,
                              int nrelax, double w, double* X, cudaStream_t st) {
    const size_t bytes = (size_t)op->ng() * sizeof(double);
    if (method == 1) {
        // Gauss-Seidel by wavefronts; wrapped reads see the sweep's start.
        const int r = op->st.range;
        int wa = 1, wb = 1;
        if (!op->st.cfd) {
            wb = 2 * r + 1;
            wa = (wb + 1) * r + 1;
        }
        const GridBC& g = op->g;
        const int nt = wa * (g.n[0] - 1) + wb * (g.n[1] - 1) + g.n[2];
        const bool periodic = g.periodic[0] || g.periodic[1] || g.periodic[2];
        const double inv0 = 1.0 / op->st.coef[0];
        for (int it = 0; it < nrelax; it++) {
            if (periodic) GB_CUDA_TRY(cudaMemcpyAsync(X, f, bytes, cudaMemcpyDeviceToDevice, st));
            for (int t = 0; t < nt; t++)
                launch_gs_wave(f, periodic ? X : f, s, g, op->st, t, wa, wb, inv0, st);
            GB_LAUNCH_CHECK();
        }
        return 0;
    }
    // weighted Jacobi: ping-pong so that the last sweep lands in f
    const double* src = f;
    if (nrelax % 2 == 1) {
        GB_CUDA_TRY(cudaMemcpyAsync(X, f, bytes, cudaMemcpyDeviceToDevice, st));
        src = X;
    }
    Phases P0;
    memset(&P0, 0, sizeof P0);
    for (int it = 0; it < nrelax; it++) {
        double* dst = (src == f) ? X : f;
        if (int rc = op_sweep(op, EPI_JACOBI, src, dst, s, 1, GB_F64, P0, w, 0, 0, nullptr, st))
            return rc;
        src = dst;
    }
    GB_LAUNCH_CHECK();
    return 0;
}

static int relax_impl(gb_operator* op, int method, double* f, const double* s, int nrelax,
                      double w, cudaStream_t st) {
    if (nrelax <= 0) return 0;
    if (int e = op->scratch.ensure((size_t)op->ng() * sizeof(double))) return e;
    return relax_with_scratch(op, method, f, s, nrelax, w, (double*)op->scratch.ptr, st);
}

extern "C" int gb_operator_relax(gb_operator* op, int method, double* f, const double* s,
                                 int nrelax, double w, void* stream) {
    if (!op || !f || !s) return fail(GB_EINVAL, "relax: NULL argument");
    if (!op->real) return fail(GB_EINVAL, "relax: float64 operators only");
    if (method != 1 && method != 2) return fail(GB_EINVAL, "relax: method must be 1 or 2");
    return relax_impl(op, method, f, s, nrelax, w, (cudaStream_t)stream);
}

// -------------------------------------------------------------- Transformer

static void lagrange_weights(int k, double* w) {
    // Weights of the order-k Lagrange interpolant at the mid-point, for the
    // node pairs at distance 1/2, 3/2, ... (exact binary fractions, equal to
    // the constants of c/bmgs/restrict.cpp:37-57).
    for (int j = k / 2; j < k; j++) {
        double num = 1.0, den = 1.0;
        const double xj = (2.0 * j - k + 1) / 2.0;
        for (int m = 0; m < k; m++) {
            if (m == j) continue;
            const double xm = (2.0 * m - k + 1) / 2.0;
            num *= (0.0 - xm);
            den *= (xj - xm);
        }
        w[j - k / 2] = num / den;
    }
}

extern "C" int gb_transformer_new(const int64_t size_in[3], const int64_t size_out[3], int k,
                                  const int64_t pads[6], const int64_t npads[6],
                                  const int64_t skip[6], const int64_t neighbors[6], int real,
                                  int interpolate, gb_transformer** out) {
    if (!out || !size_in || !size_out || !pads || !npads || !skip || !neighbors)
        return fail(GB_EINVAL, "Transformer: NULL argument");
    *out = nullptr;
    if (k != 2 && k != 4 && k != 6 && k != 8)
        return fail(GB_EINVAL, "Transformer: k must be 2, 4, 6 or 8");
    gb_transformer* t = new gb_transformer();
    memset(&t->G, 0, sizeof t->G);
    t->k = k;
    t->interpolate = interpolate ? 1 : 0;
    t->real = real ? 1 : 0;
    XferGeom& G = t->G;
    const int e = interpolate ? k - 1 : 2 * k - 3;
    for (int c = 0; c < 3; c++) {
        const int64_t lo = neighbors[2 * c], hi = neighbors[2 * c + 1];
        if (lo > 0 || hi > 0 || (lo == 0) != (hi == 0)) {
            delete t;
            return fail(GB_EINVAL, "Transformer: single-domain neighbours only");
        }
        G.g.n[c] = (int)size_in[c];
        G.g.periodic[c] = (lo == 0) ? 1 : 0;
        if (pads[2 * c] < 0 || pads[2 * c + 1] < 0) {
            delete t;
            return fail(GB_EINVAL, "Transformer: negative padding");
        }
        if (G.g.periodic[c] && (npads[2 * c] != pads[2 * c + 1] || npads[2 * c + 1] != pads[2 * c] ||
                                pads[2 * c] > size_in[c] || pads[2 * c + 1] > size_in[c])) {
            delete t;
            return fail(GB_EINVAL, "Transformer: periodic padding wider than the grid");
        }
        G.plo[c] = (int)pads[2 * c];
        G.s[c] = (int)(size_in[c] + pads[2 * c] + pads[2 * c + 1]);
        G.nout[c] = (int)size_out[c];
        G.skip0[c] = interpolate ? (int)skip[2 * c] : 0;
        G.skip1[c] = interpolate ? (int)skip[2 * c + 1] : 0;
        const int expect = interpolate ? 2 * (G.s[c] - e + G.skip1[c]) - G.skip0[c] - G.skip1[c]
                                       : (G.s[c] - e) / 2;
        if (expect != size_out[c]) {
            delete t;
            return fail(GB_EINVAL, "Transformer: output size %lld does not match input geometry (%d)",
                        (long long)size_out[c], expect);
        }
    }
    lagrange_weights(k, G.w);
    t->ngin = (long long)size_in[0] * size_in[1] * size_in[2];
    t->ngout = (long long)size_out[0] * size_out[1] * size_out[2];
    *out = t;
    return 0;
}

extern "C" void gb_transformer_free(gb_transformer* t) { delete t; }

extern "C" int gb_transformer_apply(gb_transformer* t, const void* in, void* out, int64_t nin,
                                    int dtype, const double* phases, void* stream) {
    if (!t || !in || !out) return fail(GB_EINVAL, "transformer apply: NULL argument");
    if (dtype != GB_F64 && dtype != GB_C128) return fail(GB_EINVAL, "unsupported dtype");
    if ((dtype == GB_F64) != (t->real != 0))
        return fail(GB_EINVAL, "dtype does not match the transformer (real=%d)", t->real);
    if (nin <= 0) return 0;
    const size_t es = elem_size(dtype);
    const char* ib = (const char*)in;
    const char* ob = (const char*)out;
    if (ib < ob + nin * t->ngout * es && ob < ib + nin * t->ngin * es)
        return fail(GB_EINVAL, "transformer apply: input and output overlap");
    Phases P;
    read_phases(dtype, phases, P);
    return transform_impl(t, in, out, nullptr, nin, dtype, P, 0, 0, 0.0, (cudaStream_t)stream);
}

// --------------------------------------------------------------- fd_precond
extern "C" int gb_fd_precond(gb_transformer* rest0, gb_transformer* rest1, gb_transformer* intp1,
                             gb_transformer* intp2, gb_operator* kin0, gb_operator* kin1,
                             gb_operator* kin2, void* d0, void* q0, void* r1, void* d1, void* q1,
                             void* r2, void* d2, void* q2, const void* residuals,
                             const void* nresiduals, int64_t nin, int dtype, double step,
                             const double* phases, void* stream) {
    if (!rest0 || !rest1 || !intp1 || !intp2 || !kin0 || !kin1 || !kin2)
        return fail(GB_EINVAL, "fd_precond: NULL object");
    if (!d0 || !q0 || !r1 || !d1 || !q1 || !r2 || !d2 || !q2 || !residuals)
        return fail(GB_EINVAL, "fd_precond: NULL array");
    if (int e = check_dtype(kin0, dtype)) return e;
    if (int e = check_dtype(kin1, dtype)) return e;
    if (int e = check_dtype(kin2, dtype)) return e;
    if (rest0->ngin != kin0->ng() || rest0->ngout != kin1->ng() || rest1->ngin != kin1->ng() ||
        rest1->ngout != kin2->ng() || intp2->ngin != kin2->ng() || intp2->ngout != kin1->ng() ||
        intp1->ngin != kin1->ng() || intp1->ngout != kin0->ng() || rest0->interpolate ||
        rest1->interpolate || !intp1->interpolate || !intp2->interpolate)
        return fail(GB_EINVAL, "fd_precond: level sizes do not match");
    if (nin <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Phases P;
    read_phases(dtype, phases, P);
    const int n = (int)nin;
    const double s4 = 4 * step, s16 = 16 * step;
    // real grids of at least 2^18 points: the pass kernel (two points a
    // thread from 16-byte shared-memory reads, the same arithmetic) unless
    // GPAW_B200_PASS=0.  128 x 112^3 (C4): 1.64 -> 1.16 ms for the level-0
    // step; on the 56^3 level it was slower (0.13 -> 0.16 ms).
    static const bool pass = [] {
        const char* e = getenv("GPAW_B200_PASS");
        return !(e && atoi(e) == 0);
    }();
    auto step_launch = [&](gb_operator* op, const void* d, const void* r, void* o, double sc,
                           int negate) {
        if (pass && dtype == GB_F64 && op->tiled && d != o && r != o &&
            op->ng() >= (1ll << 18)) {
            const int rc = launch_pass_precond(op->g, op->cs, op->nn, (const double*)d,
                                               (double*)o, (const double*)r, n, sc, negate, st);
            if (rc == 0) {
                GB_LAUNCH_CHECK();
                return 0;
            }
            if (rc == -2) return fail(GB_ECUDA, "precond: could not raise the shared-memory limit");
        }
        return op_sweep(op, EPI_PRECOND, d, o, r, n, dtype, P, 0, sc, negate, nullptr, st);
    };
    int rc;
    // r1 = restrict(-R); d1 = 4 s r1
    trace_mark("restrict0 r1,d1 = R(-R), 4s r1", st);
    if (nresiduals)
        rc = transform_impl(rest0, nresiduals, r1, d1, nin, dtype, P, 0, 0, s4, st);
    else
        rc = transform_impl(rest0, residuals, r1, d1, nin, dtype, P, 1, 0, s4, st);
    if (rc) return rc;
    // q1 = K1 d1 - r1; r2 = restrict(q1); d2 = 16 s r2
    trace_mark("kin1 q1 = K1 d1 - r1", st);
    if ((rc = op_sweep(kin1, EPI_RESID, d1, q1, r1, n, dtype, P, 0, 0, 0, nullptr, st))) return rc;
    GB_LAUNCH_CHECK();
    trace_mark("restrict1 r2,d2 = R(q1), 16s r2", st);
    if ((rc = transform_impl(rest1, q1, r2, d2, nin, dtype, P, 0, 0, s16, st))) return rc;
    // d2' = d2 - 16 s (K2 d2 - r2)   (into q2)
    trace_mark("kin2 q2 = d2 - 16s(K2 d2 - r2)", st);
    if ((rc = step_launch(kin2, d2, r2, q2, s16, 0))) return rc;
    GB_LAUNCH_CHECK();
    // d1 -= interpolate(d2')
    trace_mark("interp2 d1 -= I(q2)", st);
    if ((rc = transform_impl(intp2, q2, d1, nullptr, nin, dtype, P, 0, 1, 0.0, st))) return rc;
    // d1' = d1 - 4 s (K1 d1 - r1)   (into q1)
    trace_mark("kin1 q1 = d1 - 4s(K1 d1 - r1)", st);
    if ((rc = step_launch(kin1, d1, r1, q1, s4, 0))) return rc;
    GB_LAUNCH_CHECK();
    // q0 = interpolate(-d1')
    trace_mark("interp1 q0 = I(-q1)", st);
    if ((rc = transform_impl(intp1, q1, q0, nullptr, nin, dtype, P, 1, 0, 0.0, st))) return rc;
    // d0 = -(q0 - s (K0 q0 - R))
    trace_mark("kin0 d0 = -(q0 - s(K0 q0 - R))", st);
    if ((rc = step_launch(kin0, q0, residuals, d0, step, 1))) return rc;
    GB_LAUNCH_CHECK();
    trace_mark("end", st);
    return 0;
}

// --------------------------------------------------------------- FD Poisson
struct SolveCtl {
    double eps;
    double err;
    int maxiter;
    int niter;
};

// After each V-cycle: niter += 1; keep looping while err > eps and
// niter < maxiter (gpaw/poisson.py:484-486).
__global__ void k_solve_check(SolveCtl* ctl, const double* err, cudaGraphConditionalHandle h) {
    const int n = ctl->niter + 1;
    ctl->niter = n;
    ctl->err = err[0];
    cudaGraphSetConditional(h, (err[0] > ctl->eps && n < ctl->maxiter) ? 1u : 0u);
}

__global__ void k_solve_init(SolveCtl* ctl, double eps, int maxiter) {
    ctl->eps = eps;
    ctl->maxiter = maxiter;
    ctl->niter = 0;
    ctl->err = 0.0;
}

// ------------------------------------------------ fused coarse-level V-cycle
// The coarse levels of a multigrid hierarchy hold a few thousand points or
// fewer, so each of their sweeps, residuals and transfers is one short
// launch.  When every level from `lf` down is small, one CTA runs the whole
// V-cycle below lf (iterate2 from level lf on, gpaw/poisson.py:500-537)
// with all arrays in shared memory: weighted-Jacobi sweeps, the residual,
// the K = 2 restriction and interpolation (three separable passes each, axis
// 2, then 1, then 0, as bmgs_restrict / bmgs_interpolate order them,
// c/bmgs/restrict.cpp:137-156, c/bmgs/interpolate.cpp:70-99).  Every value
// is computed with the same operations in the same order as the per-level
// kernels, so the V-cycle is bit-identical to them.
namespace gb {
constexpr int TAIL_MAX = 8;
struct TailLevel {
    int n[3];
    int per[3];
    int ng;
    int phi, rho, tmp;        // offsets (doubles) of this level's arrays
    double c0, cp[3], cm[3];  // 2nd-order stencil: direction k runs along axis 2 - k
    int pre, post;
    double w;
    int rplo[3];              // restriction to the next level: input padding
    double rw;                //   and mid-point weight
    int iplo[3], iskip[3];    // interpolation from the next level: padding, skip
    double iw;
};
struct TailPlan {
    int nl;        // levels handled (lf .. L)
    int scratch;   // offset of the transfer passes' intermediate arrays
    TailLevel lv[TAIL_MAX];
};

// i / n for 0 <= i < 2^22 through a float reciprocal (inv = 1/n rounded):
// the float quotient is within 1e-3 of i / n, so one correction step gives
// the exact integer quotient
__device__ __forceinline__ int tail_div(int i, int n, float inv) {
    int q = __float2int_rz(__fmul_rn((float)i, inv));
    const int r = i - q * n;
    if (r < 0) q -= 1;
    else if (r >= n) q += 1;
    return q;
}

// index along one axis after the boundary condition; -1 reads zero
__device__ __forceinline__ int tail_at(int j, int n, int per) {
    if (j >= 0 && j < n) return j;
    if (!per) return -1;
    j = j < 0 ? j + n : j - n;
    return (j >= 0 && j < n) ? j : -1;
}

// neighbour at +1 / -1 of point i (coordinate c, extent n, stride s)
__device__ __forceinline__ double tail_up(const double* __restrict__ A, int i, int c, int n,
                                          int per, int s) {
    return (c + 1 < n) ? A[i + s] : (per ? A[i + s - n * s] : 0.0);
}
__device__ __forceinline__ double tail_dn(const double* __restrict__ A, int i, int c, int n,
                                          int per, int s) {
    return (c > 0) ? A[i - s] : (per ? A[i - s + n * s] : 0.0);
}

// x = 0 (+ v c0) + v(+1) c(+1) + v(-1) c(-1) per direction, axis 2, 1, 0
template <bool CENTRE>
__device__ __forceinline__ double tail_stencil(const double* __restrict__ A, const TailLevel& L,
                                               int i, int i0, int i1, int i2) {
    const int n1 = L.n[1], n2 = L.n[2];
    double x = 0.0;
    if (CENTRE) x = __dadd_rn(x, __dmul_rn(A[i], L.c0));
    x = __dadd_rn(x, __dmul_rn(tail_up(A, i, i2, n2, L.per[2], 1), L.cp[0]));
    x = __dadd_rn(x, __dmul_rn(tail_dn(A, i, i2, n2, L.per[2], 1), L.cm[0]));
    x = __dadd_rn(x, __dmul_rn(tail_up(A, i, i1, n1, L.per[1], n2), L.cp[1]));
    x = __dadd_rn(x, __dmul_rn(tail_dn(A, i, i1, n1, L.per[1], n2), L.cm[1]));
    x = __dadd_rn(x, __dmul_rn(tail_up(A, i, i0, L.n[0], L.per[0], n1 * n2), L.cp[2]));
    x = __dadd_rn(x, __dmul_rn(tail_dn(A, i, i0, L.n[0], L.per[0], n1 * n2), L.cm[2]));
    return x;
}

// split a flat index of an (., b, c) array into its three coordinates
__device__ __forceinline__ void tail_split(int i, int b, int c, float ibc, float ic, int& i0,
                                           int& i1, int& i2) {
    i0 = tail_div(i, b * c, ibc);
    const int r = i - i0 * b * c;
    i1 = tail_div(r, c, ic);
    i2 = r - i1 * c;
}

// MODE 0: one weighted-Jacobi sweep A -> B (c/bmgs/relax.cpp:41-65);
// MODE 1: the residual B = L A - rho
template <int MODE>
__device__ void tail_pass(const double* __restrict__ A, const double* __restrict__ R,
                          double* __restrict__ B, const TailLevel& L) {
    const int n1 = L.n[1], n2 = L.n[2];
    const float i12 = __frcp_rn((float)(n1 * n2)), i2f = __frcp_rn((float)n2);
    const double w1 = 1.0 - L.w;
    for (int i = threadIdx.x; i < L.ng; i += blockDim.x) {
        int i0, i1, i2;
        tail_split(i, n1, n2, i12, i2f, i0, i1, i2);
        if (MODE == 0) {
            const double x = tail_stencil<false>(A, L, i, i0, i1, i2);
            B[i] = __dadd_rn(__dmul_rn(w1, A[i]),
                             __ddiv_rn(__dmul_rn(L.w, __dsub_rn(R[i], x)), L.c0));
        } else {
            B[i] = __dsub_rn(tail_stencil<true>(A, L, i, i0, i1, i2), R[i]);
        }
    }
    __syncthreads();
}

// n weighted-Jacobi sweeps of the level's phi, held in buffer b (phi or
// tmp); returns the buffer that holds the result
__device__ __forceinline__ int tail_other(const TailLevel& L, int b) {
    return b == L.phi ? L.tmp : L.phi;
}
__device__ __forceinline__ int tail_after(const TailLevel& L, int b, int n) {
    return (n & 1) ? tail_other(L, b) : b;
}
__device__ int tail_relax(double* sm, const TailLevel& L, int b, int n) {
    for (int it = 0; it < n; it++) {
        tail_pass<0>(sm + b, sm + L.rho, sm + tail_other(L, b), L);
        b = tail_other(L, b);
    }
    return b;
}

// mid-point restriction of one line value, K = 2: 0.5 (a + w (a+ + a-))
__device__ __forceinline__ double tail_r1(const double* __restrict__ a, int j, int n, int per,
                                          int s, double w) {
    const int j0 = tail_at(j, n, per), jp = tail_at(j + 1, n, per), jm = tail_at(j - 1, n, per);
    const double v = j0 < 0 ? 0.0 : a[j0 * s];
    const double vp = jp < 0 ? 0.0 : a[jp * s];
    const double vm = jm < 0 ? 0.0 : a[jm * s];
    return __dmul_rn(0.5, __dadd_rn(v, __dmul_rn(w, __dadd_rn(vp, vm))));
}

// restriction of A (level F, extents n) into out (level C, extents m)
__device__ void tail_restrict(const TailLevel& F, const TailLevel& C,
                              const double* __restrict__ A, double* __restrict__ out,
                              double* __restrict__ tA, double* __restrict__ tB) {
    const int n0 = F.n[0], n1 = F.n[1], n2 = F.n[2];
    const int m0 = C.n[0], m1 = C.n[1], m2 = C.n[2];
    const float im2 = __frcp_rn((float)m2), im12 = __frcp_rn((float)(m1 * m2));
    // axis 2: (n0, n1, m2)
    for (int i = threadIdx.x; i < n0 * n1 * m2; i += blockDim.x) {
        const int r = tail_div(i, m2, im2), c = i - r * m2;
        tA[i] = tail_r1(A + r * n2, 2 * c + 1 - F.rplo[2], n2, F.per[2], 1, F.rw);
    }
    __syncthreads();
    // axis 1: (n0, m1, m2)
    for (int i = threadIdx.x; i < n0 * m1 * m2; i += blockDim.x) {
        int i0, c1, c2;
        tail_split(i, m1, m2, im12, im2, i0, c1, c2);
        tB[i] = tail_r1(tA + i0 * n1 * m2 + c2, 2 * c1 + 1 - F.rplo[1], n1, F.per[1], m2, F.rw);
    }
    __syncthreads();
    // axis 0: (m0, m1, m2)
    for (int i = threadIdx.x; i < m0 * m1 * m2; i += blockDim.x) {
        const int c0 = tail_div(i, m1 * m2, im12), r = i - c0 * m1 * m2;
        out[i] = tail_r1(tB + r, 2 * c0 + 1 - F.rplo[0], n0, F.per[0], m1 * m2, F.rw);
    }
    __syncthreads();
}

// interpolated value at fine index f of one line a[j * s] of the coarse
// level (length n, its boundary condition): the even outputs copy, the odd
// ones are w (a(k) + a(k+1)) (c/bmgs/interpolate.cpp:10-46, K = 2)
__device__ __forceinline__ double tail_i1(const double* __restrict__ a, int f, int skip, int plo,
                                          int n, int per, int s, double w) {
    const int u = f + skip;
    const int k = u >> 1;
    const int j = tail_at(k - plo, n, per);
    const double v = j < 0 ? 0.0 : a[j * s];
    if (!(u & 1)) return v;
    const int j1 = tail_at(k + 1 - plo, n, per);
    return __dmul_rn(w, __dadd_rn(v, j1 < 0 ? 0.0 : a[j1 * s]));
}

// phi (level F, extents n) -= interpolation of B (level C, extents m)
__device__ void tail_interp_sub(const TailLevel& F, const TailLevel& C,
                                const double* __restrict__ B, double* __restrict__ phi,
                                double* __restrict__ tA, double* __restrict__ tB) {
    const int n0 = F.n[0], n1 = F.n[1], n2 = F.n[2];
    const int m0 = C.n[0], m1 = C.n[1], m2 = C.n[2];
    const float in2 = __frcp_rn((float)n2), in12 = __frcp_rn((float)(n1 * n2));
    // axis 2: (m0, m1, n2)
    for (int i = threadIdx.x; i < m0 * m1 * n2; i += blockDim.x) {
        const int r = tail_div(i, n2, in2), f = i - r * n2;
        tA[i] = tail_i1(B + r * m2, f, F.iskip[2], F.iplo[2], m2, C.per[2], 1, F.iw);
    }
    __syncthreads();
    // axis 1: (m0, n1, n2)
    for (int i = threadIdx.x; i < m0 * n1 * n2; i += blockDim.x) {
        int c0, f1, f2;
        tail_split(i, n1, n2, in12, in2, c0, f1, f2);
        tB[i] = tail_i1(tA + c0 * m1 * n2 + f2, f1, F.iskip[1], F.iplo[1], m1, C.per[1], n2,
                        F.iw);
    }
    __syncthreads();
    // axis 0: (n0, n1, n2), subtracted from phi
    for (int i = threadIdx.x; i < n0 * n1 * n2; i += blockDim.x) {
        const int f0 = tail_div(i, n1 * n2, in12), r = i - f0 * n1 * n2;
        const double v = tail_i1(tB + r, f0, F.iskip[0], F.iplo[0], m0, C.per[0], n1 * n2, F.iw);
        phi[i] = __dsub_rn(phi[i], v);
    }
    __syncthreads();
}

// The V-cycle from level lf down: rho_g is that level's right-hand side,
// phi_g receives its correction (the level starts from zero).
__global__ void __launch_bounds__(1024, 1)
k_tail_vcycle(const double* __restrict__ rho_g, double* __restrict__ phi_g, TailPlan plan) {
    extern __shared__ __align__(16) double tail_sm[];
    double* sm = tail_sm;
    const TailLevel& L0 = plan.lv[0];
    for (int i = threadIdx.x; i < L0.ng; i += blockDim.x) {
        sm[L0.rho + i] = rho_g[i];
        sm[L0.phi + i] = 0.0;
    }
    __syncthreads();
    double* tA = sm + plan.scratch;
    const int last = plan.nl - 1;
    for (int l = 0; l < last; l++) {
        const TailLevel& L = plan.lv[l];
        const TailLevel& C = plan.lv[l + 1];
        const int cur = tail_relax(sm, L, L.phi, L.pre);
        const int fre = tail_other(L, cur);
        tail_pass<1>(sm + cur, sm + L.rho, sm + fre, L);
        tail_restrict(L, C, sm + fre, sm + C.rho, tA, tA + L.n[0] * L.n[1] * C.n[2]);
        for (int i = threadIdx.x; i < C.ng; i += blockDim.x) sm[C.phi + i] = 0.0;
        __syncthreads();
    }
    const TailLevel& LL = plan.lv[last];
    int fin = tail_relax(sm, LL, LL.phi, LL.post);
    for (int l = last - 1; l >= 0; l--) {
        const TailLevel& L = plan.lv[l];
        const TailLevel& C = plan.lv[l + 1];
        const int cur = tail_after(L, L.phi, L.pre);
        tail_interp_sub(L, C, sm + fin, sm + cur, tA, tA + C.n[0] * C.n[1] * L.n[2]);
        fin = tail_relax(sm, L, cur, L.post);
    }
    for (int i = threadIdx.x; i < L0.ng; i += blockDim.x) phi_g[i] = sm[fin + i];
}
}  // namespace gb

struct gb_poisson {
    int L;  // coarsest level index
    int tail_lf = -1;           // first level of the fused coarse V-cycle (-1: none)
    size_t tail_smem = 0;
    gb::TailPlan tail;
    std::vector<gb_operator*> ops;
    std::vector<gb_transformer*> rst, itp;
    std::vector<int> pre, post;
    std::vector<double> w;
    int method;
    double dv;
    std::vector<double*> phi, rho, res;  // per level (phi[0], rho[0] from the caller)
    double* partial = nullptr;
    double* err_dev = nullptr;
    double* err_host = nullptr;
    double* mean_dev = nullptr;
    // device-resident solve: own copies of phi0/rho0, a control block and a
    // graph holding   while (err > eps && niter < maxiter) { V-cycle }
    double* phi0 = nullptr;
    double* rho0 = nullptr;
    SolveCtl* ctl = nullptr;
    SolveCtl* ctl_host = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t solve_exec = nullptr;
    int last_maxiter = 0;
    ~gb_poisson() {
        if (solve_exec) cudaGraphExecDestroy(solve_exec);
        if (cap) cudaStreamDestroy(cap);
        dfree(phi0);
        dfree(rho0);
        dfree(ctl);
        if (ctl_host) hfree(ctl_host);
        for (size_t l = 1; l < phi.size(); l++) dfree(phi[l]);
        for (size_t l = 1; l < rho.size(); l++) dfree(rho[l]);
        for (double* p : res) dfree(p);
        dfree(partial);
        dfree(err_dev);
        dfree(mean_dev);
        if (err_host) hfree(err_host);
    }
};

// Pick the first level of the fused coarse V-cycle: the coarsest run of
// levels (below level 0) whose operators are 2nd-order axis-aligned
// Laplacians, whose transfers are K = 2, that relax by weighted Jacobi,
// whose first level holds at most TAIL_POINTS points and whose arrays fit
// in shared memory.  GPAW_B200_POISSON_TAIL=0 keeps every level on the
// per-level kernels (same results).
static void plan_tail(gb_poisson* p) {
    constexpr long long TAIL_POINTS = 4096;
    constexpr size_t TAIL_SMEM = 200 * 1024;
    p->tail_lf = -1;
    const char* env = getenv("GPAW_B200_POISSON_TAIL");
    if ((env && atoi(env) == 0) || p->method != 2 || p->L < 1) return;
    auto level_ok = [&](int l) {
        const gb_operator* op = p->ops[l];
        if (!op->tiled || op->nn != 1 || !op->real) return false;
        if (!(op->cs.axis[0] == 2 && op->cs.axis[1] == 1 && op->cs.axis[2] == 0)) return false;
        if (l < p->L) {
            const gb_transformer* r = p->rst[l];
            const gb_transformer* i = p->itp[l];
            if (r->k != 2 || i->k != 2) return false;
            for (int c = 0; c < 3; c++) {
                if (r->G.g.n[c] != op->g.n[c] || r->G.g.periodic[c] != op->g.periodic[c] ||
                    r->G.nout[c] != p->ops[l + 1]->g.n[c] ||
                    i->G.g.n[c] != p->ops[l + 1]->g.n[c] ||
                    i->G.g.periodic[c] != p->ops[l + 1]->g.periodic[c] ||
                    i->G.nout[c] != op->g.n[c])
                    return false;
            }
        }
        return true;
    };
    auto smem_from = [&](int lf) {
        size_t d = 0, scratch = 0;
        for (int l = lf; l <= p->L; l++) {
            d += 3 * (size_t)p->ops[l]->ng();
            if (l < p->L) {
                const int* n = p->ops[l]->g.n;
                const int* m = p->ops[l + 1]->g.n;
                const size_t r = (size_t)n[0] * n[1] * m[2] + (size_t)n[0] * m[1] * m[2];
                const size_t i = (size_t)m[0] * m[1] * n[2] + (size_t)m[0] * n[1] * n[2];
                scratch = std::max(scratch, std::max(r, i));
            }
        }
        return (d + scratch) * sizeof(double);
    };
    int lf = -1;
    for (int l = p->L; l >= 1; l--) {
        if (!level_ok(l) || p->ops[l]->ng() > TAIL_POINTS || smem_from(l) > TAIL_SMEM ||
            p->L - l + 1 > gb::TAIL_MAX)
            break;
        lf = l;
    }
    if (lf < 0) return;
    gb::TailPlan& T = p->tail;
    memset(&T, 0, sizeof T);
    T.nl = p->L - lf + 1;
    int off = 0;
    for (int k = 0; k < T.nl; k++) {
        const int l = lf + k;
        const gb_operator* op = p->ops[l];
        gb::TailLevel& V = T.lv[k];
        V.ng = (int)op->ng();
        for (int c = 0; c < 3; c++) {
            V.n[c] = op->g.n[c];
            V.per[c] = op->g.periodic[c];
        }
        V.phi = off;
        V.rho = off + V.ng;
        V.tmp = off + 2 * V.ng;
        off += 3 * V.ng;
        V.c0 = op->cs.c0;
        for (int d = 0; d < 3; d++) {
            V.cp[d] = op->cs.cp[d][0];
            V.cm[d] = op->cs.cm[d][0];
        }
        V.pre = p->pre[l];
        V.post = p->post[l];
        V.w = p->w[l];
        if (l < p->L) {
            const gb_transformer* r = p->rst[l];
            const gb_transformer* i = p->itp[l];
            for (int c = 0; c < 3; c++) {
                V.rplo[c] = r->G.plo[c];
                V.iplo[c] = i->G.plo[c];
                V.iskip[c] = i->G.skip0[c];
            }
            V.rw = r->G.w[0];
            V.iw = i->G.w[0];
        }
    }
    T.scratch = off;
    p->tail_smem = smem_from(lf);
    p->tail_lf = lf;
}

static int launch_tail(gb_poisson* p, cudaStream_t st) {
    static bool attr_done = false;
    if (!attr_done) {
        GB_CUDA_TRY(cudaFuncSetAttribute(gb::k_tail_vcycle,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024));
        attr_done = true;
    }
    const int lf = p->tail_lf;
    gb::k_tail_vcycle<<<1, 1024, p->tail_smem, st>>>(p->rho[lf], p->phi[lf], p->tail);
    GB_LAUNCH_CHECK();
    return 0;
}

extern "C" int gb_poisson_new(int nlevels, gb_operator* const* operators,
                              gb_transformer* const* restrictors,
                              gb_transformer* const* interpolators, const int* presmooths,
                              const int* postsmooths, const double* weights, int relax_method,
                              double dv, gb_poisson** out) {
    if (!out || !operators || nlevels < 1 || !presmooths || !postsmooths || !weights)
        return fail(GB_EINVAL, "Poisson: bad arguments");
    if (nlevels > 1 && (!restrictors || !interpolators))
        return fail(GB_EINVAL, "Poisson: missing transformers");
    if (relax_method != 1 && relax_method != 2)
        return fail(GB_EINVAL, "Poisson: relax method must be 1 (GS) or 2 (J)");
    *out = nullptr;
    gb_poisson* p = new gb_poisson();
    p->L = nlevels - 1;
    p->method = relax_method;
    p->dv = dv;
    for (int l = 0; l < nlevels; l++) {
        if (!operators[l] || !operators[l]->real) {
            delete p;
            return fail(GB_EINVAL, "Poisson: level %d operator missing or complex", l);
        }
        p->ops.push_back(operators[l]);
        p->pre.push_back(presmooths[l]);
        p->post.push_back(postsmooths[l]);
        p->w.push_back(weights[l]);
    }
    for (int l = 0; l < p->L; l++) {
        gb_transformer* r = restrictors[l];
        gb_transformer* i = interpolators[l];
        if (!r || !i || r->interpolate || !i->interpolate || !r->real || !i->real ||
            r->ngin != p->ops[l]->ng() || r->ngout != p->ops[l + 1]->ng() ||
            i->ngin != p->ops[l + 1]->ng() || i->ngout != p->ops[l]->ng()) {
            delete p;
            return fail(GB_EINVAL, "Poisson: transformer %d does not match the levels", l);
        }
        p->rst.push_back(r);
        p->itp.push_back(i);
    }
    plan_tail(p);
    p->phi.assign(nlevels, nullptr);
    p->rho.assign(nlevels, nullptr);
    p->res.assign(nlevels, nullptr);
    for (int l = 0; l < nlevels; l++) {
        const size_t bytes = (size_t)p->ops[l]->ng() * sizeof(double);
        cudaError_t e = pool_malloc(&p->res[l], bytes);
        if (e == cudaSuccess && l > 0) e = pool_malloc(&p->phi[l], bytes);
        if (e == cudaSuccess && l > 0) e = pool_malloc(&p->rho[l], bytes);
        if (e != cudaSuccess) {
            delete p;
            return fail(GB_ECUDA, "Poisson: cudaMalloc: %s", cudaGetErrorString(e));
        }
        if (int rc = gb_operator_reserve(p->ops[l], 1, GB_F64)) {
            delete p;
            return rc;
        }
    }
    const int nblk = std::max(residual_blocks(p->ops[0]->g), op_resid_blocks(p->ops[0], 1, 8));
    cudaError_t e = pool_malloc(&p->partial, (size_t)nblk * sizeof(double));
    if (e == cudaSuccess) e = pool_malloc(&p->err_dev, sizeof(double));
    if (e == cudaSuccess) e = pool_malloc(&p->mean_dev, sizeof(double));
    if (e == cudaSuccess) e = pool_malloc_host(&p->err_host, sizeof(double));
    const size_t bytes0 = (size_t)p->ops[0]->ng() * sizeof(double);
    if (e == cudaSuccess) e = pool_malloc(&p->phi0, bytes0);
    if (e == cudaSuccess) e = pool_malloc(&p->rho0, bytes0);
    if (e == cudaSuccess) e = pool_malloc(&p->ctl, sizeof(SolveCtl));
    if (e == cudaSuccess) e = pool_malloc_host(&p->ctl_host, sizeof(SolveCtl));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete p;
        return fail(GB_ECUDA, "Poisson: allocation: %s", cudaGetErrorString(e));
    }
    *out = p;
    return 0;
}

extern "C" void gb_poisson_free(gb_poisson* p) { delete p; }

extern "C" int gb_poisson_fused_levels(const gb_poisson* p) {
    return (p && p->tail_lf >= 0) ? p->tail.nl : 0;
}

// iterate2 (gpaw/poisson.py:500-537), recursive over levels.
static int vcycle(gb_poisson* p, int l, cudaStream_t st) {
    if (l == p->tail_lf) return launch_tail(p, st);   // starts from phi_l = 0 itself
    gb_operator* op = p->ops[l];
    Phases P;
    memset(&P, 0, sizeof P);
    if (l < p->L) {
        if (int rc = relax_impl(op, p->method, p->phi[l], p->rho[l], p->pre[l], p->w[l], st))
            return rc;
        if (int rc = op_sweep(op, EPI_RESID, p->phi[l], p->res[l], p->rho[l], 1, GB_F64, P, 0, 0, 0,
                              nullptr, st))
            return rc;
        GB_LAUNCH_CHECK();
        if (int rc = transform_impl(p->rst[l], p->res[l], p->rho[l + 1], nullptr, 1, GB_F64, P, 0,
                                    0, 0.0, st))
            return rc;
        if (l + 1 != p->tail_lf)
            GB_CUDA_TRY(cudaMemsetAsync(p->phi[l + 1], 0,
                                        (size_t)p->ops[l + 1]->ng() * sizeof(double), st));
        if (int rc = vcycle(p, l + 1, st)) return rc;
        // phi_l -= interpolate(phi_{l+1})
        if (int rc = transform_impl(p->itp[l], p->phi[l + 1], p->phi[l], nullptr, 1, GB_F64, P, 0,
                                    1, 0.0, st))
            return rc;
    }
    if (int rc = relax_impl(op, p->method, p->phi[l], p->rho[l], p->post[l], p->w[l], st))
        return rc;
    if (l == 0) {
        const int nblk = op_resid_blocks(op, 1, 8);
        if (int rc = op_sweep(op, EPI_RESID, p->phi[0], p->res[0], p->rho[0], 1, GB_F64, P, 0, 0, 0,
                              p->partial, st))
            return rc;
        GB_LAUNCH_CHECK();
        launch_reduce_partials(p->partial, nblk, 1, p->dv, p->err_dev, st);
        GB_LAUNCH_CHECK();
    }
    return 0;
}

extern "C" int gb_poisson_iterate(gb_poisson* p, double* phi, const double* rho, double* error,
                                  void* stream) {
    if (!p || !phi || !rho) return fail(GB_EINVAL, "Poisson iterate: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    p->phi[0] = phi;
    p->rho[0] = (double*)rho;  // never written
    if (int rc = vcycle(p, 0, st)) return rc;
    GB_CUDA_TRY(cudaMemcpyAsync(p->err_host, p->err_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
    GB_CUDA_TRY(cudaStreamSynchronize(st));
    if (error) *error = *p->err_host;
    return 0;
}

__global__ void k_sub_scalar(double* a, long long n, const double* v, double count) {
    // phi_ave = sum(phi) / prod(N_c); phi -= phi_ave  (gpaw/poisson.py:492-496)
    const double m = v[0] / count;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = a[i] - m;
}

__global__ void k_block_sums(const double* a, long long n, double* partial) {
    double v = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v += a[i];
    v = block_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

static int mean_removal(gb_poisson* p, double* phi, cudaStream_t st) {
    const GridBC& g = p->ops[0]->g;
    if (!(g.periodic[0] && g.periodic[1] && g.periodic[2])) return 0;
    const long long n = p->ops[0]->ng();
    const int nb = (int)std::min<long long>(1024, (n + 255) / 256);
    k_block_sums<<<nb, 256, 0, st>>>(phi, n, p->partial);
    launch_reduce_partials(p->partial, nb, 1, 1.0, p->mean_dev, st);
    k_sub_scalar<<<nb, 256, 0, st>>>(phi, n, p->mean_dev, (double)n);
    GB_LAUNCH_CHECK();
    return 0;
}

// Capture the whole solve_neutral loop once per executor into a graph with
// a conditional WHILE node: the V-cycle and a check kernel that sets the
// loop condition, then the periodic mean removal.  It works on the
// executor's own phi0/rho0, so one graph serves every call.
static int build_solve_graph(gb_poisson* p) {
    cudaStream_t cs = p->cap;
    // one uncaptured V-cycle first: sets kernel attributes, touches scratch
    GB_CUDA_TRY(cudaMemsetAsync(p->phi0, 0, (size_t)p->ops[0]->ng() * 8, cs));
    GB_CUDA_TRY(cudaMemsetAsync(p->rho0, 0, (size_t)p->ops[0]->ng() * 8, cs));
    p->phi[0] = p->phi0;
    p->rho[0] = p->rho0;
    if (int rc = vcycle(p, 0, cs)) return rc;
    if (int rc = mean_removal(p, p->phi0, cs)) return rc;
    GB_CUDA_TRY(cudaStreamSynchronize(cs));

    cudaGraph_t graph;
    GB_CUDA_TRY(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h;
    GB_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    GB_CUDA_TRY(cudaGraphAddNode(&wnode, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    int rc = vcycle(p, 0, cs);
    if (!rc) k_solve_check<<<1, 1, 0, cs>>>(p->ctl, p->err_dev, h);
    cudaGraph_t body_out = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cs, &body_out);
    if (rc) {
        cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(GB_ECUDA, "Poisson: capture of the V-cycle: %s", cudaGetErrorString(ce));
    }
    // mean removal after the loop (periodic grids)
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, graph, &wnode, nullptr, 1,
                                              cudaStreamCaptureModeThreadLocal));
    rc = mean_removal(p, p->phi0, cs);
    cudaGraph_t g2 = nullptr;
    ce = cudaStreamEndCapture(cs, &g2);
    if (rc || ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return rc ? rc : fail(GB_ECUDA, "Poisson: capture: %s", cudaGetErrorString(ce));
    }
    cudaError_t ie = cudaGraphInstantiate(&p->solve_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(GB_ECUDA, "Poisson: instantiate: %s", cudaGetErrorString(ie));
    return 0;
}

extern "C" int gb_poisson_solve_neutral_async(gb_poisson* p, double* phi, const double* rho,
                                              double eps, int maxiter, void* stream) {
    if (!p || !phi || !rho) return fail(GB_EINVAL, "Poisson solve: NULL argument");
    if (maxiter < 1) return fail(GB_EINVAL, "Poisson solve: maxiter must be >= 1");
    cudaStream_t st = (cudaStream_t)stream;
    if (!p->solve_exec)
        if (int rc = build_solve_graph(p)) return rc;
    const size_t bytes = (size_t)p->ops[0]->ng() * sizeof(double);
    // rhos[0][:] = rho; phis[0] = phi  (gpaw/poisson.py:476-482)
    GB_CUDA_TRY(cudaMemcpyAsync(p->rho0, rho, bytes, cudaMemcpyDeviceToDevice, st));
    GB_CUDA_TRY(cudaMemcpyAsync(p->phi0, phi, bytes, cudaMemcpyDeviceToDevice, st));
    k_solve_init<<<1, 1, 0, st>>>(p->ctl, eps, maxiter);
    GB_LAUNCH_CHECK();
    GB_CUDA_TRY(cudaGraphLaunch(p->solve_exec, st));
    GB_CUDA_TRY(cudaMemcpyAsync(phi, p->phi0, bytes, cudaMemcpyDeviceToDevice, st));
    GB_CUDA_TRY(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, st));
    p->last_maxiter = maxiter;
    return 0;
}

extern "C" int gb_poisson_result(gb_poisson* p, int* niter, double* error) {
    if (!p) return fail(GB_EINVAL, "Poisson result: NULL executor");
    const int it = p->ctl_host->niter;
    if (niter) *niter = it;
    if (error) *error = p->ctl_host->err;
    if (it >= p->last_maxiter)
        return fail(GB_ENOCONV, "Poisson solver did not converge in %d iterations!",
                    p->last_maxiter);
    return 0;
}

extern "C" int gb_poisson_solve_neutral(gb_poisson* p, double* phi, const double* rho, double eps,
                                        int maxiter, int* niter, double* error, void* stream) {
    if (int rc = gb_poisson_solve_neutral_async(p, phi, rho, eps, maxiter, stream)) return rc;
    GB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return gb_poisson_result(p, niter, error);
}

// ------------------------------------------------- relax without allocation
// Some callers cannot let this library call cudaMalloc: a host program that
// has handed all of HBM to its own memory pool (a cudaMalloc would fail or
// force the pool to release cached blocks), a latency-critical serving loop
// that must not risk the implicit device synchronisation cudaMalloc and
// cudaFree may perform, or a plugin host that forbids allocations outside
// its own allocator.  gb_operator_relax_noalloc serves them: the scratch
// grid that relaxation needs (the Jacobi ping-pong buffer, the Gauss-Seidel
// start-of-sweep snapshot) lives in the fixed device array below instead of
// the operator's lazily allocated buffer.
//
// The array is GB_NOALLOC_MAX_POINTS doubles (16 MiB); every GPU that loads
// the library holds it until the process exits.  All calls share it, so
// calls that overlap on the GPU (other streams, other threads) race; calls
// on one stream are ordered.  It keeps the last call's contents; nothing
// needs to start at zero, because each sweep writes every point of the
// scratch before reading it.
static __device__ __align__(256) double g_relax_scratch[GB_NOALLOC_MAX_POINTS];

namespace {
std::mutex g_noalloc_mu;
// Per device: the address of g_relax_scratch and the CUDA context it was
// looked up in.  After cudaDeviceReset (or any other re-creation of the
// primary context) the module is loaded again and the array may move, so a
// cached address is used only while the current context is the one it came
// from.
struct NoallocSlot {
    void* ptr = nullptr;
    void* ctx = nullptr;
};
NoallocSlot g_noalloc[256];

// cuCtxGetCurrent through the runtime's driver entry point table, so that
// the library needs no link against libcuda.
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (CtxGetCurrentFn) nullptr;
        return (CtxGetCurrentFn)f;
    }();
    return fn;
}
}  // namespace

// Host code must not use g_relax_scratch's name as a device address (it is a
// host-side stand-in); the array's address is looked up with the device
// current, on the first call on that device and again whenever the current
// context has changed since.  The look-up may load the module, which a
// stream capture does not allow: if `st` is capturing and no address is
// cached for this context, the call fails with GB_EINVAL and says so.
static int noalloc_scratch(double** out, cudaStream_t st) {
    int dev = 0;
    GB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(GB_EINVAL, "relax_noalloc: device index %d", dev);
    void* ctx = nullptr;
    if (CtxGetCurrentFn f = ctx_get_current()) {
        if (f(&ctx) != 0) ctx = nullptr;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocSlot& slot = g_noalloc[dev];
    if (!slot.ptr || slot.ctx != ctx) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        GB_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return fail(GB_EINVAL,
                        "relax_noalloc: the first call on a device (or after its context was "
                        "re-created) looks up the scratch array's address and must not run "
                        "inside a stream capture; call it once before capturing");
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_relax_scratch);
        if (e != cudaSuccess || !p)
            return fail(GB_ECUDA, "relax_noalloc: cudaGetSymbolAddress: %s",
                        cudaGetErrorString(e));
        slot.ptr = p;
        slot.ctx = ctx;
    }
    *out = (double*)slot.ptr;
    return 0;
}

extern "C" int gb_operator_relax_noalloc(gb_operator* op, int method, double* f,
                                         const double* s, int nrelax, double w, void* stream) {
    if (!op || !f || !s) return fail(GB_EINVAL, "relax_noalloc: NULL argument");
    if (!op->real) return fail(GB_EINVAL, "relax_noalloc: float64 operators only");
    if (method != 1 && method != 2) return fail(GB_EINVAL, "relax_noalloc: method must be 1 or 2");
    if (op->ng() > (long long)GB_NOALLOC_MAX_POINTS)
        return fail(GB_EINVAL,
                    "relax_noalloc: grid has %lld points, more than the %d this entry point "
                    "supports; use gb_operator_relax",
                    op->ng(), (int)GB_NOALLOC_MAX_POINTS);
    if (nrelax <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    double* X = nullptr;
    if (int rc = noalloc_scratch(&X, st)) return rc;
    return relax_with_scratch(op, method, f, s, nrelax, w, X, st);
}
