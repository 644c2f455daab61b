// Host-side definitions shared by the C-ABI files: error state, scratch
// buffers, the Operator and Transformer objects and the dispatch of one
// stencil sweep or one transfer.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/gpaw_b200.h"
#include "gb_internal.cuh"

namespace gb {

// float32 data inside the library (mixed-precision solver); not an ABI dtype
constexpr int GB_F32_INTERNAL = 100;

// Record the message of a failed call for gb_last_error(); returns code.
int fail(int code, const char* fmt, ...);

// While a kernel trace is open (gb_trace_begin), record an event on `st`
// labelled with the kernel launched next; a no-op otherwise, and on a
// stream that is being captured.
void trace_mark(const char* label, cudaStream_t st);

#define GB_CUDA_TRY(expr)                                                             \
    do {                                                                              \
        cudaError_t e_ = (expr);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return ::gb::fail(GB_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                              __FILE__, __LINE__);                                    \
    } while (0)

#define GB_LAUNCH_CHECK()                                                             \
    do {                                                                              \
        cudaError_t e_ = cudaGetLastError();                                          \
        if (e_ != cudaSuccess)                                                        \
            return ::gb::fail(GB_ECUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(e_), \
                              __FILE__, __LINE__);                                    \
    } while (0)

// ------------------------------------------------------------------ scratch
// Device buffer owned by an object; grows on demand (never inside a
// caller's stream capture if gb_*_reserve was called first).
struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~Scratch() {
        if (ptr) dfree(ptr);
    }
    int ensure(size_t want) {
        if (want <= bytes) return 0;
        if (ptr) dfree(ptr);
        ptr = nullptr;
        bytes = 0;
        if (int rc = dmalloc(&ptr, want)) return rc;
        bytes = want;
        return 0;
    }
};

inline size_t elem_size(int dtype) { return dtype == GB_C128 ? 16 : 8; }

inline int read_phases(int dtype, const double* phases, Phases& P) {
    memset(&P, 0, sizeof P);
    if (dtype != GB_C128 || phases == nullptr) return 0;
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 2; d++) {
            P.ph[c][d].x = phases[(c * 2 + d) * 2];
            P.ph[c][d].y = phases[(c * 2 + d) * 2 + 1];
        }
    P.use = 1;
    return 0;
}

// Split an offset flattened with the padded strides (M_c = size_c + 2 range,
// gpaw/fd_operators.py:60-63) into (o0, o1, o2) with |o_c| <= range; false
// when it does not fit the range.
inline bool split_offset(long long f, const int64_t size[3], int range, int o[3]) {
    const long long M1 = size[1] + 2 * range, M2 = size[2] + 2 * range;
    long long o2 = ((f % M2) + M2) % M2;
    if (o2 > M2 / 2) o2 -= M2;
    const long long rest = (f - o2) / M2;
    long long o1 = ((rest % M1) + M1) % M1;
    if (o1 > M1 / 2) o1 -= M1;
    const long long o0 = (rest - o1) / M1;
    if (llabs(o0) > range || llabs(o1) > range || llabs(o2) > range ||
        (o0 * M1 + o1) * M2 + o2 != f)
        return false;
    o[0] = (int)o0;
    o[1] = (int)o1;
    o[2] = (int)o2;
    return true;
}

inline bool ranges_overlap(const void* a, const void* b, size_t bytes) {
    const char* x = (const char*)a;
    const char* y = (const char*)b;
    return x < y + bytes && y < x + bytes;
}

}  // namespace gb

// The opaque objects of the C ABI (global names, declared in gpaw_b200.h).
struct gb_operator {
    gb::Stencil st;
    gb::GridBC g;
    int real;
    double diag;
    gb::CfdStencil cs;     // axis-aligned form, when the stencil has one
    int nn = 0;        // its half-width
    int tiled = 0;     // use the plane-marching kernels
    int chunk = 0;     // axis-0 planes per CTA of those kernels (0: automatic)
    gb::Scratch scratch;   // aliasing stage / Jacobi ping-pong / GS snapshot
    gb::Scratch partial;   // per-CTA partial sums of |r|^2
    long long ng() const { return (long long)g.n[0] * g.n[1] * g.n[2]; }
};

struct gb_transformer {
    gb::XferGeom G;
    int k;
    int interpolate;
    int real;
    long long ngin, ngout;
};

namespace gb {

// ----------------------------------------------------------------- Operator

// Partial sums produced per grid by a residual sweep of `op`.
inline int op_resid_blocks(const gb_operator* op, int nin, int es) {
    return op->tiled ? cfd_blocks(op->g, op->nn, es, nin, op->chunk) : residual_blocks(op->g);
}

// One pass of the stencil with a fused epilogue; plane-marching kernel for
// axis-aligned stencils, the generic one otherwise.
inline int op_sweep(gb_operator* op, int mode, const void* in, void* out, const void* aux,
                    int nin, int dtype, const Phases& P, double w, double sc, int negate,
                    double* partial, cudaStream_t st) {
    if (op->tiled) {
        Epi ep{aux, w, sc, negate, partial};
        ep.chunk = op->chunk;
        int rc = (dtype == GB_F64)
                     ? launch_fd_cfd<double>(mode, in, out, nin, op->g, P, op->cs, op->nn, ep, st,
                                             nullptr)
                     : launch_fd_cfd<double2>(mode, in, out, nin, op->g, P, op->cs, op->nn, ep,
                                              st, nullptr);
        if (rc == -2) return fail(GB_ECUDA, "could not raise the shared-memory limit");
        if (rc == 0) return 0;
    }
    switch (mode) {
        case EPI_APPLY:
            if (dtype == GB_F64) launch_fd<double>(in, out, nin, op->g, P, op->st, st);
            else launch_fd<double2>(in, out, nin, op->g, P, op->st, st);
            break;
        case EPI_POT:
            // generic stencils: the apply, then o += p * v in a second pass
            if (dtype == GB_F64) {
                launch_fd<double>(in, out, nin, op->g, P, op->st, st);
                launch_add_pot<double>(in, out, (const double*)aux, nin, op->ng(), st);
            } else {
                launch_fd<double2>(in, out, nin, op->g, P, op->st, st);
                launch_add_pot<double2>(in, out, (const double*)aux, nin, op->ng(), st);
            }
            break;
        case EPI_RESID:
            if (dtype == GB_F64)
                launch_residual<double>(in, aux, out, nin, op->g, P, op->st, partial, st);
            else
                launch_residual<double2>(in, aux, out, nin, op->g, P, op->st, partial, st);
            break;
        case EPI_JACOBI:
            launch_jacobi((const double*)in, (double*)out, (const double*)aux, op->g, op->st, w,
                          st);
            break;
        case EPI_PRECOND:
            if (dtype == GB_F64)
                launch_precond_step<double>(in, aux, out, nin, op->g, P, op->st, sc, negate, st);
            else
                launch_precond_step<double2>(in, aux, out, nin, op->g, P, op->st, sc, negate, st);
            break;
    }
    return 0;
}


inline int transform_impl(gb_transformer* t, const void* in, void* out, void* out2, int64_t nin,
                          int dtype, const Phases& P, int neg_in, int accumulate, double scale2,
                          cudaStream_t st) {
    XferGeom G = t->G;
    G.neg_in = neg_in;
    G.accumulate = accumulate;
    G.scale2 = scale2;
    int rc;
    if (dtype == GB_F64)
        rc = launch_transform<double>(t->k, t->interpolate, in, out, out2, (int)nin, G, P, st);
    else if (dtype == GB_F32_INTERNAL)
        rc = launch_transform<float>(t->k, t->interpolate, in, out, out2, (int)nin, G, P, st);
    else
        rc = launch_transform<double2>(t->k, t->interpolate, in, out, out2, (int)nin, G, P, st);
    if (rc == -2) return fail(GB_ECUDA, "transformer: could not raise the shared-memory limit");
    if (rc) return fail(GB_EINVAL, "transformer: unsupported order");
    GB_LAUNCH_CHECK();
    return 0;
}


}  // namespace gb
