// Shared device-side definitions for the gpaw_b200 finite-difference kernels.
//
// Arithmetic convention: every kernel on the FP64 path evaluates each output
// with the same operations, operands and grouping as the reference's C loops
// (c/bmgs/fd.cpp, relax.cpp, restrict.cpp, interpolate.cpp,
// translate.cpp), using the _rn intrinsics so that nvcc cannot contract a
// multiply and an add into an FMA.  With that, results are bit-identical to
// the reference compiled for x86-64 without FMA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define GB_MAX_COEFS 96   // GUCLaplace with 6 directions and nn = 6: 73

namespace gb {

// ------------------------------------------------------------------ scalars
struct cplx {
    double re, im;
};

template <class T> struct Num;

template <> struct Num<double> {
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double scale(double a, double c) { return __dmul_rn(a, c); }
    static __device__ __forceinline__ double neg(double a) { return -a; }
};

template <> struct Num<double2> {
    static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ double2 add(double2 a, double2 b) {
        return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
    }
    static __device__ __forceinline__ double2 sub(double2 a, double2 b) {
        return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
    }
    static __device__ __forceinline__ double2 scale(double2 a, double c) {
        return make_double2(__dmul_rn(a.x, c), __dmul_rn(a.y, c));
    }
    static __device__ __forceinline__ double2 neg(double2 a) { return make_double2(-a.x, -a.y); }
};

template <> struct Num<float> {
    static __device__ __forceinline__ float zero() { return 0.0f; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float scale(float a, float c) { return a * c; }
    static __device__ __forceinline__ float neg(float a) { return -a; }
};

// phase * z, grouped as (a c - b d) + i (a d + b c) with every product
// rounded on its own (the reference's std::complex multiply in
// bmgs_translatemz, c/bmgs/translate.cpp:28-47).
__device__ __forceinline__ double2 cmul(double2 ph, double2 z) {
    return make_double2(__dsub_rn(__dmul_rn(ph.x, z.x), __dmul_rn(ph.y, z.y)),
                        __dadd_rn(__dmul_rn(ph.x, z.y), __dmul_rn(ph.y, z.x)));
}

// ----------------------------------------------------------- geometry/bc
// Boundary description of one grid: interior size n[c] and, per axis, whether
// a read past the edge wraps (periodic, own rank as neighbour) or reads zero
// (neighbour -1).  Bloch phases: ph[c][0] multiplies values read past the
// HIGH edge, ph[c][1] values read past the LOW edge (c/bc.cpp:242-257 with
// sendproc == COPY_DATA; gpaw/core/uniform_grid.py:116-127).
struct GridBC {
    int n[3];
    int periodic[3];
};

struct Phases {
    double2 ph[3][2];
    int use;  // 0 for real data or all phases == 1 (no multiply)
};

// Value the reference's padded buffer holds at interior coordinate (x0,x1,x2),
// each coordinate possibly outside [0, n) by less than n.  `corners`
// selects the cfd = 0 rule (edges and corners filled, c/bc.cpp:108-112);
// with corners == 0 a read outside on two or more axes returns zero.
template <class T>
__device__ __forceinline__ T bc_read(const T* __restrict__ a, int x0, int x1, int x2,
                                     const GridBC& g, const Phases& P, bool corners);

template <>
__device__ __forceinline__ double bc_read<double>(const double* __restrict__ a, int x0, int x1,
                                                  int x2, const GridBC& g, const Phases& P,
                                                  bool corners) {
    int x[3] = {x0, x1, x2};
    int outside = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (x[c] < 0 || x[c] >= g.n[c]) {
            if (!g.periodic[c]) return 0.0;
            x[c] += (x[c] < 0) ? g.n[c] : -g.n[c];
            outside++;
        }
    }
    if (outside > 1 && !corners) return 0.0;
    return __ldg(a + ((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2]);
}

template <>
__device__ __forceinline__ double2 bc_read<double2>(const double2* __restrict__ a, int x0, int x1,
                                                    int x2, const GridBC& g, const Phases& P,
                                                    bool corners) {
    int x[3] = {x0, x1, x2};
    int side[3] = {-1, -1, -1};
    int outside = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (x[c] < 0 || x[c] >= g.n[c]) {
            if (!g.periodic[c]) return make_double2(0.0, 0.0);
            side[c] = (x[c] < 0) ? 1 : 0;
            x[c] += (x[c] < 0) ? g.n[c] : -g.n[c];
            outside++;
        }
    }
    if (outside > 1 && !corners) return make_double2(0.0, 0.0);
    double2 v = __ldg(a + ((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2]);
    if (P.use) {
        // the halo is filled axis by axis, so phases compose in axis order
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (side[c] >= 0) v = cmul(P.ph[c][side[c]], v);
    }
    return v;
}

template <>
__device__ __forceinline__ float bc_read<float>(const float* __restrict__ a, int x0, int x1,
                                                int x2, const GridBC& g, const Phases& P,
                                                bool corners) {
    int x[3] = {x0, x1, x2};
    int outside = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (x[c] < 0 || x[c] >= g.n[c]) {
            if (!g.periodic[c]) return 0.0f;
            x[c] += (x[c] < 0) ? g.n[c] : -g.n[c];
            outside++;
        }
    }
    if (outside > 1 && !corners) return 0.0f;
    return __ldg(a + ((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2]);
}

// ---------------------------------------------------------------- stencil
// Stencil in kernel-parameter form.  Offsets are kept both as (o0,o1,o2)
// and as flat offsets in the UNPADDED grid, coefficient order as given by
// the caller (the order bmgs_fd sums in, c/bmgs/fd.cpp:26-27).
struct Stencil {
    int ncoefs;
    int range;
    int cfd;
    double coef[GB_MAX_COEFS];
    int off[GB_MAX_COEFS][3];
    long long flat[GB_MAX_COEFS];
};

}  // namespace gb
