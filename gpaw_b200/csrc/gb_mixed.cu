// Mixed-precision multigrid Poisson solver: FP32 V-cycles inside FP64
// defect correction.  No counterpart in the reference (its FDPoissonSolver is
// FP64 throughout, gpaw/poisson.py:321-537); the operators, transformers and
// level hierarchy are the reference's.
//
//   d = rho - L64 phi                (FP64 stencil, |d|^2 in FP64)
//   while |d| / |rho| > tol:
//       e = V32(float(d))            (FP32 V-cycle, Chebyshev smoothing)
//       phi += e                     (FP64 accumulate, fused in the last sweep)
//       d = rho - L64 phi
//
// V32 on levels 0..L-1: pre-smooth (degree-2 Chebyshev from zero, one
// stencil pass), residual, restriction, coarse correction, interpolation and
// correction, post-smooth (degree-2 Chebyshev, two stencil passes).  Level L
// (coarsest) is solved in FP64 with a fixed-degree Chebyshev iteration over
// the spectrum of D^-1 A, in one single-CTA kernel.  The whole loop runs on
// the device: a CUDA graph with a conditional WHILE node.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "gb_objects.cuh"
#include "gb_tma.cuh"

using namespace gb;

namespace {

// Degree-2 Chebyshev smoother on D^-1 A over [a, b] (Saad, Iterative
// Methods for Sparse Linear Systems, Alg. 12.1), folded into stencil passes:
//   from e = 0:  e2 = pre_u * b + pre_Lu * (A b)
//   from e:      t  = (b - A e) / (theta c0)
//                e2 = e + k1 * t - k2 * (A t)
struct ChebLevel {
    double pre_u, pre_Lu;     // pre-smooth coefficients
    double inv_tc0;           // 1 / (theta c0)
    double k1, k2;            // post-smooth coefficients
};

// Chebyshev smoothing on [lam_max / 8, 1.05 lam_max]: on the 192^3 grid
// with four levels, lower bounds lam_max / 5 .. / 16 and upper factors
// 1.0 .. 1.2 all took 14 to 23 V-cycles against 14 for this choice.
ChebLevel cheb_level(double lam_max, double c0) {
    const double a = lam_max / 8.0, b = 1.05 * lam_max;
    const double theta = 0.5 * (b + a), delta = 0.5 * (b - a);
    const double sigma = theta / delta;
    const double rho0 = 1.0 / sigma;
    const double rho1 = 1.0 / (2.0 * sigma - rho0);
    ChebLevel c;
    c.k1 = 1.0 + rho1 * rho0 + 2.0 * rho1 * theta / delta;
    c.k2 = 2.0 * rho1 / (delta * c0);
    c.inv_tc0 = 1.0 / (theta * c0);
    c.pre_u = c.k1 * c.inv_tc0;
    c.pre_Lu = -c.k2 * c.inv_tc0;
    return c;
}

// Value of d at interior coordinate (x0, x1, x2) with the grid's boundary
// (zero or periodic); plain loads, since d changes during the kernel.
__device__ __forceinline__ double coarse_read(const double* d, int x0, int x1, int x2,
                                              const GridBC& g) {
    int x[3] = {x0, x1, x2};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (x[c] < 0 || x[c] >= g.n[c]) {
            if (!g.periodic[c]) return 0.0;
            x[c] += x[c] < 0 ? g.n[c] : -g.n[c];
        }
    }
    return d[((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2]];
}

struct Ctl {
    double rho2;      // |rho|^2
    double rel;       // last |d| / |rho|
    double tol;
    int maxiter;
    int niter;
};

// Coarsest level: x = Chebyshev_deg(D^-1 A, [lo, hi]) applied to b, from
// x = 0, in FP64, by one CTA.  b is the FP32 restricted residual; the FP32
// correction is written to e.  r, da, db, x are FP64 scratch of n points.
__global__ void __launch_bounds__(1024)
k_coarse_cheb(const float* __restrict__ b, float* __restrict__ e, double* __restrict__ x,
              double* __restrict__ r, double* __restrict__ da, double* __restrict__ db,
              GridBC g, const __grid_constant__ Stencil s, double lo, double hi, int deg) {
    const int n = g.n[0] * g.n[1] * g.n[2];
    const double c0 = s.coef[0];
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const double r0 = (double)b[p] / c0;
        r[p] = r0;
        x[p] = 0.0;
        da[p] = r0 / theta;
    }
    __syncthreads();
    double* d = da;
    double* dn = db;
    for (int k = 0; k < deg; k++) {
        const double rho_n = 1.0 / (2.0 * sigma - rho);
        for (int p = threadIdx.x; p < n; p += blockDim.x) {
            const int i2 = p % g.n[2];
            const int t = p / g.n[2];
            const int i1 = t % g.n[1];
            const int i0 = t / g.n[1];
            double ad = 0.0;
            for (int c = 0; c < s.ncoefs; c++)
                ad += s.coef[c] * coarse_read(d, i0 + s.off[c][0], i1 + s.off[c][1],
                                              i2 + s.off[c][2], g);
            const double dk = d[p];
            x[p] += dk;
            const double rn = r[p] - ad / c0;
            r[p] = rn;
            dn[p] = rho_n * rho * dk + 2.0 * rho_n / delta * rn;
        }
        rho = rho_n;
        __syncthreads();
        double* tmp = d;
        d = dn;
        dn = tmp;
    }
    for (int p = threadIdx.x; p < n; p += blockDim.x) e[p] = (float)x[p];
}

// Same iteration with the search direction in shared memory (double
// buffered) and each thread's points (x, r) in registers: for coarsest grids
// of at most KP * 1024 points.
constexpr int KP = 14;
constexpr int SMEM_COARSE_MAX = KP * 1024;

// Axis-aligned 7-point stencil by axis (coefficients of +1 / -1 along each).
struct Seven {
    double c0, cp[3], cm[3];
};

__global__ void __launch_bounds__(1024, 1)
k_coarse_cheb_smem(const float* __restrict__ b, float* __restrict__ e, GridBC g,
                   const __grid_constant__ Stencil s, Seven s7, int seven, double lo,
                   double hi, int deg) {
    extern __shared__ __align__(16) double sm[];
    const int n = g.n[0] * g.n[1] * g.n[2];
    double* dA = sm;
    double* dB = sm + n;
    const double inv_c0 = 1.0 / s.coef[0];
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    double x[KP], r[KP];
    int ijk[KP];
#pragma unroll
    for (int k = 0; k < KP; k++) {
        const int p = threadIdx.x + k * 1024;
        x[k] = 0.0;
        r[k] = 0.0;
        ijk[k] = 0;
        if (p < n) {
            const int i2 = p % g.n[2];
            const int t = p / g.n[2];
            ijk[k] = ((t / g.n[1]) << 20) | ((t % g.n[1]) << 10) | i2;
            r[k] = (double)b[p] * inv_c0;
            dA[p] = r[k] / theta;
        }
    }
    __syncthreads();
    double* d = dA;
    double* dn = dB;
    for (int it = 0; it < deg; it++) {
        const double rho_n = 1.0 / (2.0 * sigma - rho);
        const double c1 = rho_n * rho, c2 = 2.0 * rho_n / delta;
#pragma unroll
        for (int k = 0; k < KP; k++) {
            const int p = threadIdx.x + k * 1024;
            if (p >= n) break;
            const int i0 = ijk[k] >> 20, i1 = (ijk[k] >> 10) & 1023, i2 = ijk[k] & 1023;
            const double dk = d[p];
            double ad;
            if (seven) {
                // 7-point stencil: neighbour = p +- stride, wrapped or zero
                // at the grid's edge
                const int st1 = g.n[2], st0 = g.n[1] * g.n[2];
                auto nb = [&](int i, int nax, int stride, int per, int dir) -> double {
                    const int j = i + dir;
                    if (j >= 0 && j < nax) return d[p + dir * stride];
                    if (!per) return 0.0;
                    return d[p + dir * stride - dir * nax * stride];
                };
                ad = s7.c0 * dk;
                ad += s7.cp[0] * nb(i0, g.n[0], st0, g.periodic[0], +1) +
                      s7.cm[0] * nb(i0, g.n[0], st0, g.periodic[0], -1);
                ad += s7.cp[1] * nb(i1, g.n[1], st1, g.periodic[1], +1) +
                      s7.cm[1] * nb(i1, g.n[1], st1, g.periodic[1], -1);
                ad += s7.cp[2] * nb(i2, g.n[2], 1, g.periodic[2], +1) +
                      s7.cm[2] * nb(i2, g.n[2], 1, g.periodic[2], -1);
            } else {
                ad = 0.0;
                for (int c = 0; c < s.ncoefs; c++)
                    ad += s.coef[c] * coarse_read(d, i0 + s.off[c][0], i1 + s.off[c][1],
                                                  i2 + s.off[c][2], g);
            }
            x[k] += dk;
            r[k] -= ad * inv_c0;
            dn[p] = c1 * dk + c2 * r[k];
        }
        rho = rho_n;
        __syncthreads();
        double* tmp = d;
        d = dn;
        dn = tmp;
    }
#pragma unroll
    for (int k = 0; k < KP; k++) {
        const int p = threadIdx.x + k * 1024;
        if (p < n) e[p] = (float)x[k];
    }
}

// Same iteration spread over a cluster of CL CTAs: CTA r owns the flat
// points [r * chunk, (r + 1) * chunk); its slab of the search direction
// (double buffered) lives in its shared memory, and neighbours owned by other
// CTAs are read through distributed shared memory.  One hardware cluster
// barrier per step.  For coarsest grids of at most CL * 1024 * KPC points.
constexpr int CL = 8;
constexpr int KPC = 4;
constexpr int CLUSTER_COARSE_MAX = CL * 1024 * KPC;

__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(1024, 1)
k_coarse_cheb_cluster(const float* __restrict__ b, float* __restrict__ e, GridBC g, Seven s7,
                      double lo, double hi, int deg) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) double smc[];
    const int n = g.n[0] * g.n[1] * g.n[2];
    const int chunk = (n + CL - 1) / CL;
    const int rank = (int)cluster.block_rank();
    double* bufA = smc;
    double* bufB = smc + chunk;
    const double inv_c0 = 1.0 / s7.c0;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    const int st1 = g.n[2], st0 = g.n[1] * g.n[2];
    double x[KPC], r[KPC];
#pragma unroll
    for (int k = 0; k < KPC; k++) {
        const int li = threadIdx.x + k * 1024;
        const int p = rank * chunk + li;
        x[k] = 0.0;
        r[k] = 0.0;
        if (li < chunk && p < n) {
            r[k] = (double)b[p] * inv_c0;
            bufA[li] = r[k] / theta;
        }
    }
    cluster.sync();
    bool useA = true;
    for (int it = 0; it < deg; it++) {
        double* d = useA ? bufA : bufB;
        double* dn = useA ? bufB : bufA;
        auto at = [&](int q) -> double {
            double* base = cluster.map_shared_rank(d, q / chunk);
            return base[q % chunk];
        };
        const double rho_n = 1.0 / (2.0 * sigma - rho);
        const double c1 = rho_n * rho, c2 = 2.0 * rho_n / delta;
#pragma unroll
        for (int k = 0; k < KPC; k++) {
            const int li = threadIdx.x + k * 1024;
            const int p = rank * chunk + li;
            if (li >= chunk || p >= n) break;
            const int i2 = p % g.n[2];
            const int t = p / g.n[2];
            const int i1 = t % g.n[1];
            const int i0 = t / g.n[1];
            auto nb = [&](int i, int nax, int stride, int per, int dir) -> double {
                const int j = i + dir;
                if (j >= 0 && j < nax) return at(p + dir * stride);
                if (!per) return 0.0;
                return at(p + dir * stride - dir * nax * stride);
            };
            const double dk = d[li];
            double ad = s7.c0 * dk;
            ad += s7.cp[0] * nb(i0, g.n[0], st0, g.periodic[0], +1) +
                  s7.cm[0] * nb(i0, g.n[0], st0, g.periodic[0], -1);
            ad += s7.cp[1] * nb(i1, g.n[1], st1, g.periodic[1], +1) +
                  s7.cm[1] * nb(i1, g.n[1], st1, g.periodic[1], -1);
            ad += s7.cp[2] * nb(i2, g.n[2], 1, g.periodic[2], +1) +
                  s7.cm[2] * nb(i2, g.n[2], 1, g.periodic[2], -1);
            x[k] += dk;
            r[k] -= ad * inv_c0;
            dn[li] = c1 * dk + c2 * r[k];
        }
        rho = rho_n;
        cluster.sync();
        useA = !useA;
    }
#pragma unroll
    for (int k = 0; k < KPC; k++) {
        const int li = threadIdx.x + k * 1024;
        const int p = rank * chunk + li;
        if (li < chunk && p < n) e[p] = (float)x[k];
    }
}

// Exact solve of the coarsest level by fast diagonalisation.  A 7-point
// operator with symmetric couplings, c0 x_p + sum_a c_a (x_{p+e_a} +
// x_{p-e_a}), is c0 I + sum_a c_a T_a with T_a the 1-D neighbour matrix of
// axis a (zero or periodic boundary), so it is diagonal in the tensor
// product of the T_a's orthonormal eigenvectors Q_a (sine vectors for a
// zero boundary, cosine/sine pairs for a periodic one):
//     x = (Q0 x Q1 x Q2) diag(1 / lambda) (Q0 x Q1 x Q2)^T b,
//     lambda_ijk = c0 + c_0 mu0_i + c_1 mu1_j + c_2 mu2_k.
// Six passes of small dense products along one axis each, in FP64, by one
// CTA with the grid (two copies), the Q_a and mu_a in shared memory.  A
// lambda that vanishes (the constant mode of a fully periodic grid) is
// left out, as the neutral problem's mean is free.  `tab` holds Q0, Q1,
// Q2 (row j, column k = component j of eigenvector k), then mu0, mu1, mu2.
__global__ void __launch_bounds__(1024, 1)
k_coarse_direct(const float* __restrict__ b, float* __restrict__ e, const double* __restrict__ tab,
                int n0, int n1, int n2, double c0, double ca0, double ca1, double ca2) {
    extern __shared__ __align__(16) double smd[];
    const int n = n0 * n1 * n2;
    const int ntab = n0 * n0 + n1 * n1 + n2 * n2 + n0 + n1 + n2;
    double* A = smd;
    double* B = A + n;
    double* T = B + n;
    const double* Q0 = T;
    const double* Q1 = Q0 + n0 * n0;
    const double* Q2 = Q1 + n1 * n1;
    const double* mu0 = Q2 + n2 * n2;
    const double* mu1 = mu0 + n0;
    const double* mu2 = mu1 + n1;
    for (int p = threadIdx.x; p < ntab; p += blockDim.x) T[p] = tab[p];
    for (int p = threadIdx.x; p < n; p += blockDim.x) A[p] = (double)b[p];
    __syncthreads();
    // y = M^T x (fwd) or y = M x along one axis: `len` points apart by
    // `stride`; the point's coordinate along the axis is (p / stride) % len
    auto pass = [&](const double* src, double* dst, const double* M, int len, int stride,
                    bool fwd) {
        for (int p = threadIdx.x; p < n; p += blockDim.x) {
            const int k = (p / stride) % len;
            const double* col = src + (p - k * stride);
            double acc = 0.0;
            for (int j = 0; j < len; j++)
                acc += (fwd ? M[j * len + k] : M[k * len + j]) * col[j * stride];
            dst[p] = acc;
        }
        __syncthreads();
    };
    pass(A, B, Q2, n2, 1, true);
    pass(B, A, Q1, n1, n2, true);
    pass(A, B, Q0, n0, n1 * n2, true);
    double lmax = fabs(c0) + 2.0 * (fabs(ca0) + fabs(ca1) + fabs(ca2));
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const int k2 = p % n2, k1 = (p / n2) % n1, k0 = p / (n1 * n2);
        const double lam = c0 + ca0 * mu0[k0] + ca1 * mu1[k1] + ca2 * mu2[k2];
        B[p] = fabs(lam) > 1e-12 * lmax ? B[p] / lam : 0.0;
    }
    __syncthreads();
    pass(B, A, Q0, n0, n1 * n2, false);
    pass(A, B, Q1, n1, n2, false);
    pass(B, A, Q2, n2, 1, false);
    for (int p = threadIdx.x; p < n; p += blockDim.x) e[p] = (float)A[p];
}

// Orthonormal eigenvectors (columns of Q, n x n, row-major) and eigenvalues
// of the 1-D neighbour matrix of an axis of n points: (T x)_j = x_{j+1} +
// x_{j-1}, zero past the ends or wrapped.
static void neighbour_eigen(int n, bool periodic, double* Q, double* mu) {
    const double pi = 3.14159265358979323846;
    if (!periodic) {
        const double s = std::sqrt(2.0 / (n + 1));
        for (int k = 0; k < n; k++) {
            mu[k] = 2.0 * std::cos(pi * (k + 1) / (n + 1));
            for (int j = 0; j < n; j++) Q[j * n + k] = s * std::sin(pi * (j + 1) * (k + 1) / (n + 1));
        }
        return;
    }
    // periodic: constant, cosine/sine pairs, and the alternating vector
    int col = 0;
    const double c = 1.0 / std::sqrt((double)n), s2 = std::sqrt(2.0 / n);
    for (int j = 0; j < n; j++) Q[j * n + col] = c;
    mu[col++] = 2.0;
    for (int k = 1; 2 * k < n; k++) {
        for (int j = 0; j < n; j++) {
            Q[j * n + col] = s2 * std::cos(2 * pi * k * j / n);
            Q[j * n + col + 1] = s2 * std::sin(2 * pi * k * j / n);
        }
        mu[col] = mu[col + 1] = 2.0 * std::cos(2 * pi * k / n);
        col += 2;
    }
    if (n % 2 == 0 && n > 1) {
        for (int j = 0; j < n; j++) Q[j * n + col] = (j % 2 ? -c : c);
        mu[col++] = -2.0;
    }
}

// ------------------------------------------------ coarse levels in one kernel
// The FP32 V-cycle below level 0 -- smoothing, residual, restriction and
// interpolation of every level from `lc` down, and the exact coarsest
// solve -- as ONE cooperative kernel: every pass is a grid-stride loop over
// the level's points (FP32 7-point operator, K = 2 transfers, each output
// formed from its neighbourhood directly), and the passes are separated by
// a grid-wide barrier instead of a kernel boundary.  On these small, L2-
// resident levels a kernel boundary costs more than the work it separates.
// Same passes and coefficients as the per-level kernels of vcycle32.
constexpr int CV_MAX = 12;
struct CoopLevel {
    int n[3], per[3], ng;
    float c0, cp[3], cm[3];            // the level's 7-point operator
    float pre_u, pre_Lu, inv_tc0, k1, k2;
    float *b, *e, *t;
    int rplo[3];                       // restriction to the next level
    float rw;
    int iplo[3], iskip[3];             // interpolation from the next level
    float iw;
};
struct CoopPlan {
    int nl;                            // levels lc .. L (the last is the coarsest)
    CoopLevel lv[CV_MAX];
    const double* tab;                 // eigen tables of the coarsest level
    double *X, *Y;                     // coarsest-level FP64 work grids
    double dc0, dca[3];                // coarsest operator (FP64)
    unsigned* bar;                     // grid barrier: arrivals, generation
};

// Grid-wide barrier of a cooperative launch (all CTAs resident), bounded by
// one second: a barrier that runs out records a device fault and the
// kernel gives up (its output is then not valid).
__device__ __forceinline__ bool coop_sync(unsigned* bar, bool ok) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = ok;
        if (ok) {
            volatile unsigned* gen = bar + 1;
            const unsigned g = *gen;
            __threadfence();
            if (atomicAdd(bar, 1u) == gridDim.x - 1) {
                atomicExch(bar, 0u);
                __threadfence();
                atomicAdd(bar + 1, 1u);
            } else {
                const uint64_t t0 = global_ns();
                while (*gen == g) {
                    if (global_ns() - t0 > 1000000000ull) {
                        atomicCAS(&g_device_fault, 0, GB_FAULT_TMA_TIMEOUT);
                        s_ok = 0;
                        break;
                    }
                    __nanosleep(20);
                }
            }
            __threadfence();
        }
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ int cv_at(int j, int n, int per) {
    if (j >= 0 && j < n) return j;
    if (!per) return -1;
    j = j < 0 ? j + n : j - n;
    return (j >= 0 && j < n) ? j : -1;
}

// A x at point p = (i0, i1, i2) of level L (reads bypass L1: other CTAs
// wrote x before the last barrier)
__device__ __forceinline__ float cv_apply(const float* x, const CoopLevel& L, int p, int i0,
                                          int i1, int i2) {
    const int s1 = L.n[2], s0 = L.n[1] * L.n[2];
    auto nb = [&](int i, int n, int per, int s, int d) -> float {
        const int j = cv_at(i + d, n, per);
        return j < 0 ? 0.0f : __ldcg(x + p + (j - i) * s);
    };
    float y = L.c0 * __ldcg(x + p);
    y += L.cp[2] * nb(i2, L.n[2], L.per[2], 1, 1) + L.cm[2] * nb(i2, L.n[2], L.per[2], 1, -1);
    y += L.cp[1] * nb(i1, L.n[1], L.per[1], s1, 1) + L.cm[1] * nb(i1, L.n[1], L.per[1], s1, -1);
    y += L.cp[0] * nb(i0, L.n[0], L.per[0], s0, 1) + L.cm[0] * nb(i0, L.n[0], L.per[0], s0, -1);
    return y;
}

__device__ __forceinline__ void cv_split(int p, const int n[3], int& i0, int& i1, int& i2) {
    i2 = p % n[2];
    const int q = p / n[2];
    i1 = q % n[1];
    i0 = q / n[1];
}

__global__ void __launch_bounds__(512)
k_coop_vcycle(const __grid_constant__ CoopPlan P) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    bool ok = true;
    const int nl = P.nl;
    // descent: pre-smooth, residual, restriction
    for (int l = 0; l + 1 < nl && ok; l++) {
        const CoopLevel& L = P.lv[l];
        const CoopLevel& C = P.lv[l + 1];
        for (int p = tid; p < L.ng; p += nth) {
            int i0, i1, i2;
            cv_split(p, L.n, i0, i1, i2);
            L.e[p] = L.pre_u * __ldcg(L.b + p) + L.pre_Lu * cv_apply(L.b, L, p, i0, i1, i2);
        }
        ok = coop_sync(P.bar, ok);
        for (int p = tid; p < L.ng; p += nth) {
            int i0, i1, i2;
            cv_split(p, L.n, i0, i1, i2);
            L.t[p] = __ldcg(L.b + p) - cv_apply(L.e, L, p, i0, i1, i2);
        }
        ok = coop_sync(P.bar, ok);
        // restriction: 0.5 (a + w (a+ + a-)) along each axis, centre 2I+1-plo
        for (int q = tid; q < C.ng; q += nth) {
            int I0, I1, I2;
            cv_split(q, C.n, I0, I1, I2);
            const int c[3] = {2 * I0 + 1 - L.rplo[0], 2 * I1 + 1 - L.rplo[1],
                              2 * I2 + 1 - L.rplo[2]};
            int idx[3][3];
            float wt[3][3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int d = -1; d <= 1; d++) {
                    idx[a][d + 1] = cv_at(c[a] + d, L.n[a], L.per[a]);
                    wt[a][d + 1] = d == 0 ? 0.5f : 0.5f * L.rw;
                }
            }
            float acc = 0.0f;
#pragma unroll
            for (int d0 = 0; d0 < 3; d0++) {
                if (idx[0][d0] < 0) continue;
#pragma unroll
                for (int d1 = 0; d1 < 3; d1++) {
                    if (idx[1][d1] < 0) continue;
                    const float w01 = wt[0][d0] * wt[1][d1];
                    const float* row = L.t + (idx[0][d0] * L.n[1] + idx[1][d1]) * L.n[2];
#pragma unroll
                    for (int d2 = 0; d2 < 3; d2++)
                        if (idx[2][d2] >= 0) acc += w01 * wt[2][d2] * __ldcg(row + idx[2][d2]);
                }
            }
            C.b[q] = acc;
        }
        ok = coop_sync(P.bar, ok);
    }
    // coarsest level: exact solve by fast diagonalisation (FP64)
    if (ok) {
        const CoopLevel& L = P.lv[nl - 1];
        const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2], n = L.ng;
        const double* Q0 = P.tab;
        const double* Q1 = Q0 + n0 * n0;
        const double* Q2 = Q1 + n1 * n1;
        const double* mu0 = Q2 + n2 * n2;
        const double* mu1 = mu0 + n0;
        const double* mu2 = mu1 + n1;
        for (int p = tid; p < n; p += nth) P.X[p] = (double)__ldcg(L.b + p);
        ok = coop_sync(P.bar, ok);
        auto pass = [&](const double* src, double* dst, const double* M, int len, int stride,
                        bool fwd) {
            for (int p = tid; p < n; p += nth) {
                const int k = (p / stride) % len;
                const double* col = src + (p - k * stride);
                double acc = 0.0;
                for (int j = 0; j < len; j++)
                    acc += (fwd ? __ldg(M + j * len + k) : __ldg(M + k * len + j)) *
                           __ldcg(col + j * stride);
                dst[p] = acc;
            }
            return coop_sync(P.bar, ok);
        };
        if (ok) ok = pass(P.X, P.Y, Q2, n2, 1, true);
        if (ok) ok = pass(P.Y, P.X, Q1, n1, n2, true);
        if (ok) ok = pass(P.X, P.Y, Q0, n0, n1 * n2, true);
        const double lmax = fabs(P.dc0) + 2.0 * (fabs(P.dca[0]) + fabs(P.dca[1]) + fabs(P.dca[2]));
        for (int p = tid; p < n && ok; p += nth) {
            const int k2 = p % n2, k1 = (p / n2) % n1, k0 = p / (n1 * n2);
            const double lam = P.dc0 + P.dca[0] * __ldg(mu0 + k0) + P.dca[1] * __ldg(mu1 + k1) +
                               P.dca[2] * __ldg(mu2 + k2);
            P.Y[p] = fabs(lam) > 1e-12 * lmax ? __ldcg(P.Y + p) / lam : 0.0;
        }
        ok = coop_sync(P.bar, ok);
        if (ok) ok = pass(P.Y, P.X, Q0, n0, n1 * n2, false);
        if (ok) ok = pass(P.X, P.Y, Q1, n1, n2, false);
        if (ok) ok = pass(P.Y, P.X, Q2, n2, 1, false);
        for (int p = tid; p < n && ok; p += nth) L.e[p] = (float)__ldcg(P.X + p);
        ok = coop_sync(P.bar, ok);
    }
    // ascent: interpolation, post-smoothing
    for (int l = nl - 2; l >= 0 && ok; l--) {
        const CoopLevel& L = P.lv[l];
        const CoopLevel& C = P.lv[l + 1];
        // e += I(e_{l+1}): per axis the even fine points copy, the odd ones
        // are w (a(k) + a(k+1)), k = (f + skip) / 2 - plo
        for (int p = tid; p < L.ng; p += nth) {
            int f[3];
            cv_split(p, L.n, f[0], f[1], f[2]);
            int idx[3][2];
            float wt[3][2];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const int u = f[a] + L.iskip[a];
                const int k = (u >> 1) - L.iplo[a];
                idx[a][0] = cv_at(k, C.n[a], C.per[a]);
                if (u & 1) {
                    idx[a][1] = cv_at(k + 1, C.n[a], C.per[a]);
                    wt[a][0] = wt[a][1] = L.iw;
                } else {
                    idx[a][1] = -1;
                    wt[a][0] = 1.0f;
                    wt[a][1] = 0.0f;
                }
            }
            float acc = 0.0f;
#pragma unroll
            for (int d0 = 0; d0 < 2; d0++) {
                if (idx[0][d0] < 0) continue;
#pragma unroll
                for (int d1 = 0; d1 < 2; d1++) {
                    if (idx[1][d1] < 0) continue;
                    const float w01 = wt[0][d0] * wt[1][d1];
                    const float* row = C.e + (idx[0][d0] * C.n[1] + idx[1][d1]) * C.n[2];
#pragma unroll
                    for (int d2 = 0; d2 < 2; d2++)
                        if (idx[2][d2] >= 0) acc += w01 * wt[2][d2] * __ldcg(row + idx[2][d2]);
                }
            }
            L.e[p] = __ldcg(L.e + p) + acc;
        }
        ok = coop_sync(P.bar, ok);
        for (int p = tid; p < L.ng; p += nth) {
            int i0, i1, i2;
            cv_split(p, L.n, i0, i1, i2);
            L.t[p] = L.inv_tc0 * (__ldcg(L.b + p) - cv_apply(L.e, L, p, i0, i1, i2));
        }
        ok = coop_sync(P.bar, ok);
        for (int p = tid; p < L.ng; p += nth) {
            int i0, i1, i2;
            cv_split(p, L.n, i0, i1, i2);
            L.e[p] = __ldcg(L.e + p) + L.k1 * __ldcg(L.t + p) -
                     L.k2 * cv_apply(L.t, L, p, i0, i1, i2);
        }
        ok = coop_sync(P.bar, ok);
    }
}

}  // namespace

int gb::take_fault_mixed(int* code) { return take_unit_fault(code); }

namespace {

__global__ void k_sumsq(const double* __restrict__ a, long long n, double* __restrict__ partial) {
    double v = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v += a[i] * a[i];
    v = block_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

__global__ void k_mixed_init(Ctl* ctl, const double* rho2, double tol, int maxiter) {
    ctl->rho2 = rho2[0];
    ctl->tol = tol;
    ctl->maxiter = maxiter;
    ctl->niter = 0;
    ctl->rel = 0.0;
}

// After the defect: rel = |d| / |rho|; continue while rel > tol and fewer
// than maxiter V-cycles ran.  `count` adds the V-cycle just finished.
__global__ void k_mixed_check(Ctl* ctl, const double* d2, int count,
                              cudaGraphConditionalHandle h) {
    const int n = ctl->niter + count;
    ctl->niter = n;
    const double rel = ctl->rho2 > 0.0 ? sqrt(d2[0] / ctl->rho2) : 0.0;
    ctl->rel = rel;
    cudaGraphSetConditional(h, (rel > ctl->tol && n < ctl->maxiter) ? 1u : 0u);
}

}  // namespace

struct gb_mixed {
    int L = 0;
    gb_operator* op64 = nullptr;
    std::vector<gb_operator*> ops;
    std::vector<gb_transformer*> rst, itp;
    std::vector<ChebLevel> ch;
    double coarse_lo = 0, coarse_hi = 0;
    int coarse_deg = 0;
    double* direct_tab = nullptr;   // eigen tables of the exact coarsest solve
    Seven direct_s7{};
    // levels lc .. L as one cooperative kernel (coop = 0: per-level kernels)
    int coop = 0, coop_ok = 0, lc = 0, coop_grid = 0;
    CoopPlan coop_plan{};
    double* coop_tab = nullptr;
    unsigned* coop_bar = nullptr;
    // the single-CTA form of the same kernel over levels lt..L (each at most
    // TAIL_MAX_POINTS points), for solves that run beside others
    int tail_ok = 0, lt = 0, tail = 0;
    CoopPlan tail_plan{};
    unsigned* tail_bar = nullptr;
    double last_tol = 0.0;
    int last_maxiter = 0;
    std::vector<float*> b, e, t;       // levels 0..L (b[L], e[L] used at L)
    double *x = nullptr, *r = nullptr, *da = nullptr, *db = nullptr;
    double *phi0 = nullptr, *rho0 = nullptr;
    double *partial = nullptr, *nrm = nullptr;
    Ctl* ctl = nullptr;
    Ctl* ctl_host = nullptr;
    int nblk64 = 0;   // partial-sum buffer length
    int nres = 0;     // partials written by the level-0 defect sweep
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~gb_mixed() {
        if (exec) cudaGraphExecDestroy(exec);
        if (cap) cudaStreamDestroy(cap);
        for (float* p : b) dfree(p);
        for (float* p : e) dfree(p);
        for (float* p : t) dfree(p);
        dfree(direct_tab);
        dfree(coop_tab);
        dfree(tail_bar);
        dfree(coop_bar);
        dfree(x);
        dfree(r);
        dfree(da);
        dfree(db);
        dfree(phi0);
        dfree(rho0);
        dfree(partial);
        dfree(nrm);
        dfree(ctl);
        if (ctl_host) hfree(ctl_host);
    }
};

// ------------------------------------------------------ FP32 level passes
// One pass y = p0 aux + p1 u + p2 (A u) + p3 aux2 of an FP32 level (A the
// level's axis-aligned stencil of half-width NN), written to `out` or added
// to an FP64 array.  The level arrays (a few tens of MB at most) stay in
// L2 between passes, so this kernel stages nothing in shared memory: a
// thread owns one (row, column) of the grid and marches along axis 0 with
// the 2NN+1 values of its column in registers; the in-plane neighbours are
// read through the L1 cache, which a CTA's 32 x 8 tile shares.  No barriers,
// no copy bookkeeping: for these passes the plane-marching kernel spent
// about 150 instructions a point on staging.  FP32 fused multiply-adds
// (the FP32 V-cycle's arithmetic is its own; it is checked by tolerance).
// F: 1 = aux, 2 = aux2, 4 = add to acc64 instead of writing out.
template <int NN, int F>
__global__ void __launch_bounds__(256)
k_lin32(const float* __restrict__ u, float* __restrict__ out, const float* __restrict__ aux,
        const float* __restrict__ aux2, double* __restrict__ acc64, GridBC g, CfdStencil cs,
        float p0, float p1, float p2, float p3, int chunk, int tiles_x) {
    constexpr int Q = 2 * NN + 1;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int x = (blockIdx.x % tiles_x) * 32 + (threadIdx.x & 31);
    const int y = (blockIdx.x / tiles_x) * 8 + (threadIdx.x >> 5);
    const int pa = blockIdx.y * chunk;
    const int pb = min(n0, pa + chunk);
    if (x >= n2 || y >= n1 || pa >= pb) return;
    const long long ps = (long long)n1 * n2;
    // in-plane neighbours: offsets after the boundary, or -1 (zero)
    int xo[2 * NN], yo[2 * NN];
#pragma unroll
    for (int d = 1; d <= NN; d++) {
        int a = x + d, b = x - d;
        xo[d - 1] = (a < n2) ? a : (g.periodic[2] && a - n2 < n2 ? a - n2 : -1);
        xo[NN + d - 1] = (b >= 0) ? b : (g.periodic[2] && b + n2 >= 0 ? b + n2 : -1);
        a = y + d;
        b = y - d;
        yo[d - 1] = (a < n1) ? a * n2 : (g.periodic[1] && a - n1 < n1 ? (a - n1) * n2 : -1);
        yo[NN + d - 1] = (b >= 0) ? b * n2 : (g.periodic[1] && b + n1 >= 0 ? (b + n1) * n2 : -1);
    }
    const int row = y * n2;
    auto col_at = [&](int p) -> float {   // u at plane p of this column
        if (p < 0 || p >= n0) {
            if (!g.periodic[0]) return 0.0f;
            p += p < 0 ? n0 : -n0;
            if (p < 0 || p >= n0) return 0.0f;
        }
        return __ldg(u + p * ps + row + x);
    };
    float q[Q];
#pragma unroll
    for (int k = 0; k < Q - 1; k++) q[k + 1] = col_at(pa - NN + k);
    const float c0 = (float)cs.c0;
    float cp[3][NN], cm[3][NN];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int d = 0; d < NN; d++) {
            cp[k][d] = (float)cs.cp[k][d];
            cm[k][d] = (float)cs.cm[k][d];
        }
#pragma unroll 2
    for (int p = pa; p < pb; p++) {
#pragma unroll
        for (int k = 0; k < Q - 1; k++) q[k] = q[k + 1];
        q[Q - 1] = col_at(p + NN);
        const float* pl = u + p * ps;
        // one partial sum a direction (axis 2, 1, 0), added at the end
        float s2 = c0 * q[NN], s1 = 0.0f, s0 = 0.0f;
#pragma unroll
        for (int d = 0; d < NN; d++) {
            const float a = xo[d] >= 0 ? __ldg(pl + row + xo[d]) : 0.0f;
            const float b = xo[NN + d] >= 0 ? __ldg(pl + row + xo[NN + d]) : 0.0f;
            s2 = fmaf(cp[0][d], a, fmaf(cm[0][d], b, s2));
            const float c = yo[d] >= 0 ? __ldg(pl + yo[d] + x) : 0.0f;
            const float e = yo[NN + d] >= 0 ? __ldg(pl + yo[NN + d] + x) : 0.0f;
            s1 = fmaf(cp[1][d], c, fmaf(cm[1][d], e, s1));
            s0 = fmaf(cp[2][d], q[NN + 1 + d], fmaf(cm[2][d], q[NN - 1 - d], s0));
        }
        const float au = (s2 + s1) + s0;
        const long long at = p * ps + row + x;
        float v = fmaf(p1, q[NN], p2 * au);
        if (F & 1) v = fmaf(p0, aux[at], v);
        if (F & 2) v = fmaf(p3, aux2[at], v);
        if (F & 4) acc64[at] += (double)v;
        else out[at] = v;
    }
}

template <int NN>
static void launch_lin32_nn(const gb_operator* op, const float* in, float* out, const float* aux,
                            const float* aux2, double* acc64, float p0, float p1, float p2,
                            float p3, cudaStream_t st) {
    const GridBC& g = op->g;
    const int tiles_x = (g.n[2] + 31) / 32, tiles_y = (g.n[1] + 7) / 8;
    int chunk = op->chunk > 0 ? std::min(op->chunk, g.n[0]) : g.n[0];
    if (op->chunk <= 0)
        while (chunk > 2 * NN + 2 && (long long)tiles_x * tiles_y * ((g.n[0] + chunk - 1) / chunk) <
                                         148 * 6)
            chunk = (chunk + 1) / 2;
    dim3 grid(tiles_x * tiles_y, (g.n[0] + chunk - 1) / chunk);
    const int f = (aux ? 1 : 0) | (aux2 ? 2 : 0) | (acc64 ? 4 : 0);
#define GB_LIN32(F)                                                                          \
    k_lin32<NN, F><<<grid, 256, 0, st>>>(in, out, aux, aux2, acc64, g, op->cs, p0, p1, p2, p3, \
                                         chunk, tiles_x)
    switch (f) {
        case 0: GB_LIN32(0); break;
        case 1: GB_LIN32(1); break;
        case 2: GB_LIN32(2); break;
        case 3: GB_LIN32(3); break;
        case 4: GB_LIN32(4); break;
        case 5: GB_LIN32(5); break;
        case 6: GB_LIN32(6); break;
        default: GB_LIN32(7); break;
    }
#undef GB_LIN32
}

// The FP32 passes through k_lin32 only with GPAW_B200_LIN32=1: on the
// 192^3 grid it measured no faster than the plane-marching kernel's EPI_LIN
// mode (level-0 passes 55-86 us either way, 6.99 against 6.70 ms a solve).
static bool lin32_direct() {
    static const bool on = [] {
        const char* e = getenv("GPAW_B200_LIN32");
        return e && atoi(e) != 0;
    }();
    return on;
}

// The level passes and the FP64 defect through k_pass (gb_pass.cu) unless
// GPAW_B200_PASS=0 (the plane-marching kernel's EPI_LIN mode instead).
static bool pass_on() {
    static const bool on = [] {
        const char* e = getenv("GPAW_B200_PASS");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

static int lin32(const gb_operator* op, const float* in, float* out, const float* aux,
                 const float* aux2, double p0, double p1, double p2, double p3, double* acc64,
                 cudaStream_t st) {
    const CfdStencil& cs = op->cs;
    if (!(cs.axis[0] == 2 && cs.axis[1] == 1 && cs.axis[2] == 0)) return -1;
    const float f0 = (float)p0, f1 = (float)p1, f2 = (float)p2, f3 = (float)p3;
    switch (op->nn) {
        case 1: launch_lin32_nn<1>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        case 2: launch_lin32_nn<2>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        case 3: launch_lin32_nn<3>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        case 4: launch_lin32_nn<4>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        case 5: launch_lin32_nn<5>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        case 6: launch_lin32_nn<6>(op, in, out, aux, aux2, acc64, f0, f1, f2, f3, st); break;
        default: return -1;
    }
    return 0;
}

// One stencil pass of the linear epilogue on level l (float) or on the
// level-0 FP64 operator (double).
template <class T>
static int lin(gb_operator* op, const T* in, T* out, const T* aux, const T* aux2, double p0,
               double p1, double p2, double p3, double* acc64, float* out32, double* partial,
               cudaStream_t st) {
    if constexpr (sizeof(T) == 4) {
        if (lin32_direct() && !partial && !out32 &&
            lin32(op, in, out, aux, aux2, p0, p1, p2, p3, acc64, st) == 0) {
            GB_LAUNCH_CHECK();
            return 0;
        }
    }
    if (pass_on()) {
        const int rc = launch_pass<T>(op->g, op->cs, op->nn, in, out, aux, aux2, p0, p1, p2, p3,
                                      acc64, out32, partial, st);
        if (rc == -2) return fail(GB_ECUDA, "mixed: could not raise the shared-memory limit");
        if (rc == 0) {
            GB_LAUNCH_CHECK();
            return 0;
        }
    }
    Epi ep{};
    ep.aux = aux;
    ep.aux2 = aux2;
    ep.p0 = p0;
    ep.p1 = p1;
    ep.p2 = p2;
    ep.p3 = p3;
    ep.acc64 = acc64;
    ep.out32 = out32;
    ep.partial = partial;
    ep.chunk = op->chunk;
    Phases P{};
    const int rc = launch_fd_cfd<T>(EPI_LIN, in, out, 1, op->g, P, op->cs, op->nn, ep, st, nullptr);
    if (rc == -2) return fail(GB_ECUDA, "mixed: could not raise the shared-memory limit");
    if (rc) return fail(GB_EINVAL, "mixed: operator is not an axis-aligned stencil");
    GB_LAUNCH_CHECK();
    return 0;
}

// V-cycle on levels l..L for the FP32 right-hand side b[l]; at level 0 the
// final correction is added to phi0 (FP64).
// Set while a batch of solvers is captured: its branches run side by side,
// and cooperative kernels (which need the whole GPU resident at once) would
// serialise them, so the batch keeps the per-level kernels.
static thread_local bool t_no_coop = false;

static int vcycle32(gb_mixed* m, int l, cudaStream_t st) {
    const bool coop = m->coop && !t_no_coop;
    if (!coop && m->tail && m->tail_ok && l == m->lt) {
        trace_mark("levels lt..L: one single-CTA kernel", st);
        k_coop_vcycle<<<1, 512, 0, st>>>(m->tail_plan);
        GB_LAUNCH_CHECK();
        return 0;
    }
    if (coop && l == m->lc) {
        trace_mark("levels lc..L: one cooperative kernel", st);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(m->coop_grid);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        GB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_coop_vcycle, m->coop_plan));
        return 0;
    }
    if (l == m->L) {
        gb_operator* op = m->ops[l];
        const long long n = op->ng();
        // the 7-point form of the coarsest operator, if it has one
        Seven s7{};
        int seven = op->st.ncoefs == 7 && op->st.range == 1 && op->st.cfd;
        if (seven) {
            for (int c = 0; c < 7; c++) {
                int ax = -1, dir = 0;
                for (int a = 0; a < 3; a++)
                    if (op->st.off[c][a]) {
                        ax = a;
                        dir = op->st.off[c][a];
                    }
                if (ax < 0) s7.c0 += op->st.coef[c];
                else if (dir > 0) s7.cp[ax] = op->st.coef[c];
                else s7.cm[ax] = op->st.coef[c];
            }
        }
        if (m->direct_tab) {
            const GridBC& g = op->g;
            const size_t smem = ((size_t)2 * n + (size_t)g.n[0] * g.n[0] + (size_t)g.n[1] * g.n[1] +
                                 (size_t)g.n[2] * g.n[2] + g.n[0] + g.n[1] + g.n[2]) *
                                sizeof(double);
            trace_mark("coarsest: FP64 exact solve", st);
            k_coarse_direct<<<1, 1024, smem, st>>>(m->b[l], m->e[l], m->direct_tab, g.n[0], g.n[1],
                                                   g.n[2], m->direct_s7.c0, m->direct_s7.cp[0],
                                                   m->direct_s7.cp[1], m->direct_s7.cp[2]);
            GB_LAUNCH_CHECK();
            return 0;
        }
        trace_mark("coarsest: FP64 Chebyshev solve", st);
        if (seven && n <= CLUSTER_COARSE_MAX) {
            const int chunk = (int)((n + CL - 1) / CL);
            const size_t smem = (size_t)2 * chunk * sizeof(double);
            static bool cattr = false;
            if (!cattr) {
                GB_CUDA_TRY(cudaFuncSetAttribute(k_coarse_cheb_cluster,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)((size_t)2 * (CLUSTER_COARSE_MAX / CL) *
                                                       sizeof(double))));
                cattr = true;
            }
            k_coarse_cheb_cluster<<<CL, 1024, smem, st>>>(m->b[l], m->e[l], op->g, s7,
                                                          m->coarse_lo, m->coarse_hi,
                                                          m->coarse_deg);
        } else if (n <= SMEM_COARSE_MAX && op->g.n[1] < 1024 && op->g.n[2] < 1024) {
            const size_t smem = (size_t)2 * n * sizeof(double);
            static bool attr = false;
            if (!attr) {
                GB_CUDA_TRY(cudaFuncSetAttribute(k_coarse_cheb_smem,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)((size_t)2 * SMEM_COARSE_MAX * sizeof(double))));
                attr = true;
            }
            k_coarse_cheb_smem<<<1, 1024, smem, st>>>(m->b[l], m->e[l], op->g, op->st, s7, seven,
                                                       m->coarse_lo, m->coarse_hi, m->coarse_deg);
        } else {
            k_coarse_cheb<<<1, 1024, 0, st>>>(m->b[l], m->e[l], m->x, m->r, m->da, m->db, op->g,
                                               op->st, m->coarse_lo, m->coarse_hi, m->coarse_deg);
        }
        GB_LAUNCH_CHECK();
        return 0;
    }
    gb_operator* op = m->ops[l];
    const ChebLevel& c = m->ch[l];
    float *b = m->b[l], *e = m->e[l], *t = m->t[l];
    int rc;
    static const char* const lbl[][6] = {
        {"L0 pre-smooth", "L0 residual", "L0 restrict", "L0 interpolate", "L0 post-smooth 1",
         "L0 post-smooth 2 (phi += e)"},
        {"L1 pre-smooth", "L1 residual", "L1 restrict", "L1 interpolate", "L1 post-smooth 1",
         "L1 post-smooth 2"},
        {"L2 pre-smooth", "L2 residual", "L2 restrict", "L2 interpolate", "L2 post-smooth 1",
         "L2 post-smooth 2"},
        {"L3+ pre-smooth", "L3+ residual", "L3+ restrict", "L3+ interpolate",
         "L3+ post-smooth 1", "L3+ post-smooth 2"}};
    const char* const* lb = lbl[l < 3 ? l : 3];
    // pre-smooth from zero
    trace_mark(lb[0], st);
    if ((rc = lin<float>(op, b, e, nullptr, nullptr, 0, c.pre_u, c.pre_Lu, 0, nullptr, nullptr,
                         nullptr, st)))
        return rc;
    // residual t = b - A e, restricted to the next level
    trace_mark(lb[1], st);
    if ((rc = lin<float>(op, e, t, b, nullptr, 1.0, 0.0, -1.0, 0, nullptr, nullptr, nullptr, st)))
        return rc;
    Phases P{};
    trace_mark(lb[2], st);
    if ((rc = transform_impl(m->rst[l], t, m->b[l + 1], nullptr, 1, GB_F32_INTERNAL, P, 0, 0, 0.0, st)))
        return rc;
    if ((rc = vcycle32(m, l + 1, st))) return rc;
    // e += I(e_{l+1})   (as e -= I(-e_{l+1}), negation exact)
    trace_mark(lb[3], st);
    if ((rc = transform_impl(m->itp[l], m->e[l + 1], e, nullptr, 1, GB_F32_INTERNAL, P, 1, 1, 0.0, st)))
        return rc;
    // post-smooth: t = (b - A e) / (theta c0); e += k1 t - k2 A t
    trace_mark(lb[4], st);
    if ((rc = lin<float>(op, e, t, b, nullptr, c.inv_tc0, 0.0, -c.inv_tc0, 0, nullptr, nullptr,
                         nullptr, st)))
        return rc;
    trace_mark(lb[5], st);
    if (l == 0)
        rc = lin<float>(op, t, e, nullptr, e, 0, c.k1, -c.k2, 1.0, m->phi0, nullptr, nullptr, st);
    else
        rc = lin<float>(op, t, e, nullptr, e, 0, c.k1, -c.k2, 1.0, nullptr, nullptr, nullptr, st);
    return rc;
}

// d = rho - L64 phi  ->  b[0] (float) and |d|^2 -> nrm[0]
static int defect(gb_mixed* m, cudaStream_t st) {
    trace_mark("FP64 defect d = rho - L phi, |d|^2", st);
    if (int rc = lin<double>(m->op64, m->phi0, nullptr, m->rho0, nullptr, 1.0, 0.0, -1.0, 0,
                             nullptr, m->b[0], m->partial, st))
        return rc;
    trace_mark("FP64 defect norm reduction", st);
    launch_reduce_partials(m->partial, m->nres, 1, 1.0, m->nrm, st);
    GB_LAUNCH_CHECK();
    trace_mark("end of defect", st);
    return 0;
}

// The exact coarsest solve, opt-in (GPAW_B200_COARSE_DIRECT=1), when the
// coarsest operator is a symmetric 7-point stencil and the grid, two copies
// of it and the eigen tables fit in one CTA's shared memory.  Measured on
// the 192^3 grid with 4 levels (coarsest 23^3): 144 us a solve against
// 75 us for the Chebyshev iteration (shared-memory bound on one SM), and
// 14 V-cycles instead of 15, so the Chebyshev iteration stays the default.
static int setup_direct(gb_mixed* m) {
    const char* env = getenv("GPAW_B200_COARSE_DIRECT");
    if (!env || atoi(env) == 0) return 0;
    gb_operator* op = m->ops[m->L];
    if (!(op->st.ncoefs == 7 && op->st.range == 1 && op->st.cfd)) return 0;
    Seven s7{};
    for (int c = 0; c < 7; c++) {
        int ax = -1, dir = 0;
        for (int a = 0; a < 3; a++)
            if (op->st.off[c][a]) {
                ax = a;
                dir = op->st.off[c][a];
            }
        if (ax < 0) s7.c0 += op->st.coef[c];
        else if (dir > 0) s7.cp[ax] = op->st.coef[c];
        else s7.cm[ax] = op->st.coef[c];
    }
    for (int a = 0; a < 3; a++)
        if (s7.cp[a] != s7.cm[a]) return 0;
    const GridBC& g = op->g;
    const long long n = op->ng();
    const long long ntab = (long long)g.n[0] * g.n[0] + (long long)g.n[1] * g.n[1] +
                           (long long)g.n[2] * g.n[2] + g.n[0] + g.n[1] + g.n[2];
    const size_t smem = (size_t)(2 * n + ntab) * sizeof(double);
    if (smem > 225 * 1024) return 0;
    std::vector<double> tab(ntab);
    double* q = tab.data();
    double* mu = q + (long long)g.n[0] * g.n[0] + (long long)g.n[1] * g.n[1] +
                 (long long)g.n[2] * g.n[2];
    for (int a = 0; a < 3; a++) {
        neighbour_eigen(g.n[a], g.periodic[a] != 0, q, mu);
        q += (long long)g.n[a] * g.n[a];
        mu += g.n[a];
    }
    static bool attr = false;
    if (!attr) {
        GB_CUDA_TRY(cudaFuncSetAttribute(k_coarse_direct,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         225 * 1024));
        attr = true;
    }
    GB_CUDA_TRY(pool_malloc(&m->direct_tab, ntab * sizeof(double)));
    GB_CUDA_TRY(cudaMemcpy(m->direct_tab, tab.data(), ntab * sizeof(double),
                           cudaMemcpyHostToDevice));
    m->direct_s7 = s7;
    return 0;
}

// The cooperative kernel takes the coarsest level (its exact solve), and
// with GPAW_B200_COOP_MAX_POINTS=n also every level from the first with at
// most n points, when the coarsest operator is a symmetric 7-point stencil
// (the exact solve needs the eigen tables) and every level below 0 has the
// 7-point operator (what MixedPoissonSolver builds).  Measured on the 192^3
// grid with 4 levels: the coarsest alone 6.70 ms a solve, levels 2-3
// 7.15 ms, levels 1-3 8.17 ms (grid-stride passes and grid barriers cost
// more than the tiled kernels on the larger levels).
// GPAW_B200_COOP_COARSE=0 keeps the per-level kernels and the Chebyshev
// coarsest solve.
constexpr long long COOP_MAX_POINTS = 0;

// The levels lc..L of a cooperative-kernel plan; false when one of them
// does not have the 7-point operator and order-2 transfers it assumes (or
// the coarsest operator is not symmetric).
static bool fill_coop_levels(gb_mixed* m, int lc, CoopPlan& P) {
    for (int l = lc; l <= m->L; l++) {
        const gb_operator* op = m->ops[l];
        if (!(op->st.ncoefs == 7 && op->st.range == 1 && op->st.cfd)) return false;
        Seven s7{};
        for (int c = 0; c < 7; c++) {
            int ax = -1, dir = 0;
            for (int a = 0; a < 3; a++)
                if (op->st.off[c][a]) {
                    ax = a;
                    dir = op->st.off[c][a];
                }
            if (ax < 0) s7.c0 += op->st.coef[c];
            else if (dir > 0) s7.cp[ax] = op->st.coef[c];
            else s7.cm[ax] = op->st.coef[c];
        }
        CoopLevel& V = P.lv[l - lc];
        for (int a = 0; a < 3; a++) {
            V.n[a] = op->g.n[a];
            V.per[a] = op->g.periodic[a];
            V.cp[a] = (float)s7.cp[a];
            V.cm[a] = (float)s7.cm[a];
        }
        V.ng = (int)op->ng();
        V.c0 = (float)s7.c0;
        V.b = m->b[l];
        V.e = m->e[l];
        V.t = m->t[l];
        if (l < m->L) {
            const ChebLevel& c = m->ch[l];
            V.pre_u = (float)c.pre_u;
            V.pre_Lu = (float)c.pre_Lu;
            V.inv_tc0 = (float)c.inv_tc0;
            V.k1 = (float)c.k1;
            V.k2 = (float)c.k2;
            const gb_transformer* r = m->rst[l];
            const gb_transformer* i = m->itp[l];
            if (r->k != 2 || i->k != 2) return false;
            for (int a = 0; a < 3; a++) {
                V.rplo[a] = r->G.plo[a];
                V.iplo[a] = i->G.plo[a];
                V.iskip[a] = i->G.skip0[a];
            }
            V.rw = (float)r->G.w[0];
            V.iw = (float)i->G.w[0];
        } else {
            for (int a = 0; a < 3; a++)
                if (s7.cp[a] != s7.cm[a]) return false;
            P.dc0 = s7.c0;
            for (int a = 0; a < 3; a++) P.dca[a] = s7.cp[a];
        }
    }
    return true;
}

static int setup_coop(gb_mixed* m) {
    const char* env = getenv("GPAW_B200_COOP_COARSE");
    if (env && atoi(env) == 0) return 0;
    const char* emax = getenv("GPAW_B200_COOP_MAX_POINTS");
    const long long maxpts = emax ? atoll(emax) : COOP_MAX_POINTS;
    int lc = m->L;
    for (int l = 1; l <= m->L; l++)
        if (m->ops[l]->ng() <= maxpts) {
            lc = l;
            break;
        }
    if (lc < 0 || m->L - lc + 1 > CV_MAX) return 0;
    CoopPlan& P = m->coop_plan;
    memset(&P, 0, sizeof P);
    if (!fill_coop_levels(m, lc, P)) return 0;
    // eigen tables of the coarsest level
    const GridBC& g = m->ops[m->L]->g;
    const long long ntab = (long long)g.n[0] * g.n[0] + (long long)g.n[1] * g.n[1] +
                           (long long)g.n[2] * g.n[2] + g.n[0] + g.n[1] + g.n[2];
    std::vector<double> tab(ntab);
    double* q = tab.data();
    double* mu = q + ntab - (g.n[0] + g.n[1] + g.n[2]);
    for (int a = 0; a < 3; a++) {
        neighbour_eigen(g.n[a], g.periodic[a] != 0, q, mu);
        q += (long long)g.n[a] * g.n[a];
        mu += g.n[a];
    }
    int per_sm = 0, dev = 0, nsm = 0;
    GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coop_vcycle, 512, 0));
    GB_CUDA_TRY(cudaGetDevice(&dev));
    GB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return 0;
    GB_CUDA_TRY(pool_malloc(&m->coop_tab, ntab * sizeof(double)));
    GB_CUDA_TRY(cudaMemcpy(m->coop_tab, tab.data(), ntab * sizeof(double),
                           cudaMemcpyHostToDevice));
    GB_CUDA_TRY(pool_malloc(&m->coop_bar, 2 * sizeof(unsigned)));
    GB_CUDA_TRY(cudaMemset(m->coop_bar, 0, 2 * sizeof(unsigned)));
    P.nl = m->L - lc + 1;
    P.tab = m->coop_tab;
    P.X = m->x;
    P.Y = m->r;
    P.bar = m->coop_bar;
    m->lc = lc;
    const char* eps = getenv("GPAW_B200_COOP_PER_SM");
    const int want = eps ? std::max(1, atoi(eps)) : 1;
    m->coop_grid = std::min(per_sm, want) * nsm;
    m->coop_ok = 1;
    m->coop = 1;
    return 0;
}

// The single-CTA tail: levels from the first below 0 with at most
// TAIL_MAX_POINTS points down to the coarsest, in one launch of the same
// kernel with one block (its grid barrier is then a block barrier), so
// that solves running side by side (a batch graph, the serving loop) each
// take their coarse levels in one kernel instead of six a level.  Uses the
// coarsest level's eigen tables, so it needs setup_coop to have built
// them.  GPAW_B200_TAIL=0 keeps the per-level kernels;
// GPAW_B200_TAIL_MAX_POINTS sets the size bound (512-grid batch: 2146,
// 2158, 2176, 2183 and 2189 solves/s for bounds of 2048, 4096, 8192, 16384
// and 40000 points).  The coarsest level itself must have at most
// TAIL_MAX_COARSEST points: the exact solve's dense passes on one SM cost
// about n (n0 + n1 + n2) multiply-adds (on the 192^3 grid's 23^3 coarsest
// level the single block took 10.0 ms a solve against 5.2 with the whole
// GPU's cooperative kernel).
constexpr long long TAIL_MAX_POINTS = 16384;
constexpr long long TAIL_MAX_COARSEST = 4096;

static int setup_tail(gb_mixed* m) {
    const char* env = getenv("GPAW_B200_TAIL");
    if ((env && atoi(env) == 0) || !m->coop_tab) return 0;
    if (m->ops[m->L]->ng() > TAIL_MAX_COARSEST) return 0;
    const char* emax = getenv("GPAW_B200_TAIL_MAX_POINTS");
    const long long maxpts = emax ? atoll(emax) : TAIL_MAX_POINTS;
    int lt = -1;
    for (int l = 1; l <= m->L; l++)
        if (m->ops[l]->ng() <= maxpts) {
            lt = l;
            break;
        }
    if (lt < 0 || m->L - lt + 1 > CV_MAX) return 0;
    CoopPlan& P = m->tail_plan;
    memset(&P, 0, sizeof P);
    if (!fill_coop_levels(m, lt, P)) return 0;
    GB_CUDA_TRY(pool_malloc(&m->tail_bar, 2 * sizeof(unsigned)));
    GB_CUDA_TRY(cudaMemset(m->tail_bar, 0, 2 * sizeof(unsigned)));
    P.nl = m->L - lt + 1;
    P.tab = m->coop_tab;
    P.X = m->x;
    P.Y = m->r;
    P.bar = m->tail_bar;
    m->lt = lt;
    m->tail_ok = 1;
    return 0;
}

extern "C" int gb_mixed_new(int nlevels, gb_operator* op64, gb_operator* const* operators,
                            gb_transformer* const* restrictors,
                            gb_transformer* const* interpolators, const double* lam_max,
                            double lam_min_coarse, int coarse_degree, gb_mixed** out) {
    if (!out || !op64 || !operators || !lam_max || nlevels < 2 || !restrictors || !interpolators)
        return fail(GB_EINVAL, "mixed: bad arguments (needs at least two levels)");
    *out = nullptr;
    if (!op64->real || !op64->tiled)
        return fail(GB_EINVAL, "mixed: level-0 operator must be a real axis-aligned stencil");
    if (coarse_degree < 1 || lam_min_coarse <= 0.0)
        return fail(GB_EINVAL, "mixed: coarse degree >= 1 and a positive lower bound needed");
    gb_mixed* m = new gb_mixed();
    m->L = nlevels - 1;
    m->op64 = op64;
    for (int l = 0; l < nlevels; l++) {
        gb_operator* op = operators[l];
        if (!op || !op->real || (l < m->L && !op->tiled)) {
            delete m;
            return fail(GB_EINVAL, "mixed: level %d operator must be a real axis-aligned stencil", l);
        }
        m->ops.push_back(op);
        if (l < m->L) m->ch.push_back(cheb_level(lam_max[l], op->st.coef[0]));
    }
    if (m->ops[0]->ng() != op64->ng()) {
        delete m;
        return fail(GB_EINVAL, "mixed: level-0 operators differ in size");
    }
    for (int l = 0; l < m->L; l++) {
        gb_transformer* rr = restrictors[l];
        gb_transformer* ii = interpolators[l];
        if (!rr || !ii || rr->interpolate || !ii->interpolate || rr->ngin != m->ops[l]->ng() ||
            rr->ngout != m->ops[l + 1]->ng() || ii->ngin != m->ops[l + 1]->ng() ||
            ii->ngout != m->ops[l]->ng()) {
            delete m;
            return fail(GB_EINVAL, "mixed: transformer %d does not match the levels", l);
        }
        m->rst.push_back(rr);
        m->itp.push_back(ii);
    }
    m->coarse_hi = 1.02 * lam_max[m->L];
    m->coarse_lo = lam_min_coarse;
    m->coarse_deg = coarse_degree;
    if (int rc = setup_direct(m)) {
        delete m;
        return rc;
    }
    cudaError_t ce = cudaSuccess;
    for (int l = 0; l <= m->L && ce == cudaSuccess; l++) {
        const size_t bytes = (size_t)m->ops[l]->ng() * sizeof(float);
        float *bb = nullptr, *ee = nullptr, *tt = nullptr;
        ce = pool_malloc(&bb, bytes);
        if (ce == cudaSuccess) ce = pool_malloc(&ee, bytes);
        if (ce == cudaSuccess) ce = pool_malloc(&tt, bytes);
        m->b.push_back(bb);
        m->e.push_back(ee);
        m->t.push_back(tt);
    }
    const size_t nc = (size_t)m->ops[m->L]->ng() * sizeof(double);
    const size_t n0 = (size_t)op64->ng() * sizeof(double);
    // partial sums of the defect: one per CTA of the pass kernel when it
    // takes the level-0 operator, else of the plane-marching kernel
    m->nres = (pass_on() && pass_supported_grid(op64->g, op64->cs, op64->nn))
                  ? pass_blocks(op64->g, 8)
                  : op_resid_blocks(op64, 1, 8);
    m->nblk64 = std::max(m->nres, 1024);
    if (ce == cudaSuccess) ce = pool_malloc(&m->x, nc);
    if (ce == cudaSuccess) ce = pool_malloc(&m->r, nc);
    if (ce == cudaSuccess) ce = pool_malloc(&m->da, nc);
    if (ce == cudaSuccess) ce = pool_malloc(&m->db, nc);
    if (ce == cudaSuccess) ce = pool_malloc(&m->phi0, n0);
    if (ce == cudaSuccess) ce = pool_malloc(&m->rho0, n0);
    if (ce == cudaSuccess) ce = pool_malloc(&m->partial, (size_t)m->nblk64 * sizeof(double));
    if (ce == cudaSuccess) ce = pool_malloc(&m->nrm, 2 * sizeof(double));
    if (ce == cudaSuccess) ce = pool_malloc(&m->ctl, sizeof(Ctl));
    if (ce == cudaSuccess) ce = pool_malloc_host(&m->ctl_host, sizeof(Ctl));
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&m->cap, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        delete m;
        return fail(GB_ECUDA, "mixed: allocation: %s", cudaGetErrorString(ce));
    }
    if (int rc = setup_coop(m)) {
        delete m;
        return rc;
    }
    if (int rc = setup_tail(m)) {
        delete m;
        return rc;
    }
    *out = m;
    return 0;
}

extern "C" void gb_mixed_free(gb_mixed* m) { delete m; }

extern "C" int gb_mixed_set_fused_coarse(gb_mixed* m, int mode) {
    if (!m) return fail(GB_EINVAL, "mixed: NULL solver");
    const int coop = (mode == 1 && m->coop_ok) ? 1 : 0;
    const int tail = (mode == 2 && m->tail_ok) ? 1 : 0;
    if ((coop != m->coop || tail != m->tail) && m->exec) {
        cudaGraphExecDestroy(m->exec);   // captured with the other path
        m->exec = nullptr;
    }
    m->coop = coop;
    m->tail = tail;
    return 0;
}

// Graph:  defect; check -> WHILE { V32 (phi += e); defect; check }
static int build_mixed_graph(gb_mixed* m) {
    cudaStream_t cs = m->cap;
    const size_t n0 = (size_t)m->op64->ng() * sizeof(double);
    // one uncaptured pass: sets kernel attributes
    GB_CUDA_TRY(cudaMemsetAsync(m->phi0, 0, n0, cs));
    GB_CUDA_TRY(cudaMemsetAsync(m->rho0, 0, n0, cs));
    if (int rc = defect(m, cs)) return rc;
    if (int rc = vcycle32(m, 0, cs)) return rc;
    GB_CUDA_TRY(cudaStreamSynchronize(cs));

    cudaGraph_t graph;
    GB_CUDA_TRY(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h;
    GB_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
    // head: initial defect and check (sets the loop condition)
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    int rc = defect(m, cs);
    if (!rc) k_mixed_check<<<1, 1, 0, cs>>>(m->ctl, m->nrm, 0, h);
    cudaGraph_t gout = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cs, &gout);
    if (rc || ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return rc ? rc : fail(GB_ECUDA, "mixed: capture: %s", cudaGetErrorString(ce));
    }
    size_t nleaf = 0;
    GB_CUDA_TRY(cudaGraphGetNodes(graph, nullptr, &nleaf));
    std::vector<cudaGraphNode_t> nodes(nleaf);
    GB_CUDA_TRY(cudaGraphGetNodes(graph, nodes.data(), &nleaf));
    // the check kernel is the only node without dependents
    cudaGraphNode_t tail = nullptr;
    for (auto nd : nodes) {
        size_t nout = 0;
        GB_CUDA_TRY(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
        if (nout == 0) tail = nd;
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    GB_CUDA_TRY(cudaGraphAddNode(&wnode, graph, &tail, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    rc = vcycle32(m, 0, cs);
    if (!rc) rc = defect(m, cs);
    if (!rc) k_mixed_check<<<1, 1, 0, cs>>>(m->ctl, m->nrm, 1, h);
    ce = cudaStreamEndCapture(cs, &gout);
    if (rc || ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return rc ? rc : fail(GB_ECUDA, "mixed: capture of the V-cycle: %s", cudaGetErrorString(ce));
    }
    cudaError_t ie = cudaGraphInstantiate(&m->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(GB_ECUDA, "mixed: instantiate: %s", cudaGetErrorString(ie));
    return 0;
}

extern "C" int gb_mixed_prepare(gb_mixed* m) {
    if (!m) return fail(GB_EINVAL, "mixed prepare: NULL solver");
    if (!m->exec) {
        int rc = build_mixed_graph(m);
        if (rc && m->coop) {
            // a graph that would not take the cooperative kernel: per-level
            // kernels instead
            cudaGetLastError();
            m->coop = 0;
            rc = build_mixed_graph(m);
        }
        if (rc) return rc;
    }
    return 0;
}

extern "C" int gb_mixed_solve_async(gb_mixed* m, double* phi, const double* rho, double tol,
                                    int maxiter, void* stream) {
    if (!m || !phi || !rho) return fail(GB_EINVAL, "mixed solve: NULL argument");
    if (maxiter < 1) return fail(GB_EINVAL, "mixed solve: maxiter must be >= 1");
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = gb_mixed_prepare(m)) return rc;
    const long long n = m->op64->ng();
    const size_t bytes = (size_t)n * sizeof(double);
    GB_CUDA_TRY(cudaMemcpyAsync(m->rho0, rho, bytes, cudaMemcpyDeviceToDevice, st));
    GB_CUDA_TRY(cudaMemcpyAsync(m->phi0, phi, bytes, cudaMemcpyDeviceToDevice, st));
    const int nb = (int)std::min<long long>(1024, (n + 255) / 256);
    k_sumsq<<<nb, 256, 0, st>>>(m->rho0, n, m->partial);
    launch_reduce_partials(m->partial, nb, 1, 1.0, m->nrm + 1, st);
    k_mixed_init<<<1, 1, 0, st>>>(m->ctl, m->nrm + 1, tol, maxiter);
    GB_LAUNCH_CHECK();
    GB_CUDA_TRY(cudaGraphLaunch(m->exec, st));
    GB_CUDA_TRY(cudaMemcpyAsync(phi, m->phi0, bytes, cudaMemcpyDeviceToDevice, st));
    GB_CUDA_TRY(cudaMemcpyAsync(m->ctl_host, m->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    m->last_tol = tol;
    m->last_maxiter = maxiter;
    return 0;
}

extern "C" int gb_mixed_result(gb_mixed* m, int* niter, double* rel_residual) {
    if (!m) return fail(GB_EINVAL, "mixed result: NULL solver");
    if (niter) *niter = m->ctl_host->niter;
    if (rel_residual) *rel_residual = m->ctl_host->rel;
    if (m->ctl_host->rel > m->last_tol)
        return fail(GB_ENOCONV, "mixed-precision Poisson solver did not reach %g in %d V-cycles",
                    m->last_tol, m->last_maxiter);
    return 0;
}

// One V-cycle and its defect launched kernel by kernel (no graph), for
// profilers and kernel traces: phi <- phi + V32(rho - L phi).
extern "C" int gb_mixed_vcycle_eager(gb_mixed* m, double* phi, const double* rho,
                                     void* stream) {
    if (!m || !phi || !rho) return fail(GB_EINVAL, "mixed vcycle: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)m->op64->ng() * sizeof(double);
    GB_CUDA_TRY(cudaMemcpyAsync(m->rho0, rho, bytes, cudaMemcpyDeviceToDevice, st));
    GB_CUDA_TRY(cudaMemcpyAsync(m->phi0, phi, bytes, cudaMemcpyDeviceToDevice, st));
    if (int rc = defect(m, st)) return rc;
    if (int rc = vcycle32(m, 0, st)) return rc;
    if (int rc = defect(m, st)) return rc;
    GB_CUDA_TRY(cudaMemcpyAsync(phi, m->phi0, bytes, cudaMemcpyDeviceToDevice, st));
    return 0;
}

extern "C" int gb_mixed_solve(gb_mixed* m, double* phi, const double* rho, double tol,
                              int maxiter, int* niter, double* rel_residual, void* stream) {
    if (int rc = gb_mixed_solve_async(m, phi, rho, tol, maxiter, stream)) return rc;
    GB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return gb_mixed_result(m, niter, rel_residual);
}

// --------------------------------------------------------------- batches
// Many mixed-precision solves (grids of any sizes) as ONE CUDA graph:
//   copy-in kernel (every solver's phi and rho into its buffers)
//   -> per solver a branch  |rho|^2 -> init -> defect -> check ->
//      WHILE { V-cycle; defect; check } -> control block to the host
//   -> copy-out kernel (every phi back)
// The branches are independent, so the graph runs the solves concurrently;
// one launch replaces a stream of per-solve launches.  The caller's array
// addresses live in a device table that one copy refreshes before each
// launch.
struct gb_mixed_batch {
    std::vector<gb_mixed*> s;
    double tol = 0.0;
    int maxiter = 0;
    int n = 0;
    double** d_user = nullptr;     // [2n]: phi_i, rho_i (caller's arrays)
    double** h_user = nullptr;     // pinned host copy of the table
    double** d_own = nullptr;      // [2n]: phi0_i, rho0_i (solver buffers)
    long long* d_len = nullptr;    // [n] points of grid i
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~gb_mixed_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (cap) cudaStreamDestroy(cap);
        cudaFree(d_user);
        cudaFree(d_own);
        cudaFree(d_len);
        if (h_user) cudaFreeHost(h_user);
    }
};

namespace {

// in: phi0_i = phi_i, rho0_i = rho_i; out: phi_i = phi0_i (blockIdx.y = i)
__global__ void k_batch_copy(int n, double* const* user, double* const* own,
                             const long long* len, int out) {
    const int i = blockIdx.y;
    if (i >= n) return;
    const long long m = len[i];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long j0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (out) {
        double* dst = user[2 * i];
        const double* src = own[2 * i];
        for (long long j = j0; j < m; j += stride) dst[j] = src[j];
    } else {
        for (int k = 0; k < 2; k++) {
            double* dst = own[2 * i + k];
            const double* src = user[2 * i + k];
            for (long long j = j0; j < m; j += stride) dst[j] = src[j];
        }
    }
}

// the single node a capture has produced since its last dependency set
int capture_tail(cudaStream_t cs, cudaGraphNode_t* tail) {
    cudaStreamCaptureStatus stat;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    GB_CUDA_TRY(cudaStreamGetCaptureInfo(cs, &stat, nullptr, nullptr, &deps, &ndeps));
    if (stat != cudaStreamCaptureStatusActive || ndeps != 1)
        return fail(GB_ECUDA, "mixed batch: unexpected capture state (%zu tail nodes)", ndeps);
    *tail = deps[0];
    return 0;
}

// one solver's branch after `root`; *wnode receives its WHILE node
int add_branch(gb_mixed_batch* bt, cudaGraph_t G, gb_mixed* m, cudaGraphNode_t root,
               cudaGraphNode_t* wnode) {
    cudaStream_t cs = bt->cap;
    const long long n = m->op64->ng();
    cudaGraphConditionalHandle h;
    GB_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, G, 0, 0));
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, G, &root, nullptr, 1,
                                              cudaStreamCaptureModeThreadLocal));
    const int nb = (int)std::min<long long>(1024, (n + 255) / 256);
    k_sumsq<<<nb, 256, 0, cs>>>(m->rho0, n, m->partial);
    launch_reduce_partials(m->partial, nb, 1, 1.0, m->nrm + 1, cs);
    k_mixed_init<<<1, 1, 0, cs>>>(m->ctl, m->nrm + 1, bt->tol, bt->maxiter);
    int rc = defect(m, cs);
    if (!rc) k_mixed_check<<<1, 1, 0, cs>>>(m->ctl, m->nrm, 0, h);
    cudaGraphNode_t tail = nullptr;
    if (!rc) rc = capture_tail(cs, &tail);
    cudaGraph_t gout = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cs, &gout);
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(GB_ECUDA, "mixed batch: capture: %s", cudaGetErrorString(ce));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    GB_CUDA_TRY(cudaGraphAddNode(wnode, G, &tail, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GB_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    t_no_coop = true;
    rc = vcycle32(m, 0, cs);
    t_no_coop = false;
    if (!rc) rc = defect(m, cs);
    if (!rc) k_mixed_check<<<1, 1, 0, cs>>>(m->ctl, m->nrm, 1, h);
    ce = cudaStreamEndCapture(cs, &gout);
    if (rc) return rc;
    if (ce != cudaSuccess)
        return fail(GB_ECUDA, "mixed batch: capture of the V-cycle: %s", cudaGetErrorString(ce));
    cudaGraphNode_t co;
    GB_CUDA_TRY(cudaGraphAddMemcpyNode1D(&co, G, wnode, 1, m->ctl_host, m->ctl, sizeof(Ctl),
                                         cudaMemcpyDeviceToHost));
    return 0;
}

int build_batch(gb_mixed_batch* bt) {
    const int n = bt->n;
    long long maxlen = 0;
    std::vector<double*> own(2 * n);
    std::vector<long long> len(n);
    for (int i = 0; i < n; i++) {
        own[2 * i] = bt->s[i]->phi0;
        own[2 * i + 1] = bt->s[i]->rho0;
        len[i] = bt->s[i]->op64->ng();
        maxlen = std::max(maxlen, len[i]);
    }
    GB_CUDA_TRY(cudaMalloc(&bt->d_user, 2 * n * sizeof(double*)));
    GB_CUDA_TRY(cudaMalloc(&bt->d_own, 2 * n * sizeof(double*)));
    GB_CUDA_TRY(cudaMalloc(&bt->d_len, n * sizeof(long long)));
    GB_CUDA_TRY(cudaMallocHost(&bt->h_user, 2 * n * sizeof(double*)));
    GB_CUDA_TRY(cudaMemcpy(bt->d_own, own.data(), 2 * n * sizeof(double*),
                           cudaMemcpyHostToDevice));
    GB_CUDA_TRY(cudaMemcpy(bt->d_len, len.data(), n * sizeof(long long),
                           cudaMemcpyHostToDevice));
    cudaGraph_t G;
    GB_CUDA_TRY(cudaGraphCreate(&G, 0));
    const dim3 cgrid((unsigned)std::min<long long>(64, (maxlen + 255) / 256), (unsigned)n);
    cudaStream_t cs = bt->cap;
    int rc = 0;
    cudaGraphNode_t root = nullptr;
    std::vector<cudaGraphNode_t> whiles(n);
    cudaError_t ce = cudaStreamBeginCaptureToGraph(cs, G, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
        k_batch_copy<<<cgrid, 256, 0, cs>>>(n, bt->d_user, bt->d_own, bt->d_len, 0);
        rc = capture_tail(cs, &root);
        cudaGraph_t gout = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &gout);
        if (!rc && e2 != cudaSuccess)
            rc = fail(GB_ECUDA, "mixed batch: capture: %s", cudaGetErrorString(e2));
    } else {
        rc = fail(GB_ECUDA, "mixed batch: capture: %s", cudaGetErrorString(ce));
    }
    for (int i = 0; i < n && !rc; i++) rc = add_branch(bt, G, bt->s[i], root, &whiles[i]);
    if (!rc) {
        ce = cudaStreamBeginCaptureToGraph(cs, G, whiles.data(), nullptr, n,
                                           cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
            k_batch_copy<<<cgrid, 256, 0, cs>>>(n, bt->d_user, bt->d_own, bt->d_len, 1);
            cudaGraph_t gout = nullptr;
            ce = cudaStreamEndCapture(cs, &gout);
        }
        if (ce != cudaSuccess)
            rc = fail(GB_ECUDA, "mixed batch: capture: %s", cudaGetErrorString(ce));
    }
    if (!rc) {
        ce = cudaGraphInstantiate(&bt->exec, G, 0);
        if (ce != cudaSuccess)
            rc = fail(GB_ECUDA, "mixed batch: instantiate: %s", cudaGetErrorString(ce));
    }
    cudaGraphDestroy(G);
    return rc;
}

}  // namespace

extern "C" int gb_mixed_batch_new(int n, gb_mixed* const* solvers, double tol, int maxiter,
                                  gb_mixed_batch** out) {
    if (!out || !solvers || n < 1) return fail(GB_EINVAL, "mixed batch: bad arguments");
    if (maxiter < 1) return fail(GB_EINVAL, "mixed batch: maxiter must be >= 1");
    if (n > 65535) return fail(GB_EINVAL, "mixed batch: at most 65535 solvers");
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!solvers[i]) return fail(GB_EINVAL, "mixed batch: NULL solver %d", i);
        for (int j = 0; j < i; j++)
            if (solvers[j] == solvers[i])
                return fail(GB_EINVAL, "mixed batch: solver %d appears twice", i);
        // one uncaptured pass of every kernel (sets kernel attributes)
        if (!solvers[i]->exec)
            if (int rc = build_mixed_graph(solvers[i])) return rc;
    }
    gb_mixed_batch* bt = new gb_mixed_batch();
    bt->tol = tol;
    bt->maxiter = maxiter;
    bt->n = n;
    bt->s.assign(solvers, solvers + n);
    cudaError_t e = cudaStreamCreateWithFlags(&bt->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete bt;
        return fail(GB_ECUDA, "mixed batch: stream: %s", cudaGetErrorString(e));
    }
    if (int rc = build_batch(bt)) {
        delete bt;
        return rc;
    }
    *out = bt;
    return 0;
}

extern "C" void gb_mixed_batch_free(gb_mixed_batch* bt) { delete bt; }

extern "C" int gb_mixed_batch_solve_async(gb_mixed_batch* bt, double* const* phis,
                                          const double* const* rhos, void* stream) {
    if (!bt || !phis || !rhos) return fail(GB_EINVAL, "mixed batch solve: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    // the previous launch on this stream may still read the table
    GB_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < bt->n; i++) {
        if (!phis[i] || !rhos[i]) return fail(GB_EINVAL, "mixed batch solve: NULL array %d", i);
        bt->h_user[2 * i] = phis[i];
        bt->h_user[2 * i + 1] = const_cast<double*>(rhos[i]);
        bt->s[i]->last_tol = bt->tol;
        bt->s[i]->last_maxiter = bt->maxiter;
    }
    GB_CUDA_TRY(cudaMemcpyAsync(bt->d_user, bt->h_user, 2 * bt->n * sizeof(double*),
                                cudaMemcpyHostToDevice, st));
    GB_CUDA_TRY(cudaGraphLaunch(bt->exec, st));
    return 0;
}

extern "C" int gb_mixed_batch_result(gb_mixed_batch* bt, int* niters, double* rel_residuals) {
    if (!bt) return fail(GB_EINVAL, "mixed batch result: NULL batch");
    int bad = -1;
    for (int i = 0; i < bt->n; i++) {
        const Ctl* c = bt->s[i]->ctl_host;
        if (niters) niters[i] = c->niter;
        if (rel_residuals) rel_residuals[i] = c->rel;
        if (c->rel > bt->tol && bad < 0) bad = i;
    }
    if (bad >= 0)
        return fail(GB_ENOCONV, "mixed batch: solve %d did not reach %g in %d V-cycles", bad,
                    bt->tol, bt->maxiter);
    return 0;
}
