// Weighted finite-difference operator: A = sum_i w_i(x) L_i with per-point
// weights (cgpaw.WOperator, c/woperators.cpp; bmgs_wfd / bmgs_wfdz,
// c/bmgs/wfd.cpp; bmgs_wrelax, c/bmgs/wrelax.cpp).  The dielectric Poisson
// solver of the solvation model builds it from a Laplacian and the three
// gradients with weights eps, d_x eps, d_y eps, d_z eps.
//
// Axis-aligned operators (the solvation solver's) take a plane-marching
// kernel with every tap a shared-memory read; others one thread per grid
// point reading through L1.  Every operator's inner sum starts from 0 and
// adds c_p v(x + o_p) in coefficient order (each product and sum rounded
// on its own), is scaled by its weight, and is added to the total, as the
// reference's loops do, so results are bit-identical to them.  Values off
// the grid come from the same boundary read as the plain operator (zero,
// or wrapped with the Bloch phase; corners zero when every operator is
// axis-aligned, as bc_unpack leaves them for cfd = 1).
#include <cstdlib>
#include <cstring>

#include "gb_objects.cuh"

using namespace gb;

namespace gb {

constexpr int GB_MAX_WCOEFS = 256;

struct WStencil {
    int nw;
    int range;
    int cfd;
    int ncoefs[GB_MAX_WEIGHTS];
    int start[GB_MAX_WEIGHTS];   // first coefficient of operator i
    const double* w[GB_MAX_WEIGHTS];
    double coef[GB_MAX_WCOEFS];
    int off[GB_MAX_WCOEFS][3];
    long long flat[GB_MAX_WCOEFS];
};

template <class T>
__device__ __forceinline__ T wread(const T* __restrict__ a, int p, int i0, int i1, int i2, bool inner,
                                   const GridBC& g, const Phases& P, const WStencil& s, int c) {
    if (inner) return __ldg(a + p + s.flat[c]);
    return bc_read<T>(a, i0 + s.off[c][0], i1 + s.off[c][1], i2 + s.off[c][2], g, P, !s.cfd);
}

// out = sum_i w_i (sum_p c_ip in(x + o_ip))   (bmgs_wfd, c/bmgs/wfd.cpp:10-40)
template <class T>
__global__ void __launch_bounds__(256)
k_wfd(const T* __restrict__ in, T* __restrict__ out, int nin, GridBC g, Phases P,
      const __grid_constant__ WStencil s) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int ng = n0 * n1 * n2;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ng) return;
    const int i2 = p % n2;
    const int t = p / n2;
    const int i1 = t % n1;
    const int i0 = t / n1;
    const int r = s.range;
    const bool inner = i0 >= r && i0 + r < n0 && i1 >= r && i1 + r < n1 && i2 >= r && i2 + r < n2;
    for (int b = blockIdx.y; b < nin; b += gridDim.y) {
        const T* a = in + (long long)b * ng;
        T x = Num<T>::zero();
        for (int iw = 0; iw < s.nw; iw++) {
            T tmp = Num<T>::zero();
            const int c0 = s.start[iw], c1 = c0 + s.ncoefs[iw];
            for (int c = c0; c < c1; c++)
                tmp = Num<T>::add(tmp, Num<T>::scale(wread<T>(a, p, i0, i1, i2, inner, g, P, s, c),
                                                     s.coef[c]));
            tmp = Num<T>::scale(tmp, __ldg(s.w[iw] + p));
            x = Num<T>::add(x, tmp);
        }
        out[(long long)b * ng + p] = x;
    }
}

// ---------------------------------------------------------------- tiled apply
// Axis-aligned weighted operators (every offset on one axis, range R):
// one CTA owns a WX x WY column tile and a chunk of planes along axis 0.
// Plane tiles (the tile plus an R-wide halo on its four sides; corners are
// never read) stream through a ring of S shared-memory stages by cp.async,
// S - (2R + 1) planes ahead; S is a power of two, so the stage of any tap's
// plane is (centre + o0) & (S - 1).  Every tap is then a shared-memory
// read, and the sums keep the order of k_wfd.  Wrapped values carry their
// Bloch phase: in-plane halo cells are multiplied right after they land,
// a whole plane wrapped along axis 0 by that axis's phase (only its tile
// columns are read, as axis-0 neighbours).
constexpr int WX = 32, WY = 8;

__device__ __forceinline__ bool wwrap(int& y, int n, int periodic) {
    if (y >= 0 && y < n) return true;
    if (!periodic) return false;
    y += (y < 0) ? n : -n;
    return y >= 0 && y < n;
}

template <int BYTES>
__device__ __forceinline__ void wcp_async(unsigned sdst, const void* gsrc, bool valid) {
    const int n = valid ? BYTES : 0;   // 0: zero fill, nothing is read
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(gsrc),
                     "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sdst), "l"(gsrc),
                     "r"(n));
}

// Structured form of an operator list whose every operator is a centre
// tap followed by groups of 2R taps along one axis, +1..+R then -1..-R
// (the Laplacians and gradients of orthorhombic cells): the tap positions
// are then compile-time offsets from the centre, and only the axis of each
// group and the coefficients are data.
struct WGroups {
    int ng[GB_MAX_WEIGHTS];               // groups of operator i (0..3)
    int axis[GB_MAX_WEIGHTS][3];
    double c0[GB_MAX_WEIGHTS];
    double cp[GB_MAX_WEIGHTS][3][6];      // coefficient of +d, d = 1..R
    double cm[GB_MAX_WEIGHTS][3][6];      // coefficient of -d
};

// MODE 0: the apply.  MODE 1 (real data): one weighted-Jacobi sweep, out =
// (1 - wj) in + (wj (rhs - x)) / d with x the off-diagonal part and d the
// diagonal of the weighted operator at the point, each operator's inner sum
// and the accumulation in bmgs_wrelax's order (c/bmgs/wrelax.cpp:71-86),
// the same arithmetic as k_wjacobi.
// GR: 0 = tap tables, 1 = structured groups, 2 = structured groups of
// exactly four operators (the solvation operator), with every operator and
// group loop unrolled so that each coefficient is a compile-time operand and
// the four weights are loaded before the taps.
template <class T, int R, int S, int GR, int MODE>
__global__ void __launch_bounds__(WX * WY)
k_wfd_tiled(const T* __restrict__ in, T* __restrict__ out, int nin, GridBC g, Phases P,
            const __grid_constant__ WStencil s, const __grid_constant__ WGroups G, int chunk0,
            int tiles_x, const double* __restrict__ rhs, double wj) {
    constexpr int PX = WX + 2 * R, PY = WY + 2 * R, PL = PX * PY;
    constexpr int NT = WX * WY;
    constexpr int D = S - (2 * R + 1);          // planes in flight
    constexpr int NMID = PY * WX, NSIDE = WY * 2 * R;
    constexpr int NC = (NMID + NSIDE + NT - 1) / NT;
    constexpr int EB = (int)sizeof(T);
    static_assert(D >= 1 && (S & (S - 1)) == 0, "ring depth");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ring = reinterpret_cast<T*>(smem_raw);

    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int x0 = (blockIdx.x % tiles_x) * WX;
    const int y0 = (blockIdx.x / tiles_x) * WY;
    const int pa = blockIdx.y * chunk0;
    const int pb = min(n0, pa + chunk0);
    const int b = blockIdx.z;
    if (pa >= pb || b >= nin) return;
    const int tid = threadIdx.x;
    const long long ng = (long long)n0 * n1 * n2;
    const long long pstride = (long long)n1 * n2;
    const T* a = in + b * ng;
    T* o = out + b * ng;
    const int tx = tid % WX, ty = tid / WX;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool own = gx < n2 && gy < n1;

    // this thread's copy cells: stage offset, in-plane source offset,
    // validity and in-plane phase code (0 none, 1/2 axis 1 high/low,
    // 3/4 axis 2 high/low)
    int soff[NC], goff[NC];
    unsigned vmask = 0, wcode = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const int e = tid + i * NT;
        soff[i] = 0;
        goff[i] = 0;
        if (e >= NMID + NSIDE) continue;
        int ry, rx;
        if (e < NMID) {
            ry = e / WX - R;
            rx = e % WX;
        } else {
            const int f = e - NMID;
            ry = f / (2 * R);
            const int c = f % (2 * R);
            rx = c < R ? c - R : WX + c - R;
        }
        soff[i] = (ry + R) * PX + (rx + R);
        int y = y0 + ry, x = x0 + rx;
        const bool yw = y < 0 || y >= n1, xw = x < 0 || x >= n2;
        const int ys = y < 0, xs = x < 0;
        if (wwrap(y, n1, g.periodic[1]) && wwrap(x, n2, g.periodic[2])) {
            vmask |= 1u << i;
            goff[i] = y * n2 + x;
            unsigned c = 0;
            if (yw) c = 1 + ys;
            else if (xw) c = 3 + xs;
            wcode |= c << (3 * i);
        }
    }
    if (!P.use) wcode = 0;
    const unsigned ring_u = (unsigned)__cvta_generic_to_shared(ring);
    // relative plane j is absolute plane pa - R + j; it lives in stage j & (S-1)
    auto issue = [&](int j) {
        int pl = pa - R + j;
        const bool pv = wwrap(pl, n0, g.periodic[0]);
        const unsigned su = ring_u + (unsigned)((j & (S - 1)) * PL * EB);
        const T* src = a + pl * pstride;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= NMID + NSIDE) break;
            const bool ok = pv && ((vmask >> i) & 1);
            wcp_async<EB>(su + (unsigned)(soff[i] * EB), ok ? src + goff[i] : a, ok);
        }
    };
    auto fixup = [&](int j) {
        if constexpr (sizeof(T) == 16) {
            const int pl = pa - R + j;
            const bool zw = P.use && g.periodic[0] && (pl < 0 || pl >= n0);
            if (!wcode && !zw) return;
            const double2 ph0 = pl >= n0 ? P.ph[0][0] : P.ph[0][1];
            T* st = ring + (j & (S - 1)) * PL;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                if (tid + i * NT >= NMID + NSIDE) break;
                if (!((vmask >> i) & 1)) continue;
                const unsigned c = (wcode >> (3 * i)) & 7u;
                if (c == 0 && !zw) continue;
                T v = st[soff[i]];
                if (c) v = cmul(c == 1 ? P.ph[1][0] : c == 2 ? P.ph[1][1]
                                : c == 3 ? P.ph[2][0] : P.ph[2][1], v);
                if (zw) v = cmul(ph0, v);
                st[soff[i]] = v;
            }
        }
    };

    const int nplanes = pb - pa;
    const int total = nplanes + 2 * R;     // relative planes 0 .. total-1
#pragma unroll 1
    for (int j = 0; j < D; j++) {
        if (j < total) issue(j);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    // the stencil tables in shared memory (read by every thread at the same
    // address: broadcasts): per tap its plane offset o0, its in-plane
    // offset o1 * PX + o2 and its coefficient
    __shared__ double sh_coef[GB_MAX_WCOEFS];
    __shared__ int sh_o0[GB_MAX_WCOEFS], sh_ip[GB_MAX_WCOEFS];
    const int ntap = s.start[s.nw - 1] + s.ncoefs[s.nw - 1];
    for (int c = tid; c < ntap; c += NT) {
        sh_coef[c] = s.coef[c];
        sh_o0[c] = s.off[c][0];
        sh_ip[c] = s.off[c][1] * PX + s.off[c][2];
    }
    const int cen = (ty + R) * PX + (tx + R);
    // GR == 2: the weights (and the Jacobi source) of the next centre plane,
    // loaded a plane ahead so that their latency overlaps a plane's taps
    double wn[4] = {0.0, 0.0, 0.0, 0.0}, rn = 0.0;
    auto fetch = [&](int pp) {
        if (GR == 2 && own && pp < pb) {
            const long long a2 = pp * pstride + (long long)gy * n2 + gx;
#pragma unroll
            for (int iw = 0; iw < 4; iw++) wn[iw] = __ldg(s.w[iw] + a2);
            if (MODE == 1) rn = __ldg(rhs + a2);
        }
    };
    fetch(pa);
#pragma unroll 1
    for (int t = 0; t < total; t++) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(D - 1));
        fixup(t);
        __syncthreads();
        if (t + D < total) issue(t + D);
        asm volatile("cp.async.commit_group;\n" ::);
        if (t < 2 * R) continue;
        const int cj = t - R;                  // relative centre plane
        const int p = pa + cj - R;             // absolute centre plane
        if (!own) continue;
        const long long at = p * pstride + (long long)gy * n2 + gx;
        T x = Num<T>::zero();
        double dg = 0.0;     // MODE 1: the diagonal sum_i w_i c_i0
        double src = 0.0;    // MODE 1: the source term at the point
        if constexpr (GR >= 1) {
            const T* c = ring + (cj & (S - 1)) * PL + cen;
            // one operator's term: inner sum from zero in coefficient order,
            // scaled by its weight, added to the total (bmgs_wfd's order)
            // one operator's term: inner sum from zero in coefficient order,
            // scaled by its weight, added to the total (bmgs_wfd's order).
            // Every tap is a shared-memory read: holding the 6 R neighbours
            // in registers for the four operators to share measured slower
            // (79-90 registers, half the CTAs an SM).
            auto term = [&](int iw, double weight) {
                T tmp = Num<T>::zero();
                if (MODE == 0) tmp = Num<T>::add(tmp, Num<T>::scale(c[0], G.c0[iw]));
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (k >= G.ng[iw]) break;
                    const int ax = G.axis[iw][k];
                    if (ax == 0) {
#pragma unroll
                        for (int d = 1; d <= R; d++)
                            tmp = Num<T>::add(tmp, Num<T>::scale(
                                ring[((cj + d) & (S - 1)) * PL + cen], G.cp[iw][k][d - 1]));
#pragma unroll
                        for (int d = 1; d <= R; d++)
                            tmp = Num<T>::add(tmp, Num<T>::scale(
                                ring[((cj - d) & (S - 1)) * PL + cen], G.cm[iw][k][d - 1]));
                    } else {
                        const int sd = ax == 1 ? PX : 1;
#pragma unroll
                        for (int d = 1; d <= R; d++)
                            tmp = Num<T>::add(tmp, Num<T>::scale(c[d * sd], G.cp[iw][k][d - 1]));
#pragma unroll
                        for (int d = 1; d <= R; d++)
                            tmp = Num<T>::add(tmp, Num<T>::scale(c[-d * sd], G.cm[iw][k][d - 1]));
                    }
                }
                tmp = Num<T>::scale(tmp, weight);
                x = Num<T>::add(x, tmp);
                if (MODE == 1) dg = __dadd_rn(dg, __dmul_rn(weight, G.c0[iw]));
            };
            if constexpr (GR == 2) {
                double wv[4];
#pragma unroll
                for (int iw = 0; iw < 4; iw++) wv[iw] = wn[iw];
                src = rn;
                fetch(p + 1);
#pragma unroll
                for (int iw = 0; iw < 4; iw++) term(iw, wv[iw]);
            } else {
                for (int iw = 0; iw < s.nw; iw++) term(iw, __ldg(s.w[iw] + at));
            }
        } else {
            for (int iw = 0; iw < s.nw; iw++) {
                T tmp = Num<T>::zero();
                const int c0 = s.start[iw], c1 = c0 + s.ncoefs[iw];
#pragma unroll 4
                for (int c = c0 + MODE; c < c1; c++) {
                    const T v = ring[((cj + sh_o0[c]) & (S - 1)) * PL + cen + sh_ip[c]];
                    tmp = Num<T>::add(tmp, Num<T>::scale(v, sh_coef[c]));
                }
                const double weight = __ldg(s.w[iw] + at);
                tmp = Num<T>::scale(tmp, weight);
                x = Num<T>::add(x, tmp);
                if (MODE == 1) dg = __dadd_rn(dg, __dmul_rn(weight, sh_coef[c0]));
            }
        }
        if constexpr (MODE == 1 && sizeof(T) == 8) {
            const double old = ring[(cj & (S - 1)) * PL + cen];
            if constexpr (GR != 2) src = rhs[at];
            o[at] = __dadd_rn(__dmul_rn(1.0 - wj, old),
                              __ddiv_rn(__dmul_rn(wj, __dsub_rn(src, x)), dg));
        } else {
            o[at] = x;
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// Off-diagonal part and diagonal of the weighted operator at point p:
// x = sum_i w_i (sum_{p>0} c_ip a(x + o_ip)),  d = sum_i w_i c_i0
// (bmgs_wrelax's inner loops, c/bmgs/wrelax.cpp:33-48 and 71-86)
__device__ __forceinline__ void wrelax_terms(const double* __restrict__ a, int p, int i0, int i1,
                                             int i2, bool inner, const GridBC& g,
                                             const WStencil& s, double& x, double& d) {
    const Phases P{};
    x = 0.0;
    d = 0.0;
    for (int iw = 0; iw < s.nw; iw++) {
        const double weight = __ldg(s.w[iw] + p);
        double tmp = 0.0;
        const int c0 = s.start[iw], c1 = c0 + s.ncoefs[iw];
        for (int c = c0 + 1; c < c1; c++)
            tmp = __dadd_rn(tmp, __dmul_rn(wread<double>(a, p, i0, i1, i2, inner, g, P, s, c),
                                           s.coef[c]));
        tmp = __dmul_rn(tmp, weight);
        x = __dadd_rn(x, tmp);
        d = __dadd_rn(d, __dmul_rn(weight, s.coef[c0]));
    }
}

// weighted Jacobi: nw = (1 - w) old + w (src - x) / d, neighbours from old
__global__ void __launch_bounds__(256)
k_wjacobi(const double* __restrict__ old, double* __restrict__ nw, const double* __restrict__ src,
          GridBC g, const __grid_constant__ WStencil s, double w) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n0 * n1 * n2) return;
    const int i2 = p % n2;
    const int t = p / n2;
    const int i1 = t % n1;
    const int i0 = t / n1;
    const int r = s.range;
    const bool inner = i0 >= r && i0 + r < n0 && i1 >= r && i1 + r < n1 && i2 >= r && i2 + r < n2;
    double x, d;
    wrelax_terms(old, p, i0, i1, i2, inner, g, s, x, d);
    nw[p] = __dadd_rn(__dmul_rn(1.0 - w, old[p]),
                      __ddiv_rn(__dmul_rn(w, __dsub_rn(src[p], x)), d));
}

// One wavefront of weighted Gauss-Seidel (points with wa i0 + wb i1 + i2 =
// t): neighbours inside the grid are read live, wrapped ones from the
// sweep's starting copy `snap`, as the reference's padded buffer holds them.
__global__ void __launch_bounds__(256)
k_wgs_wave(double* __restrict__ f, const double* __restrict__ snap, const double* __restrict__ src,
           GridBC g, const __grid_constant__ WStencil s, int t, int wa, int wb) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n0 * n1) return;
    const int i1 = q % n1;
    const int i0 = q / n1;
    const int i2 = t - wa * i0 - wb * i1;
    if (i2 < 0 || i2 >= n2) return;
    const int p = (i0 * n1 + i1) * n2 + i2;
    const Phases P{};
    double x = 0.0, d = 0.0;
    for (int iw = 0; iw < s.nw; iw++) {
        const double weight = s.w[iw][p];
        double tmp = 0.0;
        const int c0 = s.start[iw], c1 = c0 + s.ncoefs[iw];
        for (int c = c0 + 1; c < c1; c++) {
            const int y0 = i0 + s.off[c][0], y1 = i1 + s.off[c][1], y2 = i2 + s.off[c][2];
            double v;
            if (y0 >= 0 && y0 < n0 && y1 >= 0 && y1 < n1 && y2 >= 0 && y2 < n2)
                v = f[(y0 * n1 + y1) * n2 + y2];
            else
                v = bc_read<double>(snap, y0, y1, y2, g, P, !s.cfd);
            tmp = __dadd_rn(tmp, __dmul_rn(v, s.coef[c]));
        }
        tmp = __dmul_rn(tmp, weight);
        x = __dadd_rn(x, tmp);
        d = __dadd_rn(d, __dmul_rn(weight, s.coef[c0]));
    }
    f[p] = __ddiv_rn(__dsub_rn(src[p], x), d);
}

// max over points of |sum_i w_i c_i0| (c/woperators.cpp:372-398); the
// non-negative doubles order like their bit patterns, so an integer
// atomicMax on the bits gives the maximum
__global__ void __launch_bounds__(256)
k_wdiag(int ng, const __grid_constant__ WStencil s, unsigned long long* out) {
    double m = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ng; p += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int iw = 0; iw < s.nw; iw++) d = __dadd_rn(d, __dmul_rn(s.w[iw][p], s.coef[s.start[iw]]));
        if (d < 0) d = -d;
        if (d > m) m = d;
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace gb

struct gb_woperator {
    WStencil s;
    GridBC g;
    int real;
    Scratch scratch;
    unsigned long long* diag_dev = nullptr;
    ~gb_woperator() {
        if (diag_dev) cudaFree(diag_dev);
    }
    long long ng() const { return (long long)g.n[0] * g.n[1] * g.n[2]; }
};

namespace gb {
// Tiled apply for axis-aligned operators of range 1..6 (complex: 1..3);
// -1 when the operator does not qualify (the gather kernel runs instead).
// The structured form of s for range R, if every operator has it.
static bool wfd_groups(const WStencil& s, int R, WGroups& G) {
    if (R < 1 || R > 6) return false;
    memset(&G, 0, sizeof G);
    for (int iw = 0; iw < s.nw; iw++) {
        const int c0 = s.start[iw], n = s.ncoefs[iw];
        if (s.off[c0][0] || s.off[c0][1] || s.off[c0][2]) return false;
        if ((n - 1) % (2 * R) != 0 || (n - 1) / (2 * R) > 3) return false;
        G.c0[iw] = s.coef[c0];
        G.ng[iw] = (n - 1) / (2 * R);
        for (int k = 0; k < G.ng[iw]; k++) {
            const int base = c0 + 1 + k * 2 * R;
            int ax = -1;
            for (int a = 0; a < 3; a++)
                if (s.off[base][a]) ax = a;
            if (ax < 0) return false;
            for (int d = 1; d <= R; d++) {
                const int ip = base + d - 1, im = base + R + d - 1;
                for (int a = 0; a < 3; a++) {
                    if (s.off[ip][a] != (a == ax ? d : 0)) return false;
                    if (s.off[im][a] != (a == ax ? -d : 0)) return false;
                }
                G.cp[iw][k][d - 1] = s.coef[ip];
                G.cm[iw][k][d - 1] = s.coef[im];
            }
            G.axis[iw][k] = ax;
        }
    }
    return true;
}

template <class T, int R, int S, int GR, int MODE>
static int launch_wfd_tiled_k(const void* in, void* out, int nin, const GridBC& g,
                              const Phases& P, const WStencil& s, const WGroups& G,
                              cudaStream_t st, const double* rhs, double wj) {
    constexpr size_t smem = (size_t)S * (WX + 2 * R) * (WY + 2 * R) * sizeof(T);
    static bool attr_done = false;
    if (!attr_done) {
        if (cudaFuncSetAttribute(k_wfd_tiled<T, R, S, GR, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return -2;
        attr_done = true;
    }
    const int tiles_x = (g.n[2] + WX - 1) / WX;
    const int tiles_y = (g.n[1] + WY - 1) / WY;
    const int chunk0 = cfd_chunk(g, R, nin, WY);
    const int nch = (g.n[0] + chunk0 - 1) / chunk0;
    const long long ng = (long long)g.n[0] * g.n[1] * g.n[2];
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(tiles_x * tiles_y, nch, nb);
        k_wfd_tiled<T, R, S, GR, MODE><<<grid, WX * WY, smem, st>>>(
            (const T*)in + b0 * ng, (T*)out + b0 * ng, nb, g, P, s, G, chunk0, tiles_x, rhs, wj);
    }
    return 0;
}

template <class T, int R, int S, int MODE>
static int launch_wfd_tiled_rs(const void* in, void* out, int nin, const GridBC& g,
                               const Phases& P, const WStencil& s, cudaStream_t st,
                               const double* rhs, double wj) {
    WGroups G;
    if (wfd_groups(s, R, G)) {
        if (s.nw == 4)
            return launch_wfd_tiled_k<T, R, S, 2, MODE>(in, out, nin, g, P, s, G, st, rhs, wj);
        return launch_wfd_tiled_k<T, R, S, 1, MODE>(in, out, nin, g, P, s, G, st, rhs, wj);
    }
    return launch_wfd_tiled_k<T, R, S, 0, MODE>(in, out, nin, g, P, s, G, st, rhs, wj);
}

// MODE 1 (weighted Jacobi, real data): `rhs` the source term, `wj` the
// relaxation weight.
template <class T, int MODE = 0>
static int launch_wfd_tiled(const void* in, void* out, int nin, const GridBC& g,
                            const Phases& P, const WStencil& s, cudaStream_t st,
                            const double* rhs = nullptr, double wj = 0.0) {
    if (!s.cfd) return -1;
    const int nc = s.start[s.nw - 1] + s.ncoefs[s.nw - 1];
    for (int c = 0; c < nc; c++) {
        int nz = 0;
        for (int k = 0; k < 3; k++) nz += s.off[c][k] != 0;
        if (nz > 1) return -1;
    }
    switch (s.range) {
        case 1: return launch_wfd_tiled_rs<T, 1, 4, MODE>(in, out, nin, g, P, s, st, rhs, wj);
        case 2: return launch_wfd_tiled_rs<T, 2, 8, MODE>(in, out, nin, g, P, s, st, rhs, wj);
        case 3: return launch_wfd_tiled_rs<T, 3, 8, MODE>(in, out, nin, g, P, s, st, rhs, wj);
    }
    if constexpr (sizeof(T) == 8) {
        switch (s.range) {
            case 4: return launch_wfd_tiled_rs<T, 4, 16, MODE>(in, out, nin, g, P, s, st, rhs, wj);
            case 5: return launch_wfd_tiled_rs<T, 5, 16, MODE>(in, out, nin, g, P, s, st, rhs, wj);
            case 6: return launch_wfd_tiled_rs<T, 6, 16, MODE>(in, out, nin, g, P, s, st, rhs, wj);
        }
    }
    return -1;
}

}  // namespace gb

extern "C" int gb_woperator_new(int nweights, const double* const* weights,
                                const double* const* coefs, const int64_t* const* offsets,
                                const int* ncoefs, const int64_t size[3], int range,
                                const int64_t neighbors[6], int real, int cfd,
                                gb_woperator** out) {
    if (!out || !weights || !coefs || !offsets || !ncoefs || !size || !neighbors)
        return fail(GB_EINVAL, "WOperator: NULL argument");
    *out = nullptr;
    if (nweights < 1 || nweights > GB_MAX_WEIGHTS)
        return fail(GB_EINVAL, "WOperator: %d weights (1..%d supported)", nweights, GB_MAX_WEIGHTS);
    if (range < 0) return fail(GB_EINVAL, "WOperator: negative range");
    for (int c = 0; c < 3; c++)
        if (size[c] < 1 || size[c] > (1 << 20)) return fail(GB_EINVAL, "WOperator: bad size");
    if ((double)size[0] * size[1] * size[2] >= 2147483647.0)
        return fail(GB_EINVAL, "WOperator: grid has 2^31 points or more");
    gb_woperator* op = new gb_woperator();
    memset(&op->s, 0, sizeof op->s);
    op->s.nw = nweights;
    op->s.range = range;
    op->s.cfd = cfd ? 1 : 0;
    op->real = real ? 1 : 0;
    for (int c = 0; c < 3; c++) {
        const int64_t lo = neighbors[2 * c], hi = neighbors[2 * c + 1];
        if (lo > 0 || hi > 0 || (lo == 0) != (hi == 0)) {
            delete op;
            return fail(GB_EINVAL, "WOperator: single-domain neighbours only");
        }
        op->g.n[c] = (int)size[c];
        op->g.periodic[c] = lo == 0 ? 1 : 0;
        if (op->g.periodic[c] && size[c] < range) {
            delete op;
            return fail(GB_EINVAL, "Stencil longer than domain");
        }
    }
    int k = 0;
    for (int iw = 0; iw < nweights; iw++) {
        if (!weights[iw] || !coefs[iw] || !offsets[iw] || ncoefs[iw] < 1) {
            delete op;
            return fail(GB_EINVAL, "WOperator: operator %d is empty", iw);
        }
        if (offsets[iw][0] != 0) {
            delete op;
            return fail(GB_EINVAL, "WOperator: operator %d does not start at offset 0", iw);
        }
        if (k + ncoefs[iw] > GB_MAX_WCOEFS) {
            delete op;
            return fail(GB_EINVAL, "WOperator: more than %d coefficients in all", GB_MAX_WCOEFS);
        }
        op->s.w[iw] = weights[iw];
        op->s.start[iw] = k;
        op->s.ncoefs[iw] = ncoefs[iw];
        for (int p = 0; p < ncoefs[iw]; p++, k++) {
            int o[3];
            if (!split_offset(offsets[iw][p], size, range, o)) {
                delete op;
                return fail(GB_EINVAL, "WOperator: offset %lld does not fit range %d",
                            (long long)offsets[iw][p], range);
            }
            op->s.coef[k] = coefs[iw][p];
            for (int c = 0; c < 3; c++) op->s.off[k][c] = o[c];
            op->s.flat[k] = ((long long)o[0] * size[1] + o[1]) * size[2] + o[2];
        }
    }
    *out = op;
    return 0;
}

extern "C" void gb_woperator_free(gb_woperator* op) { delete op; }

extern "C" int gb_woperator_apply(gb_woperator* op, const void* in, void* out, int64_t nin,
                                  int dtype, const double* phases, void* stream) {
    if (!op || !in || !out) return fail(GB_EINVAL, "WOperator apply: NULL argument");
    if (dtype != GB_F64 && dtype != GB_C128) return fail(GB_EINVAL, "unsupported dtype %d", dtype);
    if ((dtype == GB_F64) != (op->real != 0))
        return fail(GB_EINVAL, "dtype does not match the operator (real=%d)", op->real);
    if (nin < 0) return fail(GB_EINVAL, "WOperator apply: negative batch");
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
    int rc = (dtype == GB_F64)
                 ? launch_wfd_tiled<double>(in, out, (int)nin, op->g, P, op->s, st)
                 : launch_wfd_tiled<double2>(in, out, (int)nin, op->g, P, op->s, st);
    if (rc == -2) return fail(GB_ECUDA, "WOperator: could not raise the shared-memory limit");
    if (rc == 0) {
        GB_LAUNCH_CHECK();
        return 0;
    }
    const int ng = (int)op->ng();
    const dim3 grid((unsigned)((ng + 255) / 256), (unsigned)(nin < 65535 ? nin : 65535));
    if (dtype == GB_F64)
        k_wfd<double><<<grid, 256, 0, st>>>((const double*)in, (double*)out, (int)nin, op->g, P,
                                            op->s);
    else
        k_wfd<double2><<<grid, 256, 0, st>>>((const double2*)in, (double2*)out, (int)nin, op->g,
                                             P, op->s);
    GB_LAUNCH_CHECK();
    return 0;
}

extern "C" int gb_woperator_relax(gb_woperator* op, int method, double* f, const double* s,
                                  int nrelax, double w, void* stream) {
    if (!op || !f || !s) return fail(GB_EINVAL, "WOperator relax: NULL argument");
    if (!op->real) return fail(GB_EINVAL, "WOperator relax: float64 operators only");
    if (method != 1 && method != 2) return fail(GB_EINVAL, "relax method must be 1 or 2");
    if (nrelax <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)op->ng() * sizeof(double);
    if (int e = op->scratch.ensure(bytes)) return e;
    double* X = (double*)op->scratch.ptr;
    const GridBC& g = op->g;
    if (method == 1) {
        // wavefronts: every neighbour earlier in the lexicographic order
        // lies on an earlier front (c/bmgs/wrelax.cpp:23-56)
        const int r = op->s.range;
        int wa = 1, wb = 1;
        if (!op->s.cfd) {
            wb = 2 * r + 1;
            wa = (wb + 1) * r + 1;
        }
        const int nt = wa * (g.n[0] - 1) + wb * (g.n[1] - 1) + g.n[2];
        const bool periodic = g.periodic[0] || g.periodic[1] || g.periodic[2];
        const int nq = g.n[0] * g.n[1];
        for (int it = 0; it < nrelax; it++) {
            if (periodic) GB_CUDA_TRY(cudaMemcpyAsync(X, f, bytes, cudaMemcpyDeviceToDevice, st));
            for (int t = 0; t < nt; t++)
                k_wgs_wave<<<(nq + 255) / 256, 256, 0, st>>>(f, periodic ? X : f, s, g, op->s, t,
                                                            wa, wb);
            GB_LAUNCH_CHECK();
        }
        return 0;
    }
    // weighted Jacobi, ping-pong so that the last sweep lands in f
    const double* src = f;
    if (nrelax % 2 == 1) {
        GB_CUDA_TRY(cudaMemcpyAsync(X, f, bytes, cudaMemcpyDeviceToDevice, st));
        src = X;
    }
    const int ng = (int)op->ng();
    const Phases P0{};
    for (int it = 0; it < nrelax; it++) {
        double* dst = (src == f) ? X : f;
        // the plane-marching kernel for axis-aligned operators, else one
        // thread a point
        const int rc = launch_wfd_tiled<double, 1>(src, dst, 1, g, P0, op->s, st, s, w);
        if (rc == -2) return fail(GB_ECUDA, "WOperator relax: could not raise the shared-memory limit");
        if (rc != 0) k_wjacobi<<<(ng + 255) / 256, 256, 0, st>>>(src, dst, s, g, op->s, w);
        src = dst;
    }
    GB_LAUNCH_CHECK();
    return 0;
}

extern "C" int gb_woperator_get_diagonal_element(gb_woperator* op, double* out, void* stream) {
    if (!op || !out) return fail(GB_EINVAL, "WOperator get_diagonal_element: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (!op->diag_dev) GB_CUDA_TRY(cudaMalloc(&op->diag_dev, sizeof(unsigned long long)));
    GB_CUDA_TRY(cudaMemsetAsync(op->diag_dev, 0, sizeof(unsigned long long), st));
    const int ng = (int)op->ng();
    const int nb = std::min(1184, (ng + 255) / 256);
    k_wdiag<<<nb, 256, 0, st>>>(ng, op->s, op->diag_dev);
    GB_LAUNCH_CHECK();
    unsigned long long bits = 0;
    GB_CUDA_TRY(cudaMemcpyAsync(&bits, op->diag_dev, sizeof bits, cudaMemcpyDeviceToHost, st));
    GB_CUDA_TRY(cudaStreamSynchronize(st));
    double d;
    memcpy(&d, &bits, sizeof d);
    *out = d;
    return 0;
}
