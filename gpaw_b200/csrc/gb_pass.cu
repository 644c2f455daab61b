// One stencil pass with a linear epilogue,
//     v = p0 aux + p1 u + p2 (A u) + p3 aux2,
// for the mixed-precision solver's levels (T = float) and its FP64 defect
// (T = double, v = rho - L phi written as float, with per-CTA partial sums
// of v^2).  A is an axis-aligned stencil of half-width NN <= 3 with zero or
// periodic boundaries.  The solver's own arithmetic: fused multiply-adds in
// any order (its results are checked by tolerance, not bit for bit).
//
// Layout of the work: a CTA owns a 16 x (16 VX) tile of rows x columns and
// marches through a chunk of planes.  Each thread computes VX = 16 B /
// sizeof(T) consecutive points of one row (a float4 or double2), so the
// in-plane neighbours come as a few 16-byte shared-memory reads shared by
// those points; the 2 NN + 1 values of its points along the marching axis
// sit in a register queue.  Planes (tile plus halo) are staged into a ring
// of shared memory by cp.async, 8 - NN - 2 planes ahead of the queue's
// front, and the pointwise operands one plane ahead into registers; the
// element-to-thread
// assignment of the staging, with the boundary (zero fill or periodic wrap)
// folded in, is computed once per CTA, so a staged element costs one copy
// instruction.  Rows of the solver's arrays are not 16-byte aligned (odd
// sides), which rules out TMA here; the shared-memory tile is aligned
// instead.
#include "gb_objects.cuh"

namespace gb {
namespace {

constexpr int PT_ROWS = 16;   // rows of a tile, 16 threads each
constexpr int PT_HX = 4;      // halo columns staged on each side
constexpr int PT_RING = 8;    // planes in the ring

template <class T>
struct PassVec;
template <>
struct PassVec<float> {
    using V = float4;
    static constexpr int N = 4;
};
template <>
struct PassVec<double> {
    using V = double2;
    static constexpr int N = 2;
};

template <class T>
struct PassCoef {
    T c0;
    T cp[3][3];   // +d along direction k (0: columns, 1: rows, 2: planes)
    T cm[3][3];
};

enum : int {
    PF_AUX = 1, PF_AUX2 = 2, PF_ACC64 = 4, PF_OUT32 = 8, PF_PARTIAL = 16,
    // double only: the preconditioner step out = +-(u - sc (A u - aux)) with
    // the stencil summed and every product and sum rounded as the
    // reference's C loop does (bit-identical); p0 = sc, p1 != 0 negates
    PF_EXACT_PRECOND = 32
};

template <class T>
__device__ __forceinline__ void vload(T* dst, const T* src) {
    using V = typename PassVec<T>::V;
    const V v = *reinterpret_cast<const V*>(src);
    if constexpr (sizeof(T) == 4) {
        dst[0] = v.x;
        dst[1] = v.y;
        dst[2] = v.z;
        dst[3] = v.w;
    } else {
        dst[0] = v.x;
        dst[1] = v.y;
    }
}

__device__ __forceinline__ void cp_async_elem(unsigned dst, const void* src, int bytes_valid,
                                              int size) {
    if (size == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src),
                     "r"(bytes_valid));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                     "r"(bytes_valid));
}

// CTAs an SM holds: 3, or 2 for the variant that also carries an FP64
// accumulator (its registers would spill at 3)
template <int F>
constexpr int pass_min_blocks() {
    return (F & PF_ACC64) ? 2 : 3;
}

template <class T, int NN, int F>
__global__ void __launch_bounds__(256, pass_min_blocks<F>())
k_pass(const T* __restrict__ u, T* __restrict__ out, const T* __restrict__ aux,
       const T* __restrict__ aux2, double* __restrict__ acc64, float* __restrict__ out32,
       double* __restrict__ partial, GridBC g, PassCoef<T> c, T p0, T p1, T p2, T p3, int chunk,
       int tiles_x) {
    constexpr int VX = PassVec<T>::N;
    constexpr int TX = 16 * VX;
    constexpr int C = TX + 2 * PT_HX;           // staged columns
    constexpr int R = PT_ROWS + 2 * NN;         // staged rows
    constexpr int E = R * C;                    // elements of a staged plane
    constexpr int NE = (E + 255) / 256;         // staged elements a thread
    constexpr int NL = (NN + VX - 1) / VX;      // vectors of halo a side
    constexpr int Q = 2 * NN + 1;
    // planes staged beyond the queue's front: as many as the ring holds
    // while the slot being refilled was read two iterations back or more
    constexpr int AHEAD = PT_RING - NN - 2;
    extern __shared__ __align__(16) unsigned char pass_smem[];
    T* ring = reinterpret_cast<T*>(pass_smem);

    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const long long ps = (long long)n1 * n2;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int x0 = (blockIdx.x % tiles_x) * TX, y0 = (blockIdx.x / tiles_x) * PT_ROWS;
    const int x = x0 + VX * tx, y = y0 + ty;
    const int pa = blockIdx.y * chunk;
    const int pb = min(n0, pa + chunk);
    {   // grid blockIdx.z of a batch
        const long long off = (long long)blockIdx.z * n0 * ps;
        u += off;
        if (out) out += off;
        if (aux) aux += off;
        if (aux2) aux2 += off;
    }

    // staging map: in-plane offset of each element this thread copies, or
    // -1 for a zero (outside a zero boundary); the boundary is fixed per CTA
    int goff[NE];
#pragma unroll
    for (int i = 0; i < NE; i++) {
        const int e = tid + 256 * i;
        goff[i] = -1;
        if (e < E) {
            int r = y0 - NN + e / C, col = x0 - PT_HX + e % C;
            bool ok = true;
            if (r < 0 || r >= n1) {
                if (g.periodic[1]) r += r < 0 ? n1 : -n1;
                else ok = false;
            }
            if (col < 0 || col >= n2) {
                if (g.periodic[2]) col += col < 0 ? n2 : -n2;
                else ok = false;
            }
            if (ok) goff[i] = r * n2 + col;
        }
    }
    const unsigned ring_addr = (unsigned)__cvta_generic_to_shared(ring);
    auto plane_of = [&](int q, bool& ok) -> long long {
        ok = true;
        if (q < 0 || q >= n0) {
            if (!g.periodic[0]) {
                ok = false;
                return 0;
            }
            q += q < 0 ? n0 : -n0;
        }
        return (long long)q * ps;
    };
    auto stage = [&](int q) {
        bool ok;
        const long long base = plane_of(q, ok);
        const unsigned slot = ring_addr + (unsigned)((q & (PT_RING - 1)) * E * sizeof(T));
#pragma unroll
        for (int i = 0; i < NE; i++) {
            const int e = tid + 256 * i;
            if (e < E) {
                const bool v = ok && goff[i] >= 0;
                const T* src = v ? u + base + goff[i] : u;
                cp_async_elem(slot + (unsigned)(e * sizeof(T)), src, v ? (int)sizeof(T) : 0,
                              (int)sizeof(T));
            }
        }
    };
    // own values at plane q, straight from global memory (queue warm-up)
    auto own = [&](int q, T* dst) {
        bool ok;
        const long long base = plane_of(q, ok);
#pragma unroll
        for (int j = 0; j < VX; j++)
            dst[j] = (ok && y < n1 && x + j < n2) ? u[base + (long long)y * n2 + x + j] : T(0);
    };

    T q[Q][VX];
#pragma unroll
    for (int k = 1; k < Q; k++) own(pa - NN + k - 1, q[k]);
    for (int k = 0; k < NN + AHEAD; k++) {
        if (pa + k < pb + NN) stage(pa + k);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    // pointwise operands (aux, aux2, acc64) of the next plane, loaded one
    // plane ahead so that their latency overlaps a plane's work
    T na[VX], nb[VX];
    double nc[VX];
    auto load_pointwise = [&](int pp) {
        if (pp < pb && y < n1) {
            const long long row = (long long)pp * ps + (long long)y * n2 + x;
#pragma unroll
            for (int j = 0; j < VX; j++)
                if (x + j < n2) {
                    if (F & PF_AUX) na[j] = aux[row + j];
                    if (F & PF_AUX2) nb[j] = aux2[row + j];
                    if (F & PF_ACC64) nc[j] = acc64[row + j];
                }
        }
    };
    load_pointwise(pa);
    double sq = 0.0;
    const int col0 = PT_HX + VX * tx;
    for (int p = pa; p < pb; p++) {
        T ca[VX], cb[VX];
        double cc[VX];
#pragma unroll
        for (int j = 0; j < VX; j++) {
            ca[j] = na[j];
            cb[j] = nb[j];
            cc[j] = nc[j];
        }
        load_pointwise(p + 1);
        if (p + NN + AHEAD < pb + NN) stage(p + NN + AHEAD);
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(AHEAD));
        __syncthreads();
        const T* cur = ring + (p & (PT_RING - 1)) * E;
        const T* front = ring + ((p + NN) & (PT_RING - 1)) * E;
#pragma unroll
        for (int k = 0; k < Q - 1; k++)
#pragma unroll
            for (int j = 0; j < VX; j++) q[k][j] = q[k + 1][j];
        vload<T>(q[Q - 1], front + (ty + NN) * C + col0);
        // the row: NL vectors left, the centre, NL right
        T w[(2 * NL + 1) * VX];
#pragma unroll
        for (int v = 0; v < 2 * NL + 1; v++)
            vload<T>(w + v * VX, cur + (ty + NN) * C + col0 + (v - NL) * VX);
        T acc[VX];
        if constexpr ((F & PF_EXACT_PRECOND) != 0 && sizeof(T) == 8) {
            // x = 0; x += v c in coefficient order: the centre, then per
            // direction (columns, rows, planes) +1..+NN and -1..-NN, every
            // product and sum rounded on its own
#pragma unroll
            for (int j = 0; j < VX; j++) acc[j] = __dadd_rn(0.0, __dmul_rn(w[NL * VX + j], c.c0));
#pragma unroll
            for (int d = 1; d <= NN; d++)
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(w[NL * VX + j + d], c.cp[0][d - 1]));
#pragma unroll
            for (int d = 1; d <= NN; d++)
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(w[NL * VX + j - d], c.cm[0][d - 1]));
#pragma unroll
            for (int d = 1; d <= NN; d++) {
                T yv[VX];
                vload<T>(yv, cur + (ty + NN + d) * C + col0);
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(yv[j], c.cp[1][d - 1]));
            }
#pragma unroll
            for (int d = 1; d <= NN; d++) {
                T yv[VX];
                vload<T>(yv, cur + (ty + NN - d) * C + col0);
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(yv[j], c.cm[1][d - 1]));
            }
#pragma unroll
            for (int d = 1; d <= NN; d++)
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(q[NN + d][j], c.cp[2][d - 1]));
#pragma unroll
            for (int d = 1; d <= NN; d++)
#pragma unroll
                for (int j = 0; j < VX; j++)
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(q[NN - d][j], c.cm[2][d - 1]));
        } else {
#pragma unroll
        for (int j = 0; j < VX; j++) acc[j] = c.c0 * w[NL * VX + j];
#pragma unroll
        for (int d = 1; d <= NN; d++) {
            T ym[VX], yp[VX];
            vload<T>(yp, cur + (ty + NN + d) * C + col0);
            vload<T>(ym, cur + (ty + NN - d) * C + col0);
#pragma unroll
            for (int j = 0; j < VX; j++) {
                T a = acc[j];
                a = fma(c.cp[0][d - 1], w[NL * VX + j + d], a);
                a = fma(c.cm[0][d - 1], w[NL * VX + j - d], a);
                a = fma(c.cp[1][d - 1], yp[j], a);
                a = fma(c.cm[1][d - 1], ym[j], a);
                a = fma(c.cp[2][d - 1], q[NN + d][j], a);
                a = fma(c.cm[2][d - 1], q[NN - d][j], a);
                acc[j] = a;
            }
        }
        }
        if (y < n1) {
            const long long row = (long long)p * ps + (long long)y * n2 + x;
#pragma unroll
            for (int j = 0; j < VX; j++) {
                if (x + j >= n2) break;
                if constexpr ((F & PF_EXACT_PRECOND) != 0 && sizeof(T) == 8) {
                    const T yv = __dsub_rn(w[NL * VX + j], __dmul_rn(__dsub_rn(acc[j], ca[j]), p0));
                    out[row + j] = p1 != T(0) ? -yv : yv;
                    continue;
                }
                T v = fma(p1, w[NL * VX + j], p2 * acc[j]);
                if (F & PF_AUX) v = fma(p0, ca[j], v);
                if (F & PF_AUX2) v = fma(p3, cb[j], v);
                if (F & PF_PARTIAL) sq = fma((double)v, (double)v, sq);
                if (F & PF_ACC64)
                    acc64[row + j] = cc[j] + (double)v;
                else if (F & PF_OUT32)
                    out32[row + j] = (float)v;
                else
                    out[row + j] = v;
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    if (F & PF_PARTIAL) {
        const double s = block_sum(sq);
        if (tid == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}


struct PassGeom {
    int tiles_x, tiles_y, chunk, nchunk;
};

template <class T>
PassGeom pass_geom(const GridBC& g, int per_sm, int nin = 1) {
    constexpr int TX = 16 * PassVec<T>::N;
    PassGeom G;
    G.tiles_x = (g.n[2] + TX - 1) / TX;
    G.tiles_y = (g.n[1] + PT_ROWS - 1) / PT_ROWS;
    const int tiles = G.tiles_x * G.tiles_y;
    // one wave: at most as many CTAs as fit on the GPU at once (a batch of
    // nin grids: whole grids a CTA column once the batch fills the GPU)
    int want = 148 * per_sm / (tiles * std::max(1, nin));
    want = std::max(1, std::min(want, g.n[0]));
    G.chunk = (g.n[0] + want - 1) / want;
    G.nchunk = (g.n[0] + G.chunk - 1) / G.chunk;
    return G;
}

template <class T>
bool pass_supported(const GridBC& g, const CfdStencil& cs, int nn) {
    if (nn < 1 || nn > 3) return false;
    if (!(cs.axis[0] == 2 && cs.axis[1] == 1 && cs.axis[2] == 0)) return false;
    // wrapped halos must come from inside the grid
    if (g.n[2] < PT_HX || g.n[1] < nn || g.n[0] < nn) return false;
    const long long ps = (long long)g.n[1] * g.n[2];
    return ps * g.n[0] < (1ll << 31) && ps < (1ll << 31);
}

template <class T, int NN, int F>
int launch_pass_f(const GridBC& g, const PassCoef<T>& c, const T* in, T* out, const T* aux,
                  const T* aux2, double* acc64, float* out32, double* partial, T p0, T p1, T p2,
                  T p3, cudaStream_t st, int nin = 1) {
    constexpr int VX = PassVec<T>::N;
    constexpr size_t smem = (size_t)PT_RING * (PT_ROWS + 2 * NN) * (16 * VX + 2 * PT_HX) * sizeof(T);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_pass<T, NN, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return -2;
        attr = true;
    }
    const PassGeom G = pass_geom<T>(g, pass_min_blocks<F>(), nin);
    dim3 grid(G.tiles_x * G.tiles_y, G.nchunk, nin);
    k_pass<T, NN, F><<<grid, 256, smem, st>>>(in, out, aux, aux2, acc64, out32, partial, g, c, p0,
                                             p1, p2, p3, G.chunk, G.tiles_x);
    return 0;
}

template <class T, int NN>
int launch_pass_nn(int f, const GridBC& g, const PassCoef<T>& c, const T* in, T* out,
                   const T* aux, const T* aux2, double* acc64, float* out32, double* partial, T p0,
                   T p1, T p2, T p3, cudaStream_t st) {
#define GB_PASS_F(FF)                                                                            \
    case FF:                                                                                    \
        return launch_pass_f<T, NN, FF>(g, c, in, out, aux, aux2, acc64, out32, partial, p0, p1, \
                                        p2, p3, st)
    if constexpr (sizeof(T) == 4) {
        switch (f) {
            GB_PASS_F(0);
            GB_PASS_F(PF_AUX);
            GB_PASS_F(PF_AUX2);
            GB_PASS_F(PF_AUX | PF_AUX2);
            GB_PASS_F(PF_AUX2 | PF_ACC64);
            default: return -1;
        }
    } else {
        switch (f) {
            GB_PASS_F(PF_AUX | PF_OUT32 | PF_PARTIAL);
            default: return -1;
        }
    }
#undef GB_PASS_F
}

}  // namespace

bool pass_supported_grid(const GridBC& g, const CfdStencil& cs, int nn) {
    return pass_supported<float>(g, cs, nn);
}

int pass_blocks(const GridBC& g, int elem_bytes) {
    // the FP64 defect variant (no accumulator): three CTAs an SM
    const PassGeom G = elem_bytes == 4 ? pass_geom<float>(g, 3) : pass_geom<double>(g, 3);
    return G.tiles_x * G.tiles_y * G.nchunk;
}

template <class T>
int launch_pass(const GridBC& g, const CfdStencil& cs, int nn, const T* in, T* out, const T* aux,
                const T* aux2, double p0, double p1, double p2, double p3, double* acc64,
                float* out32, double* partial, cudaStream_t st) {
    if (!pass_supported<T>(g, cs, nn)) return -1;
    PassCoef<T> c{};
    c.c0 = (T)cs.c0;
    for (int k = 0; k < 3; k++)
        for (int d = 0; d < nn; d++) {
            c.cp[k][d] = (T)cs.cp[k][d];
            c.cm[k][d] = (T)cs.cm[k][d];
        }
    const int f = (aux ? PF_AUX : 0) | (aux2 ? PF_AUX2 : 0) | (acc64 ? PF_ACC64 : 0) |
                  (out32 ? PF_OUT32 : 0) | (partial ? PF_PARTIAL : 0);
    const T a0 = (T)p0, a1 = (T)p1, a2 = (T)p2, a3 = (T)p3;
    switch (nn) {
        case 1: return launch_pass_nn<T, 1>(f, g, c, in, out, aux, aux2, acc64, out32, partial, a0, a1, a2, a3, st);
        case 2: return launch_pass_nn<T, 2>(f, g, c, in, out, aux, aux2, acc64, out32, partial, a0, a1, a2, a3, st);
        default: return launch_pass_nn<T, 3>(f, g, c, in, out, aux, aux2, acc64, out32, partial, a0, a1, a2, a3, st);
    }
}

int launch_pass_precond(const GridBC& g, const CfdStencil& cs, int nn, const double* in,
                        double* out, const double* aux, int nin, double sc, int negate,
                        cudaStream_t st) {
    if (!pass_supported<double>(g, cs, nn) || nin < 1 || nin > 65535 || !in || !out || !aux)
        return -1;
    PassCoef<double> c{};
    c.c0 = cs.c0;
    for (int k = 0; k < 3; k++)
        for (int d = 0; d < nn; d++) {
            c.cp[k][d] = cs.cp[k][d];
            c.cm[k][d] = cs.cm[k][d];
        }
    constexpr int F = PF_AUX | PF_EXACT_PRECOND;
    const double ng = negate ? 1.0 : 0.0;
    switch (nn) {
        case 1: return launch_pass_f<double, 1, F>(g, c, in, out, aux, nullptr, nullptr, nullptr, nullptr, sc, ng, 0.0, 0.0, st, nin);
        case 2: return launch_pass_f<double, 2, F>(g, c, in, out, aux, nullptr, nullptr, nullptr, nullptr, sc, ng, 0.0, 0.0, st, nin);
        default: return launch_pass_f<double, 3, F>(g, c, in, out, aux, nullptr, nullptr, nullptr, nullptr, sc, ng, 0.0, 0.0, st, nin);
    }
}

template int launch_pass<float>(const GridBC&, const CfdStencil&, int, const float*, float*,
                                const float*, const float*, double, double, double, double,
                                double*, float*, double*, cudaStream_t);
template int launch_pass<double>(const GridBC&, const CfdStencil&, int, const double*, double*,
                                 const double*, const double*, double, double, double, double,
                                 double*, float*, double*, cudaStream_t);

}  // namespace gb
