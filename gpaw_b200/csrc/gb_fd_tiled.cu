// Plane-marching FD apply for central-difference (axis-aligned) stencils.
//
// Same result as k_fd_generic (and as the reference's bmgs_fd over its
// padded buffer, c/bmgs/fd.cpp:9-33): every output is
//     x = 0;  x += v(center) c0;  then, for each of the three directions in
//     the caller's order, x += v(+1) c(+1) ... v(+nn) c(+nn),
//     x += v(-1) c(-1) ... v(-nn) c(-nn)
// with separately rounded products and sums.
//
// Data movement (one CTA = TX x TY output columns, a chunk of planes along
// axis 0):
//  * a multi-stage ring of shared-memory plane tiles, each tile the TX x TY
//    block plus an nn-wide halo on the four in-plane sides, filled with
//    asynchronous global->shared copies (cp.async, register-free, with
//    hardware zero fill for zero-boundary cells) D planes ahead of use;
//  * a register queue of 2nn+1 values per output along axis 0, so the
//    axis-0 neighbours are read from shared memory once per point;
//  * each thread owns RY consecutive rows of one column, so the axis-1
//    neighbours are shared between its rows.
// Periodic halos are copied from the wrapped position; the Bloch phase of a
// wrapped complex value is applied when it is read (register-side, exact
// complex multiply as in bmgs_translatemz, c/bmgs/translate.cpp:28-47).
#include <cstdlib>
#include <cstring>
#include <utility>

#include <algorithm>

#include "gb_internal.cuh"
#include "gb_tma.cuh"

namespace gb {


// Planes per CTA along axis 0.  A batch of grids already gives enough
// CTAs; a single grid is split along axis 0 until the launch has at least
// `target` CTAs (default 148 * 2, tunable by GPAW_B200_CTA_TARGET), but
// never into chunks shorter than 2 nn planes.
int cfd_chunk(const GridBC& g, int nn, int nin, int ty) {
    static int target = [] {
        const char* v = getenv("GPAW_B200_CTA_TARGET");
        const int t = v ? atoi(v) : 0;
        return t > 0 ? t : 148 * 2;
    }();
    const int tiles_x = (g.n[2] + 31) / 32;
    const int tiles_y = (g.n[1] + ty - 1) / ty;
    const long long tiles = (long long)tiles_x * tiles_y * nin;
    int chunk0 = g.n[0];
    while (chunk0 > 2 * nn && tiles * ((g.n[0] + chunk0 - 1) / chunk0) < target)
        chunk0 = (chunk0 + 1) / 2;
    return chunk0;
}

// GPAW_B200_FMA=1 selects the fused-multiply-add form of the complex
// nn = 3 apply: not bit-identical to the reference (each product is no
// longer rounded before its sum), within a few ulp per point.  Read at
// every launch so it can be switched on and off inside one process.
bool fused_apply() {
    const char* e = getenv("GPAW_B200_FMA");
    return e != nullptr && atoi(e) != 0;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* sdst, const void* gsrc, bool valid) {
    const unsigned s = smem_u32(sdst);
    const int n = valid ? BYTES : 0;   // 0: zero-fill, nothing is read
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc),
                     "r"(n));
    else if (BYTES == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc),
                     "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc),
                     "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// (1 - w) b + (w (src - x)) / c0, each operation rounded on its own
template <class T>
__device__ __forceinline__ T jacobi_update(T b, T src, T x, double w, double c0);
template <>
__device__ __forceinline__ double jacobi_update<double>(double b, double src, double x, double w,
                                                        double c0) {
    return __dadd_rn(__dmul_rn(1.0 - w, b), __ddiv_rn(__dmul_rn(w, __dsub_rn(src, x)), c0));
}
template <>
__device__ __forceinline__ double2 jacobi_update<double2>(double2 b, double2, double2, double,
                                                          double) {
    return b;  // relaxation is defined for real data only
}
template <>
__device__ __forceinline__ float jacobi_update<float>(float b, float src, float x, double w,
                                                      double c0) {
    return (1.0f - (float)w) * b + (float)w * (src - x) / (float)c0;
}

// x + v c with one rounding (fused multiply-add): the opt-in fast form.
template <class T>
__device__ __forceinline__ T fma_fused(T x, T v, double c);
template <>
__device__ __forceinline__ double fma_fused<double>(double x, double v, double c) {
    return __fma_rn(v, c, x);
}
template <>
__device__ __forceinline__ double2 fma_fused<double2>(double2 x, double2 v, double c) {
    return make_double2(__fma_rn(v.x, c, x.x), __fma_rn(v.y, c, x.y));
}
template <>
__device__ __forceinline__ float fma_fused<float>(float x, float v, double c) {
    return __fmaf_rn(v, (float)c, x);
}

template <class T>
__device__ __forceinline__ T fma_exact(T x, T v, double c) {
    return Num<T>::add(x, Num<T>::scale(v, c));
}

// Wrap coordinate y into [0, n) for a periodic axis; returns false for a
// zero-boundary position (or one further out than one period).
__device__ __forceinline__ bool wrap_coord(int& y, int n, int periodic) {
    if (y >= 0 && y < n) return true;
    if (!periodic) return false;
    if (y < 0) y += n;
    else y -= n;
    return y >= 0 && y < n;
}

// Call f(std::integral_constant<int, I>) for I = 0 .. N-1.
template <class F, int... Is>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// Sum of one direction's 2*NN terms in the caller's order: +1..+NN then
// -1..-NN.  `vp(d)` / `vm(d)` return the values at +d / -d.
template <class T, int NN, bool FUSED, class VP, class VM>
__device__ __forceinline__ T add_direction(T x, const double* cp, const double* cm, VP vp, VM vm) {
#pragma unroll
    for (int d = 1; d <= NN; d++)
        x = FUSED ? fma_fused<T>(x, vp(d), cp[d - 1]) : fma_exact<T>(x, vp(d), cp[d - 1]);
#pragma unroll
    for (int d = 1; d <= NN; d++)
        x = FUSED ? fma_fused<T>(x, vm(d), cm[d - 1]) : fma_exact<T>(x, vm(d), cm[d - 1]);
    return x;
}

// Directions are summed in the order GUCLaplace builds for an orthorhombic
// cell: axis 2, axis 1, axis 0.  ORD = 1: every product and sum rounded on
// its own (bit-identical to the reference); ORD = 2: fused multiply-adds
// (fewer instructions, results within a few ulp; opt-in, apply only);
// ORD = 3: fused multiply-adds into one partial sum a direction, the three
// added at the end (the mixed-precision solver's own passes, EPI_LIN, whose
// results are checked by tolerance: shorter dependency chains).
// Register caps: three resident CTAs of 256 threads for the complex apply
// (nn <= 3), two for the other complex modes, four CTAs of 128 threads for
// real data.
// LD selects how plane tiles reach shared memory: 0 per-thread cp.async
// cells (any element type), 1 one TMA tensor copy per plane (16-byte
// elements; `map` describes the whole batch, `b0` is this launch's first
// grid in it).  With the TMA the tile arrives with zeros past every edge;
// the halo cells past a periodic edge of axis 1 or 2 are then stored by the
// threads (values loaded one plane ahead, times the Bloch phase).
template <class T, int NN, int TX, int TY, int RY, int D, int MODE, int ORD, int LD, int MINB>
__global__ void __launch_bounds__(TX * (TY / RY), MINB)
k_fd_cfd(const T* __restrict__ in, T* __restrict__ out, int nin, GridBC g, Phases P,
         CfdStencil cs, int chunk0, int tiles_x, Epi ep, const __grid_constant__ CUtensorMap map,
         int b0) {
    constexpr int PX = TX + 2 * NN;          // tile pitch (elements)
    constexpr int PY = TY + 2 * NN;
    constexpr int S = NN + 1 + D;            // ring depth
    constexpr int NT = TX * (TY / RY);
    constexpr int Q = 2 * NN + 1;
    constexpr int EB = (int)sizeof(T);
    constexpr bool CPLX = sizeof(T) == 16;
    static_assert(LD == 0 || CPLX, "TMA tiles: 16-byte elements only");
    // plane stage stride: 128-byte aligned for the TMA
    constexpr int SP = LD ? (PX * PY + 7) / 8 * 8 : PX * PY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ring;
    uint64_t* bar = nullptr;
    if constexpr (LD == 1) {
        const unsigned mis = tma_smem_u32(smem_raw) & 127u;
        ring = reinterpret_cast<T*>(smem_raw + (mis ? 128 - mis : 0));
        bar = reinterpret_cast<uint64_t*>(ring + S * SP);
    } else {
        ring = reinterpret_cast<T*>(smem_raw);
    }

    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int x0 = (blockIdx.x % tiles_x) * TX;
    const int y0 = (blockIdx.x / tiles_x) * TY;
    const int pa = blockIdx.y * chunk0;
    const int pb = min(n0, pa + chunk0);
    const int b = blockIdx.z;
    const int tid = threadIdx.x;
    if (pa >= pb || b >= nin) {
        if ((MODE == EPI_RESID || MODE == EPI_LIN) && ep.partial && tid == 0)
            ep.partial[((long long)b * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = 0.0;
        return;
    }
    const long long ng = (long long)n0 * n1 * n2;
    const long long pstride = (long long)n1 * n2;   // one plane
    const T* a = in + b * ng;
    T* o = out + b * ng;
    const T* aux = (const T*)ep.aux + b * ng;
    const T* aux2 = (const T*)ep.aux2 + b * ng;
    double sq = 0.0;
    const int tx = tid % TX;
    const int ty0 = (tid / TX) * RY;
    const int gx = x0 + tx;
    long long colr[RY];      // in-plane offset of this thread's rows
#pragma unroll
    for (int r = 0; r < RY; r++) colr[r] = (long long)(y0 + ty0 + r) * n2 + gx;

    // -- async copy of relative plane j (absolute pa + j) ------------------
    // Rows -NN..TY+NN-1 at columns 0..TX-1, and rows 0..TY-1 of the two
    // x-halo strips (corners are never read by a cfd stencil).
    constexpr int NMID = PY * TX;
    constexpr int NSIDE = TY * 2 * NN;
    auto cell = [&](int e, int& ry, int& rx) {
        if (e < NMID) {
            ry = e / TX - NN;
            rx = e % TX;
        } else {
            const int f = e - NMID;
            ry = f / (2 * NN);
            const int c = f % (2 * NN);
            rx = c < NN ? c - NN : TX + c - NN;
        }
    };
    // Each thread copies the same NC cells of every plane: precompute their
    // shared-memory offsets, in-plane source offsets (after the periodic
    // wrap), validity and Bloch-phase code once per CTA.
    constexpr int NC = (NMID + NSIDE + NT - 1) / NT;
    int soff[NC], goff[NC];
    unsigned vmask = 0, wcode = 0;   // wcode: 3 bits per cell (0 = no phase)
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const int e = tid + i * NT;
        soff[i] = 0;
        goff[i] = 0;
        if (e >= NMID + NSIDE) continue;
        int ry, rx;
        cell(e, ry, rx);
        soff[i] = (ry + NN) * PX + (rx + NN);
        int y = y0 + ry, x = x0 + rx;
        const bool yw = y < 0 || y >= n1, xw = x < 0 || x >= n2;
        const int ys = y < 0, xs = x < 0;
        if (wrap_coord(y, n1, g.periodic[1]) && wrap_coord(x, n2, g.periodic[2])) {
            vmask |= 1u << i;
            goff[i] = y * n2 + x;
            // phase code: 1 + 2*axis_index + side, axis 1 -> 0, axis 2 -> 1
            unsigned c = 0;
            if (yw) c = 1 + ys;
            else if (xw) c = 3 + xs;
            wcode |= c << (3 * i);
        }
    }
    if (!(CPLX && P.use)) wcode = 0;
    // slot = j % S (a compile-time constant inside the unrolled march when
    // the ring depth equals the queue length)
    auto issue = [&](int j, int slot) {
        int pl = pa + j;
        const bool pvalid = wrap_coord(pl, n0, g.periodic[0]);
        T* st = ring + slot * SP;
        const T* src = a + pl * pstride;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= NMID + NSIDE) break;
            const bool ok = pvalid && ((vmask >> i) & 1);
            cp_async<EB>(st + soff[i], ok ? src + goff[i] : a, ok);
        }
    };
    // After this thread's own copies of plane j completed, multiply the
    // wrapped halo cells among them by their phase (the halo is filled from
    // the opposite side, as bc_unpack1's translate does, c/bc.cpp:242-257).
    // Other threads read them NN iterations later, after a barrier.
    auto fixup = [&](int slot) {
        T* st = ring + slot * SP;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            const unsigned c = (wcode >> (3 * i)) & 7u;
            if (c == 0) continue;
            if constexpr (CPLX) {
                const double2 ph = c == 1 ? P.ph[1][0] : c == 2 ? P.ph[1][1]
                                 : c == 3 ? P.ph[2][0] : P.ph[2][1];
                st[soff[i]] = cmul(ph, st[soff[i]]);
            }
        }
    };

    // -- TMA tiles (LD == 1): the halo cells past a periodic edge ----------
    // Cells the stencil reads that lie outside the grid on one axis: rows
    // past axis 1's edges (columns 0..TX-1 of the tile) and columns past
    // axis 2's edges (rows 0..TY-1), taken from rows/columns beyond the
    // grid's extent inside [-NN, TY + NN) x [-NN, TX + NN).  They are dealt
    // to the threads, at most NWR each (the launcher checks the count).
    constexpr int NWR = LD ? (2 * NN * (TX + TY) + NT - 1) / NT : 1;
    int wso[NWR], wgo[NWR];
    unsigned wmask = 0, wph = 0;   // wph: 3 bits a cell, the code of `fixup`
    if constexpr (LD == 1) {
        const int rb0 = max(-NN, -y0), rb1 = min(TY + NN, n1 - y0);   // in-grid rows
        const int cb0 = max(-NN, -x0), cb1 = min(TX + NN, n2 - x0);   // in-grid columns
        const int ra0 = max(0, cb0), ra1 = min(TX, cb1);              // part A columns
        const int nrowA = g.periodic[1] ? (TY + 2 * NN) - (rb1 - rb0) : 0;
        const int ncolA = max(0, ra1 - ra0);
        const int nA = nrowA * ncolA;
        const int rB0 = max(0, rb0), rB1 = min(TY, rb1);              // part B rows
        const int ncolB = g.periodic[2] ? (TX + 2 * NN) - (cb1 - cb0) : 0;
        const int nB = max(0, rB1 - rB0) * ncolB;
#pragma unroll
        for (int r = 0; r < NWR; r++) {
            const int w = tid + r * NT;
            wso[r] = 0;
            wgo[r] = 0;
            int ry, rx;
            if (w < nA) {
                const int q = w / ncolA;
                rx = ra0 + w % ncolA;
                // outside rows: [-NN, rb0) then [rb1, TY + NN)
                ry = q < rb0 + NN ? q - NN : rb1 + (q - (rb0 + NN));
            } else if (w < nA + nB) {
                const int w2 = w - nA;
                ry = rB0 + w2 / ncolB;
                const int c = w2 % ncolB;
                rx = c < cb0 + NN ? c - NN : cb1 + (c - (cb0 + NN));
            } else {
                continue;
            }
            int y = y0 + ry, x = x0 + rx;
            const bool yw = y < 0 || y >= n1;
            const int ys = y < 0, xs = x < 0;
            if (wrap_coord(y, n1, g.periodic[1]) && wrap_coord(x, n2, g.periodic[2])) {
                wmask |= 1u << r;
                wso[r] = (ry + NN) * PX + (rx + NN);
                wgo[r] = y * n2 + x;
                wph |= (yw ? 1u + ys : 3u + xs) << (3 * r);
            }
        }
        if (!P.use) wph = 0;
    }
    T pre[NWR];
    // this thread's wrapped cells of centre plane p (in the grid), loaded
    // one plane before they are stored
    auto load_wrapped = [&](int p) {
#pragma unroll
        for (int r = 0; r < NWR; r++)
            pre[r] = ((wmask >> r) & 1) ? __ldg(a + p * pstride + wgo[r]) : Num<T>::zero();
    };
    auto store_wrapped = [&](int slot) {
        T* st = ring + slot * SP;
#pragma unroll
        for (int r = 0; r < NWR; r++) {
            if (!((wmask >> r) & 1)) continue;
            T v = pre[r];
            if constexpr (CPLX) {
                const unsigned c = (wph >> (3 * r)) & 7u;
                if (c) v = cmul(c == 1 ? P.ph[1][0] : c == 2 ? P.ph[1][1]
                                : c == 3 ? P.ph[2][0] : P.ph[2][1], v);
            }
            st[wso[r]] = v;
        }
    };
    // thread 0: the tile window of relative plane j into slot j % S
    auto issue_tma = [&](int j, int slot) {
        int pl = pa + j;
        const bool pvalid = wrap_coord(pl, n0, g.periodic[0]);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[slot], (unsigned)(PX * PY * EB));
        // a plane past a zero boundary: a window outside the tensor (zeros)
        tma_load_window16(ring + slot * SP, &map, x0 - NN, y0 - NN, pvalid ? pl : -1,
                          b0 + b, &bar[slot]);
    };

    // -- axis-0 queue ---------------------------------------------------------
    // Slot j % Q of the queue holds relative plane j (j = -NN .. nplanes +
    // NN - 1).  Planes pa-NN..pa-1 (before the chunk) come straight from
    // global memory.
    T q[RY][Q];
#pragma unroll
    for (int r = 0; r < RY; r++)
#pragma unroll
        for (int k = 0; k < Q; k++) q[r][k] = Num<T>::zero();
#pragma unroll
    for (int k = 0; k < NN; k++) {
        int pl = pa - NN + k;
        const bool wrapped = pl < 0;
        const bool pv = wrap_coord(pl, n0, g.periodic[0]);
#pragma unroll
        for (int r = 0; r < RY; r++) {
            const int gy = y0 + ty0 + r;
            T v = Num<T>::zero();
            if (pv && gx < n2 && gy < n1) {
                v = __ldg(a + ((long long)pl * n1 + gy) * n2 + gx);
                if constexpr (CPLX)
                    if (P.use && wrapped) v = cmul(P.ph[0][1], v);
            }
            q[r][NN + 1 + k] = v;   // relative plane k - NN sits in slot k + NN + 1
        }
    }

    // prologue: relative planes 0 .. D-1 into the ring
    const int jend = (pb - pa) + NN;   // relative planes needed: [0, jend)
    if constexpr (LD == 1) {
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q < S; q++) mbar_init(&bar[q], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0)
            for (int j = 0; j < D && j < jend; j++) issue_tma(j, j % S);
        if (wmask) load_wrapped(pa);
    } else {
#pragma unroll 1
        for (int j = 0; j < D; j++) {
            if (j < jend) issue(j, j % S);
            cp_commit();
        }
    }
    // a bounded wait ran out (all threads agree): no further copies or
    // waits; the kernel finishes with invalid output and the fault recorded
    bool dead = false;

    const int nplanes = pb - pa;
    const int total = nplanes + NN;
    // Epilogue operands (aux, aux2, FP64 accumulator) of the centre plane,
    // loaded one iteration ahead so that their latency overlaps the stencil
    // work instead of stalling every plane.
    constexpr bool NEED_AUX = MODE != EPI_APPLY;
    // EPI_POT: the potential, one real grid shared by the batch
    const double* vpot = (const double*)ep.aux;
    T pa1[RY], pa2[RY];
    double pac[RY];
    auto prefetch = [&](int p) {
#pragma unroll
        for (int r = 0; r < RY; r++) {
            const int gy = y0 + ty0 + r;
            pa1[r] = Num<T>::zero();
            pa2[r] = Num<T>::zero();
            pac[r] = 0.0;
            if (p < pb && gx < n2 && gy < n1) {
                const long long at = p * pstride + colr[r];
                if constexpr (MODE == EPI_POT) pac[r] = vpot[at];
                else if (NEED_AUX && ep.aux) pa1[r] = aux[at];
                if constexpr (MODE == EPI_LIN) {
                    if (ep.aux2) pa2[r] = aux2[at];
                    if (ep.acc64) pac[r] = ep.acc64[b * ng + at];
                }
            }
        }
    };
    if (NEED_AUX) prefetch(pa);
    // Iteration t pushes relative plane t into queue slot t % Q and, for
    // t >= NN, computes centre plane t - NN.  The loop is unrolled by Q so
    // that every slot index is a compile-time constant (no register moves).
    auto step = [&](int t, auto U_) {
        constexpr int U = decltype(U_)::value;           // t % Q
        constexpr int CU = (U + Q - NN) % Q;              // slot of the centre
        constexpr bool FIXED = S == Q;                    // ring slots = U-based
        const int s_t = FIXED ? U : t % S;
        const int s_c = FIXED ? CU : (t - NN) % S;
        const int s_d = FIXED ? (U + D) % Q : (t + D) % S;
        if constexpr (LD == 1) {
            bool bad = false;
            if (!dead) bad = !mbar_wait(&bar[s_t], (unsigned)(t / S) & 1u);
            // the window of plane t has landed: store the wrapped halo cells
            // of a centre plane (read NN iterations later, after a barrier)
            if (wmask && t < nplanes) {
                store_wrapped(s_t);
                if (t + 1 < nplanes) load_wrapped(pa + t + 1);
            }
            fence_proxy_async_smem();
            if (__syncthreads_or(bad)) dead = true;
            const int j = t + D;
            if (tid == 0 && !dead && j < jend) issue_tma(j, s_d);
        } else {
            cp_wait<D - 1>();
            // this thread's copies of plane t have landed: fix its wrapped
            // halo cells (read as a centre NN iterations later, after a
            // barrier)
            if (wcode && t < nplanes) fixup(s_t);
            __syncthreads();
            // the slot of plane t+D last held plane t-NN-1, the centre of
            // iteration t-1, which every thread has finished (barrier above)
            const int j = t + D;
            if (j < jend) issue(j, s_d);
            cp_commit();
        }
        // push plane t's own values (uniform phase for a wrapped plane)
        {
            const T* st_in = ring + s_t * SP;
            const bool wrapped = CPLX && P.use && pa + t >= n0;
#pragma unroll
            for (int r = 0; r < RY; r++) {
                T v = st_in[(ty0 + r + NN) * PX + (tx + NN)];
                if constexpr (CPLX)
                    if (wrapped) v = cmul(P.ph[0][0], v);
                q[r][U] = v;
            }
        }
        if (t >= NN) {
            const int p = pa + t - NN;
            const T* sc = ring + s_c * SP;
            // this thread's column in the centre tile (axis-1 neighbours)
            const T* colp = sc + ty0 * PX + (tx + NN);
#pragma unroll
            for (int r = 0; r < RY; r++) {
                const T vc = q[r][CU];
                const T* row = sc + (ty0 + r + NN) * PX + (tx + NN);
                // x = 0; x += v c in coefficient order (Jacobi skips c0)
                T x = Num<T>::zero();
                if (MODE != EPI_JACOBI) x = Num<T>::add(x, Num<T>::scale(vc, cs.c0));
                if constexpr (ORD == 3) {
                    // three independent fused sums, one a direction, added
                    // at the end: a third of the serial dependency chain
                    T x1 = add_direction<T, NN, true>(Num<T>::zero(), cs.cp[1], cs.cm[1],
                                         [&](int d) { return colp[(r + NN + d) * PX]; },
                                         [&](int d) { return colp[(r + NN - d) * PX]; });
                    T x0 = add_direction<T, NN, true>(Num<T>::zero(), cs.cp[2], cs.cm[2],
                                         [&](int d) { return q[r][(CU + d) % Q]; },
                                         [&](int d) { return q[r][(CU + Q - d) % Q]; });
                    x = add_direction<T, NN, true>(x, cs.cp[0], cs.cm[0],
                                         [&](int d) { return row[d]; },
                                         [&](int d) { return row[-d]; });
                    x = Num<T>::add(Num<T>::add(x, x1), x0);
                } else {
                // directions: axis 2, axis 1, axis 0 (GUCLaplace's order)
                x = add_direction<T, NN, ORD == 2>(x, cs.cp[0], cs.cm[0],
                                         [&](int d) { return row[d]; },
                                         [&](int d) { return row[-d]; });
                x = add_direction<T, NN, ORD == 2>(x, cs.cp[1], cs.cm[1],
                                         [&](int d) { return colp[(r + NN + d) * PX]; },
                                         [&](int d) { return colp[(r + NN - d) * PX]; });
                x = add_direction<T, NN, ORD == 2>(x, cs.cp[2], cs.cm[2],
                                         [&](int d) { return q[r][(CU + d) % Q]; },
                                         [&](int d) { return q[r][(CU + Q - d) % Q]; });
                }
                const int gy = y0 + ty0 + r;
                if (gx < n2 && gy < n1) {
                    const long long at = p * pstride + colr[r];
                    if (MODE == EPI_APPLY) {
                        o[at] = x;
                    } else if (MODE == EPI_POT) {
                        // numpy's o += p * v: product rounded, then the sum
                        o[at] = Num<T>::add(x, Num<T>::scale(vc, pac[r]));
                    } else if (MODE == EPI_RESID) {
                        const T res = Num<T>::sub(x, pa1[r]);
                        if (out) o[at] = res;
                        sq += sqnorm(res);
                    } else if (MODE == EPI_JACOBI) {
                        o[at] = jacobi_update<T>(vc, pa1[r], x, ep.w, cs.c0);
                    } else if (MODE == EPI_LIN) {
                        if constexpr (sizeof(T) != 16) {
                            T y = (T)ep.p1 * vc + (T)ep.p2 * x;
                            if (ep.aux) y += (T)ep.p0 * pa1[r];
                            if (ep.aux2) y += (T)ep.p3 * pa2[r];
                            if (ep.partial) sq += (double)y * (double)y;
                            if (ep.acc64) ep.acc64[b * ng + at] = pac[r] + (double)y;
                            else if (ep.out32) ep.out32[b * ng + at] = (float)y;
                            else o[at] = y;
                        }
                    } else {
                        const T y = Num<T>::sub(vc, Num<T>::scale(Num<T>::sub(x, pa1[r]), ep.sc));
                        o[at] = ep.negate ? Num<T>::neg(y) : y;
                    }
                }
            }
            // operands of the next centre plane: in flight while the next
            // iteration waits for its plane and computes the stencil
            if (NEED_AUX) prefetch(p + 1);
        }
    };
#pragma unroll 1
    for (int t0 = 0; t0 < total; t0 += Q)
        static_for<Q>([&](auto U_) {
            const int t = t0 + decltype(U_)::value;
            if (t < total) step(t, U_);
        });
    if constexpr (LD == 1) {
        // copies still in flight after a wait ran out: give them a moment
        if (dead)
            for (int j = 0; j < jend; j++) mbar_wait(&bar[j % S], (unsigned)(j / S) & 1u, 1000000ull);
    } else {
        cp_wait<0>();
    }
    if ((MODE == EPI_RESID || MODE == EPI_LIN) && ep.partial) {
        sq = block_sum(sq);
        if (tid == 0)
            ep.partial[((long long)b * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = sq;
    }
}

int take_fault_cfd(int* code) { return take_unit_fault(code); }

// The halo cells past a periodic edge in the busiest tile (what the TMA
// variant of k_fd_cfd deals to its threads; the same count as the kernel's).
static int cfd_wrapped_max(const GridBC& g, int NN, int TX, int TY) {
    int best = 0;
    for (int y0 = 0; y0 < g.n[1]; y0 += TY)
        for (int x0 = 0; x0 < g.n[2]; x0 += TX) {
            const int rb0 = std::max(-NN, -y0), rb1 = std::min(TY + NN, g.n[1] - y0);
            const int cb0 = std::max(-NN, -x0), cb1 = std::min(TX + NN, g.n[2] - x0);
            const int ncolA = std::max(0, std::min(TX, cb1) - std::max(0, cb0));
            const int nA = g.periodic[1] ? ((TY + 2 * NN) - (rb1 - rb0)) * ncolA : 0;
            const int nrowB = std::max(0, std::min(TY, rb1) - std::max(0, rb0));
            const int nB = g.periodic[2] ? nrowB * ((TX + 2 * NN) - (cb1 - cb0)) : 0;
            best = std::max(best, nA + nB);
        }
    return best;
}

bool tma_enabled();   // gb_transform.cu

template <class T, int NN, int TX, int TY, int RY, int D, int MODE, int ORD, int LD, int MINB>
static int launch_cfd_t(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
                        const CfdStencil& cs, const Epi& ep, cudaStream_t st, int* nblk) {
    constexpr int PX = TX + 2 * NN, PY = TY + 2 * NN, S = NN + 1 + D;
    constexpr int SP = LD ? (PX * PY + 7) / 8 * 8 : PX * PY;
    constexpr size_t smem =
        (size_t)S * SP * sizeof(T) + (LD ? S * sizeof(uint64_t) + 128 : 0);
    CUtensorMap map;
    memset(&map, 0, sizeof map);
    if constexpr (LD == 1) {
        constexpr int NT = TX * (TY / RY);
        constexpr int NWR = (2 * NN * (TX + TY) + NT - 1) / NT;
        if (cfd_wrapped_max(g, NN, TX, TY) > NWR * NT) return 1;   // not this kernel
        const char* why = nullptr;
        if (make_plane_map16(&map, in, nin, g.n[0], g.n[1], g.n[2], PY, PX, &why)) return 1;
    }
    static bool attr_done = false;
    if (!attr_done) {
        cudaError_t e = cudaFuncSetAttribute(k_fd_cfd<T, NN, TX, TY, RY, D, MODE, ORD, LD, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return -2;
        attr_done = true;
    }
    const int tiles_x = (g.n[2] + TX - 1) / TX;
    const int tiles_y = (g.n[1] + TY - 1) / TY;
    const int chunk0 = ep.chunk > 0 ? min(ep.chunk, g.n[0]) : cfd_chunk(g, NN, nin, TY);
    const int nch = (g.n[0] + chunk0 - 1) / chunk0;
    if (nblk) *nblk = tiles_x * tiles_y * nch;
    const long long ng = (long long)g.n[0] * g.n[1] * g.n[2];
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(tiles_x * tiles_y, nch, nb);
        Epi e2 = ep;
        if (e2.aux) e2.aux = (const T*)ep.aux + b0 * ng;
        if (e2.partial) e2.partial = ep.partial + (long long)b0 * tiles_x * tiles_y * nch;
        k_fd_cfd<T, NN, TX, TY, RY, D, MODE, ORD, LD, MINB><<<grid, TX * (TY / RY), smem, st>>>(
            (const T*)in + b0 * ng, out ? (T*)out + b0 * ng : nullptr, nb, g, P, cs, chunk0,
            tiles_x, e2, map, b0);
    }
    return 0;
}

// Tile shapes: 32 columns per warp row; f64 threads own 4 rows, complex 2.
template <class T, int NN, int MODE>
static int launch_cfd_nn(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
                         const CfdStencil& cs, const Epi& ep, cudaStream_t st, int* nblk) {
    // only the direction order GUCLaplace builds (axis 2, 1, 0); other
    // axis-aligned stencils take the generic kernel
    if (!(cs.axis[0] == 2 && cs.axis[1] == 1 && cs.axis[2] == 0)) return -1;
    // rows per thread: fewer when the epilogue reads other arrays (their
    // prefetched values need registers too)
    constexpr bool AUX = MODE != EPI_APPLY;
    if constexpr (sizeof(T) == 16) {
        // 32 x 8 tiles, one row a thread: 80 registers and 60 KB of ring
        // (nn = 3) let three CTAs share an SM; measured faster than 32 x 16
        // tiles of two rows a thread at two CTAs an SM (the rows' shared
        // axis-1 loads do not make up for the lost warps)
        constexpr int D = NN <= 3 ? 2 : 2;
        constexpr int MB = (NN <= 3 && (MODE == EPI_APPLY || MODE == EPI_POT)) ? 4 : 2;
        if constexpr (MODE == EPI_APPLY && NN == 3)
            if (fused_apply())
                return launch_cfd_t<T, NN, 32, 8, 1, D, MODE, 2, 0, MB>(in, out, nin, g, P, cs,
                                                                         ep, st, nblk);
        if (tma_enabled()) {
            int rc = 1;
            if constexpr (NN <= 3 && MODE != EPI_RESID) {
                // two rows a thread share their axis-1 neighbours: fewer
                // shared-memory reads per point (variant picked by
                // GPAW_B200_CFD_VARIANT while the shapes are measured)
                static const int var = [] {
                    const char* e = getenv("GPAW_B200_CFD_VARIANT");
                    return e ? atoi(e) : 0;
                }();
                if (var == 1)
                    rc = launch_cfd_t<T, NN, 32, 8, 2, D, MODE, 1, 1, 4>(in, out, nin, g, P, cs,
                                                                         ep, st, nblk);
                else if (var == 2)
                    rc = launch_cfd_t<T, NN, 32, 16, 2, D, MODE, 1, 1, 2>(in, out, nin, g, P, cs,
                                                                          ep, st, nblk);
                else if (var == 3)
                    rc = launch_cfd_t<T, NN, 32, 8, 2, 1, MODE, 1, 1, 4>(in, out, nin, g, P, cs,
                                                                         ep, st, nblk);
            }
            if (rc == 1)
                rc = launch_cfd_t<T, NN, 32, 8, 1, D, MODE, 1, 1, MB>(in, out, nin, g, P, cs,
                                                                       ep, st, nblk);
            if (rc <= 0) return rc;
        }
        return launch_cfd_t<T, NN, 32, 8, 1, D, MODE, 1, 0, MB>(in, out, nin, g, P, cs, ep, st,
                                                                 nblk);
    } else {
        constexpr int RY = (NN <= 3 && !AUX) ? 4 : 2;
        // nn = 3: three planes ahead makes the ring exactly 2nn+1 deep, so
        // every ring slot in the unrolled march is a constant
        constexpr int D = NN == 3 ? 3 : 4;
        // float64: 32 x 8 tiles of two rows a thread (128 threads, more
        // CTAs an SM) measured faster than 32 x 16 tiles (nn = 3 apply
        // 14 %, preconditioner 9 %, FP64 V-cycles 3-7 %)
        // split sums for the FP64 defect of the mixed solver (measured
        // faster there); the FP32 levels keep one chain (measured slower
        // with three: more registers)
        constexpr int ORDL = (MODE == EPI_LIN && sizeof(T) == 8) ? 3 : 1;
        if constexpr (MODE == EPI_LIN) {
            // tile shapes of the mixed solver's passes under measurement
            // (GPAW_B200_LIN_VARIANT): 1 = one row a thread, 32 x 8 tiles
            static const int var = [] {
                const char* e = getenv("GPAW_B200_LIN_VARIANT");
                return e ? atoi(e) : 0;
            }();
            if (var == 1) {
                if constexpr (sizeof(T) == 8)
                    return launch_cfd_t<T, NN, 32, 8, 1, D, MODE, ORDL, 0, 3>(in, out, nin, g, P,
                                                                              cs, ep, st, nblk);
                else
                    return launch_cfd_t<T, NN, 32, 8, 1, D, MODE, ORDL, 0, 4>(in, out, nin, g, P,
                                                                              cs, ep, st, nblk);
            }
            if (var == 2) {
                if constexpr (sizeof(T) == 8)
                    return launch_cfd_t<T, NN, 32, 8, 1, D, MODE, ORDL, 0, 3>(in, out, nin, g, P,
                                                                              cs, ep, st, nblk);
                else
                    return launch_cfd_t<T, NN, 32, 16, RY, D, MODE, ORDL, 0, 3>(
                        in, out, nin, g, P, cs, ep, st, nblk);
            }
        }
        if constexpr (sizeof(T) == 8)
            return launch_cfd_t<T, NN, 32, 8, 2, D, MODE, ORDL, 0, 4>(in, out, nin, g, P, cs, ep,
                                                                      st, nblk);
        return launch_cfd_t<T, NN, 32, 16, RY, D, MODE, ORDL, 0, 512 / (32 * (16 / RY))>(
            in, out, nin, g, P, cs, ep, st, nblk);
    }
}

template <class T, int MODE>
static int launch_cfd_mode(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
                           const CfdStencil& cs, int nn, const Epi& ep, cudaStream_t st,
                           int* nblk) {
    switch (nn) {
        case 1: return launch_cfd_nn<T, 1, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
        case 2: return launch_cfd_nn<T, 2, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
        case 3: return launch_cfd_nn<T, 3, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
        case 4: return launch_cfd_nn<T, 4, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
        case 5: return launch_cfd_nn<T, 5, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
        case 6: return launch_cfd_nn<T, 6, MODE>(in, out, nin, g, P, cs, ep, st, nblk);
    }
    return -1;
}

template <class T>
int launch_fd_cfd(int mode, const void* in, void* out, int nin, const GridBC& g,
                  const Phases& P, const CfdStencil& cs, int nn, const Epi& ep,
                  cudaStream_t st, int* nblk) {
    switch (mode) {
        case EPI_APPLY: return launch_cfd_mode<T, EPI_APPLY>(in, out, nin, g, P, cs, nn, ep, st, nblk);
        case EPI_RESID:
            if constexpr (sizeof(T) == 4) return -1;
            else return launch_cfd_mode<T, EPI_RESID>(in, out, nin, g, P, cs, nn, ep, st, nblk);
        case EPI_PRECOND:
            if constexpr (sizeof(T) == 4) return -1;
            else return launch_cfd_mode<T, EPI_PRECOND>(in, out, nin, g, P, cs, nn, ep, st, nblk);
        case EPI_LIN:
            if constexpr (sizeof(T) == 16) return -1;
            else return launch_cfd_mode<T, EPI_LIN>(in, out, nin, g, P, cs, nn, ep, st, nblk);
        case EPI_JACOBI:
            if constexpr (sizeof(T) != 8) return -1;
            else return launch_cfd_mode<T, EPI_JACOBI>(in, out, nin, g, P, cs, nn, ep, st, nblk);
        case EPI_POT:
            if constexpr (sizeof(T) == 4) return -1;
            else return launch_cfd_mode<T, EPI_POT>(in, out, nin, g, P, cs, nn, ep, st, nblk);
    }
    return -1;
}

template int launch_fd_cfd<double>(int, const void*, void*, int, const GridBC&, const Phases&,
                                   const CfdStencil&, int, const Epi&, cudaStream_t, int*);
template int launch_fd_cfd<double2>(int, const void*, void*, int, const GridBC&, const Phases&,
                                    const CfdStencil&, int, const Epi&, cudaStream_t, int*);
template int launch_fd_cfd<float>(int, const void*, void*, int, const GridBC&, const Phases&,
                                  const CfdStencil&, int, const Epi&, cudaStream_t, int*);

// Number of CTAs per grid of the EPI_RESID launch (partials per grid).
int cfd_blocks(const GridBC& g, int nn, int elem_bytes, int nin, int chunk) {
    // the tile of launch_cfd_nn: 32 x 16 for float, 32 x 8 otherwise
    const int TX = 32, TY = elem_bytes == 4 ? 16 : 8;
    const int tiles_x = (g.n[2] + TX - 1) / TX;
    const int tiles_y = (g.n[1] + TY - 1) / TY;
    const int chunk0 = chunk > 0 ? std::min(chunk, g.n[0]) : cfd_chunk(g, nn, nin, TY);
    return tiles_x * tiles_y * ((g.n[0] + chunk0 - 1) / chunk0);
}

// Recognise the GUCLaplace layout of an axis-aligned stencil: centre first,
// then three directions, each +1..+nn followed by -1..-nn along one axis.
bool to_cfd_stencil(const Stencil& s, CfdStencil& cs, int& nn) {
    if (!s.cfd) return false;
    const int n = (s.ncoefs - 1) / 6;
    if (n < 1 || n > 6 || s.ncoefs != 6 * n + 1 || s.range != n) return false;
    if (s.off[0][0] || s.off[0][1] || s.off[0][2]) return false;
    cs.c0 = s.coef[0];
    int used = 0;
    for (int k = 0; k < 3; k++) {
        const int base = 1 + k * 2 * n;
        int ax = -1;
        for (int c = 0; c < 3; c++)
            if (s.off[base][c] != 0) ax = c;
        if (ax < 0 || (used >> ax) & 1) return false;
        used |= 1 << ax;
        cs.axis[k] = ax;
        for (int d = 1; d <= n; d++) {
            const int ip = base + d - 1, im = base + n + d - 1;
            for (int c = 0; c < 3; c++) {
                if (s.off[ip][c] != (c == ax ? d : 0)) return false;
                if (s.off[im][c] != (c == ax ? -d : 0)) return false;
            }
            cs.cp[k][d - 1] = s.coef[ip];
            cs.cm[k][d - 1] = s.coef[im];
        }
    }
    nn = n;
    return true;
}

}  // namespace gb
