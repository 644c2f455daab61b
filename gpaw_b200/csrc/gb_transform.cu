// Restriction (fine -> coarse) and interpolation (coarse -> fine) between
// grids whose point counts differ by 2 along every axis.
//
// The reference (c/transformers.cpp:38-109) pads the input into a halo
// buffer (bc_init with cfd = 0, so edges and corners are filled too,
// c/transformers.cpp:230) and then runs three separable 1-D passes with
// transpose-on-write: along axis 2, then axis 1, then axis 0
// (c/bmgs/restrict.cpp:137-156, c/bmgs/interpolate.cpp:70-99), each pass
// writing a full intermediate array.
//
// Here one kernel does all three passes.  A CTA owns a TJ x TK tile of the
// output in axes (1, 2) and a chunk of axis 0.  It marches over the padded
// input planes along axis 0; for each plane it loads the tile's input
// footprint (halo resolved in the load path), runs the axis-2 pass and the
// axis-1 pass in shared memory, and pushes the result into a per-thread ring
// of recent planes, from which the axis-0 pass produces finished outputs.
// Every intermediate value is formed with the same operations in the same
// order as in the reference's passes, so outputs are bit-identical.
#include <algorithm>
#include <cstring>

#include "gb_internal.cuh"
#include "gb_tma.cuh"

namespace gb {

// ----------------------------------------------------------------- restrict
// out[I][J][L] over padded input a:  per axis, r(c) = 0.5 * (a[c] + sum_l
// w_l * (a[c + 2l + 1] + a[c - 2l - 1])) at c = K - 1 + 2 I  (RST1D,
// c/bmgs/restrict.cpp:18-60), applied along axis 2, then 1, then 0.
//
// Fine padded planes stream through a ring of S shared-memory stages filled
// by cp.async D planes ahead.  A stage holds the tile's footprint row-major
// with an odd row pitch, so consecutive lanes copy consecutive global and
// shared addresses (full L2 requests).  The axis-2 pass, whose outputs read
// every second column, gives each bank phase of a warp half its lanes on
// one row and half on the next: the odd pitch puts the two halves on
// disjoint banks, and every read is the thread's base plus a constant.

__device__ __forceinline__ unsigned smem_u32x(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async_x(void* sdst, const void* gsrc, bool valid) {
    const unsigned s = smem_u32x(sdst);
    const int n = valid ? BYTES : 0;
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(n));
    else if (BYTES == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(n));
}
__device__ __forceinline__ void cp_commit_x() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait_x() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ bool wrap_c(int& y, int n, int periodic) {
    if (y >= 0 && y < n) return true;
    if (!periodic) return false;
    if (y < 0) y += n;
    else y -= n;
    return y >= 0 && y < n;
}

// Phase code of a cell: bits 0-1 axis 1 (0 none, 1 past high edge, 2 past
// low edge), bits 2-3 axis 2.  Phases compose in axis order (the halo is
// filled axis by axis with cfd = 0, c/bc.cpp:108-112, 242-257).
template <class T>
__device__ __forceinline__ T apply_code(T v, unsigned c, bool plane_wrap, double2 ph0,
                                        const Phases& P) {
    if constexpr (sizeof(T) == 16) {
        if (plane_wrap) v = cmul(ph0, v);
        const unsigned c1 = c & 3u, c2 = (c >> 2) & 3u;
        if (c1) v = cmul(c1 == 1 ? P.ph[1][0] : P.ph[1][1], v);
        if (c2) v = cmul(c2 == 1 ? P.ph[2][0] : P.ph[2][1], v);
    }
    return v;
}

template <class T, int K, int TJ, int TK, int D>
__global__ void __launch_bounds__(TJ * TK, 3)
k_restrict(const T* __restrict__ in, T* __restrict__ out, T* __restrict__ out2, int nin,
           XferGeom G, Phases P, int chunk0) {
    constexpr int NT = TJ * TK;
    constexpr int H = 2 * K - 3;
    constexpr int FY = 2 * TJ + H;        // fine rows needed by the tile
    constexpr int FZ = 2 * TK + H;        // fine columns needed by the tile
    constexpr int SS = FY * FZ;           // one stage (elements); FZ is odd
    // lanes of one shared-memory bank phase (16-byte words: 8, 8-byte: 16,
    // 4-byte: 32) and the R1 pitch that keeps a phase's two rows apart
    constexpr int PG = sizeof(T) == 16 ? 8 : (sizeof(T) == 8 ? 16 : 32);
    constexpr int HG = PG / 2;
    // (16-byte elements: pitch TK, which costs a two-way conflict on the R1
    // writes but keeps three CTAs in the shared memory of an SM)
    constexpr int RP = sizeof(T) == 16 ? TK : TK + HG;
    constexpr int S = D + 1;              // ring depth
    constexpr int NR = 2 * K - 1;         // axis-0 ring depth
    constexpr int NC = (FY * FZ + NT - 1) / NT;
    constexpr int EB = (int)sizeof(T);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* stage = reinterpret_cast<T*>(smem_raw);
    T* R1 = stage + S * SS;               // [2][FY][RP]

    const int tiles2 = (G.nout[2] + TK - 1) / TK;
    const int J0 = (blockIdx.x / tiles2) * TJ;
    const int L0 = (blockIdx.x % tiles2) * TK;
    const int I0 = blockIdx.y * chunk0;
    const int I1 = min(G.nout[0], I0 + chunk0);
    const int b = blockIdx.z;
    if (I0 >= I1 || b >= nin) return;
    const int n1 = G.g.n[1], n2 = G.g.n[2];
    const long long ngin = (long long)G.g.n[0] * n1 * n2;
    const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
    const T* a = in + b * ngin;
    T* o = out + b * ngout;
    const int tid = threadIdx.x;
    const int tj = tid / TK, tk = tid % TK;
    const bool cplx = sizeof(T) == 16 && P.use;

    // this thread's footprint cells: stage offset, in-plane source offset,
    // validity, phase code
    int soff[NC], goff[NC];
    unsigned vmask = 0, pcode = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const int e = tid + i * NT;
        soff[i] = 0;
        goff[i] = 0;
        if (e >= FY * FZ) continue;
        const int y = e / FZ, z = e % FZ;
        soff[i] = e;
        const int py = 2 * J0 + y, pz = 2 * L0 + z;
        if (py >= G.s[1] || pz >= G.s[2]) continue;
        int iy = py - G.plo[1], iz = pz - G.plo[2];
        const unsigned c1 = iy >= n1 ? 1u : (iy < 0 ? 2u : 0u);
        const unsigned c2 = iz >= n2 ? 1u : (iz < 0 ? 2u : 0u);
        if (wrap_c(iy, n1, G.g.periodic[1]) && wrap_c(iz, n2, G.g.periodic[2])) {
            vmask |= 1u << i;
            goff[i] = iy * n2 + iz;
            pcode |= (c1 | (c2 << 2)) << (4 * i);
        }
    }
    if (!cplx) pcode = 0;

    // padded plane range for outputs [I0, I1): 2*I0 .. 2*(I1-1) + 2K - 2
    const int x0a = 2 * I0;
    const int nx = 2 * (I1 - I0) + 2 * K - 3;
    auto plane_info = [&](int j, int& ip, int& wrapside) {
        ip = x0a + j - G.plo[0];
        wrapside = ip >= G.g.n[0] ? 0 : (ip < 0 ? 1 : -1);
        return wrap_c(ip, G.g.n[0], G.g.periodic[0]);
    };
    // slot: j % S, kept by the caller as a running counter
    auto issue = [&](int j, int slot) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        T* st = stage + slot * SS;
        // a plane outside a zero boundary copies nothing (size 0) from
        // plane 0's cells, which always exist
        const T* src = pv ? a + (long long)ip * n1 * n2 : a;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= FY * FZ) break;
            cp_async_x<EB>(st + soff[i], src + goff[i], pv && ((vmask >> i) & 1));
        }
    };
    auto fixup = [&](int j, int slot) {
        int ip, ws;
        plane_info(j, ip, ws);
        T* st = stage + slot * SS;
        const bool pw = cplx && ws >= 0 && G.g.periodic[0];
        if (!pw && !pcode) return;
        const double2 ph0 = ws == 0 ? P.ph[0][0] : P.ph[0][1];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= FY * FZ) break;
            const unsigned c = (pcode >> (4 * i)) & 15u;
            if ((pw || c) && ((vmask >> i) & 1))
                st[soff[i]] = apply_code<T>(st[soff[i]], c, pw, ph0, P);
        }
    };

    T ring[NR];
#pragma unroll
    for (int i = 0; i < NR; i++) ring[i] = Num<T>::zero();

    // axis-2 pass of plane t: R1[t & 1][y][k], centre at odd column K-1+2k.
    // Items come in blocks of two rows x TK columns; within a block, a bank
    // phase takes HG consecutive columns of both rows.
    constexpr int NE2 = ((FY + 1) / 2) * 2 * TK;
    constexpr int NR2 = (NE2 + NT - 1) / NT;
    int foff[NR2], roff[NR2];     // this thread's axis-2 items: stage / R1 offsets
    unsigned imask = 0;
#pragma unroll
    for (int r = 0; r < NR2; r++) {
        const int e = tid + r * NT;
        const int j = e % (2 * TK);
        const int k = (j / PG) * HG + j % HG;
        const int y = 2 * (e / (2 * TK)) + (j / HG) % 2;
        foff[r] = y * FZ + K - 1 + 2 * k;
        roff[r] = y * RP + k;
        if ((NE2 % NT == 0 || e < NE2) && y < FY) imask |= 1u << r;
    }
    auto axis2 = [&](int t, int slot) {
        const T* F = stage + slot * SS;
        T* R = R1 + (t & 1) * (FY * RP);
#pragma unroll
        for (int r = 0; r < NR2; r++) {
            if ((imask >> r) & 1) {
                const T* f = F + foff[r];
                T x = f[0];
#pragma unroll
                for (int l = 0; l < K / 2; l++)
                    x = Num<T>::add(x, Num<T>::scale(Num<T>::add(f[2 * l + 1], f[-2 * l - 1]),
                                                     G.w[l]));
                // restrict(-a) == -restrict(a) bit for bit (every step is odd)
                const T v = Num<T>::scale(x, 0.5);
                R[roff[r]] = G.neg_in ? Num<T>::neg(v) : v;
            }
        }
    };
    // axis-1 pass of plane t for this thread's (j, k), into the axis-0 ring;
    // the axis-0 pass once the ring spans planes 2I .. 2I + 2K - 2.  Planes
    // enter in pairs (odd, even): an odd plane waits in `pend`; an even one
    // shifts the ring by two and fills its last two entries, so the ring
    // holds planes t - NR + 1 .. t whenever t is even.
    T pend = Num<T>::zero();
    auto axis10 = [&](int t) {
        const T* R = R1 + (t & 1) * (FY * RP) + (K - 1 + 2 * tj) * RP + tk;
        T x = R[0];
#pragma unroll
        for (int l = 0; l < K / 2; l++)
            x = Num<T>::add(x, Num<T>::scale(Num<T>::add(R[(2 * l + 1) * RP],
                                                         R[-(2 * l + 1) * RP]),
                                             G.w[l]));
        if (t & 1) {
            pend = Num<T>::scale(x, 0.5);
            return;
        }
#pragma unroll
        for (int i = 0; i < NR - 2; i++) ring[i] = ring[i + 2];
        ring[NR - 2] = pend;
        ring[NR - 1] = Num<T>::scale(x, 0.5);
        if (t >= 2 * K - 2) {
            const int I = I0 + (t - (2 * K - 2)) / 2;
            const int J = J0 + tj, L = L0 + tk;
            T y = ring[K - 1];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                y = Num<T>::add(y, Num<T>::scale(Num<T>::add(ring[K - 1 + 2 * l + 1],
                                                             ring[K - 1 - 2 * l - 1]),
                                                 G.w[l]));
            if (J < G.nout[1] && L < G.nout[2]) {
                const long long at = ((long long)I * G.nout[1] + J) * G.nout[2] + L;
                const T r = Num<T>::scale(y, 0.5);
                o[at] = r;
                // fd_precond's "d = 4 * step * r" (c/fd_preconditioner.cpp:222-226)
                if (out2) out2[b * ngout + at] = Num<T>::scale(r, G.scale2);
            }
        }
    };

    // One barrier per plane: after barrier t, stage t+1 and R1[t & 1] are
    // visible, so the axis-2 pass of plane t+1 (into the other R1 buffer)
    // and the axis-1/axis-0 passes of plane t run in the same interval.
    // R1[(t+1) & 1] was last read by the axis-1 pass of plane t-1 and stage
    // slot t % S by the axis-2 pass of plane t, both before barrier t.
#pragma unroll 1
    for (int j = 0; j < D; j++) {
        if (j < nx) issue(j, j);
        cp_commit_x();
    }
    cp_wait_x<D - 1>();
    fixup(0, 0);
    __syncthreads();
    if (D < nx) issue(D, D);
    cp_commit_x();
    axis2(0, 0);
    // ring slots of planes t and t + 1 (mod S), advanced each iteration
    int s_t = 0, s_n = 1 % S;
#pragma unroll 1
    for (int t = 0; t < nx; t++) {
        cp_wait_x<D - 1>();
        if (t + 1 < nx) fixup(t + 1, s_n);
        __syncthreads();
        // plane t + 1 + D goes into slot (t + 1 + D) % S = t % S
        if (t + 1 + D < nx) issue(t + 1 + D, s_t);
        cp_commit_x();
        if (t + 1 < nx) axis2(t + 1, s_n);
        axis10(t);
        s_t = s_n;
        s_n = s_n + 1 == S ? 0 : s_n + 1;
    }
    cp_wait_x<0>();
}

// ------------------------------------------- restrict, TMA plane windows
// The same restriction for complex128 grids, with each padded input plane's
// window brought into shared memory by one TMA tensor copy instead of
// per-thread cp.async cells.  The window starts at the tile's footprint
// origin; the parts outside the grid arrive as zeros.  What the TMA cannot
// do is done by the threads afterwards, per plane:
//  * cells past a periodic edge of axis 1 or 2 (the "wrapped" cells, only
//    in tiles at an edge): loaded from the opposite side one plane ahead
//    (into registers) and stored with their Bloch phases;
//  * a plane past a periodic edge of axis 0: every in-grid cell is
//    multiplied by that axis's phase.
// The wrapped cells of a tile are enumerated compactly (rows past the edge,
// then columns past the edge of the other rows) and dealt to the threads,
// at most NWR a thread; the launcher checks the count.
template <int K, int TJ, int TK, int D, int NWR, int MINB>
__global__ void __launch_bounds__(TJ * TK, MINB)
k_restrict_tma(const __grid_constant__ CUtensorMap map, const double2* __restrict__ in,
               double2* __restrict__ out, double2* __restrict__ out2, int nin, int b0,
               XferGeom G, Phases P, int chunk0) {
    using T = double2;
    constexpr int NT = TJ * TK;
    constexpr int H = 2 * K - 3;
    constexpr int FY = 2 * TJ + H;        // fine rows needed by the tile
    constexpr int FZ = 2 * TK + H;        // fine columns needed by the tile
    constexpr int SS = FY * FZ;           // one window (elements)
    constexpr int SSP = (SS + 7) / 8 * 8; // stage stride: 128-byte aligned
    constexpr int RP = TK + 1;            // odd: a warp's rows hit distinct banks
    constexpr int S = D + 1;              // ring depth
    constexpr int NR = 2 * K - 1;         // axis-0 ring depth
    constexpr int NC = (SS + NT - 1) / NT;
    constexpr unsigned WBYTES = SS * 16;
    extern __shared__ __align__(128) unsigned char smem_tma[];
    const unsigned mis = tma_smem_u32(smem_tma) & 127u;
    T* stage = reinterpret_cast<T*>(smem_tma + (mis ? 128 - mis : 0));
    T* R1 = stage + S * SSP;              // [2][FY][RP]
    uint64_t* bar = reinterpret_cast<uint64_t*>(R1 + 2 * FY * RP);

    const int tiles2 = (G.nout[2] + TK - 1) / TK;
    const int J0 = (blockIdx.x / tiles2) * TJ;
    const int L0 = (blockIdx.x % tiles2) * TK;
    const int I0 = blockIdx.y * chunk0;
    const int I1 = min(G.nout[0], I0 + chunk0);
    const int bg = b0 + blockIdx.z;
    if (I0 >= I1 || (int)blockIdx.z >= nin) return;
    const int n0 = G.g.n[0], n1 = G.g.n[1], n2 = G.g.n[2];
    const long long psz = (long long)n1 * n2;
    const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
    const T* a = in + (long long)bg * n0 * psz;
    T* o = out + (long long)bg * ngout;
    const int tid = threadIdx.x;
    const int tj = tid / TK, tk = tid % TK;
    const bool cplx = P.use != 0;
    // interior coordinates of the window's first row and column
    const int row0 = 2 * J0 - G.plo[1], col0 = 2 * L0 - G.plo[2];

    // this thread's in-grid cells (for the phase of a wrapped plane)
    unsigned inmask = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const int e = tid + i * NT;
        if (e < SS) {
            const int iy = row0 + e / FZ, iz = col0 + e % FZ;
            if (iy >= 0 && iy < n1 && iz >= 0 && iz < n2) inmask |= 1u << i;
        }
    }
    // wrapped cells: rows [0, ra) and [rb, FY) are past axis 1's edges,
    // columns [0, ca) and [cb, FZ) past axis 2's
    const int ra = min(max(-row0, 0), FY), rb = min(max(n1 - row0, ra), FY);
    const int ca = min(max(-col0, 0), FZ), cb = min(max(n2 - col0, ca), FZ);
    const int nA = G.g.periodic[1] ? (ra + FY - rb) * FZ : 0;
    const int nBc = G.g.periodic[2] ? ca + FZ - cb : 0;
    const int nB = (rb - ra) * nBc;
    int wso[NWR], wgo[NWR];
    unsigned wmask = 0, wcode = 0;
#pragma unroll
    for (int r = 0; r < NWR; r++) {
        const int w = tid + r * NT;
        wso[r] = 0;
        wgo[r] = 0;
        int y, z;
        if (w < nA) {
            const int q = w / FZ;
            z = w % FZ;
            y = q < ra ? q : rb + (q - ra);
        } else if (w < nA + nB) {
            const int w2 = w - nA;
            const int q = w2 / nBc, c = w2 % nBc;
            y = ra + q;
            z = c < ca ? c : cb + (c - ca);
        } else {
            continue;
        }
        int iy = row0 + y, iz = col0 + z;
        const unsigned c1 = iy >= n1 ? 1u : (iy < 0 ? 2u : 0u);
        const unsigned c2 = iz >= n2 ? 1u : (iz < 0 ? 2u : 0u);
        if (wrap_c(iy, n1, G.g.periodic[1]) && wrap_c(iz, n2, G.g.periodic[2])) {
            wmask |= 1u << r;
            wso[r] = y * FZ + z;
            wgo[r] = iy * n2 + iz;
            wcode |= (c1 | (c2 << 2)) << (4 * r);
        }
    }
    if (!cplx) wcode = 0;

    // padded plane range for outputs [I0, I1): 2*I0 .. 2*(I1-1) + 2K - 2
    const int x0a = 2 * I0;
    const int nx = 2 * (I1 - I0) + 2 * K - 3;
    auto plane_info = [&](int j, int& ip, int& wrapside) {
        ip = x0a + j - G.plo[0];
        wrapside = ip >= n0 ? 0 : (ip < 0 ? 1 : -1);
        return wrap_c(ip, n0, G.g.periodic[0]);
    };
    // thread 0: the window of plane j into stage j % S
    auto issue = [&](int j) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        const int slot = j % S;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[slot], WBYTES);
        // a plane past a zero boundary: a window outside the tensor (zeros)
        tma_load_window16(stage + slot * SSP, &map, col0, row0, pv ? ip : -1, bg, &bar[slot]);
    };
    T pre[NWR];
    auto load_wrapped = [&](int j) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        const T* src = a + (long long)(pv ? ip : 0) * psz;
#pragma unroll
        for (int r = 0; r < NWR; r++)
            pre[r] = (pv && ((wmask >> r) & 1)) ? __ldg(src + wgo[r]) : Num<T>::zero();
    };
    auto fixup = [&](int j, int slot) {
        int ip, ws;
        if (!plane_info(j, ip, ws)) return;
        T* st = stage + slot * SSP;
        const bool pw = cplx && ws >= 0;
        const double2 ph0 = ws == 0 ? P.ph[0][0] : P.ph[0][1];
        if (pw) {
#pragma unroll
            for (int i = 0; i < NC; i++)
                if ((inmask >> i) & 1) st[tid + i * NT] = cmul(ph0, st[tid + i * NT]);
        }
#pragma unroll
        for (int r = 0; r < NWR; r++)
            if ((wmask >> r) & 1)
                st[wso[r]] = apply_code<T>(pre[r], (wcode >> (4 * r)) & 15u, pw, ph0, P);
    };

    T ring[NR];
#pragma unroll
    for (int i = 0; i < NR; i++) ring[i] = Num<T>::zero();
    // axis-2 pass: a thread makes four neighbouring outputs of one row
    // (columns 4g .. 4g+3 of the tile), reading the K + 3 even columns
    // 8g, 8g + 2, ..., 8g + 2K + 4 they share and their four centres
    // 8g + K - 1 + {0, 2, 4, 6}: K + 7 reads instead of 4 (K + 1).
    // Consecutive lanes take consecutive rows; the odd row pitch FZ puts
    // the eight lanes of a bank phase on distinct banks.
    constexpr int G4 = TK / 4;
    constexpr int NI2 = FY * G4;                   // items per plane
    static_assert(NI2 <= NT, "one axis-2 item per thread at most");
    const bool has2 = tid < NI2;
    const int y2 = tid % FY, g2 = tid / FY;
    const int foff = y2 * FZ + 8 * g2;             // first even column
    const int roff = y2 * RP + 4 * g2;
    auto axis2 = [&](int t, int slot) {
        if (!has2) return;
        const T* f = stage + slot * SSP + foff;
        T* R = R1 + (t & 1) * (FY * RP) + roff;
        // a window of K even columns slides one step per output
        T ev[K];
#pragma unroll
        for (int q = 0; q < K; q++) ev[q] = f[2 * q];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            // centre 2i + K - 1; its pairs at +-(2l + 1) are the even
            // columns 2i + K + 2l and 2i + K - 2 - 2l: window slots
            // K/2 + l and K/2 - 1 - l
            T x = f[2 * i + K - 1];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(ev[K / 2 + l], ev[K / 2 - 1 - l]),
                                                 G.w[l]));
            const T v = Num<T>::scale(x, 0.5);
            R[i] = G.neg_in ? Num<T>::neg(v) : v;
            if (i < 3) {
#pragma unroll
                for (int q = 0; q < K - 1; q++) ev[q] = ev[q + 1];
                ev[K - 1] = f[2 * (i + K)];
            }
        }
    };
    T pend = Num<T>::zero();
    auto axis10 = [&](int t) {
        const T* R = R1 + (t & 1) * (FY * RP) + (K - 1 + 2 * tj) * RP + tk;
        T x = R[0];
#pragma unroll
        for (int l = 0; l < K / 2; l++)
            x = Num<T>::add(x, Num<T>::scale(Num<T>::add(R[(2 * l + 1) * RP],
                                                         R[-(2 * l + 1) * RP]),
                                             G.w[l]));
        if (t & 1) {
            pend = Num<T>::scale(x, 0.5);
            return;
        }
#pragma unroll
        for (int i = 0; i < NR - 2; i++) ring[i] = ring[i + 2];
        ring[NR - 2] = pend;
        ring[NR - 1] = Num<T>::scale(x, 0.5);
        if (t >= 2 * K - 2) {
            const int I = I0 + (t - (2 * K - 2)) / 2;
            const int J = J0 + tj, L = L0 + tk;
            T y = ring[K - 1];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                y = Num<T>::add(y, Num<T>::scale(Num<T>::add(ring[K - 1 + 2 * l + 1],
                                                             ring[K - 1 - 2 * l - 1]),
                                                 G.w[l]));
            if (J < G.nout[1] && L < G.nout[2]) {
                const long long at = ((long long)I * G.nout[1] + J) * G.nout[2] + L;
                const T r = Num<T>::scale(y, 0.5);
                o[at] = r;
                if (out2) out2[(long long)bg * ngout + at] = Num<T>::scale(r, G.scale2);
            }
        }
    };
    // after a wait ran out: every thread agrees (a barrier with a vote),
    // waits a little for the copies it may still have in flight, and leaves
    auto drain = [&](int j) {
        for (int q = j; q < min(nx, j + D); q++)
            mbar_wait(&bar[q % S], (unsigned)(q / S) & 1u, 100000000ull);
    };

    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < S; q++) mbar_init(&bar[q], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int j = 0; j < D && j < nx; j++) issue(j);
    load_wrapped(0);
    bool bad = !mbar_wait(&bar[0], 0u);
    if (!bad) fixup(0, 0);
    if (nx > 1) load_wrapped(1);
    fence_proxy_async_smem();
    if (__syncthreads_or(bad)) {
        drain(0);
        return;
    }
    if (tid == 0 && D < nx) issue(D);
    axis2(0, 0);
#pragma unroll 1
    for (int t = 0; t < nx; t++) {
        const int j = t + 1;
        if (j < nx) {
            bad = !mbar_wait(&bar[j % S], (unsigned)(j / S) & 1u);
            if (!bad) fixup(j, j % S);
            if (j + 1 < nx) load_wrapped(j + 1);
        }
        // this thread's shared-memory writes and reads of the slot that the
        // next copy overwrites come before that copy (async proxy)
        fence_proxy_async_smem();
        if (__syncthreads_or(bad)) {
            drain(j);
            return;
        }
        // plane j + D goes into slot t % S, whose plane t was read by the
        // axis-2 pass before this barrier
        if (tid == 0 && j + D < nx) issue(j + D);
        if (j < nx) axis2(j, j % S);
        axis10(t);
    }
}

// The wrapped cells of the busiest tile of a restriction (what
// k_restrict_tma deals to its threads).
static int restrict_wrapped_max(const XferGeom& G, int K, int TJ, int TK) {
    const int H = 2 * K - 3, FY = 2 * TJ + H, FZ = 2 * TK + H;
    int best = 0;
    for (int J0 = 0; J0 < G.nout[1]; J0 += TJ)
        for (int L0 = 0; L0 < G.nout[2]; L0 += TK) {
            const int row0 = 2 * J0 - G.plo[1], col0 = 2 * L0 - G.plo[2];
            const int ra = std::min(std::max(-row0, 0), FY);
            const int rb = std::min(std::max(G.g.n[1] - row0, ra), FY);
            const int ca = std::min(std::max(-col0, 0), FZ);
            const int cb = std::min(std::max(G.g.n[2] - col0, ca), FZ);
            const int nA = G.g.periodic[1] ? (ra + FY - rb) * FZ : 0;
            const int nB = G.g.periodic[2] ? (rb - ra) * (ca + FZ - cb) : 0;
            best = std::max(best, nA + nB);
        }
    return best;
}

int take_fault_transform(int* code) { return take_unit_fault(code); }

// TMA staging of complex restrictions: on unless GPAW_B200_TMA=0 (read at
// every launch, so that tests can compare both paths in one process).
bool tma_enabled() {
    const char* e = getenv("GPAW_B200_TMA");
    return e == nullptr || atoi(e) != 0;
}

template <int K, int D, int MINB>
static int launch_restrict_tma_v(const void* in, void* out, void* out2, int nin,
                                 const XferGeom& G, const Phases& P, cudaStream_t st) {
    constexpr int TJ = 16, TK = 16, NWR = 2;
    constexpr int H = 2 * K - 3, FY = 2 * TJ + H, FZ = 2 * TK + H;
    constexpr int SSP = (FY * FZ + 7) / 8 * 8;
    constexpr size_t smem = ((size_t)(D + 1) * SSP + (size_t)2 * FY * (TK + 1)) * 16 +
                            (D + 1) * sizeof(uint64_t) + 128;
    if (restrict_wrapped_max(G, K, TJ, TK) > NWR * TJ * TK) return 1;   // not this kernel
    CUtensorMap map;
    const char* why = nullptr;
    if (make_plane_map16(&map, in, nin, G.g.n[0], G.g.n[1], G.g.n[2], FY, FZ, &why)) return 1;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_restrict_tma<K, TJ, TK, D, NWR, MINB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -2;
        attr = true;
    }
    const int t1 = (G.nout[1] + TJ - 1) / TJ, t2 = (G.nout[2] + TK - 1) / TK;
    int chunk0 = G.nout[0];
    const long long tiles = (long long)t1 * t2 * nin;
    if (G.chunk > 0) chunk0 = std::min(G.chunk, G.nout[0]);
    else
        while (chunk0 > 4 && tiles * ((G.nout[0] + chunk0 - 1) / chunk0) < 148 * 4)
            chunk0 = (chunk0 + 1) / 2;
    const int nchunks = (G.nout[0] + chunk0 - 1) / chunk0;
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(t1 * t2, nchunks, nb);
        k_restrict_tma<K, TJ, TK, D, NWR, MINB><<<grid, TJ * TK, smem, st>>>(
            map, (const double2*)in, (double2*)out, (double2*)out2, nb, b0, G, P, chunk0);
    }
    return 0;
}

// Pipeline depth and occupancy of the TMA restriction: two planes ahead
// with two CTAs an SM for K >= 6 (measured on the 256 x 96^3 complex batch:
// 3130 GB/s, against 2190 GB/s one plane ahead with three CTAs, whose
// register cap spills), one plane ahead with three CTAs for K <= 4 (no
// spills there).  GPAW_B200_RST_DEPTH=1 or 2 overrides.
template <int K>
static int launch_restrict_tma(const void* in, void* out, void* out2, int nin,
                               const XferGeom& G, const Phases& P, cudaStream_t st) {
    static const int depth = [] {
        const char* e = getenv("GPAW_B200_RST_DEPTH");
        return e ? atoi(e) : 0;
    }();
    const bool deep = depth == 2 || (depth == 0 && K >= 6) || K >= 8;
    if (deep) return launch_restrict_tma_v<K, 2, 2>(in, out, out2, nin, G, P, st);
    return launch_restrict_tma_v<K, 1, 3>(in, out, out2, nin, G, P, st);
}

// -------------------------------------------------------------- interpolate
// IP1D (c/bmgs/interpolate.cpp:10-46): raw fine index u along an axis maps
// to coarse base m = K/2 - 1 + u/2 in the padded input; even u copies a[m],
// odd u gives sum_j w_j (a[m - j] + a[m + 1 + j]).  Fine index f = u - skip0.
// One interpolated value from a column of padded input `c` (stride apart):
// the even fine point copies c[0]; the odd one is
// sum_j w_j (c[-j] + c[1 + j]) in IP1D's order.
template <class T, int K>
__device__ __forceinline__ T ip_value(const T* c, int stride, bool odd, const double* w) {
    if (!odd) return c[0];
    T x = Num<T>::scale(Num<T>::add(c[0], c[stride]), w[0]);
#pragma unroll
    for (int j = 1; j < K / 2; j++)
        x = Num<T>::add(x, Num<T>::scale(Num<T>::add(c[-j * stride], c[(1 + j) * stride]), w[j]));
    return x;
}

// LD = 1 (complex data): each coarse plane's footprint window arrives by
// one TMA tensor copy (zeros past every edge), then the threads store the
// cells past a periodic edge of axis 1 or 2 (loaded one plane ahead) and,
// in a plane past a periodic edge of axis 0, multiply the in-grid cells by
// that axis's phase.  `map` covers the whole batch; `b0` is this launch's
// first grid in it.
template <class T, int K, int TJ, int TK, int D, int LD>
__global__ void __launch_bounds__(TJ * TK, 4)
k_interpolate(const T* __restrict__ in, T* __restrict__ out, int nin, XferGeom G, Phases P,
              int chunk0, const __grid_constant__ CUtensorMap map, int b0) {
    constexpr int NT = TJ * TK;
    constexpr int CY = TJ / 2 + K + 1;     // coarse rows feeding TJ fine rows
    constexpr int CZ = TK / 2 + K + 1;
    constexpr int SS = CY * CZ;
    constexpr int S = D + 1;
    constexpr int NC = (SS + NT - 1) / NT;
    // axis-2 items per thread: each warp takes items of one parity of the
    // fine index (copies or taps), so its lanes never diverge
    constexpr int NW = NT / 32;
    constexpr int NIP = CY * (TK / 2);                  // items per parity
    constexpr int NQ = (NIP + (NW / 2) * 32 - 1) / ((NW / 2) * 32);
    constexpr int EB = (int)sizeof(T);
    static_assert(LD == 0 || sizeof(T) == 16, "TMA windows: 16-byte elements only");
    constexpr int SSP = LD ? (SS + 7) / 8 * 8 : SS;   // stage stride (128-byte aligned)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* stage;
    if constexpr (LD == 1) {
        const unsigned mis = tma_smem_u32(smem_raw) & 127u;
        stage = reinterpret_cast<T*>(smem_raw + (mis ? 128 - mis : 0));
    } else {
        stage = reinterpret_cast<T*>(smem_raw);
    }
    T* Q = stage + S * SSP;                // [CY][TK]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Q + CY * TK);

    const int tiles2 = (G.nout[2] + TK - 1) / TK;
    const int F1 = (blockIdx.x / tiles2) * TJ;
    const int F2 = (blockIdx.x % tiles2) * TK;
    const int b = blockIdx.z;
    // pairs i along axis 0 handled by this CTA
    const int n0p = G.s[0] - (K - 1) + G.skip1[0];
    const int ia = blockIdx.y * chunk0;
    const int ib = min(n0p, ia + chunk0);
    if (ia >= ib || b >= nin) return;
    const int n1 = G.g.n[1], n2 = G.g.n[2];
    const long long ngin = (long long)G.g.n[0] * n1 * n2;
    const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
    const T* a = in + b * ngin;
    T* o = out + b * ngout;
    const int tid = threadIdx.x;
    const int bg = b0 + b;                 // this grid's index in the TMA map
    const int lane = tid & 31, wid = tid >> 5;
    // fine row of this thread: a warp's rows share the parity of their
    // fine index (two rows a warp for 16-wide tiles, one for 32-wide)
    int tj;
    if constexpr (TK == 16) tj = 4 * (wid >> 1) + (wid & 1) + 2 * (lane >> 4);
    else tj = wid;
    const int tk = lane & (TK - 1);
    const bool cplx = sizeof(T) == 16 && P.use;

    // coarse footprint origin along axes 1 and 2
    const int base1 = (F1 + G.skip0[1]) >> 1;
    const int base2 = (F2 + G.skip0[2]) >> 1;
    int soff[NC], goff[NC];
    unsigned vmask = 0, pcode = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const int e = tid + i * NT;
        soff[i] = e;
        goff[i] = 0;
        if (e >= SS) continue;
        const int y = e / CZ, z = e % CZ;
        const int py = base1 + y, pz = base2 + z;
        if (py >= G.s[1] || pz >= G.s[2]) continue;
        int iy = py - G.plo[1], iz = pz - G.plo[2];
        const unsigned c1 = iy >= n1 ? 1u : (iy < 0 ? 2u : 0u);
        const unsigned c2 = iz >= n2 ? 1u : (iz < 0 ? 2u : 0u);
        if (wrap_c(iy, n1, G.g.periodic[1]) && wrap_c(iz, n2, G.g.periodic[2])) {
            vmask |= 1u << i;
            goff[i] = iy * n2 + iz;
            pcode |= (c1 | (c2 << 2)) << (4 * i);
        }
    }
    if (!cplx) pcode = 0;

    // This thread's axis-2 items (row y, fine column k of the tile): raw
    // fine index u = F2 + k + skip0 maps to coarse base m = K/2 - 1 + u/2
    // (IP1D, c/bmgs/interpolate.cpp:10-46) in the stage row; parity of u
    // picks copy or taps.  Fixed for the whole march.
    int qsrc[NQ], qdst[NQ];
    unsigned qok = 0;
    // warps 0 .. NW/2-1: fine index even; the others: odd
    const bool qodd = wid >= NW / 2;
    {
        const int s2 = G.skip0[2] & 1;
        const int c = qodd ? 1 - s2 : s2;       // column parity with that u parity
#pragma unroll
        for (int r = 0; r < NQ; r++) {
            const int j = (wid % (NW / 2)) * 32 + lane + r * (NW / 2) * 32;
            const int y = j / (TK / 2), kk = j % (TK / 2);
            const int k = 2 * kk + c;
            const int u = F2 + k + G.skip0[2];
            qsrc[r] = y * CZ + K / 2 - 1 + (u >> 1) - base2;
            qdst[r] = y * TK + k;
            if (j < NIP && F2 + k < G.nout[2]) qok |= 1u << r;
        }
    }
    // the axis-1 value of this thread's fine row F1 + tj from Q's column tk
    const int u1 = F1 + tj + G.skip0[1];
    const int qcol = (K / 2 - 1 + (u1 >> 1) - base1) * TK + tk;
    const bool odd1 = u1 & 1;
    const bool row_ok = F1 + tj < G.nout[1];

    // coarse padded planes ia .. min(s0-1, ib-1+K-1)
    const int nx = min(G.s[0] - 1, ib - 1 + K - 1) - ia + 1;
    auto plane_info = [&](int j, int& ip, int& ws) {
        ip = ia + j - G.plo[0];
        ws = ip >= G.g.n[0] ? 0 : (ip < 0 ? 1 : -1);
        return wrap_c(ip, G.g.n[0], G.g.periodic[0]);
    };
    auto issue = [&](int j, int slot) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        T* st = stage + slot * SSP;
        const T* src = pv ? a + (long long)ip * n1 * n2 : a;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= SS) break;
            cp_async_x<EB>(st + soff[i], src + goff[i], pv && ((vmask >> i) & 1));
        }
    };
    auto fixup = [&](int j, int slot) {
        int ip, ws;
        plane_info(j, ip, ws);
        const bool pw = cplx && ws >= 0 && G.g.periodic[0];
        if (!pw && !pcode) return;
        const double2 ph0 = ws == 0 ? P.ph[0][0] : P.ph[0][1];
        T* st = stage + slot * SSP;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (tid + i * NT >= SS) break;
            const unsigned c = (pcode >> (4 * i)) & 15u;
            if ((pw || c) && ((vmask >> i) & 1))
                st[soff[i]] = apply_code<T>(st[soff[i]], c, pw, ph0, P);
        }
    };

    // -- TMA windows (LD == 1) ----------------------------------------------
    // in-grid cells of this thread (e-mapping) and the wrapped cells (past
    // a periodic edge of axis 1 or 2), dealt compactly: rows [0, ra) and
    // [rb, CY) past axis 1's edges, then columns [0, ca) and [cb, CZ) of
    // the other rows
    const int row0 = base1 - G.plo[1], col0 = base2 - G.plo[2];
    unsigned inmask = 0, wmask = 0, wcode = 0;
    int wso[NC], wgo[NC];
    T pre[NC];
    if constexpr (LD == 1) {
#pragma unroll
        for (int i = 0; i < NC; i++) {
            const int e = tid + i * NT;
            if (e < SS) {
                const int iy = row0 + e / CZ, iz = col0 + e % CZ;
                if (iy >= 0 && iy < n1 && iz >= 0 && iz < n2) inmask |= 1u << i;
            }
        }
        const int ra = min(max(-row0, 0), CY), rb = min(max(n1 - row0, ra), CY);
        const int ca = min(max(-col0, 0), CZ), cb = min(max(n2 - col0, ca), CZ);
        const int nA = G.g.periodic[1] ? (ra + CY - rb) * CZ : 0;
        const int nBc = G.g.periodic[2] ? ca + CZ - cb : 0;
        const int nB = (rb - ra) * nBc;
#pragma unroll
        for (int r = 0; r < NC; r++) {
            const int w = tid + r * NT;
            wso[r] = 0;
            wgo[r] = 0;
            int y, z;
            if (w < nA) {
                const int q = w / CZ;
                z = w % CZ;
                y = q < ra ? q : rb + (q - ra);
            } else if (w < nA + nB) {
                const int w2 = w - nA;
                const int q = w2 / nBc, c = w2 % nBc;
                y = ra + q;
                z = c < ca ? c : cb + (c - ca);
            } else {
                continue;
            }
            int iy = row0 + y, iz = col0 + z;
            const unsigned c1 = iy >= n1 ? 1u : (iy < 0 ? 2u : 0u);
            const unsigned c2 = iz >= n2 ? 1u : (iz < 0 ? 2u : 0u);
            if (wrap_c(iy, n1, G.g.periodic[1]) && wrap_c(iz, n2, G.g.periodic[2])) {
                wmask |= 1u << r;
                wso[r] = y * CZ + z;
                wgo[r] = iy * n2 + iz;
                wcode |= (c1 | (c2 << 2)) << (4 * r);
            }
        }
        if (!cplx) wcode = 0;
    }
    auto issue_tma = [&](int j, int slot) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[slot], (unsigned)(SS * 16));
        tma_load_window16(stage + slot * SSP, &map, col0, row0, pv ? ip : -1, bg, &bar[slot]);
    };
    auto load_wrapped = [&](int j) {
        int ip, ws;
        const bool pv = plane_info(j, ip, ws);
        const T* src = a + (long long)(pv ? ip : 0) * n1 * n2;
#pragma unroll
        for (int r = 0; r < NC; r++)
            pre[r] = (pv && ((wmask >> r) & 1)) ? __ldg(src + wgo[r]) : Num<T>::zero();
    };
    auto fixup_tma = [&](int j, int slot) {
        int ip, ws;
        if (!plane_info(j, ip, ws)) return;
        T* st = stage + slot * SSP;
        const bool pw = cplx && ws >= 0;
        const double2 ph0 = ws == 0 ? P.ph[0][0] : P.ph[0][1];
        if constexpr (sizeof(T) == 16) {
            if (pw) {
#pragma unroll
                for (int i = 0; i < NC; i++)
                    if ((inmask >> i) & 1) st[tid + i * NT] = cmul(ph0, st[tid + i * NT]);
            }
        }
#pragma unroll
        for (int r = 0; r < NC; r++)
            if ((wmask >> r) & 1)
                st[wso[r]] = apply_code<T>(pre[r], (wcode >> (4 * r)) & 15u, pw, ph0, P);
    };

    T ring[K];
#pragma unroll
    for (int i = 0; i < K; i++) ring[i] = Num<T>::zero();
    const int f1 = F1 + tj, f2 = F2 + tk;
    const bool inside = row_ok && f2 < G.nout[2];
    // this thread's output column; fine plane f0 adds f0 * plane stride
    T* ocol = o + (long long)f1 * G.nout[2] + f2;
    const long long pstride = (long long)G.nout[1] * G.nout[2];
    auto emit = [&](int u, T v) {
        const int f0 = u - G.skip0[0];
        if (inside && f0 >= 0 && f0 < G.nout[0]) {
            T* dst = ocol + f0 * pstride;
            // accumulate: phi -= I(phi_coarse) (gpaw/poisson.py:520-521)
            *dst = G.accumulate ? Num<T>::sub(*dst, v) : v;
        }
    };

    bool dead = false;   // a bounded wait ran out (all threads agree)
    if constexpr (LD == 1) {
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q < S; q++) mbar_init(&bar[q], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0)
            for (int j = 0; j < D && j < nx; j++) issue_tma(j, j);
        if (wmask) load_wrapped(0);
    } else {
#pragma unroll 1
        for (int j = 0; j < D; j++) {
            if (j < nx) issue(j, j);
            cp_commit_x();
        }
    }
    int slot = 0;   // t % S
#pragma unroll 1
    for (int t = 0; t < nx; t++) {
        if constexpr (LD == 1) {
            bool bad = false;
            if (!dead) bad = !mbar_wait(&bar[slot], (unsigned)(t / S) & 1u);
            fixup_tma(t, slot);
            if (wmask && t + 1 < nx) load_wrapped(t + 1);
            fence_proxy_async_smem();
            if (__syncthreads_or(bad)) dead = true;
            // plane t + D goes into slot (t + D) % S = (t - 1) % S
            if (tid == 0 && !dead && t + D < nx) issue_tma(t + D, slot == 0 ? S - 1 : slot - 1);
        } else {
            cp_wait_x<D - 1>();
            fixup(t, slot);
            __syncthreads();
            // plane t + D goes into slot (t + D) % S = (t - 1) % S
            if (t + D < nx) issue(t + D, slot == 0 ? S - 1 : slot - 1);
            cp_commit_x();
        }
        const T* A = stage + slot * SSP;
#pragma unroll
        for (int r = 0; r < NQ; r++) {
            if ((qok >> r) & 1) {
                const T v = ip_value<T, K>(A + qsrc[r], 1, qodd, G.w);
                Q[qdst[r]] = G.neg_in ? Num<T>::neg(v) : v;
            }
        }
        __syncthreads();
        {
            T v = row_ok ? ip_value<T, K>(Q + qcol, TK, odd1, G.w) : Num<T>::zero();
#pragma unroll
            for (int i = 0; i < K - 1; i++) ring[i] = ring[i + 1];
            ring[K - 1] = v;
        }
        const int x0 = ia + t;
        // emit the pair i = x0 - (K - 1) (or the final even point when the
        // odd one is skipped and plane i + K - 1 lies past the input)
        const int i = x0 - (K - 1);
        if (i >= ia && i < ib) {
            emit(2 * i, ring[K / 2 - 1]);
            T x = Num<T>::scale(Num<T>::add(ring[K / 2 - 1], ring[K / 2]), G.w[0]);
#pragma unroll
            for (int jj = 1; jj < K / 2; jj++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(ring[K / 2 - 1 - jj],
                                                             ring[K / 2 + jj]),
                                                 G.w[jj]));
            emit(2 * i + 1, x);
        }
        if (x0 == G.s[0] - 1 && ib - 1 + K - 1 > x0) {
            // last pair with skip1: its even point lives K/2 planes back
            const int il = ib - 1;
            if (il >= ia && il == x0 - (K - 2)) emit(2 * il, ring[K / 2]);
        }
        slot = slot + 1 == S ? 0 : slot + 1;
    }
    if constexpr (LD == 1) {
        if (dead)
            for (int j = 0; j < nx; j++)
                mbar_wait(&bar[j % S], (unsigned)(j / S) & 1u, 1000000ull);
    } else {
        cp_wait_x<0>();
    }
}

// ----------------------------------------------------------------- launchers
template <class T, int K>
static int launch_restrict_k(const void* in, void* out, void* out2, int nin, const XferGeom& G,
                             const Phases& P, cudaStream_t st) {
    if constexpr (sizeof(T) == 16) {
        if (tma_enabled()) {
            const int rc = launch_restrict_tma<K>(in, out, out2, nin, G, P, st);
            if (rc <= 0) return rc;
        }
    }
    // 16-byte elements: a square 16 x 16 tile; 8-byte: 8 x 32.  Complex
    // stages are 27 KB: one plane ahead (two stages) leaves room for three
    // CTAs an SM, which hides more latency than a deeper ring (measured).
    constexpr int TK = sizeof(T) == 16 ? 16 : 32;
    constexpr int TJ = 256 / TK;
    constexpr int D = sizeof(T) == 16 ? 1 : 3;
    constexpr int H = 2 * K - 3, FY = 2 * TJ + H, FZ = 2 * TK + H;
    constexpr int SS = FY * FZ;
    constexpr int RP = TK + (sizeof(T) == 16 ? 0 : (sizeof(T) == 8 ? 8 : 16));
    constexpr size_t smem = ((size_t)(D + 1) * SS + (size_t)2 * FY * RP) * sizeof(T);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_restrict<T, K, TJ, TK, D>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -2;
        attr = true;
    }
    const int t1 = (G.nout[1] + TJ - 1) / TJ, t2 = (G.nout[2] + TK - 1) / TK;
    int chunk0 = G.nout[0];
    const long long tiles = (long long)t1 * t2 * nin;
    if (G.chunk > 0) chunk0 = std::min(G.chunk, G.nout[0]);
    else
        while (chunk0 > 4 && tiles * ((G.nout[0] + chunk0 - 1) / chunk0) < 148 * 4)
            chunk0 = (chunk0 + 1) / 2;
    const int nchunks = (G.nout[0] + chunk0 - 1) / chunk0;
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(t1 * t2, nchunks, nb);
        const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
        const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
        k_restrict<T, K, TJ, TK, D><<<grid, TJ * TK, smem, st>>>(
            (const T*)in + b0 * ngin, (T*)out + b0 * ngout,
            out2 ? (T*)out2 + b0 * ngout : nullptr, nb, G, P, chunk0);
    }
    return 0;
}

template <class T, int K, int LD>
static int launch_interp_v(const void* in, void* out, int nin, const XferGeom& G,
                           const Phases& P, cudaStream_t st) {
    constexpr int TK = sizeof(T) == 16 ? 16 : 32;
    constexpr int TJ = 256 / TK;
    constexpr int D = 3;
    constexpr int CY = TJ / 2 + K + 1, CZ = TK / 2 + K + 1;
    constexpr int SSP = LD ? (CY * CZ + 7) / 8 * 8 : CY * CZ;
    constexpr size_t smem = ((size_t)(D + 1) * SSP + (size_t)CY * TK) * sizeof(T) +
                            (LD ? (D + 1) * sizeof(uint64_t) + 128 : 0);
    CUtensorMap map;
    memset(&map, 0, sizeof map);
    if constexpr (LD == 1) {
        const char* why = nullptr;
        if (make_plane_map16(&map, in, nin, G.g.n[0], G.g.n[1], G.g.n[2], CY, CZ, &why))
            return 1;
    }
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_interpolate<T, K, TJ, TK, D, LD>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -2;
        attr = true;
    }
    const int t1 = (G.nout[1] + TJ - 1) / TJ, t2 = (G.nout[2] + TK - 1) / TK;
    const int n0p = G.s[0] - (K - 1) + G.skip1[0];
    int chunk0 = n0p;
    const long long tiles = (long long)t1 * t2 * nin;
    if (G.chunk > 0) chunk0 = std::min(G.chunk, n0p);
    else
        while (chunk0 > 4 && tiles * ((n0p + chunk0 - 1) / chunk0) < 148 * 8)
            chunk0 = (chunk0 + 1) / 2;
    const int nchunks = (n0p + chunk0 - 1) / chunk0;
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(t1 * t2, nchunks, nb);
        const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
        const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
        k_interpolate<T, K, TJ, TK, D, LD><<<grid, TJ * TK, smem, st>>>(
            (const T*)in + b0 * ngin, (T*)out + b0 * ngout, nb, G, P, chunk0, map, b0);
    }
    return 0;
}

// The interpolation keeps per-thread cp.async cells by default: its coarse
// windows are small (15 x 15 cells for K = 6), and one TMA copy per plane
// measured slower (3500 against 3820 GB/s on the 256 x 96^3 complex batch).
// GPAW_B200_TMA_INTERP=1 selects the TMA windows.
static bool tma_interp() {
    const char* e = getenv("GPAW_B200_TMA_INTERP");
    return e != nullptr && atoi(e) != 0;
}

template <class T, int K>
static int launch_interp_k(const void* in, void* out, int nin, const XferGeom& G,
                           const Phases& P, cudaStream_t st) {
    if constexpr (sizeof(T) == 16) {
        if (tma_enabled() && tma_interp()) {
            const int rc = launch_interp_v<T, K, 1>(in, out, nin, G, P, st);
            if (rc <= 0) return rc;
        }
    }
    return launch_interp_v<T, K, 0>(in, out, nin, G, P, st);
}

template <class T>
int launch_transform(int k, bool interpolate, const void* in, void* out, void* out2, int nin,
                     const XferGeom& G, const Phases& P, cudaStream_t st) {
    const int K = k;
    if (interpolate) {
        switch (K) {
            case 2: return launch_interp_k<T, 2>(in, out, nin, G, P, st);
            case 4: return launch_interp_k<T, 4>(in, out, nin, G, P, st);
            case 6: return launch_interp_k<T, 6>(in, out, nin, G, P, st);
            case 8: return launch_interp_k<T, 8>(in, out, nin, G, P, st);
        }
    } else {
        switch (K) {
            case 2: return launch_restrict_k<T, 2>(in, out, out2, nin, G, P, st);
            case 4: return launch_restrict_k<T, 4>(in, out, out2, nin, G, P, st);
            case 6: return launch_restrict_k<T, 6>(in, out, out2, nin, G, P, st);
            case 8: return launch_restrict_k<T, 8>(in, out, out2, nin, G, P, st);
        }
    }
    return -1;
}

template int launch_transform<double>(int, bool, const void*, void*, void*, int, const XferGeom&,
                                      const Phases&, cudaStream_t);
template int launch_transform<double2>(int, bool, const void*, void*, void*, int, const XferGeom&,
                                       const Phases&, cudaStream_t);
template int launch_transform<float>(int, bool, const void*, void*, void*, int, const XferGeom&,
                                     const Phases&, cudaStream_t);

}  // namespace gb
