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
#include "gb_internal.cuh"

namespace gb {



// ----------------------------------------------------------------- restrict
// out[I][J][L] over padded input a:  per axis, r(c) = 0.5 * (a[c] + sum_l
// w_l * (a[c + 2l + 1] + a[c - 2l - 1])) at c = K - 1 + 2 I  (RST1D,
// c/bmgs/restrict.cpp:18-60), applied along axis 2, then 1, then 0.
template <class T, int K, int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK)
k_restrict(const T* __restrict__ in, T* __restrict__ out, T* __restrict__ out2, int nin,
           XferGeom G, Phases P, int chunk0) {
    constexpr int H = 2 * K - 3;          // taps reach K-1+2(K/2-1)+1 = 2K-2 past 2I
    constexpr int FY = 2 * TJ + H;        // fine rows needed by the tile
    constexpr int FZ = 2 * TK + H;        // fine columns needed by the tile
    constexpr int NR = 2 * K - 1;         // axis-0 ring depth
    __shared__ T F[FY][FZ + 1];
    __shared__ T R1[FY][TK];

    const int tiles2 = (G.nout[2] + TK - 1) / TK;
    const int J0 = (blockIdx.x / tiles2) * TJ;
    const int L0 = (blockIdx.x % tiles2) * TK;
    const int I0 = blockIdx.y * chunk0;
    const int I1 = min(G.nout[0], I0 + chunk0);
    const int b = blockIdx.z;
    if (I0 >= I1 || b >= nin) return;
    const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
    const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
    const T* a = in + b * ngin;
    T* o = out + b * ngout;
    const int tid = threadIdx.x;
    const int tj = tid / TK, tk = tid % TK;

    T ring[NR];
#pragma unroll
    for (int i = 0; i < NR; i++) ring[i] = Num<T>::zero();

    // padded plane range for outputs [I0, I1): 2*I0 .. 2*(I1-1) + 2K - 2
    const int x0a = 2 * I0, x0b = 2 * (I1 - 1) + 2 * K - 2;
    for (int x0 = x0a; x0 <= x0b; x0++) {
        // 1. input footprint of the tile in this padded plane
        for (int e = tid; e < FY * FZ; e += TJ * TK) {
            const int y = e / FZ, z = e % FZ;
            const int py = 2 * J0 + y, pz = 2 * L0 + z;
            T v = Num<T>::zero();
            if (py < G.s[1] && pz < G.s[2])
                v = bc_read<T>(a, x0 - G.plo[0], py - G.plo[1], pz - G.plo[2], G.g, P, true);
            F[y][z] = G.neg_in ? Num<T>::neg(v) : v;
        }
        __syncthreads();
        // 2. axis-2 pass: R1[y][k] for every footprint row
        for (int e = tid; e < FY * TK; e += TJ * TK) {
            const int y = e / TK, k = e % TK;
            const int c = K - 1 + 2 * k;
            T x = F[y][c];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(F[y][c + 2 * l + 1],
                                                             F[y][c - 2 * l - 1]),
                                                 G.w[l]));
            R1[y][k] = Num<T>::scale(x, 0.5);
        }
        __syncthreads();
        // 3. axis-1 pass for this thread's (j, k)
        {
            const int c = K - 1 + 2 * tj;
            T x = R1[c][tk];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(R1[c + 2 * l + 1][tk],
                                                             R1[c - 2 * l - 1][tk]),
                                                 G.w[l]));
#pragma unroll
            for (int i = 0; i < NR - 1; i++) ring[i] = ring[i + 1];
            ring[NR - 1] = Num<T>::scale(x, 0.5);
        }
        // 4. axis-0 pass once the ring spans planes 2I .. 2I + 2K - 2
        const int q = x0 - 2 * I0;
        if (q >= 2 * K - 2 && ((q - (2 * K - 2)) & 1) == 0) {
            const int I = I0 + (q - (2 * K - 2)) / 2;
            const int J = J0 + tj, L = L0 + tk;
            T x = ring[K - 1];
#pragma unroll
            for (int l = 0; l < K / 2; l++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(ring[K - 1 + 2 * l + 1],
                                                             ring[K - 1 - 2 * l - 1]),
                                                 G.w[l]));
            if (J < G.nout[1] && L < G.nout[2]) {
                const long long at = ((long long)I * G.nout[1] + J) * G.nout[2] + L;
                const T r = Num<T>::scale(x, 0.5);
                o[at] = r;
                // fd_precond's "d = 4 * step * r" (c/fd_preconditioner.cpp:222-226)
                if (out2) out2[b * ngout + at] = Num<T>::scale(r, G.scale2);
            }
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------- interpolate
// IP1D (c/bmgs/interpolate.cpp:10-46): raw fine index u along an axis maps
// to coarse base m = K/2 - 1 + u/2 in the padded input; even u copies a[m],
// odd u gives sum_j w_j (a[m - j] + a[m + 1 + j]).  Fine index f = u - skip0.
template <class T, int K>
__device__ __forceinline__ T ip_tap(const T* row, int stride, int u, int base, const double* w) {
    const int i = u >> 1;
    const int m = K / 2 - 1 + i - base;
    if ((u & 1) == 0) return row[m * stride];
    T x = Num<T>::scale(Num<T>::add(row[m * stride], row[(m + 1) * stride]), w[0]);
#pragma unroll
    for (int j = 1; j < K / 2; j++)
        x = Num<T>::add(x, Num<T>::scale(Num<T>::add(row[(m - j) * stride],
                                                     row[(m + 1 + j) * stride]),
                                         w[j]));
    return x;
}

template <class T, int K, int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK)
k_interpolate(const T* __restrict__ in, T* __restrict__ out, int nin, XferGeom G, Phases P,
              int chunk0) {
    constexpr int CY = TJ / 2 + K + 1;     // coarse rows feeding TJ fine rows
    constexpr int CZ = TK / 2 + K + 1;
    __shared__ T A[CY][CZ + 1];
    __shared__ T Q[CY][TK];

    const int tiles2 = (G.nout[2] + TK - 1) / TK;
    const int F1 = (blockIdx.x / tiles2) * TJ;
    const int F2 = (blockIdx.x % tiles2) * TK;
    const int b = blockIdx.z;
    // pairs i along axis 0 handled by this CTA
    const int n0p = G.s[0] - (K - 1) + G.skip1[0];
    const int ia = blockIdx.y * chunk0;
    const int ib = min(n0p, ia + chunk0);
    if (ia >= ib || b >= nin) return;
    const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
    const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
    const T* a = in + b * ngin;
    T* o = out + b * ngout;
    const int tid = threadIdx.x;
    const int tj = tid / TK, tk = tid % TK;

    // coarse footprint origin along axes 1 and 2
    const int base1 = (F1 + G.skip0[1]) >> 1;
    const int base2 = (F2 + G.skip0[2]) >> 1;

    T ring[K];
#pragma unroll
    for (int i = 0; i < K; i++) ring[i] = Num<T>::zero();

    // pair i needs planes i .. i + K - 1 (odd) and K/2 - 1 + i (even)
    const int xa = ia, xb = min(G.s[0] - 1, ib - 1 + K - 1);
    for (int x0 = xa; x0 <= xb; x0++) {
        for (int e = tid; e < CY * CZ; e += TJ * TK) {
            const int y = e / CZ, z = e % CZ;
            const int py = base1 + y, pz = base2 + z;
            T v = Num<T>::zero();
            if (py < G.s[1] && pz < G.s[2])
                v = bc_read<T>(a, x0 - G.plo[0], py - G.plo[1], pz - G.plo[2], G.g, P, true);
            A[y][z] = G.neg_in ? Num<T>::neg(v) : v;
        }
        __syncthreads();
        for (int e = tid; e < CY * TK; e += TJ * TK) {
            const int y = e / TK, k = e % TK;
            const int u = F2 + k + G.skip0[2];
            Q[y][k] = (F2 + k < G.nout[2]) ? ip_tap<T, K>(&A[y][0], 1, u, base2, G.w)
                                           : Num<T>::zero();
        }
        __syncthreads();
        {
            const int u = F1 + tj + G.skip0[1];
            T v = (F1 + tj < G.nout[1]) ? ip_tap<T, K>(&Q[0][tk], TK, u, base1, G.w)
                                        : Num<T>::zero();
#pragma unroll
            for (int i = 0; i < K - 1; i++) ring[i] = ring[i + 1];
            ring[K - 1] = v;
        }
        // emit the pair i = x0 - (K - 1) (or the final even point when the
        // odd one is skipped and plane i + K - 1 lies past the input)
        const int f1 = F1 + tj, f2 = F2 + tk;
        const bool inside = f1 < G.nout[1] && f2 < G.nout[2];
        auto emit = [&](int u, T v) {
            const int f0 = u - G.skip0[0];
            if (inside && f0 >= 0 && f0 < G.nout[0]) {
                T* dst = o + ((long long)f0 * G.nout[1] + f1) * G.nout[2] + f2;
                // accumulate: phi -= I(phi_coarse) (gpaw/poisson.py:520-521)
                *dst = G.accumulate ? Num<T>::sub(*dst, v) : v;
            }
        };
        const int i = x0 - (K - 1);
        if (i >= ia && i < ib) {
            emit(2 * i, ring[K / 2 - 1]);
            T x = Num<T>::scale(Num<T>::add(ring[K / 2 - 1], ring[K / 2]), G.w[0]);
#pragma unroll
            for (int j = 1; j < K / 2; j++)
                x = Num<T>::add(x, Num<T>::scale(Num<T>::add(ring[K / 2 - 1 - j],
                                                             ring[K / 2 + j]),
                                                 G.w[j]));
            emit(2 * i + 1, x);
        }
        if (x0 == G.s[0] - 1 && ib - 1 + K - 1 > x0) {
            // last pair with skip1: its even point lives K/2 planes back
            const int il = ib - 1;
            if (il >= ia && il == x0 - (K - 2)) emit(2 * il, ring[K / 2]);
        }
        __syncthreads();
    }
}

// ----------------------------------------------------------------- launchers
template <class T, int K>
static void launch_restrict_k(const void* in, void* out, void* out2, int nin, const XferGeom& G,
                              const Phases& P, cudaStream_t st) {
    // 16-byte elements: a square tile keeps the footprint under 48 KB
    constexpr int TK = sizeof(T) == 16 ? 16 : 32;
    constexpr int TJ = 256 / TK;
    const int t1 = (G.nout[1] + TJ - 1) / TJ, t2 = (G.nout[2] + TK - 1) / TK;
    int chunk0 = G.nout[0];
    // enough CTAs to fill the GPU several times over
    const long long tiles = (long long)t1 * t2 * nin;
    while (chunk0 > 4 && tiles * ((G.nout[0] + chunk0 - 1) / chunk0) < 148 * 8) chunk0 = (chunk0 + 1) / 2;
    const int nchunks = (G.nout[0] + chunk0 - 1) / chunk0;
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(t1 * t2, nchunks, nb);
        const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
        const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
        k_restrict<T, K, TJ, TK><<<grid, TJ * TK, 0, st>>>(
            (const T*)in + b0 * ngin, (T*)out + b0 * ngout,
            out2 ? (T*)out2 + b0 * ngout : nullptr, nb, G, P, chunk0);
    }
}

template <class T, int K>
static void launch_interp_k(const void* in, void* out, int nin, const XferGeom& G,
                            const Phases& P, cudaStream_t st) {
    constexpr int TK = sizeof(T) == 16 ? 16 : 32;
    constexpr int TJ = 256 / TK;
    const int t1 = (G.nout[1] + TJ - 1) / TJ, t2 = (G.nout[2] + TK - 1) / TK;
    const int n0p = G.s[0] - (K - 1) + G.skip1[0];
    int chunk0 = n0p;
    const long long tiles = (long long)t1 * t2 * nin;
    while (chunk0 > 4 && tiles * ((n0p + chunk0 - 1) / chunk0) < 148 * 8) chunk0 = (chunk0 + 1) / 2;
    const int nchunks = (n0p + chunk0 - 1) / chunk0;
    for (int b0 = 0; b0 < nin; b0 += 65535) {
        const int nb = min(65535, nin - b0);
        dim3 grid(t1 * t2, nchunks, nb);
        const long long ngin = (long long)G.g.n[0] * G.g.n[1] * G.g.n[2];
        const long long ngout = (long long)G.nout[0] * G.nout[1] * G.nout[2];
        k_interpolate<T, K, TJ, TK><<<grid, TJ * TK, 0, st>>>(
            (const T*)in + b0 * ngin, (T*)out + b0 * ngout, nb, G, P, chunk0);
    }
}

template <class T>
int launch_transform(int k, bool interpolate, const void* in, void* out, void* out2, int nin,
                     const XferGeom& G, const Phases& P, cudaStream_t st) {
    const int K = k;
    if (interpolate) {
        switch (K) {
            case 2: launch_interp_k<T, 2>(in, out, nin, G, P, st); return 0;
            case 4: launch_interp_k<T, 4>(in, out, nin, G, P, st); return 0;
            case 6: launch_interp_k<T, 6>(in, out, nin, G, P, st); return 0;
            case 8: launch_interp_k<T, 8>(in, out, nin, G, P, st); return 0;
        }
    } else {
        switch (K) {
            case 2: launch_restrict_k<T, 2>(in, out, out2, nin, G, P, st); return 0;
            case 4: launch_restrict_k<T, 4>(in, out, out2, nin, G, P, st); return 0;
            case 6: launch_restrict_k<T, 6>(in, out, out2, nin, G, P, st); return 0;
            case 8: launch_restrict_k<T, 8>(in, out, out2, nin, G, P, st); return 0;
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
