// Finite-difference stencil apply, residual and relaxation kernels.
//
// Reference behaviour restated here (single domain):
//   apply   c/operators.cpp:98-144 (bc_unpack1/2 then bmgs_fd/bmgs_fdz,
//           c/bmgs/fd.cpp:9-33)
//   relax   c/operators.cpp:50-92 + c/bmgs/relax.cpp:8-66
//
// The reference first copies every grid into a zero-initialised padded
// buffer and fills the halo (c/bc.cpp:146-258), then runs the stencil over
// the padded buffer.  Here the halo is never materialised: a read past an
// edge is resolved in the load path (zero, or periodic wrap times the Bloch
// phase), so each launch touches only its inputs and outputs.
#include <algorithm>

#include "gb_internal.cuh"

namespace gb {

// ----------------------------------------------------------------------------
// Generic stencil (any offsets, cfd or not).  One thread per output point.
// Points whose every neighbour is in range take the fast path (plain loads at
// flat offsets); the others resolve each neighbour through bc_read.
// ----------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256)
k_fd_generic(const T* __restrict__ in, T* __restrict__ out, int nin, GridBC g, Phases P,
             const __grid_constant__ Stencil s) {
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
    const bool corners = !s.cfd;
    for (int b = blockIdx.y; b < nin; b += gridDim.y) {
        const T* a = in + (long long)b * ng;
        T x = Num<T>::zero();
        if (inner) {
            for (int c = 0; c < s.ncoefs; c++)
                x = Num<T>::add(x, Num<T>::scale(__ldg(a + p + s.flat[c]), s.coef[c]));
        } else {
            for (int c = 0; c < s.ncoefs; c++) {
                T v = bc_read<T>(a, i0 + s.off[c][0], i1 + s.off[c][1], i2 + s.off[c][2], g, P,
                                 corners);
                x = Num<T>::add(x, Num<T>::scale(v, s.coef[c]));
            }
        }
        out[(long long)b * ng + p] = x;
    }
}

// r = L(phi) - rho   (gpaw/poisson.py:517-518 and 525-526: apply, then
// residual -= rho).  Optionally writes one partial sum of r*r per block
// (partial[b * gridDim.x + block]); reduce_partials() adds them up in a
// fixed order, so the norm is deterministic run to run.
template <class T>
__global__ void __launch_bounds__(256)
k_residual(const T* __restrict__ phi, const T* __restrict__ rho, T* __restrict__ res, int nin,
           GridBC g, Phases P, const __grid_constant__ Stencil s, double* __restrict__ partial) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int ng = n0 * n1 * n2;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < ng;
    int i0 = 0, i1 = 0, i2 = 0;
    if (valid) {
        i2 = p % n2;
        const int t = p / n2;
        i1 = t % n1;
        i0 = t / n1;
    }
    const int r = s.range;
    const bool inner = i0 >= r && i0 + r < n0 && i1 >= r && i1 + r < n1 && i2 >= r && i2 + r < n2;
    const bool corners = !s.cfd;
    for (int b = blockIdx.y; b < nin; b += gridDim.y) {
        double sq = 0.0;
        if (valid) {
            const T* a = phi + (long long)b * ng;
            T x = Num<T>::zero();
            if (inner) {
                for (int c = 0; c < s.ncoefs; c++)
                    x = Num<T>::add(x, Num<T>::scale(__ldg(a + p + s.flat[c]), s.coef[c]));
            } else {
                for (int c = 0; c < s.ncoefs; c++) {
                    T v = bc_read<T>(a, i0 + s.off[c][0], i1 + s.off[c][1], i2 + s.off[c][2], g,
                                     P, corners);
                    x = Num<T>::add(x, Num<T>::scale(v, s.coef[c]));
                }
            }
            x = Num<T>::sub(x, rho[(long long)b * ng + p]);
            if (res) res[(long long)b * ng + p] = x;
            sq = sqnorm(x);
        }
        if (partial) {
            sq = block_sum(sq);
            if (threadIdx.x == 0) partial[(long long)b * gridDim.x + blockIdx.x] = sq;
        }
    }
}

// Weighted Jacobi sweep (c/bmgs/relax.cpp:41-65):
//   new = (1 - w) * old + w * (src - sum_{c>=1} coef_c old[g + o_c]) / coef_0
// reading `old` and writing `nw` (the reference reads the padded copy of
// the previous sweep, so every point sees old values only).
__global__ void __launch_bounds__(256)
k_jacobi(const double* __restrict__ old, double* __restrict__ nw, const double* __restrict__ src,
         GridBC g, const __grid_constant__ Stencil s, double w) {
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
    Phases P{};
    double x = 0.0;
    if (inner) {
        for (int c = 1; c < s.ncoefs; c++)
            x = __dadd_rn(x, __dmul_rn(__ldg(old + p + s.flat[c]), s.coef[c]));
    } else {
        for (int c = 1; c < s.ncoefs; c++) {
            double v = bc_read<double>(old, i0 + s.off[c][0], i1 + s.off[c][1],
                                       i2 + s.off[c][2], g, P, !s.cfd);
            x = __dadd_rn(x, __dmul_rn(v, s.coef[c]));
        }
    }
    const double b = old[p];
    nw[p] = __dadd_rn(__dmul_rn(1.0 - w, b),
                      __ddiv_rn(__dmul_rn(w, __dsub_rn(src[p], x)), s.coef[0]));
}

// One wavefront of lexicographic Gauss-Seidel (c/bmgs/relax.cpp:12-40).
// Wavefront t holds the points with a*i0 + b*i1 + i2 == t; with the weights
// chosen by the host every earlier-in-order neighbour lies on an earlier
// wavefront and every later one on a later wavefront, so updating a whole
// wavefront at once reproduces the sequential loop exactly.  Reads past the
// edge see the values of the sweep's start (`snap`), as the reference's
// padded copy does; reads inside see the live array.
__global__ void __launch_bounds__(256)
k_gs_wave(double* __restrict__ f, const double* __restrict__ snap, const double* __restrict__ src,
          GridBC g, const __grid_constant__ Stencil s, int t, int wa, int wb, double inv0) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n0 * n1) return;
    const int i1 = q % n1;
    const int i0 = q / n1;
    const int i2 = t - wa * i0 - wb * i1;
    if (i2 < 0 || i2 >= n2) return;
    const int p = (i0 * n1 + i1) * n2 + i2;
    Phases P{};
    double x = 0.0;
    for (int c = 1; c < s.ncoefs; c++) {
        const int y0 = i0 + s.off[c][0], y1 = i1 + s.off[c][1], y2 = i2 + s.off[c][2];
        double v;
        if (y0 >= 0 && y0 < n0 && y1 >= 0 && y1 < n1 && y2 >= 0 && y2 < n2)
            v = f[(y0 * n1 + y1) * n2 + y2];
        else
            v = bc_read<double>(snap, y0, y1, y2, g, P, !s.cfd);
        x = __dadd_rn(x, __dmul_rn(v, s.coef[c]));
    }
    f[p] = __dmul_rn(__dsub_rn(src[p], x), inv0);
}


// One smoothing step of the preconditioner's V-cycle
// (c/fd_preconditioner.cpp:251-262, 285-296, 313-333):
//   q = L(d) - r;   out = d - s * q;   optionally out = -out.
// `out` must not alias `d` (d is read at neighbouring points).
template <class T>
__global__ void __launch_bounds__(256)
k_precond_step(const T* __restrict__ d, const T* __restrict__ r, T* __restrict__ out, int nin,
               GridBC g, Phases P, const __grid_constant__ Stencil s, double sc, int negate) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int ng = n0 * n1 * n2;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ng) return;
    const int i2 = p % n2;
    const int t = p / n2;
    const int i1 = t % n1;
    const int i0 = t / n1;
    const int rg = s.range;
    const bool inner =
        i0 >= rg && i0 + rg < n0 && i1 >= rg && i1 + rg < n1 && i2 >= rg && i2 + rg < n2;
    const bool corners = !s.cfd;
    for (int b = blockIdx.y; b < nin; b += gridDim.y) {
        const T* a = d + (long long)b * ng;
        T x = Num<T>::zero();
        if (inner) {
            for (int c = 0; c < s.ncoefs; c++)
                x = Num<T>::add(x, Num<T>::scale(__ldg(a + p + s.flat[c]), s.coef[c]));
        } else {
            for (int c = 0; c < s.ncoefs; c++) {
                T v = bc_read<T>(a, i0 + s.off[c][0], i1 + s.off[c][1], i2 + s.off[c][2], g, P,
                                 corners);
                x = Num<T>::add(x, Num<T>::scale(v, s.coef[c]));
            }
        }
        const long long at = (long long)b * ng + p;
        x = Num<T>::sub(x, r[at]);
        T y = Num<T>::sub(a[p], Num<T>::scale(x, sc));
        out[at] = negate ? Num<T>::neg(y) : y;
    }
}

// norm2[b] = scale * sum of the per-block partials of grid b, added in a
// fixed order.
__global__ void k_reduce_partials(const double* __restrict__ partial, int nblk, double scale,
                                  double* __restrict__ out) {
    const int b = blockIdx.x;
    double v = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v += partial[(long long)b * nblk + i];
    v = block_sum(v);
    if (threadIdx.x == 0) out[b] = v * scale;
}

// ----------------------------------------------------------------- launchers
static inline dim3 grid_for(int ng, int nin) {
    return dim3((unsigned)((ng + 255) / 256), (unsigned)(nin < 65535 ? nin : 65535));
}

template <class T>
void launch_fd(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
               const Stencil& st, cudaStream_t stream) {
    const int ng = g.n[0] * g.n[1] * g.n[2];
    k_fd_generic<T><<<grid_for(ng, nin), 256, 0, stream>>>((const T*)in, (T*)out, nin, g, P,
                                                          st);
}

template void launch_fd<double>(const void*, void*, int, const GridBC&, const Phases&,
                                const Stencil&, cudaStream_t);
template void launch_fd<double2>(const void*, void*, int, const GridBC&, const Phases&,
                                 const Stencil&, cudaStream_t);
template void launch_fd<float>(const void*, void*, int, const GridBC&, const Phases&,
                               const Stencil&, cudaStream_t);

// o += p * v per point, in numpy's order for `o += p * vt_R.data`
// (gpaw/new/fd/hamiltonian.py:31-32): the product rounded, then the sum.
template <class T>
__global__ void k_add_pot(const T* __restrict__ in, T* __restrict__ out,
                          const double* __restrict__ v, int nin, long long ng) {
    const long long n = (long long)nin * ng;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = Num<T>::add(out[i], Num<T>::scale(in[i], v[i % ng]));
}

template <class T>
void launch_add_pot(const void* in, void* out, const double* v, int nin, long long ng,
                    cudaStream_t stream) {
    const long long n = (long long)nin * ng;
    const int nb = (int)std::min<long long>(148 * 16, (n + 255) / 256);
    k_add_pot<T><<<nb, 256, 0, stream>>>((const T*)in, (T*)out, v, nin, ng);
}
template void launch_add_pot<double>(const void*, void*, const double*, int, long long,
                                     cudaStream_t);
template void launch_add_pot<double2>(const void*, void*, const double*, int, long long,
                                      cudaStream_t);

template <class T>
void launch_residual(const void* phi, const void* rho, void* res, int nin, const GridBC& g,
                     const Phases& P, const Stencil& st, double* partial, cudaStream_t stream) {
    const int ng = g.n[0] * g.n[1] * g.n[2];
    k_residual<T><<<grid_for(ng, nin), 256, 0, stream>>>((const T*)phi, (const T*)rho, (T*)res,
                                                        nin, g, P, st, partial);
}
template void launch_residual<double>(const void*, const void*, void*, int, const GridBC&,
                                      const Phases&, const Stencil&, double*, cudaStream_t);
template void launch_residual<double2>(const void*, const void*, void*, int, const GridBC&,
                                       const Phases&, const Stencil&, double*, cudaStream_t);
template void launch_residual<float>(const void*, const void*, void*, int, const GridBC&,
                                     const Phases&, const Stencil&, double*, cudaStream_t);

void launch_jacobi(const double* old, double* nw, const double* src, const GridBC& g,
                   const Stencil& st, double w, cudaStream_t stream) {
    const int ng = g.n[0] * g.n[1] * g.n[2];
    k_jacobi<<<(ng + 255) / 256, 256, 0, stream>>>(old, nw, src, g, st, w);
}

void launch_gs_wave(double* f, const double* snap, const double* src, const GridBC& g,
                    const Stencil& st, int t, int wa, int wb, double inv0,
                    cudaStream_t stream) {
    const int nq = g.n[0] * g.n[1];
    k_gs_wave<<<(nq + 255) / 256, 256, 0, stream>>>(f, snap, src, g, st, t, wa, wb, inv0);
}

template <class T>
void launch_precond_step(const void* d, const void* r, void* out, int nin, const GridBC& g,
                         const Phases& P, const Stencil& st, double sc, int negate,
                         cudaStream_t stream) {
    const int ng = g.n[0] * g.n[1] * g.n[2];
    k_precond_step<T><<<grid_for(ng, nin), 256, 0, stream>>>((const T*)d, (const T*)r, (T*)out,
                                                            nin, g, P, st, sc, negate);
}
template void launch_precond_step<double>(const void*, const void*, void*, int, const GridBC&,
                                          const Phases&, const Stencil&, double, int,
                                          cudaStream_t);
template void launch_precond_step<double2>(const void*, const void*, void*, int, const GridBC&,
                                           const Phases&, const Stencil&, double, int,
                                           cudaStream_t);

int residual_blocks(const GridBC& g) { return (g.n[0] * g.n[1] * g.n[2] + 255) / 256; }

void launch_reduce_partials(const double* partial, int nblk, int nin, double scale, double* out,
                            cudaStream_t stream) {
    k_reduce_partials<<<nin, 256, 0, stream>>>(partial, nblk, scale, out);
}

}  // namespace gb
