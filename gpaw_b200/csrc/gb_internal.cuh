// Internal declarations shared by the kernel files and the C-ABI layer.
#pragma once

#include "gb_common.cuh"

namespace gb {

// ---------------------------------------------------------- block reduction
__device__ __forceinline__ double sqnorm(double x) { return x * x; }
__device__ __forceinline__ double sqnorm(float x) { return (double)x * (double)x; }
__device__ __forceinline__ double sqnorm(double2 x) { return x.x * x.x + x.y * x.y; }

// Sum over a block of up to 1024 threads; the result is valid in thread 0.
// The order of additions is fixed, so repeated runs give identical sums.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_part[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) warp_part[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? warp_part[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// -------------------------------------------------------------- transformer
struct XferGeom {
    GridBC g;       // input grid (interior size + periodicity)
    int plo[3];     // padding below the interior, per axis
    int s[3];       // padded input extent
    int nout[3];    // output interior extent
    int skip0[3];   // interpolation: first fine point omitted
    int skip1[3];   // interpolation: last fine point omitted
    double w[4];    // Lagrange mid-point weights for order k
    int neg_in;     // negate every input value on load (exact)
    int accumulate; // interpolation: out -= value instead of out = value
    double scale2;  // restriction: also write out2 = scale2 * out when out2 set
};

// ------------------------------------------------------------------ launchers
template <class T>
void launch_fd(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
               const Stencil& st, cudaStream_t stream);
template <class T>
void launch_residual(const void* phi, const void* rho, void* res, int nin, const GridBC& g,
                     const Phases& P, const Stencil& st, double* partial, cudaStream_t stream);
void launch_jacobi(const double* old, double* nw, const double* src, const GridBC& g,
                   const Stencil& st, double w, cudaStream_t stream);
void launch_gs_wave(double* f, const double* snap, const double* src, const GridBC& g,
                    const Stencil& st, int t, int wa, int wb, double inv0, cudaStream_t stream);
template <class T>
int launch_transform(int k, bool interpolate, const void* in, void* out, void* out2, int nin,
                     const XferGeom& G, const Phases& P, cudaStream_t st);
template <class T>
void launch_precond_step(const void* d, const void* r, void* out, int nin, const GridBC& g,
                         const Phases& P, const Stencil& st, double s, int negate,
                         cudaStream_t stream);
void launch_reduce_partials(const double* partial, int nblk, int nin, double scale,
                            double* out, cudaStream_t stream);
int residual_blocks(const GridBC& g);

}  // namespace gb
