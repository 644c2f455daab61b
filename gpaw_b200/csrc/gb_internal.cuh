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
    int chunk;      // output planes of axis 0 per CTA (0: the launcher's rule)
};

// ------------------------------------------------------- tiled cfd stencil
// Axis-aligned stencil in "three directions" form (coefficient order = the
// caller's order: centre, then per direction +1..+nn, -1..-nn).
struct CfdStencil {
    double c0;
    int axis[3];          // axis of direction k
    double cp[3][8];      // coefficient of +d (d = 1..nn) along direction k
    double cm[3][8];      // coefficient of -d
};

// Epilogues fused into the sweep (one pass over the data each):
enum : int {
    EPI_APPLY = 0,    // out = L in                       (bmgs_fd)
    EPI_RESID = 1,    // out = L in - aux, |out|^2 partials (gpaw/poisson.py:517-532)
    EPI_JACOBI = 2,   // out = (1-w) in + w (aux - L' in) / c0  (c/bmgs/relax.cpp:41-65)
    EPI_PRECOND = 3,  // out = +-(in - sc (L in - aux))  (c/fd_preconditioner.cpp:251-333)
    EPI_LIN = 4,      // y = p0 aux + p1 in + p2 L in + p3 aux2 (mixed-precision solver)
    EPI_POT = 5,      // out = L in + in * v, v real, one grid for the whole batch
                      // (FDHamiltonian.apply_local_potential, gpaw/new/fd/hamiltonian.py:23-32)
};

struct Epi {
    const void* aux;
    double w;
    double sc;
    int negate;
    double* partial;  // EPI_RESID / EPI_LIN: per-CTA sums of |out|^2 (nullable)
    // EPI_LIN only
    const void* aux2;
    double p0, p1, p2, p3;
    double* acc64;    // if set: acc64 += y (instead of writing out)
    float* out32;     // if set: out32 = (float) y (instead of writing out)
    int chunk;        // planes of axis 0 per CTA (0: cfd_chunk's rule)
};

// ------------------------------------------------------------------ launchers
template <class T>
void launch_fd(const void* in, void* out, int nin, const GridBC& g, const Phases& P,
               const Stencil& st, cudaStream_t stream);
// out += in * v (v real, the same grid for every batch member)
template <class T>
void launch_add_pot(const void* in, void* out, const double* v, int nin, long long ng,
                    cudaStream_t stream);
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
bool to_cfd_stencil(const Stencil& s, CfdStencil& cs, int& nn);
template <class T>
int launch_fd_cfd(int mode, const void* in, void* out, int nin, const GridBC& g,
                  const Phases& P, const CfdStencil& cs, int nn, const Epi& ep,
                  cudaStream_t st, int* nblk);
int cfd_blocks(const GridBC& g, int nn, int elem_bytes, int nin, int chunk = 0);
int cfd_chunk(const GridBC& g, int nn, int nin, int ty);
// read and clear the device fault flag of a kernel file (bounded waits)
int take_fault_transform(int* code);
int take_fault_cfd(int* code);
int take_fault_mixed(int* code);

// stencil pass with a linear epilogue for the mixed solver (gb_pass.cu):
// v = p0 aux + p1 u + p2 (A u) + p3 aux2 written to out, added to acc64, or
// written as float to out32 with per-CTA partials of v^2; -1 when the
// operator or grid is not supported (caller falls back)
bool pass_supported_grid(const GridBC& g, const CfdStencil& cs, int nn);
int pass_blocks(const GridBC& g, int elem_bytes);
template <class T>
int launch_pass(const GridBC& g, const CfdStencil& cs, int nn, const T* in, T* out, const T* aux,
                const T* aux2, double p0, double p1, double p2, double p3, double* acc64,
                float* out32, double* partial, cudaStream_t st);

// the preconditioner step out = +-(in - sc (A in - aux)) on a batch of nin
// real grids, bit-identical to the plane-marching kernel's EPI_PRECOND
// (gb_pass.cu); -1 when not supported
int launch_pass_precond(const GridBC& g, const CfdStencil& cs, int nn, const double* in,
                        double* out, const double* aux, int nin, double sc, int negate,
                        cudaStream_t st);

// caching allocator of the solver objects (gb_pool.cu): device memory and
// pinned host memory; with the pool off these are cudaMalloc/cudaFree
int dmalloc(void** p, size_t bytes);
void dfree(void* p);
int hmalloc(void** p, size_t bytes);
void hfree(void* p);
template <class T>
inline cudaError_t pool_malloc(T** p, size_t bytes) {
    return dmalloc((void**)p, bytes) ? cudaErrorMemoryAllocation : cudaSuccess;
}
template <class T>
inline cudaError_t pool_malloc_host(T** p, size_t bytes) {
    return hmalloc((void**)p, bytes) ? cudaErrorMemoryAllocation : cudaSuccess;
}

}  // namespace gb
