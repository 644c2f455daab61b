/* gpaw_b200 — C ABI of the B200 (sm_100a) finite-difference hot path.
 *
 * Each entry point replaces one GPU entry point of the reference's compiled
 * extension (`cgpaw`), keeping the argument meaning: device pointers in,
 * device pointers out, C-contiguous arrays, an optional leading batch
 * dimension `nin` (the reference's ndim == 4 case), and phases as the
 * (3, 2) complex array `phase_cd` flattened to 12 doubles (re, im, ...).
 *
 * Conventions
 *   - Return value: 0 on success, GB_EINVAL for an argument the reference
 *     would reject (TypeError / ValueError / AssertionError), GB_ECUDA for a
 *     CUDA failure (the reference's RuntimeError via gpaw_set_runtime_error,
 *     c/gpu/operators.cpp:381-384), GB_ENOCONV for a Poisson solve that hit
 *     maxiter (PoissonConvergenceError, gpaw/poisson.py:487-489).
 *     gb_last_error() returns the message of the last failure of the calling
 *     thread.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Every
 *     launch is asynchronous on that stream except where noted; no entry
 *     point synchronises the device.
 *   - dtype: GB_F64 (numpy float64) or GB_C128 (numpy complex128).
 *   - Objects own only their stencil, geometry and scratch.  One object
 *     must not be used from two streams at the same time (its scratch is
 *     shared between calls).
 *   - Single domain: a neighbour equal to 0 (own rank) means periodic, -1
 *     means zero boundary (gpaw/old/domain.py:110-138).  Domain
 *     decomposition over several GPUs is not part of this library.
 */
#ifndef GPAW_B200_H
#define GPAW_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GB_API __attribute__((visibility("default")))
#else
#define GB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GB_OK 0
#define GB_EINVAL 1
#define GB_ECUDA 2
#define GB_ENOCONV 3

#define GB_F64 0
#define GB_C128 1

typedef struct gb_operator gb_operator;
typedef struct gb_transformer gb_transformer;
typedef struct gb_poisson gb_poisson;
typedef struct gb_woperator gb_woperator;

/* Library version (major * 10000 + minor * 100 + patch). */
GB_API int gb_version(void);

/* Message of the calling thread's last failed call ("" if none). */
GB_API const char* gb_last_error(void);

/* ------------------------------------------------------------------ Operator
 * Replaces cgpaw.Operator(coefs, offsets, size, range, neighbors, real, comm,
 * cfd, use_gpu) — NewOperatorObject, c/operators.cpp:379-420.
 *   coefs[ncoefs]     stencil coefficients, summed in this order
 *   offsets[ncoefs]   offsets flattened with the PADDED strides
 *                     (M_c = size_c + 2 * range), as FDOperator builds them
 *                     (gpaw/fd_operators.py:60-63)
 *   size[3]           interior grid size n_c
 *   range             stencil half-width mp (padding)
 *   neighbors[6]      neighbor_cd, row-major (3, 2)
 *   real              1 for float64 data, 0 for complex128
 *   cfd               1 if every offset lies on an axis
 */
GB_API int gb_operator_new(const double* coefs, const int64_t* offsets, int ncoefs,
                    const int64_t size[3], int range, const int64_t neighbors[6],
                    int real, int cfd, gb_operator** out);
GB_API void gb_operator_free(gb_operator* op);

/* Replaces Operator.apply_gpu(in_ptr, out_ptr, shape, dtype, phases) —
 * Operator_apply_gpu, c/gpu/operators.cpp:344-385 (CPU twin Operator_apply,
 * c/operators.cpp:245-316).  out[x] = sum_p coefs[p] * in_padded[x + p]
 * for every grid of the batch.  `in == out` is allowed (the input is then
 * staged through the operator's scratch, as the reference stages it through
 * its padded buffer).  phases may be NULL (all ones). */
GB_API int gb_operator_apply(gb_operator* op, const void* in, void* out, int64_t nin,
                      int dtype, const double* phases, void* stream);

/* Tuning knob (no reference counterpart): planes of axis 0 that one CTA of
 * the plane-marching kernels handles (the "z-block depth"; outputs planes
 * for transformers).  0 restores the automatic rule (enough CTAs for two
 * per SM).  Results do not depend on it; gpaw_b200.autotune picks it by
 * timing.  Solvers capture their launches in a graph at their first solve:
 * set it on their operators before that. */
GB_API int gb_operator_set_chunk(gb_operator* op, int chunk);
GB_API int gb_transformer_set_chunk(gb_transformer* t, int chunk);

/* FDHamiltonian.apply_local_potential (gpaw/new/fd/hamiltonian.py:23-32):
 * out = L in + in * v for every batch member, v a real float64 grid
 * (n0, n1, n2) shared by the batch; the same arithmetic as the reference's
 * `self.kin(psit_nR, out)` followed by `o += p * vt_R.data` (product
 * rounded, then the sum), in one pass over the data.  in == out allowed;
 * v must not overlap out. */
GB_API int gb_operator_apply_potential(gb_operator* op, const void* in, void* out, int64_t nin,
                                       int dtype, const double* phases, const double* v,
                                       void* stream);

/* Replaces Operator.relax_gpu(method, f_ptr, s_ptr, nrelax, w) —
 * Operator_relax_gpu, c/gpu/operators.cpp:200-221 (CPU twin Operator_relax,
 * c/operators.cpp:50-92).  float64 only, one grid.  method 2: weighted
 * Jacobi with weight w; method 1: lexicographic Gauss-Seidel (w ignored),
 * bit-identical to the reference's CPU loop (the reference's own GPU
 * Gauss-Seidel is a no-op, c/gpu/kernels/relax.cpp:72-80). */
GB_API int gb_operator_relax(gb_operator* op, int method, double* f, const double* s,
                      int nrelax, double w, void* stream);

/* Variant of gb_operator_relax that allocates nothing; it has no
 * counterpart in the reference.  For callers that cannot let the library
 * call cudaMalloc (all of HBM handed to their own pool, a serving loop that
 * must not risk the implicit synchronisation of cudaMalloc/cudaFree, a plugin
 * host that forbids foreign allocations).  Its scratch grid is a fixed
 * device array of GB_NOALLOC_MAX_POINTS doubles (16 MiB, held by every GPU
 * that loads the library until exit); grids with more points are rejected
 * with GB_EINVAL.  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress), and so does the first call after the device's
 * context was re-created (cudaDeviceReset); make that call before any stream
 * capture: made inside one, it fails with GB_EINVAL.  All calls share the
 * array: calls that overlap on the GPU race.  Same results as
 * gb_operator_relax. */
#define GB_NOALLOC_MAX_POINTS (2 * 1024 * 1024)
GB_API int gb_operator_relax_noalloc(gb_operator* op, int method, double* f, const double* s,
                                     int nrelax, double w, void* stream);

/* Device-side fault record; no counterpart in the reference.  Kernels that
 * wait on the completion of asynchronous copies bound every wait (one
 * second); a wait that runs out records a code here instead of hanging the
 * GPU, and that kernel's output is not valid.  Reads and clears the record
 * (synchronous): *code = 0 when nothing was recorded, 1 for a copy that
 * did not complete in time. */
GB_API int gb_device_fault(int* code);

/* Caching allocator of the solver objects (gb_poisson, gb_mixed and the
 * operators' scratch); no counterpart in the reference, whose C objects
 * hold static buffers.  With the pool on, memory an object frees is kept,
 * binned by size class (four per power of two), and handed to the next
 * object that needs that class, so that building and dropping solvers
 * neither calls the driver nor synchronises the device.  The caller then
 * must free an object only when none of its work is in flight.  The cache
 * holds at most `cache_limit` bytes (the largest blocks go first);
 * gb_pool_release returns every cached block to the driver; gb_pool_stats
 * gives the bytes handed out and the bytes cached.  Off by default. */
GB_API int gb_pool_set(int on, size_t cache_limit);
GB_API int gb_pool_release(void);
GB_API int gb_pool_stats(size_t* live, size_t* cached);

/* Kernel timeline of composite calls; a profiling aid with no counterpart
 * in the reference.  Between gb_trace_begin(capacity) and gb_trace_end,
 * gb_fd_precond and gb_mixed_vcycle_eager record a CUDA event on their
 * stream before each of their kernels and one after the last (at most
 * `capacity` events in all).
 * gb_trace_end waits for the last event and writes, for up to `max`
 * intervals, the milliseconds between consecutive events and the label of
 * the kernel each interval starts with; *count receives the number of
 * intervals.  Not for use inside a stream capture. */
GB_API int gb_trace_begin(int capacity);
GB_API int gb_trace_end(int max, float* ms, const char** labels, int* count);

/* Residual r = L(phi) - rho for a batch (gpaw/poisson.py:517-518 done in
 * one pass).  r may be NULL.  If norm2 is not NULL it receives, per grid,
 * scale * sum |r|^2 as a DEVICE array of nin doubles (the reference's
 * xp.dot(r, r) * dv, gpaw/poisson.py:527-532, without the host sync). */
GB_API int gb_operator_residual(gb_operator* op, const void* phi, const void* rho,
                         void* r, int64_t nin, int dtype, const double* phases,
                         double scale, double* norm2, void* stream);

/* Replaces Operator.get_diagonal_element(), c/operators.cpp:319-332. */
GB_API double gb_operator_get_diagonal_element(const gb_operator* op);

/* Preallocate the operator's scratch for batches up to nin grids (so that
 * later calls allocate nothing, e.g. inside CUDA-graph capture). */
GB_API int gb_operator_reserve(gb_operator* op, int64_t nin, int dtype);

/* ----------------------------------------------------------------- WOperator
 * Replaces cgpaw.WOperator(nweights, weights, coefs, offsets, size, range,
 * neighbors, real, comm, cfd) — NewWOperatorObject, c/woperators.cpp:416-460,
 * built by WeightedFDOperator.set_weights (gpaw/wfd_operators.py:64-81).
 * A = sum_i weights_i * operators_i with per-point weights:
 *   nweights          number of operators (1..GB_MAX_WEIGHTS)
 *   weights[i]        DEVICE pointer to a float64 grid (size[0..2]) for
 *                     operator i; not copied, must outlive the object
 *   coefs[i], offsets[i], ncoefs[i]
 *                     stencil i, offsets flattened with the padded strides
 *                     (M_c = size_c + 2 * range); offsets[i][0] must be 0
 *                     (WeightedFDOperator puts the centre first, with
 *                     coefficient 0 when the operator has none)
 *   size, range, neighbors, real, cfd as for gb_operator_new (cfd = 1 when
 *   every operator is axis-aligned) */
#define GB_MAX_WEIGHTS 8
GB_API int gb_woperator_new(int nweights, const double* const* weights,
                            const double* const* coefs, const int64_t* const* offsets,
                            const int* ncoefs, const int64_t size[3], int range,
                            const int64_t neighbors[6], int real, int cfd,
                            gb_woperator** out);
GB_API void gb_woperator_free(gb_woperator* op);

/* WOperator.apply(in, out[, phases]) — WOperator_apply,
 * c/woperators.cpp:318-370 with bmgs_wfd / bmgs_wfdz (c/bmgs/wfd.cpp):
 * out[x] = sum_i w_i[x] (sum_p c_ip in[x + o_ip]), every inner sum from 0
 * in coefficient order, scaled by the weight, then added to the total.
 * Every grid of the batch uses the same weights.  in == out is allowed. */
GB_API int gb_woperator_apply(gb_woperator* op, const void* in, void* out, int64_t nin,
                              int dtype, const double* phases, void* stream);

/* WOperator.relax(method, f, s, nrelax, w=1.0) — WOperator_relax,
 * c/woperators.cpp:53-96 with bmgs_wrelax (c/bmgs/wrelax.cpp).  float64,
 * one grid.  method 2: weighted Jacobi; method 1: lexicographic
 * Gauss-Seidel.  The diagonal is sum_i w_i[x] c_i0 per point. */
GB_API int gb_woperator_relax(gb_woperator* op, int method, double* f, const double* s,
                              int nrelax, double w, void* stream);

/* WOperator.get_diagonal_element() — c/woperators.cpp:372-398: the largest
 * |sum_i w_i[x] c_i0| over the grid (0 for an all-zero grid), written to
 * *out (host).  Synchronises the stream. */
GB_API int gb_woperator_get_diagonal_element(gb_woperator* op, double* out, void* stream);

/* --------------------------------------------------------------- Transformer
 * Replaces cgpaw.Transformer(size_in, size_out, k, pads, npads, skip,
 * neighbors, real, comm, interpolate, use_gpu) — NewTransformerObject,
 * c/transformers.cpp:196-246.  k = 2 * nn in {2, 4, 6, 8}.  pads, npads,
 * skip, neighbors are row-major (3, 2) arrays as built by _Transformer
 * (gpaw/transformers.py:31-55). */
GB_API int gb_transformer_new(const int64_t size_in[3], const int64_t size_out[3], int k,
                       const int64_t pads[6], const int64_t npads[6],
                       const int64_t skip[6], const int64_t neighbors[6], int real,
                       int interpolate, gb_transformer** out);
GB_API void gb_transformer_free(gb_transformer* t);

/* Replaces Transformer.apply_gpu(in_ptr, out_ptr, shape, dtype, phases) —
 * Transformer_apply_gpu, c/gpu/transformers.cpp:189-226 (CPU twin
 * Transformer_apply, c/transformers.cpp:112-158).  in and out must not
 * overlap. */
GB_API int gb_transformer_apply(gb_transformer* t, const void* in, void* out, int64_t nin,
                         int dtype, const double* phases, void* stream);

/* ---------------------------------------------------------------- fd_precond
 * Replaces cgpaw.fd_precond(rest0, rest1, intp1, intp2, kin0, kin1, kin2,
 * d0, q0, r1, d1, q1, r2, d2, q2, residuals, nresiduals, step, phases) —
 * c/fd_preconditioner.cpp:106-351 (the reference has no GPU version; its
 * GPU path runs the same sequence as ~20 cupy launches,
 * gpaw/preconditioner.py:74-93).  Writes the preconditioned residuals to
 * d0.  nresiduals (= -residuals) may be NULL: the negation is then applied
 * on load.  Scratch arrays q0, r1, d1, q1, r2, d2, q2 are caller-owned as
 * in the reference; their contents on return are unspecified. */
GB_API int gb_fd_precond(gb_transformer* rest0, gb_transformer* rest1, gb_transformer* intp1,
                  gb_transformer* intp2, gb_operator* kin0, gb_operator* kin1,
                  gb_operator* kin2, void* d0, void* q0, void* r1, void* d1, void* q1,
                  void* r2, void* d2, void* q2, const void* residuals,
                  const void* nresiduals, int64_t nin, int dtype, double step,
                  const double* phases, void* stream);

/* -------------------------------------------------------------- FD Poisson
 * Native executor for FDPoissonSolver's multigrid V-cycle
 * (gpaw/poisson.py:451-537).  nlevels = levels + 1 operators; levels
 * restrictors (level l -> l+1) and interpolators (level l+1 -> l), built
 * as FDPoissonSolver.set_grid_descriptor builds them (:366-430).
 * presmooths/postsmooths/weights per level as in :386-403 and :470-471.
 * dv is the volume element of level 0.  The objects passed in must outlive
 * the executor. */
GB_API int gb_poisson_new(int nlevels, gb_operator* const* operators,
                   gb_transformer* const* restrictors,
                   gb_transformer* const* interpolators, const int* presmooths,
                   const int* postsmooths, const double* weights, int relax_method,
                   double dv, gb_poisson** out);
GB_API void gb_poisson_free(gb_poisson* p);

/* Number of coarse levels the executor runs as one fused kernel (the
 * coarsest levels, when they are small enough for shared memory; 0 when
 * every level runs on its own kernels).  Introspection only: both forms
 * give the same V-cycle bit for bit.  No reference counterpart. */
GB_API int gb_poisson_fused_levels(const gb_poisson* p);

/* One V-cycle, FDPoissonSolver.iterate2(step, level=0) (:500-537): updates
 * phi in place and writes sum r^2 * dv to *error (host).  Synchronises the
 * stream once (to read the error). */
GB_API int gb_poisson_iterate(gb_poisson* p, double* phi, const double* rho, double* error,
                       void* stream);

/* FDPoissonSolver.solve_neutral(phi, rho) (:474-498): V-cycles until
 * error <= eps, at most maxiter (GB_ENOCONV when the loop stops at
 * maxiter, as the reference raises).  Periodic grids get the mean of phi
 * removed.  *niter and *error (host) receive the iteration count and the
 * last error. */
GB_API int gb_poisson_solve_neutral(gb_poisson* p, double* phi, const double* rho, double eps,
                             int maxiter, int* niter, double* error, void* stream);

/* ------------------------------------------------ mixed-precision Poisson
 * No counterpart in the reference (its Poisson solver is FP64 throughout):
 * FP32 V-cycles inside FP64 defect correction, for the neutral problem
 * L phi = rho of FDPoissonSolver.solve_neutral.  operators[0..nlevels-1]
 * are the levels' stencils (used in FP32 below the coarsest level, FP64 on
 * it), op64 the level-0 stencil applied in FP64 for the defect (normally
 * operators[0] itself); restrictors/interpolators connect the levels.
 * lam_max[l] is an upper bound of the spectrum of D^-1 A on level l (it sets
 * the degree-2 Chebyshev smoother, interval [lam_max/8, 1.05 lam_max]);
 * lam_min_coarse a lower bound on the coarsest level, which is solved with a
 * degree-`coarse_degree` FP64 Chebyshev iteration.  The objects passed in
 * must outlive the solver. */
typedef struct gb_mixed gb_mixed;
GB_API int gb_mixed_new(int nlevels, gb_operator* op64, gb_operator* const* operators,
                        gb_transformer* const* restrictors,
                        gb_transformer* const* interpolators, const double* lam_max,
                        double lam_min_coarse, int coarse_degree, gb_mixed** out);
GB_API void gb_mixed_free(gb_mixed* m);
/* How the coarse levels are solved: mode 1 (the default where the levels
 * allow it) the coarsest level exactly (fast diagonalisation) in one
 * cooperative kernel over every SM; mode 0 per-level kernels and the
 * Chebyshev iteration on the coarsest level; mode 2 the levels from the
 * first with at most 16384 points down to a coarsest of at most 4096 points
 * in one single-block kernel with the exact solve (for solves that run side
 * by side, as in a batch graph), else as mode 0.  The modes give slightly
 * different FP32 corrections, each deterministic.  No counterpart in the
 * reference.  Returns 0; a mode the levels do not allow falls back to 0. */
GB_API int gb_mixed_set_fused_coarse(gb_mixed* m, int mode);
/* One V-cycle of the mixed-precision solver and the defects around it,
 * launched kernel by kernel instead of through the solver's graph:
 * phi <- phi + V32(rho - L phi).  For profilers and kernel traces (its
 * kernels carry gb_trace labels); no counterpart in the reference. */
GB_API int gb_mixed_vcycle_eager(gb_mixed* m, double* phi, const double* rho, void* stream);

/* Solve until ||rho - L phi|| / ||rho|| <= tol (both norms in FP64, on the
 * device), starting from phi; at most maxiter V-cycles (GB_ENOCONV
 * otherwise).  Synchronises the stream once; *niter and *rel_residual
 * (host) receive the V-cycle count and the final relative residual. */
GB_API int gb_mixed_solve(gb_mixed* m, double* phi, const double* rho, double tol, int maxiter,
                          int* niter, double* rel_residual, void* stream);

/* Asynchronous forms (no counterpart in the reference): enqueue the whole
 * solve on `stream` and return at once; after the stream (or an event
 * recorded after the call) completes, *_result reports the V-cycle count and
 * the final error / relative residual, and GB_ENOCONV if the solve stopped
 * at maxiter.  A solver object serves one solve at a time: enqueue the next
 * solve on the same object only after the previous one's result was read or
 * on the same stream. */
GB_API int gb_poisson_solve_neutral_async(gb_poisson* p, double* phi, const double* rho,
                                          double eps, int maxiter, void* stream);
GB_API int gb_poisson_result(gb_poisson* p, int* niter, double* error);
GB_API int gb_mixed_solve_async(gb_mixed* m, double* phi, const double* rho, double tol,
                                int maxiter, void* stream);
GB_API int gb_mixed_result(gb_mixed* m, int* niter, double* rel_residual);
/* Build the solver's captured solve now (what the first gb_mixed_solve_async
 * otherwise does): one uncaptured pass on the solver's own stream, then the
 * capture; synchronous.  Lets a host thread prepare solvers while another
 * thread enqueues solves of other solvers.  No counterpart in the
 * reference. */
GB_API int gb_mixed_prepare(gb_mixed* m);

/* Many mixed-precision solves as one CUDA graph (no reference counterpart):
 * one branch per solver (distinct solvers, grids of any sizes), each the
 * solve of gb_mixed_solve_async with tolerance `tol` and at most `maxiter`
 * V-cycles; the branches run concurrently.  gb_mixed_batch_solve_async
 * takes one phi and one rho per solver (device arrays of that solver's
 * grid), enqueues the whole batch with one graph launch and returns;
 * gb_mixed_batch_result (after the stream reached that point) fills
 * niters[n] and rel_residuals[n] and returns GB_ENOCONV if any solve
 * stopped at maxiter.  The solvers must outlive the batch and must not be
 * used on their own while a batch launch is in flight.  A new launch first
 * waits for the stream's earlier work (the launch refreshes a table of
 * array addresses the previous one may still read). */
typedef struct gb_mixed_batch gb_mixed_batch;
GB_API int gb_mixed_batch_new(int n, gb_mixed* const* solvers, double tol, int maxiter,
                              gb_mixed_batch** out);
GB_API void gb_mixed_batch_free(gb_mixed_batch* b);
GB_API int gb_mixed_batch_solve_async(gb_mixed_batch* b, double* const* phis,
                                      const double* const* rhos, void* stream);
GB_API int gb_mixed_batch_result(gb_mixed_batch* b, int* niters, double* rel_residuals);

#ifdef __cplusplus
}
#endif

#endif /* GPAW_B200_H */
