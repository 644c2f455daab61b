// Test and benchmark infrastructure only: drives the reference's own GPU
// kernels (c/gpu/kernels/{fd,paste,translate,restrict,interpolate}.cpp,
// compiled for sm_100a from the reference's sources by `make -C oracle gpu`)
// so that they can be timed beside this library's kernels.  Nothing in the
// library links or calls this.
//
// The call sequence is the reference's single-domain GPU path without its
// two-stream overlap (c/gpu/operators.cpp:268-316 and
// c/gpu/transformers.cpp:107-176): for every block of at most 16 grids,
// the input is pasted into a zeroed padded buffer (bc_unpack_paste_gpu,
// c/gpu/bc.cpp:246-290), each axis's periodic halos are copied inside the
// buffer with their Bloch phase (bc_unpack_gpu, c/gpu/bc.cpp:346-360), and
// the stencil, restriction or interpolation kernel runs on the buffer.
// The halo geometry comes from the reference's own bc_init (c/bc.cpp).
// Buffers are allocated here once per object (the reference keeps static
// ones).
#include <cstdlib>
#include <cstring>
#include <complex>

#include "extensions.h"
#include "bc.h"
#include "bmgs/bmgs.h"
#include "gpu/gpu.h"
#include "gpu/gpu-complex.h"
#include "gpu/bmgs.h"

// The reference's bc_init calls this to size its static GPU buffers; the
// buffers here are the objects' own, so it has nothing to do.
void bc_init_gpu(boundary_conditions*) {}

namespace {
constexpr int BLOCKS = GPU_BLOCKS_MIN;   // grids a block, as the reference picks for one rank

struct RefOp {
    boundary_conditions* bc = nullptr;
    bmgsstencil st{};
    bmgsstencil_gpu sg{};
    double* buf = nullptr;   // padded buffer, BLOCKS grids
    int real = 1;
};

struct RefTr {
    boundary_conditions* bc = nullptr;
    int k = 2, interpolate = 0, real = 1;
    int size_out[3];
    int skip[3][2];
    double* buf = nullptr;
    double* buf16 = nullptr;
};

// paste + halo copies of one block of `nb` grids into `buf`
void fill_halos(boundary_conditions* bc, const double* in, double* buf, int nb, int real,
                const double* phases) {
    if (real)
        bmgs_paste_zero_gpu(in, bc->size1, buf, bc->size2, bc->sendstart[0][0], nb, 0);
    else
        bmgs_paste_zero_gpuz((const gpuDoubleComplex*)in, bc->size1, (gpuDoubleComplex*)buf,
                             bc->size2, bc->sendstart[0][0], nb, 0);
    for (int i = 0; i < 3; i++)
        for (int d = 0; d < 2; d++) {
            if (bc->sendproc[i][d] != COPY_DATA) continue;
            if (real) {
                bmgs_translate_gpu(buf, bc->size2, bc->sendsize[i][d], bc->sendstart[i][d],
                                   bc->recvstart[i][1 - d], nb, 0);
            } else {
                gpuDoubleComplex ph = {1.0, 0.0};
                if (phases) ph = {phases[(2 * i + d) * 2], phases[(2 * i + d) * 2 + 1]};
                bmgs_translate_gpuz((gpuDoubleComplex*)buf, bc->size2, bc->sendsize[i][d],
                                    bc->sendstart[i][d], bc->recvstart[i][1 - d], ph, nb, 0);
            }
        }
}
}  // namespace

extern "C" {

void* refgpu_operator_new(const double* coefs, const long* offsets, int ncoefs, int range,
                          const long size[3], const long neighbors[6], int real) {
    RefOp* op = new RefOp();
    long pad[3][2], nb[3][2];
    for (int c = 0; c < 3; c++) {
        pad[c][0] = pad[c][1] = range;
        nb[c][0] = neighbors[2 * c];
        nb[c][1] = neighbors[2 * c + 1];
    }
    op->bc = bc_init(size, pad, pad, nb, MPI_COMM_NULL, real != 0, true);
    op->st = bmgs_stencil(ncoefs, coefs, offsets, range, size);
    op->sg = bmgs_stencil_to_gpu(&op->st);
    op->real = real;
    const size_t ng2 = (size_t)op->bc->size2[0] * op->bc->size2[1] * op->bc->size2[2];
    if (cudaMalloc(&op->buf, ng2 * (real ? 1 : 2) * sizeof(double) * BLOCKS) != cudaSuccess) {
        delete op;
        return nullptr;
    }
    return op;
}

int refgpu_operator_apply(void* h, const double* in, double* out, int nin,
                          const double* phases) {
    RefOp* op = (RefOp*)h;
    const int* s1 = op->bc->size1;
    const long ng = (long)(op->real ? 1 : 2) * s1[0] * s1[1] * s1[2];
    for (int n = 0; n < nin; n += BLOCKS) {
        const int m = nin - n < BLOCKS ? nin - n : BLOCKS;
        fill_halos(op->bc, in + n * ng, op->buf, m, op->real, phases);
        if (op->real)
            bmgs_fd_gpu(&op->sg, op->buf, out + n * ng, GPAW_BOUNDARY_NORMAL, m, 0);
        else
            bmgs_fd_gpuz(&op->sg, (const gpuDoubleComplex*)op->buf,
                         (gpuDoubleComplex*)(out + n * ng), GPAW_BOUNDARY_NORMAL, m, 0);
    }
    return (int)cudaGetLastError();
}

void* refgpu_transformer_new(const long size_in[3], const long size_out[3], int k,
                             const long pads[6], const long npads[6], const long skip[6],
                             const long neighbors[6], int real, int interpolate) {
    RefTr* t = new RefTr();
    long pad[3][2], npad[3][2], nb[3][2];
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 2; d++) {
            pad[c][d] = pads[2 * c + d];
            npad[c][d] = npads[2 * c + d];
            nb[c][d] = neighbors[2 * c + d];
            t->skip[c][d] = (int)skip[2 * c + d];
        }
    t->bc = bc_init(size_in, pad, npad, nb, MPI_COMM_NULL, real != 0, false);
    t->k = k;
    t->interpolate = interpolate;
    t->real = real;
    for (int c = 0; c < 3; c++) t->size_out[c] = (int)size_out[c];
    const int* s2 = t->bc->size2;
    const size_t ng2 = (size_t)s2[0] * s2[1] * s2[2] * (real ? 1 : 2);
    // the reference's scratch of the stencil variants: 16 times the padded
    // grid (c/gpu/transformers.cpp:26-44)
    if (cudaMalloc(&t->buf, ng2 * sizeof(double) * BLOCKS) != cudaSuccess ||
        cudaMalloc(&t->buf16, 16 * ng2 * sizeof(double) * BLOCKS) != cudaSuccess) {
        delete t;
        return nullptr;
    }
    return t;
}

int refgpu_transformer_apply(void* h, const double* in, double* out, int nin,
                             const double* phases) {
    RefTr* t = (RefTr*)h;
    const int* s1 = t->bc->size1;
    const long ng = (long)(t->real ? 1 : 2) * s1[0] * s1[1] * s1[2];
    const long ngo = (long)(t->real ? 1 : 2) * t->size_out[0] * t->size_out[1] * t->size_out[2];
    // the optimised kernels exist for k = 2 only; otherwise the stencil
    // variants (c/gpu/transformers.cpp:103-106)
    const bool stencil = t->k != 2;
    for (int n = 0; n < nin; n += BLOCKS) {
        const int m = nin - n < BLOCKS ? nin - n : BLOCKS;
        fill_halos(t->bc, in + n * ng, t->buf, m, t->real, phases);
        gpuDoubleComplex* zb = (gpuDoubleComplex*)t->buf;
        gpuDoubleComplex* zo = (gpuDoubleComplex*)(out + n * ngo);
        gpuDoubleComplex* z16 = (gpuDoubleComplex*)t->buf16;
        if (t->interpolate) {
            if (stencil) {
                if (t->real)
                    bmgs_interpolate_stencil_gpu(t->k, t->skip, t->buf, t->bc->size2,
                                                 out + n * ngo, t->size_out, t->buf16, m);
                else
                    bmgs_interpolate_stencil_gpuz(t->k, t->skip, zb, t->bc->size2, zo,
                                                  t->size_out, z16, m);
            } else {
                if (t->real)
                    bmgs_interpolate_gpu(t->k, t->skip, t->buf, t->bc->size2, out + n * ngo,
                                         t->size_out, m);
                else
                    bmgs_interpolate_gpuz(t->k, t->skip, zb, t->bc->size2, zo, t->size_out, m);
            }
        } else {
            if (stencil) {
                if (t->real)
                    bmgs_restrict_stencil_gpu(t->k, t->buf, t->bc->size2, out + n * ngo,
                                              t->size_out, t->buf16, m);
                else
                    bmgs_restrict_stencil_gpuz(t->k, zb, t->bc->size2, zo, t->size_out, z16, m);
            } else {
                if (t->real)
                    bmgs_restrict_gpu(t->k, t->buf, t->bc->size2, out + n * ngo, t->size_out, m);
                else
                    bmgs_restrict_gpuz(t->k, zb, t->bc->size2, zo, t->size_out, m);
            }
        }
    }
    return (int)cudaGetLastError();
}

}  // extern "C"
