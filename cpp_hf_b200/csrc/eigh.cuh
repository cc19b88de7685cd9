// Internal interface of the batched Jacobi eigensolver.
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kMaxEighNb = 80;

// Optional block-diagonal structure (linalg.hpp:72-120): entries outside the
// diagonal blocks are ignored; sort=0 orders eigenvalues block by block.
struct BlockSpec {
    int nblocks;
    int sort;
    short start[kMaxEighNb + 1];
    unsigned char blk[kMaxEighNb];
};

// mode 0: eigh(herm(M)); mode 1: eigh(herm(i M)) (Cayley spectral setup).
int eigh_batched(const double2* M, double* w, double2* V, int64_t batch, int64_t nb, int mode,
                 const BlockSpec* bs, cudaStream_t st);
int make_block_spec(int64_t nb, const int64_t* sizes, int64_t n_sizes, int sort, BlockSpec& bs);
// Host decision of solver_dm.hpp:92-98: max off-block |M| <= 1e-10 + 1e-10 max |M|
// over a batch of nb x nb matrices.  dev2 is 16 bytes of device scratch;
// synchronises the stream.
int block_structure_ok(const double2* M, int64_t batch, int64_t nb, const BlockSpec& bs, unsigned long long* dev2,
                       cudaStream_t st, bool* ok);

// Householder + implicit QL path for 2 <= nb <= 8 (eigh_small.cu); other nb run
// the Jacobi kernels of eigh.cu.
bool eigh_small_enabled(int64_t nb);
int eigh_small(const double2* M, double* w, double2* V, int64_t batch, int64_t nb, int mode, cudaStream_t st);

}  // namespace cpphf
