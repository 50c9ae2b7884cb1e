// Projection of voxels onto a B1 block's low-rank basis (svd.cu), used by
// the compressed forms of snapmrf_mrf_match.
#pragma once

#include <cuda_runtime.h>

namespace snapmrf {

// out[v][c] = sum_t conj(basis[bin(v)][c][t]) img[v][t] for c < rank, with
// bin(v) = vox_bin[v] (block 0 when vox_bin is null); columns [rank,
// out_stride) are set to zero.  real_basis: the basis' imaginary parts are
// taken as 0 (not read).  Enqueued on st; allocates stream-ordered scratch.
int project_voxels(float2 *out, long long out_stride, const float2 *img, long long img_stride,
                   long long nvox, long long nreps, const int *vox_bin, int nbins, const float2 *basis,
                   long long basis_rows, long long basis_stride, int rank, bool real_basis, cudaStream_t st);

}  // namespace snapmrf
