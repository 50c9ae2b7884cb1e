// Host interface of the tensor-core matching path (match_tc.cu).
#pragma once

#include <cuda_runtime.h>

namespace snapmrf {

struct TcMatchRequest {
    float *maps;             // out [nvox][5]
    long long *index_out;    // optional out [nvox]
    const float2 *img;       // device [nvox][img_stride]
    long long img_stride;
    const float2 *atoms;     // device [NATOMS][atom_stride]
    long long atom_stride;
    const float *params;     // device [NATOMS][nparams]
    int nparams;
    long long nreps, NATOMS, natoms, nvox;
    int nblocks;
    const float *b1map;      // device [nvox] or null
    int fmt;                 // operands: 0 bf16, 1 fp16, 2 e4m3 (per-row scales)
    bool imag;               // atoms purely imaginary (bf16 / fp16: half the MMA work)
    const void *packed;      // optional: the atoms' imaginary rows, already packed (imag)
    int topk;                // candidates rescored in FP32: 8 or 16
    // compressed matching (basis != null): voxels are projected onto their
    // bin's rank-r basis and scored against the atoms' coordinates; the
    // candidates are rescored against `atoms` (the coordinates when null)
    const float2 *basis;     // device [nblocks][basis_rows][basis_stride]
    long long basis_rows, basis_stride;
    const float2 *coeffs;    // device [NATOMS][coeff_stride]
    long long coeff_stride;
    int rank;
    // optional device [NATOMS]: norms of `atoms`, which are not normalised;
    // the rescoring divides each candidate's inner product by its norm
    const float *atom_norms = nullptr;
    // `atoms` holds Im rows ([NATOMS][atom_stride] float) of purely
    // imaginary atoms; only the rescoring reads them (packed operand given)
    bool imag_rows = false;
};

// BF16 / FP16 / E4M3 tcgen05 scores + top-k + FP32 rescoring; enqueued on st.
int match_bf16(const TcMatchRequest &q, cudaStream_t st);

}  // namespace snapmrf
