// FP32 fused score + first-argmax kernel for MIP matching.
#pragma once

#include <cuda_runtime.h>

#include "common.h"

namespace snapmrf {

constexpr int kMatchVT = 64;       // voxels per CTA tile
constexpr int kMatchAT = 128;      // atoms per CTA tile
constexpr int kMatchKC = 16;       // time points per shared-memory stage
constexpr int kMatchThreads = 256; // 16 voxel groups x 16 atom groups

struct MatchArgs {
    const float2 *atoms;
    long long atom_stride;
    const float2 *img;
    long long img_stride;
    long long nreps;
    int nbins;
    long long bin_natoms;        // atoms per bin; bin b starts at atom b * bin_natoms
    const long long *slot_start; // [nbins + 1]
    const long long *tile_start; // [nbins + 1]
    const long long *perm;       // slot -> voxel (null: identity, or slot % perm_mod)
    long long perm_mod;
    long long nvox;
    unsigned long long *keys;    // [slots] packed (|s|^2 bits << 32 | ~atom)
    int atiles_per_split;
};

// Packs a non-negative score and a local atom index so that an unsigned max
// prefers the larger score and, for equal scores, the lower index.
__device__ __forceinline__ unsigned long long pack_key(float score, unsigned idx) {
    return ((unsigned long long)__float_as_uint(score) << 32) | (unsigned long long)(0xffffffffu - idx);
}

// Candidate (score, idx) beats (bs, bi): strictly larger score, or equal
// score with a lower index (bi < 0 means no candidate yet).
__device__ __forceinline__ bool beats(float s, int i, float bs, int bi) {
    return s > bs || (s == bs && i >= 0 && (bi < 0 || i < bi));
}

#ifdef SNAPMRF_MATCH_KERNEL_DECLARATION_ONLY
// Defined once, in match.cu.
__global__ void __launch_bounds__(kMatchThreads, 1) match_fp32_kernel(MatchArgs m);
#else
// One CTA: a tile of kMatchVT voxel slots of one bin against
// atiles_per_split tiles of kMatchAT atoms of that bin.  Thread (vy, ax)
// accumulates 4 voxels (vy + 16j) x 8 atoms (ax + 16i) complex scores
// s = sum_t conj(d_t) x_t in FP32 registers.
__global__ void __launch_bounds__(kMatchThreads, 1) match_fp32_kernel(MatchArgs m) {
    __shared__ float2 sA[kMatchKC][kMatchAT + 1];
    __shared__ float2 sB[kMatchKC][kMatchVT + 1];
    __shared__ long long sVox[kMatchVT];
    const int tid = threadIdx.x;
    const int ax = tid % 16, vy = tid / 16;
    const long long total_tiles = m.tile_start[m.nbins];

    for (long long tile = blockIdx.y; tile < total_tiles; tile += gridDim.y) {
        // bin of this tile (binary search over the tile prefix)
        int lo = 0, hi = m.nbins - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if (m.tile_start[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const int bin = lo;
        const long long s0 = m.slot_start[bin] + (tile - m.tile_start[bin]) * kMatchVT;
        const long long s_end = m.slot_start[bin + 1];
        const long long a_bin0 = (long long)bin * m.bin_natoms;
        const long long at_begin = (long long)blockIdx.x * m.atiles_per_split * kMatchAT;
        const long long at_end = min(m.bin_natoms, at_begin + (long long)m.atiles_per_split * kMatchAT);
        __syncthreads();
        if (tid < kMatchVT) {
            long long s = s0 + tid;
            long long v = -1;
            if (s < s_end) v = m.perm ? m.perm[s] : (m.perm_mod ? s % m.perm_mod : s);
            sVox[tid] = v;
        }
        __syncthreads();
        if (at_begin >= at_end) continue;

        float bscore[4];
        int bidx[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            bscore[j] = 0.f;
            bidx[j] = -1;
        }

        for (long long a0 = at_begin; a0 < at_end; a0 += kMatchAT) {
            float re[4][8], im[4][8];
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    re[j][i] = 0.f;
                    im[j][i] = 0.f;
                }
            for (long long k0 = 0; k0 < m.nreps; k0 += kMatchKC) {
                __syncthreads();
                // atoms: 128 rows x 16 samples, 8 per thread
#pragma unroll
                for (int r = 0; r < (kMatchAT * kMatchKC) / kMatchThreads; r++) {
                    int f = tid + r * kMatchThreads;
                    int row = f / kMatchKC, t = f % kMatchKC;
                    long long a = a0 + row, k = k0 + t;
                    float2 v = make_float2(0.f, 0.f);
                    if (a < at_end && k < m.nreps) v = m.atoms[(a_bin0 + a) * m.atom_stride + k];
                    sA[t][row] = v;
                }
                // voxels: 64 rows x 16 samples, 4 per thread
#pragma unroll
                for (int r = 0; r < (kMatchVT * kMatchKC) / kMatchThreads; r++) {
                    int f = tid + r * kMatchThreads;
                    int row = f / kMatchKC, t = f % kMatchKC;
                    long long v = sVox[row], k = k0 + t;
                    float2 x = make_float2(0.f, 0.f);
                    if (v >= 0 && k < m.nreps) x = m.img[v * m.img_stride + k];
                    sB[t][row] = x;
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < kMatchKC; kk++) {
                    float2 av[8], xv[4];
#pragma unroll
                    for (int i = 0; i < 8; i++) av[i] = sA[kk][ax + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; j++) xv[j] = sB[kk][vy + 16 * j];
#pragma unroll
                    for (int j = 0; j < 4; j++)
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            re[j][i] = fmaf(av[i].x, xv[j].x, re[j][i]);
                            re[j][i] = fmaf(av[i].y, xv[j].y, re[j][i]);
                            im[j][i] = fmaf(av[i].x, xv[j].y, im[j][i]);
                            im[j][i] = fmaf(-av[i].y, xv[j].x, im[j][i]);
                        }
                }
            }
            // epilogue: running first-argmax of |s|^2 over this thread's atoms
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    long long a = a0 + ax + 16 * i;
                    float sc = re[j][i] * re[j][i] + im[j][i] * im[j][i];
                    if (a < at_end && sc > bscore[j]) {
                        bscore[j] = sc;
                        bidx[j] = (int)a;
                    }
                }
        }
        // combine the 16 atom groups of each voxel (lanes of one half-warp)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float bs = bscore[j];
            int bi = bidx[j];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                float os = __shfl_xor_sync(0xffffffffu, bs, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (beats(os, oi, bs, bi)) {
                    bs = os;
                    bi = oi;
                }
            }
            int vrow = vy + 16 * j;
            if (ax == 0 && bi >= 0 && sVox[vrow] >= 0) {
                long long slot = s0 + vrow;
                atomicMax(&m.keys[slot], pack_key(bs, (unsigned)bi));
            }
        }
    }
}

#endif  // SNAPMRF_MATCH_KERNEL_DECLARATION_ONLY

inline cudaError_t launch_match_fp32(const MatchArgs &m, dim3 grid, cudaStream_t st) {
    match_fp32_kernel<<<grid, kMatchThreads, 0, st>>>(m);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace snapmrf
