// FP32 fused score + first-argmax kernel for MIP matching.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"

namespace snapmrf {

constexpr int kMatchVT = 64;       // voxels per CTA tile
constexpr int kMatchAT = 128;      // atoms per CTA tile
constexpr int kMatchKC = 8;        // time points per shared-memory stage
constexpr int kMatchThreads = 256; // 8 warps: 4 atom rows x 2 voxel columns

struct MatchArgs {
    const float2 *atoms;
    long long atom_stride;
    const float2 *img;
    long long img_stride;
    long long nreps;
    int nbins;
    long long bin_natoms;        // atoms per bin (< 2^31); bin b starts at atom b * bin_natoms
    const long long *slot_start; // [nbins + 1]
    const long long *tile_start; // [nbins + 1]
    const long long *perm;       // slot -> voxel (null: identity, or slot % perm_mod)
    long long perm_mod;
    long long nvox;
    unsigned long long *keys;    // [slots] packed (|s|^2 bits << 32 | ~atom)
    int atiles_per_split;
    int *err;                    // imaginary form: set to 7 when an atom has a real part
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

// Shared memory of one CTA: two stages of kMatchKC time points, the atoms
// transposed to [t][atom] (imaginary parts only in the IMAG form; rows
// 16-byte aligned) and the voxels to [t][voxel], plus each thread's running
// best per voxel column (kept here while the accumulators hold the
// registers).
template <bool IMAG>
struct MatchSmem {
    static constexpr int APITCH = IMAG ? kMatchAT + 4 : 2 * (kMatchAT + 2);  // floats per row
    float a[2][kMatchKC][APITCH];
    float2 x[2][kMatchKC][kMatchVT];
    long long vox[kMatchVT];
    float best_s[4][kMatchThreads];
    int best_i[4][kMatchThreads];
};

#ifdef SNAPMRF_MATCH_KERNEL_DECLARATION_ONLY
// Defined once, in match.cu.
template <bool IMAG, bool VEC>
__global__ void __launch_bounds__(kMatchThreads, 2) match_fp32_kernel(MatchArgs m);
#else
// One CTA: a tile of kMatchVT voxel slots of one bin against
// atiles_per_split tiles of kMatchAT atoms of that bin.  Warp w covers atoms
// 32 (w / 2) .. + 31 and voxels 32 (w % 2) .. + 31; lane (ag, vg) = (lane / 8,
// lane % 8) accumulates atoms 8 ag .. 8 ag + 7 of its warp's rows against
// voxels vg + 8 j (j < 4).  Scores s = sum_t conj(d_t) x_t:
//   complex form: Re s += dr xr + di xi, Im s += dr xi - di xr (4 FMA);
//   IMAG form (every dr = 0): Re s += di xi, Im s += -di xr (2 FMA), the same
//   roundings as the complex form, whose dr products add exact zeros.
// The next stage's global loads are held in registers while the current
// stage is multiplied (VEC: 16-byte loads of two samples, every row start
// 16-byte aligned).
template <bool IMAG, bool VEC>
__global__ void __launch_bounds__(kMatchThreads, 2) match_fp32_kernel(MatchArgs m) {
    extern __shared__ __align__(16) unsigned char match_smem[];
    MatchSmem<IMAG> &sm = *reinterpret_cast<MatchSmem<IMAG> *>(match_smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp >> 1, wc = warp & 1;
    const int ag = lane >> 3, vg = lane & 7;
    const int arow0 = wr * 32 + ag * 8;      // this thread's first atom row in the tile
    const int vcol0 = wc * 32 + vg;          // voxel columns vcol0 + 8 j
    const long long total_tiles = m.tile_start[m.nbins];
    // global-load assignment: each lane loads one 16-byte pair of samples
    // (q of the stage's kMatchKC / 2) of rows lrow + kRowsPerPass i
    constexpr int kLanesPerRow = kMatchKC / 2;
    constexpr int kRowsPerPass = kMatchThreads / kLanesPerRow;
    constexpr int kAtomPasses = kMatchAT / kRowsPerPass, kVoxPasses = kMatchVT / kRowsPerPass;
    static_assert(kVoxPasses >= 1 && kMatchVT % kRowsPerPass == 0, "stage geometry");
    const int q = tid % kLanesPerRow, lrow = tid / kLanesPerRow;
    bool real_part = false;

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
        // atom positions within the bin fit an int (fewer than 2^31 atoms per bin)
        const int at_begin = (int)min((long long)blockIdx.x * m.atiles_per_split * kMatchAT, m.bin_natoms);
        const int at_end = (int)min(m.bin_natoms, (long long)at_begin + (long long)m.atiles_per_split * kMatchAT);
        __syncthreads();
        if (tid < kMatchVT) {
            long long s = s0 + tid;
            long long v = -1;
            if (s < s_end) v = m.perm ? m.perm[s] : (m.perm_mod ? s % m.perm_mod : s);
            sm.vox[tid] = v;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sm.best_s[j][tid] = 0.f;
            sm.best_i[j][tid] = -1;
        }
        __syncthreads();
        if (at_begin >= at_end) continue;

        // this thread's voxel rows (null: an empty slot)
        const float2 *px[kVoxPasses];
#pragma unroll
        for (int i = 0; i < kVoxPasses; i++) {
            const long long v = sm.vox[lrow + kRowsPerPass * i];
            px[i] = v >= 0 ? m.img + v * m.img_stride + 2 * q : nullptr;
        }
        const int nk = (int)((m.nreps + kMatchKC - 1) / kMatchKC);
        const int nreps = (int)m.nreps;

        for (int a0 = at_begin; a0 < at_end; a0 += kMatchAT) {
            float4 ra[kAtomPasses], rx[kVoxPasses];
            // this thread's atom rows (null past the end of the split)
            const float2 *pa[kAtomPasses];
#pragma unroll
            for (int i = 0; i < kAtomPasses; i++) {
                const int a = a0 + lrow + kRowsPerPass * i;
                pa[i] = a < at_end ? m.atoms + (a_bin0 + a) * m.atom_stride + 2 * q : nullptr;
            }
            // two samples (t, t + 1) of a row, zeros past nreps
            auto fetch = [&](const float2 *p, int t) {
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (p) {
                    if (VEC && t + 1 < nreps) {
                        v = __ldg(reinterpret_cast<const float4 *>(p));
                    } else {
                        if (t < nreps) { const float2 u = __ldg(p); v.x = u.x; v.y = u.y; }
                        if (t + 1 < nreps) { const float2 u = __ldg(p + 1); v.z = u.x; v.w = u.y; }
                    }
                }
                return v;
            };
            // loads of stage k0 into registers
            auto load = [&](int k0) {
                const int t = k0 * kMatchKC + 2 * q;
#pragma unroll
                for (int i = 0; i < kAtomPasses; i++) ra[i] = fetch(pa[i] ? pa[i] + k0 * kMatchKC : nullptr, t);
#pragma unroll
                for (int i = 0; i < kVoxPasses; i++) rx[i] = fetch(px[i] ? px[i] + k0 * kMatchKC : nullptr, t);
            };
            auto store = [&](int buf) {
#pragma unroll
                for (int i = 0; i < kAtomPasses; i++) {
                    const int r = lrow + kRowsPerPass * i;
                    if (IMAG) {
                        real_part |= (ra[i].x != 0.f) | (ra[i].z != 0.f);
                        sm.a[buf][2 * q][r] = ra[i].y;
                        sm.a[buf][2 * q + 1][r] = ra[i].w;
                    } else {
                        reinterpret_cast<float2 *>(sm.a[buf][2 * q])[r] = make_float2(ra[i].x, ra[i].y);
                        reinterpret_cast<float2 *>(sm.a[buf][2 * q + 1])[r] = make_float2(ra[i].z, ra[i].w);
                    }
                }
#pragma unroll
                for (int i = 0; i < kVoxPasses; i++) {
                    const int r = lrow + kRowsPerPass * i;
                    sm.x[buf][2 * q][r] = make_float2(rx[i].x, rx[i].y);
                    sm.x[buf][2 * q + 1][r] = make_float2(rx[i].z, rx[i].w);
                }
            };

            float acc_r[4][8], acc_i[4][8];
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    acc_r[j][i] = 0.f;
                    acc_i[j][i] = 0.f;
                }
            load(0);
            __syncthreads();  // the previous atom tile's readers are done
            store(0);
            __syncthreads();
            for (int k0 = 0; k0 < nk; k0++) {
                const int buf = k0 & 1;
                if (k0 + 1 < nk) load(k0 + 1);
#pragma unroll
                for (int kk = 0; kk < kMatchKC; kk++) {
                    float2 xv[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) xv[j] = sm.x[buf][kk][vcol0 + 8 * j];
                    if (IMAG) {
                        const float4 d0 = *reinterpret_cast<const float4 *>(&sm.a[buf][kk][arow0]);
                        const float4 d1 = *reinterpret_cast<const float4 *>(&sm.a[buf][kk][arow0 + 4]);
                        const float di[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
#pragma unroll
                        for (int j = 0; j < 4; j++)
#pragma unroll
                            for (int i = 0; i < 8; i++) {
                                acc_r[j][i] = fmaf(di[i], xv[j].y, acc_r[j][i]);
                                acc_i[j][i] = fmaf(-di[i], xv[j].x, acc_i[j][i]);
                            }
                    } else {
                        const float4 *row = reinterpret_cast<const float4 *>(&sm.a[buf][kk][2 * arow0]);
                        float2 d[8];
#pragma unroll
                        for (int h = 0; h < 4; h++) {
                            const float4 u = row[h];
                            d[2 * h] = make_float2(u.x, u.y);
                            d[2 * h + 1] = make_float2(u.z, u.w);
                        }
#pragma unroll
                        for (int j = 0; j < 4; j++)
#pragma unroll
                            for (int i = 0; i < 8; i++) {
                                acc_r[j][i] = fmaf(d[i].x, xv[j].x, acc_r[j][i]);
                                acc_r[j][i] = fmaf(d[i].y, xv[j].y, acc_r[j][i]);
                                acc_i[j][i] = fmaf(d[i].x, xv[j].y, acc_i[j][i]);
                                acc_i[j][i] = fmaf(-d[i].y, xv[j].x, acc_i[j][i]);
                            }
                    }
                }
                if (k0 + 1 < nk) {
                    store(buf ^ 1);
                    __syncthreads();
                }
            }
            // running first-argmax of |s|^2 over this thread's atoms (in
            // increasing order, so strict '>' keeps the lowest index)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float bs = sm.best_s[j][tid];
                int bi = sm.best_i[j][tid];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int a = a0 + arow0 + i;
                    const float sc = acc_r[j][i] * acc_r[j][i] + acc_i[j][i] * acc_i[j][i];
                    if (a < at_end && sc > bs) {
                        bs = sc;
                        bi = a;
                    }
                }
                sm.best_s[j][tid] = bs;
                sm.best_i[j][tid] = bi;
            }
        }
        // combine the four atom groups of each voxel (lanes vg, vg + 8, ...),
        // then one atomicMax per voxel and atom row of warps
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float bs = sm.best_s[j][tid];
            int bi = sm.best_i[j][tid];
#pragma unroll
            for (int o = 8; o < 32; o <<= 1) {
                const float os = __shfl_xor_sync(0xffffffffu, bs, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (beats(os, oi, bs, bi)) {
                    bs = os;
                    bi = oi;
                }
            }
            const int vcol = vcol0 + 8 * j;
            if (ag == 0 && bi >= 0 && sm.vox[vcol] >= 0) atomicMax(&m.keys[s0 + vcol], pack_key(bs, (unsigned)bi));
        }
    }
    if (IMAG && m.err && __any_sync(0xffffffffu, real_part) && lane == 0) atomicCAS(m.err, 0, 7);
}
#endif  // SNAPMRF_MATCH_KERNEL_DECLARATION_ONLY

inline size_t match_fp32_smem(bool imag) {
    return imag ? sizeof(MatchSmem<true>) : sizeof(MatchSmem<false>);
}

// Grid of the FP32 kernel: y walks the voxel tiles (bin-major, so CTAs that
// run together share a bin's atoms in L2), x splits each bin's atom tiles so
// that about 16 waves of two resident CTAs per SM keep the last wave's idle
// share small.  Sets m.atiles_per_split.  tiles_est: voxel tiles the grid
// covers; max_tiles: an upper bound of the tile count.
inline dim3 fp32_match_grid(MatchArgs &m, long long tiles_est, long long max_tiles) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        sms = 148;
    }
    const long long atiles = (m.bin_natoms + kMatchAT - 1) / kMatchAT;
    const long long target = (long long)sms * 2 * 16;
    long long splits = std::max(1ll, std::min(atiles, (target + tiles_est - 1) / std::max(1ll, tiles_est)));
    m.atiles_per_split = (int)((atiles + splits - 1) / splits);
    splits = (atiles + m.atiles_per_split - 1) / m.atiles_per_split;
    return dim3((unsigned)splits, (unsigned)std::min(max_tiles, 65535ll));
}

// Launches the imaginary-atom or complex form; 16-byte loads when every atom
// and voxel row starts 16-byte aligned.
inline cudaError_t launch_match_fp32(const MatchArgs &m, dim3 grid, bool imag, cudaStream_t st) {
    const bool vec = (m.atom_stride % 2 == 0) && (m.img_stride % 2 == 0) &&
                     (reinterpret_cast<uintptr_t>(m.atoms) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(m.img) % 16 == 0);
    const size_t smem = match_fp32_smem(imag);
    auto k = imag ? (vec ? match_fp32_kernel<true, true> : match_fp32_kernel<true, false>)
                  : (vec ? match_fp32_kernel<false, true> : match_fp32_kernel<false, false>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, kMatchThreads, smem, st>>>(m);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace snapmrf
