// Tensor-core matching on sm_100a: BF16, FP16 or FP8-E4M3 real-stacked scores on
// tcgen05 with FP32 accumulation in TMEM, a per-voxel running top-k (8 or
// 16) in the epilogue, then exact FP32 rescoring of the k candidates (the maps then follow the
// reference's rules: first argmax of |s| among them, PD = |s|).
//
// Operands.  The complex score s = sum_t conj(d_t) x_t is a real GEMM over
// K = 2T: a voxel row is its samples interleaved (Re x_t, Im x_t), and an
// atom gives two rows, (Re d_t, Im d_t) -> Re s and (-Im d_t, Re d_t) ->
// Im s.  D = A B^T with A = voxels (M, TMEM lanes) and B = atom rows (N, TMEM
// columns), so each epilogue thread owns one voxel and sees the (Re s, Im s)
// column pairs of 128 atoms per tile: the top-k update needs no cross-thread
// reduction.
//
// Kernel (one persistent CTA per SM, 320 threads):
//   warp 0     TMA producer: voxel tile (128 x 64 bf16) + atom tile
//              (256 x 64 bf16) per K-chunk into a 4-stage ring, 128-byte
//              swizzle;
//   warp 1     allocates 512 TMEM columns, issues tcgen05.mma (M 128, N 256,
//              K 16) into one of two accumulators, commits to mbarriers;
//   warps 2-9  epilogue, two warps per TMEM lane group, each on half of the
//              accumulator's columns: tcgen05.ld, |s|^2, top-k insertion,
//              release of the accumulator.  Each voxel leaves two top-k
//              lists; the rescoring kernel takes the k best of their union.
// Work items are (B1 block, 128-voxel tile); each item loops over all atom
// tiles of its block.  Every mbarrier wait is bounded (sm100.cuh) and sets a
// device error word instead of hanging.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>

#include "common.h"
#include "match_tc.h"
#include "sm100.cuh"
#include "svd.h"

namespace snapmrf {

// Kernels of the FP32 matching path (match.cu).
__global__ void assign_bins_kernel(int *vox_bin, int *counts, const float *b1map, const float *params,
                                   int nparams, long long natoms, int nblocks, long long nvox);
__global__ void scatter_bins_kernel(long long *perm, long long *cursor, const int *vox_bin,
                                    long long nvox);

namespace tc {

constexpr int BM = 128;                 // voxels per tile (TMEM lanes)
constexpr int BA = 128;                 // atoms per tile
constexpr int BN = 2 * BA;              // B rows per tile
constexpr int BK = 64;                  // bf16 per 128-byte swizzled row
constexpr int BK8 = 128;                // e4m3 per 128-byte swizzled row
constexpr float E4M3_MAX = 448.f;       // largest finite E4M3 value
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;    // 16 KB
constexpr int B_BYTES = BN * BK * 2;    // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int TOPK_MAX = 16;
constexpr int NLISTS = 2;               // top-k lists per voxel (one per half tile)
constexpr int THREADS = 320;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;
constexpr uint32_t TMEM_COLS = 512;

__device__ int g_device_error;

struct Args {
    const long long *tile_start;  // [nbins + 1]
    int nbins;
    long long bin_natoms;
    int nk;                       // K chunks of BK
    int tile_stride;              // atom tiles visited in the order (at * tile_stride) % natiles
    uint32_t idesc;               // tcgen05 instruction descriptor
    const float *ascale2;         // E4M3: [NATOMS] 1 / (atom scale)^2
    float *top_s;                 // [slots][TOPK]
    int *top_i;                   // [slots][TOPK]
    int *err;
};

__device__ __forceinline__ int find_bin(const long long *tile_start, int nbins, long long item) {
    int lo = 0, hi = nbins - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (tile_start[mid] <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Insertion into a descending list; strict '>' keeps earlier (lower-index)
// entries ahead of equal scores.
template <int TOPK>
__device__ __forceinline__ void topk_insert(float *ts, int *ti, float s, int i) {
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
        bool gt = s > ts[k];
        float t = ts[k];
        int u = ti[k];
        ts[k] = gt ? s : t;
        ti[k] = gt ? i : u;
        s = gt ? t : s;
        i = gt ? u : i;
    }
}

// FP8: E4M3 operands on kind::f8f6f4, one 128-byte row holding 128 elements
// of K, and scores divided by the atom's squared scale before the top-k.
// IMAG: purely imaginary atoms d = i v.  Then s = -i sum v x, |s|^2 =
// (sum v x_r)^2 + (sum v x_i)^2: a voxel gives two A rows (x_r, x_i) in
// neighbouring TMEM lanes, an atom one B row v, K = T: half the MMA work.
// A tile is 64 voxels x 256 atoms; the two lanes of a voxel swap halves of
// each 32-column load and keep a top-k each over half the atoms, merged at
// the end of the item.
template <int TOPK, bool FP8, bool IMAG>
__global__ void __launch_bounds__(THREADS, 1)
match_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Args p) {
    constexpr int BKE = FP8 ? BK8 : BK;   // K elements per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], tfull[2], tempty[2], mma_done;
    __shared__ uint32_t tmem_base_sh;
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr int IPT = IMAG ? 2 : 1;       // work items per 128-slot tile
    constexpr int APT = IMAG ? BN : BA;     // atoms per B tile
    const long long total = p.tile_start[p.nbins] * IPT;
    const int natiles = (int)((p.bin_natoms + APT - 1) / APT);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            sm100::mbar_init(&full[s], 1);
            sm100::mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            sm100::mbar_init(&tfull[a], 1);
            sm100::mbar_init(&tempty[a], 256);
        }
        sm100::mbar_init(&mma_done, 1);
        sm100::fence_mbar_init();
        sm100::prefetch_tmap(&tmA);
        sm100::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        sm100::tmem_alloc(&tmem_base_sh, TMEM_COLS);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            int stage = 0;
            uint32_t phase = 0;
            int issued[STAGES];
            for (int s = 0; s < STAGES; s++) issued[s] = -1;
            bool ok = true;
            for (long long item = blockIdx.x; item < total && ok; item += gridDim.x) {
                const int bin = find_bin(p.tile_start, p.nbins, item / IPT);
                const int vrow = (int)(item * BM);
                for (int at = 0; at < natiles && ok; at++) {
                    const long long pt = (long long)at * p.tile_stride % natiles;
                    const int brow = IMAG ? (int)((long long)bin * p.bin_natoms + pt * APT)
                                          : (int)(2 * ((long long)bin * p.bin_natoms + pt * BA));
                    for (int kc = 0; kc < p.nk; kc++) {
                        if (!sm100::mbar_wait(&empty[stage], phase ^ 1, p.err, 1)) {
                            ok = false;
                            break;
                        }
                        sm100::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                        unsigned char *sa = smem + stage * STAGE_BYTES;
                        sm100::tma_load_2d(sa, &tmA, &full[stage], kc * BKE, vrow);
                        sm100::tma_load_2d(sa + A_BYTES, &tmB, &full[stage], kc * BKE, brow);
                        issued[stage] = (int)phase;
                        if (++stage == STAGES) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
            }
            // every load issued must land before the CTA may exit
            for (int s = 0; s < STAGES; s++)
                if (issued[s] >= 0) sm100::mbar_wait(&full[s], (uint32_t)issued[s], p.err, 5);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int stage = 0, acc = 0;
            uint32_t phase = 0, aphase = 0;
            bool ok = true;
            const uint32_t idesc = p.idesc;
            for (long long item = blockIdx.x; item < total && ok; item += gridDim.x) {
                for (int at = 0; at < natiles && ok; at++) {
                    if (!sm100::mbar_wait(&tempty[acc], aphase ^ 1, p.err, 2)) {
                        ok = false;
                        break;
                    }
                    sm100::tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(acc * BN);
                    for (int kc = 0; kc < p.nk; kc++) {
                        if (!sm100::mbar_wait(&full[stage], phase, p.err, 3)) {
                            ok = false;
                            break;
                        }
                        sm100::tc_fence_after();
                        const uint32_t a_addr = sm100::smem_u32(smem + stage * STAGE_BYTES);
                        const uint32_t b_addr = a_addr + A_BYTES;
                        // four MMAs of 32 bytes of K each (16 bf16 / 32 e4m3)
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            if (FP8)
                                sm100::mma_f8f6f4(d, sm100::make_sw128_desc(a_addr + k * 32),
                                                  sm100::make_sw128_desc(b_addr + k * 32), idesc,
                                                  (kc > 0 || k > 0) ? 1u : 0u);
                            else
                                sm100::mma_bf16(d, sm100::make_sw128_desc(a_addr + k * 32),
                                                sm100::make_sw128_desc(b_addr + k * 32), idesc,
                                                (kc > 0 || k > 0) ? 1u : 0u);
                        }
                        sm100::mma_commit(&empty[stage]);
                        if (++stage == STAGES) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                    if (!ok) break;
                    sm100::mma_commit(&tfull[acc]);
                    acc ^= 1;
                    if (acc == 0) aphase ^= 1;
                }
            }
            // all issued MMAs complete before TMEM is released
            sm100::mma_commit(&mma_done);
            sm100::mbar_wait(&mma_done, 0, p.err, 6);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        // two warps per TMEM lane group, each taking half of the columns of
        // every accumulator and keeping its own top-k (merged by the
        // rescoring kernel), so that two warps per SM sub-partition hide
        // each other's tcgen05.ld and shuffle latencies
        const int lg = warp % 4;           // TMEM lane group of this warp
        const int half = (warp - 2) / 4;   // columns [half * BN / 2, (half + 1) * BN / 2)
        const int row = lg * 32 + lane;    // voxel row within the tile
        int acc = 0;
        uint32_t aphase = 0;
        bool ok = true;
        for (long long item = blockIdx.x; item < total && ok; item += gridDim.x) {
            const float *asc = nullptr;
            if (FP8) asc = p.ascale2 + (long long)find_bin(p.tile_start, p.nbins, item / IPT) * p.bin_natoms;
            float ts[TOPK];
            int ti[TOPK];
#pragma unroll
            for (int k = 0; k < TOPK; k++) {
                ts[k] = 0.f;
                ti[k] = -1;
            }
            for (int at = 0; at < natiles; at++) {
                // every lane polls, then the warp reconverges and agrees
                // before the warp-collective tcgen05.ld
                const bool got = sm100::mbar_wait(&tfull[acc], aphase, p.err, 4);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                sm100::tc_fence_after();
                const uint32_t taddr = tmem + (uint32_t)(acc * BN) + ((uint32_t)(lg * 32) << 16);
                const int abase = (int)((long long)at * p.tile_stride % natiles) * APT;
                const bool full_tile = (long long)abase + APT <= p.bin_natoms;
#pragma unroll 1
                for (int c = half * (BN / 64); c < (half + 1) * (BN / 64); c++) {
                    float v[32];
                    sm100::tmem_ld32(taddr + c * 32, v);
                    if (IMAG) {
                        // Bound first: each lane holds one component (x_r or
                        // x_i sum) of all 32 atoms of the load, so every
                        // score of the pair is at most max|own|^2 +
                        // max|partner's|^2 (inflated by 2^-20 to cover
                        // rounding).  When no pair of the warp can beat its
                        // k-th best, the load needs no shuffles.  A voxel's
                        // two sums share one phase over all atoms, so the
                        // bound sits close to the best score of the load.
                        float am = 0.f;
#pragma unroll
                        for (int j = 0; j < 32; j++) am = fmaxf(am, fabsf(v[j]));
                        const float own = am * am;
                        const float bound = (own + __shfl_xor_sync(0xffffffffu, own, 1)) * (1.f + 0x1p-20f);
                        const float thr = fmaxf(ts[TOPK - 1], __shfl_xor_sync(0xffffffffu, ts[TOPK - 1], 1));
                        if (!__any_sync(0xffffffffu, bound > thr)) continue;
                    }
                    // the 16 scores of this load, then one test of their
                    // maximum against the current k-th best before any insertion
                    float sc[16];
                    int a0;
                    if (IMAG) {
                        // lane pair (2m, 2m+1) = voxel m's (x_r, x_i) rows: the
                        // even lane scores columns 0-15, the odd lane 16-31
                        const int part = lane & 1;
                        a0 = abase + c * 32 + (part ? 16 : 0);
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const float mine = part ? v[16 + j] : v[j];
                            const float other = __shfl_xor_sync(0xffffffffu, part ? v[j] : v[16 + j], 1);
                            sc[j] = fmaf(mine, mine, other * other);
                        }
                    } else {
                        a0 = abase + c * 16;
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            sc[j] = fmaf(v[2 * j], v[2 * j], v[2 * j + 1] * v[2 * j + 1]);
                            if (FP8) sc[j] *= (full_tile || a0 + j < p.bin_natoms) ? __ldg(asc + a0 + j) : 0.f;
                        }
                    }
                    float mx = sc[0];
#pragma unroll
                    for (int j = 1; j < 16; j++) mx = fmaxf(mx, sc[j]);
                    // IMAG: the lane pair keeps two lists of one voxel; each
                    // list's k-th best bounds the voxel's k-th best from
                    // below, so a score must beat the larger of the two
                    float thr = ts[TOPK - 1];
                    if (IMAG) thr = fmaxf(thr, __shfl_xor_sync(0xffffffffu, thr, 1));
                    if (mx > thr) {
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            if (sc[j] > fmaxf(thr, ts[TOPK - 1]) && (full_tile || a0 + j < p.bin_natoms))
                                topk_insert<TOPK>(ts, ti, sc[j], a0 + j);
                    }
                }
                sm100::tc_fence_before();
                sm100::mbar_arrive(&tempty[acc]);
                acc ^= 1;
                if (acc == 0) aphase ^= 1;
            }
            if (IMAG) {
                // the odd lane's list into the even lane's: the top-k of the union
                float os[TOPK];
                int oi[TOPK];
#pragma unroll
                for (int k = 0; k < TOPK; k++) {
                    os[k] = __shfl_xor_sync(0xffffffffu, ts[k], 1);
                    oi[k] = __shfl_xor_sync(0xffffffffu, ti[k], 1);
                }
                if (!(lane & 1)) {
#pragma unroll
                    for (int k = 0; k < TOPK; k++)
                        if (oi[k] >= 0 && os[k] > ts[TOPK - 1]) topk_insert<TOPK>(ts, ti, os[k], oi[k]);
                }
            }
            if (!IMAG || !(lane & 1)) {
                const long long slot = IMAG ? item * (BM / 2) + row / 2 : item * BM + row;
                const long long o = (slot * NLISTS + half) * TOPK_MAX;
#pragma unroll
                for (int k = 0; k < TOPK_MAX; k++) {
                    p.top_s[o + k] = k < TOPK ? ts[k] : 0.f;
                    p.top_i[o + k] = k < TOPK ? ti[k] : -1;
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (warp == 1) {
        sm100::tc_fence_after();
        sm100::tmem_dealloc(tmem, TMEM_COLS);
    }
}

// Padded bin layout: every B1 block's voxel slots start on a multiple of BM.
__global__ void scan_padded_kernel(const int *counts, long long *tile_start, long long *cursor, int nbins) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long t = 0;
    for (int b = 0; b < nbins; b++) {
        tile_start[b] = t;
        cursor[b] = t * BM;
        t += (counts[b] + BM - 1) / BM;
    }
    tile_start[nbins] = t;
}

__global__ void global_bin_kernel(long long *tile_start, long long *perm, long long nvox, long long cap) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s == 0) {
        tile_start[0] = 0;
        tile_start[1] = (nvox + BM - 1) / BM;
    }
    if (s < cap) perm[s] = s < nvox ? s : -1;
}

// 16-bit element pairs of the two operand formats.
template <bool HALF> struct Pair;
template <> struct Pair<false> {
    using T = __nv_bfloat162;
    static __device__ __forceinline__ T make(float a, float b) { return __floats2bfloat162_rn(a, b); }
};
template <> struct Pair<true> {
    using T = __half2;
    static __device__ __forceinline__ T make(float a, float b) { return __floats2half2_rn(a, b); }
};

// A rows: voxel perm[slot] scaled to unit norm (the argmax over atoms does
// not depend on the voxel's scale; it keeps FP16 in range), interleaved
// (Re, Im), zero padded to Kp.  One warp per slot.
template <bool HALF>
__global__ void pack_voxels_kernel(void *A, const float2 *img, long long img_stride, const long long *perm,
                                   long long nslots, long long nreps, long long Kp) {
    using P = Pair<HALF>;
    const long long slot = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (slot >= nslots) return;
    const long long v = perm[slot];
    const float2 *x = img + (v >= 0 ? v : 0) * img_stride;
    float n = 0.f;
    if (v >= 0)
        for (long long t = lane; t < nreps; t += 32) n += x[t].x * x[t].x + x[t].y * x[t].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    const float inv = n > 0.f ? rsqrtf(n) : 0.f;
    typename P::T *row = reinterpret_cast<typename P::T *>(A) + slot * (Kp / 2);
    for (long long t = lane; t < Kp / 2; t += 32) {
        float2 xv = make_float2(0.f, 0.f);
        if (v >= 0 && t < nreps) xv = x[t];
        row[t] = P::make(xv.x * inv, xv.y * inv);
    }
}

// B rows: atom a -> row 2a (Re d, Im d) and row 2a+1 (-Im d, Re d).  One
// warp per atom, four samples per lane and step (16-byte stores).
template <bool HALF>
__global__ void pack_atoms_kernel(void *B, const float2 *atoms, long long atom_stride, long long natoms,
                                  long long nreps, long long Kp) {
    using P = Pair<HALF>;
    const long long a = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (a >= natoms) return;
    typename P::T *r0 = reinterpret_cast<typename P::T *>(B) + (2 * a) * (Kp / 2);
    typename P::T *r1 = r0 + Kp / 2;
    const float2 *src = atoms + a * atom_stride;
    for (long long t = 4 * lane; t < Kp / 2; t += 128) {
        uint32_t o0[4], o1[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            float2 d = make_float2(0.f, 0.f);
            if (t + u < nreps) d = src[t + u];
            typename P::T x0 = P::make(d.x, d.y), x1 = P::make(-d.y, d.x);
            o0[u] = *reinterpret_cast<const uint32_t *>(&x0);
            o1[u] = *reinterpret_cast<const uint32_t *>(&x1);
        }
        *reinterpret_cast<uint4 *>(r0 + t) = make_uint4(o0[0], o0[1], o0[2], o0[3]);
        *reinterpret_cast<uint4 *>(r1 + t) = make_uint4(o1[0], o1[1], o1[2], o1[3]);
    }
}

// A rows for purely imaginary atoms: voxel perm[slot] at unit norm as two
// rows, 2 slot = (Re x_t) and 2 slot + 1 = (Im x_t), zero padded to Kp.
// One warp per slot.
template <bool HALF>
__global__ void pack_voxels_split_kernel(void *A, const float2 *img, long long img_stride, const long long *perm,
                                         long long nslots, long long nreps, long long Kp) {
    using P = Pair<HALF>;
    const long long slot = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (slot >= nslots) return;
    const long long v = perm[slot];
    const float2 *x = img + (v >= 0 ? v : 0) * img_stride;
    // two samples per 16-byte load where every row starts 16-byte aligned
    const bool vec = img_stride % 2 == 0 && reinterpret_cast<uintptr_t>(img) % 16 == 0;
    const float4 *x4 = reinterpret_cast<const float4 *>(x);
    float n = 0.f;
    if (v >= 0) {
        if (vec) {
            for (long long t = lane; t < nreps / 2; t += 32) {
                const float4 q = x4[t];
                n += q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
            }
            if ((nreps & 1) && lane == 0) n += x[nreps - 1].x * x[nreps - 1].x + x[nreps - 1].y * x[nreps - 1].y;
        } else {
            for (long long t = lane; t < nreps; t += 32) n += x[t].x * x[t].x + x[t].y * x[t].y;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    const float inv = n > 0.f ? rsqrtf(n) : 0.f;
    typename P::T *rr = reinterpret_cast<typename P::T *>(A) + (2 * slot) * (Kp / 2);
    typename P::T *ri = rr + Kp / 2;
    // four samples per lane and step: two pairs of each row in one 8-byte store
    for (long long g = lane; g < Kp / 4; g += 32) {
        const long long t = 4 * g;
        float2 s[4];
        if (vec && v >= 0 && t + 4 <= nreps) {
            const float4 q0 = x4[2 * g], q1 = x4[2 * g + 1];
            s[0] = make_float2(q0.x, q0.y);
            s[1] = make_float2(q0.z, q0.w);
            s[2] = make_float2(q1.x, q1.y);
            s[3] = make_float2(q1.z, q1.w);
        } else {
#pragma unroll
            for (int u = 0; u < 4; u++) s[u] = v >= 0 && t + u < nreps ? x[t + u] : make_float2(0.f, 0.f);
        }
        const typename P::T r0 = P::make(s[0].x * inv, s[1].x * inv), r1 = P::make(s[2].x * inv, s[3].x * inv);
        const typename P::T i0 = P::make(s[0].y * inv, s[1].y * inv), i1 = P::make(s[2].y * inv, s[3].y * inv);
        reinterpret_cast<uint2 *>(rr)[g] =
            make_uint2(*reinterpret_cast<const uint32_t *>(&r0), *reinterpret_cast<const uint32_t *>(&r1));
        reinterpret_cast<uint2 *>(ri)[g] =
            make_uint2(*reinterpret_cast<const uint32_t *>(&i0), *reinterpret_cast<const uint32_t *>(&i1));
    }
}

// B rows for purely imaginary atoms: row a = (Im d_t), zero padded to Kp;
// an atom with a non-zero real part sets the error word (code 7), which
// turns the call's maps to NaN.  One warp per atom, eight samples (16
// bytes) per lane and step.
template <bool HALF>
__global__ void pack_atoms_imag_kernel(void *B, const float2 *atoms, long long atom_stride, long long natoms,
                                       long long nreps, long long Kp, int *err) {
    using P = Pair<HALF>;
    const long long a = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (a >= natoms) return;
    typename P::T *row = reinterpret_cast<typename P::T *>(B) + a * (Kp / 2);
    const float2 *src = atoms + a * atom_stride;
    bool real_part = false;
    for (long long t = 8 * lane; t < Kp; t += 256) {
        uint32_t o[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            float2 d0 = make_float2(0.f, 0.f), d1 = make_float2(0.f, 0.f);
            if (t + 2 * u < nreps) d0 = src[t + 2 * u];
            if (t + 2 * u + 1 < nreps) d1 = src[t + 2 * u + 1];
            real_part |= d0.x != 0.f || d1.x != 0.f;
            typename P::T q = P::make(d0.y, d1.y);
            o[u] = *reinterpret_cast<const uint32_t *>(&q);
        }
        *reinterpret_cast<uint4 *>(row + t / 2) = make_uint4(o[0], o[1], o[2], o[3]);
    }
    if (__any_sync(0xffffffffu, real_part) && lane == 0) atomicCAS(err, 0, 7);
}

// Compressed operands (rank-r coordinates), each value split into 16-bit
// parts hi = rn(v), lo = rn(v - hi): an A row holds [hi(a), lo(a), hi(a)]
// and a B row [hi(b), hi(b), lo(b)], so the MMA sums hi(a) hi(b) +
// lo(a) hi(b) + hi(a) lo(b) = a b - lo(a) lo(b): the product to ~2^-22
// (FP16) or ~2^-16 (BF16) relative, at K = 3L (L = r, or 2r interleaved),
// which for r <= 21 still fits the one 64-wide K chunk.  Few coordinates
// carry most of a score, so unlike K = nreps the rounding of single
// products does not average out.
template <bool HALF> struct Half16;
template <> struct Half16<false> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ T make(float a) { return __float2bfloat16_rn(a); }
    static __device__ __forceinline__ float back(T a) { return __bfloat162float(a); }
};
template <> struct Half16<true> {
    using T = __half;
    static __device__ __forceinline__ T make(float a) { return __float2half_rn(a); }
    static __device__ __forceinline__ float back(T a) { return __half2float(a); }
};

template <bool HALF>
__device__ __forceinline__ typename Half16<HALF>::T split_part(float v, int seg, bool atom) {
    using H = Half16<HALF>;
    const typename H::T hi = H::make(v);
    const bool lo = atom ? seg == 2 : seg == 1;
    return lo ? H::make(v - H::back(hi)) : hi;
}

// A rows of compressed voxels (r coordinates, unit norm): IMAG gives two
// rows (Re, Im) per slot, otherwise one interleaved row.  One warp per slot.
template <bool HALF, bool IMAG>
__global__ void pack_voxels_comp_kernel(void *A, const float2 *img, long long img_stride, const long long *perm,
                                        long long nslots, long long r, long long Kp) {
    using H = Half16<HALF>;
    const long long slot = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (slot >= nslots) return;
    const long long v = perm[slot];
    const float2 *x = img + (v >= 0 ? v : 0) * img_stride;
    float n = 0.f;
    if (v >= 0)
        for (long long i = lane; i < r; i += 32) n += x[i].x * x[i].x + x[i].y * x[i].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    const float inv = n > 0.f ? rsqrtf(n) : 0.f;
    const long long L = IMAG ? r : 2 * r;
    typename H::T *row = reinterpret_cast<typename H::T *>(A) + (IMAG ? 2 * slot : slot) * Kp;
    for (long long e = lane; e < Kp; e += 32) {
        const int seg = (int)(e / L);
        const long long i = e % L;
        float a0 = 0.f, a1 = 0.f;
        if (v >= 0 && seg < 3) {
            if (IMAG) {
                a0 = x[i].x * inv;
                a1 = x[i].y * inv;
            } else {
                a0 = ((i & 1) ? x[i / 2].y : x[i / 2].x) * inv;
            }
        }
        row[e] = seg < 3 ? split_part<HALF>(a0, seg, false) : H::make(0.f);
        if (IMAG) row[Kp + e] = seg < 3 ? split_part<HALF>(a1, seg, false) : H::make(0.f);
    }
}

// B rows of compressed atoms: IMAG one row (Im c; a non-zero Re c sets the
// error word to 7), otherwise two rows (Re c, Im c) and (-Im c, Re c)
// interleaved.  One warp per atom.
template <bool HALF, bool IMAG>
__global__ void pack_atoms_comp_kernel(void *B, const float2 *coeffs, long long stride, long long natoms, long long r,
                                       long long Kp, int *err) {
    using H = Half16<HALF>;
    const long long a = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (a >= natoms) return;
    const float2 *c = coeffs + a * stride;
    const long long L = IMAG ? r : 2 * r;
    typename H::T *row = reinterpret_cast<typename H::T *>(B) + (IMAG ? a : 2 * a) * Kp;
    bool real_part = false;
    for (long long e = lane; e < Kp; e += 32) {
        const int seg = (int)(e / L);
        const long long i = e % L;
        float b0 = 0.f, b1 = 0.f;
        if (seg < 3) {
            if (IMAG) {
                const float2 cv = c[i];
                real_part |= cv.x != 0.f;
                b0 = cv.y;
            } else {
                const float2 cv = c[i / 2];
                b0 = (i & 1) ? cv.y : cv.x;
                b1 = (i & 1) ? cv.x : -cv.y;
            }
        }
        row[e] = seg < 3 ? split_part<HALF>(b0, seg, true) : H::make(0.f);
        if (!IMAG) row[Kp + e] = seg < 3 ? split_part<HALF>(b1, seg, true) : H::make(0.f);
    }
    if (IMAG && __any_sync(0xffffffffu, real_part) && lane == 0) atomicCAS(err, 0, 7);
}

// E4M3 A rows: voxel perm[slot] scaled so that its largest component is
// E4M3_MAX (the argmax over atoms does not depend on the voxel's scale),
// interleaved (Re, Im), zero padded to Kp bytes.  One warp per slot.
__global__ void pack_voxels_e4m3_kernel(unsigned char *A, const float2 *img, long long img_stride,
                                        const long long *perm, long long nslots, long long nreps, long long Kp) {
    const long long slot = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (slot >= nslots) return;
    const long long v = perm[slot];
    const float2 *x = img + (v >= 0 ? v : 0) * img_stride;
    float mx = 0.f;
    if (v >= 0)
        for (long long t = lane; t < nreps; t += 32) mx = fmaxf(mx, fmaxf(fabsf(x[t].x), fabsf(x[t].y)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sc = mx > 0.f ? E4M3_MAX / mx : 0.f;
    __nv_fp8x2_storage_t *row = reinterpret_cast<__nv_fp8x2_storage_t *>(A + slot * Kp);
    for (long long t = lane; t < Kp / 2; t += 32) {
        float2 xv = make_float2(0.f, 0.f);
        if (v >= 0 && t < nreps) xv = x[t];
        row[t] = __nv_cvt_float2_to_fp8x2(make_float2(xv.x * sc, xv.y * sc), __NV_SATFINITE, __NV_E4M3);
    }
}

// E4M3 B rows: atom a scaled by s_a = E4M3_MAX / (largest component) into
// row 2a (Re d, Im d) and row 2a+1 (-Im d, Re d); ascale2[a] = 1 / s_a^2
// undoes the scale on |s|^2.  One warp per atom, eight samples (16 bytes)
// per lane and step.
__global__ void pack_atoms_e4m3_kernel(unsigned char *B, float *ascale2, const float2 *atoms,
                                       long long atom_stride, long long natoms, long long nreps, long long Kp) {
    const long long a = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (a >= natoms) return;
    const float2 *src = atoms + a * atom_stride;
    float mx = 0.f;
    for (long long t = lane; t < nreps; t += 32) mx = fmaxf(mx, fmaxf(fabsf(src[t].x), fabsf(src[t].y)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sc = mx > 0.f ? E4M3_MAX / mx : 0.f;
    if (lane == 0) ascale2[a] = mx > 0.f ? 1.f / (sc * sc) : 0.f;
    unsigned char *r0 = B + (2 * a) * Kp;
    unsigned char *r1 = r0 + Kp;
    for (long long t = 8 * lane; t < Kp / 2; t += 256) {
        uint32_t o0[4], o1[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            float2 d0 = make_float2(0.f, 0.f), d1 = make_float2(0.f, 0.f);
            if (t + 2 * u < nreps) d0 = src[t + 2 * u];
            if (t + 2 * u + 1 < nreps) d1 = src[t + 2 * u + 1];
            const uint32_t p0 = __nv_cvt_float2_to_fp8x2(make_float2(d0.x * sc, d0.y * sc), __NV_SATFINITE, __NV_E4M3);
            const uint32_t p1 = __nv_cvt_float2_to_fp8x2(make_float2(d1.x * sc, d1.y * sc), __NV_SATFINITE, __NV_E4M3);
            const uint32_t q0 = __nv_cvt_float2_to_fp8x2(make_float2(-d0.y * sc, d0.x * sc), __NV_SATFINITE, __NV_E4M3);
            const uint32_t q1 = __nv_cvt_float2_to_fp8x2(make_float2(-d1.y * sc, d1.x * sc), __NV_SATFINITE, __NV_E4M3);
            o0[u] = p0 | (p1 << 16);
            o1[u] = q0 | (q1 << 16);
        }
        *reinterpret_cast<uint4 *>(r0 + 2 * t) = make_uint4(o0[0], o0[1], o0[2], o0[3]);
        *reinterpret_cast<uint4 *>(r1 + 2 * t) = make_uint4(o1[0], o1[1], o1[2], o1[3]);
    }
}

// Exact FP32 rescoring of the top-k per voxel; one warp per slot.  The
// scoring kernel leaves NLISTS lists of TOPK (by approximate score) per
// voxel, one per half of the atom tiles; their TOPK best (ties to the lower
// atom index) are rescored.  The map gets the candidate with the largest |s| (lowest
// atom index on ties, nothing unless |s| > 0, like generate_maps' strict '>'
// from 0).  VEC: two samples per 16-byte load (strides even, rows aligned).
// ROWS: the atoms are Im rows of purely imaginary atoms, [NATOMS][atom_stride]
// float (SNAPMRF_DICT_IMAG_ROWS); VEC then reads four samples per 16 bytes.
template <int TOPK, bool VEC, bool ROWS = false>
__global__ void rescore_kernel(float *maps, long long *index_out, const float *top_s, const int *top_i,
                               const long long *perm, const long long *tile_start, int nbins, const int *vox_bin,
                               const float2 *atoms, long long atom_stride, const float2 *img, long long img_stride,
                               long long nreps, const float *params, int nparams, long long bin_natoms,
                               const int *err, const float *atom_norms) {
    const long long slot = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (slot >= tile_start[nbins] * BM) return;
    const long long v = perm[slot];
    if (v < 0) return;
    const long long bin = vox_bin ? vox_bin[v] : 0;
    static_assert(NLISTS * TOPK <= 32, "one lane per listed candidate");
    const bool listed = lane < NLISTS * TOPK;
    const long long o = (slot * NLISTS + lane / TOPK) * TOPK_MAX + lane % TOPK;
    const int li = listed ? top_i[o] : -1;
    const float ls = listed && li >= 0 ? top_s[o] : -1.f;
    int rank = 0;
#pragma unroll
    for (int j = 0; j < NLISTS * TOPK; j++) {
        const float sj = __shfl_sync(0xffffffffu, ls, j);
        const int ij = __shfl_sync(0xffffffffu, li, j);
        rank += sj > ls || (sj == ls && (ij < li || (ij == li && j < lane)));
    }
    int cand = -1;
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
        const unsigned m = __ballot_sync(0xffffffffu, listed && rank == k);
        const int ik = __shfl_sync(0xffffffffu, li, m ? __ffs(m) - 1 : 0);
        if (lane == k) cand = m ? ik : -1;
    }
    int ci[TOPK];
    const float2 *row[TOPK];
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
        ci[k] = __shfl_sync(0xffffffffu, cand, k);
        row[k] = atoms + (bin * bin_natoms + (ci[k] >= 0 ? ci[k] : 0)) * atom_stride;
    }
    float re[TOPK], im[TOPK];
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
        re[k] = 0.f;
        im[k] = 0.f;
    }
    // Atoms as generated (atom_norms): 1 / ||d|| per candidate, formed as the
    // dictionary's normalisation forms it, loaded ahead of the inner products
    // so that the loads' latency is hidden.  Top-16: every lane loads and
    // forms all 16; top-4 / 8: lane k loads candidate k's norm and forms its
    // inverse after the inner products (each the faster on C1).
    float inv[TOPK];
    if constexpr (TOPK == 16) {
#pragma unroll
        for (int k = 0; k < TOPK; k++) {
            inv[k] = 1.f;
            if (atom_norms && ci[k] >= 0) {
                const float n = atom_norms[bin * bin_natoms + ci[k]];
                inv[k] = n > 0.f ? 1.f / n : 0.f;
            }
        }
    }
    const bool scaled = TOPK != 16 && atom_norms && lane < TOPK && cand >= 0;
    const float my_norm = scaled ? atom_norms[bin * bin_natoms + cand] : 1.f;
    const float2 *x = img + v * img_stride;
    if (ROWS) {
        // s = i d: conj(s) x = (d xi, -d xr)
        const float *rowf[TOPK];
#pragma unroll
        for (int k = 0; k < TOPK; k++)
            rowf[k] = reinterpret_cast<const float *>(atoms) + (bin * bin_natoms + (ci[k] >= 0 ? ci[k] : 0)) * atom_stride;
        if (VEC) {
            const long long n4 = nreps / 4;
            for (long long t = lane; t < n4; t += 32) {
                const float4 x0 = reinterpret_cast<const float4 *>(x)[2 * t];
                const float4 x1 = reinterpret_cast<const float4 *>(x)[2 * t + 1];
#pragma unroll
                for (int k = 0; k < TOPK; k++) {
                    if (ci[k] < 0) continue;
                    const float4 d = reinterpret_cast<const float4 *>(rowf[k])[t];
                    re[k] += d.x * x0.y + d.y * x0.w;
                    im[k] -= d.x * x0.x + d.y * x0.z;
                    re[k] += d.z * x1.y + d.w * x1.w;
                    im[k] -= d.z * x1.x + d.w * x1.z;
                }
            }
        } else {
            for (long long t = lane; t < nreps; t += 32) {
                const float2 xv = x[t];
#pragma unroll
                for (int k = 0; k < TOPK; k++) {
                    if (ci[k] < 0) continue;
                    const float d = rowf[k][t];
                    re[k] += d * xv.y;
                    im[k] -= d * xv.x;
                }
            }
        }
    } else if (VEC) {
        const long long n2 = nreps / 2;
        for (long long t = lane; t < n2; t += 32) {
            const float4 xv = reinterpret_cast<const float4 *>(x)[t];
#pragma unroll
            for (int k = 0; k < TOPK; k++) {
                if (ci[k] < 0) continue;
                const float4 d = reinterpret_cast<const float4 *>(row[k])[t];
                re[k] += d.x * xv.x + d.y * xv.y;
                im[k] += d.x * xv.y - d.y * xv.x;
                re[k] += d.z * xv.z + d.w * xv.w;
                im[k] += d.z * xv.w - d.w * xv.z;
            }
        }
    } else {
        for (long long t = lane; t < nreps; t += 32) {
            const float2 xv = x[t];
#pragma unroll
            for (int k = 0; k < TOPK; k++) {
                if (ci[k] < 0) continue;
                const float2 d = row[k][t];
                re[k] += d.x * xv.x + d.y * xv.y;
                im[k] += d.x * xv.y - d.y * xv.x;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            re[k] += __shfl_xor_sync(0xffffffffu, re[k], o);
            im[k] += __shfl_xor_sync(0xffffffffu, im[k], o);
        }
    }
    if constexpr (TOPK != 16) {
        const float my_inv = scaled ? (my_norm > 0.f ? 1.f / my_norm : 0.f) : 1.f;
#pragma unroll
        for (int k = 0; k < TOPK; k++) inv[k] = __shfl_sync(0xffffffffu, my_inv, k);
    }
    if (lane != 0) return;
    if (atom_norms) {
#pragma unroll
        for (int k = 0; k < TOPK; k++) {
            re[k] *= inv[k];
            im[k] *= inv[k];
        }
    }
    int best = -1;
    float bs = 0.f, bre = 0.f, bim = 0.f;
#pragma unroll
    for (int k = 0; k < TOPK; k++) {
        if (ci[k] < 0) continue;
        const float sc = re[k] * re[k] + im[k] * im[k];
        if (sc > bs || (sc == bs && best >= 0 && ci[k] < best)) {
            if (sc > 0.f) {
                bs = sc;
                best = ci[k];
                bre = re[k];
                bim = im[k];
            }
        }
    }
    const long long g = bin * bin_natoms + (best >= 0 ? best : 0);
    const float *pr = params + g * nparams;
    float *m = maps + v * 5;
    const bool bad = err && *err;
    const float nanv = __int_as_float(0x7fc00000);
    m[0] = bad ? nanv : pr[0];
    m[1] = bad ? nanv : pr[1];
    m[2] = bad ? nanv : pr[2];
    m[3] = bad ? nanv : pr[3];
    m[4] = bad ? nanv : (best >= 0 ? hypotf(bre, bim) : 0.f);
    if (index_out) index_out[v] = bad ? -1 : g;
}

__global__ void publish_error_kernel(const int *err) {
    if (*err) atomicCAS(&g_device_error, 0, *err);
}

// Self-test of the bounded wait: an mbarrier that expects one arrival,
// which nothing makes; thread 0 waits on it with a limit of limit_ns, the
// wait gives up, records code 10 and the kernel returns.  No copy or MMA is
// in flight, so giving up leaves nothing behind.
__global__ void bounded_wait_selftest_kernel(int *err, unsigned long long limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        sm100::mbar_init(&bar, 1);
        sm100::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) sm100::mbar_wait(&bar, 0, err, 10, limit_ns);
    __syncthreads();
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// fmt: 0 bf16, 1 fp16, 2 e4m3 (as bytes); the box is one 128-byte row of K.
int make_map(CUtensorMap *m, const void *base, long long rows, long long Kp, int box_rows, int fmt) {
    auto enc = encode_fn();
    if (!enc) SNAPMRF_FAIL(SNAPMRF_ERR_CUDA, "MRF_match: cuTensorMapEncodeTiled is not available");
    const int eb = fmt == 2 ? 1 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(Kp * eb)};
    cuuint32_t box[2] = {(cuuint32_t)(128 / eb), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType ty = fmt == 2   ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                   : fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                              : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUresult r = enc(m, ty, 2, const_cast<void *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) SNAPMRF_FAIL(SNAPMRF_ERR_CUDA, "MRF_match: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SNAPMRF_OK;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace tc

int match_bf16(const TcMatchRequest &q, cudaStream_t st) {
    using namespace tc;
    const long long nvox = q.nvox;
    const int nbins = q.b1map ? q.nblocks : 1;
    const long long bin_natoms = q.b1map ? q.natoms : q.NATOMS;
    const int fmt = q.fmt;
    const bool fp8 = fmt == 2;
    const bool imag = q.imag && !fp8;     // one real row per atom, K = T
    const int eb = fp8 ? 1 : 2;           // bytes per element
    const int bke = fp8 ? BK8 : BK;       // K elements per 128-byte row
    // compressed matching scores rank-r coordinates: projected voxels
    // [nvox][rs] (rs even, for the two-sample loads of the rescoring)
    const bool comp = q.basis != nullptr;
    const long long kn = comp ? q.rank : q.nreps;
    const long long rs = comp ? ((q.rank + 1) & ~1ll) : 0;
    // BF16 / FP16 compressed operands are split into hi + lo parts (K = 3L)
    const bool split = comp && !fp8;
    const long long Kp = (((imag ? 1 : 2) * kn * (split ? 3 : 1) + bke - 1) / bke) * bke;
    const long long cap = ((nvox + BM - 1) / BM + nbins) * BM;  // padded slots, upper bound
    const long long brows = (imag ? 1 : 2) * q.NATOMS;
    const long long arows = (imag ? 2 : 1) * cap;
    if (arows > 0x7fffffffll || brows > 0x7fffffffll || Kp > 0x7fffffffll)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_match: problem too large for the tensor-core path");

    size_t bytes = 0;
    auto take = [&](size_t n) {
        size_t off = bytes;
        bytes += (n + 255) & ~size_t(255);
        return off;
    };
    const bool prepacked = imag && q.packed;
    const size_t oA = take((size_t)arows * Kp * eb), oB = take(prepacked ? 0 : (size_t)brows * Kp * eb);
    const size_t oSc = take(fp8 ? (size_t)q.NATOMS * 4 : 0);
    const size_t oTs = take((size_t)cap * NLISTS * TOPK_MAX * 4), oTi = take((size_t)cap * NLISTS * TOPK_MAX * 4);
    const size_t oPerm = take((size_t)cap * 8), oTile = take((size_t)(nbins + 1) * 8);
    const size_t oCur = take((size_t)(nbins + 1) * 8), oVb = take((size_t)nvox * 4);
    const size_t oCnt = take((size_t)nbins * 4), oErr = take(4);
    const size_t oCimg = take(comp ? (size_t)nvox * rs * sizeof(float2) : 0);
    DeviceScratch s;
    SNAPMRF_CUDA(s.alloc(bytes, st));
    unsigned char *b = s.as<unsigned char>();
    void *A = b + oA;
    void *B = prepacked ? const_cast<void *>(q.packed) : static_cast<void *>(b + oB);
    float *ascale2 = reinterpret_cast<float *>(b + oSc);
    const bool half = fmt == 1;
    float *top_s = reinterpret_cast<float *>(b + oTs);
    int *top_i = reinterpret_cast<int *>(b + oTi);
    long long *perm = reinterpret_cast<long long *>(b + oPerm);
    long long *tile_start = reinterpret_cast<long long *>(b + oTile);
    long long *cursor = reinterpret_cast<long long *>(b + oCur);
    int *vox_bin = reinterpret_cast<int *>(b + oVb);
    int *counts = reinterpret_cast<int *>(b + oCnt);
    int *err = reinterpret_cast<int *>(b + oErr);
    float2 *cimg = reinterpret_cast<float2 *>(b + oCimg);
    SNAPMRF_CUDA(cudaMemsetAsync(err, 0, 4, st));
    // operands of the scores: the samples, or the rank-r coordinates
    const float2 *pimg = comp ? cimg : q.img;
    const long long pis = comp ? rs : q.img_stride;
    const float2 *patoms = comp ? q.coeffs : q.atoms;
    const long long pas = comp ? q.coeff_stride : q.atom_stride;

    if (q.b1map) {
        SNAPMRF_CUDA(cudaMemsetAsync(counts, 0, (size_t)nbins * 4, st));
        SNAPMRF_CUDA(cudaMemsetAsync(perm, 0xff, (size_t)cap * 8, st));
        assign_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(vox_bin, counts, q.b1map, q.params, q.nparams,
                                                            q.natoms, nbins, nvox);
        SNAPMRF_LAUNCH_CHECK();
        scan_padded_kernel<<<1, 32, 0, st>>>(counts, tile_start, cursor, nbins);
        SNAPMRF_LAUNCH_CHECK();
        scatter_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(perm, cursor, vox_bin, nvox);
        SNAPMRF_LAUNCH_CHECK();
    } else {
        global_bin_kernel<<<nblk(cap, 256), 256, 0, st>>>(tile_start, perm, nvox, cap);
        SNAPMRF_LAUNCH_CHECK();
    }
    if (comp) {
        int rc = project_voxels(cimg, rs, q.img, q.img_stride, nvox, q.nreps, q.b1map ? vox_bin : nullptr, nbins,
                                q.basis, q.basis_rows, q.basis_stride, q.rank, q.imag, st);
        if (rc) return rc;
    }
    if (split) {
        const unsigned gv = nblk(cap * 32, 256), ga = nblk(q.NATOMS * 32, 256);
        if (imag && half) {
            pack_voxels_comp_kernel<true, true><<<gv, 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
            SNAPMRF_LAUNCH_CHECK();
            pack_atoms_comp_kernel<true, true><<<ga, 256, 0, st>>>(B, patoms, pas, q.NATOMS, kn, Kp, err);
        } else if (imag) {
            pack_voxels_comp_kernel<false, true><<<gv, 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
            SNAPMRF_LAUNCH_CHECK();
            pack_atoms_comp_kernel<false, true><<<ga, 256, 0, st>>>(B, patoms, pas, q.NATOMS, kn, Kp, err);
        } else if (half) {
            pack_voxels_comp_kernel<true, false><<<gv, 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
            SNAPMRF_LAUNCH_CHECK();
            pack_atoms_comp_kernel<true, false><<<ga, 256, 0, st>>>(B, patoms, pas, q.NATOMS, kn, Kp, err);
        } else {
            pack_voxels_comp_kernel<false, false><<<gv, 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
            SNAPMRF_LAUNCH_CHECK();
            pack_atoms_comp_kernel<false, false><<<ga, 256, 0, st>>>(B, patoms, pas, q.NATOMS, kn, Kp, err);
        }
        SNAPMRF_LAUNCH_CHECK();
    } else if (fp8) {
        pack_voxels_e4m3_kernel<<<nblk(cap * 32, 256), 256, 0, st>>>(static_cast<unsigned char *>(A), pimg,
                                                                      pis, perm, cap, kn, Kp);
        SNAPMRF_LAUNCH_CHECK();
        // Kp is a multiple of 128 bytes, so every 16-byte group of a row is
        // whole and aligned
        pack_atoms_e4m3_kernel<<<nblk(q.NATOMS * 32, 256), 256, 0, st>>>(static_cast<unsigned char *>(B), ascale2,
                                                                          patoms, pas, q.NATOMS,
                                                                          kn, Kp);
        SNAPMRF_LAUNCH_CHECK();
    } else if (imag) {
        if (half)
            pack_voxels_split_kernel<true><<<nblk(cap * 32, 256), 256, 0, st>>>(A, pimg, pis, perm, cap,
                                                                                kn, Kp);
        else
            pack_voxels_split_kernel<false><<<nblk(cap * 32, 256), 256, 0, st>>>(A, pimg, pis, perm, cap,
                                                                                 kn, Kp);
        SNAPMRF_LAUNCH_CHECK();
        // Kp is a multiple of 64, so every 8-element group of a row is whole
        // and 16-byte aligned
        if (!prepacked) {
            if (half)
                pack_atoms_imag_kernel<true><<<nblk(q.NATOMS * 32, 256), 256, 0, st>>>(B, patoms, pas,
                                                                                       q.NATOMS, kn, Kp, err);
            else
                pack_atoms_imag_kernel<false><<<nblk(q.NATOMS * 32, 256), 256, 0, st>>>(B, patoms, pas,
                                                                                        q.NATOMS, kn, Kp, err);
            SNAPMRF_LAUNCH_CHECK();
        }
    } else {
        if (half)
            pack_voxels_kernel<true><<<nblk(cap * 32, 256), 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
        else
            pack_voxels_kernel<false><<<nblk(cap * 32, 256), 256, 0, st>>>(A, pimg, pis, perm, cap, kn, Kp);
        SNAPMRF_LAUNCH_CHECK();
        // Kp is a multiple of 64, so every 4-pair group of a row is whole and
        // 16-byte aligned (row pitch Kp * 2 bytes)
        if (half)
            pack_atoms_kernel<true><<<nblk(q.NATOMS * 32, 256), 256, 0, st>>>(B, patoms, pas, q.NATOMS,
                                                                                kn, Kp);
        else
            pack_atoms_kernel<false><<<nblk(q.NATOMS * 32, 256), 256, 0, st>>>(B, patoms, pas, q.NATOMS,
                                                                                 kn, Kp);
        SNAPMRF_LAUNCH_CHECK();
    }
    CUtensorMap mA, mB;
    int rc = make_map(&mA, A, arows, Kp, BM, fmt);
    if (rc) return rc;
    rc = make_map(&mB, B, brows, Kp, BN, fmt);
    if (rc) return rc;

    int num_sms = 0, dev = 0;
    SNAPMRF_CUDA(cudaGetDevice(&dev));
    SNAPMRF_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    auto pick = [&](auto k16, auto k8, auto k4) { return q.topk > 8 ? k16 : q.topk > 4 ? k8 : k4; };
    auto kern = fp8    ? pick(match_bf16_kernel<16, true, false>, match_bf16_kernel<8, true, false>,
                              match_bf16_kernel<4, true, false>)
                : imag ? pick(match_bf16_kernel<16, false, true>, match_bf16_kernel<8, false, true>,
                              match_bf16_kernel<4, false, true>)
                       : pick(match_bf16_kernel<16, false, false>, match_bf16_kernel<8, false, false>,
                              match_bf16_kernel<4, false, false>);
    SNAPMRF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    Args a;
    a.tile_start = tile_start;
    a.nbins = nbins;
    a.bin_natoms = bin_natoms;
    a.nk = (int)(Kp / bke);
    // Atom tiles in a golden-ratio stride order (coprime to their count):
    // the dictionary's (T1, T2) order makes consecutive tiles' scores rise
    // smoothly toward a voxel's best, so visiting tiles spread over the grid
    // first raises the k-th best early and saves top-k insertions.
    {
        const long long natiles = (bin_natoms + (imag ? BN : BA) - 1) / (imag ? BN : BA);
        long long st_ = std::max(1ll, (long long)std::llround(0.618034 * (double)natiles));
        while (std::gcd(st_, natiles) != 1) st_++;
        a.tile_stride = natiles > 1 ? (int)(st_ % natiles) : 1;
        if (a.tile_stride == 0) a.tile_stride = 1;
    }
    a.idesc = fp8 ? sm100::make_idesc_e4m3(BM, BN) : half ? sm100::make_idesc_f16(BM, BN) : sm100::make_idesc_bf16(BM, BN);
    a.ascale2 = fp8 ? ascale2 : nullptr;
    a.top_s = top_s;
    a.top_i = top_i;
    a.err = err;
    const long long max_items = (imag ? 2 : 1) * cap / BM;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(num_sms, max_items));
    kern<<<grid, THREADS, SMEM_BYTES, st>>>(mA, mB, a);
    SNAPMRF_LAUNCH_CHECK();
    // two samples per 16-byte load when every row starts 16-byte aligned
    // rescoring operands: the atoms and samples, or (compressed, no atoms)
    // the coordinates and projected voxels
    const bool rfull = !comp || q.atoms;
    const float2 *ratoms = rfull ? q.atoms : q.coeffs, *rimg = rfull ? q.img : cimg;
    const long long ras = rfull ? q.atom_stride : q.coeff_stride, ris = rfull ? q.img_stride : rs;
    const long long rn = rfull ? q.nreps : q.rank;
    const bool rows = rfull && q.imag_rows;
    const bool vec = rn % (rows ? 4 : 2) == 0 && ras % (rows ? 4 : 2) == 0 && ris % 2 == 0 &&
                     reinterpret_cast<uintptr_t>(ratoms) % 16 == 0 && reinterpret_cast<uintptr_t>(rimg) % 16 == 0;
    auto rk = rows ? (vec ? pick(rescore_kernel<16, true, true>, rescore_kernel<8, true, true>,
                                 rescore_kernel<4, true, true>)
                          : pick(rescore_kernel<16, false, true>, rescore_kernel<8, false, true>,
                                 rescore_kernel<4, false, true>))
                   : vec ? pick(rescore_kernel<16, true>, rescore_kernel<8, true>, rescore_kernel<4, true>)
                         : pick(rescore_kernel<16, false>, rescore_kernel<8, false>, rescore_kernel<4, false>);
    rk<<<nblk(cap * 32, 256), 256, 0, st>>>(q.maps, q.index_out, top_s, top_i, perm, tile_start, nbins,
                                            q.b1map ? vox_bin : nullptr, ratoms, ras, rimg, ris, rn, q.params,
                                            q.nparams, bin_natoms, err, rfull ? q.atom_norms : nullptr);
    SNAPMRF_LAUNCH_CHECK();
    publish_error_kernel<<<1, 1, 0, st>>>(err);
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}

}  // namespace snapmrf

namespace snapmrf {
cudaError_t noalloc_device_error(int *value, int reset);
}

extern "C" int snapmrf_selftest_bounded_wait(unsigned limit_us, void *stream) {
    using namespace snapmrf;
    cudaStream_t st = (cudaStream_t)stream;
    if (limit_us == 0 || limit_us > 2000000u)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "selftest_bounded_wait: limit must be in [1, 2000000] us (got %u)",
                     limit_us);
    DeviceScratch s;
    SNAPMRF_CUDA(s.alloc(sizeof(int), st));
    SNAPMRF_CUDA(cudaMemsetAsync(s.ptr, 0, sizeof(int), st));
    tc::bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(s.as<int>(), 1000ull * limit_us);
    SNAPMRF_LAUNCH_CHECK();
    tc::publish_error_kernel<<<1, 1, 0, st>>>(s.as<int>());
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}

extern "C" int snapmrf_device_error(int reset) {
    int v = 0, w = 0;
    SNAPMRF_CUDA(cudaMemcpyFromSymbol(&v, snapmrf::tc::g_device_error, sizeof(int)));
    if (reset) {
        int z = 0;
        SNAPMRF_CUDA(cudaMemcpyToSymbol(snapmrf::tc::g_device_error, &z, sizeof(int)));
    }
    SNAPMRF_CUDA(snapmrf::noalloc_device_error(&w, reset));
    return v ? v : w;
}
