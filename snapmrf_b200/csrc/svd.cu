// Low-rank (SVD) compression of MRF dictionaries per B1 block, and the
// projection of voxels onto a block's basis for compressed matching.
//
// Method: McGivney et al., IEEE TMI 2014, as matlab/MRF_dict_B1.m:127-159
// applies it: per B1 block the economy SVD of the unit-norm atoms
// (nreps x natoms), the rank from block 0's cumulative energy
// (nDictSpace = sum(cumsum(s.^2)./sum(s.^2) <= sfrac)), U_r = the r leading
// left singular vectors of each block and dict_compress = U_r' * D.
//
// MATLAB computes every block's full SVD.  Only the k = max_rank +
// oversample leading vectors are needed, so they are computed by subspace
// iteration with Rayleigh-Ritz (Halko, Martinsson and Tropp, SIAM Review
// 2011, algorithms 4.4 and 5.1), every block at once:
//
//   Q  = orth(G),  G a seeded Gaussian nreps x k                  FP64
//   power_iters times:
//     P = Q^H D                      project_kernel, a pass over the atoms
//     M = P P^H = W L W^H            gram_kernel + jacobi_kernel (FP64)
//     Z = D^H Q W L^-1/2             combine_kernel from P (orthonormal)
//     Y = D Z                        range_kernel, a pass over the atoms
//     Q = orth(Y)                    gram + jacobi + combine on Y (FP64)
//   P = Q^H D in FP64, M = P P^H = W L W^H: Ritz values L ~ s^2, vectors
//     U = Q W                        project64_kernel, a pass over the atoms
//   C = U_r^H D                      project_kernel, a pass over the atoms
//
// orth(A) is the eigen-decomposition form of the Gram-matrix orthonormalisation:
// A^H A = V S V^H (FP64 Jacobi), Q = A V S^-1/2, dropping directions with
// S below 1e-12 of the largest (numerically absent: rank-deficient blocks,
// nreps or natoms below k).  ||D_0||_F^2, the rank rule's denominator, is
// summed over block 0's atoms in FP64.  The passes of the iteration read
// FP32 and accumulate in FP32 per 32-element chunk, FP64 across chunks; the
// Rayleigh-Ritz projection, every Gram, eigenproblem and basis rotation is
// FP64, so the Ritz values the rank rule sums are exact for the computed
// subspace.  All reductions have a fixed order: the result is deterministic
// for a given seed.
//
// Compressed matching projects each voxel onto its bin's basis
// (project_voxels_kernel; the scores and rescoring are in match_tc.cu and
// match.cu).
//
// Purely imaginary atoms (SNAPMRF_SVD_IMAG_ATOMS) d = i v run the same
// iteration in real arithmetic on v (REAL = true); then U is real and
// C = U^H d = i U^T v.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "svd.h"

namespace snapmrf {
namespace svd {

constexpr int KMAX = SNAPMRF_SVD_MAX_SUBSPACE;  // subspace vectors
constexpr int PT = 32;                          // rows per tile = samples per chunk
constexpr int THREADS = 256;
constexpr int NW = THREADS / 32;
constexpr int CPT = (KMAX + NW - 1) / NW;       // subspace columns per thread
static_assert(KMAX % 2 == 0, "the Jacobi pairing needs an even bound");

// ---- scalar / complex helpers, REAL selects the real type -----------------
template <bool REAL> struct Ty;
template <> struct Ty<true> {
    using f = float;
    using d = double;
};
template <> struct Ty<false> {
    using f = float2;
    using d = double2;
};

__device__ __forceinline__ double to_d(float a) { return (double)a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double to_d(double a) { return a; }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double conj_(double a) { return a; }
__device__ __forceinline__ double2 conj_(double2 a) { return make_double2(a.x, -a.y); }
// acc + conj(a) * b
__device__ __forceinline__ double fma_cj(double acc, double a, double b) { return fma(a, b, acc); }
__device__ __forceinline__ double2 fma_cj(double2 acc, double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.x, b.y, fma(-a.y, b.x, acc.y)));
}
// acc + a * b
__device__ __forceinline__ double fma_(double acc, double a, double b) { return fma(a, b, acc); }
__device__ __forceinline__ double2 fma_(double2 acc, double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
template <class T> __device__ __forceinline__ T zero_();
template <> __device__ __forceinline__ float zero_<float>() { return 0.f; }
template <> __device__ __forceinline__ float2 zero_<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double zero_<double>() { return 0.0; }
template <> __device__ __forceinline__ double2 zero_<double2>() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double scale_(double a, double s) { return a * s; }
__device__ __forceinline__ double2 scale_(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float to_f(double a) { return (float)a; }
__device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
// the basis format (complex float, imaginary part 0 in real arithmetic)
__device__ __forceinline__ float2 to_f2(double a) { return make_float2((float)a, 0.f); }
__device__ __forceinline__ float2 to_f2(double2 a) { return make_float2((float)a.x, (float)a.y); }

__device__ __forceinline__ int find_bin(const long long *start, int nbins, long long item) {
    int lo = 0, hi = nbins - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (start[mid] <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---- projection of rows onto a basis --------------------------------------
struct ProjArgs {
    const float2 *x;            // rows [*][x_stride] complex
    long long x_stride;
    long long rows_per_block;   // contiguous mode: rows b * rpb + [0, rpb), grid.y = block
    const long long *perm;      // binned mode (voxel projection, non-null): slot -> row
    const long long *tile_start;  // [nbins + 1] first PT-slot tile of each bin
    const long long *slot_start;  // [nbins + 1] first slot of each bin
    int nbins;
    const float2 *basis;        // [bin][basis_rows][basis_stride] complex
    long long basis_rows, basis_stride;
    long long nreps;
    int k;                      // columns computed
    void *out;
    long long out_stride;
    int out_col;                // 1: out[(bin * k + c) * out_stride + local row]; 0: out[row * out_stride + c]
};

// out[row][c] = sum_t conj(basis[bin][c][t]) x[row][t], c < k.
// MODE 0: complex basis and rows; 1: real basis, complex rows; 2: real
// basis, purely imaginary rows d = i v: the value sum_t u_c[t] v[t] (real),
// written as a float (OUTF2 false) or as the complex (0, value).
// A CTA takes PT rows of one B1 block (rows b * rows_per_block + [0,
// rows_per_block), grid.y = b); lane = row, warp w the columns w + NW j.
template <int MODE, bool OUTF2>
__global__ void __launch_bounds__(THREADS) project_kernel(ProjArgs a) {
    __shared__ float sxr[PT][PT + 1], sxi[PT][PT + 1];
    __shared__ float sbr[KMAX][PT + 1], sbi[MODE == 0 ? KMAX : 1][PT + 1];
    __shared__ long long srow[PT], slocal[PT];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long bin = blockIdx.y;
    if (threadIdx.x < PT) {
        const long long l = (long long)blockIdx.x * PT + threadIdx.x;
        srow[threadIdx.x] = l < a.rows_per_block ? bin * a.rows_per_block + l : -1;
        slocal[threadIdx.x] = l;
    }
    __syncthreads();
    const float2 *B = a.basis + bin * a.basis_rows * a.basis_stride;
    // FP32 sums over a chunk of PT samples, FP64 across chunks
    float accr[CPT], acci[CPT];
    double sumr[CPT], sumi[CPT];
#pragma unroll
    for (int j = 0; j < CPT; j++) {
        accr[j] = acci[j] = 0.f;
        sumr[j] = sumi[j] = 0.0;
    }
    for (long long t0 = 0; t0 < a.nreps; t0 += PT) {
        const long long t = t0 + lane;
        const bool tin = t < a.nreps;
        for (int r = warp; r < PT; r += NW) {
            const long long row = srow[r];
            float2 v = make_float2(0.f, 0.f);
            if (row >= 0 && tin) v = a.x[row * a.x_stride + t];
            sxr[r][lane] = v.x;
            sxi[r][lane] = v.y;
        }
        for (int c = warp; c < a.k; c += NW) {
            float2 v = make_float2(0.f, 0.f);
            if (tin) v = B[c * a.basis_stride + t];
            sbr[c][lane] = v.x;
            if constexpr (MODE == 0) sbi[c][lane] = v.y;
        }
        __syncthreads();
#pragma unroll 4
        for (int tt = 0; tt < PT; tt++) {
            const float xr = sxr[lane][tt], xi = sxi[lane][tt];
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const int c = warp + NW * j;
                if (c < a.k) {
                    const float br = sbr[c][tt];
                    if constexpr (MODE == 0) {
                        const float bi = sbi[c][tt];
                        accr[j] = fmaf(br, xr, fmaf(bi, xi, accr[j]));
                        acci[j] = fmaf(br, xi, fmaf(-bi, xr, acci[j]));
                    } else if constexpr (MODE == 1) {
                        accr[j] = fmaf(br, xr, accr[j]);
                        acci[j] = fmaf(br, xi, acci[j]);
                    } else {
                        acci[j] = fmaf(br, xi, acci[j]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < CPT; j++) {
            sumr[j] += accr[j];
            sumi[j] += acci[j];
            accr[j] = acci[j] = 0.f;
        }
        __syncthreads();
    }
    const long long row = srow[lane];
    if (row < 0) return;
#pragma unroll
    for (int j = 0; j < CPT; j++) {
        const int c = warp + NW * j;
        if (c >= a.k) continue;
        const long long o = a.out_col ? (bin * a.k + c) * a.out_stride + slocal[lane] : row * a.out_stride + c;
        if (MODE == 2 && !OUTF2) {
            static_cast<float *>(a.out)[o] = (float)sumi[j];
        } else {
            static_cast<float2 *>(a.out)[o] = make_float2(MODE == 2 ? 0.f : (float)sumr[j], (float)sumi[j]);
        }
    }
}

// P64[b][c][j] = sum_t conj(Q64[b][c][t]) d_j[t] in FP64 from the FP64
// basis (REAL: sum_t Q64[b][c][t] Im d_j[t]): the Rayleigh-Ritz step, whose
// Gram gives the singular values the rank rule sums.  Same tiling as
// project_kernel (contiguous blocks); the basis chunk lives in dynamic
// shared memory (KMAX x (PT + 1) FP64, twice for complex).
template <bool REAL>
__global__ void __launch_bounds__(THREADS) project64_kernel(const float2 *x, long long x_stride, long long natoms,
                                                            const typename Ty<REAL>::d *q, long long nreps, int k,
                                                            typename Ty<REAL>::d *out) {
    using D = typename Ty<REAL>::d;
    __shared__ float sxr[PT][PT + 1], sxi[PT][PT + 1];
    extern __shared__ double psm[];
    double *sbr = psm, *sbi = psm + KMAX * (PT + 1);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long b = blockIdx.y;
    const long long l0 = (long long)blockIdx.x * PT;
    const D *Q = q + b * k * nreps;
    double accr[CPT], acci[CPT];
#pragma unroll
    for (int j = 0; j < CPT; j++) accr[j] = acci[j] = 0.0;
    for (long long t0 = 0; t0 < nreps; t0 += PT) {
        const long long t = t0 + lane;
        const bool tin = t < nreps;
        for (int r = warp; r < PT; r += NW) {
            float2 v = make_float2(0.f, 0.f);
            if (l0 + r < natoms && tin) v = x[(b * natoms + l0 + r) * x_stride + t];
            sxr[r][lane] = v.x;
            sxi[r][lane] = v.y;
        }
        for (int c = warp; c < k; c += NW) {
            D v = zero_<D>();
            if (tin) v = Q[c * nreps + t];
            if constexpr (REAL) {
                sbr[c * (PT + 1) + lane] = v;
            } else {
                sbr[c * (PT + 1) + lane] = v.x;
                sbi[c * (PT + 1) + lane] = v.y;
            }
        }
        __syncthreads();
#pragma unroll 2
        for (int tt = 0; tt < PT; tt++) {
            const double xr = sxr[lane][tt], xi = sxi[lane][tt];
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const int c = warp + NW * j;
                if (c < k) {
                    const double br = sbr[c * (PT + 1) + tt];
                    if constexpr (REAL) {
                        accr[j] = fma(br, xi, accr[j]);
                    } else {
                        const double bi = sbi[c * (PT + 1) + tt];
                        accr[j] = fma(br, xr, fma(bi, xi, accr[j]));
                        acci[j] = fma(br, xi, fma(-bi, xr, acci[j]));
                    }
                }
            }
        }
        __syncthreads();
    }
    const long long l = l0 + lane;
    if (l >= natoms) return;
#pragma unroll
    for (int j = 0; j < CPT; j++) {
        const int c = warp + NW * j;
        if (c >= k) continue;
        if constexpr (REAL) out[(b * k + c) * natoms + l] = accr[j];
        else out[(b * k + c) * natoms + l] = make_double2(accr[j], acci[j]);
    }
}

// Projection of voxels onto their bin's basis for the compressed matching,
// where the rank is small.  A CTA takes a tile of PT voxels of one bin and
// its VTS warps split the samples (chunks of PT, round-robin), so that even
// 25,600 voxels give enough warps to hide the image loads; a lane holds one
// voxel's VKC columns [c0, c0 + VKC) of one pass (columns >= k read zero
// basis values), two columns per packed two-wide FMA.  Each warp's basis
// chunk is kept as [column][sample] (conflict-free stores) and read as
// broadcast float4s of four samples.  The warps' partial sums are added in
// shared memory at the end.  RB: real basis (imaginary parts not read).
constexpr int VKC = 16;   // columns per pass
constexpr int VTS = 4;    // warps per tile (sample split)
constexpr int VLD = PT + 4;  // basis row pitch (16-byte aligned rows)
struct VoxSmem {
    float xr[VTS][PT][PT + 1], xi[VTS][PT][PT + 1];
    __align__(16) float br[VTS][VKC][VLD];
    __align__(16) float bi[VTS][VKC][VLD];
};
template <bool RB>
__global__ void __launch_bounds__(VTS * 32) project_voxels_kernel(ProjArgs a, int c0) {
    extern __shared__ __align__(16) unsigned char vsm_raw[];
    VoxSmem &sm = *reinterpret_cast<VoxSmem *>(vsm_raw);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long g = blockIdx.x;
    long long bin, row;
    if (a.perm) {
        if (g >= a.tile_start[a.nbins]) return;  // uniform per CTA
        const int b = find_bin(a.tile_start, a.nbins, g);
        bin = b;
        const long long sl = a.slot_start[b] + (g - a.tile_start[b]) * PT + lane;
        row = sl < a.slot_start[b + 1] ? a.perm[sl] : -1;
    } else {
        bin = 0;
        row = g * PT + lane < a.rows_per_block ? g * PT + lane : -1;
    }
    const float2 *B = a.basis + bin * a.basis_rows * a.basis_stride;
    float2 ar[VKC / 2], ai[VKC / 2];
#pragma unroll
    for (int j = 0; j < VKC / 2; j++) ar[j] = ai[j] = make_float2(0.f, 0.f);
    for (long long t0 = (long long)warp * PT; t0 < a.nreps; t0 += (long long)VTS * PT) {
        const long long t = t0 + lane;
        const bool tin = t < a.nreps;
        for (int r = 0; r < PT; r++) {
            const long long rr = __shfl_sync(0xffffffffu, row, r);
            float2 v = make_float2(0.f, 0.f);
            if (rr >= 0 && tin) v = a.x[rr * a.x_stride + t];
            sm.xr[warp][r][lane] = v.x;
            sm.xi[warp][r][lane] = v.y;
        }
#pragma unroll
        for (int c = 0; c < VKC; c++) {
            float2 v = make_float2(0.f, 0.f);
            if (c0 + c < a.k && tin) v = B[(long long)(c0 + c) * a.basis_stride + t];
            sm.br[warp][c][lane] = v.x;
            if constexpr (!RB) sm.bi[warp][c][lane] = v.y;
        }
        __syncwarp();
#pragma unroll 1
        for (int t4 = 0; t4 < PT; t4 += 4) {
            float xr[4], xi[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                xr[u] = sm.xr[warp][lane][t4 + u];
                xi[u] = sm.xi[warp][lane][t4 + u];
            }
#pragma unroll
            for (int q = 0; q < VKC / 2; q++) {
                const float4 b0 = *reinterpret_cast<const float4 *>(&sm.br[warp][2 * q][t4]);
                const float4 b1 = *reinterpret_cast<const float4 *>(&sm.br[warp][2 * q + 1][t4]);
                const float2 bb[4] = {make_float2(b0.x, b1.x), make_float2(b0.y, b1.y), make_float2(b0.z, b1.z),
                                      make_float2(b0.w, b1.w)};
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    ar[q] = __ffma2_rn(bb[u], make_float2(xr[u], xr[u]), ar[q]);
                    ai[q] = __ffma2_rn(bb[u], make_float2(xi[u], xi[u]), ai[q]);
                }
                if constexpr (!RB) {
                    // conj(b) x: Re += bi xi, Im -= bi xr
                    const float4 c0v = *reinterpret_cast<const float4 *>(&sm.bi[warp][2 * q][t4]);
                    const float4 c1v = *reinterpret_cast<const float4 *>(&sm.bi[warp][2 * q + 1][t4]);
                    const float2 cc[4] = {make_float2(c0v.x, c1v.x), make_float2(c0v.y, c1v.y),
                                          make_float2(c0v.z, c1v.z), make_float2(c0v.w, c1v.w)};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        ar[q] = __ffma2_rn(cc[u], make_float2(xi[u], xi[u]), ar[q]);
                        ai[q] = __ffma2_rn(cc[u], make_float2(-xr[u], -xr[u]), ai[q]);
                    }
                }
            }
        }
        __syncwarp();
    }
    // the warps' partial sums: [warp][voxel][column] in the x buffers
    __syncthreads();
    float2 *red = reinterpret_cast<float2 *>(&sm.xr[0][0][0]);  // VTS * PT * VKC float2 fit in xr + xi
#pragma unroll
    for (int j = 0; j < VKC / 2; j++) {
        red[(warp * PT + lane) * VKC + 2 * j] = make_float2(ar[j].x, ai[j].x);
        red[(warp * PT + lane) * VKC + 2 * j + 1] = make_float2(ar[j].y, ai[j].y);
    }
    __syncthreads();
    const long long vrow = __shfl_sync(0xffffffffu, row, lane);
    if (vrow < 0) return;
    // warp w adds columns [w * VKC / VTS, (w + 1) * VKC / VTS) over the warps
    float2 *out = static_cast<float2 *>(a.out) + vrow * a.out_stride;
#pragma unroll
    for (int cc = 0; cc < VKC / VTS; cc++) {
        const int c = warp * (VKC / VTS) + cc;
        if (c0 + c >= a.k) continue;
        float sr = 0.f, si = 0.f;
#pragma unroll
        for (int w = 0; w < VTS; w++) {
            const float2 v = red[(w * PT + lane) * VKC + c];
            sr += v.x;
            si += v.y;
        }
        out[c0 + c] = make_float2(sr, si);
    }
}
static_assert(sizeof(float) * 2 * VTS * PT * (PT + 1) >= sizeof(float2) * VTS * PT * VKC,
              "the partial sums fit in the sample buffers");

// ---- Y = D Z: partial sums over a split of each block's atoms ---------------
struct RangeArgs {
    const float2 *x;     // atoms [NATOMS][x_stride]
    long long x_stride, natoms, nreps;
    int k;
    const void *z;       // [nb][k][natoms]
    void *ypart;         // [nb][splits][k][nreps]
    int splits;
    long long per_split;
};

// REAL: y_i[t] = sum_j v_j[t] z_i[j] with v = Im d; complex: d_j[t] z_i[j].
// A CTA takes PT samples (lane) of one block and split; warp w the
// columns w + NW m.
template <bool REAL>
__global__ void __launch_bounds__(THREADS) range_kernel(RangeArgs a) {
    using F = typename Ty<REAL>::f;
    __shared__ float sdr[REAL ? 1 : PT][PT + 1], sdi[PT][PT + 1];
    __shared__ F sz[KMAX][PT + 1];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long b = blockIdx.z, s = blockIdx.y;
    const long long t = (long long)blockIdx.x * PT + lane;
    const bool tin = t < a.nreps;
    const long long j0 = s * a.per_split, j1 = min(a.natoms, j0 + a.per_split);
    const F *Z = static_cast<const F *>(a.z) + b * a.k * a.natoms;
    float accr[CPT], acci[CPT];
    double sumr[CPT], sumi[CPT];
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        accr[m] = acci[m] = 0.f;
        sumr[m] = sumi[m] = 0.0;
    }
    for (long long jb = j0; jb < j1; jb += PT) {
        for (int jj = warp; jj < PT; jj += NW) {
            const long long j = jb + jj;
            float2 v = make_float2(0.f, 0.f);
            if (j < j1 && tin) v = a.x[(b * a.natoms + j) * a.x_stride + t];
            if constexpr (!REAL) sdr[jj][lane] = v.x;
            sdi[jj][lane] = v.y;
        }
        for (int i = warp; i < a.k; i += NW) {
            const long long j = jb + lane;
            sz[i][lane] = j < j1 ? Z[i * a.natoms + j] : zero_<F>();
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < PT; jj++) {
            const float di = sdi[jj][lane];
            float dr = 0.f;
            if constexpr (!REAL) dr = sdr[jj][lane];
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                const int i = warp + NW * m;
                if (i < a.k) {
                    if constexpr (REAL) {
                        accr[m] = fmaf(di, sz[i][jj], accr[m]);
                    } else {
                        const float2 zv = sz[i][jj];
                        accr[m] = fmaf(dr, zv.x, fmaf(-di, zv.y, accr[m]));
                        acci[m] = fmaf(dr, zv.y, fmaf(di, zv.x, acci[m]));
                    }
                }
            }
        }
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            sumr[m] += accr[m];
            sumi[m] += acci[m];
            accr[m] = acci[m] = 0.f;
        }
        __syncthreads();
    }
    if (!tin) return;
    F *Y = static_cast<F *>(a.ypart) + ((b * a.splits + s) * a.k) * a.nreps;
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        const int i = warp + NW * m;
        if (i >= a.k) continue;
        if constexpr (REAL) Y[i * a.nreps + t] = (float)sumr[m];
        else Y[i * a.nreps + t] = make_float2((float)sumr[m], (float)sumi[m]);
    }
}

// y64[b][i][t] = sum_s ypart[b][s][i][t], in FP64 in split order.
template <bool REAL>
__global__ void reduce_range_kernel(typename Ty<REAL>::d *y64, const typename Ty<REAL>::f *ypart, long long nb,
                                    int splits, long long kT) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nb * kT) return;
    const long long b = e / kT, r = e % kT;
    typename Ty<REAL>::d acc = zero_<typename Ty<REAL>::d>();
    for (int s = 0; s < splits; s++) {
        const auto v = to_d(ypart[(b * splits + s) * kT + r]);
        if constexpr (REAL) acc += v;
        else acc = make_double2(acc.x + v.x, acc.y + v.y);
    }
    y64[e] = acc;
}

// ---- Gram matrices ---------------------------------------------------------
struct GramArgs {
    const void *A;       // [nb][k][L] (row a of block b: A + (b k + a) L)
    long long L;
    int k;
    void *gpart;         // [nb][splits][k][k] (upper triangle)
    int splits;
    long long per_split;
};
constexpr int PPT = (KMAX * (KMAX + 1) / 2 + THREADS - 1) / THREADS;  // pairs per thread

// gpart[b][s][a][c] = sum_{x in split s} conj(A[a][x]) A[c][x] for a <= c.
template <bool REAL, class TIN>
__global__ void __launch_bounds__(THREADS) gram_kernel(GramArgs g) {
    using D = typename Ty<REAL>::d;
    __shared__ D sa[KMAX][PT + 1];
    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    const long long b = blockIdx.y, s = blockIdx.x;
    const int k = g.k;
    const int npairs = k * (k + 1) / 2;
    int pa[PPT], pc[PPT];
#pragma unroll
    for (int m = 0; m < PPT; m++) {
        int p = tid + THREADS * m;
        int a = 0;
        if (p < npairs) {
            while (p >= k - a) {  // row a holds k - a pairs (c = a .. k-1)
                p -= k - a;
                a++;
            }
            pa[m] = a;
            pc[m] = a + p;
        } else {
            pa[m] = pc[m] = -1;
        }
    }
    D acc[PPT];
#pragma unroll
    for (int m = 0; m < PPT; m++) acc[m] = zero_<D>();
    const TIN *A = static_cast<const TIN *>(g.A) + b * k * g.L;
    const long long x0 = s * g.per_split, x1 = min(g.L, x0 + g.per_split);
    for (long long xb = x0; xb < x1; xb += PT) {
        for (int a = warp; a < k; a += NW) {
            const long long x = xb + lane;
            sa[a][lane] = x < x1 ? to_d(A[a * g.L + x]) : zero_<D>();
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < PPT; m++) {
            if (pa[m] < 0) continue;
            D v = acc[m];
            for (int xx = 0; xx < PT; xx++) v = fma_cj(v, sa[pa[m]][xx], sa[pc[m]][xx]);
            acc[m] = v;
        }
        __syncthreads();
    }
    D *out = static_cast<D *>(g.gpart) + (b * g.splits + s) * k * k;
#pragma unroll
    for (int m = 0; m < PPT; m++)
        if (pa[m] >= 0) out[pa[m] * k + pc[m]] = acc[m];
}

// G[b] = sum over splits (upper triangle), mirrored Hermitian; conjugated
// when conj_out (the atom-side Gram P P^H = conj(P^T)^H ... of rows of P).
template <bool REAL>
__global__ void reduce_gram_kernel(typename Ty<REAL>::d *G, const typename Ty<REAL>::d *gpart, long long nb, int splits,
                                   int k, int conj_out) {
    using D = typename Ty<REAL>::d;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long kk = (long long)k * k;
    if (e >= nb * kk) return;
    const long long b = e / kk;
    const int a = (int)((e % kk) / k), c = (int)(e % k);
    const int lo = min(a, c), hi = max(a, c);
    D acc = zero_<D>();
    for (int s = 0; s < splits; s++) {
        const D v = gpart[(b * splits + s) * kk + lo * k + hi];
        if constexpr (REAL) acc += v;
        else acc = make_double2(acc.x + v.x, acc.y + v.y);
    }
    if (a > c) acc = conj_(acc);
    if (conj_out) acc = conj_(acc);
    G[e] = acc;
}

// ---- Hermitian eigenproblems: cyclic Jacobi, one CTA per block --------------
// Two-sided Jacobi rotations J = diag(1, e^{-i phi}) R (R the real rotation
// that zeroes the phase-corrected |a_pq|, Numerical Recipes' angle
// convention), applied as A <- J^H A J and V <- V J, n/2 disjoint pairs per
// round in round-robin order.  A pair is skipped when |a_pq| <= n eps
// sqrt(|a_pp a_qq|) (the relative-accuracy criterion of Demmel and Veselic)
// or below 1e-18 of the trace; the iteration stops after a sweep that
// rotates nothing (at most 40 sweeps).  Output: eigenvalues descending
// (lam[b][i]) and eigenvectors as columns (W[b][a][i]).
template <bool REAL>
__global__ void __launch_bounds__(THREADS) jacobi_kernel(const typename Ty<REAL>::d *G, typename Ty<REAL>::d *W,
                                                         double *lam, int k) {
    using D = typename Ty<REAL>::d;
    extern __shared__ double jsm[];
    const int n = k + (k & 1), ld = n + 1, h = n / 2;
    double *Ar = jsm, *Vr = Ar + n * ld;
    double *Ai = REAL ? nullptr : Vr + n * ld;
    double *Vi = REAL ? nullptr : Ai + n * ld;
    __shared__ int sp[KMAX / 2], sq[KMAX / 2];
    __shared__ double sc[KMAX / 2], ss[KMAX / 2], ser[KMAX / 2], sei[KMAX / 2];
    __shared__ double red_off[1];
    __shared__ int done;
    const int tid = threadIdx.x;
    const D *g = G + (long long)blockIdx.x * k * k;
    for (int e = tid; e < n * n; e += THREADS) {
        const int r = e / n, c = e % n;
        const D v = (r < k && c < k) ? g[r * k + c] : zero_<D>();
        if constexpr (REAL) {
            Ar[r * ld + c] = v;
        } else {
            Ar[r * ld + c] = v.x;
            Ai[r * ld + c] = v.y;
            Vi[r * ld + c] = 0.0;
        }
        Vr[r * ld + c] = r == c ? 1.0 : 0.0;
    }
    __syncthreads();
    // scale for the absolute skip floor: the trace (>= the largest eigenvalue)
    if (tid == 0) {
        double tr = 0.0;
        for (int a = 0; a < n; a++) tr += fabs(Ar[a * ld + a]);
        red_off[0] = tr;
    }
    __syncthreads();
    const double floor_abs = 1e-18 * red_off[0];
    const double tol = 2.2e-16 * n;
    for (int sweep = 0; sweep < 40; sweep++) {
        if (tid == 0) done = 1;
        __syncthreads();
        for (int r = 0; r < n - 1; r++) {
            if (tid < h) {
                auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + r) % (n - 1); };
                int p = idx(tid), q = idx(n - 1 - tid);
                if (p > q) {
                    const int t = p;
                    p = q;
                    q = t;
                }
                const double app = Ar[p * ld + p], aqq = Ar[q * ld + q];
                const double apr = Ar[p * ld + q], api = REAL ? 0.0 : Ai[p * ld + q];
                const double mag = REAL ? fabs(apr) : hypot(apr, api);
                double c = 1.0, s = 0.0, er = 1.0, ei = 0.0;
                // rotate unless |a_pq| is negligible against the diagonal
                // (relative) or against the whole matrix (null directions)
                if (mag > floor_abs && mag > tol * sqrt(fabs(app * aqq))) {
                    const double theta = (aqq - app) / (2.0 * mag);
                    const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                    er = apr / mag;   // e^{-i phi} = conj(a_pq) / |a_pq|
                    ei = -api / mag;
                    done = 0;
                }
                sp[tid] = p;
                sq[tid] = q;
                sc[tid] = c;
                ss[tid] = s;
                ser[tid] = er;
                sei[tid] = ei;
            }
            __syncthreads();
            // columns: X <- X J for A and V (X_rp, X_rq) -> (c X_rp - s e X_rq, s X_rp + c e X_rq)
            for (int e = tid; e < n * h; e += THREADS) {
                const int row = e / h, i = e % h;
                if (ss[i] == 0.0) continue;
                const int p = sp[i], q = sq[i];
                const double c = sc[i], s = ss[i], er = ser[i], ei = sei[i];
                {
                    const double xpr = Ar[row * ld + p], xqr = Ar[row * ld + q];
                    if constexpr (REAL) {
                        const double eq = er * xqr;
                        Ar[row * ld + p] = c * xpr - s * eq;
                        Ar[row * ld + q] = s * xpr + c * eq;
                    } else {
                        const double xpi = Ai[row * ld + p], xqi = Ai[row * ld + q];
                        const double eqr = er * xqr - ei * xqi, eqi = er * xqi + ei * xqr;
                        Ar[row * ld + p] = c * xpr - s * eqr;
                        Ai[row * ld + p] = c * xpi - s * eqi;
                        Ar[row * ld + q] = s * xpr + c * eqr;
                        Ai[row * ld + q] = s * xpi + c * eqi;
                    }
                }
                {
                    const double xpr = Vr[row * ld + p], xqr = Vr[row * ld + q];
                    if constexpr (REAL) {
                        const double eq = er * xqr;
                        Vr[row * ld + p] = c * xpr - s * eq;
                        Vr[row * ld + q] = s * xpr + c * eq;
                    } else {
                        const double xpi = Vi[row * ld + p], xqi = Vi[row * ld + q];
                        const double eqr = er * xqr - ei * xqi, eqi = er * xqi + ei * xqr;
                        Vr[row * ld + p] = c * xpr - s * eqr;
                        Vi[row * ld + p] = c * xpi - s * eqi;
                        Vr[row * ld + q] = s * xpr + c * eqr;
                        Vi[row * ld + q] = s * xpi + c * eqi;
                    }
                }
            }
            __syncthreads();
            // rows: A <- J^H A, (A_pc, A_qc) -> (c A_pc - s conj(e) A_qc, s A_pc + c conj(e) A_qc);
            // the rotated pair's off-diagonal entries are set to 0 and its
            // diagonal made real
            for (int e = tid; e < h * n; e += THREADS) {
                const int i = e / n, col = e % n;
                if (ss[i] == 0.0) continue;
                const int p = sp[i], q = sq[i];
                const double c = sc[i], s = ss[i], er = ser[i], ei = -sei[i];
                const double xpr = Ar[p * ld + col], xqr = Ar[q * ld + col];
                double npr, nqr, npi = 0.0, nqi = 0.0;
                if constexpr (REAL) {
                    const double eq = er * xqr;
                    npr = c * xpr - s * eq;
                    nqr = s * xpr + c * eq;
                } else {
                    const double xpi = Ai[p * ld + col], xqi = Ai[q * ld + col];
                    const double eqr = er * xqr - ei * xqi, eqi = er * xqi + ei * xqr;
                    npr = c * xpr - s * eqr;
                    npi = c * xpi - s * eqi;
                    nqr = s * xpr + c * eqr;
                    nqi = s * xpi + c * eqi;
                }
                if (col == q) npr = npi = 0.0;  // A_pq
                if (col == p) nqr = nqi = 0.0;  // A_qp
                if (col == p) npi = 0.0;        // A_pp real
                if (col == q) nqi = 0.0;        // A_qq real
                Ar[p * ld + col] = npr;
                Ar[q * ld + col] = nqr;
                if constexpr (!REAL) {
                    Ai[p * ld + col] = npi;
                    Ai[q * ld + col] = nqi;
                }
            }
            __syncthreads();
        }
        // every thread reads the flag before thread 0 may reset it
        const int finished = done;
        __syncthreads();
        if (finished) break;
    }
    // descending order (ties by index)
    if (tid < k) {
        const double v = Ar[tid * ld + tid];
        int rank = 0;
        for (int b = 0; b < k; b++) {
            const double u = Ar[b * ld + b];
            rank += (u > v) || (u == v && b < tid);
        }
        lam[(long long)blockIdx.x * k + rank] = v;
        D *w = W + (long long)blockIdx.x * k * k;
        for (int a = 0; a < k; a++) {
            if constexpr (REAL) w[a * k + rank] = Vr[a * ld + tid];
            else w[a * k + rank] = make_double2(Vr[a * ld + tid], Vi[a * ld + tid]);
        }
    }
}

// ---- rotations: out[b][i][x] = s_i sum_a W[b][a][i] f(in[b][a][x]) ----------
struct CombArgs {
    const void *in;      // [nb][kin][L]
    long long L;
    int kin, nout;
    const void *W;       // [nb][kin][kin] (columns = eigenvectors)
    const double *lam;   // [nb][kin] descending
    int scale;           // 1: s_i = lam_i^-1/2 (0 below 1e-12 of lam_0); 0: s_i = 1
    void *out64;         // optional [nb][kin][L] (FP64 / complex FP64)
    void *out32;         // optional [nb][kin][L] (float / float2)
    float2 *outb;        // optional [nb][out_rows][out_stride] complex float (basis format)
    long long out_rows, out_stride;
};

template <bool REAL, class TIN, bool CONJ_IN>
__global__ void __launch_bounds__(THREADS) combine_kernel(CombArgs a) {
    using D = typename Ty<REAL>::d;
    using F = typename Ty<REAL>::f;
    extern __shared__ __align__(16) unsigned char csm_raw[];
    D *ws = reinterpret_cast<D *>(csm_raw);  // [kin][nout]
    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    const long long b = blockIdx.y;
    const D *W = static_cast<const D *>(a.W) + b * a.kin * a.kin;
    const double *lam = a.lam + b * a.kin;
    const double l0 = fmax(lam[0], 0.0);
    for (int e = tid; e < a.kin * a.nout; e += THREADS) {
        const int r = e / a.nout, i = e % a.nout;
        double s = 1.0;
        if (a.scale) {
            const double l = lam[i];
            s = (l > 1e-12 * l0 && l > 0.0) ? 1.0 / sqrt(l) : 0.0;
        }
        ws[r * a.nout + i] = scale_(W[r * a.kin + i], s);
    }
    __syncthreads();
    const long long x = (long long)blockIdx.x * 32 + lane;
    if (x >= a.L) return;
    const TIN *in = static_cast<const TIN *>(a.in) + b * a.kin * a.L;
    D acc[CPT];
#pragma unroll
    for (int m = 0; m < CPT; m++) acc[m] = zero_<D>();
    for (int r = 0; r < a.kin; r++) {
        D v = to_d(in[r * a.L + x]);
        if (CONJ_IN) v = conj_(v);
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            const int i = warp + NW * m;
            if (i < a.nout) acc[m] = fma_(acc[m], ws[r * a.nout + i], v);
        }
    }
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        const int i = warp + NW * m;
        if (i >= a.nout) continue;
        if (a.out64) static_cast<D *>(a.out64)[(b * a.kin + i) * a.L + x] = acc[m];
        if (a.out32) static_cast<F *>(a.out32)[(b * a.kin + i) * a.L + x] = to_f(acc[m]);
        if (a.outb) a.outb[(b * a.out_rows + i) * a.out_stride + x] = to_f2(acc[m]);
    }
}

// ---- start subspace, energy ------------------------------------------------
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
// Standard normal pair by Box-Muller from two 53-bit uniforms in (0, 1].
__device__ __forceinline__ double2 gauss2(unsigned long long seed, unsigned long long i) {
    const unsigned long long h1 = mix64(seed ^ mix64(2 * i)), h2 = mix64(seed ^ mix64(2 * i + 1));
    const double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740992.0);
    const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    const double r = sqrt(-2.0 * log(u1));
    return make_double2(r * cospi(2.0 * u2), r * sinpi(2.0 * u2));
}

template <bool REAL>
__global__ void random_kernel(typename Ty<REAL>::d *q, long long n, unsigned long long seed) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double2 g = gauss2(seed, (unsigned long long)e);
    if constexpr (REAL) q[e] = g.x;
    else q[e] = g;
}

// partial[cta] = sum over this CTA's atoms of block 0 of sum_t |d_t|^2 (FP64).
__global__ void energy_kernel(double *partial, const float2 *x, long long x_stride, long long natoms,
                              long long nreps) {
    __shared__ double red[NW];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    double acc = 0.0;
    for (long long j = (long long)blockIdx.x * NW + warp; j < natoms; j += (long long)gridDim.x * NW) {
        const float2 *row = x + j * x_stride;
        for (long long t = lane; t < nreps; t += 32) {
            const float2 v = row[t];
            acc += (double)v.x * v.x + (double)v.y * v.y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < NW; w++) s += red[w];
        partial[blockIdx.x] = s;
    }
}

// ---- voxel binning into PT-row tiles ---------------------------------------
__global__ void count_bins_kernel(int *counts, const int *vox_bin, long long nvox) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v < nvox) atomicAdd(&counts[vox_bin[v]], 1);
}
__global__ void scan_tiles_kernel(const int *counts, long long *slot_start, long long *tile_start, long long *cursor,
                                  int nbins) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long s = 0, t = 0;
    for (int b = 0; b < nbins; b++) {
        slot_start[b] = s;
        tile_start[b] = t;
        cursor[b] = s;
        s += counts[b];
        t += (counts[b] + PT - 1) / PT;
    }
    slot_start[nbins] = s;
    tile_start[nbins] = t;
}
__global__ void scatter_kernel(long long *perm, long long *cursor, const int *vox_bin, long long nvox) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    const long long pos = atomicAdd(reinterpret_cast<unsigned long long *>(&cursor[vox_bin[v]]), 1ull);
    perm[pos] = v;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

template <class K>
cudaError_t allow_smem(K kern, size_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace svd

int project_voxels(float2 *out, long long out_stride, const float2 *img, long long img_stride, long long nvox,
                   long long nreps, const int *vox_bin, int nbins, const float2 *basis, long long basis_rows,
                   long long basis_stride, int rank, bool real_basis, cudaStream_t st) {
    using namespace svd;
    if (rank < 1 || rank > KMAX)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: rank must be in [1, %d] (got %d)", KMAX, rank);
    if (out_stride > rank)
        SNAPMRF_CUDA(cudaMemsetAsync(out, 0, (size_t)nvox * out_stride * sizeof(float2), st));
    ProjArgs a{};
    a.x = img;
    a.x_stride = img_stride;
    a.basis = basis;
    a.basis_rows = basis_rows;
    a.basis_stride = basis_stride;
    a.nreps = nreps;
    a.k = rank;
    a.out = out;
    a.out_stride = out_stride;
    a.out_col = 0;
    DeviceScratch s;
    long long ntiles;
    if (!vox_bin || nbins <= 1) {
        a.rows_per_block = nvox;
        ntiles = (nvox + PT - 1) / PT;
    } else {
        const size_t bytes = (size_t)nvox * 8 + 3 * (size_t)(nbins + 1) * 8 + (size_t)nbins * 4 + 64;
        SNAPMRF_CUDA(s.alloc(bytes, st));
        long long *perm = s.as<long long>();
        long long *slot_start = perm + nvox, *tile_start = slot_start + nbins + 1, *cursor = tile_start + nbins + 1;
        int *counts = reinterpret_cast<int *>(cursor + nbins + 1);
        SNAPMRF_CUDA(cudaMemsetAsync(counts, 0, (size_t)nbins * 4, st));
        count_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(counts, vox_bin, nvox);
        SNAPMRF_LAUNCH_CHECK();
        scan_tiles_kernel<<<1, 32, 0, st>>>(counts, slot_start, tile_start, cursor, nbins);
        SNAPMRF_LAUNCH_CHECK();
        scatter_kernel<<<nblk(nvox, 256), 256, 0, st>>>(perm, cursor, vox_bin, nvox);
        SNAPMRF_LAUNCH_CHECK();
        a.perm = perm;
        a.tile_start = tile_start;
        a.slot_start = slot_start;
        a.nbins = nbins;
        ntiles = (nvox + PT - 1) / PT + nbins;  // upper bound on the tiles
    }
    const size_t vsm = sizeof(VoxSmem);
    SNAPMRF_CUDA(allow_smem(project_voxels_kernel<true>, vsm));
    SNAPMRF_CUDA(allow_smem(project_voxels_kernel<false>, vsm));
    for (int c0 = 0; c0 < rank; c0 += VKC) {
        if (real_basis) project_voxels_kernel<true><<<(unsigned)ntiles, VTS * 32, vsm, st>>>(a, c0);
        else project_voxels_kernel<false><<<(unsigned)ntiles, VTS * 32, vsm, st>>>(a, c0);
        SNAPMRF_LAUNCH_CHECK();
    }
    return SNAPMRF_OK;
}

namespace svd {

// The iteration of the file comment in real (REAL) or complex arithmetic.
template <bool REAL>
int compress(const float2 *atoms, long long astride, long long nreps, long long nb, long long natoms, int max_rank,
             int k, const snapmrf_svd_opts &o, float2 *d_basis, long long basis_stride, float2 *d_coeffs,
             long long coeff_stride, int *rank_out, double *h_sv, cudaStream_t st) {
    using D = typename Ty<REAL>::d;
    using F = typename Ty<REAL>::f;
    const long long T = nreps, N = natoms;
    int dev = 0, nsm = 148;
    SNAPMRF_CUDA(cudaGetDevice(&dev));
    SNAPMRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));

    // splits: the range pass over atoms, the Gram sums over samples / atoms
    const long long tx = (T + PT - 1) / PT;
    int rsplits = (int)std::max(1ll, std::min((N + PT - 1) / PT, (4ll * nsm + nb * tx - 1) / (nb * tx)));
    const long long rper = ((N + rsplits - 1) / rsplits + PT - 1) / PT * PT;
    rsplits = (int)((N + rper - 1) / rper);
    auto gsplits_for = [&](long long L) {
        long long s = std::max(1ll, std::min((L + 4 * PT - 1) / (4 * PT), (2ll * nsm + nb - 1) / nb));
        return s;
    };
    const int gsT = (int)gsplits_for(T), gsN = (int)gsplits_for(N);
    const long long gperT = ((T + gsT - 1) / gsT + PT - 1) / PT * PT, gperN = ((N + gsN - 1) / gsN + PT - 1) / PT * PT;
    const int gs_max = std::max(gsT, gsN);

    size_t bytes = 0;
    auto take = [&](size_t n) {
        size_t off = bytes;
        bytes += (n + 255) & ~size_t(255);
        return off;
    };
    const size_t oQ64 = take((size_t)nb * k * T * sizeof(D)), oQ32 = take((size_t)nb * k * T * sizeof(float2));
    const size_t oY64 = take((size_t)nb * k * T * sizeof(D));
    const size_t oP = take((size_t)nb * k * N * sizeof(F)), oZ = take((size_t)nb * k * N * sizeof(F));
    const size_t oP64 = take((size_t)nb * k * N * sizeof(D));
    const size_t oYp = take((size_t)nb * rsplits * k * T * sizeof(F));
    const size_t oGp = take((size_t)nb * gs_max * k * k * sizeof(D)), oG = take((size_t)nb * k * k * sizeof(D));
    const size_t oW = take((size_t)nb * k * k * sizeof(D)), oL = take((size_t)nb * k * sizeof(double));
    const int eparts = nsm;
    const size_t oE = take((size_t)eparts * sizeof(double));
    DeviceScratch s;
    SNAPMRF_CUDA(s.alloc(bytes, st));
    unsigned char *base = s.as<unsigned char>();
    D *Q64 = reinterpret_cast<D *>(base + oQ64);
    float2 *Q32 = reinterpret_cast<float2 *>(base + oQ32);
    D *Y64 = reinterpret_cast<D *>(base + oY64);
    F *P = reinterpret_cast<F *>(base + oP);
    F *Z = reinterpret_cast<F *>(base + oZ);
    D *P64 = reinterpret_cast<D *>(base + oP64);
    F *Yp = reinterpret_cast<F *>(base + oYp);
    D *Gp = reinterpret_cast<D *>(base + oGp);
    D *G = reinterpret_cast<D *>(base + oG);
    D *W = reinterpret_cast<D *>(base + oW);
    double *lam = reinterpret_cast<double *>(base + oL);
    double *epart = reinterpret_cast<double *>(base + oE);

    const size_t jac_smem = (size_t)(REAL ? 2 : 4) * (k + (k & 1)) * (k + (k & 1) + 1) * sizeof(double);
    const size_t comb_smem = (size_t)k * k * sizeof(D);
    SNAPMRF_CUDA(allow_smem(jacobi_kernel<REAL>, jac_smem));
    SNAPMRF_CUDA(allow_smem(combine_kernel<REAL, D, false>, comb_smem));
    SNAPMRF_CUDA(allow_smem(combine_kernel<REAL, F, true>, comb_smem));
    const size_t p64_smem = (size_t)(REAL ? 1 : 2) * KMAX * (PT + 1) * sizeof(double);
    SNAPMRF_CUDA(allow_smem(project64_kernel<REAL>, p64_smem));

    // Gram of a [nb][k][L] array -> G, then its eigen-decomposition -> W, lam
    auto gram_eig = [&](const void *A, long long L, bool atom_side, bool fp64_in = false) -> int {
        GramArgs g{};
        g.A = A;
        g.L = L;
        g.k = k;
        g.gpart = Gp;
        g.splits = atom_side ? gsN : gsT;
        g.per_split = atom_side ? gperN : gperT;
        g.splits = (int)((L + g.per_split - 1) / g.per_split);
        if (atom_side && !fp64_in) gram_kernel<REAL, F><<<dim3(g.splits, nb), THREADS, 0, st>>>(g);
        else gram_kernel<REAL, D><<<dim3(g.splits, nb), THREADS, 0, st>>>(g);
        SNAPMRF_LAUNCH_CHECK();
        reduce_gram_kernel<REAL><<<nblk(nb * k * k, 256), 256, 0, st>>>(G, Gp, nb, g.splits, k, atom_side ? 1 : 0);
        SNAPMRF_LAUNCH_CHECK();
        jacobi_kernel<REAL><<<(unsigned)nb, THREADS, jac_smem, st>>>(G, W, lam, k);
        SNAPMRF_LAUNCH_CHECK();
        return SNAPMRF_OK;
    };
    // Q64, Q32 <- orth(Y64)
    auto orth_T = [&](const D *Yin) -> int {
        int rc = gram_eig(Yin, T, false);
        if (rc) return rc;
        CombArgs c{};
        c.in = Yin;
        c.L = T;
        c.kin = k;
        c.nout = k;
        c.W = W;
        c.lam = lam;
        c.scale = 1;
        c.out64 = Q64;
        c.out32 = nullptr;
        c.outb = Q32;
        c.out_rows = k;
        c.out_stride = T;
        combine_kernel<REAL, D, false><<<dim3(nblk(T, 32), nb), THREADS, comb_smem, st>>>(c);
        SNAPMRF_LAUNCH_CHECK();
        return SNAPMRF_OK;
    };
    // P <- Q^H D (atom side, [nb][k][N])
    auto project_atoms = [&](const float2 *basis, long long brows, long long bstride, int kc, void *out,
                             long long ostride, int out_col, bool outf2) -> int {
        ProjArgs a{};
        a.x = atoms;
        a.x_stride = astride;
        a.rows_per_block = N;
        a.basis = basis;
        a.basis_rows = brows;
        a.basis_stride = bstride;
        a.nreps = T;
        a.k = kc;
        a.out = out;
        a.out_stride = ostride;
        a.out_col = out_col;
        const dim3 grid(nblk(N, PT), (unsigned)nb);
        if (REAL) {
            if (outf2) project_kernel<2, true><<<grid, THREADS, 0, st>>>(a);
            else project_kernel<2, false><<<grid, THREADS, 0, st>>>(a);
        } else {
            project_kernel<0, true><<<grid, THREADS, 0, st>>>(a);
        }
        SNAPMRF_LAUNCH_CHECK();
        return SNAPMRF_OK;
    };

    int rc;
    // start: orthonormal Gaussian subspace
    random_kernel<REAL><<<nblk(nb * k * T, 256), 256, 0, st>>>(Y64, nb * k * T, o.seed ^ 0x5eedull);
    SNAPMRF_LAUNCH_CHECK();
    if ((rc = orth_T(Y64))) return rc;
    const int iters = o.power_iters < 0 ? 0 : (o.power_iters == 0 ? 3 : o.power_iters);
    for (int it = 0; it < iters; it++) {
        if ((rc = project_atoms(Q32, k, T, k, P, N, 1, false))) return rc;
        if ((rc = gram_eig(P, N, true))) return rc;
        // Z = D^H Q W L^-1/2: z_i[j] = s_i sum_a W[a][i] conj(P[a][j])
        CombArgs c{};
        c.in = P;
        c.L = N;
        c.kin = k;
        c.nout = k;
        c.W = W;
        c.lam = lam;
        c.scale = 1;
        c.out32 = Z;
        combine_kernel<REAL, F, true><<<dim3(nblk(N, 32), nb), THREADS, comb_smem, st>>>(c);
        SNAPMRF_LAUNCH_CHECK();
        RangeArgs r{};
        r.x = atoms;
        r.x_stride = astride;
        r.natoms = N;
        r.nreps = T;
        r.k = k;
        r.z = Z;
        r.ypart = Yp;
        r.splits = rsplits;
        r.per_split = rper;
        range_kernel<REAL><<<dim3((unsigned)tx, rsplits, (unsigned)nb), THREADS, 0, st>>>(r);
        SNAPMRF_LAUNCH_CHECK();
        reduce_range_kernel<REAL><<<nblk(nb * k * T, 256), 256, 0, st>>>(Y64, Yp, nb, rsplits, (long long)k * T);
        SNAPMRF_LAUNCH_CHECK();
        if ((rc = orth_T(Y64))) return rc;
    }
    // Rayleigh-Ritz in FP64: M = (Q^H D)(Q^H D)^H = W L W^H
    project64_kernel<REAL><<<dim3(nblk(N, PT), (unsigned)nb), THREADS, p64_smem, st>>>(atoms, astride, N, Q64, T, k,
                                                                                      P64);
    SNAPMRF_LAUNCH_CHECK();
    if ((rc = gram_eig(P64, N, true, true))) return rc;
    energy_kernel<<<eparts, THREADS, 0, st>>>(epart, atoms, astride, N, T);
    SNAPMRF_LAUNCH_CHECK();

    std::vector<double> h_lam((size_t)nb * k), h_e(eparts);
    SNAPMRF_CUDA(cudaMemcpyAsync(h_lam.data(), lam, h_lam.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    SNAPMRF_CUDA(cudaMemcpyAsync(h_e.data(), epart, h_e.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    SNAPMRF_CUDA(cudaStreamSynchronize(st));
    double energy = 0.0;
    for (double v : h_e) energy += v;
    int r = o.rank;
    if (r <= 0) {
        // MATLAB: nDictSpace = sum(cumsum(s.^2) ./ sum(s.^2) <= sfrac), block 0
        double cum = 0.0;
        r = 0;
        for (int i = 0; i < k; i++) {
            cum += std::max(h_lam[i], 0.0);
            if (energy > 0.0 && cum / energy <= o.sfrac) r = i + 1;
            else break;
        }
        if (r == 0)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                         "svd_compress: sfrac %g keeps no singular vector (the first holds %.9g of the energy)",
                         o.sfrac, energy > 0.0 ? std::max(h_lam[0], 0.0) / energy : 0.0);
        if (r > max_rank)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "svd_compress: sfrac %g keeps more than max_rank = %d vectors", o.sfrac,
                         max_rank);
    }
    if (h_sv)
        for (long long b = 0; b < nb; b++)
            for (int i = 0; i < max_rank; i++) h_sv[b * max_rank + i] = std::sqrt(std::max(h_lam[b * k + i], 0.0));
    *rank_out = r;

    // U_r = Q W[:, :r] into the caller's basis (rows >= r zero)
    SNAPMRF_CUDA(cudaMemsetAsync(d_basis, 0, (size_t)nb * max_rank * basis_stride * sizeof(float2), st));
    {
        CombArgs c{};
        c.in = Q64;
        c.L = T;
        c.kin = k;
        c.nout = r;
        c.W = W;
        c.lam = lam;
        c.scale = 0;
        c.outb = d_basis;
        c.out_rows = max_rank;
        c.out_stride = basis_stride;
        combine_kernel<REAL, D, false><<<dim3(nblk(T, 32), nb), THREADS, comb_smem, st>>>(c);
        SNAPMRF_LAUNCH_CHECK();
    }
    // C = U_r^H D, columns >= r zero
    SNAPMRF_CUDA(cudaMemsetAsync(d_coeffs, 0, (size_t)nb * N * coeff_stride * sizeof(float2), st));
    return project_atoms(d_basis, max_rank, basis_stride, r, d_coeffs, coeff_stride, 0, true);
}

}  // namespace svd
}  // namespace snapmrf

using namespace snapmrf;

extern "C" int snapmrf_svd_compress(const float *d_atoms, size_t nreps, size_t NATOMS, size_t natoms, int max_rank,
                                    float *d_basis, size_t basis_stride, float *d_coeffs, size_t coeff_stride,
                                    int *rank, double *h_sv, const snapmrf_svd_opts *opts, void *stream) {
    if (!d_atoms || !d_basis || !d_coeffs || !rank) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "svd_compress: null pointer");
    if (nreps == 0 || natoms == 0 || NATOMS % natoms != 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "svd_compress: bad sizes (nreps %zu, NATOMS %zu, natoms %zu)", nreps, NATOMS,
                     natoms);
    snapmrf_svd_opts o{};
    if (opts) o = *opts;
    const int over = o.oversample > 0 ? o.oversample : 8;
    if (max_rank < 1 || o.rank > max_rank || max_rank + over > svd::KMAX)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                     "svd_compress: need 1 <= max_rank, rank <= max_rank and max_rank + oversample <= %d "
                     "(max_rank %d, rank %d, oversample %d)",
                     svd::KMAX, max_rank, o.rank, over);
    if (o.rank <= 0 && !(o.sfrac > 0.0 && o.sfrac <= 1.0))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "svd_compress: sfrac must be in (0, 1] (got %g)", o.sfrac);
    const size_t astride = o.atom_stride ? o.atom_stride : nreps;
    if (astride < nreps || basis_stride < nreps || coeff_stride < (size_t)max_rank)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "svd_compress: strides must be >= nreps (atoms, basis) and >= max_rank (coeffs)");
    const size_t nb = NATOMS / natoms;
    if (nb > 65535) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "svd_compress: more than 65535 B1 blocks");
    if (natoms > 0x7fffffffull / svd::KMAX)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "svd_compress: too many atoms per block");
    const int k = max_rank + over;
    cudaStream_t st = (cudaStream_t)stream;
    const float2 *atoms = reinterpret_cast<const float2 *>(d_atoms);
    float2 *basis = reinterpret_cast<float2 *>(d_basis);
    float2 *coeffs = reinterpret_cast<float2 *>(d_coeffs);
    if (o.flags & SNAPMRF_SVD_IMAG_ATOMS)
        return svd::compress<true>(atoms, (long long)astride, (long long)nreps, (long long)nb, (long long)natoms,
                                   max_rank, k, o, basis, (long long)basis_stride, coeffs, (long long)coeff_stride,
                                   rank, h_sv, st);
    return svd::compress<false>(atoms, (long long)astride, (long long)nreps, (long long)nb, (long long)natoms,
                                max_rank, k, o, basis, (long long)basis_stride, coeffs, (long long)coeff_stride, rank,
                                h_sv, st);
}
