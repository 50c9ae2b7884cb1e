// Matching entry point that allocates no device memory.
//
// snapmrf_mrf_match allocates its working arrays with cudaMallocAsync on
// every call.  Some callers cannot allow that: a host framework that has
// already reserved the GPU's free memory in its own caching allocator (a
// cudaMalloc would fail, or force that allocator to flush and synchronise),
// or a reconstruction pipeline on a scanner that must not allocate once it
// is running, because an allocation can stall the device and break its
// latency budget.  This variant takes every buffer it needs from one
// file-scope __device__ array of fixed size, so all of its device memory is
// reserved when the library is loaded and nothing is allocated afterwards.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the parts that must start at zero are cleared at the start of
// each call.  Two calls whose device work overlaps (on different streams or
// host threads) would use the same array at once and race: issue them one
// after another on one stream, or serialise them.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"
#define SNAPMRF_MATCH_KERNEL_DECLARATION_ONLY
#include "match_kernels.cuh"

namespace snapmrf {

// Kernels of the ordinary matching path (match.cu).
__global__ void assign_bins_kernel(int *vox_bin, int *counts, const float *b1map, const float *params,
                                   int nparams, long long natoms, int nblocks, long long nvox);
__global__ void scan_bins_kernel(const int *counts, long long *slot_start, long long *tile_start,
                                 long long *cursor, int nbins);
__global__ void scatter_bins_kernel(long long *perm, long long *cursor, const int *vox_bin,
                                    long long nvox);
__global__ void uniform_bins_kernel(long long *slot_start, long long *tile_start, int nbins,
                                    long long nvox, long long vt);
__global__ void check_uniform_b1_kernel(int *bad, const float *params, int nparams, long long natoms,
                                        long long NATOMS);
__global__ void finalize_maps_kernel(float *maps, long long *index_out, const unsigned long long *keys,
                                     const long long *perm, const int *vox_bin, const float2 *atoms,
                                     long long atom_stride, const float2 *img, long long img_stride,
                                     long long nreps, const float *params, int nparams,
                                     long long natoms_per_bin, long long nslots);

namespace {

// Layout of the scratch array: keys[V] u64 | perm[V] i64 | slot_start,
// tile_start, cursor [B+1] i64 | vox_bin[V] i32 | counts[B] i32 | flag i32
// (set when a B1 block holds several B1 values).
constexpr size_t kMaxVoxels = SNAPMRF_NOALLOC_MAX_VOXELS;
constexpr size_t kMaxBlocks = SNAPMRF_NOALLOC_MAX_B1_BLOCKS;
constexpr size_t kScratchBytes = kMaxVoxels * 8 + kMaxVoxels * 8 + 3 * (kMaxBlocks + 1) * 8 +
                                 kMaxVoxels * 4 + kMaxBlocks * 4 + 16;

__device__ __align__(256) unsigned char g_match_scratch[kScratchBytes];

// Error word of this path (read by snapmrf_device_error).
__device__ int g_noalloc_error;

// Device address of g_match_scratch on the current device.  In host code
// the symbol names a host-side shadow, not device memory, so the address is
// looked up (with the device current) on every call: a host-side query that
// enqueues nothing, and that stays right after a device reset re-creates the
// context and loads the array again.
int scratch_address(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_match_scratch);
    if (e != cudaSuccess || !p)
        SNAPMRF_FAIL(SNAPMRF_ERR_CUDA, "MRF_match_noalloc: cudaGetSymbolAddress failed: %s",
                     cudaGetErrorString(e));
    *out = p;
    return SNAPMRF_OK;
}

__global__ void clear_scratch_kernel(unsigned long long *keys, long long nkeys, int *counts, int ncounts,
                                     int *flag) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < nkeys) keys[i] = 0ull;
    if (i < ncounts) counts[i] = 0;
    if (i == 0) *flag = 0;
}

// A B1 block with several B1 values cannot be matched by nearest-B1 bins:
// such a call's maps become NaN, its indices -1, and the error word 9.
__global__ void reject_mixed_b1_kernel(float *maps, long long *index_out, long long nvox, const int *flag) {
    if (!*flag) return;
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v == 0) atomicCAS(&g_noalloc_error, 0, 9);
    if (v >= nvox) return;
    const float nan = __int_as_float(0x7fc00000);
    for (int k = 0; k < 5; k++) maps[v * 5 + k] = nan;
    if (index_out) index_out[v] = -1;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Reads (and with reset clears) this path's error word; snapmrf_device_error
// reports it beside the tensor-core kernels' word.
cudaError_t noalloc_device_error(int *value, int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(value, g_noalloc_error, sizeof(int));
    if (e == cudaSuccess && reset) {
        int z = 0;
        e = cudaMemcpyToSymbol(g_noalloc_error, &z, sizeof(int));
    }
    return e;
}

}  // namespace snapmrf

using namespace snapmrf;

extern "C" int snapmrf_mrf_match_noalloc(float *d_maps, const float *d_img, size_t img_stride,
                                         const float *d_atoms, size_t atom_stride,
                                         const float *d_params, size_t nreps, size_t NATOMS,
                                         size_t natoms, size_t nvoxels, int nparams, int nmaps,
                                         const float *d_b1map, int64_t *d_index, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_maps || !d_img || !d_atoms || !d_params)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match_noalloc: null pointer");
    if (nmaps != 5 || nparams < 4)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match_noalloc: nmaps must be 5 and nparams >= 4");
    if (nreps == 0 || nvoxels == 0 || natoms == 0 || NATOMS % natoms != 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match_noalloc: bad sizes (nreps %zu, nvoxels %zu, NATOMS %zu, natoms %zu)",
                     nreps, nvoxels, NATOMS, natoms);
    if (!img_stride) img_stride = nreps;
    if (!atom_stride) atom_stride = nreps;
    if (img_stride < nreps || atom_stride < nreps)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match_noalloc: strides must be >= nreps");
    if (nvoxels > kMaxVoxels)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                     "MRF_match_noalloc: %zu voxels exceed the fixed scratch limit of %zu; split the "
                     "image into calls of at most %zu voxels or use snapmrf_mrf_match",
                     nvoxels, kMaxVoxels, kMaxVoxels);
    const size_t nblocks = NATOMS / natoms;
    if (d_b1map && nblocks > kMaxBlocks)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match_noalloc: %zu B1 blocks exceed the fixed limit of %zu",
                     nblocks, kMaxBlocks);
    if (natoms >= 0xffffffffull || (!d_b1map && NATOMS >= 0x7fffffffull))
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_match_noalloc: too many atoms");

    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    const long long nvox = (long long)nvoxels;
    const int nbins = d_b1map ? (int)nblocks : 1;
    unsigned char *p = static_cast<unsigned char *>(base);
    unsigned long long *keys = reinterpret_cast<unsigned long long *>(p);
    long long *perm = reinterpret_cast<long long *>(p + kMaxVoxels * 8);
    long long *slot_start = reinterpret_cast<long long *>(p + 2 * kMaxVoxels * 8);
    long long *tile_start = slot_start + (kMaxBlocks + 1);
    long long *cursor = tile_start + (kMaxBlocks + 1);
    int *vox_bin = reinterpret_cast<int *>(cursor + (kMaxBlocks + 1));
    int *counts = vox_bin + kMaxVoxels;
    int *flag = counts + kMaxBlocks;

    // keys, the per-bin counts and the flag start at zero on every call
    clear_scratch_kernel<<<nblk(std::max<long long>(nvox, nbins), 256), 256, 0, st>>>(keys, nvox, counts, nbins,
                                                                                      flag);
    SNAPMRF_LAUNCH_CHECK();
    if (d_b1map && nblocks > 1) {
        check_uniform_b1_kernel<<<nblk((long long)NATOMS, 256), 256, 0, st>>>(flag, d_params, nparams,
                                                                              (long long)natoms, (long long)NATOMS);
        SNAPMRF_LAUNCH_CHECK();
    }

    MatchArgs m;
    m.atoms = reinterpret_cast<const float2 *>(d_atoms);
    m.atom_stride = (long long)atom_stride;
    m.img = reinterpret_cast<const float2 *>(d_img);
    m.img_stride = (long long)img_stride;
    m.nreps = (long long)nreps;
    m.nbins = nbins;
    m.bin_natoms = d_b1map ? (long long)natoms : (long long)NATOMS;
    m.nvox = nvox;
    m.keys = keys;
    m.perm_mod = 0;
    m.slot_start = slot_start;
    m.tile_start = tile_start;
    if (d_b1map) {
        assign_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(vox_bin, counts, d_b1map, d_params, nparams,
                                                            (long long)natoms, nbins, nvox);
        SNAPMRF_LAUNCH_CHECK();
        scan_bins_kernel<<<1, 32, 0, st>>>(counts, slot_start, tile_start, cursor, nbins);
        SNAPMRF_LAUNCH_CHECK();
        scatter_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(perm, cursor, vox_bin, nvox);
        SNAPMRF_LAUNCH_CHECK();
        m.perm = perm;
    } else {
        uniform_bins_kernel<<<1, 256, 0, st>>>(slot_start, tile_start, 1, nvox, (nvox + kMatchVT - 1) / kMatchVT);
        SNAPMRF_LAUNCH_CHECK();
        m.perm = nullptr;
    }
    const long long max_tiles = (nvox + kMatchVT - 1) / kMatchVT + nbins;
    dim3 grid = fp32_match_grid(m, (nvox + kMatchVT - 1) / kMatchVT, max_tiles);
    m.err = nullptr;
    SNAPMRF_CUDA(launch_match_fp32(m, grid, false, st));
    finalize_maps_kernel<<<nblk(nvox * 32, 256), 256, 0, st>>>(
        d_maps, (long long *)d_index, keys, d_b1map ? perm : nullptr, d_b1map ? vox_bin : nullptr, m.atoms,
        m.atom_stride, m.img, m.img_stride, (long long)nreps, d_params, nparams, m.bin_natoms, nvox);
    SNAPMRF_LAUNCH_CHECK();
    if (d_b1map && nblocks > 1) {
        reject_mixed_b1_kernel<<<nblk(nvox, 256), 256, 0, st>>>(d_maps, (long long *)d_index, nvox, flag);
        SNAPMRF_LAUNCH_CHECK();
    }
    return SNAPMRF_OK;
}
