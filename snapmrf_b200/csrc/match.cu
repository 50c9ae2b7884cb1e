// Maximum-inner-product matching on sm_100a (replaces MRF_match,
// MRF_minimatch, generate_maps, merge_maps and compute_nsplits,
// src/functions.cu:1317-1584).
//
// The reference runs a full FP32 CGEMM of every voxel against every B1
// block, materialises the score matrix, scans it per voxel, then merges the
// blocks.  Here voxels are first grouped by the B1 block they will be merged
// into (counting sort), each group is scored only against its block's atoms
// by a fused complex GEMM whose epilogue keeps the running first-argmax of
// |s|^2, and CTAs that split a block's atoms merge their winners with one
// 64-bit atomicMax per voxel on (score bits << 32 | ~index): larger score
// wins, equal scores go to the lower atom index, like the reference's strict
// '>' scan.  Without a B1 map the blocks' max-PD merge is the global first
// argmax, which is computed directly over all atoms.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "common.h"
#include "match_kernels.cuh"
#include "match_tc.h"
#include "svd.h"

namespace snapmrf {

// Nearest-B1 block per voxel (merge_maps with a B1 map,
// src/functions.cu:1351-1384): strict '<' from an initial 10, so ties go to
// the lower block and a voxel more than 10 away from every block (or NaN)
// goes to block 0.
__global__ void assign_bins_kernel(int *vox_bin, int *counts, const float *b1map,
                                   const float *params, int nparams, long long natoms,
                                   int nblocks, long long nvox) {
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    float gt = b1map[v];
    int best = 0;
    float best_abs = 10.f;
    for (int k = 0; k < nblocks; k++) {
        float b1 = params[(long long)k * natoms * nparams + 3];
        float d = fabsf(gt - b1);
        if (d < best_abs) {
            best_abs = d;
            best = k;
        }
    }
    vox_bin[v] = best;
    atomicAdd(&counts[best], 1);
}

// Exclusive scans of the per-bin voxel counts (slots) and voxel tiles.
__global__ void scan_bins_kernel(const int *counts, long long *slot_start, long long *tile_start,
                                 long long *cursor, int nbins) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long s = 0, t = 0;
    for (int b = 0; b < nbins; b++) {
        slot_start[b] = s;
        tile_start[b] = t;
        cursor[b] = s;
        s += counts[b];
        t += (counts[b] + kMatchVT - 1) / kMatchVT;
    }
    slot_start[nbins] = s;
    tile_start[nbins] = t;
}

__global__ void scatter_bins_kernel(long long *perm, long long *cursor, const int *vox_bin,
                                    long long nvox) {
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    long long pos = atomicAdd((unsigned long long *)&cursor[vox_bin[v]], 1ull);
    perm[pos] = v;
}

// Bins that all hold every voxel: slot_start[b] = b*nvox, tile_start[b] = b*vt.
__global__ void uniform_bins_kernel(long long *slot_start, long long *tile_start, int nbins,
                                    long long nvox, long long vt) {
    long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (b > nbins) return;
    slot_start[b] = b * nvox;
    tile_start[b] = b * vt;
}

// Every block's B1 equal to its first atom's (true for trans_params tables).
__global__ void check_uniform_b1_kernel(int *bad, const float *params, int nparams,
                                        long long natoms, long long NATOMS) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= NATOMS) return;
    long long head = (i / natoms) * natoms;
    if (params[i * nparams + 3] != params[head * nparams + 3]) atomicExch(bad, 1);
}

// Per voxel: decode the winning atom, recompute its exact FP32 inner product
// (PD = hypotf(|s|), generate_maps, src/functions.cu:1318-1349) and write
// maps[v] = {T1, T2, B0, B1, PD}.  One warp per voxel.
__global__ void finalize_maps_kernel(float *maps, long long *index_out, const unsigned long long *keys,
                                     const long long *perm, const int *vox_bin, const float2 *atoms,
                                     long long atom_stride, const float2 *img, long long img_stride,
                                     long long nreps, const float *params, int nparams,
                                     long long natoms_per_bin, long long nslots) {
    long long s = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    int lane = threadIdx.x % 32;
    if (s >= nslots) return;
    long long v = perm ? perm[s] : s;
    long long bin = vox_bin ? vox_bin[v] : 0;
    unsigned long long key = keys[s];
    long long local = key ? (long long)(0xffffffffull - (key & 0xffffffffull)) : 0;
    long long g = bin * natoms_per_bin + local;
    const float2 *d = atoms + g * atom_stride;
    const float2 *x = img + v * img_stride;
    float re = 0.f, im = 0.f;
    if (key) {
        for (long long t = lane; t < nreps; t += 32) {
            float2 a = d[t], b = x[t];
            re += a.x * b.x + a.y * b.y;
            im += a.x * b.y - a.y * b.x;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
    }
    if (lane == 0) {
        const float *p = params + g * nparams;
        float *m = maps + v * 5;
        m[0] = p[0];
        m[1] = p[1];
        m[2] = p[2];
        m[3] = p[3];
        m[4] = key ? hypotf(re, im) : 0.f;
        if (index_out) index_out[v] = g;
    }
}

// General B1-map merge when a block holds several B1 values: every block was
// matched against every voxel (keys[k * nvox + v]); pick the block whose
// matched atom's B1 is nearest the map (src/functions.cu:1351-1384).
__global__ void merge_nearest_b1_kernel(unsigned long long *keys_out, int *vox_bin,
                                        const unsigned long long *keys, const float *b1map,
                                        const float *params, int nparams, long long natoms,
                                        int nblocks, long long nvox) {
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    float gt = b1map[v];
    int best = 0;
    float best_abs = 10.f;
    for (int k = 0; k < nblocks; k++) {
        unsigned long long key = keys[(long long)k * nvox + v];
        long long local = key ? (long long)(0xffffffffull - (key & 0xffffffffull)) : 0;
        float b1 = params[((long long)k * natoms + local) * nparams + 3];
        float d = fabsf(gt - b1);
        if (d < best_abs) {
            best_abs = d;
            best = k;
        }
    }
    vox_bin[v] = best;
    keys_out[v] = keys[(long long)best * nvox + v];
}

// Maps of a call whose device-side check failed (*err != 0): NaN, index -1.
__global__ void poison_maps_kernel(float *maps, long long *index_out, long long nvox, const int *err) {
    if (!*err) return;
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    const float nan = __int_as_float(0x7fc00000);
    for (int k = 0; k < 5; k++) maps[v * 5 + k] = nan;
    if (index_out) index_out[v] = -1;
}

namespace tc {
// Copies a call's error code into the library's device error word (match_tc.cu).
__global__ void publish_error_kernel(const int *err);
}

static inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Copy stream and chunk events of the calling thread on the current device.
struct UploadContext {
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> ev;
};

// Chunks of one host-image upload: chunk c covers voxels [first(c), first(c+1)).
struct ImageUpload {
    int nchunks = 0;
    long long per = 0, nvox = 0;
    const cudaEvent_t *ev = nullptr;
    long long first(int c) const { return std::min(nvox, (long long)c * per); }
    cudaEvent_t done() const { return ev[nchunks - 1]; }
};

constexpr int kMaxUploadChunks = 8;
constexpr size_t kUploadChunkBytes = 16u << 20;

// Enqueues the copy of nvox host rows (stride `stride` samples, nreps copied)
// into dst [nvox][nreps] on the thread's copy stream, as up to
// kMaxUploadChunks 2D copies of at least kUploadChunkBytes, each followed by
// an event.  The copy stream first waits for the work already on `st`
// unless `early`.
static int upload_image(ImageUpload *up, float2 *dst, const float2 *src, size_t stride, size_t nreps,
                        size_t nvox, bool early, cudaStream_t st) {
    static thread_local std::map<int, UploadContext> ctx;
    int dev = 0;
    SNAPMRF_CUDA(cudaGetDevice(&dev));
    UploadContext &u = ctx[dev];
    if (!u.stream) {
        SNAPMRF_CUDA(cudaStreamCreateWithFlags(&u.stream, cudaStreamNonBlocking));
        SNAPMRF_CUDA(cudaEventCreateWithFlags(&u.start, cudaEventDisableTiming));
        u.ev.resize(kMaxUploadChunks);
        for (auto &e : u.ev) SNAPMRF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const size_t row = nreps * sizeof(float2);
    const size_t total = row * nvox;
    int n = (int)std::min<size_t>(kMaxUploadChunks, std::max<size_t>(1, total / kUploadChunkBytes));
    up->nvox = (long long)nvox;
    up->per = ((long long)nvox + n - 1) / n;
    n = (int)(((long long)nvox + up->per - 1) / up->per);
    up->nchunks = n;
    up->ev = u.ev.data();
    if (!early) {
        SNAPMRF_CUDA(cudaEventRecord(u.start, st));
        SNAPMRF_CUDA(cudaStreamWaitEvent(u.stream, u.start, 0));
    }
    for (int c = 0; c < n; c++) {
        const long long v0 = up->first(c), nv = up->first(c + 1) - v0;
        SNAPMRF_CUDA(cudaMemcpy2DAsync(dst + v0 * (long long)nreps, row, src + v0 * (long long)stride,
                                       stride * sizeof(float2), row, (size_t)nv, cudaMemcpyHostToDevice, u.stream));
        SNAPMRF_CUDA(cudaEventRecord(u.ev[c], u.stream));
    }
    return SNAPMRF_OK;
}

}  // namespace snapmrf

using namespace snapmrf;

extern "C" int snapmrf_mrf_match(float *d_maps, const float *img, int img_on_host,
                                 const float *d_atoms, const float *d_params, size_t nreps,
                                 size_t NATOMS, size_t natoms, size_t nvoxels, int nparams,
                                 int nmaps, const snapmrf_match_opts *opts, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const bool comp = opts && opts->basis;
    if (!d_maps || !img || (!d_atoms && !comp) || !d_params)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: null pointer");
    if (nmaps != 5 || nparams < 4)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: nmaps must be 5 and nparams >= 4");
    if (nreps == 0 || nvoxels == 0 || natoms == 0 || NATOMS % natoms != 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: bad sizes (nreps %zu, nvoxels %zu, NATOMS %zu, natoms %zu)",
                     nreps, nvoxels, NATOMS, natoms);
    int precision = opts ? opts->precision : SNAPMRF_PREC_FP32;
    if (precision != SNAPMRF_PREC_FP32 && precision != SNAPMRF_PREC_BF16 && precision != SNAPMRF_PREC_FP16 &&
        precision != SNAPMRF_PREC_FP8)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_match: unknown precision %d", precision);
    size_t img_stride = (opts && opts->img_stride) ? opts->img_stride : nreps;
    size_t atom_stride = (opts && opts->atom_stride) ? opts->atom_stride : nreps;
    if (img_stride < nreps || atom_stride < nreps)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: strides must be >= nreps");
    if (natoms >= 0xffffffffull || NATOMS >= (1ull << 40))
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_match: too many atoms per block");
    const float *b1map = opts ? opts->b1map : nullptr;
    const size_t nblocks = NATOMS / natoms;
    if (nblocks > 65535) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_match: more than 65535 B1 blocks");
    unsigned flags = opts ? opts->flags : 0u;
    int64_t *d_index = opts ? opts->d_index : nullptr;
    const float *atom_norms = opts ? opts->atom_norms : nullptr;
    if (atom_norms && (comp || !opts->packed_atoms ||
                       (precision != SNAPMRF_PREC_BF16 && precision != SNAPMRF_PREC_FP16)))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: atom_norms needs BF16 / FP16 matching with packed_atoms");
    const bool imag_rows = (flags & SNAPMRF_MATCH_IMAG_ROWS) != 0;
    if (imag_rows && (comp || !opts->packed_atoms || !(flags & SNAPMRF_MATCH_IMAG_ATOMS) ||
                      (precision != SNAPMRF_PREC_BF16 && precision != SNAPMRF_PREC_FP16)))
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                     "MRF_match: SNAPMRF_MATCH_IMAG_ROWS needs BF16 / FP16 matching with packed_atoms and "
                     "SNAPMRF_MATCH_IMAG_ATOMS");
    if (comp) {
        if (!opts->coeffs || opts->rank < 1 || opts->basis_rows < (size_t)opts->rank ||
            opts->basis_stride < nreps || opts->coeff_stride < (size_t)opts->rank)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                         "MRF_match: compressed matching needs coeffs, rank >= 1, basis_rows and coeff_stride >= rank "
                         "and basis_stride >= nreps");
        if (opts->packed_atoms)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: packed_atoms and a compressed basis are exclusive");
        if (!b1map && nblocks > 1)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                         "MRF_match: compressed matching of several B1 blocks needs a B1 map (one basis per block)");
    }

    // A host image is streamed to the device in chunks on the library's copy
    // stream (one 2D copy per chunk instead of one copy per voxel,
    // src/functions.cu:1524-1530), into img_device_copy or call scratch; the
    // FP32 form matches each chunk as it arrives, the tensor-core forms wait
    // for the whole image.
    float *img_copy = opts ? opts->img_device_copy : nullptr;
    const bool early = (flags & SNAPMRF_MATCH_UPLOAD_EARLY) != 0;
    if (img_copy && !img_on_host)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: img_device_copy applies to a host image (img_on_host)");
    if (early && !img_copy)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: SNAPMRF_MATCH_UPLOAD_EARLY needs img_device_copy");
    DeviceScratch s_img;
    const float2 *d_img = reinterpret_cast<const float2 *>(img);
    long long istride = (long long)img_stride;
    ImageUpload up;
    if (img_on_host) {
        float2 *dst = reinterpret_cast<float2 *>(img_copy);
        if (!dst) {
            SNAPMRF_CUDA(s_img.alloc(nvoxels * nreps * sizeof(float2), st));
            dst = s_img.as<float2>();
        }
        int rc = upload_image(&up, dst, reinterpret_cast<const float2 *>(img), img_stride, nreps, nvoxels, early, st);
        if (rc) return rc;
        d_img = dst;
        istride = (long long)nreps;
    }
    DeviceScratch s_b1;
    const float *d_b1 = b1map;
    if (b1map && opts->b1map_on_host) {
        SNAPMRF_CUDA(s_b1.alloc(nvoxels * sizeof(float), st));
        SNAPMRF_CUDA(cudaMemcpyAsync(s_b1.ptr, b1map, nvoxels * sizeof(float), cudaMemcpyHostToDevice, st));
        d_b1 = s_b1.as<float>();
    }

    // Mode: global argmax (no B1 map), nearest-B1 bins (uniform blocks), or
    // every block against every voxel followed by the nearest-B1 merge.
    bool general = false;
    if (d_b1 && nblocks > 1 && !(flags & SNAPMRF_MATCH_ASSUME_UNIFORM_B1)) {
        DeviceScratch s_bad;
        SNAPMRF_CUDA(s_bad.alloc(sizeof(int), st));
        SNAPMRF_CUDA(cudaMemsetAsync(s_bad.ptr, 0, sizeof(int), st));
        check_uniform_b1_kernel<<<nblk((long long)NATOMS, 256), 256, 0, st>>>(
            s_bad.as<int>(), d_params, nparams, (long long)natoms, (long long)NATOMS);
        SNAPMRF_LAUNCH_CHECK();
        int bad = 0;
        SNAPMRF_CUDA(cudaMemcpyAsync(&bad, s_bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        SNAPMRF_CUDA(cudaStreamSynchronize(st));
        general = bad != 0;
    }

    const long long nvox = (long long)nvoxels;
    if (comp && general)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                     "MRF_match: compressed matching needs every B1 block to hold one B1 value");
    if (precision == SNAPMRF_PREC_BF16 || precision == SNAPMRF_PREC_FP16 || precision == SNAPMRF_PREC_FP8) {
        if (general)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                         "MRF_match: tensor-core matching needs every B1 block to hold one B1 value");
        TcMatchRequest q;
        q.maps = d_maps;
        q.index_out = (long long *)d_index;
        q.img = d_img;
        q.img_stride = istride;
        q.atoms = reinterpret_cast<const float2 *>(d_atoms);
        q.atom_stride = (long long)atom_stride;
        q.params = d_params;
        q.nparams = nparams;
        q.nreps = (long long)nreps;
        q.NATOMS = (long long)NATOMS;
        q.natoms = (long long)natoms;
        q.nvox = nvox;
        q.nblocks = (int)nblocks;
        q.b1map = d_b1;
        q.fmt = precision == SNAPMRF_PREC_FP16 ? 1 : precision == SNAPMRF_PREC_FP8 ? 2 : 0;
        q.imag = (flags & SNAPMRF_MATCH_IMAG_ATOMS) != 0;
        q.packed = opts ? opts->packed_atoms : nullptr;
        q.atom_norms = atom_norms;
        q.imag_rows = imag_rows;
        if (q.packed && (!q.imag || q.fmt == 2 || opts->packed_nreps != nreps))
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                         "MRF_match: packed_atoms need SNAPMRF_MATCH_IMAG_ATOMS, BF16 / FP16 and packed_nreps == nreps");
        q.basis = comp ? reinterpret_cast<const float2 *>(opts->basis) : nullptr;
        q.basis_rows = comp ? (long long)opts->basis_rows : 0;
        q.basis_stride = comp ? (long long)opts->basis_stride : 0;
        q.coeffs = comp ? reinterpret_cast<const float2 *>(opts->coeffs) : nullptr;
        q.coeff_stride = comp ? (long long)opts->coeff_stride : 0;
        q.rank = comp ? opts->rank : 0;
        q.topk = (opts && opts->topk) ? opts->topk : (q.fmt == 1 ? 4 : 16);
        if (q.topk != 4 && q.topk != 8 && q.topk != 16)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_match: topk must be 4, 8 or 16 (got %d)", q.topk);
        if (img_on_host && up.nchunks >= 4) {
            // A streamed image: the voxels of all but the last two chunks are
            // matched as soon as they have arrived (and the work queued
            // before, such as the dictionary, is done), the rest when the
            // upload ends, so that only about a quarter of the matching waits
            // for the last copies.  Each voxel's scores, candidates and
            // rescoring do not depend on the other voxels of its call.
            const long long vA = up.first(up.nchunks - 2);
            SNAPMRF_CUDA(cudaStreamWaitEvent(st, up.ev[up.nchunks - 3], 0));
            TcMatchRequest qa = q;
            qa.nvox = vA;
            int rc = match_bf16(qa, st);
            if (rc) return rc;
            SNAPMRF_CUDA(cudaStreamWaitEvent(st, up.done(), 0));
            TcMatchRequest qb = q;
            qb.maps = q.maps + vA * 5;
            qb.index_out = q.index_out ? q.index_out + vA : nullptr;
            qb.img = q.img + vA * q.img_stride;
            qb.b1map = q.b1map ? q.b1map + vA : nullptr;
            qb.nvox = nvox - vA;
            return match_bf16(qb, st);
        }
        if (img_on_host) SNAPMRF_CUDA(cudaStreamWaitEvent(st, up.done(), 0));
        return match_bf16(q, st);
    }
    // the FP32 kernels carry an atom's index within its bin as an int
    if (!d_b1 && NATOMS >= 0x7fffffffull)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                     "MRF_match: FP32 matching without a B1 map takes fewer than 2^31 - 1 atoms (got %zu)", NATOMS);
    // The FP32 path over voxels [v0, v0 + nvox): a host image streamed in
    // chunks is matched chunk by chunk as each chunk arrives.
    auto fp32_range = [&](long long v0, long long nvox, float *d_maps, int64_t *d_index, const float2 *d_img,
                          const float *d_b1) -> int {
        (void)v0;
        int nbins;
        long long per_bin_atoms, nslots;
        if (!d_b1) {
            nbins = 1;
            per_bin_atoms = (long long)NATOMS;
            nslots = nvox;
        } else if (!general) {
            nbins = (int)nblocks;
            per_bin_atoms = (long long)natoms;
            nslots = nvox;
        } else {
            nbins = (int)nblocks;
            per_bin_atoms = (long long)natoms;
            nslots = nvox * (long long)nblocks;
        }

        // purely imaginary atoms: half the products (the imaginary parts only)
        const bool imag = (flags & SNAPMRF_MATCH_IMAG_ATOMS) != 0;
        // scratch: keys[nslots] u64 | perm[nvox] i64 | slot_start, tile_start,
        // cursor [nbins+1] i64 | vox_bin[nvox] i32 | counts[nbins] i32 | err i32
        size_t bytes = (size_t)nslots * 8 + (size_t)nvox * 8 + 3 * (size_t)(nbins + 1) * 8 +
                       (size_t)nvox * 4 + (size_t)nbins * 4 + 64;
        DeviceScratch s_work;
        SNAPMRF_CUDA(s_work.alloc(bytes, st));
        unsigned long long *keys = s_work.as<unsigned long long>();
        long long *perm = reinterpret_cast<long long *>(keys + nslots);
        long long *slot_start = perm + nvox;
        long long *tile_start = slot_start + (nbins + 1);
        long long *cursor = tile_start + (nbins + 1);
        int *vox_bin = reinterpret_cast<int *>(cursor + (nbins + 1));
        int *counts = vox_bin + nvox;
        int *err = counts + nbins;
        SNAPMRF_CUDA(cudaMemsetAsync(keys, 0, (size_t)nslots * 8, st));
        if (imag) SNAPMRF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));

        MatchArgs m;
        m.atoms = reinterpret_cast<const float2 *>(d_atoms);
        m.atom_stride = (long long)atom_stride;
        m.img = d_img;
        m.img_stride = istride;
        m.nreps = (long long)nreps;
        m.nbins = nbins;
        m.bin_natoms = per_bin_atoms;
        m.nvox = nvox;
        m.keys = keys;
        m.err = imag ? err : nullptr;

        if (!d_b1) {
            // one bin, identity permutation
            uniform_bins_kernel<<<1, 256, 0, st>>>(slot_start, tile_start, 1, nvox,
                                                   (nvox + kMatchVT - 1) / kMatchVT);
            SNAPMRF_LAUNCH_CHECK();
            m.perm = nullptr;
            m.perm_mod = 0;
        } else if (!general) {
            SNAPMRF_CUDA(cudaMemsetAsync(counts, 0, (size_t)nbins * 4, st));
            assign_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(vox_bin, counts, d_b1, d_params, nparams,
                                                                (long long)natoms, nbins, nvox);
            SNAPMRF_LAUNCH_CHECK();
            scan_bins_kernel<<<1, 32, 0, st>>>(counts, slot_start, tile_start, cursor, nbins);
            SNAPMRF_LAUNCH_CHECK();
            scatter_bins_kernel<<<nblk(nvox, 256), 256, 0, st>>>(perm, cursor, vox_bin, nvox);
            SNAPMRF_LAUNCH_CHECK();
            m.perm = perm;
            m.perm_mod = 0;
        } else {
            uniform_bins_kernel<<<nblk(nbins + 1, 256), 256, 0, st>>>(slot_start, tile_start, nbins, nvox,
                                                                      (nvox + kMatchVT - 1) / kMatchVT);
            SNAPMRF_LAUNCH_CHECK();
            m.perm = nullptr;
            m.perm_mod = nvox;
        }
        m.slot_start = slot_start;
        m.tile_start = tile_start;

        // Compressed: score the rank-r coordinates of the atoms against the
        // voxels projected onto their bin's basis; the maps' PD is the
        // compressed |s|.
        DeviceScratch s_cimg;
        if (comp) {
            const long long rs = (opts->rank + 1) & ~1ll;
            SNAPMRF_CUDA(s_cimg.alloc((size_t)nvox * rs * sizeof(float2), st));
            int rc = project_voxels(s_cimg.as<float2>(), rs, d_img, istride, nvox, (long long)nreps,
                                    d_b1 ? vox_bin : nullptr, nbins, reinterpret_cast<const float2 *>(opts->basis),
                                    (long long)opts->basis_rows, (long long)opts->basis_stride, opts->rank,
                                    (flags & SNAPMRF_MATCH_IMAG_ATOMS) != 0, st);
            if (rc) return rc;
            m.img = s_cimg.as<float2>();
            m.img_stride = rs;
            m.atoms = reinterpret_cast<const float2 *>(opts->coeffs);
            m.atom_stride = (long long)opts->coeff_stride;
            m.nreps = opts->rank;
        }

        long long max_tiles = general ? (long long)nbins * ((nvox + kMatchVT - 1) / kMatchVT)
                                      : (nvox + kMatchVT - 1) / kMatchVT + nbins;
        long long est_tiles = general ? max_tiles : (nvox + kMatchVT - 1) / kMatchVT;
        dim3 grid = fp32_match_grid(m, est_tiles, max_tiles);
        SNAPMRF_CUDA(launch_match_fp32(m, grid, imag, st));

        const unsigned long long *fkeys = keys;
        if (general) {
            DeviceScratch s_merged;
            SNAPMRF_CUDA(s_merged.alloc((size_t)nvox * 8, st));
            merge_nearest_b1_kernel<<<nblk(nvox, 256), 256, 0, st>>>(s_merged.as<unsigned long long>(), vox_bin,
                                                                     keys, d_b1, d_params, nparams,
                                                                     (long long)natoms, nbins, nvox);
            SNAPMRF_LAUNCH_CHECK();
            finalize_maps_kernel<<<nblk(nvox * 32, 256), 256, 0, st>>>(
                d_maps, (long long *)d_index, s_merged.as<unsigned long long>(), nullptr, vox_bin,
                m.atoms, m.atom_stride, d_img, istride, (long long)nreps, d_params, nparams,
                (long long)natoms, nvox);
            SNAPMRF_LAUNCH_CHECK();
            if (imag) {
                poison_maps_kernel<<<nblk(nvox, 256), 256, 0, st>>>(d_maps, (long long *)d_index, nvox, err);
                SNAPMRF_LAUNCH_CHECK();
                tc::publish_error_kernel<<<1, 1, 0, st>>>(err);
                SNAPMRF_LAUNCH_CHECK();
            }
            return SNAPMRF_OK;
        }
        finalize_maps_kernel<<<nblk(nvox * 32, 256), 256, 0, st>>>(
            d_maps, (long long *)d_index, fkeys, d_b1 ? perm : nullptr, d_b1 ? vox_bin : nullptr, m.atoms,
            m.atom_stride, m.img, m.img_stride, m.nreps, d_params, nparams, per_bin_atoms, nvox);
        SNAPMRF_LAUNCH_CHECK();
        if (imag) {
            // an atom with a real part: NaN maps, indices -1, error word 7
            poison_maps_kernel<<<nblk(nvox, 256), 256, 0, st>>>(d_maps, (long long *)d_index, nvox, err);
            SNAPMRF_LAUNCH_CHECK();
            tc::publish_error_kernel<<<1, 1, 0, st>>>(err);
            SNAPMRF_LAUNCH_CHECK();
        }
        return SNAPMRF_OK;
    };
    if (!img_on_host || up.nchunks <= 1 || comp || general) {
        if (img_on_host) SNAPMRF_CUDA(cudaStreamWaitEvent(st, up.done(), 0));
        return fp32_range(0, nvox, d_maps, d_index, d_img, d_b1);
    }
    for (int c = 0; c < up.nchunks; c++) {
        const long long v0 = up.first(c), n = up.first(c + 1) - v0;
        SNAPMRF_CUDA(cudaStreamWaitEvent(st, up.ev[c], 0));
        int rc = fp32_range(v0, n, d_maps + 5 * v0, d_index ? d_index + v0 : nullptr, d_img + v0 * istride,
                            d_b1 ? d_b1 + v0 : nullptr);
        if (rc) return rc;
    }
    return SNAPMRF_OK;
}
