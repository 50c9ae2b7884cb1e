/*
 * snapmrf.h -- C ABI of the B200-native snapMRF hot path.
 *
 * The path: MRF dictionary generation (extended-phase-graph recursion for
 * the FISP / SSFP / SR / SE / TSE echo types, ROA Bloch isochromats) and
 * maximum-inner-product template matching of voxel signal evolutions into
 * T1 / T2 / B0 / B1 / PD maps.
 *
 * Conventions (all entry points):
 *   - plain C types only; complex arrays are interleaved float pairs
 *     (re, im), i.e. the reference's float2 layout;
 *   - device pointers are caller-owned; scratch is allocated stream-ordered
 *     inside the call and released before it returns;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *     device work is enqueued on it and the call returns without waiting,
 *     except where a function says it synchronises;
 *   - every entry point returns a snapmrf_status; snapmrf_last_error()
 *     returns the message of the last failure on the calling thread.
 *     Nothing in the library prints, waits on stdin or exits.
 *
 * Layouts follow the reference (src/functions.h, src/mrf.cu):
 *   params [NATOMS][nparams] = {T1 ms, T2 ms, B0 Hz, B1}
 *   schedule h_mrf [4][NREPS] = CSV columns (flip, phase, TR, TE)
 *   atoms  [NATOMS][nreps] complex
 *   image  [nvoxels][img_stride] complex
 *   maps   [nvoxels][nmaps] = {T1, T2, B0, B1, PD}
 */
#ifndef SNAPMRF_H
#define SNAPMRF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum snapmrf_status {
    SNAPMRF_OK = 0,
    SNAPMRF_ERR_INVALID = 1,     /* bad argument or size */
    SNAPMRF_ERR_ECHO_TYPE = 2,   /* unknown echo type (reference: err(EX_USAGE)) */
    SNAPMRF_ERR_CUDA = 3,        /* a CUDA runtime call or launch failed */
    SNAPMRF_ERR_ALLOC = 4,       /* device or host allocation failed */
    SNAPMRF_ERR_IO = 5,          /* file open / read / write failed */
    SNAPMRF_ERR_FORMAT = 6,      /* malformed RA / CSV / grid string */
    SNAPMRF_ERR_UNSUPPORTED = 7, /* valid request this build does not handle */
    SNAPMRF_ERR_DEVICE = 8       /* device-side check failed (bounded wait, bad index) */
} snapmrf_status;

/* Message of the last failing call on this thread ("" if none). */
const char *snapmrf_last_error(void);
/* Library version string. */
const char *snapmrf_version(void);
/* Number of CUDA kernels this library has launched in this process (all
 * threads, all devices): an exact count for benchmarks and tests. */
uint64_t snapmrf_kernel_launches(void);
/* Number of device scratch allocations this library has made in this
 * process (stream-ordered, from the pool below): a diagnostic that lets a
 * caller check that a call allocated nothing. */
uint64_t snapmrf_scratch_allocations(void);
/* Scratch memory is taken from a per-device pool that keeps freed blocks
 * for reuse by later calls; this returns the cached memory of the current
 * device to the driver (it synchronises the device first). */
int snapmrf_release_scratch(void);

/* ------------------------------------------------------------------------
 * Host: schedules, grids and the parameter table.
 * Each keeps the float arithmetic of the reference function it replaces.
 * ---------------------------------------------------------------------- */

/* Number of '\n' in the file (replaces csv_dim, src/functions.cu:100-120).
 * Returns (size_t)-1 when the file cannot be opened. */
size_t snapmrf_csv_dim(const char *path);

/* Reads up to nreps schedule rows into h_mrf[4][nreps], skipping the first
 * two 100-byte fgets chunks exactly like csv_read (src/functions.cu:122-158). */
int snapmrf_csv_read(float *h_mrf, size_t nreps, const char *path);

/* "min", "min:max" or "min:step:max" (parse_range, src/functions.cu:197-237). */
int snapmrf_parse_range(const char *str, float *min, float *step, float *max, size_t *len);

/* Length of a '+'-joined grid string (parse_length, src/functions.cu:239-269).
 * Returns 0 on a malformed string. */
size_t snapmrf_parse_length(const char *str);

/* Fills h_p[LEN] from a grid string (parse_params, src/functions.cu:315-353). */
int snapmrf_parse_params(float *h_p, const char *str, size_t LEN);

/* linspace / logspace (src/functions.cu:271-313), including logspace's
 * symmetric negative branch used by the -N grids. */
void snapmrf_linspace(float *h_p, float min, float step, size_t len);
void snapmrf_logspace(float *h_p, float min, float max, size_t len);

/* Atoms with T1 > T2, times l_b0 * l_b1 (compute_natoms, src/functions.cu:393-414). */
size_t snapmrf_compute_natoms(const float *h_t1, const float *h_t2, size_t l_t1,
                              size_t l_t2, size_t l_b0, size_t l_b1);

/* params[NATOMS][nparams] in B1 > B0 > T2 > T1 order, T1 > T2 only
 * (trans_params, src/functions.cu:355-391). */
int snapmrf_trans_params(float *h_params, const float *h_t1, const float *h_t2,
                         const float *h_b0, const float *h_b1, size_t l_t1, size_t l_t2,
                         size_t l_b0, size_t l_b1, size_t NATOMS, int nparams);

/* ------------------------------------------------------------------------
 * RA files (replaces ra_read / ra_write / ra_free, src/ra.h:60-74,
 * src/ra.cu:23-104).  Same 48-byte header + dims + data layout.
 * ---------------------------------------------------------------------- */
typedef struct snapmrf_ra {
    uint64_t flags;
    uint64_t eltype; /* 0 user, 1 int, 2 uint, 3 float, 4 complex */
    uint64_t elbyte;
    uint64_t size;   /* data bytes */
    uint64_t ndims;
    uint64_t *dims;
    uint8_t *data;   /* page-locked when read with pinned != 0; snapmrf_ra_read
                        records that in flags bit 63, which is never written */
} snapmrf_ra;

/* Reads an RA file; data in page-locked host memory when pinned != 0
 * (the reference builds with -DCUDA_HOST_MALLOC, src/ra.cu:39-44).
 * Checks the magic number and that the file holds `size` data bytes. */
int snapmrf_ra_read(snapmrf_ra *a, const char *path, int pinned);
int snapmrf_ra_write(const snapmrf_ra *a, const char *path);
void snapmrf_ra_free(snapmrf_ra *a);

/* ------------------------------------------------------------------------
 * Dictionary generation (replaces MRF_dict, src/functions.cu:1224-1315, and
 * the echo-type engines epg_sr/epg_se/epg_tse/epg_fisp/epg_ssfp/roa_ssfp,
 * src/functions.cu:687-1222).
 * ---------------------------------------------------------------------- */

/* Generate every B1 block for the non-SSFP echo types, flip angle scaled by
 * the block's B1 (the reference's epg_fisp/sr/se/tse/roa fill block 0 only,
 * unscaled, src/functions.cu:1293-1309). */
#define SNAPMRF_DICT_ALL_B1_BLOCKS 0x1u
/* Normalise every generated atom to unit l2 norm (the reference normalises
 * only epg_ssfp and roa_ssfp, src/functions.cu:1268, 1297). */
#define SNAPMRF_DICT_NORMALIZE 0x2u
/* Use the reference's operation order (complex state, separate relaxation
 * and RF steps) even where the real-valued fast recursion applies. */
#define SNAPMRF_DICT_REFERENCE_ORDER 0x4u
/* Real-valued recursion (FISP / SR with every RF phase 0) with the
 * reference's two relaxations per step, bit-identical to the complex
 * recursion.  By default that recursion folds each step's relaxation over
 * TR into the next step's RF instead (relaxation commutes with the
 * dephasing shift), which changes results by rounding only (~1e-7). */
#define SNAPMRF_DICT_SEPARATE_RELAX 0x8u
/* With d_packed (and without SNAPMRF_DICT_NORMALIZE): write the 16-bit
 * operand of the unit-norm atoms, bit-identical to the one written with
 * SNAPMRF_DICT_NORMALIZE, while d_atoms keeps the atoms as generated; with
 * d_norms, their norms.  snapmrf_mrf_match takes such a dictionary with
 * snapmrf_match_opts.atom_norms.  Saves rewriting the FP32 atoms. */
#define SNAPMRF_DICT_NORMALIZE_OPERAND 0x10u
/* epg_fisp / epg_sr with every RF phase 0 only (their atoms are purely
 * imaginary): d_atoms receives Im(atom) as FP32 rows, [NATOMS][nreps] float
 * (half the bytes of the complex rows, whose real parts are zeros), with the
 * same values bit for bit.  snapmrf_mrf_match reads such rows with
 * SNAPMRF_MATCH_IMAG_ROWS and snapmrf_refine_start with
 * SNAPMRF_START_IMAG_ROWS.  Other echo types and schedules fail with
 * SNAPMRF_ERR_UNSUPPORTED. */
#define SNAPMRF_DICT_IMAG_ROWS 0x20u

typedef struct snapmrf_dict_opts {
    unsigned flags;  /* SNAPMRF_DICT_* */
    int n_iso;       /* ROA isochromats per atom, dephased across 2*pi per TR (1 = reference) */
    float *d_norms;  /* optional out [NATOMS]: l2 norm of each generated atom before normalisation */
    /* Optional out, device [NATOMS][snapmrf_packed_pitch(nreps)] 16-bit
     * (packed_precision SNAPMRF_PREC_BF16 or _FP16): the imaginary part of
     * each generated atom (as written to d_atoms), zero padded, which
     * snapmrf_mrf_match takes as snapmrf_match_opts.packed_atoms instead of
     * packing the atoms itself.  Only for the real-valued recursion (epg_fisp
     * / epg_sr with every RF phase 0, whose atoms are purely imaginary). */
    void *d_packed;
    int packed_precision;
} snapmrf_dict_opts;

/* Row pitch (elements) of packed atoms for nreps time points. */
size_t snapmrf_packed_pitch(size_t nreps);

/* d_atoms: out, device [NATOMS][nreps] complex (blocks the echo type does
 *          not generate are left untouched, as in the reference)
 * d_params: device [NATOMS][nparams]; h_mrf: host [4][NREPS];
 * nreps <= NREPS time points; natoms atoms per B1 block (NATOMS % natoms == 0);
 * nstates EPG states w; echo_type in {epg_ssfp, roa_ssfp, epg_sr, epg_se,
 * epg_tse1, epg_tse2, epg_fisp}; opts may be NULL (reference behaviour). */
int snapmrf_mrf_dict(float *d_atoms, const float *d_params, const float *h_mrf,
                     size_t nreps, size_t NREPS, size_t NATOMS, size_t natoms,
                     int nparams, int nstates, const char *echo_type,
                     const snapmrf_dict_opts *opts, void *stream);

/* Engine-level generation, as the reference's echo-type engines
 * epg_sr / epg_se / epg_tse / epg_fisp / epg_ssfp / roa_ssfp run it
 * (src/functions.h:89-113, src/functions.cu:687-1222): the schedule is
 * already converted and in device memory, d_mrf [4][nreps] = {flip (rad),
 * phase (rad), TR (ms), TE (ms)} (no CSV conversion), and the atoms are not
 * normalised unless SNAPMRF_DICT_NORMALIZE asks for it (MRF_dict normalises
 * the epg_ssfp / roa_ssfp atoms after the engine, src/functions.cu:1268,
 * 1297).  ti: epg_ssfp's inversion delay in ms (MRF_dict passes 40); the
 * other echo types ignore it.  Blocks, options and limits as for
 * snapmrf_mrf_dict.  Synchronises `stream` once (the schedule is read back
 * to choose the recursion). */
int snapmrf_dict_engine(float *d_atoms, const float *d_params, const float *d_mrf, float ti,
                        size_t nreps, size_t NATOMS, size_t natoms, int nparams, int nstates,
                        const char *echo_type, const snapmrf_dict_opts *opts, void *stream);

/* In-place unit-l2 normalisation of NATOMS atoms of nreps samples
 * (replaces the normalize kernel, src/functions.cu:670-685). */
int snapmrf_normalize(float *d_atoms, size_t nreps, size_t NATOMS, float *d_norms,
                      void *stream);

/* ------------------------------------------------------------------------
 * Matching (replaces MRF_match / MRF_minimatch / generate_maps /
 * merge_maps / compute_nsplits, src/functions.cu:1317-1584).
 * ---------------------------------------------------------------------- */
#define SNAPMRF_PREC_FP32 0  /* FP32 scores (the reference's cublasCgemm form) */
/* BF16 scores on the tensor cores (FP32 accumulation, each voxel scaled to
 * unit norm first), a per-voxel top-k (snapmrf_match_opts.topk, 4, 8 or 16;
 * 16 by default for BF16, 4 for FP16),
 * then exact FP32 rescoring of those k atoms: the map is the FP32 first
 * argmax among them.  Needs B1 blocks holding one B1 value each when a B1
 * map is given. */
#define SNAPMRF_PREC_BF16 1
/* The same with FP16 operands (8x finer mantissa than BF16, same rate). */
#define SNAPMRF_PREC_FP16 2
/* The same with FP8-E4M3 operands (twice the BF16 rate, 3 mantissa bits):
 * each atom row and each voxel row is scaled so its largest component is
 * 448, scores are divided by the atom's squared scale before the top-k
 * (16 by default), and the k candidates are rescored in FP32. */
#define SNAPMRF_PREC_FP8 3

/* Skip the device check that every B1 block holds one B1 value (true for
 * any params table built by trans_params); without the flag the call
 * synchronises `stream` once to read the check's result. */
#define SNAPMRF_MATCH_ASSUME_UNIFORM_B1 0x1u
/* The atoms are purely imaginary (every Re d_t is 0), as the FISP / SR
 * dictionaries of schedules whose RF phases are all 0 are.  The BF16 / FP16
 * forms then score |s|^2 = (sum Im d x_r)^2 + (sum Im d x_i)^2 with one
 * operand row per atom: half the tensor-core work.  An atom with a non-zero
 * real part makes the call's maps NaN and sets the device error word
 * (snapmrf_device_error() == 7).  Other precisions ignore the flag. */
#define SNAPMRF_MATCH_IMAG_ATOMS 0x2u
/* With a host image (img_on_host) and snapmrf_match_opts.img_device_copy:
 * the image upload may start at once, before the work already queued on
 * `stream` (such as the dictionary generation whose atoms this call
 * matches) has finished, so that the two overlap.  The caller guarantees
 * that no work queued before this call still uses img_device_copy (for
 * instance by alternating two buffers between calls). */
#define SNAPMRF_MATCH_UPLOAD_EARLY 0x4u
/* d_atoms holds Im(atom) rows as SNAPMRF_DICT_IMAG_ROWS writes them
 * ([NATOMS][atom_stride] float).  Needs SNAPMRF_MATCH_IMAG_ATOMS, BF16 or
 * FP16 matching and packed_atoms (the atoms are read only by the FP32
 * rescoring of the candidates); other forms fail with
 * SNAPMRF_ERR_UNSUPPORTED. */
#define SNAPMRF_MATCH_IMAG_ROWS 0x8u

typedef struct snapmrf_match_opts {
    int precision;          /* SNAPMRF_PREC_* */
    unsigned flags;         /* SNAPMRF_MATCH_* */
    size_t img_stride;      /* complex samples between voxels (0 = nreps) */
    size_t atom_stride;     /* complex samples between atoms (0 = nreps) */
    const float *b1map;     /* optional [nvoxels] B1 map: match within the nearest B1 block */
    int b1map_on_host;      /* b1map is host memory */
    int64_t *d_index;       /* optional out [nvoxels]: chosen global atom index */
    int topk;               /* tensor-core forms: candidates rescored in FP32, 4, 8 or 16 (0: default) */
    /* Optional: the atoms packed by snapmrf_mrf_dict (snapmrf_dict_opts.d_packed)
     * in this call's precision (BF16 or FP16) for these same nreps
     * (packed_nreps == nreps); needs SNAPMRF_MATCH_IMAG_ATOMS.  The FP32
     * atoms are still read for the exact rescoring. */
    const void *packed_atoms;
    size_t packed_nreps;
    /* Optional: compressed matching against a low-rank dictionary from
     * snapmrf_svd_compress.  basis: device complex
     * [nblocks][basis_rows][basis_stride] (the r leading left singular
     * vectors of each B1 block, over nreps samples); coeffs: device complex
     * [NATOMS][coeff_stride] (each atom's r coordinates in its block's
     * basis); rank: r.  Each voxel is projected onto its B1 block's basis and
     * scored against the coordinates (r instead of nreps products per pair).
     * FP32: the maps come from the compressed scores (PD = |<c, U^H x>|), as
     * matching against the MATLAB code's dict_compress does.  BF16 / FP16 /
     * FP8: the top-k candidates of the compressed scores are rescored
     * exactly in FP32 against d_atoms and the voxels (against the
     * coordinates and projected voxels when d_atoms is NULL).  Needs a B1
     * map (with one B1 value per block) or a single block; with
     * SNAPMRF_MATCH_IMAG_ATOMS the basis is taken as real (its imaginary
     * parts are not read) and the coordinates must be purely imaginary, as
     * snapmrf_svd_compress writes them for such atoms.  Not combinable with
     * packed_atoms. */
    const float *basis;
    size_t basis_rows, basis_stride;
    const float *coeffs;
    size_t coeff_stride;
    int rank;
    /* Optional, device [NATOMS]: the l2 norm of each atom of d_atoms, which
     * are then taken as not normalised (a dictionary made with
     * SNAPMRF_DICT_NORMALIZE_OPERAND): the exact FP32 rescoring divides each
     * candidate's inner product by its atom's norm, so the maps are those of
     * unit-norm atoms.  BF16 / FP16 with packed_atoms only (the candidates
     * come from the unit-norm packed operand). */
    const float *atom_norms;
    /* Optional, device [nvoxels][nreps] complex, with a host image: the
     * upload lands here and stays for the caller (for instance for
     * snapmrf_refine_gn), instead of in scratch freed by the call. */
    float *img_device_copy;
} snapmrf_match_opts;

/* d_maps: out, device [nvoxels][nmaps] (nmaps == 5, nparams == 4)
 * img: [nvoxels][img_stride] complex, host memory when img_on_host != 0.
 * A host image is copied in up to 8 chunks of at least 16 MB on a copy
 * stream of the library (one per host thread and device); the FP32 form
 * matches each chunk as soon as it has arrived, while the next ones are in
 * flight, and the tensor-core forms start once the whole image is there.
 * Page-locked host memory makes the copies asynchronous: the call then
 * returns before they finish, so keep the host image unchanged until the
 * call's work on `stream` has completed;
 * nreps time points are matched.  Per B1 block the first atom with the
 * largest |<atom, voxel>| wins; blocks are merged by nearest B1 when a B1
 * map is given (ties to the lower block, differences >= 10 to block 0),
 * otherwise by the largest PD (ties to the lower block). */
int snapmrf_mrf_match(float *d_maps, const float *img, int img_on_host,
                      const float *d_atoms, const float *d_params, size_t nreps,
                      size_t NATOMS, size_t natoms, size_t nvoxels, int nparams, int nmaps,
                      const snapmrf_match_opts *opts, void *stream);

/* ------------------------------------------------------------------------
 * Low-rank (SVD) compression of a dictionary per B1 block, the method of
 * McGivney et al. (IEEE TMI 2014) as matlab/MRF_dict_B1.m:127-159 applies it
 * (input.reduce = 1): each block's atoms D_b (nreps x natoms, columns as
 * stored) are represented by their coordinates C_b = U_r^H D_b in the span
 * of the block's r leading left singular vectors U_r.  The rank comes from
 * block 0 with the MATLAB rule r = #{i : (s_1^2 + ... + s_i^2) /
 * ||D_0||_F^2 <= sfrac}, and every block keeps r vectors.  The reference's
 * CUDA path has no counterpart.
 *
 * The singular vectors are computed by subspace iteration: k = max_rank +
 * oversample vectors (k <= SNAPMRF_SVD_MAX_SUBSPACE), a seeded random
 * start, power_iters rounds of D D^H with FP64 Gram matrices and FP64
 * Jacobi eigensolvers for the k x k problems, then a Rayleigh-Ritz step.
 * Deterministic for a given seed.
 * ---------------------------------------------------------------------- */
#define SNAPMRF_SVD_MAX_SUBSPACE 80
/* The atoms are purely imaginary (every Re d_t is 0, as for
 * SNAPMRF_MATCH_IMAG_ATOMS): the singular vectors are computed in real
 * arithmetic, the basis is real (imaginary parts 0) and the coordinates
 * purely imaginary (real parts 0). */
#define SNAPMRF_SVD_IMAG_ATOMS 0x2u

typedef struct snapmrf_svd_opts {
    unsigned flags;         /* SNAPMRF_SVD_* */
    size_t atom_stride;     /* complex samples between atoms (0 = nreps) */
    double sfrac;           /* energy fraction kept (the MATLAB rule) when rank == 0 */
    int rank;               /* > 0: keep exactly this many vectors (<= max_rank) */
    int oversample;         /* subspace vectors beyond max_rank (0: 8) */
    int power_iters;        /* rounds of D D^H (0: 3; < 0: none) */
    unsigned long long seed;/* random start of the subspace */
} snapmrf_svd_opts;

/* d_atoms: device complex [NATOMS][atom_stride], NATOMS = nblocks * natoms;
 * d_basis: out, device complex [nblocks][max_rank][basis_stride]: row i of
 *   block b is u_i over the nreps samples (rows >= r are zero);
 * d_coeffs: out, device complex [NATOMS][coeff_stride] (coeff_stride >=
 *   max_rank): c_j = U_r^H d_j in columns [0, r), zero in [r, max_rank);
 * rank: out, r;
 * h_sv: optional out, host [nblocks][max_rank]: each block's leading
 *   singular values (Ritz values), descending.
 * Synchronises `stream` once (to choose r).  Returns SNAPMRF_ERR_INVALID when
 * sfrac keeps no vector or more than max_rank. */
int snapmrf_svd_compress(const float *d_atoms, size_t nreps, size_t NATOMS, size_t natoms, int max_rank,
                         float *d_basis, size_t basis_stride, float *d_coeffs, size_t coeff_stride,
                         int *rank, double *h_sv, const snapmrf_svd_opts *opts, void *stream);

/* Device-side error word (0 when no error was recorded).  Codes: 1-6 a
 * bounded wait of the tensor-core matching kernel ran out (the maps of that
 * call are NaN); 7 SNAPMRF_MATCH_IMAG_ATOMS was given atoms with a non-zero
 * real part (NaN maps); 9 snapmrf_mrf_match_noalloc was given a B1 map and
 * a B1 block holding several B1 values (NaN maps, indices -1); 10 the
 * bounded-wait self-test (snapmrf_selftest_bounded_wait).
 * Synchronises the current device; clears the word when reset != 0. */
int snapmrf_device_error(int reset);

/* Self-test of the bounded waits behind the device error word: launches one
 * warp that waits, with a limit of limit_us microseconds (1 .. 2,000,000),
 * on an mbarrier that nothing arrives on, the wait primitive of the
 * tensor-core kernels.  The wait gives up, the kernel returns and the error
 * word becomes 10 (snapmrf_device_error).  Nothing else is in flight in that
 * kernel, so the device stays usable.  No counterpart in the reference. */
int snapmrf_selftest_bounded_wait(unsigned limit_us, void *stream);

/* Largest request snapmrf_mrf_match_noalloc accepts: its working arrays live
 * in one fixed array of about 1.3 MiB per GPU (sized for 65,536 voxels and
 * 1,024 B1 blocks). */
#define SNAPMRF_NOALLOC_MAX_VOXELS 65536
#define SNAPMRF_NOALLOC_MAX_B1_BLOCKS 1024

/* Matching that allocates no device memory.  No counterpart in the
 * reference: its MRF_match allocates on every call, as snapmrf_mrf_match does.
 *
 * For callers that cannot allocate while they run: a host framework that
 * has already reserved the GPU's free memory in its own caching allocator
 * (a cudaMalloc here would fail, or make that allocator flush and
 * synchronise), or a scanner reconstruction pipeline that forbids
 * allocation after start-up because an allocation can stall the device.
 * Every working array comes from one __device__ array of fixed size that
 * each GPU holds from the moment the library is loaded until the process
 * exits; nothing is allocated or freed by the call.
 *
 * Same results as snapmrf_mrf_match in its FP32 form, with these limits:
 *   - d_img, d_b1map (optional) and every output are device memory;
 *   - nvoxels <= SNAPMRF_NOALLOC_MAX_VOXELS and, with a B1 map,
 *     NATOMS / natoms <= SNAPMRF_NOALLOC_MAX_B1_BLOCKS; larger requests
 *     return SNAPMRF_ERR_INVALID (split the image into several calls);
 *   - with a B1 map every B1 block must hold a single B1 value, as every
 *     table built by snapmrf_trans_params does; this is checked on the
 *     device without waiting for it: when a block holds several values the
 *     call's maps are NaN, its indices -1, and snapmrf_device_error()
 *     returns 9;
 *   - each call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress: host-side work, nothing enqueued); the first
 *     call on a device also makes the runtime load the array, so make that
 *     first call before any stream capture;
 *   - all calls on a device share the array and it keeps the previous
 *     call's contents (each call clears what must start at zero): calls
 *     whose device work overlaps race and give wrong maps, so issue them in
 *     order on one stream or otherwise serialise them.
 * Strides of 0 mean nreps. */
int snapmrf_mrf_match_noalloc(float *d_maps, const float *d_img, size_t img_stride,
                              const float *d_atoms, size_t atom_stride, const float *d_params,
                              size_t nreps, size_t NATOMS, size_t natoms, size_t nvoxels,
                              int nparams, int nmaps, const float *d_b1map, int64_t *d_index,
                              void *stream);

/* ------------------------------------------------------------------------
 * Derivatives of the EPG signal.  No counterpart in the reference, which
 * only evaluates the forward recursion.  Two recursions are differentiated:
 *   - the real-valued FISP / SR recursion (epg_fisp, epg_sr:
 *     src/functions.cu:687-739, 878-933, every RF phase 0) with the B1
 *     extension of snapmrf_mrf_dict (flip angle alpha_t * B1, no initial
 *     pulse); parameters T1, T2, B1;
 *   - the complex bSSFP recursion (epg_ssfp, src/functions.cu:935-1019: RF
 *     with any phase, B0 precession, the 180-degree inversion with TI = 40
 *     ms), h_mrf in the CSV convention it converts (flip fraction of 60
 *     degrees, phase in degrees, TR - 16 ms, TE - 3.5 ms), flip angle alpha_t
 *     * B1 (the continuous form of epg_ssfp's FA x b1); parameters T1, T2, B0,
 *     B1.  nstates <= 128.
 * ------------------------------------------------------------------------ */

/* Reverse mode (adjoint) with checkpointing.
 *
 * d_params: device [natoms][nparams] (T1, T2, B0, B1; nparams >= 4);
 * h_mrf: host [4][NREPS] schedule as for snapmrf_mrf_dict (row 1 must be 0);
 * d_grad_signal: device complex [natoms][nreps], dL/d(Re s_t, Im s_t) of a
 * real loss L of the (unnormalised) atoms s;
 * d_signal: optional out, the atoms (complex [natoms][nreps]);
 * d_grad_params: out [natoms][3]: dL/dT1, dL/dT2, dL/dB1 (epg_fisp /
 * epg_sr); [natoms][4]: dL/dT1, dL/dT2, dL/dB0, dL/dB1 (epg_ssfp);
 * d_grad_alpha: optional out [nreps]: dL/dh_mrf[0][t] (the schedule's flip
 * entries) summed over atoms;
 * d_grad_alpha_atoms: optional out [natoms][nreps]: the per-atom terms;
 * checkpoint_every: states kept every C steps (0: C = ceil(sqrt(nreps))),
 * so device scratch is natoms * (nreps/C + C) * 3 * nstates floats (rounded
 * up to the kernel's state layout). */
int snapmrf_epg_adjoint(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                        size_t NREPS, size_t natoms, int nstates, const char *echo_type,
                        const float *d_grad_signal, float *d_signal, float *d_grad_params,
                        float *d_grad_alpha, float *d_grad_alpha_atoms, int checkpoint_every,
                        void *stream);

/* Per-voxel Gauss-Newton refinement of matched (T1, T2), in place (epg_fisp /
 * epg_sr); of (T1, T2, B0) and, without d_b1map, B1 too for epg_ssfp (B0
 * steps limited to max_rel_step x 50 Hz, a voxel stops once its B0 step is
 * within tol x 100 Hz and its B1 step within tol of B1 as well).
 *
 * Model: voxel x = rho * s(T1, T2, B1) with rho complex, eliminated by
 * variable projection (rho = <s, x> / <s, s>); each iteration runs the
 * forward recursion with the tangents ds/dT1 and ds/dT2, then solves the
 * 2x2 normal equations of the projected residual.  Steps are clipped to
 * max_rel_step (0: 0.2) times the current value, and T1 > T2 > 0 is kept.
 *
 * d_maps: device in/out [nvoxels][nmaps] as snapmrf_mrf_match writes them
 * (T1, T2, B0, B1, PD): T1 and T2 are refined at the voxel's B1, taken from
 * d_b1map (optional device [nvoxels], the measured B1 map, then also written
 * to column 3) or else from column 3 (1 when nmaps < 4); with nmaps >= 5
 * column 4 is replaced by the PD of the refined signal, |<s, x>| / ||s||
 * (the matching PD of a unit-norm atom).  Voxels whose maps are not finite
 * or do not hold T1 > T2 > 0 are left as they are.
 * img: device complex [nvoxels][img_stride] (0 = nreps);
 * d_m0: optional out [nvoxels], |rho|.  PD, M0 and the B1 column are
 * written by the pass in which each voxel stops (with iterations == 0, by
 * one value-only forward pass).
 * iterations: at most this many Gauss-Newton steps per voxel; with tol > 0 a
 * voxel stops once a step changed both T1 and T2 by at most tol of their
 * values (later iterations run only over the voxels still moving). */
int snapmrf_refine_gn(float *d_maps, int nmaps, const float *img, size_t img_stride,
                      const float *d_b1map, const float *h_mrf, size_t nreps, size_t NREPS,
                      size_t nvoxels, int nstates, const char *echo_type, int iterations,
                      float max_rel_step, float tol, float *d_m0, void *stream);

/* Sub-grid start for snapmrf_refine_gn from the dictionary, in place.  No
 * counterpart in the reference (matching ends on the grid).
 *
 * For each voxel, the matched atom d_index[v] (as snapmrf_mrf_match writes
 * it), the atoms at the adjacent T1 and T2 values of the parameter table
 * (trans_params order, src/functions.cu:355-391) and one diagonal neighbour
 * (T1 and T2 both above, else both below) form a six-point stencil; with
 * d_b1map the stencil is taken from the three B1 blocks around the block of
 * the match and interpolated quadratically to the voxel's B1.  In (log T1,
 * log T2) the stencil gives the quadratic surrogate c + a U + b V + d U^2 +
 * e V^2 + f U V of the signal model, accurate to third order in the grid
 * step; the voxel's fit |<s, x>|^2 / ||s||^2 is maximised over it by
 * Gauss-Newton with variable projection (on the 6 x 6 Gram matrix of the
 * surrogate's terms and their inner products with the voxel, no recursion),
 * within 1.5 times the stencil's extent, and the result replaces (T1, T2) in
 * d_maps.  The start is typically within 1e-4 of the least-squares fit
 * (relative), so one refinement pass meets a stopping tolerance of 1e-3.
 *
 * Voxels are left as they are when the index is outside [0, NATOMS), the
 * maps no longer hold the matched atom's (T1, T2), the atom is on the edge of
 * the grid (no neighbour on one side in T1 or T2, an adjacent T2 row lacks
 * the matched T1, or neither diagonal node exists), the B1 blocks do not
 * share the stencil's rows, or the fit leaves T1 > T2 > 0.
 *
 * d_maps: device in/out [nvoxels][nmaps] (T1, T2 in columns 0 and 1);
 * d_atoms: device complex [NATOMS][nreps] (normalised or not);
 * d_params: device [NATOMS][nparams] (T1, T2, B0, B1), natoms per B1 block;
 * img: device complex [nvoxels][img_stride] (0 = nreps);
 * d_b1map: optional device [nvoxels] (needs nparams >= 4);
 * flags: SNAPMRF_START_IMAG_ATOMS when every atom is purely imaginary (the
 * zero-phase FISP / SR dictionaries), which multiplies half as much;
 * SNAPMRF_START_IMAG_ROWS (with SNAPMRF_START_IMAG_ATOMS) when d_atoms holds
 * Im(atom) rows as SNAPMRF_DICT_IMAG_ROWS writes them ([NATOMS][nreps]
 * float), which also reads half as much;
 * d_count: optional device counter, incremented once per voxel moved. */
#define SNAPMRF_START_IMAG_ATOMS 0x1u
#define SNAPMRF_START_IMAG_ROWS 0x2u
int snapmrf_refine_start(float *d_maps, int nmaps, const int64_t *d_index, const float *d_atoms,
                         const float *d_params, int nparams, size_t nreps, size_t NATOMS,
                         size_t natoms, const float *img, size_t img_stride, size_t nvoxels,
                         const float *d_b1map, unsigned flags, int *d_count, void *stream);

/* Forward mode (Jacobian-vector products) of the real FISP / SR recursion.
 * No counterpart in the reference; the forward model is its epg_fisp / epg_sr
 * (src/functions.cu:687-933) with flip angle alpha_t * B1 and every RF phase 0.
 *
 * d_params: device [natoms][nparams] (T1, T2, B0, B1; nparams >= 4);
 * h_mrf: host [4][NREPS] schedule as for snapmrf_mrf_dict (row 1 must be 0);
 * d_out: device out [natoms][3][nreps] = f, df/dT1, df/dT2, where s = i f is
 * the atom as generated (unnormalised).  The product of the Jacobian with a
 * direction (dT1, dT2) is dT1 * df/dT1 + dT2 * df/dT2.  echo_type: "epg_fisp"
 * or "epg_sr"; nstates <= 256. */
int snapmrf_epg_jvp(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                    size_t NREPS, size_t natoms, int nstates, const char *echo_type, float *d_out,
                    void *stream);

/* Cramer-Rao bound of (T1, T2) and its gradient with respect to the flip-angle
 * schedule, for designing schedules.  No counterpart in the reference.
 *
 * For each tissue i (d_params row: T1, T2, B0, B1; real FISP / SR recursion
 * with flip angle alpha_t * B1, every RF phase 0) the signal s = i f and its
 * tangents f1 = df/dT1, f2 = df/dT2 give the Fisher matrix M = V^T V of
 * V = [f1, f2, f] (unit noise variance, a real proton-density factor as the
 * nuisance parameter) and
 *   d_loss[i] = [M^-1]_00 / T1^2 + [M^-1]_11 / T2^2,
 * the normalised CRBs of T1 and T2 (NaN when M is singular).
 * d_grad_alpha (out [nreps]) = d(sum_i d_loss[i]) / d alpha_t, by reverse
 * mode through the recursion and its tangents, with states kept every
 * checkpoint_every steps (0: ceil(sqrt(nreps))).
 * d_signals (optional out [ntissues][3][nreps]): f, f1, f2. */
int snapmrf_crb_gradient(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                         size_t NREPS, size_t ntissues, int nstates, const char *echo_type,
                         float *d_loss, float *d_grad_alpha, float *d_signals, int checkpoint_every,
                         void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SNAPMRF_H */
