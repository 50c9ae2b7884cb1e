// Dictionary generation on sm_100a: extended-phase-graph recursion for the
// SSFP / SR / SE / TSE / FISP echo types and single- or multi-isochromat ROA
// Bloch simulation.  Replaces MRF_dict and the per-operator kernels of the
// reference (src/functions.cu:416-1315).
//
// Design: the reference launches ~14 kernels and a cuBLAS handle per time
// step over a global [atom][state][3] state array.  Here one launch runs the
// whole recursion: an atom's EPG state lives in the registers of a group of
// L lanes (S states per lane), the F-state shift is a shuffle between
// neighbouring lanes, per-step constants (RF transition matrix, relaxation
// and precession factors) are staged in shared memory per chunk of time
// steps, and the readout is staged in shared memory and written coalesced.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.h"
#include "epg_kernels.cuh"

namespace snapmrf {

// ---------------------------------------------------------------------------
// Schedule preparation
// ---------------------------------------------------------------------------

// Per-block flip angles.  epg_ssfp scales the flip-angle row in place by the
// block's B1 and back by 1/B1 after the block (src/functions.cu:969-973,
// 1011-1013); that float round trip is reproduced so block j sees exactly the
// reference's angles.  Other echo types use the converted angle, times b1
// when every block is generated (the B1 extension).
__global__ void prepare_alpha_kernel(float *alpha, const float *fa, const float *params,
                                     int nparams, long long nreps, long long natoms,
                                     long long nblocks, int mode) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nreps) return;
    float v = fa[t];
    for (long long j = 0; j < nblocks; j++) {
        float b1 = params[j * natoms * nparams + 3];
        if (mode == 0) {            // SSFP drift
            v *= b1;
            alpha[j * nreps + t] = v;
            float inv = 1.f / b1;
            v *= inv;
        } else if (mode == 1) {     // alpha * b1
            alpha[j * nreps + t] = fa[t] * b1;
        } else {                    // unscaled
            alpha[j * nreps + t] = fa[t];
        }
    }
}

// The 16-bit matching operand of the unit-norm atoms
// (SNAPMRF_DICT_NORMALIZE_OPERAND), after the recursion: row a is
// Im(atom a) * (1 / norm a), the product the recursion's kernel forms when
// it normalises, rounded once to the operand's type, and zeros up to the
// row pitch.  A pass of its own reads every finished atom at the full
// bandwidth, where reading each atom back at the end of its own recursion
// waited on one row at a time.  One warp per row (grid-stride over rows),
// lanes over samples; norms as the recursion wrote them (sqrt of the sum of
// squares).
__global__ void pack_operand_kernel(EpgArgs a, long long natoms_total) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    // eight samples per lane and step: four 16-byte loads of the atom row and
    // one 16-byte store of the operand where the row allows it
    const bool vec = a.nreps % (a.imag_rows ? 4 : 2) == 0 && reinterpret_cast<uintptr_t>(a.atoms) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(a.packed) % 16 == 0 && a.packed_pitch % 8 == 0;
    const long long groups = (a.packed_pitch + 7) / 8;
    for (long long at = blockIdx.x * (long long)(blockDim.x / 32) + (threadIdx.x >> 5); at < natoms_total;
         at += warps) {
        float inv = a.norms[at];
        if (inv > 0.f) inv = 1.f / inv;
        const float2 *row = a.atoms + at * a.nreps;
        const float *irow = reinterpret_cast<const float *>(a.atoms) + at * a.nreps;  // (imaginary rows)
        for (long long gq = lane; gq < groups; gq += 32) {
            const long long q0 = gq * 8;
            float v[8];
            if (vec && q0 + 8 <= a.nreps) {
                if (a.imag_rows) {
                    const float4 *r4 = reinterpret_cast<const float4 *>(irow + q0);
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                        const float4 x = __ldg(r4 + k);
                        v[4 * k] = x.x * inv;
                        v[4 * k + 1] = x.y * inv;
                        v[4 * k + 2] = x.z * inv;
                        v[4 * k + 3] = x.w * inv;
                    }
                } else {
                    const float4 *r4 = reinterpret_cast<const float4 *>(row + q0);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float4 x = __ldg(r4 + k);
                        v[2 * k] = c_scale(make_float2(x.x, x.y), inv).y;
                        v[2 * k + 1] = c_scale(make_float2(x.z, x.w), inv).y;
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++)
                    v[k] = q0 + k >= a.nreps ? 0.f : a.imag_rows ? irow[q0 + k] * inv : c_scale(row[q0 + k], inv).y;
            }
            if (vec) {
                uint4 w;
                uint32_t *wp = reinterpret_cast<uint32_t *>(&w);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (a.packed_half) {
                        const __half2 h = __floats2half2_rn(v[2 * k], v[2 * k + 1]);
                        wp[k] = *reinterpret_cast<const uint32_t *>(&h);
                    } else {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
                        wp[k] = *reinterpret_cast<const uint32_t *>(&h);
                    }
                }
                reinterpret_cast<uint4 *>(static_cast<unsigned char *>(a.packed) +
                                          (at * a.packed_pitch + q0) * 2)[0] = w;
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++)
                    if (q0 + k < a.packed_pitch) store_packed(a, at, q0 + k, v[k]);
            }
        }
    }
}

static int parse_echo(const char *s) {
    if (!s) return -1;
    if (!strcmp(s, "epg_ssfp")) return ECHO_SSFP;
    if (!strcmp(s, "roa_ssfp")) return ECHO_ROA;
    if (!strcmp(s, "epg_sr")) return ECHO_SR;
    if (!strcmp(s, "epg_se")) return ECHO_SE;
    if (!strcmp(s, "epg_tse1") || !strcmp(s, "epg_tse2")) return ECHO_TSE;
    if (!strcmp(s, "epg_fisp")) return ECHO_FISP;
    return -1;
}

// Lanes per atom (power of two) and states per lane (<= smax, a multiple of
// `step`) for w states: least padding first, then more states per lane.
static void choose_layout(int w, int smax, int step, int *L, int *S) {
    // SNAPMRF_DICT_LAYOUT="L,S" (lanes per atom, states per lane) overrides
    // the choice when it is a valid layout for w states
    if (const char *e = getenv("SNAPMRF_DICT_LAYOUT")) {
        int l = 0, s = 0;
        if (sscanf(e, "%d,%d", &l, &s) == 2 && l >= 1 && l <= 32 && (l & (l - 1)) == 0 && s >= step &&
            s <= smax && s % step == 0 && l * s >= w) {
            *L = l;
            *S = s;
            return;
        }
    }
    int bestL = 32, bestS = smax, bestPad = 1 << 30;
    for (int s = smax; s >= step; s -= step)
        for (int l = 1; l <= 32; l *= 2)
            if (l * s >= w) {
                int pad = l * s - w;
                if (pad < bestPad) { bestPad = pad; bestL = l; bestS = s; }
                break;
            }
    *L = bestL;
    *S = bestS;
}

template <int ECHO, int S>
static cudaError_t launch_epg_ref(const EpgArgs &a, dim3 grid, cudaStream_t st) {
    size_t smem = epg_ref_smem_bytes(ECHO, a.L);
    auto k = epg_ref_kernel<ECHO, S>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, kEpgThreads, smem, st>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

template <int ECHO>
static cudaError_t dispatch_states(const EpgArgs &a, int S, dim3 grid, cudaStream_t st) {
    switch (S) {
    case 1: return launch_epg_ref<ECHO, 1>(a, grid, st);
    case 2: return launch_epg_ref<ECHO, 2>(a, grid, st);
    case 3: return launch_epg_ref<ECHO, 3>(a, grid, st);
    case 4: return launch_epg_ref<ECHO, 4>(a, grid, st);
    case 5: return launch_epg_ref<ECHO, 5>(a, grid, st);
    case 6: return launch_epg_ref<ECHO, 6>(a, grid, st);
    case 7: return launch_epg_ref<ECHO, 7>(a, grid, st);
    default: return launch_epg_ref<ECHO, 8>(a, grid, st);
    }
}

// Fine-tail plan of the real-valued kernel.  A CTA carries its atoms through
// every step whatever its layout, so a grid of C CTAs on R resident ones
// takes ceil(C / R) rounds, and a last round holding only a few CTAs costs a
// good part of a full one (C1, 41 B1 blocks x 434 CTAs on 1,776 resident:
// the 41 CTAs past 10 rounds add 0.17 ms to 7.04).  When the CTAs past the
// last whole round number at most the blocks (one partial CTA each), or the
// whole grid is smaller than one round, each block's trailing atoms go to
// the fine layout (kFineL lanes per atom, kFineP pairs of states per lane:
// w <= 64), provided its CTAs number at most R / 2.  *bulk_cpb / *fine_cpb:
// CTAs per block of the chosen and the fine layout (*fine_cpb = 0: no
// split).  SNAPMRF_DICT_FINE_ATOMS = n forces n fine atoms per block (rounded
// up to whole CTAs of the chosen layout; 0 turns the split off); an explicit
// SNAPMRF_DICT_LAYOUT turns it off too.
static void plan_fine_tail(const EpgArgs &a, int P, long long nblocks, const void *kernel, size_t smem,
                           long long *bulk_cpb, long long *fine_cpb) {
    const long long apc = kRealThreads / a.L, apc_f = kRealThreads / kFineL;
    const long long n = a.natoms, B = nblocks;
    *bulk_cpb = (n + apc - 1) / apc;
    *fine_cpb = 0;
    if (P <= kFineP || a.nstates > 2 * kFineP * kFineL || kRealThreads % 32 || getenv("SNAPMRF_DICT_LAYOUT"))
        return;
    long long bulk;
    if (const char *e = getenv("SNAPMRF_DICT_FINE_ATOMS")) {
        const long long nf = atoll(e);
        if (nf <= 0) return;
        bulk = nf >= n ? 0 : (n - nf) / apc;
    } else {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kRealThreads, smem) != cudaSuccess ||
            sms <= 0 || per_sm <= 0) {
            cudaGetLastError();
            return;
        }
        const long long R = (long long)sms * per_sm;
        const long long C = B * *bulk_cpb;
        const long long rounds = C / R;
        if (rounds && (C % R == 0 || C % R > B)) return;
        bulk = rounds ? std::min(rounds * R / B, n / apc) : 0;
        if (B * ((n - bulk * apc + apc_f - 1) / apc_f) > R / 2) return;
    }
    if (n - bulk * apc <= 0) return;
    *bulk_cpb = bulk;
    *fine_cpb = (n - bulk * apc + apc_f - 1) / apc_f;
}

template <int ECHO, int S, bool TAIL, bool FOLD>
static cudaError_t launch_epg_real(EpgArgs a, dim3 grid, cudaStream_t st) {
    size_t smem = epg_real_smem_bytes(a.L);
    auto k = epg_real_kernel<ECHO, S, TAIL, FOLD>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    long long bulk_cpb = grid.x, fine_cpb = 0;
    plan_fine_tail(a, S, grid.y, (const void *)k, smem, &bulk_cpb, &fine_cpb);
    if (bulk_cpb > 0) {
        k<<<dim3((unsigned)bulk_cpb, grid.y), kRealThreads, smem, st>>>(a);
        note_launches(1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (fine_cpb == 0) return cudaSuccess;
    // the fine tail, a programmatic dependent of the main grid (see
    // epg_real_fine_kernel)
    a.fine_first = bulk_cpb * (kRealThreads / a.L);
    auto kf = epg_real_fine_kernel<ECHO, FOLD>;
    const size_t smem_f = epg_real_smem_bytes(kFineL);
    if ((e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_f)) != cudaSuccess)
        return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)fine_cpb, grid.y);
    cfg.blockDim = dim3(kRealThreads);
    cfg.dynamicSmemBytes = smem_f;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = bulk_cpb > 0 ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kf, a);
    note_launches(1);
    return e != cudaSuccess ? e : cudaGetLastError();
}

// P = pairs of states per lane (S = 2P).  FISP layouts that pad at most two
// states take the TAIL form of the shift.
template <int ECHO, bool FOLD>
static cudaError_t dispatch_real_p(const EpgArgs &a, int P, dim3 grid, cudaStream_t st) {
    if constexpr (ECHO == ECHO_FISP) {
        if (a.L * 2 * P - a.nstates <= 2) switch (P) {
            case 1: return launch_epg_real<ECHO, 1, true, FOLD>(a, grid, st);
            case 2: return launch_epg_real<ECHO, 2, true, FOLD>(a, grid, st);
            case 3: return launch_epg_real<ECHO, 3, true, FOLD>(a, grid, st);
            case 4: return launch_epg_real<ECHO, 4, true, FOLD>(a, grid, st);
            case 5: return launch_epg_real<ECHO, 5, true, FOLD>(a, grid, st);
            case 6: return launch_epg_real<ECHO, 6, true, FOLD>(a, grid, st);
            case 7: return launch_epg_real<ECHO, 7, true, FOLD>(a, grid, st);
            case 8: return launch_epg_real<ECHO, 8, true, FOLD>(a, grid, st);
            case 9: return launch_epg_real<ECHO, 9, true, FOLD>(a, grid, st);
            case 10: return launch_epg_real<ECHO, 10, true, FOLD>(a, grid, st);
            case 11: return launch_epg_real<ECHO, 11, true, FOLD>(a, grid, st);
            case 12: return launch_epg_real<ECHO, 12, true, FOLD>(a, grid, st);
            case 13: return launch_epg_real<ECHO, 13, true, FOLD>(a, grid, st);
            case 14: return launch_epg_real<ECHO, 14, true, FOLD>(a, grid, st);
            case 15: return launch_epg_real<ECHO, 15, true, FOLD>(a, grid, st);
            default: return launch_epg_real<ECHO, 16, true, FOLD>(a, grid, st);
            }
    }
    switch (P) {
    case 1: return launch_epg_real<ECHO, 1, false, FOLD>(a, grid, st);
    case 2: return launch_epg_real<ECHO, 2, false, FOLD>(a, grid, st);
    case 3: return launch_epg_real<ECHO, 3, false, FOLD>(a, grid, st);
    case 4: return launch_epg_real<ECHO, 4, false, FOLD>(a, grid, st);
    case 5: return launch_epg_real<ECHO, 5, false, FOLD>(a, grid, st);
    case 6: return launch_epg_real<ECHO, 6, false, FOLD>(a, grid, st);
    case 7: return launch_epg_real<ECHO, 7, false, FOLD>(a, grid, st);
    case 8: return launch_epg_real<ECHO, 8, false, FOLD>(a, grid, st);
    case 9: return launch_epg_real<ECHO, 9, false, FOLD>(a, grid, st);
    case 10: return launch_epg_real<ECHO, 10, false, FOLD>(a, grid, st);
    case 11: return launch_epg_real<ECHO, 11, false, FOLD>(a, grid, st);
    case 12: return launch_epg_real<ECHO, 12, false, FOLD>(a, grid, st);
    case 13: return launch_epg_real<ECHO, 13, false, FOLD>(a, grid, st);
    case 14: return launch_epg_real<ECHO, 14, false, FOLD>(a, grid, st);
    case 15: return launch_epg_real<ECHO, 15, false, FOLD>(a, grid, st);
    default: return launch_epg_real<ECHO, 16, false, FOLD>(a, grid, st);
    }
}

template <int ECHO>
static cudaError_t dispatch_real(const EpgArgs &a, int P, bool fold, dim3 grid, cudaStream_t st) {
    return fold ? dispatch_real_p<ECHO, true>(a, P, grid, st) : dispatch_real_p<ECHO, false>(a, P, grid, st);
}

static cudaError_t launch_epg(int echo, const EpgArgs &a, int S, dim3 grid, cudaStream_t st) {
    switch (echo) {
    case ECHO_SSFP: return dispatch_states<ECHO_SSFP>(a, S, grid, st);
    case ECHO_SR: return dispatch_states<ECHO_SR>(a, S, grid, st);
    case ECHO_SE: return dispatch_states<ECHO_SE>(a, S, grid, st);
    case ECHO_TSE: return dispatch_states<ECHO_TSE>(a, S, grid, st);
    default: return dispatch_states<ECHO_FISP>(a, S, grid, st);
    }
}

}  // namespace snapmrf

using namespace snapmrf;

// MRF_dict and the engine-level entry point.  convert: apply MRF_dict's
// schedule conversion for epg_ssfp / roa_ssfp (the engines take the
// converted schedule); ti: epg_ssfp's inversion delay; engine: normalise only
// on request (MRF_dict normalises the epg_ssfp / roa_ssfp atoms after the
// engine has run, src/functions.cu:1268, 1297).
static int dict_impl(float *d_atoms, const float *d_params, const float *h_mrf, size_t nreps, size_t NREPS,
                     size_t NATOMS, size_t natoms, int nparams, int nstates, const char *echo_type,
                     const snapmrf_dict_opts *opts, void *stream, bool convert, float ti, bool engine) {
    cudaStream_t st = (cudaStream_t)stream;
    int echo = parse_echo(echo_type);
    if (echo < 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_ECHO_TYPE, "Please put in correct echo types (got '%s')",
                     echo_type ? echo_type : "(null)");
    if (!d_atoms || !d_params || !h_mrf) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: null pointer");
    if (nparams < 4) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: nparams must be >= 4");
    if (nreps == 0 || nreps > NREPS)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: need 0 < nreps <= NREPS (%zu, %zu)", nreps, NREPS);
    if (natoms == 0 || NATOMS % natoms != 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: NATOMS (%zu) must be a multiple of natoms (%zu)",
                     NATOMS, natoms);
    if (nstates < 1 || nstates > 32 * kMaxRealStatesPerLane)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: nstates must be in [1, %d]", 32 * kMaxRealStatesPerLane);
    unsigned flags = opts ? opts->flags : 0u;
    int n_iso = opts ? opts->n_iso : 1;
    if (n_iso < 1) n_iso = 1;
    if (n_iso > 1 && echo != ECHO_ROA)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: n_iso > 1 applies to roa_ssfp only");
    float *d_norms = opts ? opts->d_norms : nullptr;
    if (natoms > (size_t)(65535ull * 1024ull * 1024ull))
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: too many atoms per block");

    const size_t nblocks = NATOMS / natoms;
    if (nblocks > 65535) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: more than 65535 B1 blocks");
    const bool all_blocks = (echo == ECHO_SSFP) || (flags & SNAPMRF_DICT_ALL_B1_BLOCKS);
    const size_t gen_blocks = all_blocks ? nblocks : 1;
    const bool normalize = (!engine && (echo == ECHO_SSFP || echo == ECHO_ROA)) || (flags & SNAPMRF_DICT_NORMALIZE);
    const bool pack_normalized = (flags & SNAPMRF_DICT_NORMALIZE_OPERAND) != 0;
    if (pack_normalized && (normalize || !(opts && opts->d_packed)))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID,
                     "MRF_dict: SNAPMRF_DICT_NORMALIZE_OPERAND needs d_packed and atoms that are not normalised "
                     "(no SNAPMRF_DICT_NORMALIZE; not epg_ssfp / roa_ssfp)");

    // Converted schedule (MRF_dict, src/functions.cu:1229-1291): SSFP and ROA
    // take the CSV's flip fraction of 60 deg, phase in degrees and TR/TE
    // extensions of 16 / 3.5 ms; the other echo types use the values raw.
    std::vector<float> sched(4 * nreps);
    for (int r = 0; r < 4; r++)
        for (size_t t = 0; t < nreps; t++) sched[r * nreps + t] = h_mrf[r * NREPS + t];
    if (convert && (echo == ECHO_SSFP || echo == ECHO_ROA)) {
        const float nominal_flip = 60.f, TR_base = 16.f, TE_base = 3.5f;
        const float fa_scale = (float)(nominal_flip * M_PI / 180.f);
        const float ph_scale = (float)(M_PI / 180.f);
        for (size_t t = 0; t < nreps; t++) {
            sched[t] *= fa_scale;
            sched[nreps + t] *= ph_scale;
            sched[2 * nreps + t] += TR_base;
            sched[3 * nreps + t] += TE_base;
        }
    }

    DeviceScratch scratch;
    SNAPMRF_CUDA(scratch.alloc((4 * nreps + gen_blocks * nreps) * sizeof(float), st));
    float *d_sched = scratch.as<float>();
    float *d_alpha = d_sched + 4 * nreps;
    float *h_stage = static_cast<float *>(stage_acquire(4 * nreps * sizeof(float)));
    if (!h_stage) SNAPMRF_FAIL(SNAPMRF_ERR_ALLOC, "MRF_dict: cannot allocate a pinned staging buffer");
    memcpy(h_stage, sched.data(), 4 * nreps * sizeof(float));
    SNAPMRF_CUDA(stage_upload(d_sched, h_stage, 4 * nreps * sizeof(float), st));
    SNAPMRF_CUDA(stage_release(st));
    int mode = (echo == ECHO_SSFP) ? 0 : (all_blocks ? 1 : 2);
    prepare_alpha_kernel<<<(unsigned)((nreps + 255) / 256), 256, 0, st>>>(
        d_alpha, d_sched, d_params, nparams, (long long)nreps, (long long)natoms,
        (long long)gen_blocks, mode);
    SNAPMRF_LAUNCH_CHECK();

    EpgArgs a;
    a.atoms = reinterpret_cast<float2 *>(d_atoms);
    a.norms = d_norms;
    a.alpha = d_alpha;
    a.sched = d_sched;
    a.params = d_params;
    a.nparams = nparams;
    a.nreps = (long long)nreps;
    a.natoms = (long long)natoms;
    a.nstates = nstates;
    a.own_params = (echo == ECHO_SSFP) ? 0 : 1;
    a.normalize = normalize ? 1 : 0;
    a.n_iso = n_iso;
    // init_rf_pulse arguments per engine (src/functions.cu:697, 753, 821, 890,
    // 965-966, 1175): SSFP 180 deg with TI 40 ms, SE/TSE 90/90, ROA 180,
    // FISP/SR no pulse
    a.init_alpha_deg = (echo == ECHO_SSFP || echo == ECHO_ROA) ? 180.f
                       : (echo == ECHO_SE || echo == ECHO_TSE) ? 90.f : 0.f;
    a.init_phi_deg = (echo == ECHO_SE || echo == ECHO_TSE) ? 90.f : 0.f;
    a.init_ti = (echo == ECHO_SSFP) ? ti : 0.f;
    a.packed = nullptr;
    a.packed_half = 0;
    a.packed_pitch = 0;
    a.fine_first = 0;
    a.pack_normalized = pack_normalized ? 1 : 0;
    a.operand_pass = 0;
    a.imag_rows = (flags & SNAPMRF_DICT_IMAG_ROWS) ? 1 : 0;
    void *d_packed = opts ? opts->d_packed : nullptr;

    if (echo == ECHO_ROA) {
        if (a.imag_rows)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                         "MRF_dict: SNAPMRF_DICT_IMAG_ROWS needs epg_fisp / epg_sr with every RF phase 0");
        if (d_packed)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: d_packed needs epg_fisp / epg_sr with every RF phase 0");
        if (n_iso > 32 * 8) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: n_iso must be <= 256");
        a.L = 1;
        SNAPMRF_CUDA(launch_roa(a, (long long)natoms, (unsigned)gen_blocks, st));
        return SNAPMRF_OK;
    }
    // Real-valued recursion (bit-identical, half the state) when every RF
    // phase is exactly 0 and the echo type has no off-resonance term.
    bool real_path = !(flags & SNAPMRF_DICT_REFERENCE_ORDER) && (echo == ECHO_FISP || echo == ECHO_SR) &&
                     nstates <= 32 * kMaxRealStatesPerLane;
    for (size_t t = 0; real_path && t < nreps; t++)
        if (sched[nreps + t] != 0.f) real_path = false;
    if (!real_path && nstates > 32 * kMaxStatesPerLane)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                     "MRF_dict: nstates must be in [1, %d] for this echo type and schedule "
                     "(up to %d for epg_fisp / epg_sr with all RF phases 0)",
                     32 * kMaxStatesPerLane, 32 * kMaxRealStatesPerLane);
    if (a.imag_rows && !real_path)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                     "MRF_dict: SNAPMRF_DICT_IMAG_ROWS needs epg_fisp / epg_sr with every RF phase 0 "
                     "(purely imaginary atoms)");
    if (d_packed) {
        if (!real_path)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED,
                         "MRF_dict: d_packed needs epg_fisp / epg_sr with every RF phase 0 (purely imaginary atoms)");
        if (opts->packed_precision != SNAPMRF_PREC_BF16 && opts->packed_precision != SNAPMRF_PREC_FP16)
            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "MRF_dict: packed_precision must be SNAPMRF_PREC_BF16 or _FP16");
        a.packed = d_packed;
        a.packed_half = opts->packed_precision == SNAPMRF_PREC_FP16 ? 1 : 0;
        a.packed_pitch = (long long)snapmrf_packed_pitch(nreps);
    }
    int L, S;
    if (real_path)
        choose_layout(nstates, kMaxRealStatesPerLane, 2, &L, &S);
    else
        choose_layout(nstates, kMaxStatesPerLane, 1, &L, &S);
    a.L = L;
    const int apc = (real_path ? kRealThreads : kEpgThreads) / L;
    dim3 grid((unsigned)((natoms + apc - 1) / apc), (unsigned)gen_blocks);
    if (grid.x > 0x7fffffffu) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "MRF_dict: grid too large");
    if (real_path) {
        const bool fold = !(flags & SNAPMRF_DICT_SEPARATE_RELAX);
        // the unit-norm operand by a pass of its own over the finished atoms
        // (norms in scratch when the caller wants none)
        DeviceScratch norm_scratch;
        if (pack_normalized) {
            a.operand_pass = 1;
            if (!a.norms) {
                SNAPMRF_CUDA(norm_scratch.alloc((size_t)gen_blocks * natoms * sizeof(float), st));
                a.norms = norm_scratch.as<float>();
            }
        }
        SNAPMRF_CUDA(echo == ECHO_FISP ? dispatch_real<ECHO_FISP>(a, S / 2, fold, grid, st)
                                       : dispatch_real<ECHO_SR>(a, S / 2, fold, grid, st));
        if (pack_normalized) {
            int dev = 0, sms = 0;
            SNAPMRF_CUDA(cudaGetDevice(&dev));
            SNAPMRF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const long long total = (long long)gen_blocks * (long long)natoms;
            const long long blocks = std::min<long long>((total + 7) / 8, (long long)sms * 16);
            pack_operand_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, total);
            SNAPMRF_LAUNCH_CHECK();
        }
    } else {
        SNAPMRF_CUDA(launch_epg(echo, a, S, grid, st));
    }
    return SNAPMRF_OK;
}

extern "C" int snapmrf_mrf_dict(float *d_atoms, const float *d_params, const float *h_mrf,
                                size_t nreps, size_t NREPS, size_t NATOMS, size_t natoms,
                                int nparams, int nstates, const char *echo_type,
                                const snapmrf_dict_opts *opts, void *stream) {
    return dict_impl(d_atoms, d_params, h_mrf, nreps, NREPS, NATOMS, natoms, nparams, nstates, echo_type, opts,
                     stream, true, 40.f, false);
}

extern "C" int snapmrf_dict_engine(float *d_atoms, const float *d_params, const float *d_mrf, float ti,
                                   size_t nreps, size_t NATOMS, size_t natoms, int nparams, int nstates,
                                   const char *echo_type, const snapmrf_dict_opts *opts, void *stream) {
    if (!d_mrf || nreps == 0) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "dict_engine: null schedule or nreps 0");
    if (!(ti >= 0.f)) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "dict_engine: TI must be >= 0");
    // the schedule comes back to the host once: the real-valued recursion is
    // chosen from its RF phases, and the kernels take it staged per call
    std::vector<float> h(4 * nreps);
    cudaStream_t st = (cudaStream_t)stream;
    SNAPMRF_CUDA(cudaMemcpyAsync(h.data(), d_mrf, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    SNAPMRF_CUDA(cudaStreamSynchronize(st));
    return dict_impl(d_atoms, d_params, h.data(), nreps, nreps, NATOMS, natoms, nparams, nstates, echo_type, opts,
                     stream, false, ti, true);
}

namespace snapmrf {

// normalize (src/functions.cu:670-685): a / ||a||_2 when ||a|| > 0, one warp
// per atom (the sum is a lane-strided tree instead of the reference's serial
// loop, so it differs from it by rounding only).
__global__ void normalize_kernel(float2 *atoms, float *norms, long long nreps, long long natoms) {
    long long a = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    int lane = threadIdx.x % 32;
    if (a >= natoms) return;
    float2 *p = atoms + a * nreps;
    float s = 0.f;
    for (long long t = lane; t < nreps; t += 32) s += p[t].x * p[t].x + p[t].y * p[t].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (norms && lane == 0) norms[a] = sqrtf(s);
    float inv = s;
    if (inv > 0.f) inv = 1.f / sqrtf(inv);
    for (long long t = lane; t < nreps; t += 32) p[t] = c_scale(p[t], inv);
}

}  // namespace snapmrf

extern "C" size_t snapmrf_packed_pitch(size_t nreps) { return (nreps + 63) / 64 * 64; }

extern "C" int snapmrf_normalize(float *d_atoms, size_t nreps, size_t NATOMS, float *d_norms,
                                 void *stream) {
    if (!d_atoms) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "normalize: null pointer");
    if (nreps == 0 || NATOMS == 0) return SNAPMRF_OK;
    long long threads = (long long)NATOMS * 32;
    snapmrf::normalize_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(d_atoms), d_norms, (long long)nreps, (long long)NATOMS);
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}
