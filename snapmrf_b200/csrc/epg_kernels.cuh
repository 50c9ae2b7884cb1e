// EPG / ROA device kernels (reference operation order).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cuda_runtime.h>

#include "common.h"

namespace snapmrf {

enum Echo { ECHO_SSFP = 0, ECHO_ROA = 1, ECHO_SR = 2, ECHO_SE = 3, ECHO_TSE = 4, ECHO_FISP = 5 };

constexpr int kEpgThreads = 128;      // threads per CTA
constexpr int kChunk = 16;            // time steps staged per shared-memory chunk (<= 32)
constexpr int kMaxStatesPerLane = 8;  // register-resident EPG states per lane

struct EpgArgs {
    float2 *atoms;        // out [blocks][natoms][nreps]
    float *norms;         // optional out [blocks][natoms]
    const float *alpha;   // [gen_blocks][nreps] flip angle per block (rad)
    const float *sched;   // [4][nreps] converted schedule (alpha, phi rad; TR, TE ms)
    const float *params;  // [NATOMS][nparams]
    int nparams;
    long long nreps;
    long long natoms;     // atoms per B1 block
    int nstates;          // EPG states w
    int L;                // lanes per atom (power of two)
    int own_params;       // 1: each atom's own row; 0: block-0 row (epg_ssfp)
    int normalize;        // unit-norm each atom (src/functions.cu:670-685)
    int n_iso;            // ROA isochromats
    // initial pulse (init_rf_pulse): angles in degrees, TI in ms.  Passed at
    // run time like the reference's kernel arguments, so that __sincosf is
    // evaluated on the device rather than folded at compile time.
    float init_alpha_deg, init_phi_deg, init_ti;
    // optional 16-bit copy of Im(atom), [blocks][natoms][packed_pitch]
    void *packed;
    int packed_half;      // 1: fp16, 0: bf16
    long long packed_pitch;
    // first atom of each B1 block in the fine tail of the real-valued kernel
    long long fine_first;
    // 16-bit operand of the unit-norm atoms while the atoms stay as generated
    int pack_normalized;
    // 1: that operand is written by a separate pass over the finished atoms
    // and their norms (pack_operand_kernel), not by the recursion's kernel
    int operand_pass;
    // 1: atoms written as Im rows, [blocks][natoms][nreps] float (the
    // real-valued recursion only; its atoms are purely imaginary)
    int imag_rows;
};

// Number of per-(atom, step) factors staged: E1/E2 at TE and at TR-TE, plus
// the B0 precession phasors at TE and TR-TE for SSFP.
__host__ __device__ constexpr int epg_nf(int echo) { return echo == ECHO_SSFP ? 8 : 4; }

// Per-group strides in shared memory, padded so that the groups of a warp
// hit different banks.
__host__ __device__ constexpr int epg_f_stride(int echo) { return kChunk * epg_nf(echo) + 4; }
constexpr int kReadoutStride = kChunk + 1;  // float2 per group

inline size_t epg_ref_smem_bytes(int echo, int L) {
    int apc = kEpgThreads / L;
    return (size_t)kChunk * 9 * sizeof(float2) + (size_t)apc * epg_f_stride(echo) * sizeof(float) +
           (size_t)apc * kReadoutStride * sizeof(float2) + (size_t)apc * 3 * sizeof(float);
}

// RF transition matrix of fill_transition_matrix (src/functions.cu:483-508),
// same float2 expressions; T[3r + l] multiplies state channel l into row r.
__device__ __forceinline__ void rf_matrix(float alpha, float phi, float2 *T) {
    float sa, ca;
    __sincosf(alpha, &sa, &ca);
    float sa2 = (1 - ca) / 2;
    float ca2 = (1 + ca) / 2;
    float sp, cp;
    __sincosf(phi, &sp, &cp);
    float2 z = make_float2(cp, sp);
    float2 zinv = c_conj(z);
    const float2 im = make_float2(0.f, 1.f);
    const float2 mim = make_float2(-im.x, -im.y);
    T[0] = make_float2(ca2, 0.f);
    T[3] = c_mul(c_scale(zinv, sa2), zinv);
    T[6] = c_mul(c_scale(c_scale(mim, 0.5f), sa), zinv);
    T[1] = c_scale(c_mul(z, z), sa2);
    T[4] = make_float2(ca2, 0.f);
    T[7] = c_scale(c_mul(c_scale(im, 0.5f), z), sa);
    T[2] = c_scale(c_mul(mim, z), sa);
    T[5] = c_mul(c_scale(im, sa), zinv);
    T[8] = make_float2(ca, 0.f);
}

// One output row of the 3x3 complex RF product, accumulated with FMAs over
// the three state channels (the in-place cublasCgemm of
// src/functions.cu:510-528).
__device__ __forceinline__ float2 rf_row(float2 a0, float2 a1, float2 a2, float2 o0, float2 o1,
                                         float2 o2) {
    float rx = a0.x * o0.x;
    rx = fmaf(-a0.y, o0.y, rx);
    rx = fmaf(a1.x, o1.x, rx);
    rx = fmaf(-a1.y, o1.y, rx);
    rx = fmaf(a2.x, o2.x, rx);
    rx = fmaf(-a2.y, o2.y, rx);
    float ry = a0.x * o0.y;
    ry = fmaf(a0.y, o0.x, ry);
    ry = fmaf(a1.x, o1.y, ry);
    ry = fmaf(a1.y, o1.x, ry);
    ry = fmaf(a2.x, o2.y, ry);
    ry = fmaf(a2.y, o2.x, ry);
    return make_float2(rx, ry);
}

// Register-resident EPG state of one lane: states k = gl*S + j.
template <int S>
struct LaneState {
    float2 fp[S], fm[S], zz[S];
};

template <int S>
__device__ __forceinline__ void st_rf(LaneState<S> &s, const float2 *T) {
    float2 t0 = T[0], t1 = T[1], t2 = T[2], t3 = T[3], t4 = T[4], t5 = T[5], t6 = T[6], t7 = T[7],
           t8 = T[8];
#pragma unroll
    for (int j = 0; j < S; j++) {
        float2 o0 = s.fp[j], o1 = s.fm[j], o2 = s.zz[j];
        s.fp[j] = rf_row(t0, t1, t2, o0, o1, o2);
        s.fm[j] = rf_row(t3, t4, t5, o0, o1, o2);
        s.zz[j] = rf_row(t6, t7, t8, o0, o1, o2);
    }
}

// decay_signal_stage1/2 (src/functions.cu:544-569): F+- *= E2, Z *= E1, then
// Z0 += 1 - E1 as a separate rounding.
template <int S>
__device__ __forceinline__ void st_relax(LaneState<S> &s, float E1, float E2, bool lane0) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        s.fp[j] = c_scale(s.fp[j], E2);
        s.fm[j] = c_scale(s.fm[j], E2);
        s.zz[j] = c_scale(s.zz[j], E1);
    }
    if (lane0) s.zz[0].x = __fadd_rn(s.zz[0].x, 1 - E1);
}

// shift_phase (EPG, src/functions.cu:585-607): F+ *= e, F- *= conj(e).
template <int S>
__device__ __forceinline__ void st_b0(LaneState<S> &s, float2 e) {
    float2 ec = c_conj(e);
#pragma unroll
    for (int j = 0; j < S; j++) {
        s.fp[j] = c_mul(e, s.fp[j]);
        s.fm[j] = c_mul(ec, s.fm[j]);
    }
}

// dephase_gradients (src/functions.cu:619-668): F+[k] <- F+[k-1] for
// k = w-1..1, F-[k] <- F-[k+1] for k = 0..w-2 (F-[w-1] keeps its value), then
// F+[0] = conj(F-[0]) and F-[w-1] = 0.  With w = 1 nothing shifts and F+[0]
// takes the conjugate of the unshifted F-[0].  Slots k >= w are kept zero.
template <int S>
__device__ __forceinline__ void st_shift(LaneState<S> &s, int gl, int L, int w) {
    const unsigned full = 0xffffffffu;
    float2 top = s.fp[S - 1];
    float2 up;
    up.x = __shfl_up_sync(full, top.x, 1, L);
    up.y = __shfl_up_sync(full, top.y, 1, L);
    float2 bot = s.fm[0];
    float2 dn;
    dn.x = __shfl_down_sync(full, bot.x, 1, L);
    dn.y = __shfl_down_sync(full, bot.y, 1, L);
#pragma unroll
    for (int j = S - 1; j >= 1; j--) s.fp[j] = s.fp[j - 1];
    s.fp[0] = up;
#pragma unroll
    for (int j = 0; j < S; j++) {
        const int k = gl * S + j;
        float2 nxt = (j < S - 1) ? s.fm[j + 1] : ((gl == L - 1) ? make_float2(0.f, 0.f) : dn);
        if (k != w - 1) s.fm[j] = nxt;
    }
    if (gl == 0) s.fp[0] = c_conj(s.fm[0]);
#pragma unroll
    for (int j = 0; j < S; j++) {
        const int k = gl * S + j;
        if (k >= w) s.fp[j] = make_float2(0.f, 0.f);
        if (k == w - 1) s.fm[j] = make_float2(0.f, 0.f);
    }
}

// init_rf_pulse (EPG, src/functions.cu:456-481) into state 0.
template <int S>
__device__ __forceinline__ void st_init(LaneState<S> &s, bool lane0, float t1, float t2,
                                        float alpha_deg, float phi_deg, float TI) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        s.fp[j] = make_float2(0.f, 0.f);
        s.fm[j] = make_float2(0.f, 0.f);
        s.zz[j] = make_float2(0.f, 0.f);
    }
    float alpha = (float)(alpha_deg * M_PI / 180.f);
    float phi = (float)(phi_deg * M_PI / 180.f);
    float e1 = expf(-TI / t1);
    float e2 = expf(-TI / t2);
    float sa, ca, sph, cph;
    __sincosf(alpha, &sa, &ca);
    __sincosf(phi, &sph, &cph);
    float2 tmp2 = c_scale(make_float2(sph, cph), e2 * sa);
    if (lane0) {
        s.fp[0] = c_conj(tmp2);
        s.fm[0] = tmp2;
        s.zz[0] = make_float2(e1 * ca + 1 - e1, 0.f);
    }
}

// B0 phase of shift_phase: cexpf(2*pi*B0*t/1000) with the argument
// evaluated in double like the reference expression.
__device__ __forceinline__ float2 b0_phasor(float B0, float t) {
    float th = (float)(2 * M_PI * B0 * t / 1000.f);
    float s, c;
    __sincosf(th, &s, &c);
    return make_float2(c, s);
}

// The fused EPG recursion, reference operation order.  One CTA handles
// kEpgThreads / L atoms of one B1 block (blockIdx.y).
template <int ECHO, int S>
__global__ void __launch_bounds__(kEpgThreads) epg_ref_kernel(EpgArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NF = epg_nf(ECHO);
    const int L = a.L;
    const int apc = kEpgThreads / L;
    const int tid = threadIdx.x;
    const int g = tid / L;
    const int gl = tid % L;
    const bool lane0 = (gl == 0);
    const long long blk = blockIdx.y;
    const long long nreps = a.nreps;
    const long long atom0 = (long long)blockIdx.x * apc;
    const long long ab = atom0 + g;
    const bool active = ab < a.natoms;
    const long long gatom = blk * a.natoms + ab;

    constexpr int FS = epg_f_stride(ECHO);
    float2 *sT = reinterpret_cast<float2 *>(smem_raw);
    float *sF = reinterpret_cast<float *>(sT + kChunk * 9);
    float2 *sR = reinterpret_cast<float2 *>(sF + apc * FS);
    float *sP = reinterpret_cast<float *>(sR + apc * kReadoutStride);

    for (int i = tid; i < apc; i += kEpgThreads) {
        long long at = atom0 + i;
        float t1 = 1.f, t2 = 1.f, b0 = 0.f;
        if (at < a.natoms) {
            long long row = a.own_params ? blk * a.natoms + at : at;
            const float *p = a.params + row * a.nparams;
            t1 = p[0];
            t2 = p[1];
            b0 = p[2];
        }
        sP[3 * i] = t1;
        sP[3 * i + 1] = t2;
        sP[3 * i + 2] = b0;
    }
    __syncthreads();
    const float T1 = sP[3 * g], T2 = sP[3 * g + 1];

    const float *alpha = a.alpha + blk * nreps;
    const float *phi = a.sched + nreps;
    const float *TR = a.sched + 2 * nreps;
    const float *TE = a.sched + 3 * nreps;
    const int w = a.nstates;

    LaneState<S> s;
    st_init<S>(s, lane0, T1, T2, a.init_alpha_deg, a.init_phi_deg, a.init_ti);
    if (ECHO == ECHO_SE || ECHO == ECHO_TSE) {
        st_shift<S>(s, gl, L, w);
        float te0 = TE[0];
        st_relax<S>(s, expf(-te0 / T1), expf(-te0 / T2), lane0);
    }

    float nrm = 0.f;
    float2 *out = a.atoms + gatom * nreps;
    for (long long t0 = 0; t0 < nreps; t0 += kChunk) {
        const int nch = (int)min((long long)kChunk, nreps - t0);
        __syncthreads();
        for (int i = tid; i < nch; i += kEpgThreads) rf_matrix(alpha[t0 + i], phi[t0 + i], sT + 9 * i);
        for (int idx = tid; idx < apc * nch; idx += kEpgThreads) {
            int ga = idx / nch, i = idx - ga * nch;
            float t1 = sP[3 * ga], t2 = sP[3 * ga + 1];
            float tr = TR[t0 + i], te = TE[t0 + i];
            float ta = te, tb = tr - te;
            float *f = sF + ga * FS + i * NF;
            f[0] = expf(-ta / t1);
            f[1] = expf(-ta / t2);
            f[2] = expf(-tb / t1);
            f[3] = expf(-tb / t2);
            if (ECHO == ECHO_SSFP) {
                float b0 = sP[3 * ga + 2];
                float2 ea = b0_phasor(b0, ta), eb = b0_phasor(b0, tb);
                f[4] = ea.x;
                f[5] = ea.y;
                f[6] = eb.x;
                f[7] = eb.y;
            }
        }
        __syncthreads();
        for (int i = 0; i < nch; i++) {
            const float *f = sF + g * FS + i * NF;
            st_rf<S>(s, sT + 9 * i);
            if (ECHO == ECHO_SR) {
                st_relax<S>(s, f[0], f[1], lane0);
            } else if (ECHO == ECHO_SE || ECHO == ECHO_TSE) {
                st_shift<S>(s, gl, L, w);
                st_relax<S>(s, f[0], f[1], lane0);
            } else if (ECHO == ECHO_FISP) {
                st_relax<S>(s, f[0], f[1], lane0);
            } else {
                st_relax<S>(s, f[0], f[1], lane0);
                st_b0<S>(s, make_float2(f[4], f[5]));
            }
            if (lane0) {
                float2 v = s.fp[0];
                sR[g * kReadoutStride + i] = v;
                nrm += v.x * v.x + v.y * v.y;
            }
            if (ECHO == ECHO_SR) {
                st_relax<S>(s, f[2], f[3], lane0);
            } else if (ECHO == ECHO_SE || ECHO == ECHO_TSE || ECHO == ECHO_FISP) {
                st_shift<S>(s, gl, L, w);
                st_relax<S>(s, f[2], f[3], lane0);
            } else {
                st_b0<S>(s, make_float2(f[6], f[7]));
                st_shift<S>(s, gl, L, w);
                st_relax<S>(s, f[2], f[3], lane0);
            }
        }
        __syncwarp();
        if (active)
            for (int q = gl; q < nch; q += L) out[t0 + q] = sR[g * kReadoutStride + q];
    }
    if (a.normalize || a.norms) {
        nrm = __shfl_sync(0xffffffffu, nrm, 0, L);
        if (a.norms && lane0 && active) a.norms[gatom] = sqrtf(nrm);
        if (a.normalize) {
            __syncwarp();
            float inv = nrm;
            if (inv > 0.f) inv = 1.f / sqrtf(inv);
            if (active)
                for (long long q = gl; q < nreps; q += L) out[q] = c_scale(out[q], inv);
        }
    }
}

// ---------------------------------------------------------------------------
// Real-valued EPG recursion (FISP / SR with every RF phase exactly 0).
//
// With phi = 0 the transition matrix has real F-rows and imaginary Z-column
// (and the converse for the Z-row), the initial state is Z = 1, and
// relaxation, the shift and conj() preserve the form: F+ and F- stay purely
// imaginary and Z real.  The state is then three floats per EPG state
// (f+ = Im F+, f- = Im F-, z = Re Z) instead of six.  The nine real
// coefficients are the entries of the same complex matrix, and the FMA
// chains below are those of rf_row with the terms whose factors are exact
// zeros removed, so the results are bit-identical to the complex recursion.
// ---------------------------------------------------------------------------
constexpr int kMaxRealStatesPerLane = 32;  // even: states are processed in pairs

// Coefficient pairs (c, c) of the real recursion for one step, in the order
// T0.x, T1.x, T2.y | T3.x, T4.x, T5.y | -T6.y, -T7.y, T8.x (float2 each).
__device__ __forceinline__ void rf_real_coeffs2(float alpha, float phi, float2 *c) {
    float2 T[9];
    rf_matrix(alpha, phi, T);
    const float v[9] = {T[0].x, T[1].x, T[2].y, T[3].x, T[4].x, T[5].y, -T[6].y, -T[7].y, T[8].x};
#pragma unroll
    for (int i = 0; i < 9; i++) c[i] = make_float2(v[i], v[i]);
    c[9] = make_float2(0.f, 0.f);
}

// P pairs of EPG states per lane: slot j = 2i + h of pair i is state
// k = gl * 2P + j.  Packed two-wide FP32 instructions (__ffma2_rn /
// __fmul2_rn) perform per element exactly the scalar operations of the
// complex recursion with its zero terms removed.
template <int P>
struct RealLane2 {
    float2 fp[P], fm[P], zz[P];
};

template <int P>
__device__ __forceinline__ void rl2_rf_k(RealLane2<P> &s, float2 c0, float2 c1, float2 c2, float2 c3, float2 c4,
                                         float2 c5, float2 c6, float2 c7, float2 c8) {
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float2 p = s.fp[i], m = s.fm[i], z = s.zz[i];
        float2 np = __fmul2_rn(c0, p);
        np = __ffma2_rn(c1, m, np);
        np = __ffma2_rn(c2, z, np);
        float2 nm = __fmul2_rn(c3, p);
        nm = __ffma2_rn(c4, m, nm);
        nm = __ffma2_rn(c5, z, nm);
        float2 nz = __fmul2_rn(c6, p);
        nz = __ffma2_rn(c7, m, nz);
        nz = __ffma2_rn(c8, z, nz);
        s.fp[i] = np;
        s.fm[i] = nm;
        s.zz[i] = nz;
    }
}

// The same RF with the structure of a phi = 0 pulse (c3 = c1, c4 = c0,
// c5 = -c2, c7 = -c6, as rf_real_coeffs2 produces them and the folded
// relaxation keeps them): F-' = (c0 + c1)(F+ + F-) - F+' and
// Z' = c6 (F+ - F-) + c8 Z, 8 packed operations per pair instead of 9.  It
// rounds differently from the reference's order (unit-norm C1 atoms move by
// at most 6e-8) and is used by the folded recursion only.
template <int P>
__device__ __forceinline__ void rl2_rf_k8(RealLane2<P> &s, float2 c0, float2 c1, float2 c2, float2 c6, float2 c8) {
    const float2 cs = __fadd2_rn(c0, c1);
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float2 p = s.fp[i], m = s.fm[i], z = s.zz[i];
        float2 np = __fmul2_rn(c0, p);
        np = __ffma2_rn(c1, m, np);
        np = __ffma2_rn(c2, z, np);
        const float2 d = __fadd2_rn(p, make_float2(-m.x, -m.y));
        float2 nz = __fmul2_rn(c6, d);
        nz = __ffma2_rn(c8, z, nz);
        float2 nm = __ffma2_rn(cs, m, make_float2(-np.x, -np.y));
        nm = __ffma2_rn(cs, p, nm);
        s.fp[i] = np;
        s.fm[i] = nm;
        s.zz[i] = nz;
    }
}

template <int P>
__device__ __forceinline__ void rl2_rf(RealLane2<P> &s, const float2 *c) {
    rl2_rf_k<P>(s, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8]);
}

// e = (E2, E1) of one interval: F+- *= E2, Z *= E1, then Z0 += 1 - E1.
template <int P>
__device__ __forceinline__ void rl2_relax(RealLane2<P> &s, float E1, float E2, bool lane0) {
    const float2 e2 = make_float2(E2, E2), e1 = make_float2(E1, E1);
#pragma unroll
    for (int i = 0; i < P; i++) {
        s.fp[i] = __fmul2_rn(s.fp[i], e2);
        s.fm[i] = __fmul2_rn(s.fm[i], e2);
        s.zz[i] = __fmul2_rn(s.zz[i], e1);
    }
    if (lane0) s.zz[0].x = __fadd_rn(s.zz[0].x, 1 - E1);
}

// Gradient shift of the paired real state (see st_shift): F+ up one slot,
// F- down one slot, f+[0] = -f-[0] (Im of conj), F-[w-1] = 0, slots k >= w
// zero; with w = 1 the unshifted f-[0] is used.
//
// TAIL: the layout pads at most two slots (w >= 2P L - 2).  Slots k >= w
// then hold zeros before the shift, so F-[w-1] takes the zero of F-[w] and
// only F+[w], which receives F+[w-1], must be cleared.  That slot lies in the
// last pair of the last lane, and tail_keep (0 there, 1 elsewhere) clears it
// with one multiply instead of a compare per slot; every non-zero value is
// the same as with the per-slot masks.
template <int P, bool TAIL = false>
__device__ __forceinline__ void rl2_shift(RealLane2<P> &s, int gl, int L, int w, float2 tail_keep = {1.f, 1.f}) {
    const unsigned full = 0xffffffffu;
    const float up = __shfl_up_sync(full, s.fp[P - 1].y, 1, L);
    const float dn = __shfl_down_sync(full, s.fm[0].x, 1, L);
    const float old_fm0 = s.fm[0].x;
#pragma unroll
    for (int i = P - 1; i >= 1; i--) s.fp[i] = make_float2(s.fp[i - 1].y, s.fp[i].x);
    s.fp[0] = make_float2(up, s.fp[0].x);
#pragma unroll
    for (int i = 0; i < P - 1; i++) s.fm[i] = make_float2(s.fm[i].y, s.fm[i + 1].x);
    s.fm[P - 1] = make_float2(s.fm[P - 1].y, (gl == L - 1) ? 0.f : dn);
    if (gl == 0) s.fp[0].x = -((w == 1) ? old_fm0 : s.fm[0].x);
    if (TAIL) {
        s.fp[P - 1] = __fmul2_rn(s.fp[P - 1], tail_keep);
        return;
    }
    const int k0 = gl * 2 * P;
#pragma unroll
    for (int i = 0; i < P; i++) {
        if (k0 + 2 * i >= w) s.fp[i].x = 0.f;
        if (k0 + 2 * i + 1 >= w) s.fp[i].y = 0.f;
        if (k0 + 2 * i == w - 1) s.fm[i].x = 0.f;
        if (k0 + 2 * i + 1 == w - 1) s.fm[i].y = 0.f;
    }
}

// The real-valued kernel stages 32 steps per chunk (half the barriers of 16;
// its per-step shared data is small).
constexpr int kRealChunk = 32;
// Threads per CTA of the real-valued kernel: one warp, so that no CTA
// barrier makes the warps of a CTA wait for each other at every chunk (C1:
// 7.82 ms with 128 threads, 7.79 with 64, 7.63 with 32; the atoms are
// bit-identical).
// SNAPMRF_EPG_REAL_THREADS overrides it for tuning (a multiple of 32).
#ifndef SNAPMRF_EPG_REAL_THREADS
#define SNAPMRF_EPG_REAL_THREADS 32
#endif
constexpr int kRealThreads = SNAPMRF_EPG_REAL_THREADS;
static_assert(kRealThreads % 32 == 0, "whole warps");
constexpr int kRealFS = kRealChunk * 4 + 4;          // floats per atom of relaxation factors
constexpr int kRealReadoutStride = kRealChunk + 1;  // float2 per group

inline size_t epg_real_smem_bytes(int L) {
    int apc = kRealThreads / L;
    return (size_t)kRealChunk * 10 * sizeof(float2) + (size_t)apc * kRealFS * sizeof(float) +
           (size_t)apc * kRealReadoutStride * sizeof(float2) + (size_t)apc * 4 * sizeof(float);
}

// (An explicit minimum of 1 block per SM lets ptxas use more registers and
// costs a resident block per SM; SNAPMRF_EPG_REAL_MIN_BLOCKS is for tuning.)
#ifdef SNAPMRF_EPG_REAL_MIN_BLOCKS
#define SNAPMRF_EPG_REAL_BOUNDS __launch_bounds__(kRealThreads, SNAPMRF_EPG_REAL_MIN_BLOCKS)
#elif defined(SNAPMRF_EPG_REAL_MAXNREG)
#define SNAPMRF_EPG_REAL_BOUNDS __maxnreg__(SNAPMRF_EPG_REAL_MAXNREG)
#else
#define SNAPMRF_EPG_REAL_BOUNDS __launch_bounds__(kRealThreads)
#endif

// One element of the optional 16-bit copy of Im(atom) (the tensor-core
// matching operand, one row per atom).
__device__ __forceinline__ void store_packed(const EpgArgs &a, long long atom, long long q, float v) {
    if (a.packed_half)
        reinterpret_cast<__half *>(a.packed)[atom * a.packed_pitch + q] = __float2half_rn(v);
    else
        reinterpret_cast<__nv_bfloat16 *>(a.packed)[atom * a.packed_pitch + q] = __float2bfloat16_rn(v);
}

// FOLD: relaxation is diagonal with one factor for F+ and F- (and Z0's
// recovery only touches state 0), so it commutes with the dephasing shift:
// relax(TE), shift, relax(TR - TE) equals shift followed by one relaxation
// over TR, and that relaxation is folded into the next step's RF columns
// (c_j * E_j, plus the recovery (1 - E1) times the RF's Z column on state 0).
// The readout after relax(TE) is E2(TE) f+[0] right after the RF.  Two
// multiplies per state and step fewer, and one exp fewer per atom and step;
// the result differs from the separate relaxations only by rounding.
//
// One CTA's work: atoms atom0 .. atom0 + kRealThreads / L - 1 of B1 block
// blk, L lanes per atom, P pairs of states per lane.
template <int ECHO, int P, bool TAIL, bool FOLD>
__device__ __forceinline__ void epg_real_cta(const EpgArgs &a, const int L, const long long blk,
                                             const long long atom0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NF = 4;
    constexpr int FS = kRealFS;
    const int apc = kRealThreads / L;
    const int tid = threadIdx.x;
    const int g = tid / L;
    const int gl = tid % L;
    const bool lane0 = (gl == 0);
    const long long nreps = a.nreps;
    const long long ab = atom0 + g;
    const bool active = ab < a.natoms;
    const long long gatom = blk * a.natoms + ab;

    float2 *sC = reinterpret_cast<float2 *>(smem_raw);        // [kRealChunk][10]
    float *sF = reinterpret_cast<float *>(sC + kRealChunk * 10);   // [apc][FS]
    float2 *sR = reinterpret_cast<float2 *>(sF + apc * FS);    // [apc][kRealReadoutStride]
    float *sP = reinterpret_cast<float *>(sR + apc * kRealReadoutStride);

    for (int i = tid; i < apc; i += kRealThreads) {
        long long at = atom0 + i;
        float t1 = 1.f, t2 = 1.f;
        if (at < a.natoms) {
            const float *p = a.params + (blk * a.natoms + at) * a.nparams;
            t1 = p[0];
            t2 = p[1];
        }
        sP[4 * i] = t1;
        sP[4 * i + 1] = t2;
        sP[4 * i + 2] = 1.f / t1;
        sP[4 * i + 3] = 1.f / t2;
    }

    const float *alpha = a.alpha + blk * nreps;
    const float *phi = a.sched + nreps;
    const float *TR = a.sched + 2 * nreps;
    const float *TE = a.sched + 3 * nreps;
    __syncthreads();
    const int w = a.nstates;
    // TAIL layouts: 0 at slot w (cleared after each shift), 1 elsewhere
    float2 tail_keep = make_float2(1.f, 1.f);
    if (TAIL && gl == L - 1) {
        const int pad = L * 2 * P - w;
        tail_keep = make_float2(pad == 2 ? 0.f : 1.f, pad >= 1 ? 0.f : 1.f);
    }

    // init_rf_pulse with alpha = phi = 0, TI = 0 (the expression of st_init)
    RealLane2<P> s;
#pragma unroll
    for (int i = 0; i < P; i++) {
        s.fp[i] = make_float2(0.f, 0.f);
        s.fm[i] = make_float2(0.f, 0.f);
        s.zz[i] = make_float2(0.f, 0.f);
    }
    if (lane0) {
        const float T1 = sP[4 * g];
        float e1 = expf(-0.f / T1), sa, ca;
        __sincosf((float)(0.f * M_PI / 180.f), &sa, &ca);
        s.zz[0].x = e1 * ca + 1 - e1;
    }

    float nrm = 0.f;
    float2 *out = a.atoms + gatom * nreps;
    float *outi = reinterpret_cast<float *>(a.atoms) + gatom * nreps;  // (imaginary rows)
    for (long long t0 = 0; t0 < nreps; t0 += kRealChunk) {
        const int nch = (int)min((long long)kRealChunk, nreps - t0);
        __syncthreads();
        for (int i = tid; i < nch; i += kRealThreads) rf_real_coeffs2(alpha[t0 + i], phi[t0 + i], sC + 10 * i);
        for (int idx = tid; idx < apc * nch; idx += kRealThreads) {
            int ga = idx / nch, i = idx - ga * nch;
            float t1 = sP[4 * ga], t2 = sP[4 * ga + 1];
            float4 f;
            if (FOLD) {
                // (E1, E2) over the previous step's TR (1 before the first
                // step), E2 over this step's TE, and Z0's recovery 1 - E1;
                // rates as reciprocals (|t / T| < 1, so the argument's
                // rounding moves exp by far less than an ulp)
                const long long t = t0 + i;
                const float trp = t > 0 ? TR[t - 1] : 0.f;
                const float r1 = sP[4 * ga + 2], r2 = sP[4 * ga + 3];
                const float e1 = t > 0 ? expf(-trp * r1) : 1.f, e2 = t > 0 ? expf(-trp * r2) : 1.f;
                f = make_float4(e1, e2, expf(-TE[t] * r2), 1.f - e1);
            } else {
                float tr = TR[t0 + i], te = TE[t0 + i];
                float ta = te, tb = tr - te;
                f = make_float4(expf(-ta / t1), expf(-ta / t2), expf(-tb / t1), expf(-tb / t2));
            }
            *reinterpret_cast<float4 *>(sF + ga * FS + i * NF) = f;
        }
        __syncthreads();
        for (int i = 0; i < nch; i++) {
            const float4 f = *reinterpret_cast<const float4 *>(sF + g * FS + i * NF);
            if (FOLD) {
                const float2 *c = sC + 10 * i;
                const float2 e1 = make_float2(f.x, f.x), e2 = make_float2(f.y, f.y);
                rl2_rf_k8<P>(s, __fmul2_rn(c[0], e2), __fmul2_rn(c[1], e2), __fmul2_rn(c[2], e1),
                             __fmul2_rn(c[6], e2), __fmul2_rn(c[8], e1));
                if (lane0) {
                    // the recovery term (1 - E1) of Z0 through the RF's Z column
                    s.fp[0].x = fmaf(c[2].x, f.w, s.fp[0].x);
                    s.fm[0].x = fmaf(c[5].x, f.w, s.fm[0].x);
                    s.zz[0].x = fmaf(c[8].x, f.w, s.zz[0].x);
                    const float v = f.z * s.fp[0].x;
                    sR[g * kRealReadoutStride + i] = make_float2(0.f, v);
                    nrm = fmaf(v, v, nrm);
                }
                if (ECHO == ECHO_FISP) rl2_shift<P, TAIL>(s, gl, L, w, tail_keep);
            } else {
                rl2_rf<P>(s, sC + 10 * i);
                rl2_relax<P>(s, f.x, f.y, lane0);
                if (lane0) {
                    const float v = s.fp[0].x;
                    sR[g * kRealReadoutStride + i] = make_float2(0.f, v);
                    // the complex path adds round(0*0 + v*v) = round(v*v)
                    nrm = __fadd_rn(nrm, __fmul_rn(v, v));
                }
                if (ECHO == ECHO_FISP) rl2_shift<P, TAIL>(s, gl, L, w, tail_keep);
                rl2_relax<P>(s, f.z, f.w, lane0);
            }
        }
        __syncwarp();
        if (active)
            for (int q = gl; q < nch; q += L) {
                const float2 o = sR[g * kRealReadoutStride + q];
                if (a.imag_rows)
                    outi[t0 + q] = o.y;
                else
                    out[t0 + q] = o;
                if (a.packed && !a.normalize && !a.pack_normalized) store_packed(a, gatom, t0 + q, o.y);
            }
    }
    if (a.normalize || a.norms || a.pack_normalized) {
        nrm = __shfl_sync(0xffffffffu, nrm, 0, L);
        if (a.norms && lane0 && active) a.norms[gatom] = sqrtf(nrm);
        if (a.normalize || (a.pack_normalized && !a.operand_pass)) {
            __syncwarp();
            float inv = nrm;
            if (inv > 0.f) inv = 1.f / sqrtf(inv);
            if (active) {
                if (a.normalize && a.imag_rows) {
                    // (the same product as the complex row's imaginary part)
                    for (long long q = gl; q < nreps; q += L) {
                        const float o = outi[q] * inv;
                        outi[q] = o;
                        if (a.packed) store_packed(a, gatom, q, o);
                    }
                } else if (a.normalize) {
                    for (long long q = gl; q < nreps; q += L) {
                        const float2 o = c_scale(out[q], inv);
                        out[q] = o;
                        if (a.packed) store_packed(a, gatom, q, o.y);
                    }
                } else {
                    // the operand of the unit-norm atom (the same product
                    // as above); the atom itself is not rewritten
                    for (long long q = gl; q < nreps; q += L)
                        store_packed(a, gatom, q, a.imag_rows ? outi[q] * inv : c_scale(out[q], inv).y);
                }
            }
        }
    }
    if (a.packed && active && !a.operand_pass)
        for (long long q = nreps + gl; q < a.packed_pitch; q += L) store_packed(a, gatom, q, 0.f);
}

// Fine layout of the real-valued recursion: kFineP pairs of states per lane
// and kFineL = 32 / kFineP lanes per atom (64 states, so w <= 64).  Two
// pairs measured best on C1's tail (one: a lone warp is latency-bound on the
// shuffles; four: more instructions per step).
#ifndef SNAPMRF_EPG_FINE_P
#define SNAPMRF_EPG_FINE_P 2
#endif
constexpr int kFineP = SNAPMRF_EPG_FINE_P;
constexpr int kFineL = 32 / kFineP;
static_assert(kFineP == 1 || kFineP == 2 || kFineP == 4 || kFineP == 8, "fine layout");

// Grid: x = CTA within the B1 block, y = block.  Each CTA signals at once
// that a grid launched after it as a programmatic dependent (the fine tail
// below) may start: that grid then starts when every CTA of this one has
// started, i.e. during its last round.
template <int ECHO, int P, bool TAIL, bool FOLD>
__global__ void SNAPMRF_EPG_REAL_BOUNDS epg_real_kernel(EpgArgs a) {
    asm volatile("griddepcontrol.launch_dependents;");
    epg_real_cta<ECHO, P, TAIL, FOLD>(a, a.L, blockIdx.y, (long long)blockIdx.x * (kRealThreads / a.L));
}

// Fine tail: atoms a.fine_first .. natoms - 1 of each B1 block in the fine
// layout.  A CTA carries its atoms through every step whatever its layout,
// and the fine CTAs, a few times shorter than those of the chosen layout,
// fill the slots that the chosen layout's last, partial round of resident
// CTAs leaves free instead of a few full-length CTAs running alone.  Every
// layout performs the same operations on each state in the same order, so
// the atoms do not depend on the split.  Launched as a programmatic
// dependent of the main grid, this grid must not complete before it (work
// after it on the stream reads the whole dictionary), hence the wait at the
// end; launched alone, the wait returns at once.
template <int ECHO, bool FOLD>
__global__ void __launch_bounds__(kRealThreads, 1) epg_real_fine_kernel(EpgArgs a) {
    epg_real_cta<ECHO, kFineP, false, FOLD>(a, kFineL, blockIdx.y,
                                            a.fine_first + (long long)blockIdx.x * (kRealThreads / kFineL));
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ROA (src/functions.cu:1021-1222).  State m = (Mx, My, Mz).  Per step:
// rotation R(alpha, phi), relaxation over the full TR, z-rotation by
// beta = pi*B0*TR/1000, readout Mx + iMy, z-rotation by beta.
struct RoaStep {
    float T[9];
};

// fill_transition_matrix (ROA, src/functions.cu:1049-1075); the Sgemm with
// OP_N reads it column-major: new[i] = sum_l T[i + 3l] * m[l].
__device__ __forceinline__ void roa_matrix(float alpha, float phi, float *T) {
    float s_a, c_a, s_p, c_p;
    __sincosf(alpha, &s_a, &c_a);
    __sincosf(phi, &s_p, &c_p);
    float s2 = 2 * c_p * s_p, c2 = c_p * c_p - s_p * s_p;
    T[0] = c2;
    T[1] = -s2;
    T[2] = 0.f;
    T[3] = s2 * c_a;
    T[4] = c2 * c_a;
    T[5] = -s_a;
    T[6] = s2 * s_a;
    T[7] = c2 * s_a;
    T[8] = c_a;
}

// init_rf_pulse (ROA, src/functions.cu:1022-1047); roa_ssfp calls it with
// alpha 180, phi 0, TI 0 (run-time values, see EpgArgs).
__device__ __forceinline__ void roa_init(float t1, float t2, float &m0, float &m1, float &m2, float alpha_deg,
                                         float phi_deg, float TI) {
    float ia = (float)(alpha_deg * M_PI / 180.f), ip = (float)(phi_deg * M_PI / 180.f);
    float e1 = expf(-TI / t1), e2 = expf(-TI / t2);
    float sa, ca, sph, cph;
    __sincosf(ia, &sa, &ca);
    __sincosf(ip, &sph, &cph);
    float sph2 = 2 * cph * sph, cph2 = cph * cph - sph * sph;
    m0 = e2 * sph2 * sa;
    m1 = e2 * cph2 * sa;
    m2 = e1 * ca + 1 - e1;
}

#ifndef SNAPMRF_EPG_DEVICE_HELPERS_ONLY
// (the non-template kernel below is defined once, in epg.cu; other sources
// that need only the device helpers above define
// SNAPMRF_EPG_DEVICE_HELPERS_ONLY)

// Single isochromat (the reference's roa_ssfp): one thread per atom.
__global__ void __launch_bounds__(kEpgThreads) roa_kernel(EpgArgs a) {
    __shared__ RoaStep sT[kChunk];
    __shared__ float2 sR[kEpgThreads][kChunk + 1];
    const int tid = threadIdx.x;
    const long long blk = blockIdx.y;
    const long long nreps = a.nreps;
    const long long atom0 = (long long)blockIdx.x * kEpgThreads;
    const long long ab = atom0 + tid;
    const bool active = ab < a.natoms;
    const long long gatom = blk * a.natoms + ab;
    float t1 = 1.f, t2 = 1.f, b0 = 0.f;
    if (active) {
        const float *p = a.params + (blk * a.natoms + ab) * a.nparams;
        t1 = p[0];
        t2 = p[1];
        b0 = p[2];
    }
    const float *alpha = a.alpha + blk * nreps;
    const float *phi = a.sched + nreps;
    const float *TR = a.sched + 2 * nreps;
    float m0, m1, m2;
    roa_init(t1, t2, m0, m1, m2, a.init_alpha_deg, a.init_phi_deg, a.init_ti);
    float nrm = 0.f;
    const int warp = tid / 32, lane = tid % 32;
    for (long long t0 = 0; t0 < nreps; t0 += kChunk) {
        const int nch = (int)min((long long)kChunk, nreps - t0);
        __syncthreads();
        for (int i = tid; i < nch; i += kEpgThreads) roa_matrix(alpha[t0 + i], phi[t0 + i], sT[i].T);
        __syncthreads();
        for (int i = 0; i < nch; i++) {
            const float *T = sT[i].T;
            // the in-place cublasSgemm of apply_rf_pulse (ROA), accumulated
            // over the three components in order
            float n0 = fmaf(T[6], m2, fmaf(T[3], m1, T[0] * m0));
            float n1 = fmaf(T[7], m2, fmaf(T[4], m1, T[1] * m0));
            float n2 = fmaf(T[8], m2, fmaf(T[5], m1, T[2] * m0));
            float tr = TR[t0 + i];
            float E1 = expf(-tr / t1), E2 = expf(-tr / t2);
            m0 = E2 * n0;
            m1 = E2 * n1;
            m2 = E1 * n2 + (1 - E1);
            float beta = (float)(M_PI * b0 * tr / 1000.f);
            float sb, cb;
            __sincosf(beta, &sb, &cb);
            float w1 = m0, w2 = m1;
            m0 = cb * w1 + sb * w2;
            m1 = cb * w2 - sb * w1;
            sR[tid][i] = make_float2(m0, m1);
            nrm += m0 * m0 + m1 * m1;
            w1 = m0;
            w2 = m1;
            m0 = cb * w1 + sb * w2;
            m1 = cb * w2 - sb * w1;
        }
        __syncthreads();
        for (int r = warp; r < kEpgThreads; r += kEpgThreads / 32) {
            long long at = atom0 + r;
            if (at >= a.natoms) continue;
            float2 *o = a.atoms + (blk * a.natoms + at) * nreps + t0;
            for (int q = lane; q < nch; q += 32) o[q] = sR[r][q];
        }
    }
    __syncthreads();
    if (a.norms && active) a.norms[gatom] = sqrtf(nrm);
    if (a.normalize && active) {
        float inv = nrm;
        if (inv > 0.f) inv = 1.f / sqrtf(inv);
        float2 *out = a.atoms + gatom * nreps;
        for (long long q = 0; q < nreps; q++) out[q] = c_scale(out[q], inv);
    }
}

// Multi-isochromat ROA: a group of G lanes per atom (G = 8, 16 or 32, a
// divisor of the warp), IPL isochromats per lane; lane r of a group holds
// isochromats r*IPL .. r*IPL + IPL - 1 (those past n_iso idle), so that G*IPL
// close above n_iso wastes few slots (n_iso = 100: 8 x 13 = 104, where 32
// lanes x 4 carried 128).  Isochromat j precesses by an extra pi*j/n_iso per
// half TR (2*pi*j/n_iso per TR, so the n_iso isochromats dephase uniformly
// across 2*pi); the readout is the mean of Mx + iMy over isochromats.  The
// relaxation over TR is folded into the rotation's rows (E2 into the rows of
// Mx and My, E1 into Mz's, whose recovery 1 - E1 starts the sum; the row's
// Mx entry is zero), and the step's relaxation factors and B0 phasor are
// computed once per atom and step by the group's lanes and staged.
template <int IPL>
__global__ void __launch_bounds__(kEpgThreads) roa_iso_kernel(EpgArgs a, int G) {
    constexpr int MAXA = kEpgThreads / 8;  // atoms per CTA at G = 8
    __shared__ RoaStep sT[kChunk];
    // (rows padded by one entry: the groups of a warp read and write
    // different banks)
    __shared__ float4 sF[MAXA][kChunk + 1];   // per atom and step: E1, E2, sin, cos of beta
    __shared__ float2 sOut[MAXA][kChunk + 1];  // the readout
    const int tid = threadIdx.x;
    const int apc = kEpgThreads / G, ga = tid / G, r = tid % G;
    const long long blk = blockIdx.y;
    const long long nreps = a.nreps;
    const long long ab = (long long)blockIdx.x * apc + ga;
    const bool active = ab < a.natoms;
    const long long gatom = blk * a.natoms + ab;
    float t1 = 1.f, t2 = 1.f, b0 = 0.f;
    if (active) {
        const float *p = a.params + gatom * a.nparams;
        t1 = p[0];
        t2 = p[1];
        b0 = p[2];
    }
    const float *alpha = a.alpha + blk * nreps;
    const float *phi = a.sched + nreps;
    const float *TR = a.sched + 2 * nreps;
    const int n_iso = a.n_iso;
    float i0, i1, i2;
    roa_init(t1, t2, i0, i1, i2, a.init_alpha_deg, a.init_phi_deg, a.init_ti);
    // (a slot past n_iso gets a zero rotation: its Mx, My stay 0 after the
    // first step and its readout adds exactly 0)
    float m0[IPL], m1[IPL], m2[IPL], cd[IPL], sd[IPL];
#pragma unroll
    for (int q = 0; q < IPL; q++) {
        const int j = r * IPL + q;
        m0[q] = i0;
        m1[q] = i1;
        m2[q] = i2;
        double d = M_PI * (double)j / (double)n_iso;
        cd[q] = j < n_iso ? (float)cos(d) : 0.f;
        sd[q] = j < n_iso ? (float)sin(d) : 0.f;
    }
    const float inv_n = 1.f / (float)n_iso;
    float nrm = 0.f;
    float2 *out = a.atoms + gatom * nreps;
    for (long long t0 = 0; t0 < nreps; t0 += kChunk) {
        const int nch = (int)min((long long)kChunk, nreps - t0);
        __syncthreads();
        for (int i = tid; i < nch; i += kEpgThreads) roa_matrix(alpha[t0 + i], phi[t0 + i], sT[i].T);
        for (int i = r; i < nch; i += G) {
            const float tr = TR[t0 + i];
            float sb, cb;
            const float beta = (float)(M_PI * b0 * tr / 1000.f);
            __sincosf(beta, &sb, &cb);
            sF[ga][i] = make_float4(expf(-tr / t1), expf(-tr / t2), sb, cb);
        }
        __syncthreads();
        for (int i = 0; i < nch; i++) {
            const float *T = sT[i].T;
            const float4 f = sF[ga][i];
            const float E1 = f.x, E2 = f.y, sb = f.z, cb = f.w;
            const float a0 = E2 * T[0], a3 = E2 * T[3], a6 = E2 * T[6];
            const float a1 = E2 * T[1], a4 = E2 * T[4], a7 = E2 * T[7];
            const float c5 = E1 * T[5], c8 = E1 * T[8], rec = 1.f - E1;
            float px = 0.f, py = 0.f;
#pragma unroll
            for (int q = 0; q < IPL; q++) {
                const float x = fmaf(a6, m2[q], fmaf(a3, m1[q], a0 * m0[q]));
                const float y = fmaf(a7, m2[q], fmaf(a4, m1[q], a1 * m0[q]));
                m2[q] = fmaf(c8, m2[q], fmaf(c5, m1[q], rec));
                // rotation by beta then by the isochromat's delta
                const float cx = cb * cd[q] - sb * sd[q], sx = sb * cd[q] + cb * sd[q];
                const float w1 = cx * x + sx * y, w2 = cx * y - sx * x;
                px += w1;
                py += w2;
                m0[q] = cx * w1 + sx * w2;
                m1[q] = cx * w2 - sx * w1;
            }
            // the group's sum (a group never straddles a warp)
            for (int o = G / 2; o; o >>= 1) {
                px += __shfl_xor_sync(0xffffffffu, px, o);
                py += __shfl_xor_sync(0xffffffffu, py, o);
            }
            if (r == 0) sOut[ga][i] = make_float2(px * inv_n, py * inv_n);
        }
        __syncwarp();
        for (int i = r; i < nch; i += G) {
            const float2 v = sOut[ga][i];
            nrm = fmaf(v.x, v.x, fmaf(v.y, v.y, nrm));
            if (active) out[t0 + i] = v;
        }
    }
    for (int o = G / 2; o; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    if (a.norms && active && r == 0) a.norms[gatom] = sqrtf(nrm);
    // (with G = 32 a lane rescales samples another lane of the group wrote)
    __syncwarp();
    if (a.normalize && active) {
        float inv = nrm;
        if (inv > 0.f) inv = 1.f / sqrtf(inv);
        for (long long q = r; q < nreps; q += G) out[q] = c_scale(out[q], inv);
    }
}

// Isochromats per lane and lanes per atom of roa_iso_kernel: the fewest
// slots G * IPL >= n_iso (n_iso <= 256), then the most isochromats per lane.
inline void roa_iso_layout(int n_iso, int *G, int *ipl) {
    static const int ipls[] = {13, 8, 7, 4, 2, 1};
    int best = 1 << 30;
    for (int g : {8, 16, 32})
        for (int i : ipls)
            if (g * i >= n_iso && (g * i < best || (g * i == best && i > *ipl))) {
                best = g * i;
                *G = g;
                *ipl = i;
            }
}

inline cudaError_t launch_roa(const EpgArgs &a, long long natoms, unsigned gen_blocks,
                              cudaStream_t st) {
    if (a.n_iso <= 1) {
        dim3 grid((unsigned)((natoms + kEpgThreads - 1) / kEpgThreads), gen_blocks);
        roa_kernel<<<grid, kEpgThreads, 0, st>>>(a);
    } else {
        int G = 32, ipl = 0;
        roa_iso_layout(a.n_iso, &G, &ipl);
        const long long apc = kEpgThreads / G;
        dim3 grid((unsigned)((natoms + apc - 1) / apc), gen_blocks);
        switch (ipl) {
        case 1: roa_iso_kernel<1><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        case 2: roa_iso_kernel<2><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        case 4: roa_iso_kernel<4><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        case 7: roa_iso_kernel<7><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        case 8: roa_iso_kernel<8><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        default: roa_iso_kernel<13><<<grid, kEpgThreads, 0, st>>>(a, G); break;
        }
    }
    note_launches(1);
    return cudaGetLastError();
}

#endif  // SNAPMRF_EPG_DEVICE_HELPERS_ONLY

}  // namespace snapmrf
