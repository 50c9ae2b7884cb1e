// Derivatives of the EPG recursion on sm_100a: a reverse-mode (adjoint)
// kernel with checkpointing, and a forward-mode kernel with two tangents
// that drives a per-voxel Gauss-Newton refinement of (T1, T2).
//
// Both work on the real-valued FISP / SR recursion (every RF phase 0, the
// form of the benchmark dictionaries): per EPG state f+ = Im F+,
// f- = Im F-, z = Re Z; flip angle a_t = alpha_t * B1; per step
//   RF    f+' = c f+ + s f- - S z,  f-' = s f+ + c f- + S z,
//         z'  = S/2 f+ - S/2 f- + C z      (C = cos a, S = sin a,
//                                          c = (1 + C)/2, s = (1 - C)/2)
//   relax f+- *= E2(TE), z *= E1(TE), z0 += 1 - E1(TE)
//   read  s_t = i f+[0]
//   shift (FISP only) F+ up, F- down, f+[0] = -f-[0], F-[w-1] = 0
//   relax over TR - TE
// which is the reference's epg_fisp / epg_sr (src/functions.cu:687-739,
// 878-933) with the B1 extension (flip angle times the atom's B1).
//
// Layout: one atom (or voxel) per group of L lanes, S states per lane, as in
// the dictionary kernels; states k >= w are kept exactly zero so that they
// never enter a gradient.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.h"

namespace snapmrf {
namespace grad {

constexpr int kThreads = 128;
// Threads per CTA of gn_kernel: one warp, so that no CTA barrier makes the
// warps of a CTA wait for each other at every chunk (C1, three iterations:
// 14.42 ms against 14.63 with 128 threads; identical maps).
// SNAPMRF_GN_THREADS overrides it for tuning.
#ifndef SNAPMRF_GN_THREADS
#define SNAPMRF_GN_THREADS 32
#endif
constexpr int kGnThreads = SNAPMRF_GN_THREADS;
static_assert(kGnThreads % 32 == 0, "whole warps");

// Voxels per CTA of gn_kernel with L lanes per voxel: 32 / L groups per warp
// (a group never straddles two warps; with L not a power of two the last
// 32 mod L lanes of each warp idle).
__host__ __device__ constexpr int gn_voxels_per_cta(int L) { return (kGnThreads / 32) * (32 / L); }
constexpr int kMaxS = 8;

struct Schedule {
    const float *alpha;  // [nreps] raw flip angles (rad)
    const float *TR;     // [nreps] ms
    const float *TE;     // [nreps] ms
    int nreps;
};

// Per-step constants of the recursion for one flip angle a.
struct StepRF {
    float C, S, c, s, hS;  // cos a, sin a, (1+C)/2, (1-C)/2, S/2
};

__device__ __forceinline__ StepRF step_rf(float a) {
    StepRF r;
    __sincosf(a, &r.S, &r.C);
    r.c = (1 + r.C) / 2;
    r.s = (1 - r.C) / 2;
    r.hS = 0.5f * r.S;
    return r;
}

template <int S>
struct St {
    float p[S], m[S], z[S];
};

template <int S>
__device__ __forceinline__ void rf_fwd(St<S> &x, const StepRF &r) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        const float p = x.p[j], m = x.m[j], q = x.z[j];
        x.p[j] = fmaf(-r.S, q, fmaf(r.s, m, r.c * p));
        x.m[j] = fmaf(r.S, q, fmaf(r.c, m, r.s * p));
        x.z[j] = fmaf(r.C, q, fmaf(-r.hS, m, r.hS * p));
    }
}

template <int S>
__device__ __forceinline__ void relax_fwd(St<S> &x, float E1, float E2, bool lane0) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        x.p[j] *= E2;
        x.m[j] *= E2;
        x.z[j] *= E1;
    }
    if (lane0) x.z[0] += 1 - E1;
}

// Shift with padding kept at zero (see dephase_gradients).
template <int S>
__device__ __forceinline__ void shift_fwd(St<S> &x, int gl, int L, int w) {
    const unsigned full = 0xffffffffu;
    const float up = __shfl_up_sync(full, x.p[S - 1], 1, L);
    const float dn = __shfl_down_sync(full, x.m[0], 1, L);
    const float old_m0 = x.m[0];
#pragma unroll
    for (int j = S - 1; j >= 1; j--) x.p[j] = x.p[j - 1];
    x.p[0] = up;
#pragma unroll
    for (int j = 0; j < S - 1; j++) x.m[j] = x.m[j + 1];
    x.m[S - 1] = (gl == L - 1) ? 0.f : dn;
    if (gl == 0) x.p[0] = -((w == 1) ? old_m0 : x.m[0]);
#pragma unroll
    for (int j = 0; j < S; j++) {
        const int k = gl * S + j;
        if (k >= w) x.p[j] = x.m[j] = 0.f;
        if (k == w - 1) x.m[j] = 0.f;
    }
}

// Transpose of shift_fwd acting on an adjoint state: lambda_f+ moves down a
// slot, lambda_f- up a slot, lambda_f-[1] (or [0] for w = 1) receives
// -lambda_f+[0]; lambda_f+[w-1] and lambda_f-[k >= w] vanish.
template <int S>
__device__ __forceinline__ void shift_adj(St<S> &l, int gl, int L, int w) {
    const unsigned full = 0xffffffffu;
    const float lp0 = l.p[0];
    const float lp0_all = __shfl_sync(full, lp0, 0, L);   // lambda_f+[0] of the group
    const float dn = __shfl_down_sync(full, l.p[0], 1, L);
    const float up = __shfl_up_sync(full, l.m[S - 1], 1, L);
#pragma unroll
    for (int j = 0; j < S - 1; j++) l.p[j] = l.p[j + 1];
    l.p[S - 1] = (gl == L - 1) ? 0.f : dn;
#pragma unroll
    for (int j = S - 1; j >= 1; j--) l.m[j] = l.m[j - 1];
    l.m[0] = (gl == 0) ? 0.f : up;
    // f+[0] = -f-[1] (w >= 2) or -f-[0] (w == 1) before the shift
    const int kk = (w == 1) ? 0 : 1;
#pragma unroll
    for (int j = 0; j < S; j++) {
        const int k = gl * S + j;
        if (k == kk) l.m[j] -= lp0_all;
        if (k == w - 1) l.p[j] = 0.f;
        if (k >= w) l.m[j] = 0.f;
    }
}

__device__ __forceinline__ float group_sum(float v, int L) {
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, L);
    return v;
}

// --------------------------------------------------------------------------
// Adjoint
// --------------------------------------------------------------------------
struct AdjArgs {
    Schedule sch;
    const float *params;      // [n][nparams]: T1, T2, (B0), B1
    int nparams;
    long long n;
    int w, L, shift;
    const float2 *gsig;       // [n][nreps] dL/d(Re s_t, Im s_t)
    float2 *sig;              // optional out [n][nreps]
    float *gparams;           // [n][3]: dL/dT1, dL/dT2, dL/dB1
    float *galpha_atoms;      // [n][nreps] dL/dalpha_t per atom
    float *ckpt;              // [n][nckpt][3][L*S]
    float *seg;               // [n][C][3][L*S]
    int C, nckpt;
};

// A saved state is [3][S][L] floats: for each register slot the L lanes of
// the group touch consecutive words.
template <int S>
__device__ __forceinline__ void store_state(float *dst, int L, int gl, const St<S> &x) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        dst[j * L + gl] = x.p[j];
        dst[(S + j) * L + gl] = x.m[j];
        dst[(2 * S + j) * L + gl] = x.z[j];
    }
}

template <int S>
__device__ __forceinline__ void load_state(const float *src, int L, int gl, St<S> &x) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        x.p[j] = src[j * L + gl];
        x.m[j] = src[(S + j) * L + gl];
        x.z[j] = src[(2 * S + j) * L + gl];
    }
}

__device__ __forceinline__ void relax_factors(const Schedule &sc, int t, float T1, float T2, float *E1a, float *E2a,
                                              float *E1b, float *E2b, float *ta, float *tb) {
    const float tr = sc.TR[t], te = sc.TE[t];
    *ta = te;
    *tb = tr - te;
    *E1a = expf(-*ta / T1);
    *E2a = expf(-*ta / T2);
    *E1b = expf(-*tb / T1);
    *E2b = expf(-*tb / T2);
}

template <int S>
__global__ void __launch_bounds__(kThreads) adjoint_kernel(AdjArgs a) {
    const int L = a.L, LS = L * S;
    const int g = threadIdx.x / L, gl = threadIdx.x % L;
    const long long atom = (long long)blockIdx.x * (kThreads / L) + g;
    const bool active = atom < a.n;
    const long long at = active ? atom : 0;
    const bool lane0 = gl == 0;
    const float *pp = a.params + at * a.nparams;
    const float T1 = pp[0], T2 = pp[1], B1 = pp[3];
    const int T = a.sch.nreps, w = a.w;
    float *ck = a.ckpt + at * (long long)a.nckpt * 3 * LS;
    float *sg = a.seg + at * (long long)a.C * 3 * LS;

    // forward with checkpoints
    St<S> x;
#pragma unroll
    for (int j = 0; j < S; j++) x.p[j] = x.m[j] = x.z[j] = 0.f;
    if (lane0) x.z[0] = 1.f;
    for (int t = 0; t < T; t++) {
        if (t % a.C == 0 && active) store_state<S>(ck + (long long)(t / a.C) * 3 * LS, L, gl, x);
        float E1a, E2a, E1b, E2b, ta, tb;
        relax_factors(a.sch, t, T1, T2, &E1a, &E2a, &E1b, &E2b, &ta, &tb);
        rf_fwd<S>(x, step_rf(a.sch.alpha[t] * B1));
        relax_fwd<S>(x, E1a, E2a, lane0);
        if (lane0 && active && a.sig) a.sig[at * T + t] = make_float2(0.f, x.p[0]);
        if (a.shift) shift_fwd<S>(x, gl, L, w);
        relax_fwd<S>(x, E1b, E2b, lane0);
    }
    __syncwarp();

    // reverse sweep, one checkpoint segment at a time
    St<S> l;
#pragma unroll
    for (int j = 0; j < S; j++) l.p[j] = l.m[j] = l.z[j] = 0.f;
    float gT1 = 0.f, gT2 = 0.f, gB1 = 0.f;
    for (int c = a.nckpt - 1; c >= 0; c--) {
        const int t0 = c * a.C, t1 = min(T, t0 + a.C);
        if (active) load_state<S>(ck + (long long)c * 3 * LS, L, gl, x);
        for (int t = t0; t < t1; t++) {
            if (active) store_state<S>(sg + (long long)(t - t0) * 3 * LS, L, gl, x);
            float E1a, E2a, E1b, E2b, ta, tb;
            relax_factors(a.sch, t, T1, T2, &E1a, &E2a, &E1b, &E2b, &ta, &tb);
            rf_fwd<S>(x, step_rf(a.sch.alpha[t] * B1));
            relax_fwd<S>(x, E1a, E2a, lane0);
            if (a.shift) shift_fwd<S>(x, gl, L, w);
            relax_fwd<S>(x, E1b, E2b, lane0);
        }
        __syncwarp();
        for (int t = t1 - 1; t >= t0; t--) {
            St<S> x0, xr, xs;
            if (active) load_state<S>(sg + (long long)(t - t0) * 3 * LS, L, gl, x0);
            else {
#pragma unroll
                for (int j = 0; j < S; j++) x0.p[j] = x0.m[j] = x0.z[j] = 0.f;
            }
            float E1a, E2a, E1b, E2b, ta, tb;
            relax_factors(a.sch, t, T1, T2, &E1a, &E2a, &E1b, &E2b, &ta, &tb);
            const float at_ = a.sch.alpha[t] * B1;
            const StepRF r = step_rf(at_);
            xr = x0;
            rf_fwd<S>(xr, r);          // state after RF
            xs = xr;
            relax_fwd<S>(xs, E1a, E2a, lane0);
            if (a.shift) shift_fwd<S>(xs, gl, L, w);   // state entering relax over TR-TE

            // relax(TR-TE)^T
            float gE1 = 0.f, gE2 = 0.f;
#pragma unroll
            for (int j = 0; j < S; j++) {
                gE2 += l.p[j] * xs.p[j] + l.m[j] * xs.m[j];
                gE1 += l.z[j] * xs.z[j];
            }
            if (lane0) gE1 -= l.z[0];
            gT1 += gE1 * E1b * tb / (T1 * T1);
            gT2 += gE2 * E2b * tb / (T2 * T2);
#pragma unroll
            for (int j = 0; j < S; j++) {
                l.p[j] *= E2b;
                l.m[j] *= E2b;
                l.z[j] *= E1b;
            }
            if (a.shift) shift_adj<S>(l, gl, L, w);
            // readout s_t = i f+[0] after relax(TE)
            if (lane0 && active) l.p[0] += a.gsig[at * T + t].y;
            // relax(TE)^T, pre-op state xr
            gE1 = 0.f;
            gE2 = 0.f;
#pragma unroll
            for (int j = 0; j < S; j++) {
                gE2 += l.p[j] * xr.p[j] + l.m[j] * xr.m[j];
                gE1 += l.z[j] * xr.z[j];
            }
            if (lane0) gE1 -= l.z[0];
            gT1 += gE1 * E1a * ta / (T1 * T1);
            gT2 += gE2 * E2a * ta / (T2 * T2);
#pragma unroll
            for (int j = 0; j < S; j++) {
                l.p[j] *= E2a;
                l.m[j] *= E2a;
                l.z[j] *= E1a;
            }
            // RF^T with pre-op state x0; derivative of the matrix w.r.t. a
            float ga = 0.f;
#pragma unroll
            for (int j = 0; j < S; j++) {
                const float p = x0.p[j], m = x0.m[j], q = x0.z[j];
                const float dp = -r.hS * p + r.hS * m - r.C * q;
                const float dm = r.hS * p - r.hS * m + r.C * q;
                const float dz = 0.5f * r.C * p - 0.5f * r.C * m - r.S * q;
                ga += l.p[j] * dp + l.m[j] * dm + l.z[j] * dz;
                const float lp = l.p[j], lm = l.m[j], lz = l.z[j];
                l.p[j] = r.c * lp + r.s * lm + r.hS * lz;
                l.m[j] = r.s * lp + r.c * lm - r.hS * lz;
                l.z[j] = -r.S * lp + r.S * lm + r.C * lz;
            }
            ga = group_sum(ga, L);
            if (lane0 && active) a.galpha_atoms[at * T + t] = ga * B1;
            gB1 += ga * a.sch.alpha[t];
        }
        __syncwarp();
    }
    gT1 = group_sum(gT1, L);
    gT2 = group_sum(gT2, L);
    if (lane0 && active) {
        a.gparams[at * 3 + 0] = gT1;
        a.gparams[at * 3 + 1] = gT2;
        a.gparams[at * 3 + 2] = gB1;
    }
}

// Column sums of the per-atom schedule gradients in two deterministic
// passes: kSplits row ranges into partial sums, then the partials.
constexpr int kSplits = 512;

__global__ void sum_columns_partial_kernel(float *part, const float *in, long long n, int T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const long long r0 = n * blockIdx.y / kSplits, r1 = n * (blockIdx.y + 1) / kSplits;
    float s = 0.f;
    for (long long i = r0; i < r1; i++) s += in[i * T + t];
    part[(long long)blockIdx.y * T + t] = s;
}

__global__ void sum_columns_final_kernel(float *out, const float *part, int T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    float s = 0.f;
    for (int k = 0; k < kSplits; k++) s += part[(long long)k * T + t];
    out[t] = s;
}

// --------------------------------------------------------------------------
// Gauss-Newton refinement (forward mode, tangents d/dT1 and d/dT2)
// --------------------------------------------------------------------------
struct GnArgs {
    Schedule sch;
    long long nvox;
    int w, L, shift;
    const float2 *img;        // [nvox][img_stride]
    long long img_stride;
    float *maps;              // [nvox][nmaps] in/out: T1, T2, B0, B1, PD
    int nmaps;
    const float *b1map;       // optional [nvox]: B1 of each voxel
    float *m0;                // optional out [nvox]: |rho| with x ~ rho * s
    float max_rel_step;
    // early exit: voxels of list_in[0 .. *count_in) (all voxels when null);
    // voxels whose step exceeds tol of T1 or T2 are appended to list_out
    const int *list_in;
    const int *count_in;
    int *list_out;
    int *count_out;
    float tol;
    int finish;               // a voxel that stops in this pass writes PD, M0, B1
    // part 0: the whole list; 1: the bulk, whole rounds of round_groups groups
    // of bulk_apc voxels; 2: the tail after the bulk (a finer layout), so that
    // no round of the bulk kernel runs nearly empty
    int part;
    int bulk_apc;
    long long round_groups;
};

// A voxel whose map holds no usable start (not finite, T2 <= 0, T1 <= T2)
// is left as matched.
__device__ __forceinline__ bool usable(float T1, float T2, float B1) {
    return isfinite(T1) && isfinite(T2) && isfinite(B1) && T2 > 0.f && T1 > T2;
}

// Packed state of the refinement: P pairs of EPG states per lane (slot
// j = 2i + h of pair i is state k = gl * 2P + j), one set for the signal and
// one for each tangent; two-wide FP32 instructions update a pair at once.
template <int P>
struct Pair3 {
    float2 p[P], m[P], z[P];
};

template <int P>
__device__ __forceinline__ void pz(Pair3<P> &x) {
#pragma unroll
    for (int i = 0; i < P; i++) x.p[i] = x.m[i] = x.z[i] = make_float2(0.f, 0.f);
}

// RF pulse on one packed stream: F+' = c F+ + s F- - S Z, F-' = s F+ + c F-
// + S Z, Z' = hS (F+ - F-) + C Z (hS = S / 2 with its sign), computed as
// F-' = (c + s)(F+ + F-) - F+': 8 packed operations per pair instead of 9.
template <int P>
__device__ __forceinline__ void p_rf(Pair3<P> &x, float2 c, float2 s, float2 nS, float2 hS, float2 C) {
    const float2 cs = __fadd2_rn(c, s);
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float2 p = x.p[i], m = x.m[i], q = x.z[i];
        const float2 np = __ffma2_rn(nS, q, __ffma2_rn(s, m, __fmul2_rn(c, p)));
        const float2 d = __fadd2_rn(p, make_float2(-m.x, -m.y));
        x.z[i] = __ffma2_rn(C, q, __fmul2_rn(hS, d));
        x.m[i] = __ffma2_rn(cs, p, __ffma2_rn(cs, m, make_float2(-np.x, -np.y)));
        x.p[i] = np;
    }
}

// The RF with the previous interval's relaxation folded in (the shift
// commutes with relaxation, so relax(TR), shift, RF = shift, relax(TR), RF):
// on the pre-relaxation state (p, m, z), F+' = c' p + s' m + nS' z,
// Z' = hS' (p - m) + C' z and F-' = e2 (p + m) - F+' (c + s = 1), with
// c' = c e2, s' = s e2, nS' = -S e1, hS' = hS e2, C' = C e1.  8 packed
// operations per pair, the relaxation's 3 multiplies saved.
struct FoldedRF {
    float2 c, s, nS, hS, C, e2;
};

template <int P>
__device__ __forceinline__ void p_rf_folded(Pair3<P> &x, const FoldedRF &k) {
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float2 p = x.p[i], m = x.m[i], q = x.z[i];
        const float2 np = __ffma2_rn(k.nS, q, __ffma2_rn(k.s, m, __fmul2_rn(k.c, p)));
        const float2 d = __fadd2_rn(p, make_float2(-m.x, -m.y));
        x.z[i] = __ffma2_rn(k.C, q, __fmul2_rn(k.hS, d));
        x.m[i] = __ffma2_rn(k.e2, p, __ffma2_rn(k.e2, m, make_float2(-np.x, -np.y)));
        x.p[i] = np;
    }
}

// The T1 tangent's RF with its relaxation folded in: the product rule adds
// dE1 z_signal to Z before the RF, i.e. -S dE1 z_signal to F+' and
// C dE1 z_signal to Z' (F-' follows from the identity; F+ and F- get no
// source).  sz: the signal's pre-relaxation Z, read before the signal's RF.
template <int P>
__device__ __forceinline__ void p_rf_folded_t1(Pair3<P> &x, const FoldedRF &k, const float2 *sz, float2 nSd,
                                               float2 Cd) {
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float2 p = x.p[i], m = x.m[i], q = x.z[i];
        const float2 np =
            __ffma2_rn(nSd, sz[i], __ffma2_rn(k.nS, q, __ffma2_rn(k.s, m, __fmul2_rn(k.c, p))));
        const float2 d = __fadd2_rn(p, make_float2(-m.x, -m.y));
        x.z[i] = __ffma2_rn(Cd, sz[i], __ffma2_rn(k.C, q, __fmul2_rn(k.hS, d)));
        x.m[i] = __ffma2_rn(k.e2, p, __ffma2_rn(k.e2, m, make_float2(-np.x, -np.y)));
        x.p[i] = np;
    }
}

// Shift of one packed stream.  States k >= w hold zeros: F- needs no mask
// (F-[w-1] takes the zero of F-[w]), F+ takes F+[w-1] into slot w, which
// keep[] (0 at slot w, 1 elsewhere) clears.
// The neighbours' values come by shuffles from explicit lanes (src_up: the
// lane below in the group, src_dn: the lane above), so a group may have any
// width; a group's ends replace what they receive.
template <int P>
__device__ __forceinline__ void p_shift(Pair3<P> &x, int gl, int L, int w, const float2 *keep, int src_up,
                                        int src_dn, bool padded) {
    const unsigned full = 0xffffffffu;
    const float up = __shfl_sync(full, x.p[P - 1].y, src_up);
    const float dn = __shfl_sync(full, x.m[0].x, src_dn);
    const float old_m0 = x.m[0].x;
#pragma unroll
    for (int i = P - 1; i >= 1; i--) x.p[i] = make_float2(x.p[i - 1].y, x.p[i].x);
    x.p[0] = make_float2(up, x.p[0].x);
#pragma unroll
    for (int i = 0; i < P - 1; i++) x.m[i] = make_float2(x.m[i].y, x.m[i + 1].x);
    x.m[P - 1] = make_float2(x.m[P - 1].y, (gl == L - 1) ? 0.f : dn);
    if (gl == 0) x.p[0].x = -((w == 1) ? old_m0 : x.m[0].x);
    // (no slot w without padding: the last lane's F- takes a zero instead)
    if (padded) {
#pragma unroll
        for (int i = 0; i < P; i++) x.p[i] = __fmul2_rn(x.p[i], keep[i]);
    }
}

// Per-step constants of one voxel, staged in shared memory per chunk.
// Relaxation is diagonal in the EPG states with one factor for F+ and F-,
// so it commutes with the dephasing shift: relax(TE), shift, relax(TR-TE)
// equals shift, relax(TR), and the readout after relax(TE) is E2(TE) f+[0]
// taken right after the RF pulse.
struct GnStep {
    float C, S;            // cos, sin of alpha_t * B1
    float E1, E2;          // relaxation over TR
    float dE1, dE2;        // dE1/dT1, dE2/dT2
    float Ea, dEa;         // E2 over TE (readout) and dEa/dT2
    float xr, xi;          // voxel sample
};

constexpr int kGnChunk = 16;

// One Gauss-Newton iteration per voxel (TANGENTS) or, without tangents, the
// final evaluation of PD and M0 at the current parameters.  L lanes per
// voxel; a block of kGnThreads handles kGnThreads / L voxels in lockstep over
// chunks of `chunk` steps.
// (five pairs: at most 170 registers, so that three warps fit on an SM
// sub-partition)
// PAD: the layout has slots past the last state (L * 2P > w), whose F+ slot
// w the shift must clear.
template <int P, bool TANGENTS, bool PAD = true>
__global__ void __launch_bounds__(kGnThreads, P == 5 ? 12 * 32 / kGnThreads : 1) gn_kernel(GnArgs a, int chunk) {
    extern __shared__ __align__(16) unsigned char gn_smem[];
    const int L = a.L, gpw = 32 / L, apc = gn_voxels_per_cta(L);
    const int tid = threadIdx.x, lane = tid & 31, gl = lane % L;
    // lanes past the warp's last whole group idle (their group index is
    // clamped for the shared-memory reads; they write nothing)
    const bool idle = lane >= gpw * L;
    const int g = (tid >> 5) * gpw + min(lane / L, gpw - 1);
    const bool lane0 = gl == 0;
    const int src_up = gl == 0 ? lane : lane - 1, src_dn = lane + 1 < 32 ? lane + 1 : lane;
    // [apc][chunk] steps, each voxel's row padded by 16 bytes so that the
    // voxels of a warp read different banks
    const int qrow = chunk * (int)sizeof(GnStep) + 16;
    auto step_row = [&](int ga) { return reinterpret_cast<GnStep *>(gn_smem + (size_t)ga * qrow); };
    float *sV = reinterpret_cast<float *>(gn_smem + (size_t)apc * qrow);  // [apc][4]: T1, T2, B1, ok
    long long *sI = reinterpret_cast<long long *>(sV + apc * 4);  // [apc]: voxel or -1
    const long long nlist = a.list_in ? (long long)*a.count_in : a.nvox;
    long long first = 0, end = nlist;
    if (a.part) {
        const long long groups = (nlist + a.bulk_apc - 1) / a.bulk_apc;
        const long long bulk = min(nlist, (groups / a.round_groups) * a.round_groups * a.bulk_apc);
        if (a.part == 1) end = bulk;
        else first = bulk;
    }
    const long long vox0 = first + (long long)blockIdx.x * apc;
    for (int i = tid; i < apc; i += kGnThreads) {
        const long long slot = vox0 + i;
        long long v = -1;
        if (slot < end) v = a.list_in ? (long long)a.list_in[slot] : slot;
        sI[i] = v;
        float T1 = 2.f, T2 = 1.f, B1 = 1.f, ok = 0.f;
        if (v >= 0) {
            const float *mp = a.maps + v * a.nmaps;
            const float t1 = mp[0], t2 = mp[1];
            const float b1 = a.b1map ? a.b1map[v] : (a.nmaps >= 4 ? mp[3] : 1.f);
            if (usable(t1, t2, b1)) {
                T1 = t1;
                T2 = t2;
                B1 = b1;
                ok = 1.f;
            }
        }
        sV[4 * i] = T1;
        sV[4 * i + 1] = T2;
        sV[4 * i + 2] = B1;
        sV[4 * i + 3] = ok;
    }
    // a block without a usable voxel leaves at once (uniformly)
    if (!__syncthreads_or(tid < apc && sV[4 * tid + 3] != 0.f)) return;
    const long long v = sI[g];
    const bool active = !idle && sV[4 * g + 3] != 0.f;
    const int T = a.sch.nreps, w = a.w;
    const int k0 = gl * 2 * P;
    constexpr bool padded = PAD;
    float2 keep[P];
#pragma unroll
    for (int i = 0; i < P; i++)
        keep[i] = make_float2(k0 + 2 * i == w ? 0.f : 1.f, k0 + 2 * i + 1 == w ? 0.f : 1.f);

    Pair3<P> sv, s1, s2;
    pz<P>(sv);
    if (TANGENTS) {
        pz<P>(s1);
        pz<P>(s2);
    }
    if (lane0) sv.z[0].x = 1.f;
    // inner products (lane 0): Ss = <s,s>, P = <s,x>, G_j = <s,J_j>,
    // H_jk = <J_j,J_k>, Q_j = <J_j,x>; s_t = i f, J_jt = i df_j
    float Ss = 0.f, Pr = 0.f, Pi = 0.f, G1 = 0.f, G2 = 0.f, H11 = 0.f, H12 = 0.f, H22 = 0.f;
    float Q1r = 0.f, Q1i = 0.f, Q2r = 0.f, Q2i = 0.f;
    for (int t0 = 0; t0 < T; t0 += chunk) {
        const int nch = min(chunk, T - t0);
        __syncthreads();
        for (int idx = tid; idx < apc * nch; idx += kGnThreads) {
            const int ga = idx / nch, i = idx - ga * nch;
            const float T1 = sV[4 * ga], T2 = sV[4 * ga + 1], B1 = sV[4 * ga + 2];
            const int t = t0 + i;
            GnStep q;
            __sincosf(a.sch.alpha[t] * B1, &q.S, &q.C);
            // the relaxation folded into this step's RF is the previous
            // interval's (none before the first pulse: E = 1, dE = 0)
            const float ta = a.sch.TE[t], tr = t > 0 ? a.sch.TR[t - 1] : 0.f;
            const float r1 = 1.f / T1, r2 = 1.f / T2;
            q.E1 = __expf(-tr * r1);
            q.E2 = __expf(-tr * r2);
            q.dE1 = q.E1 * tr * r1 * r1;
            q.dE2 = q.E2 * tr * r2 * r2;
            q.Ea = __expf(-ta * r2);
            q.dEa = q.Ea * ta * r2 * r2;
            const long long vv = sI[ga];
            float2 xv = make_float2(0.f, 0.f);
            if (vv >= 0) xv = a.img[vv * a.img_stride + t];
            q.xr = xv.x;
            q.xi = xv.y;
            step_row(ga)[i] = q;
        }
        __syncthreads();
        const GnStep *qs = step_row(g);
        for (int i = 0; i < nch; i++) {
            const GnStep q = qs[i];
            const float cc = (1 + q.C) / 2, ss = (1 - q.C) / 2, hS = 0.5f * q.S;
            // RF coefficients with the previous interval's relaxation folded in
            FoldedRF k;
            k.c = make_float2(cc * q.E2, cc * q.E2);
            k.s = make_float2(ss * q.E2, ss * q.E2);
            k.nS = make_float2(-q.S * q.E1, -q.S * q.E1);
            k.hS = make_float2(hS * q.E2, hS * q.E2);
            k.C = make_float2(q.C * q.E1, q.C * q.E1);
            k.e2 = make_float2(q.E2, q.E2);
            // the signal's recovery 1 - E1 on state 0's Z, through the RF's Z column
            const float rec = 1.f - q.E1;
            if (TANGENTS) {
                // T2 tangent, relaxed first (product rule on the pre-relaxation
                // signal: F+- += dE2 f+-), then the same folded RF
                const float2 de2 = make_float2(q.dE2, q.dE2), e2 = make_float2(q.E2, q.E2);
#pragma unroll
                for (int j = 0; j < P; j++) {
                    s2.p[j] = __ffma2_rn(de2, sv.p[j], __fmul2_rn(e2, s2.p[j]));
                    s2.m[j] = __ffma2_rn(de2, sv.m[j], __fmul2_rn(e2, s2.m[j]));
                }
                // (its Z relaxes by E1 only, and F+- were relaxed above: the
                // folded RF with E2 = 1 on F+- and E1 on Z)
                FoldedRF k2;
                k2.c = make_float2(cc, cc);
                k2.s = make_float2(ss, ss);
                k2.nS = k.nS;
                k2.hS = make_float2(hS, hS);
                k2.C = k.C;
                k2.e2 = make_float2(1.f, 1.f);
                p_rf_folded<P>(s2, k2);
                // T1 tangent: the source dE1 z_signal and the recovery's
                // derivative -dE1 on state 0
                p_rf_folded_t1<P>(s1, k, sv.z, make_float2(-q.S * q.dE1, -q.S * q.dE1),
                                  make_float2(q.C * q.dE1, q.C * q.dE1));
                if (lane0) {
                    s1.p[0].x = fmaf(q.S, q.dE1, s1.p[0].x);
                    s1.m[0].x = fmaf(-q.S, q.dE1, s1.m[0].x);
                    s1.z[0].x = fmaf(-q.C, q.dE1, s1.z[0].x);
                }
            }
            p_rf_folded<P>(sv, k);
            if (lane0) {
                sv.p[0].x = fmaf(-q.S, rec, sv.p[0].x);
                sv.m[0].x = fmaf(q.S, rec, sv.m[0].x);
                sv.z[0].x = fmaf(q.C, rec, sv.z[0].x);
                // readout s_t = i Ea f+[0] (relaxation over TE)
                const float f = q.Ea * sv.p[0].x;
                Ss = fmaf(f, f, Ss);
                Pr = fmaf(f, q.xi, Pr);
                Pi = fmaf(-f, q.xr, Pi);
                if (TANGENTS) {
                    const float d1 = q.Ea * s1.p[0].x;
                    const float d2 = fmaf(q.dEa, sv.p[0].x, q.Ea * s2.p[0].x);
                    G1 = fmaf(f, d1, G1);
                    G2 = fmaf(f, d2, G2);
                    H11 = fmaf(d1, d1, H11);
                    H12 = fmaf(d1, d2, H12);
                    H22 = fmaf(d2, d2, H22);
                    Q1r = fmaf(d1, q.xi, Q1r);
                    Q1i = fmaf(-d1, q.xr, Q1i);
                    Q2r = fmaf(d2, q.xi, Q2r);
                    Q2i = fmaf(-d2, q.xr, Q2i);
                }
            }
            if (a.shift) {
                p_shift<P>(sv, gl, L, w, keep, src_up, src_dn, padded);
                if (TANGENTS) {
                    p_shift<P>(s1, gl, L, w, keep, src_up, src_dn, padded);
                    p_shift<P>(s2, gl, L, w, keep, src_up, src_dn, padded);
                }
            }
            // (the relaxation over this step's TR goes into the next RF)
        }
    }
    if (!lane0 || !active || !(Ss > 0.f)) return;
    float *mp = a.maps + v * a.nmaps;
    // PD of a unit-norm atom (what matching reports), |rho| and the B1 used,
    // from <s, x> = (pr, pi) and <s, s> = ss
    auto finish = [&](float pr, float pi, float ss) {
        const float ip = sqrtf(pr * pr + pi * pi);
        if (a.b1map && a.nmaps >= 4) mp[3] = sV[4 * g + 2];
        if (a.nmaps >= 5) mp[4] = ss > 0.f ? ip / sqrtf(ss) : 0.f;
        if (a.m0) a.m0[v] = ss > 0.f ? ip / ss : 0.f;
    };
    if (!TANGENTS) {
        finish(Pr, Pi, Ss);
        return;
    }
    const float T1 = sV[4 * g], T2 = sV[4 * g + 1];
    // variable projection: rho = P / Ss; A_jk = |rho|^2 (H_jk - G_j G_k / Ss),
    // b_j = Re(conj(rho) (Q_j - G_j P / Ss)); delta = A^-1 b
    const float rr = Pr / Ss, ri = Pi / Ss, rho2 = rr * rr + ri * ri;
    const float A11 = rho2 * (H11 - G1 * G1 / Ss), A12 = rho2 * (H12 - G1 * G2 / Ss);
    const float A22 = rho2 * (H22 - G2 * G2 / Ss);
    const float c1r = Q1r - G1 * Pr / Ss, c1i = Q1i - G1 * Pi / Ss;
    const float c2r = Q2r - G2 * Pr / Ss, c2i = Q2i - G2 * Pi / Ss;
    const float b1 = rr * c1r + ri * c1i, b2 = rr * c2r + ri * c2i;
    const float det = A11 * A22 - A12 * A12;
    float d1 = 0.f, d2 = 0.f;
    if (fabsf(det) > 0.f && isfinite(det)) {
        d1 = (A22 * b1 - A12 * b2) / det;
        d2 = (A11 * b2 - A12 * b1) / det;
    }
    if (!isfinite(d1) || !isfinite(d2)) d1 = d2 = 0.f;
    // trust region: at most max_rel_step of each parameter per iteration
    const float lim1 = a.max_rel_step * T1, lim2 = a.max_rel_step * T2;
    d1 = fminf(fmaxf(d1, -lim1), lim1);
    d2 = fminf(fmaxf(d2, -lim2), lim2);
    float n1 = T1 + d1, n2 = T2 + d2;
    n2 = fmaxf(n2, 1e-3f);
    n1 = fmaxf(n1, n2 * (1.f + 1e-4f));  // keep T1 > T2 > 0
    d1 = n1 - T1;
    d2 = n2 - T2;
    mp[0] = n1;
    mp[1] = n2;
    const bool moving = !(fabsf(d1) <= a.tol * T1 && fabsf(d2) <= a.tol * T2);
    if (a.list_out && moving) {
        a.list_out[atomicAdd(a.count_out, 1)] = (int)v;
        return;
    }
    if (a.finish) {
        // the voxel stops here: PD and M0 at the updated parameters from the
        // linear model s(T + d) = s + J d, exact to first order in d:
        // <s + J d, x> = P + Q d, ||s + J d||^2 = Ss + 2 G d + d^T H d
        const float pr = Pr + Q1r * d1 + Q2r * d2, pi = Pi + Q1i * d1 + Q2i * d2;
        const float ss = Ss + 2.f * (G1 * d1 + G2 * d2) + H11 * d1 * d1 + 2.f * H12 * d1 * d2 + H22 * d2 * d2;
        finish(pr, pi, ss);
    }
}

constexpr int kGnMaxPairs = 7;  // 8 pairs with both tangents exceed 255 registers

// Lanes per voxel and state pairs per lane for the refinement: the fewest
// padded states over power-of-two widths, then the most pairs per lane
// (fewer shuffles per state), unless another width uses more of the lanes.
// SNAPMRF_GN_LAYOUT="L,P" overrides the choice when it covers w states.
static void choose_pairs(int w, int *L, int *P) {
    if (const char *e = getenv("SNAPMRF_GN_LAYOUT")) {
        int l = 0, p = 0;
        if (sscanf(e, "%d,%d", &l, &p) == 2 && l >= 1 && l <= 32 && p >= 1 && p <= kGnMaxPairs && l * 2 * p >= w) {
            *L = l;
            *P = p;
            return;
        }
    }
    int bL = 32, bP = kGnMaxPairs, best = 1 << 30;
    for (int p = 1; p <= kGnMaxPairs; p++) {
        int l = 1;
        while (l < 32 && l * 2 * p < w) l *= 2;
        if (l * 2 * p < w) continue;
        if (l * 2 * p <= best) {
            best = l * 2 * p;
            bL = l;
            bP = p;
        }
    }
    // A group width that is not a power of two when it fills the warp's
    // lanes with more useful states: useful fraction (32 / L) w / (32 * 2P).
    // C1 (w = 50): 5 lanes x 5 pairs (6 voxels per warp, 94 %) against 4 x 7
    // (8 voxels, 89 %): one pass 5.97 against 6.11 ms, the same maps.
    auto useful = [&](int l, int p) { return (double)(32 / l) * w / (32.0 * 2 * p); };
    double bu = useful(bL, bP);
    for (int l = 1; l <= 32; l++)
        for (int p = 1; p <= kGnMaxPairs; p++)
            if (l * 2 * p >= w && useful(l, p) > bu + 1e-9) {
                bu = useful(l, p);
                bL = l;
                bP = p;
            }
    *L = bL;
    *P = bP;
}

// --------------------------------------------------------------------------
// Cramer-Rao bound of (T1, T2) and its gradient with respect to the schedule
// --------------------------------------------------------------------------
// Per tissue the signal f (s = i f) and its tangents f1 = df/dT1, f2 = df/dT2
// give the Fisher matrix M = V^T V of V = [f1, f2, f] (unit noise, a real
// proton-density factor as the nuisance parameter), and the loss
//   L = [M^-1]_00 / T1^2 + [M^-1]_11 / T2^2,
// the sum of the normalised CRBs of T1 and T2.  dL/dV = 2 V G with
// G = -M^-1 W M^-1, W = diag(1/T1^2, 1/T2^2, 0); these gradients are carried
// back through the recursion with its tangents (three adjoint streams) to
// dL/dalpha_t.  Relaxation over TR after the shift, readout E2(TE) f+[0] after
// the RF, as in the Gauss-Newton kernel.
struct CrbArgs {
    Schedule sch;
    const float *params;      // [n][nparams]: T1, T2, (B0), B1
    int nparams;
    long long n;
    int w, L, shift;
    float *fvec;              // [n][3][T]: f, f1, f2
    const float *gvec;        // [n][3][T]: dL/df, dL/df1, dL/df2
    float *ckpt;              // [n][nckpt][9][L*S]
    float *seg;               // [n][C][9][L*S]
    float *galpha;            // [n][T]: dL/dalpha_t per tissue
    int C, nckpt;
};

// Relaxation constants of step t: E1, E2 over TR, their T1 / T2 derivatives,
// and E2 over TE (the readout) with its T2 derivative.
struct CrbStep {
    float E1, E2, dE1, dE2, Ea, dEa;
};

__device__ __forceinline__ CrbStep crb_step(const Schedule &sc, int t, float T1, float T2) {
    CrbStep c;
    const float tr = sc.TR[t], te = sc.TE[t];
    c.E1 = expf(-tr / T1);
    c.E2 = expf(-tr / T2);
    c.dE1 = c.E1 * tr / (T1 * T1);
    c.dE2 = c.E2 * tr / (T2 * T2);
    c.Ea = expf(-te / T2);
    c.dEa = c.Ea * te / (T2 * T2);
    return c;
}

template <int S>
struct Aug {
    St<S> v, d1, d2;
};

template <int S>
__device__ __forceinline__ void aug_zero(Aug<S> &x) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        x.v.p[j] = x.v.m[j] = x.v.z[j] = 0.f;
        x.d1.p[j] = x.d1.m[j] = x.d1.z[j] = 0.f;
        x.d2.p[j] = x.d2.m[j] = x.d2.z[j] = 0.f;
    }
}

template <int S>
__device__ __forceinline__ void aug_store(float *dst, int L, int gl, const Aug<S> &x) {
    const int LS3 = 3 * L * S;
    store_state<S>(dst, L, gl, x.v);
    store_state<S>(dst + LS3, L, gl, x.d1);
    store_state<S>(dst + 2 * LS3, L, gl, x.d2);
}

template <int S>
__device__ __forceinline__ void aug_load(const float *src, int L, int gl, Aug<S> &x) {
    const int LS3 = 3 * L * S;
    load_state<S>(src, L, gl, x.v);
    load_state<S>(src + LS3, L, gl, x.d1);
    load_state<S>(src + 2 * LS3, L, gl, x.d2);
}

// One step forward: RF, readout (f, f1, f2 on the group's first lane), shift,
// relaxation over TR with the product rule for the tangents.
template <int S>
__device__ __forceinline__ void aug_step(Aug<S> &x, const StepRF &r, const CrbStep &c, bool lane0, int gl, int L,
                                         int w, int shift, float *f3) {
    rf_fwd<S>(x.v, r);
    rf_fwd<S>(x.d1, r);
    rf_fwd<S>(x.d2, r);
    if (f3 && lane0) {
        f3[0] = c.Ea * x.v.p[0];
        f3[1] = c.Ea * x.d1.p[0];
        f3[2] = fmaf(c.dEa, x.v.p[0], c.Ea * x.d2.p[0]);
    }
    if (shift) {
        shift_fwd<S>(x.v, gl, L, w);
        shift_fwd<S>(x.d1, gl, L, w);
        shift_fwd<S>(x.d2, gl, L, w);
    }
#pragma unroll
    for (int j = 0; j < S; j++) {
        x.d1.p[j] *= c.E2;
        x.d1.m[j] *= c.E2;
        x.d1.z[j] = fmaf(c.dE1, x.v.z[j], c.E1 * x.d1.z[j]);
        x.d2.p[j] = fmaf(c.dE2, x.v.p[j], c.E2 * x.d2.p[j]);
        x.d2.m[j] = fmaf(c.dE2, x.v.m[j], c.E2 * x.d2.m[j]);
        x.d2.z[j] *= c.E1;
    }
    if (lane0) x.d1.z[0] -= c.dE1;
    relax_fwd<S>(x.v, c.E1, c.E2, lane0);
}

template <int S>
__global__ void __launch_bounds__(kThreads) crb_forward_kernel(CrbArgs a) {
    const int L = a.L, LS = L * S;
    const int g = threadIdx.x / L, gl = threadIdx.x % L;
    const long long tis = (long long)blockIdx.x * (kThreads / L) + g;
    const bool active = tis < a.n;
    const long long at = active ? tis : 0;
    const bool lane0 = gl == 0;
    const float *pp = a.params + at * a.nparams;
    const float T1 = pp[0], T2 = pp[1], B1 = pp[3];
    const int T = a.sch.nreps;
    float *ck = a.ckpt + at * (long long)a.nckpt * 9 * LS;
    float *fv = a.fvec + at * 3LL * T;
    Aug<S> x;
    aug_zero<S>(x);
    if (lane0) x.v.z[0] = 1.f;
    for (int t = 0; t < T; t++) {
        if (t % a.C == 0 && active) aug_store<S>(ck + (long long)(t / a.C) * 9 * LS, L, gl, x);
        float f3[3];
        aug_step<S>(x, step_rf(a.sch.alpha[t] * B1), crb_step(a.sch, t, T1, T2), lane0, gl, L, a.w, a.shift, f3);
        if (lane0 && active) {
            fv[t] = f3[0];
            fv[T + t] = f3[1];
            fv[2 * T + t] = f3[2];
        }
    }
}

// One block per tissue: the Fisher matrix, the loss and dL/d(f, f1, f2).
__global__ void crb_loss_kernel(const float *fvec, float *gvec, float *loss, const float *params, int nparams,
                                int T) {
    const long long tis = blockIdx.x;
    const float *f = fvec + tis * 3LL * T, *f1 = f + T, *f2 = f + 2 * T;
    double acc[6] = {0, 0, 0, 0, 0, 0};  // M00 M01 M02 M11 M12 M22 over V = [f1, f2, f]
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const double a = f1[t], b = f2[t], c = f[t];
        acc[0] += a * a;
        acc[1] += a * b;
        acc[2] += a * c;
        acc[3] += b * b;
        acc[4] += b * c;
        acc[5] += c * c;
    }
    __shared__ double red[6][32];
    __shared__ double Gs[9];
    __shared__ int bad;
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m[6];
        for (int k = 0; k < 6; k++) {
            m[k] = 0;
            for (int i = 0; i < (int)(blockDim.x / 32); i++) m[k] += red[k][i];
        }
        const double M[3][3] = {{m[0], m[1], m[2]}, {m[1], m[3], m[4]}, {m[2], m[4], m[5]}};
        // inverse by cofactors
        double C[3][3];
        C[0][0] = M[1][1] * M[2][2] - M[1][2] * M[2][1];
        C[0][1] = M[1][2] * M[2][0] - M[1][0] * M[2][2];
        C[0][2] = M[1][0] * M[2][1] - M[1][1] * M[2][0];
        C[1][0] = M[0][2] * M[2][1] - M[0][1] * M[2][2];
        C[1][1] = M[0][0] * M[2][2] - M[0][2] * M[2][0];
        C[1][2] = M[0][1] * M[2][0] - M[0][0] * M[2][1];
        C[2][0] = M[0][1] * M[1][2] - M[0][2] * M[1][1];
        C[2][1] = M[0][2] * M[1][0] - M[0][0] * M[1][2];
        C[2][2] = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        const double det = M[0][0] * C[0][0] + M[0][1] * C[0][1] + M[0][2] * C[0][2];
        bad = !(fabs(det) > 0.0) || !isfinite(det);
        const double T1 = params[tis * nparams], T2 = params[tis * nparams + 1];
        const double Wd[3] = {1.0 / (T1 * T1), 1.0 / (T2 * T2), 0.0};
        double Mi[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Mi[i][j] = C[j][i] / det;
        loss[tis] = bad ? __int_as_float(0x7fc00000) : (float)(Mi[0][0] * Wd[0] + Mi[1][1] * Wd[1]);
        // G = -Mi W Mi
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double g = 0;
                for (int k = 0; k < 3; k++) g += Mi[i][k] * Wd[k] * Mi[k][j];
                Gs[3 * i + j] = -g;
            }
    }
    __syncthreads();
    float *g = gvec + tis * 3LL * T;  // [dL/df, dL/df1, dL/df2]
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const double a = f1[t], b = f2[t], c = f[t];
        const double g1 = 2 * (a * Gs[0] + b * Gs[3] + c * Gs[6]);
        const double g2 = 2 * (a * Gs[1] + b * Gs[4] + c * Gs[7]);
        const double g0 = 2 * (a * Gs[2] + b * Gs[5] + c * Gs[8]);
        g[t] = bad ? 0.f : (float)g0;
        g[T + t] = bad ? 0.f : (float)g1;
        g[2 * T + t] = bad ? 0.f : (float)g2;
    }
}

// lambda^T (dR/da) x for one stream pair (the RF derivative as in the adjoint).
template <int S>
__device__ __forceinline__ float rf_dadj(const St<S> &l, const St<S> &x0, const StepRF &r) {
    float ga = 0.f;
#pragma unroll
    for (int j = 0; j < S; j++) {
        const float p = x0.p[j], m = x0.m[j], q = x0.z[j];
        const float dp = -r.hS * p + r.hS * m - r.C * q;
        const float dm = r.hS * p - r.hS * m + r.C * q;
        const float dz = 0.5f * r.C * p - 0.5f * r.C * m - r.S * q;
        ga += l.p[j] * dp + l.m[j] * dm + l.z[j] * dz;
    }
    return ga;
}

template <int S>
__device__ __forceinline__ void rf_transpose(St<S> &l, const StepRF &r) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        const float lp = l.p[j], lm = l.m[j], lz = l.z[j];
        l.p[j] = r.c * lp + r.s * lm + r.hS * lz;
        l.m[j] = r.s * lp + r.c * lm - r.hS * lz;
        l.z[j] = -r.S * lp + r.S * lm + r.C * lz;
    }
}

template <int S>
__global__ void __launch_bounds__(kThreads) crb_adjoint_kernel(CrbArgs a) {
    const int L = a.L, LS = L * S;
    const int g = threadIdx.x / L, gl = threadIdx.x % L;
    const long long tis = (long long)blockIdx.x * (kThreads / L) + g;
    const bool active = tis < a.n;
    const long long at = active ? tis : 0;
    const bool lane0 = gl == 0;
    const float *pp = a.params + at * a.nparams;
    const float T1 = pp[0], T2 = pp[1], B1 = pp[3];
    const int T = a.sch.nreps, w = a.w;
    const float *ck = a.ckpt + at * (long long)a.nckpt * 9 * LS;
    float *sg = a.seg + at * (long long)a.C * 9 * LS;
    const float *gv = a.gvec + at * 3LL * T;
    Aug<S> l, x;
    aug_zero<S>(l);
    for (int c = a.nckpt - 1; c >= 0; c--) {
        const int t0 = c * a.C, t1 = min(T, t0 + a.C);
        if (active) aug_load<S>(ck + (long long)c * 9 * LS, L, gl, x);
        else aug_zero<S>(x);
        for (int t = t0; t < t1; t++) {
            if (active) aug_store<S>(sg + (long long)(t - t0) * 9 * LS, L, gl, x);
            aug_step<S>(x, step_rf(a.sch.alpha[t] * B1), crb_step(a.sch, t, T1, T2), lane0, gl, L, w, a.shift,
                        nullptr);
        }
        __syncwarp();
        for (int t = t1 - 1; t >= t0; t--) {
            Aug<S> x0;
            if (active) aug_load<S>(sg + (long long)(t - t0) * 9 * LS, L, gl, x0);
            else aug_zero<S>(x0);
            const CrbStep cs = crb_step(a.sch, t, T1, T2);
            const StepRF r = step_rf(a.sch.alpha[t] * B1);
            // relaxation over TR, transposed: the signal's adjoint gathers the
            // tangents' product-rule terms
#pragma unroll
            for (int j = 0; j < S; j++) {
                l.v.p[j] = fmaf(cs.dE2, l.d2.p[j], cs.E2 * l.v.p[j]);
                l.v.m[j] = fmaf(cs.dE2, l.d2.m[j], cs.E2 * l.v.m[j]);
                l.v.z[j] = fmaf(cs.dE1, l.d1.z[j], cs.E1 * l.v.z[j]);
                l.d1.p[j] *= cs.E2;
                l.d1.m[j] *= cs.E2;
                l.d1.z[j] *= cs.E1;
                l.d2.p[j] *= cs.E2;
                l.d2.m[j] *= cs.E2;
                l.d2.z[j] *= cs.E1;
            }
            if (a.shift) {
                shift_adj<S>(l.v, gl, L, w);
                shift_adj<S>(l.d1, gl, L, w);
                shift_adj<S>(l.d2, gl, L, w);
            }
            if (lane0 && active) {
                const float g0 = gv[t], g1 = gv[T + t], g2 = gv[2 * T + t];
                l.v.p[0] += fmaf(cs.Ea, g0, cs.dEa * g2);
                l.d1.p[0] += cs.Ea * g1;
                l.d2.p[0] += cs.Ea * g2;
            }
            float ga = rf_dadj<S>(l.v, x0.v, r) + rf_dadj<S>(l.d1, x0.d1, r) + rf_dadj<S>(l.d2, x0.d2, r);
            rf_transpose<S>(l.v, r);
            rf_transpose<S>(l.d1, r);
            rf_transpose<S>(l.d2, r);
            ga = group_sum(ga, L);
            if (lane0 && active) a.galpha[at * T + t] = ga * B1;
        }
        __syncwarp();
    }
}

static void choose(int w, int *L, int *S) {
    int bL = 32, bS = kMaxS, pad = 1 << 30;
    for (int s = kMaxS; s >= 1; s--)
        for (int l = 1; l <= 32; l *= 2)
            if (l * s >= w) {
                if (l * s - w < pad) { pad = l * s - w; bL = l; bS = s; }
                break;
            }
    *L = bL;
    *S = bS;
}

#define SNAPMRF_GRAD_DISPATCH(KERNEL, S, GRID, ST, ARGS)                   \
    switch (S) {                                                          \
    case 1: KERNEL<1><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 2: KERNEL<2><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 3: KERNEL<3><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 4: KERNEL<4><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 5: KERNEL<5><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 6: KERNEL<6><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    case 7: KERNEL<7><<<GRID, kThreads, 0, ST>>>(ARGS); break;            \
    default: KERNEL<8><<<GRID, kThreads, 0, ST>>>(ARGS); break;           \
    }

#define SNAPMRF_GN_DISPATCH_PAD(P, B, PAD, GRID, SMEM, ST, ARGS, CHUNK)                   \
    switch (P) {                                                                         \
    case 1: gn_kernel<1, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    case 2: gn_kernel<2, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    case 3: gn_kernel<3, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    case 4: gn_kernel<4, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    case 5: gn_kernel<5, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    case 6: gn_kernel<6, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;      \
    default: gn_kernel<7, B, PAD><<<GRID, kGnThreads, SMEM, ST>>>(ARGS, CHUNK); break;     \
    }
// (the layout's padding, L * 2P > w, picks the kernel that clears slot w)
#define SNAPMRF_GN_DISPATCH(P, B, GRID, SMEM, ST, ARGS, CHUNK)                              \
    do {                                                                                 \
        if ((ARGS).L * 2 * (P) > (ARGS).w) {                                             \
            SNAPMRF_GN_DISPATCH_PAD(P, B, true, GRID, SMEM, ST, ARGS, CHUNK);             \
        } else {                                                                         \
            SNAPMRF_GN_DISPATCH_PAD(P, B, false, GRID, SMEM, ST, ARGS, CHUNK);            \
        }                                                                                \
    } while (0)

// Resident CTAs per SM of gn_kernel<P, true> with `smem` bytes.
static cudaError_t gn_occupancy(int P, size_t smem, int *per_sm) {
    switch (P) {
    case 1: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<1, true>, kGnThreads, smem);
    case 2: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<2, true>, kGnThreads, smem);
    case 3: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<3, true>, kGnThreads, smem);
    case 4: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<4, true>, kGnThreads, smem);
    case 5: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<5, true>, kGnThreads, smem);
    case 6: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<6, true>, kGnThreads, smem);
    default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, gn_kernel<7, true>, kGnThreads, smem);
    }
}

// Schedule of the real-valued recursion on the device; fails unless every
// RF phase is 0.
static int upload_schedule(DeviceScratch &buf, Schedule *sc, const float *h_mrf, size_t nreps, size_t NREPS,
                           cudaStream_t st, const char *who) {
    for (size_t t = 0; t < nreps; t++)
        if (h_mrf[NREPS + t] != 0.f)
            SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "%s: RF phases must all be 0 (real-valued recursion)", who);
    SNAPMRF_CUDA(buf.alloc(3 * nreps * sizeof(float), st));
    float *h = static_cast<float *>(stage_acquire(3 * nreps * sizeof(float)));
    if (!h) SNAPMRF_FAIL(SNAPMRF_ERR_ALLOC, "%s: cannot allocate a pinned staging buffer", who);
    memcpy(h, h_mrf, nreps * sizeof(float));
    memcpy(h + nreps, h_mrf + 2 * NREPS, nreps * sizeof(float));
    memcpy(h + 2 * nreps, h_mrf + 3 * NREPS, nreps * sizeof(float));
    SNAPMRF_CUDA(stage_upload(buf.ptr, h, 3 * nreps * sizeof(float), st));
    SNAPMRF_CUDA(stage_release(st));
    sc->alpha = buf.as<float>();
    sc->TR = sc->alpha + nreps;
    sc->TE = sc->TR + nreps;
    sc->nreps = (int)nreps;
    return SNAPMRF_OK;
}

// 1 for epg_fisp (dephasing shift every TR), 0 for epg_sr, -1 otherwise.
static int echo_shift(const char *echo_type) {
    if (echo_type && !strcmp(echo_type, "epg_fisp")) return 1;
    if (echo_type && !strcmp(echo_type, "epg_sr")) return 0;
    return -1;
}

}  // namespace grad
}  // namespace snapmrf

namespace snapmrf {
// epg_ssfp_grad.cu
int epg_adjoint_ssfp(const float *d_params, int nparams, const float *h_mrf, size_t nreps, size_t NREPS,
                     size_t natoms, int nstates, const float *d_grad_signal, float *d_signal, float *d_grad_params,
                     float *galpha_atoms, int checkpoint_every, cudaStream_t st);
int refine_gn_ssfp(float *d_maps, int nmaps, const float *img, size_t img_stride, const float *d_b1map,
                   const float *h_mrf, size_t nreps, size_t NREPS, size_t nvoxels, int nstates, int iterations,
                   float max_rel_step, float tol, float *d_m0, cudaStream_t st);
}

using namespace snapmrf;
using namespace snapmrf::grad;

extern "C" int snapmrf_epg_adjoint(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                                   size_t NREPS, size_t natoms, int nstates, const char *echo_type,
                                   const float *d_grad_signal, float *d_signal, float *d_grad_params,
                                   float *d_grad_alpha, float *d_grad_alpha_atoms, int checkpoint_every,
                                   void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_params || !h_mrf || !d_grad_signal || !d_grad_params)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "epg_adjoint: null pointer");
    if (nparams < 4 || nreps == 0 || nreps > NREPS || natoms == 0 || nstates < 1 || nstates > 32 * kMaxS)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "epg_adjoint: bad sizes");
    if (nreps > 0x7fffffff) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "epg_adjoint: too many time points");
    if (echo_type && !strcmp(echo_type, "epg_ssfp")) {
        // the complex bSSFP recursion (epg_ssfp_grad.cu); the per-atom
        // schedule gradient goes to the caller's buffer or scratch, then the
        // same deterministic column sum
        DeviceScratch gbuf;
        float *gat = d_grad_alpha_atoms;
        if (!gat) {
            SNAPMRF_CUDA(gbuf.alloc((size_t)natoms * nreps * sizeof(float) +
                                    (d_grad_alpha ? (size_t)kSplits * nreps * sizeof(float) : 0), st));
            gat = gbuf.as<float>();
        }
        int rc = epg_adjoint_ssfp(d_params, nparams, h_mrf, nreps, NREPS, natoms, nstates, d_grad_signal, d_signal,
                                  d_grad_params, gat, checkpoint_every, st);
        if (rc) return rc;
        if (d_grad_alpha) {
            DeviceScratch pbuf;
            float *partial = nullptr;
            if (d_grad_alpha_atoms) {
                SNAPMRF_CUDA(pbuf.alloc((size_t)kSplits * nreps * sizeof(float), st));
                partial = pbuf.as<float>();
            } else {
                partial = gat + (size_t)natoms * nreps;
            }
            dim3 pg((unsigned)((nreps + 127) / 128), kSplits);
            sum_columns_partial_kernel<<<pg, 128, 0, st>>>(partial, gat, (long long)natoms, (int)nreps);
            SNAPMRF_LAUNCH_CHECK();
            sum_columns_final_kernel<<<(unsigned)((nreps + 127) / 128), 128, 0, st>>>(d_grad_alpha, partial,
                                                                                    (int)nreps);
            SNAPMRF_LAUNCH_CHECK();
        }
        return SNAPMRF_OK;
    }
    const int shift = echo_shift(echo_type);
    if (shift < 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_ECHO_TYPE, "epg_adjoint: echo type must be epg_fisp, epg_sr or epg_ssfp");
    DeviceScratch sbuf;
    Schedule sc;
    int rc = upload_schedule(sbuf, &sc, h_mrf, nreps, NREPS, st, "epg_adjoint");
    if (rc) return rc;
    int L, S;
    choose(nstates, &L, &S);
    int C = checkpoint_every > 0 ? checkpoint_every : (int)std::max(1.0, std::ceil(std::sqrt((double)nreps)));
    int nckpt = (int)((nreps + C - 1) / C);
    const long long LS = (long long)L * S;
    DeviceScratch work;
    size_t ck = (size_t)natoms * nckpt * 3 * LS, sg = (size_t)natoms * C * 3 * LS;
    size_t ga = d_grad_alpha_atoms ? 0 : (size_t)natoms * nreps;
    size_t part = d_grad_alpha ? (size_t)kSplits * nreps : 0;
    SNAPMRF_CUDA(work.alloc((ck + sg + ga + part) * sizeof(float), st));
    AdjArgs a;
    a.sch = sc;
    a.params = d_params;
    a.nparams = nparams;
    a.n = (long long)natoms;
    a.w = nstates;
    a.L = L;
    a.shift = shift;
    a.gsig = reinterpret_cast<const float2 *>(d_grad_signal);
    a.sig = reinterpret_cast<float2 *>(d_signal);
    a.gparams = d_grad_params;
    a.ckpt = work.as<float>();
    a.seg = a.ckpt + ck;
    a.galpha_atoms = d_grad_alpha_atoms ? d_grad_alpha_atoms : a.seg + sg;
    a.C = C;
    a.nckpt = nckpt;
    const int apc = kThreads / L;
    dim3 grid((unsigned)((natoms + apc - 1) / apc));
    SNAPMRF_GRAD_DISPATCH(adjoint_kernel, S, grid, st, a);
    SNAPMRF_LAUNCH_CHECK();
    if (d_grad_alpha) {
        float *partial = a.ckpt + ck + sg + ga;
        dim3 pg((unsigned)((nreps + 127) / 128), kSplits);
        sum_columns_partial_kernel<<<pg, 128, 0, st>>>(partial, a.galpha_atoms, (long long)natoms, (int)nreps);
        SNAPMRF_LAUNCH_CHECK();
        sum_columns_final_kernel<<<(unsigned)((nreps + 127) / 128), 128, 0, st>>>(d_grad_alpha, partial, (int)nreps);
        SNAPMRF_LAUNCH_CHECK();
    }
    return SNAPMRF_OK;
}

extern "C" int snapmrf_refine_gn(float *d_maps, int nmaps, const float *img, size_t img_stride,
                                 const float *d_b1map, const float *h_mrf, size_t nreps, size_t NREPS,
                                 size_t nvoxels, int nstates, const char *echo_type, int iterations,
                                 float max_rel_step, float tol, float *d_m0, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_maps || !img || !h_mrf) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_gn: null pointer");
    if (nmaps < 2 || nreps == 0 || nreps > NREPS || nvoxels == 0 || nstates < 1 ||
        nstates > 32 * 2 * kGnMaxPairs || iterations < 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_gn: bad sizes");
    if (nreps > 0x7fffffff || nvoxels > 0x7fffffff)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "refine_gn: too many time points or voxels");
    if (!img_stride) img_stride = nreps;
    if (img_stride < nreps) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_gn: img_stride < nreps");
    if (echo_type && !strcmp(echo_type, "epg_ssfp"))
        return refine_gn_ssfp(d_maps, nmaps, img, img_stride, d_b1map, h_mrf, nreps, NREPS, nvoxels, nstates,
                              iterations, max_rel_step, tol, d_m0, st);
    const int shift = echo_shift(echo_type);
    if (shift < 0)
        SNAPMRF_FAIL(SNAPMRF_ERR_ECHO_TYPE, "refine_gn: echo type must be epg_fisp, epg_sr or epg_ssfp");
    DeviceScratch sbuf;
    Schedule sc;
    int rc = upload_schedule(sbuf, &sc, h_mrf, nreps, NREPS, st, "refine_gn");
    if (rc) return rc;
    int L, P;
    choose_pairs(nstates, &L, &P);
    GnArgs a;
    a.sch = sc;
    a.nvox = (long long)nvoxels;
    a.w = nstates;
    a.L = L;
    a.shift = shift;
    a.img = reinterpret_cast<const float2 *>(img);
    a.img_stride = (long long)img_stride;
    a.maps = d_maps;
    a.nmaps = nmaps;
    a.b1map = d_b1map;
    a.m0 = d_m0;
    a.max_rel_step = max_rel_step > 0.f ? max_rel_step : 0.2f;
    a.tol = tol;
    a.list_in = a.count_in = nullptr;
    a.list_out = a.count_out = nullptr;
    a.part = 0;
    a.bulk_apc = 1;
    a.round_groups = 1;
    // voxel lists of the early exit: two lists and two counters
    const bool early = tol > 0.f && iterations > 1;
    DeviceScratch lists;
    int *lst[2] = {nullptr, nullptr}, *cnt[2] = {nullptr, nullptr};
    if (early) {
        SNAPMRF_CUDA(lists.alloc((2 * nvoxels + 2) * sizeof(int), st));
        lst[0] = lists.as<int>();
        lst[1] = lst[0] + nvoxels;
        cnt[0] = lst[1] + nvoxels;
        cnt[1] = cnt[0] + 1;
    }
    const int apc = gn_voxels_per_cta(L);
    // steps staged per chunk: at most kGnChunk, within 48 KB of shared memory
    auto smem_for = [&](int apc_, int *chunk_) {
        const size_t fixed = (size_t)apc_ * (4 * sizeof(float) + sizeof(long long) + 16);
        *chunk_ = (int)std::min<size_t>(kGnChunk, (48 * 1024 - fixed) / ((size_t)apc_ * sizeof(GnStep)));
        return (size_t)apc_ * *chunk_ * sizeof(GnStep) + fixed;
    };
    int chunk = 0;
    const size_t smem = smem_for(apc, &chunk);
    dim3 grid((unsigned)((nvoxels + apc - 1) / apc));
    // The tail of the list: the bulk launch takes whole rounds of resident
    // CTAs, the voxels past the last whole round go to a launch with 16 lanes
    // per voxel (32 from 8 up; a quarter of the work per lane at L = 4), so the last
    // round does not run nearly empty (C1: 7,200 groups on 1,184 resident
    // CTAs were 6.08 rounds).  Same operations per state, same results.
    // SNAPMRF_GN_TAIL=0 turns it off.
    GnArgs t = a;
    int P_tail = 0, chunk_tail = 0;
    size_t smem_tail = 0;
    dim3 grid_tail(0);
    {
        const char *e = getenv("SNAPMRF_GN_TAIL");
        // SNAPMRF_GN_TAIL_LANES overrides the tail's lanes per voxel (tuning)
        const char *el = getenv("SNAPMRF_GN_TAIL_LANES");
        int L_tail = L < 8 ? 16 : 32;
        if (el && atoi(el) > L && atoi(el) <= 32) L_tail = atoi(el);
        P_tail = (nstates + 2 * L_tail - 1) / (2 * L_tail);
        int dev = 0, sms = 0, per_sm = 0;
        if (!(e && atoi(e) == 0) && L_tail > L && P_tail >= 1 && P_tail <= kGnMaxPairs &&
            cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            gn_occupancy(P, smem, &per_sm) == cudaSuccess && sms > 0 && per_sm > 0) {
            const int apc_tail = gn_voxels_per_cta(L_tail);
            smem_tail = smem_for(apc_tail, &chunk_tail);
            a.part = 1;
            a.bulk_apc = apc;
            a.round_groups = (long long)sms * per_sm;
            t = a;
            t.part = 2;
            t.L = L_tail;
            const long long tail_max = std::min<long long>((long long)nvoxels, (a.round_groups + 1) * apc);
            grid_tail = dim3((unsigned)((tail_max + apc_tail - 1) / apc_tail));
        } else {
            cudaGetLastError();
        }
    }
    // PD, M0 and the B1 column: written by each voxel in the pass where it
    // stops (early exit, or the last iteration); with no iteration at all, by
    // one value-only pass
    const bool outputs = nmaps >= 5 || d_m0 || (d_b1map && nmaps >= 4);
    for (int it = 0; it < iterations; it++) {
        const bool last = it + 1 == iterations;
        a.list_in = a.count_in = nullptr;
        a.list_out = a.count_out = nullptr;
        if (early) {
            a.list_in = it == 0 ? nullptr : lst[(it - 1) & 1];
            a.count_in = it == 0 ? nullptr : cnt[(it - 1) & 1];
            a.list_out = last ? nullptr : lst[it & 1];
            a.count_out = last ? nullptr : cnt[it & 1];
            if (a.count_out) SNAPMRF_CUDA(cudaMemsetAsync(a.count_out, 0, sizeof(int), st));
        }
        a.finish = outputs && (early || last) ? 1 : 0;
        SNAPMRF_GN_DISPATCH(P, true, grid, smem, st, a, chunk);
        SNAPMRF_LAUNCH_CHECK();
        if (a.part) {
            t.list_in = a.list_in;
            t.count_in = a.count_in;
            t.list_out = a.list_out;
            t.count_out = a.count_out;
            t.finish = a.finish;
            SNAPMRF_GN_DISPATCH(P_tail, true, grid_tail, smem_tail, st, t, chunk_tail);
            SNAPMRF_LAUNCH_CHECK();
        }
    }
    if (outputs && iterations == 0) {
        a.list_in = a.count_in = nullptr;
        a.list_out = a.count_out = nullptr;
        a.finish = 1;
        a.part = 0;
        SNAPMRF_GN_DISPATCH(P, false, grid, smem, st, a, chunk);
        SNAPMRF_LAUNCH_CHECK();
    }
    return SNAPMRF_OK;
}

// Forward mode: the signal and its T1 / T2 tangents, by the CRB's forward
// pass (the augmented recursion of aug_step) with one stored state per atom
// (the state at t = 0; nothing reads it back).
extern "C" int snapmrf_epg_jvp(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                               size_t NREPS, size_t natoms, int nstates, const char *echo_type, float *d_out,
                               void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_params || !h_mrf || !d_out) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "epg_jvp: null pointer");
    if (nparams < 4 || nreps == 0 || nreps > NREPS || natoms == 0 || nstates < 1 || nstates > 32 * kMaxS)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "epg_jvp: bad sizes");
    if (nreps > 0x7fffffff || natoms > 0x7fffffff)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "epg_jvp: too many time points or atoms");
    const int shift = echo_shift(echo_type);
    if (shift < 0) SNAPMRF_FAIL(SNAPMRF_ERR_ECHO_TYPE, "epg_jvp: echo type must be epg_fisp or epg_sr");
    DeviceScratch sbuf;
    Schedule sc;
    int rc = upload_schedule(sbuf, &sc, h_mrf, nreps, NREPS, st, "epg_jvp");
    if (rc) return rc;
    int L, S;
    choose(nstates, &L, &S);
    const size_t LS = (size_t)L * S;
    DeviceScratch work;
    SNAPMRF_CUDA(work.alloc(natoms * 9 * LS * sizeof(float), st));
    CrbArgs a;
    a.sch = sc;
    a.params = d_params;
    a.nparams = nparams;
    a.n = (long long)natoms;
    a.w = nstates;
    a.L = L;
    a.shift = shift;
    a.fvec = d_out;
    a.gvec = nullptr;
    a.ckpt = work.as<float>();
    a.seg = nullptr;
    a.galpha = nullptr;
    a.C = (int)nreps;  // one checkpoint, at t = 0
    a.nckpt = 1;
    const int apc = kThreads / L;
    dim3 grid((unsigned)((natoms + apc - 1) / apc));
    SNAPMRF_GRAD_DISPATCH(crb_forward_kernel, S, grid, st, a);
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}

extern "C" int snapmrf_crb_gradient(const float *d_params, int nparams, const float *h_mrf, size_t nreps,
                                    size_t NREPS, size_t ntissues, int nstates, const char *echo_type, float *d_loss,
                                    float *d_grad_alpha, float *d_signals, int checkpoint_every, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_params || !h_mrf || !d_loss || !d_grad_alpha) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "crb_gradient: null pointer");
    if (nparams < 4 || nreps == 0 || nreps > NREPS || ntissues == 0 || nstates < 1 || nstates > 32 * kMaxS)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "crb_gradient: bad sizes");
    if (nreps > 0x7fffffff || ntissues > 0x7fffffff)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "crb_gradient: too many time points or tissues");
    const int shift = echo_shift(echo_type);
    if (shift < 0) SNAPMRF_FAIL(SNAPMRF_ERR_ECHO_TYPE, "crb_gradient: echo type must be epg_fisp or epg_sr");
    DeviceScratch sbuf;
    Schedule sc;
    int rc = upload_schedule(sbuf, &sc, h_mrf, nreps, NREPS, st, "crb_gradient");
    if (rc) return rc;
    int L, S;
    choose(nstates, &L, &S);
    const int C = checkpoint_every > 0 ? checkpoint_every : (int)std::max(1.0, std::ceil(std::sqrt((double)nreps)));
    const int nckpt = (int)((nreps + C - 1) / C);
    const long long LS = (long long)L * S;
    const size_t n = ntissues;
    const size_t nf = n * 3 * nreps, ck = n * (size_t)nckpt * 9 * LS, sg = n * (size_t)C * 9 * LS,
                 ga = n * nreps, part = (size_t)kSplits * nreps;
    DeviceScratch work;
    SNAPMRF_CUDA(work.alloc((2 * nf + ck + sg + ga + part) * sizeof(float), st));
    float *base = work.as<float>();
    CrbArgs a;
    a.sch = sc;
    a.params = d_params;
    a.nparams = nparams;
    a.n = (long long)n;
    a.w = nstates;
    a.L = L;
    a.shift = shift;
    a.fvec = d_signals ? d_signals : base;
    a.gvec = base + nf;
    a.ckpt = base + 2 * nf;
    a.seg = a.ckpt + ck;
    a.galpha = a.seg + sg;
    a.C = C;
    a.nckpt = nckpt;
    float *partial = a.galpha + ga;
    const int apc = kThreads / L;
    dim3 grid((unsigned)((n + apc - 1) / apc));
    SNAPMRF_GRAD_DISPATCH(crb_forward_kernel, S, grid, st, a);
    SNAPMRF_LAUNCH_CHECK();
    crb_loss_kernel<<<(unsigned)n, 256, 0, st>>>(a.fvec, base + nf, d_loss, d_params, nparams, (int)nreps);
    SNAPMRF_LAUNCH_CHECK();
    SNAPMRF_GRAD_DISPATCH(crb_adjoint_kernel, S, grid, st, a);
    SNAPMRF_LAUNCH_CHECK();
    dim3 pg((unsigned)((nreps + 127) / 128), kSplits);
    sum_columns_partial_kernel<<<pg, 128, 0, st>>>(partial, a.galpha, (long long)n, (int)nreps);
    SNAPMRF_LAUNCH_CHECK();
    sum_columns_final_kernel<<<(unsigned)((nreps + 127) / 128), 128, 0, st>>>(d_grad_alpha, partial, (int)nreps);
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}
