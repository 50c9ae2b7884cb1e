// Gauss-Newton refinement on the complex bSSFP recursion (epg_ssfp,
// src/functions.cu:935-1019): RF with the alternating phase, relaxation at
// TE, B0 precession, readout, B0 precession over TR - TE, dephasing shift,
// relaxation over TR - TE, after the 180-degree inversion with delay TI.  The
// reference only evaluates this recursion; the refinement differentiates it
// in forward mode.
//
// Model per voxel: x = rho * s(T1, T2, B0, B1) with rho complex, eliminated
// by variable projection (rho = <s, x> / <s, s>).  One pass carries the
// signal and its tangents ds/dT1, ds/dT2, ds/dB0 and, without a B1 map,
// ds/dB1 (flip angle alpha_t * B1) through the recursion as complex EPG
// states, accumulates <s,s>, <s,x>, <s,J_j>, Re<J_j,J_k>, <J_j,x> on the
// voxel's first lane and solves the normal equations of the projected
// residual,
//   A_jk = |rho|^2 Re(<J_j,J_k> - conj(<s,J_j>) <s,J_k> / <s,s>),
//   b_j  = Re(conj(rho) (<J_j,x> - conj(<s,J_j>) <s,x> / <s,s>)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#define SNAPMRF_EPG_DEVICE_HELPERS_ONLY
#include "epg_kernels.cuh"

namespace snapmrf {
namespace ssfpgrad {

constexpr int kThreads = 32;   // one warp per CTA: no CTA barrier couples voxels
constexpr int kStepChunk = 16; // time steps staged per chunk

// Per-(voxel, step) constants staged in shared memory.
struct Step {
    float E1a, E2a, E1b, E2b;      // relaxation over TE and over TR - TE
    float dE1a, dE2a, dE1b, dE2b;  // their derivatives by T1 / T2
    float2 ea, eb;                 // B0 phasors over TE and TR - TE
    float tha, thb;                // d(phase)/dB0 over TE and TR - TE (rad / Hz)
    float ca, sa, fa;              // cos, sin of alpha_t * B1; alpha_t (d alpha / dB1)
    float2 z;                      // (cos phi_t, sin phi_t)
    float2 x;                      // voxel sample
};

struct Args {
    const float *alpha;  // [nreps] converted flip angles (rad)
    const float *phi;    // [nreps] RF phases (rad)
    const float *TR;     // [nreps] ms
    const float *TE;     // [nreps] ms
    int nreps;
    float TI;            // inversion delay (ms)
    long long nvox;
    int w, L;
    const float2 *img;
    long long img_stride;
    float *maps;         // [nvox][nmaps]: T1, T2, B0, B1, PD (in/out)
    int nmaps;
    const float *b1map;  // optional [nvox]: B1 of each voxel (then not refined)
    float *m0;           // optional out [nvox]
    float max_rel_step;
    float tol;
    const int *list_in;
    const int *count_in;
    int *list_out;
    int *count_out;
    int finish;
};

__device__ __forceinline__ bool usable(float T1, float T2, float B0, float B1) {
    return isfinite(T1) && isfinite(T2) && isfinite(B0) && isfinite(B1) && T2 > 0.f && T1 > T2 && B1 > 0.f;
}

// RF matrix of rf_matrix (fill_transition_matrix, src/functions.cu:483-508)
// from cos / sin of the flip angle and the phasor z, and its derivative by
// the flip angle.
__device__ __forceinline__ void rf_and_derivative(float ca, float sa, float2 z, float2 *T, float2 *dT) {
    const float sa2 = (1 - ca) / 2, ca2 = (1 + ca) / 2;
    const float2 zinv = c_conj(z);
    const float2 z2 = c_mul(z, z), zi2 = c_mul(zinv, zinv);
    T[0] = make_float2(ca2, 0.f);
    T[3] = c_scale(zi2, sa2);
    T[6] = c_scale(make_float2(zinv.y, -zinv.x), 0.5f * sa);     // (-i/2) sa zinv
    T[1] = c_scale(z2, sa2);
    T[4] = make_float2(ca2, 0.f);
    T[7] = c_scale(make_float2(-z.y, z.x), 0.5f * sa);           // (i/2) sa z
    T[2] = c_scale(make_float2(z.y, -z.x), sa);                  // -i sa z
    T[5] = c_scale(make_float2(-zinv.y, zinv.x), sa);            // i sa zinv
    T[8] = make_float2(ca, 0.f);
    dT[0] = make_float2(-0.5f * sa, 0.f);
    dT[3] = c_scale(zi2, 0.5f * sa);
    dT[6] = c_scale(make_float2(zinv.y, -zinv.x), 0.5f * ca);
    dT[1] = c_scale(z2, 0.5f * sa);
    dT[4] = make_float2(-0.5f * sa, 0.f);
    dT[7] = c_scale(make_float2(-z.y, z.x), 0.5f * ca);
    dT[2] = c_scale(make_float2(z.y, -z.x), ca);
    dT[5] = c_scale(make_float2(-zinv.y, zinv.x), ca);
    dT[8] = make_float2(-sa, 0.f);
}

template <int S>
__device__ __forceinline__ void zero(LaneState<S> &s) {
#pragma unroll
    for (int j = 0; j < S; j++) s.fp[j] = s.fm[j] = s.zz[j] = make_float2(0.f, 0.f);
}

// d <- T d (+ g dT s when WITH_S)
template <int S, bool WITH_S>
__device__ __forceinline__ void rf_apply(LaneState<S> &d, const float2 *T, const float2 *dT, float g,
                                         const LaneState<S> &s) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        const float2 o0 = d.fp[j], o1 = d.fm[j], o2 = d.zz[j];
        float2 r0 = rf_row(T[0], T[1], T[2], o0, o1, o2);
        float2 r1 = rf_row(T[3], T[4], T[5], o0, o1, o2);
        float2 r2 = rf_row(T[6], T[7], T[8], o0, o1, o2);
        if (WITH_S) {
            const float2 q0 = rf_row(dT[0], dT[1], dT[2], s.fp[j], s.fm[j], s.zz[j]);
            const float2 q1 = rf_row(dT[3], dT[4], dT[5], s.fp[j], s.fm[j], s.zz[j]);
            const float2 q2 = rf_row(dT[6], dT[7], dT[8], s.fp[j], s.fm[j], s.zz[j]);
            r0.x = fmaf(g, q0.x, r0.x); r0.y = fmaf(g, q0.y, r0.y);
            r1.x = fmaf(g, q1.x, r1.x); r1.y = fmaf(g, q1.y, r1.y);
            r2.x = fmaf(g, q2.x, r2.x); r2.y = fmaf(g, q2.y, r2.y);
        }
        d.fp[j] = r0;
        d.fm[j] = r1;
        d.zz[j] = r2;
    }
}

// Tangent relaxation: d <- E d + dE s on the channels that depend on the
// parameter (which = 0: T1, Z and the recovery; 1: T2, F+ and F-; else none).
template <int S>
__device__ __forceinline__ void relax_tangent(LaneState<S> &d, const LaneState<S> &s, float E1, float E2, float dE1,
                                              float dE2, int which, bool lane0) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        if (which == 1) {
            d.fp[j] = make_float2(fmaf(dE2, s.fp[j].x, E2 * d.fp[j].x), fmaf(dE2, s.fp[j].y, E2 * d.fp[j].y));
            d.fm[j] = make_float2(fmaf(dE2, s.fm[j].x, E2 * d.fm[j].x), fmaf(dE2, s.fm[j].y, E2 * d.fm[j].y));
        } else {
            d.fp[j] = c_scale(d.fp[j], E2);
            d.fm[j] = c_scale(d.fm[j], E2);
        }
        if (which == 0)
            d.zz[j] = make_float2(fmaf(dE1, s.zz[j].x, E1 * d.zz[j].x), fmaf(dE1, s.zz[j].y, E1 * d.zz[j].y));
        else
            d.zz[j] = c_scale(d.zz[j], E1);
    }
    if (which == 0 && lane0) d.zz[0].x -= dE1;  // d(1 - E1)
}

// Tangent B0 precession after the signal's: d <- e d (+ i th s_new on F+,
// - i th s_new on F- for the B0 tangent).
template <int S>
__device__ __forceinline__ void b0_tangent(LaneState<S> &d, const LaneState<S> &s_new, float2 e, float th, bool b0) {
    const float2 ec = c_conj(e);
#pragma unroll
    for (int j = 0; j < S; j++) {
        float2 p = c_mul(e, d.fp[j]), m = c_mul(ec, d.fm[j]);
        if (b0) {
            p.x = fmaf(-th, s_new.fp[j].y, p.x);
            p.y = fmaf(th, s_new.fp[j].x, p.y);
            m.x = fmaf(th, s_new.fm[j].y, m.x);
            m.y = fmaf(-th, s_new.fm[j].x, m.y);
        }
        d.fp[j] = p;
        d.fm[j] = m;
    }
}

// Cholesky solve of the NT x NT system A d = b (A symmetric positive
// definite up to a relative diagonal jitter); false when it is not.
template <int NT>
__device__ __forceinline__ bool solve_spd(float (&A)[NT][NT], float (&b)[NT], float (&d)[NT]) {
    float Lm[NT][NT];
#pragma unroll
    for (int i = 0; i < NT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++) Lm[i][j] = 0.f;
#pragma unroll
    for (int i = 0; i < NT; i++) {
#pragma unroll
        for (int j = 0; j <= i; j++) {
            float v = A[i][j];
#pragma unroll
            for (int k = 0; k < j; k++) v -= Lm[i][k] * Lm[j][k];
            if (i == j) {
                v += 1e-7f * fabsf(A[i][i]);
                if (!(v > 0.f) || !isfinite(v)) return false;
                Lm[i][i] = sqrtf(v);
            } else {
                Lm[i][j] = v / Lm[j][j];
            }
        }
    }
    float y[NT];
#pragma unroll
    for (int i = 0; i < NT; i++) {
        float v = b[i];
#pragma unroll
        for (int k = 0; k < i; k++) v -= Lm[i][k] * y[k];
        y[i] = v / Lm[i][i];
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; i--) {
        float v = y[i];
#pragma unroll
        for (int k = i + 1; k < NT; k++) v -= Lm[k][i] * d[k];
        d[i] = v / Lm[i][i];
    }
#pragma unroll
    for (int i = 0; i < NT; i++)
        if (!isfinite(d[i])) return false;
    return true;
}

// One Gauss-Newton iteration per voxel of the list (NT = 3: T1, T2, B0 with
// B1 from the map; NT = 4: B1 refined too) or, with NT = 0, the value-only
// evaluation of PD and M0.  L lanes per voxel, S complex states per lane.
template <int S, int NT>
__global__ void __launch_bounds__(kThreads) gn_ssfp_kernel(Args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int L = a.L, apc = kThreads / L;
    const int tid = threadIdx.x, g = tid / L, gl = tid % L;
    const bool lane0 = gl == 0;
    Step *sQ = reinterpret_cast<Step *>(smem);                      // [apc][kStepChunk]
    float *sV = reinterpret_cast<float *>(sQ + apc * kStepChunk);   // [apc][6]: T1 T2 B0 B1 ok pad
    long long *sI = reinterpret_cast<long long *>(sV + apc * 6);    // [apc]
    const long long vox0 = (long long)blockIdx.x * apc;
    const long long nlist = a.list_in ? (long long)*a.count_in : a.nvox;
    for (int i = tid; i < apc; i += kThreads) {
        const long long slot = vox0 + i;
        long long v = -1;
        if (slot < nlist) v = a.list_in ? (long long)a.list_in[slot] : slot;
        sI[i] = v;
        float T1 = 2.f, T2 = 1.f, B0 = 0.f, B1 = 1.f, ok = 0.f;
        if (v >= 0) {
            const float *mp = a.maps + v * a.nmaps;
            const float t1 = mp[0], t2 = mp[1], b0 = a.nmaps >= 3 ? mp[2] : 0.f;
            const float b1 = a.b1map ? a.b1map[v] : (a.nmaps >= 4 ? mp[3] : 1.f);
            if (usable(t1, t2, b0, b1)) {
                T1 = t1;
                T2 = t2;
                B0 = b0;
                B1 = b1;
                ok = 1.f;
            }
        }
        sV[6 * i] = T1;
        sV[6 * i + 1] = T2;
        sV[6 * i + 2] = B0;
        sV[6 * i + 3] = B1;
        sV[6 * i + 4] = ok;
    }
    if (!__syncthreads_or(tid < apc && sV[6 * tid + 4] != 0.f)) return;
    const long long v = sI[g];
    const bool active = sV[6 * g + 4] != 0.f;
    const int T = a.nreps, w = a.w;
    const float T1 = sV[6 * g], T2 = sV[6 * g + 1];

    LaneState<S> s;
    LaneState<S> d[NT > 0 ? NT : 1];
    // inversion (init_rf_pulse, src/functions.cu:456-481) with the signal's
    // float expressions of st_init; its tangents by T1 and T2
    st_init<S>(s, lane0, T1, T2, 180.f, 0.f, a.TI);
#pragma unroll
    for (int p = 0; p < NT; p++) zero<S>(d[p]);
    if constexpr (NT > 0) {
        if (lane0) {
            const float alpha = (float)(180.f * M_PI / 180.f);
            float sa0, ca0;
            __sincosf(alpha, &sa0, &ca0);
            const float e1 = expf(-a.TI / T1), e2 = expf(-a.TI / T2);
            const float de1 = e1 * a.TI / (T1 * T1), de2 = e2 * a.TI / (T2 * T2);
            d[0].zz[0] = make_float2(de1 * (ca0 - 1.f), 0.f);
            const float2 q = make_float2(0.f, de2 * sa0);  // d/dT2 of e2 sa (sin 0 + i cos 0)
            d[1].fp[0] = c_conj(q);
            d[1].fm[0] = q;
        }
    }

    // inner products on the first lane: Ss = <s,s>, P = <s,x>, G_j = <s,J_j>,
    // H_jk = Re<J_j,J_k>, Q_j = <J_j,x>
    float Ss = 0.f;
    float2 P = make_float2(0.f, 0.f);
    float2 G[NT > 0 ? NT : 1], Q[NT > 0 ? NT : 1];
    float H[NT > 0 ? NT : 1][NT > 0 ? NT : 1];
#pragma unroll
    for (int j = 0; j < NT; j++) {
        G[j] = Q[j] = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < NT; k++) H[j][k] = 0.f;
    }
    for (int t0 = 0; t0 < T; t0 += kStepChunk) {
        const int nch = min(kStepChunk, T - t0);
        __syncthreads();
        for (int idx = tid; idx < apc * nch; idx += kThreads) {
            const int ga = idx / nch, i = idx - ga * nch;
            const float t1 = sV[6 * ga], t2 = sV[6 * ga + 1], b0 = sV[6 * ga + 2], b1 = sV[6 * ga + 3];
            const int t = t0 + i;
            Step q;
            const float tr = a.TR[t], te = a.TE[t];
            const float ta = te, tb = tr - te;
            q.E1a = expf(-ta / t1);
            q.E2a = expf(-ta / t2);
            q.E1b = expf(-tb / t1);
            q.E2b = expf(-tb / t2);
            q.dE1a = q.E1a * ta / (t1 * t1);
            q.dE2a = q.E2a * ta / (t2 * t2);
            q.dE1b = q.E1b * tb / (t1 * t1);
            q.dE2b = q.E2b * tb / (t2 * t2);
            q.ea = b0_phasor(b0, ta);
            q.eb = b0_phasor(b0, tb);
            q.tha = (float)(2 * M_PI * ta / 1000.0);
            q.thb = (float)(2 * M_PI * tb / 1000.0);
            q.fa = a.alpha[t];
            __sincosf(q.fa * b1, &q.sa, &q.ca);
            float sp, cp;
            __sincosf(a.phi[t], &sp, &cp);
            q.z = make_float2(cp, sp);
            const long long vv = sI[ga];
            q.x = vv >= 0 ? a.img[vv * a.img_stride + t] : make_float2(0.f, 0.f);
            sQ[ga * kStepChunk + i] = q;
        }
        __syncthreads();
        const Step *qs = sQ + g * kStepChunk;
        for (int i = 0; i < nch; i++) {
            const Step q = qs[i];
            float2 Tm[9], dT[9];
            rf_and_derivative(q.ca, q.sa, q.z, Tm, dT);
            // RF: tangents from the signal before the pulse, then the signal
#pragma unroll
            for (int p = 0; p < NT; p++) {
                if (p == 3) rf_apply<S, true>(d[p], Tm, dT, q.fa, s);
                else rf_apply<S, false>(d[p], Tm, dT, 0.f, s);
            }
            rf_apply<S, false>(s, Tm, dT, 0.f, s);
            // relaxation over TE
#pragma unroll
            for (int p = 0; p < NT; p++) relax_tangent<S>(d[p], s, q.E1a, q.E2a, q.dE1a, q.dE2a, p, lane0);
            st_relax<S>(s, q.E1a, q.E2a, lane0);
            // B0 over TE: the signal, then its tangents
            st_b0<S>(s, q.ea);
#pragma unroll
            for (int p = 0; p < NT; p++) b0_tangent<S>(d[p], s, q.ea, q.tha, p == 2);
            if (lane0) {
                const float2 sv = s.fp[0], x = q.x;
                Ss = fmaf(sv.x, sv.x, fmaf(sv.y, sv.y, Ss));
                P.x = fmaf(sv.x, x.x, fmaf(sv.y, x.y, P.x));
                P.y = fmaf(sv.x, x.y, fmaf(-sv.y, x.x, P.y));
#pragma unroll
                for (int j = 0; j < NT; j++) {
                    const float2 J = d[j].fp[0];
                    G[j].x = fmaf(sv.x, J.x, fmaf(sv.y, J.y, G[j].x));
                    G[j].y = fmaf(sv.x, J.y, fmaf(-sv.y, J.x, G[j].y));
                    Q[j].x = fmaf(J.x, x.x, fmaf(J.y, x.y, Q[j].x));
                    Q[j].y = fmaf(J.x, x.y, fmaf(-J.y, x.x, Q[j].y));
#pragma unroll
                    for (int k = j; k < NT; k++) {
                        const float2 K = d[k].fp[0];
                        H[j][k] = fmaf(J.x, K.x, fmaf(J.y, K.y, H[j][k]));
                    }
                }
            }
            // B0 over TR - TE, shift, relaxation over TR - TE
            st_b0<S>(s, q.eb);
#pragma unroll
            for (int p = 0; p < NT; p++) b0_tangent<S>(d[p], s, q.eb, q.thb, p == 2);
            st_shift<S>(s, gl, L, w);
#pragma unroll
            for (int p = 0; p < NT; p++) st_shift<S>(d[p], gl, L, w);
#pragma unroll
            for (int p = 0; p < NT; p++) relax_tangent<S>(d[p], s, q.E1b, q.E2b, q.dE1b, q.dE2b, p, lane0);
            st_relax<S>(s, q.E1b, q.E2b, lane0);
        }
    }
    if (!lane0 || !active || !(Ss > 0.f)) return;
    float *mp = a.maps + v * a.nmaps;
    auto finish = [&](float2 p, float ss) {
        const float ip = sqrtf(p.x * p.x + p.y * p.y);
        if (a.b1map && a.nmaps >= 4) mp[3] = sV[6 * g + 3];
        if (a.nmaps >= 5) mp[4] = ss > 0.f ? ip / sqrtf(ss) : 0.f;
        if (a.m0) a.m0[v] = ss > 0.f ? ip / ss : 0.f;
    };
    if constexpr (NT == 0) {
        finish(P, Ss);
    } else {
        const float rr = P.x / Ss, ri = P.y / Ss, rho2 = rr * rr + ri * ri;
        float A[NT][NT], bv[NT], dl[NT];
    #pragma unroll
        for (int j = 0; j < NT; j++) {
    #pragma unroll
            for (int k = j; k < NT; k++) {
                // Re(conj(G_j) G_k)
                const float gg = G[j].x * G[k].x + G[j].y * G[k].y;
                A[j][k] = A[k][j] = rho2 * (H[j][k] - gg / Ss);
            }
            // c_j = Q_j - conj(G_j) P / Ss;  b_j = Re(conj(rho) c_j)
            const float cpr = G[j].x * P.x + G[j].y * P.y, cpi = G[j].x * P.y - G[j].y * P.x;
            const float cr = Q[j].x - cpr / Ss, ci = Q[j].y - cpi / Ss;
            bv[j] = rr * cr + ri * ci;
            dl[j] = 0.f;
        }
        if (!solve_spd<NT>(A, bv, dl)) {
    #pragma unroll
            for (int j = 0; j < NT; j++) dl[j] = 0.f;
        }
        const float B0 = sV[6 * g + 2], B1 = sV[6 * g + 3];
        // trust region: T1, T2 and B1 by max_rel_step of their values, B0 by
        // max_rel_step x 50 Hz
        const float lim[4] = {a.max_rel_step * T1, a.max_rel_step * T2, a.max_rel_step * 50.f, a.max_rel_step * B1};
    #pragma unroll
        for (int j = 0; j < NT; j++) dl[j] = fminf(fmaxf(dl[j], -lim[j]), lim[j]);
        float n2 = fmaxf(T2 + dl[1], 1e-3f);
        float n1 = fmaxf(T1 + dl[0], n2 * (1.f + 1e-4f));
        const float nb0 = B0 + dl[2];
        float nb1 = B1;
        if constexpr (NT > 3) nb1 = fmaxf(B1 + dl[3], 0.05f);
        dl[0] = n1 - T1;
        dl[1] = n2 - T2;
        mp[0] = n1;
        mp[1] = n2;
        if (a.nmaps >= 3) mp[2] = nb0;
        if (NT > 3 && a.nmaps >= 4) mp[3] = nb1;
        bool moving = !(fabsf(dl[0]) <= a.tol * T1 && fabsf(dl[1]) <= a.tol * T2 && fabsf(dl[2]) <= a.tol * 100.f);
        if (NT > 3) moving = moving || !(fabsf(nb1 - B1) <= a.tol * B1);
        if (a.list_out && moving) {
            a.list_out[atomicAdd(a.count_out, 1)] = (int)v;
            return;
        }
        if (a.finish) {
            // PD and M0 at the updated parameters from the linear model:
            // <s + J d, x> = P + sum d_j Q_j, ||s + J d||^2 = Ss + 2 sum d_j Re G_j + d^T H d
            float2 p = P;
            float ss = Ss;
            float dd[NT];
    #pragma unroll
            for (int j = 0; j < NT; j++) dd[j] = j == 3 ? nb1 - B1 : (j == 2 ? nb0 - B0 : dl[j]);
    #pragma unroll
            for (int j = 0; j < NT; j++) {
                p.x = fmaf(dd[j], Q[j].x, p.x);
                p.y = fmaf(dd[j], Q[j].y, p.y);
                ss = fmaf(2.f * dd[j], G[j].x, ss);
    #pragma unroll
                for (int k = 0; k < NT; k++) ss = fmaf(dd[j] * dd[k], H[min(j, k)][max(j, k)], ss);
            }
            finish(p, ss);
        }
    }
}

// lanes per voxel and states per lane: the fewest padded states for w, then
// the most states per lane (S in {2, 4})
static void choose_ls(int w, int *L, int *S) {
    int bl = 32, bs = 4, best = 1 << 30;
    for (int s = 4; s >= 2; s -= 2) {
        int l = 1;
        while (l < 32 && l * s < w) l *= 2;
        if (l * s < w) continue;
        if (l * s < best) {
            best = l * s;
            bl = l;
            bs = s;
        }
    }
    *L = bl;
    *S = bs;
}

template <int S, int NT>
static cudaError_t launch(const Args &a, dim3 grid, size_t smem, cudaStream_t st) {
    auto k = gn_ssfp_kernel<S, NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, kThreads, smem, st>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

static cudaError_t dispatch(int S, int NT, const Args &a, dim3 grid, size_t smem, cudaStream_t st) {
    if (S == 2) return NT == 4 ? launch<2, 4>(a, grid, smem, st) : NT == 3 ? launch<2, 3>(a, grid, smem, st)
                                                                       : launch<2, 0>(a, grid, smem, st);
    return NT == 4 ? launch<4, 4>(a, grid, smem, st) : NT == 3 ? launch<4, 3>(a, grid, smem, st)
                                                               : launch<4, 0>(a, grid, smem, st);
}

}  // namespace ssfpgrad

// The Gauss-Newton refinement of snapmrf_refine_gn for echo_type epg_ssfp:
// h_mrf is the CSV schedule, converted as MRF_dict converts it for epg_ssfp
// (flip fraction of 60 degrees, phase in degrees, TR + 16 ms, TE + 3.5 ms;
// src/functions.cu:1240-1261); the inversion has TI = 40 ms
// (src/functions.cu:965-966).
int refine_gn_ssfp(float *d_maps, int nmaps, const float *img, size_t img_stride, const float *d_b1map,
                   const float *h_mrf, size_t nreps, size_t NREPS, size_t nvoxels, int nstates, int iterations,
                   float max_rel_step, float tol, float *d_m0, cudaStream_t st) {
    using namespace ssfpgrad;
    if (nstates > 32 * 4) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "refine_gn (epg_ssfp): nstates must be <= 128");
    if (nmaps < 3) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_gn (epg_ssfp): maps need T1, T2 and B0 columns");
    std::vector<float> h(4 * nreps);
    const float fa_scale = (float)(60.f * M_PI / 180.f), ph_scale = (float)(M_PI / 180.f);
    for (size_t t = 0; t < nreps; t++) {
        h[t] = h_mrf[t] * fa_scale;
        h[nreps + t] = h_mrf[NREPS + t] * ph_scale;
        h[2 * nreps + t] = h_mrf[2 * NREPS + t] + 16.f;
        h[3 * nreps + t] = h_mrf[3 * NREPS + t] + 3.5f;
    }
    DeviceScratch sbuf;
    SNAPMRF_CUDA(sbuf.alloc(h.size() * sizeof(float), st));
    float *hs = static_cast<float *>(stage_acquire(h.size() * sizeof(float)));
    if (!hs) SNAPMRF_FAIL(SNAPMRF_ERR_ALLOC, "refine_gn: cannot allocate a pinned staging buffer");
    memcpy(hs, h.data(), h.size() * sizeof(float));
    SNAPMRF_CUDA(stage_upload(sbuf.ptr, hs, h.size() * sizeof(float), st));
    SNAPMRF_CUDA(stage_release(st));
    Args a;
    const float *ds = sbuf.as<float>();
    a.alpha = ds;
    a.phi = ds + nreps;
    a.TR = ds + 2 * nreps;
    a.TE = ds + 3 * nreps;
    a.nreps = (int)nreps;
    a.TI = 40.f;
    a.nvox = (long long)nvoxels;
    a.w = nstates;
    int L, S;
    choose_ls(nstates, &L, &S);
    a.L = L;
    a.img = reinterpret_cast<const float2 *>(img);
    a.img_stride = (long long)img_stride;
    a.maps = d_maps;
    a.nmaps = nmaps;
    a.b1map = d_b1map;
    a.m0 = d_m0;
    a.max_rel_step = max_rel_step > 0.f ? max_rel_step : 0.2f;
    a.tol = tol;
    // B1 is refined too when no map gives it
    const int NT = (d_b1map || nmaps < 4) ? 3 : 4;
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
    const int apc = kThreads / L;
    const size_t smem = (size_t)apc * kStepChunk * sizeof(Step) + (size_t)apc * (6 * sizeof(float) + sizeof(long long));
    dim3 grid((unsigned)((nvoxels + apc - 1) / apc));
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
        SNAPMRF_CUDA(dispatch(S, NT, a, grid, smem, st));
    }
    if (outputs && iterations == 0) {
        a.list_in = a.count_in = nullptr;
        a.list_out = a.count_out = nullptr;
        a.finish = 1;
        SNAPMRF_CUDA(dispatch(S, 0, a, grid, smem, st));
    }
    return SNAPMRF_OK;
}

}  // namespace snapmrf

// --------------------------------------------------------------------------
// Reverse mode (adjoint) of the complex bSSFP recursion with checkpointing
// --------------------------------------------------------------------------
namespace snapmrf {
namespace ssfpgrad {

struct AdjArgs {
    const float *alpha, *phi, *TR, *TE;  // converted schedule [nreps]
    float fa_scale;      // d(converted flip) / d(schedule entry)
    int nreps;
    float TI;
    const float *params; // [n][nparams]: T1, T2, B0, B1
    int nparams;
    long long n;
    int w, L;
    const float2 *gsig;  // [n][nreps] dL/d(Re s_t, Im s_t)
    float2 *sig;         // optional out [n][nreps]
    float *gparams;      // [n][4]: dL/dT1, dL/dT2, dL/dB0, dL/dB1
    float *galpha_atoms; // [n][nreps]: dL/d(schedule flip entry t) per atom
    float *ckpt;         // [n][nckpt][6 S L]
    float *seg;          // [n][C][6 S L]
    int C, nckpt;
};

// A saved state is [6][S][L] floats (F+ re, F+ im, F- re, F- im, Z re,
// Z im): the L lanes of a group touch consecutive words.
template <int S>
__device__ __forceinline__ void save(float *dst, int L, int gl, const LaneState<S> &x) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        dst[(0 * S + j) * L + gl] = x.fp[j].x;
        dst[(1 * S + j) * L + gl] = x.fp[j].y;
        dst[(2 * S + j) * L + gl] = x.fm[j].x;
        dst[(3 * S + j) * L + gl] = x.fm[j].y;
        dst[(4 * S + j) * L + gl] = x.zz[j].x;
        dst[(5 * S + j) * L + gl] = x.zz[j].y;
    }
}

template <int S>
__device__ __forceinline__ void load(LaneState<S> &x, const float *src, int L, int gl) {
#pragma unroll
    for (int j = 0; j < S; j++) {
        x.fp[j] = make_float2(src[(0 * S + j) * L + gl], src[(1 * S + j) * L + gl]);
        x.fm[j] = make_float2(src[(2 * S + j) * L + gl], src[(3 * S + j) * L + gl]);
        x.zz[j] = make_float2(src[(4 * S + j) * L + gl], src[(5 * S + j) * L + gl]);
    }
}

// Per-step constants of one atom.
struct StepC {
    float2 T[9];
    float E1a, E2a, E1b, E2b;
    float2 ea, eb;
    float ta, tb;
    float ca, sa;
    float2 z;
};

__device__ __forceinline__ StepC step_constants(const AdjArgs &a, int t, float T1, float T2, float B0, float B1) {
    StepC c;
    const float tr = a.TR[t], te = a.TE[t];
    c.ta = te;
    c.tb = tr - te;
    __sincosf(a.alpha[t] * B1, &c.sa, &c.ca);
    float sp, cp;
    __sincosf(a.phi[t], &sp, &cp);
    c.z = make_float2(cp, sp);
    float2 dT[9];
    rf_and_derivative(c.ca, c.sa, c.z, c.T, dT);
    c.E1a = expf(-c.ta / T1);
    c.E2a = expf(-c.ta / T2);
    c.E1b = expf(-c.tb / T1);
    c.E2b = expf(-c.tb / T2);
    c.ea = b0_phasor(B0, c.ta);
    c.eb = b0_phasor(B0, c.tb);
    return c;
}

// One step of the recursion (src/functions.cu:976-1010 order): RF,
// relax(TE), B0(TE), readout, B0(TR - TE), shift, relax(TR - TE).
template <int S>
__device__ __forceinline__ float2 forward_step(LaneState<S> &v, const StepC &c, int gl, int L, int w, bool lane0) {
    st_rf<S>(v, c.T);
    st_relax<S>(v, c.E1a, c.E2a, lane0);
    st_b0<S>(v, c.ea);
    const float2 s = v.fp[0];
    st_b0<S>(v, c.eb);
    st_shift<S>(v, gl, L, w);
    st_relax<S>(v, c.E1b, c.E2b, lane0);
    return s;
}

// Transpose of st_shift on adjoint states: lam_old.F+[k] = lam_new.F+[k+1]
// (k <= w-2), lam_old.F-[k] = lam_new.F-[k-1] (1 <= k <= w-1), plus
// conj(lam_new.F+[0]) into lam_old.F-[1] (F-[0] with w = 1), Z unchanged.
template <int S>
__device__ __forceinline__ void shift_transpose(LaneState<S> &l, int gl, int L, int w) {
    const unsigned full = 0xffffffffu;
    const float2 f0 = l.fp[0];  // lam_new.F+[0] on lane 0
    // F+ moves down one state: slot j takes j + 1, the top slot the next lane's slot 0
    float2 dn;
    dn.x = __shfl_down_sync(full, l.fp[0].x, 1, L);
    dn.y = __shfl_down_sync(full, l.fp[0].y, 1, L);
    // F- moves up one state: slot j takes j - 1, slot 0 the previous lane's top slot
    float2 up;
    up.x = __shfl_up_sync(full, l.fm[S - 1].x, 1, L);
    up.y = __shfl_up_sync(full, l.fm[S - 1].y, 1, L);
#pragma unroll
    for (int j = 0; j < S - 1; j++) l.fp[j] = l.fp[j + 1];
    l.fp[S - 1] = (gl == L - 1) ? make_float2(0.f, 0.f) : dn;
#pragma unroll
    for (int j = S - 1; j >= 1; j--) l.fm[j] = l.fm[j - 1];
    l.fm[0] = (gl == 0) ? make_float2(0.f, 0.f) : up;
    if (gl == 0) {
        const float2 cf = c_conj(f0);
        if (w == 1) l.fm[0] = cf;
        else { l.fm[1].x += cf.x; l.fm[1].y += cf.y; }
    }
#pragma unroll
    for (int j = 0; j < S; j++) {
        const int k = gl * S + j;
        if (k >= w - 1) l.fp[j] = make_float2(0.f, 0.f);
        if (k >= w) l.fm[j] = make_float2(0.f, 0.f);
    }
}

// Re sum conj(a) b over this lane's states of the channels in `mask`
// (1: F+, 2: F-, 4: Z).
template <int S>
__device__ __forceinline__ float redot(const LaneState<S> &a, const LaneState<S> &b, int mask) {
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < S; j++) {
        if (mask & 1) r = fmaf(a.fp[j].x, b.fp[j].x, fmaf(a.fp[j].y, b.fp[j].y, r));
        if (mask & 2) r = fmaf(a.fm[j].x, b.fm[j].x, fmaf(a.fm[j].y, b.fm[j].y, r));
        if (mask & 4) r = fmaf(a.zz[j].x, b.zz[j].x, fmaf(a.zz[j].y, b.zz[j].y, r));
    }
    return r;
}

// Re sum [conj(l.F+) i v.F+ - conj(l.F-) i v.F-]: the B0 derivative of a
// precession that produced v (per unit of phase).
template <int S>
__device__ __forceinline__ float b0_term(const LaneState<S> &l, const LaneState<S> &v) {
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < S; j++) {
        // Re(conj(l) i v) = l.x (-v.y) + l.y v.x
        r += -l.fp[j].x * v.fp[j].y + l.fp[j].y * v.fp[j].x;
        r -= -l.fm[j].x * v.fm[j].y + l.fm[j].y * v.fm[j].x;
    }
    return r;
}

template <int S>
__global__ void __launch_bounds__(kThreads) ssfp_adjoint_kernel(AdjArgs a) {
    const int L = a.L, apc = kThreads / L;
    const int tid = threadIdx.x, g = tid / L, gl = tid % L;
    const bool lane0 = gl == 0;
    const long long atom = (long long)blockIdx.x * apc + g;
    const bool active = atom < a.n;
    const long long at = active ? atom : 0;
    const float *p = a.params + at * a.nparams;
    const float T1 = active ? p[0] : 2.f, T2 = active ? p[1] : 1.f, B0 = active ? p[2] : 0.f,
                B1 = active ? p[3] : 1.f;
    const int T = a.nreps, w = a.w, C = a.C;
    const long long LS = (long long)L * S;
    float *ck = a.ckpt + at * (long long)a.nckpt * 6 * LS;
    float *sg = a.seg + at * (long long)C * 6 * LS;

    // forward sweep with checkpoints every C steps
    LaneState<S> v;
    st_init<S>(v, lane0, T1, T2, 180.f, 0.f, a.TI);
    for (int t = 0; t < T; t++) {
        if (t % C == 0 && active) save<S>(ck + (long long)(t / C) * 6 * LS, L, gl, v);
        const StepC c = step_constants(a, t, T1, T2, B0, B1);
        const float2 s = forward_step<S>(v, c, gl, L, w, lane0);
        if (lane0 && active && a.sig) a.sig[at * T + t] = s;
    }
    __syncwarp();

    // reverse sweep, one segment at a time
    LaneState<S> lam;
    zero<S>(lam);
    float gE1_T1 = 0.f, gE2_T2 = 0.f, gB0 = 0.f, gB1 = 0.f;  // lane partials, chained per step
    for (int sgi = a.nckpt - 1; sgi >= 0; sgi--) {
        const int t0 = sgi * C, t1 = min(T, t0 + C);
        LaneState<S> u;
        if (active) load<S>(u, ck + (long long)sgi * 6 * LS, L, gl);
        else zero<S>(u);
        for (int t = t0; t < t1; t++) {
            if (active) save<S>(sg + (long long)(t - t0) * 6 * LS, L, gl, u);
            const StepC c = step_constants(a, t, T1, T2, B0, B1);
            forward_step<S>(u, c, gl, L, w, lane0);
        }
        __syncwarp();
        for (int t = t1 - 1; t >= t0; t--) {
            const StepC c = step_constants(a, t, T1, T2, B0, B1);
            float2 dT[9], Tm[9];
            rf_and_derivative(c.ca, c.sa, c.z, Tm, dT);
            // intermediates of step t from its start state v0
            LaneState<S> v0, v1, v3, v4, v5;
            if (active) load<S>(v0, sg + (long long)(t - t0) * 6 * LS, L, gl);
            else zero<S>(v0);
            v1 = v0;
            st_rf<S>(v1, c.T);
            LaneState<S> v2 = v1;
            st_relax<S>(v2, c.E1a, c.E2a, lane0);
            v3 = v2;
            st_b0<S>(v3, c.ea);
            v4 = v3;
            st_b0<S>(v4, c.eb);
            v5 = v4;
            st_shift<S>(v5, gl, L, w);
            // relax(TR - TE): lam5 = E lam6; dL/dE1b = Re<lam6.Z, v5.Z> - Re lam6.Z0
            const float dE1b = c.E1b * c.tb / (T1 * T1), dE2b = c.E2b * c.tb / (T2 * T2);
            float gz = redot<S>(lam, v5, 4) - (lane0 ? lam.zz[0].x : 0.f);
            float gf = redot<S>(lam, v5, 3);
            gE1_T1 = fmaf(gz, dE1b, gE1_T1);
            gE2_T2 = fmaf(gf, dE2b, gE2_T2);
#pragma unroll
            for (int j = 0; j < S; j++) {
                lam.fp[j] = c_scale(lam.fp[j], c.E2b);
                lam.fm[j] = c_scale(lam.fm[j], c.E2b);
                lam.zz[j] = c_scale(lam.zz[j], c.E1b);
            }
            // shift
            shift_transpose<S>(lam, gl, L, w);
            // B0 over TR - TE (conjugate phasors), its B0 derivative with v4
            gB0 = fmaf(b0_term<S>(lam, v4), (float)(2 * M_PI * c.tb / 1000.0), gB0);
            st_b0<S>(lam, c_conj(c.eb));
            // readout s_t = v3.F+[0]
            if (lane0 && active) {
                const float2 gs = a.gsig[at * T + t];
                lam.fp[0].x += gs.x;
                lam.fp[0].y += gs.y;
            }
            // B0 over TE
            gB0 = fmaf(b0_term<S>(lam, v3), (float)(2 * M_PI * c.ta / 1000.0), gB0);
            st_b0<S>(lam, c_conj(c.ea));
            // relax(TE)
            const float dE1a = c.E1a * c.ta / (T1 * T1), dE2a = c.E2a * c.ta / (T2 * T2);
            gz = redot<S>(lam, v1, 4) - (lane0 ? lam.zz[0].x : 0.f);
            gf = redot<S>(lam, v1, 3);
            gE1_T1 = fmaf(gz, dE1a, gE1_T1);
            gE2_T2 = fmaf(gf, dE2a, gE2_T2);
#pragma unroll
            for (int j = 0; j < S; j++) {
                lam.fp[j] = c_scale(lam.fp[j], c.E2a);
                lam.fm[j] = c_scale(lam.fm[j], c.E2a);
                lam.zz[j] = c_scale(lam.zz[j], c.E1a);
            }
            // RF: dL/dalpha = Re<lam1, dM v0>; lam0 = M^H lam1
            float ga = 0.f;
#pragma unroll
            for (int j = 0; j < S; j++) {
                const float2 q0 = rf_row(dT[0], dT[1], dT[2], v0.fp[j], v0.fm[j], v0.zz[j]);
                const float2 q1 = rf_row(dT[3], dT[4], dT[5], v0.fp[j], v0.fm[j], v0.zz[j]);
                const float2 q2 = rf_row(dT[6], dT[7], dT[8], v0.fp[j], v0.fm[j], v0.zz[j]);
                ga = fmaf(lam.fp[j].x, q0.x, fmaf(lam.fp[j].y, q0.y, ga));
                ga = fmaf(lam.fm[j].x, q1.x, fmaf(lam.fm[j].y, q1.y, ga));
                ga = fmaf(lam.zz[j].x, q2.x, fmaf(lam.zz[j].y, q2.y, ga));
                const float2 l0 = lam.fp[j], l1 = lam.fm[j], l2 = lam.zz[j];
                lam.fp[j] = rf_row(c_conj(c.T[0]), c_conj(c.T[3]), c_conj(c.T[6]), l0, l1, l2);
                lam.fm[j] = rf_row(c_conj(c.T[1]), c_conj(c.T[4]), c_conj(c.T[7]), l0, l1, l2);
                lam.zz[j] = rf_row(c_conj(c.T[2]), c_conj(c.T[5]), c_conj(c.T[8]), l0, l1, l2);
            }
            // the step's flip-angle gradient over the group's lanes
            for (int o = 1; o < L; o <<= 1) ga += __shfl_xor_sync(0xffffffffu, ga, o, L);
            gB1 = fmaf(ga, a.alpha[t], gB1);
            if (lane0 && active) a.galpha_atoms[at * T + t] = ga * B1 * a.fa_scale;
        }
    }
    // the inversion: Z0 = E1 cos(a0) + 1 - E1, F+0 = conj(q), F-0 = q,
    // q = E2 sin(a0) (0 + i)
    if (lane0) {
        const float alpha0 = (float)(180.f * M_PI / 180.f);
        float sa0, ca0;
        __sincosf(alpha0, &sa0, &ca0);
        const float e1 = expf(-a.TI / T1), e2 = expf(-a.TI / T2);
        gE1_T1 = fmaf(lam.zz[0].x * (ca0 - 1.f), e1 * a.TI / (T1 * T1), gE1_T1);
        // d/dT2: F+0 = (0, -e2 sa0), F-0 = (0, e2 sa0)
        gE2_T2 = fmaf(-lam.fp[0].y * sa0 + lam.fm[0].y * sa0, e2 * a.TI / (T2 * T2), gE2_T2);
    }
    for (int o = 1; o < L; o <<= 1) {
        gE1_T1 += __shfl_xor_sync(0xffffffffu, gE1_T1, o, L);
        gE2_T2 += __shfl_xor_sync(0xffffffffu, gE2_T2, o, L);
        gB0 += __shfl_xor_sync(0xffffffffu, gB0, o, L);
    }
    if (lane0 && active) {
        float *gp = a.gparams + at * 4;
        gp[0] = gE1_T1;
        gp[1] = gE2_T2;
        gp[2] = gB0;
        gp[3] = gB1;
    }
}

}  // namespace ssfpgrad

// snapmrf_epg_adjoint for echo_type epg_ssfp: h_mrf in the CSV convention
// (converted as MRF_dict converts it), TI = 40 ms.  Writes the signal
// (optional), dL/d(T1, T2, B0, B1) per atom and the per-atom schedule
// gradient dL/dh_mrf[0][t] into galpha_atoms.
int epg_adjoint_ssfp(const float *d_params, int nparams, const float *h_mrf, size_t nreps, size_t NREPS,
                     size_t natoms, int nstates, const float *d_grad_signal, float *d_signal, float *d_grad_params,
                     float *galpha_atoms, int checkpoint_every, cudaStream_t st) {
    using namespace ssfpgrad;
    if (nstates > 32 * 4) SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "epg_adjoint (epg_ssfp): nstates must be <= 128");
    std::vector<float> h(4 * nreps);
    const float fa_scale = (float)(60.f * M_PI / 180.f), ph_scale = (float)(M_PI / 180.f);
    for (size_t t = 0; t < nreps; t++) {
        h[t] = h_mrf[t] * fa_scale;
        h[nreps + t] = h_mrf[NREPS + t] * ph_scale;
        h[2 * nreps + t] = h_mrf[2 * NREPS + t] + 16.f;
        h[3 * nreps + t] = h_mrf[3 * NREPS + t] + 3.5f;
    }
    int L, S;
    choose_ls(nstates, &L, &S);
    const int C = checkpoint_every > 0 ? checkpoint_every : (int)std::max(1.0, std::ceil(std::sqrt((double)nreps)));
    const int nckpt = (int)((nreps + C - 1) / C);
    const long long LS = (long long)L * S;
    DeviceScratch sbuf, work;
    SNAPMRF_CUDA(sbuf.alloc(h.size() * sizeof(float), st));
    float *hs = static_cast<float *>(stage_acquire(h.size() * sizeof(float)));
    if (!hs) SNAPMRF_FAIL(SNAPMRF_ERR_ALLOC, "epg_adjoint: cannot allocate a pinned staging buffer");
    memcpy(hs, h.data(), h.size() * sizeof(float));
    SNAPMRF_CUDA(stage_upload(sbuf.ptr, hs, h.size() * sizeof(float), st));
    SNAPMRF_CUDA(stage_release(st));
    const size_t ck = natoms * (size_t)nckpt * 6 * LS, sgn = natoms * (size_t)C * 6 * LS;
    SNAPMRF_CUDA(work.alloc((ck + sgn) * sizeof(float), st));
    AdjArgs a;
    const float *ds = sbuf.as<float>();
    a.alpha = ds;
    a.phi = ds + nreps;
    a.TR = ds + 2 * nreps;
    a.TE = ds + 3 * nreps;
    a.fa_scale = fa_scale;
    a.nreps = (int)nreps;
    a.TI = 40.f;
    a.params = d_params;
    a.nparams = nparams;
    a.n = (long long)natoms;
    a.w = nstates;
    a.L = L;
    a.gsig = reinterpret_cast<const float2 *>(d_grad_signal);
    a.sig = reinterpret_cast<float2 *>(d_signal);
    a.gparams = d_grad_params;
    a.galpha_atoms = galpha_atoms;
    a.ckpt = work.as<float>();
    a.seg = a.ckpt + ck;
    a.C = C;
    a.nckpt = nckpt;
    const int apc = kThreads / L;
    dim3 grid((unsigned)((natoms + apc - 1) / apc));
    if (S == 2) ssfp_adjoint_kernel<2><<<grid, kThreads, 0, st>>>(a);
    else ssfp_adjoint_kernel<4><<<grid, kThreads, 0, st>>>(a);
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}

}  // namespace snapmrf
