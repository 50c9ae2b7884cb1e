// Sub-grid start of the Gauss-Newton refinement, from the dictionary.
//
// Matching leaves each voxel on a grid point of the dictionary (the atom of
// the largest |<d, x>| in the reference's MRF_match, src/functions.cu).  The
// matched atom, its neighbours at the adjacent T1 and T2 values of the
// parameter table (trans_params order, src/functions.cu:355-391: B1
// outermost, then B0, T2, T1 innermost, T1 > T2 kept) and one diagonal
// neighbour form a six-point stencil; with a B1 map the stencil is read from
// the three B1 blocks around the voxel's B1 and interpolated quadratically to
// that value.  In (U, V) = (log T1 / T1_0, log T2 / T2_0) the six signals give
// the quadratic surrogate
//     s(U, V) = c + a U + b V + d U^2 + e V^2 + f U V
// of the signal model (exact for quadratics, so accurate to third order in
// the grid step): a, d from the three nodes along T1, b, e along T2, f from
// the diagonal node.  The voxel's fit |<s, x>|^2 / ||s||^2 is maximised over
// the surrogate by Gauss-Newton with variable projection, using only the 6 x 6
// Gram matrix of (c, a, b, d, e, f) and their inner products with the voxel,
// so no recursion is run.  The result replaces the voxel's (T1, T2): a start
// close enough to the least-squares fit that one pass of the refinement
// usually meets its stopping tolerance.  No counterpart in the reference.
//
// Two kernels.  accumulate_kernel: one warp per voxel finds the stencil
// (32 table rows at a time with warp ballots), then its lanes stride over the
// time points, each accumulating the Gram matrix and the inner products of
// its samples in the basis (c, a, b, d, e, f), formed from differences of the
// atoms sample by sample so that the small derivative terms never come out of
// a difference of large accumulated sums; the warp's sums go to a scratch
// system per voxel.  solve_kernel: one thread per voxel solves the surrogate.

#include "common.h"

#include <cmath>
#include <cstdint>
#include <type_traits>

namespace snapmrf {
namespace rstart {

constexpr int kWarps = 4;        // voxels per block of the accumulation
constexpr int kSolveIters = 10;  // Gauss-Newton iterations on the surrogate
constexpr int kPts = 6;          // stencil points (and basis signals)
constexpr int kTri = kPts * (kPts + 1) / 2;
// shared-memory slots of staged samples per warp (imaginary atoms, complex)
template <bool IMAG>
__host__ __device__ constexpr int stages() {
    return IMAG ? 5 : 3;
}

// Stencil points: the matched atom, T1 below / above, T2 below / above, and
// the diagonal (T1 above and T2 above, else T1 below and T2 below).
enum { kC = 0, kUm = 1, kUp = 2, kVm = 3, kVp = 4, kD = 5 };

struct Args {
    float *maps;
    int nmaps;
    const int64_t *index;
    const float2 *atoms;
    long long atom_stride;  // complex samples per atom row
    const float *params;
    int nparams;
    long long NATOMS, natoms;
    const float2 *img;
    long long img_stride;
    int T;
    long long nvox;
    const float *b1map;
    int *count;
    float *sys;  // [kSysRows (kSysRowsComplex)][nvox]: the accumulated system per voxel
    int imag_rows;  // atoms as Im rows, [NATOMS][atom_stride] float
};

// Rows of the per-voxel system handed from the accumulation to the solve:
// the matched (T1, T2) (T1 NaN: leave the voxel), the node offsets (log
// ratios) of T1 below / above, T2 below / above and of the diagonal node, the
// inner products with the voxel (real and imaginary parts), the real part of
// the Gram matrix (packed upper triangle) and, for complex atoms, its
// imaginary part.
constexpr int kRowT1 = 0, kRowT2 = 1, kRowH = 2, kRowPr = 8, kRowPi = kRowPr + kPts, kRowG = kRowPi + kPts,
              kRowGi = kRowG + kTri;
constexpr int kSysRows = kRowGi, kSysRowsComplex = kRowGi + kTri;

__device__ __forceinline__ float prm(const Args &a, long long r, int c) { return __ldg(a.params + r * a.nparams + c); }

// First k in [0, n) for which pred(start + dir * k) holds, 32 rows at a time
// across the warp; -1 when there is none.
template <class F>
__device__ long long warp_find(long long start, int dir, long long n, F pred) {
    const int lane = threadIdx.x & 31;
    for (long long k0 = 0; k0 < n; k0 += 32) {
        const long long k = k0 + lane;
        const bool hit = k < n && pred(start + dir * k);
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (m) return k0 + (__ffs(m) - 1);
    }
    return -1;
}

// The stencil st[kPts] as row numbers within the block starting at `base`
// (j: the matched atom); diag_up: the diagonal node is (T1 above, T2 above)
// rather than (T1 below, T2 below).  False unless the matched atom has a
// neighbour on both sides in T1 within its T2 row, the adjacent T2 rows on
// both sides hold the matched T1, and one of them holds the diagonal node,
// with the same B0 throughout.
__device__ bool find_stencil(const Args &a, long long base, long long j, long long st[kPts], bool *diag_up) {
    const long long n = a.natoms;
    auto t1 = [&](long long r) { return prm(a, base + r, 0); };
    auto t2 = [&](long long r) { return prm(a, base + r, 1); };
    auto b0 = [&](long long r) { return prm(a, base + r, 2); };
    if (j < 1 || j + 1 >= n) return false;
    const float T1m = t1(j - 1), T1c = t1(j), T1p = t1(j + 1), T2c = t2(j), B0c = b0(j);
    if (t2(j - 1) != T2c || t2(j + 1) != T2c || b0(j - 1) != B0c || b0(j + 1) != B0c) return false;
    if (!((T1m < T1c && T1c < T1p) || (T1m > T1c && T1c > T1p))) return false;
    st[kC] = j;
    st[kUm] = j - 1;
    st[kUp] = j + 1;
    float T2n[2];
    long long rcs[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int dir = s ? 1 : -1;
        // the first row past the T2 row of j (j - 1 and j + 1 belong to it)
        const long long from = j + 2 * dir;
        const long long lim = dir < 0 ? from + 1 : n - from;
        if (lim <= 0) return false;
        const long long k = warp_find(from, dir, lim, [&](long long r) { return t2(r) != T2c || b0(r) != B0c; });
        if (k < 0) return false;
        const long long r0 = from + dir * k;
        const float T2r = t2(r0);
        if (b0(r0) != B0c || !(T2r != T2c) || !isfinite(T2r)) return false;
        // in that row, the atom at the matched T1
        const long long lim2 = dir < 0 ? r0 + 1 : n - r0;
        const long long k2 = warp_find(r0, dir, lim2, [&](long long r) {
            return t2(r) != T2r || b0(r) != B0c || t1(r) == T1c;
        });
        if (k2 < 0) return false;
        const long long rc = r0 + dir * k2;
        if (t1(rc) != T1c || t2(rc) != T2r || b0(rc) != B0c) return false;
        T2n[s] = T2r;
        rcs[s] = rc;
    }
    if (!(T2n[0] != T2n[1] && (T2n[0] < T2c) == (T2c < T2n[1]))) return false;
    st[kVm] = rcs[0];
    st[kVp] = rcs[1];
    // the diagonal: T1 above in the upper T2 row (the rows list T1 in the
    // same order), else T1 below in the lower one
    const long long du = rcs[1] + 1, dm = rcs[0] - 1;
    if (du < n && t1(du) == T1p && t2(du) == T2n[1] && b0(du) == B0c) {
        st[kD] = du;
        *diag_up = true;
        return true;
    }
    if (dm >= 0 && t1(dm) == T1m && t2(dm) == T2n[0] && b0(dm) == B0c) {
        st[kD] = dm;
        *diag_up = false;
        return true;
    }
    return false;
}

// Coefficients of the quadratic through (h_m, y_m), (0, y_0), (h_p, y_p) in
// the form y_0 + l x + q x^2: l = b1 dp + b2 dm, q = a1 dp + a2 dm with
// dp = y_p - y_0, dm = y_m - y_0.
struct Quad {
    float a1, a2, b1, b2;
};

__device__ Quad quad_coeffs(float hm, float hp) {
    Quad c;
    c.a1 = 1.f / (hp * (hp - hm));
    c.a2 = -1.f / (hm * (hp - hm));
    c.b1 = 1.f / hp - c.a1 * hp;
    c.b2 = -c.a2 * hp;
    return c;
}

// Lagrange weights of the three nodes at x.
__device__ void lagrange3(const float n[3], float x, float w[3]) {
    w[0] = (x - n[1]) * (x - n[2]) / ((n[0] - n[1]) * (n[0] - n[2]));
    w[1] = (x - n[0]) * (x - n[2]) / ((n[1] - n[0]) * (n[1] - n[2]));
    w[2] = (x - n[0]) * (x - n[1]) / ((n[2] - n[0]) * (n[2] - n[1]));
}

// index of the packed upper triangle of the kPts x kPts Gram matrix
__device__ __host__ __forceinline__ constexpr int tri(int i, int j) {
    return i <= j ? i * kPts - i * (i - 1) / 2 + (j - i) : j * kPts - j * (j - 1) / 2 + (i - j);
}

// cp.async (Ampere-style asynchronous global -> shared copies, cached in
// L1 for the 4- and 8-byte forms) and its commit / wait groups.
__device__ __forceinline__ void cp_async4(void *smem, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(g)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(g)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// What the accumulation of one voxel needs: its stencil's rows (per B1
// block of the stencil) and their weights, the node offsets and the basis
// coefficients.
struct Prep {
    const float2 *rows[3][kPts];
    float qw[3];
    int nq;
    float T1c, T2c, hum, hup, hvm, hvp, hud, hvd, hud2, hvd2, inv_uv;
    Quad cu, cv;
};

// The stencil of voxel v and its B1 weights (the whole warp takes part);
// false: the voxel keeps its grid point.
__device__ __forceinline__ bool prepare(const Args &a, long long v, int lane, Prep &P) {
    const long long k = a.index[v];
    if (k < 0 || k >= a.NATOMS) return false;
    const float *mp = a.maps + v * a.nmaps;
    const long long b = k / a.natoms, j = k - b * a.natoms, bb = b * a.natoms;
    const float T1c = prm(a, k, 0), T2c = prm(a, k, 1);
    // the maps must still hold the matched grid point
    if (mp[0] != T1c || mp[1] != T2c || !(T1c > T2c) || !(T2c > 0.f)) return false;
    long long st[kPts];
    bool diag_up = true;
    if (!find_stencil(a, bb, j, st, &diag_up)) return false;
    // B1 blocks and their weights at the voxel's B1
    const long long nb = a.NATOMS / a.natoms;
    P.nq = 1;
    long long qbase[3] = {bb, bb, bb};
    P.qw[0] = 1.f;
    P.qw[1] = P.qw[2] = 0.f;
    if (a.b1map && nb >= 3) {
        const long long bs = min(max(b - 1, 0ll), nb - 3);
        float nodes[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            qbase[q] = (bs + q) * a.natoms;
            nodes[q] = prm(a, qbase[q] + j, 3);
        }
        // the same (T1, T2, B0) rows in every block of the stencil (one
        // check per lane, selected without indexing the arrays by lane)
        bool ok = true;
        if (lane < 3 * kPts) {
            const int q = lane / kPts, i = lane % kPts;
            long long row = 0, qb = 0;
            float node = 0.f;
#pragma unroll
            for (int ii = 0; ii < kPts; ii++)
                if (ii == i) row = st[ii];
#pragma unroll
            for (int qq = 0; qq < 3; qq++)
                if (qq == q) {
                    qb = qbase[qq];
                    node = nodes[qq];
                }
            const long long r0 = bb + row, r1 = qb + row;
            ok = prm(a, r0, 0) == prm(a, r1, 0) && prm(a, r0, 1) == prm(a, r1, 1) &&
                 prm(a, r0, 2) == prm(a, r1, 2) && prm(a, r1, 3) == node;
        }
        if (!__all_sync(0xffffffffu, ok)) return false;
        if (!(nodes[0] != nodes[1] && nodes[1] != nodes[2] && nodes[0] != nodes[2])) return false;
        const float bv = a.b1map[v];
        if (!isfinite(bv)) return false;
        lagrange3(nodes, bv, P.qw);
        P.nq = 3;
    }
    // node offsets as logs of ratios (exact to rounding) and the basis
    // coefficients along T1, along T2 and of the diagonal
    P.T1c = T1c;
    P.T2c = T2c;
    P.hum = logf(prm(a, bb + st[kUm], 0) / T1c);
    P.hup = logf(prm(a, bb + st[kUp], 0) / T1c);
    P.hvm = logf(prm(a, bb + st[kVm], 1) / T2c);
    P.hvp = logf(prm(a, bb + st[kVp], 1) / T2c);
    P.hud = diag_up ? P.hup : P.hum;
    P.hvd = diag_up ? P.hvp : P.hvm;
    P.hud2 = P.hud * P.hud;
    P.hvd2 = P.hvd * P.hvd;
    P.inv_uv = 1.f / (P.hud * P.hvd);
    P.cu = quad_coeffs(P.hum, P.hup);
    P.cv = quad_coeffs(P.hvm, P.hvp);
    // (with Im rows, the float row's start in the same pointer)
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int i = 0; i < kPts; i++)
            P.rows[q][i] = a.imag_rows ? reinterpret_cast<const float2 *>(reinterpret_cast<const float *>(a.atoms) +
                                                                          (qbase[q] + st[i]) * a.atom_stride)
                                       : a.atoms + (qbase[q] + st[i]) * a.atom_stride;
    return true;
}

// The warp's sums of the system to the scratch rows, each value by one lane.
template <bool IMAG>
__device__ __forceinline__ void write_system(const Args &a, long long v, int lane, const Prep &P,
                                             const float *G, const float *Gi, const float *pr, const float *pi) {
    float *sys = a.sys + v;
    const long long n = a.nvox;
    const float hv[8] = {P.T1c, P.T2c, P.hum, P.hup, P.hvm, P.hvp, P.hud, P.hvd};
#pragma unroll
    for (int r = 0; r < 8; r++)
        if ((r & 31) == lane) sys[r * n] = hv[r];
#pragma unroll
    for (int r = 0; r < kPts; r++) {
        if (((kRowPr + r) & 31) == lane) sys[(kRowPr + r) * n] = pr[r];
        if (((kRowPi + r) & 31) == lane) sys[(kRowPi + r) * n] = pi[r];
    }
#pragma unroll
    for (int r = 0; r < kTri; r++) {
        if (((kRowG + r) & 31) == lane) sys[(kRowG + r) * n] = G[r];
        if (!IMAG && ((kRowGi + r) & 31) == lane) sys[(kRowGi + r) * n] = Gi[r];
    }
}

// One warp per voxel (complex atoms): the stencil, then the system of its
// surrogate accumulated over the time points and written to a.sys.
template <bool IMAG>
__global__ void __launch_bounds__(kWarps * 32) accumulate_kernel(const __grid_constant__ Args a) {
    const int lane = threadIdx.x & 31;
    const long long v = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (v >= a.nvox) return;  // whole warps leave together
    Prep P;
    if (!prepare(a, v, lane, P)) {
        if (lane == 0) a.sys[kRowT1 * a.nvox + v] = __int_as_float(0x7fc00000);
        return;
    }
    const int nq = P.nq;
    const float *qw = P.qw;
    const Quad cu = P.cu, cv = P.cv;
    const float hud = P.hud, hvd = P.hvd, hud2 = P.hud2, hvd2 = P.hvd2, inv_uv = P.inv_uv;
    const float2 *const(*rows)[kPts] = P.rows;
    const float2 *xv = a.img + v * a.img_stride;

    // Hermitian Gram matrix of the basis, sum_t conj(m_r) m_c: real part G
    // (upper triangle), imaginary part Gi (strict upper triangle, zero for
    // purely imaginary atoms); inner products with the voxel,
    // sum_t conj(m_r) x = (pr, pi)
    float G[kTri], Gi[IMAG ? 1 : kTri], pr[kPts], pi[kPts];
#pragma unroll
    for (int i = 0; i < kTri; i++) G[i] = 0.f;
#pragma unroll
    for (int i = 0; i < (IMAG ? 1 : kTri); i++) Gi[i] = 0.f;
#pragma unroll
    for (int i = 0; i < kPts; i++) pr[i] = pi[i] = 0.f;

    // one part (real or imaginary) of the stencil at one sample -> the basis
    // (c, a, b, d, e, f)
    auto basis = [&](const float s[kPts], float m[kPts]) {
        const float c = s[kC];
        const float dpu = s[kUp] - c, dmu = s[kUm] - c, dpv = s[kVp] - c, dmv = s[kVm] - c;
        const float au = fmaf(cu.b1, dpu, cu.b2 * dmu), du = fmaf(cu.a1, dpu, cu.a2 * dmu);
        const float bv = fmaf(cv.b1, dpv, cv.b2 * dmv), ev = fmaf(cv.a1, dpv, cv.a2 * dmv);
        // the cross term: what the diagonal node leaves after the others
        float r = s[kD] - c;
        r = fmaf(-au, hud, r);
        r = fmaf(-bv, hvd, r);
        r = fmaf(-du, hud2, r);
        r = fmaf(-ev, hvd2, r);
        m[0] = c;
        m[1] = au;
        m[2] = bv;
        m[3] = du;
        m[4] = ev;
        m[5] = r * inv_uv;
    };

    // Staging: each lane copies its own samples of the stencil rows and of
    // the voxel into this warp's ring of kStages shared-memory slots with
    // cp.async, kStages - 1 chunks of 32 samples ahead of the arithmetic, and
    // reads back only what it copied itself.  The loads in flight hold no
    // registers, so many more of them are outstanding per SM than register
    // prefetching would allow.
    using Vt = typename std::conditional<IMAG, float, float2>::type;
    constexpr int kStages = stages<IMAG>();
    constexpr int kRows = 3 * kPts;
    extern __shared__ __align__(16) unsigned char rs_smem[];
    Vt *sa = reinterpret_cast<Vt *>(rs_smem) + (size_t)(threadIdx.x >> 5) * kStages * kRows * 32;
    float2 *sx = reinterpret_cast<float2 *>(reinterpret_cast<Vt *>(rs_smem) + (size_t)kWarps * kStages * kRows * 32) +
                 (threadIdx.x >> 5) * kStages * 32;
    const int nch = (a.T + 31) / 32;
    auto issue = [&](int kc) {
        const int t = kc * 32 + lane, slot = kc % kStages;
        if (t < a.T) {
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (q < nq)
#pragma unroll
                    for (int i = 0; i < kPts; i++) {
                        const float2 *g = rows[q][i] + t;
                        Vt *d = sa + (slot * kRows + q * kPts + i) * 32 + lane;
                        if (IMAG)
                            cp_async4(d, reinterpret_cast<const float *>(g) + 1);
                        else
                            cp_async8(d, g);
                    }
            cp_async8(sx + slot * 32 + lane, xv + t);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int kc = 0; kc < kStages - 1; kc++) issue(kc);

    for (int kc = 0; kc < nch; kc++) {
        issue(kc + kStages - 1);  // (an empty group past the end)
        cp_async_wait<kStages - 1>();
        const int t = kc * 32 + lane, slot = kc % kStages;
        if (t >= a.T) continue;
        const float2 x = sx[slot * 32 + lane];
        float sr[kPts], si[kPts];
#pragma unroll
        for (int i = 0; i < kPts; i++) {
            float accr = 0.f, acci = 0.f;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                if (q < nq) {
                    const Vt d = sa[(slot * kRows + q * kPts + i) * 32 + lane];
                    if constexpr (IMAG) {
                        acci = fmaf(qw[q], d, acci);
                    } else {
                        accr = fmaf(qw[q], d.x, accr);
                        acci = fmaf(qw[q], d.y, acci);
                    }
                }
            }
            sr[i] = accr;
            si[i] = acci;
        }
        float mi[kPts];
        basis(si, mi);
        if (IMAG) {
#pragma unroll
            for (int r = 0; r < kPts; r++) {
#pragma unroll
                for (int c = 0; c < kPts; c++)
                    if (c >= r) G[tri(r, c)] = fmaf(mi[r], mi[c], G[tri(r, c)]);
                // conj(i m) x = (m xi, -m xr)
                pr[r] = fmaf(mi[r], x.y, pr[r]);
                pi[r] = fmaf(-mi[r], x.x, pi[r]);
            }
        } else {
            float mr[kPts];
            basis(sr, mr);
#pragma unroll
            for (int r = 0; r < kPts; r++) {
#pragma unroll
                for (int c = 0; c < kPts; c++) {
                    if (c >= r) G[tri(r, c)] = fmaf(mr[r], mr[c], fmaf(mi[r], mi[c], G[tri(r, c)]));
                    if (c > r) Gi[tri(r, c)] = fmaf(mr[r], mi[c], fmaf(-mi[r], mr[c], Gi[tri(r, c)]));
                }
                pr[r] = fmaf(mr[r], x.x, fmaf(mi[r], x.y, pr[r]));
                pi[r] = fmaf(mr[r], x.y, fmaf(-mi[r], x.x, pi[r]));
            }
        }
    }
    // warp sums (every lane ends with the totals)
#pragma unroll
    for (int i = 0; i < kTri; i++)
#pragma unroll
        for (int o = 16; o; o >>= 1) G[i] += __shfl_xor_sync(0xffffffffu, G[i], o);
    if (!IMAG) {
#pragma unroll
        for (int i = 0; i < (IMAG ? 1 : kTri); i++)
#pragma unroll
            for (int o = 16; o; o >>= 1) Gi[i] += __shfl_xor_sync(0xffffffffu, Gi[i], o);
    }
#pragma unroll
    for (int i = 0; i < kPts; i++)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            pr[i] += __shfl_xor_sync(0xffffffffu, pr[i], o);
            pi[i] += __shfl_xor_sync(0xffffffffu, pi[i], o);
        }
    write_system<IMAG>(a, v, lane, P, G, Gi, pr, pi);
}

// cp.async of `size` bytes of which the first `src_bytes` are read and the
// rest zero-filled (src_bytes 0: zeros, nothing read).
__device__ __forceinline__ void cp_async4_zfill(void *smem, const void *g, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(g), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async8_zfill(void *smem, const void *g, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(g), "r"(src_bytes)
                 : "memory");
}
// (16 bytes, not kept in L1: the voxel's own samples are read once)
__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *g, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(g), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ float2 two(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

constexpr int kStagesImag2 = 3;  // slots of 64 staged samples per warp

// One warp per voxel, purely imaginary atoms (zero-phase FISP / SR): each
// lane takes two adjacent samples of every chunk of 64 as a packed pair, so
// that the stencil's weights, the basis and the sums run on two-wide FP32
// instructions, with two partial sums per entry (the even and the odd
// samples) added at the end.  The imaginary parts of the stencil rows and
// the voxel samples are staged with cp.async as above; the samples past the
// last one are zero-filled by the copies, so they add nothing.
//
// PAIRS: Im rows whose sample pairs are 8-byte aligned (even row stride) and
// an image whose pairs of complex samples are 16-byte aligned: one copy of a
// pair per row and one of the voxel's two samples, instead of one per sample.
template <bool PAIRS>
__global__ void __launch_bounds__(kWarps * 32) accumulate_imag_kernel(const __grid_constant__ Args a) {
    const int lane = threadIdx.x & 31;
    const long long v = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (v >= a.nvox) return;  // whole warps leave together
    Prep P;
    if (!prepare(a, v, lane, P)) {
        if (lane == 0) a.sys[kRowT1 * a.nvox + v] = __int_as_float(0x7fc00000);
        return;
    }
    const int nq = P.nq;
    const float2 qw0 = two(P.qw[0]), qw1 = two(P.qw[1]), qw2 = two(P.qw[2]);
    const float2 a1u = two(P.cu.a1), a2u = two(P.cu.a2), b1u = two(P.cu.b1), b2u = two(P.cu.b2);
    const float2 a1v = two(P.cv.a1), a2v = two(P.cv.a2), b1v = two(P.cv.b1), b2v = two(P.cv.b2);
    const float2 nhud = two(-P.hud), nhvd = two(-P.hvd), nhud2 = two(-P.hud2), nhvd2 = two(-P.hvd2);
    const float2 inv_uv = two(P.inv_uv);
    const float2 *xv = a.img + v * a.img_stride;

    constexpr int kRows = 3 * kPts;
    constexpr int S = kStagesImag2;
    extern __shared__ __align__(16) unsigned char rs_smem[];
    float2 *sa = reinterpret_cast<float2 *>(rs_smem) + (size_t)(threadIdx.x >> 5) * S * kRows * 32;
    float4 *sx = reinterpret_cast<float4 *>(reinterpret_cast<float2 *>(rs_smem) + (size_t)kWarps * S * kRows * 32) +
                 (threadIdx.x >> 5) * S * 32;
    const int nch = (a.T + 63) / 64;
    auto issue = [&](int kc) {
        const int t0 = kc * 64 + 2 * lane, slot = kc % S;
        if (kc < nch) {
            const int b0 = t0 < a.T ? 4 : 0, b1 = t0 + 1 < a.T ? 4 : 0;
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (q < nq)
#pragma unroll
                    for (int i = 0; i < kPts; i++) {
                        // (a sample past the end reads nothing: its address is the row's;
                        // Im of sample t: g[t] in Im rows, g[2t + 1] in complex rows)
                        const float *g = reinterpret_cast<const float *>(P.rows[q][i]);
                        float *d = reinterpret_cast<float *>(sa + (slot * kRows + q * kPts + i) * 32 + lane);
                        if (PAIRS) {
                            cp_async8_zfill(d, g + (b0 ? t0 : 0), b0 + b1);
                        } else if (a.imag_rows) {
                            cp_async4_zfill(d, g + (b0 ? t0 : 0), b0);
                            cp_async4_zfill(d + 1, g + (b1 ? t0 + 1 : 0), b1);
                        } else {
                            cp_async4_zfill(d, g + (b0 ? 2 * t0 + 1 : 1), b0);
                            cp_async4_zfill(d + 1, g + (b1 ? 2 * t0 + 3 : 1), b1);
                        }
                    }
            float *dx = reinterpret_cast<float *>(sx + slot * 32 + lane);
            if (PAIRS) {
                cp_async16_zfill(dx, xv + (b0 ? t0 : 0), 2 * (b0 + b1));
            } else {
                cp_async8_zfill(dx, xv + (b0 ? t0 : 0), 2 * b0);
                cp_async8_zfill(dx + 2, xv + (b1 ? t0 + 1 : 0), 2 * b1);
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int kc = 0; kc < S - 1; kc++) issue(kc);

    float2 G2[kTri], pr2[kPts], pi2[kPts];
#pragma unroll
    for (int i = 0; i < kTri; i++) G2[i] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < kPts; i++) pr2[i] = pi2[i] = make_float2(0.f, 0.f);

    for (int kc = 0; kc < nch; kc++) {
        issue(kc + S - 1);  // (an empty group past the end)
        cp_async_wait<S - 1>();
        if (kc * 64 + 2 * lane >= a.T) continue;
        const int slot = kc % S;
        const float4 x4 = sx[slot * 32 + lane];
        const float2 xr = make_float2(x4.x, x4.z), nxr = make_float2(-x4.x, -x4.z), xi = make_float2(x4.y, x4.w);
        float2 sv[kPts];
#pragma unroll
        for (int i = 0; i < kPts; i++) {
            const float2 *d = sa + (slot * kRows + i) * 32 + lane;
            float2 acc = __fmul2_rn(qw0, d[0]);
            if (nq > 1) {
                acc = __ffma2_rn(qw1, d[kPts * 32], acc);
                acc = __ffma2_rn(qw2, d[2 * kPts * 32], acc);
            }
            sv[i] = acc;
        }
        // the basis (c, a, b, d, e, f) of both samples
        float2 m[kPts];
        const float2 c = sv[kC];
        const float2 dpu = sub2(sv[kUp], c), dmu = sub2(sv[kUm], c), dpv = sub2(sv[kVp], c), dmv = sub2(sv[kVm], c);
        m[0] = c;
        m[1] = __ffma2_rn(b1u, dpu, __fmul2_rn(b2u, dmu));
        m[3] = __ffma2_rn(a1u, dpu, __fmul2_rn(a2u, dmu));
        m[2] = __ffma2_rn(b1v, dpv, __fmul2_rn(b2v, dmv));
        m[4] = __ffma2_rn(a1v, dpv, __fmul2_rn(a2v, dmv));
        float2 r = sub2(sv[kD], c);
        r = __ffma2_rn(m[1], nhud, r);
        r = __ffma2_rn(m[2], nhvd, r);
        r = __ffma2_rn(m[3], nhud2, r);
        r = __ffma2_rn(m[4], nhvd2, r);
        m[5] = __fmul2_rn(r, inv_uv);
#pragma unroll
        for (int rr = 0; rr < kPts; rr++) {
#pragma unroll
            for (int cc = 0; cc < kPts; cc++)
                if (cc >= rr) G2[tri(rr, cc)] = __ffma2_rn(m[rr], m[cc], G2[tri(rr, cc)]);
            // conj(i m) x = (m xi, -m xr)
            pr2[rr] = __ffma2_rn(m[rr], xi, pr2[rr]);
            pi2[rr] = __ffma2_rn(m[rr], nxr, pi2[rr]);
        }
    }
    float G[kTri], pr[kPts], pi[kPts];
#pragma unroll
    for (int i = 0; i < kTri; i++) G[i] = G2[i].x + G2[i].y;
#pragma unroll
    for (int i = 0; i < kPts; i++) {
        pr[i] = pr2[i].x + pr2[i].y;
        pi[i] = pi2[i].x + pi2[i].y;
    }
    // warp sums (every lane ends with the totals)
#pragma unroll
    for (int i = 0; i < kTri; i++)
#pragma unroll
        for (int o = 16; o; o >>= 1) G[i] += __shfl_xor_sync(0xffffffffu, G[i], o);
#pragma unroll
    for (int i = 0; i < kPts; i++)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            pr[i] += __shfl_xor_sync(0xffffffffu, pr[i], o);
            pi[i] += __shfl_xor_sync(0xffffffffu, pi[i], o);
        }
    write_system<true>(a, v, lane, P, G, nullptr, pr, pi);
}

// One thread per voxel: Gauss-Newton with variable projection on the
// surrogate s(U, V) = c + a U + b V + d U^2 + e V^2 + f U V and its
// derivatives, from the matched grid point (U = V = 0).  Each step is
// clipped to half the stencil's width, and the point may leave the stencil by
// half its extent on each side (a match more than a grid step from the fit:
// the quadratic extrapolates, still nearer than the grid point).
template <bool IMAG>
__global__ void __launch_bounds__(128) solve_kernel(const __grid_constant__ Args a) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvox) return;
    const float *sys = a.sys + v;
    const long long n = a.nvox;
    const float T1c = sys[kRowT1 * n];
    if (isnan(T1c)) return;
    const float T2c = sys[kRowT2 * n];
    const float hum = sys[(kRowH + 0) * n], hup = sys[(kRowH + 1) * n];
    const float hvm = sys[(kRowH + 2) * n], hvp = sys[(kRowH + 3) * n];
    float G[kTri], Gi[IMAG ? 1 : kTri], pr[kPts], pi[kPts];
#pragma unroll
    for (int r = 0; r < kTri; r++) {
        G[r] = sys[(kRowG + r) * n];
        if (!IMAG) Gi[r] = sys[(kRowGi + r) * n];
    }
#pragma unroll
    for (int r = 0; r < kPts; r++) {
        pr[r] = sys[(kRowPr + r) * n];
        pi[r] = sys[(kRowPi + r) * n];
    }
    const float lu = 0.5f * (fmaxf(hum, hup) - fminf(hum, hup)), lv = 0.5f * (fmaxf(hvm, hvp) - fminf(hvm, hvp));
    const float ulo = 1.5f * fminf(hum, hup), uhi = 1.5f * fmaxf(hum, hup);
    const float vlo = 1.5f * fminf(hvm, hvp), vhi = 1.5f * fmaxf(hvm, hvp);
    float U = 0.f, V = 0.f;
    for (int it = 0; it < kSolveIters; it++) {
        // coefficient vectors of s, ds/dU and ds/dV in the basis
        const float c0[kPts] = {1.f, U, V, U * U, V * V, U * V};
        const float c1[kPts] = {0.f, 1.f, 0.f, 2.f * U, 0.f, V};
        const float c2[kPts] = {0.f, 0.f, 1.f, 0.f, 2.f * V, U};
        // G c for the three vectors, and Gi c0 (the imaginary parts of
        // s^H ds/dU, s^H ds/dV; Gi is antisymmetric)
        float g0[kPts], g1[kPts], g2[kPts], h0[kPts];
#pragma unroll
        for (int r = 0; r < kPts; r++) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, z0 = 0.f;
#pragma unroll
            for (int c = 0; c < kPts; c++) {
                const float g = G[tri(r, c)];
                s0 = fmaf(g, c0[c], s0);
                s1 = fmaf(g, c1[c], s1);
                s2 = fmaf(g, c2[c], s2);
                if (!IMAG && c != r) z0 = fmaf(c < r ? -Gi[tri(r, c)] : Gi[tri(r, c)], c0[c], z0);
            }
            g0[r] = s0;
            g1[r] = s1;
            g2[r] = s2;
            h0[r] = z0;
        }
        // s^H s, g_j = s^H J_j (complex), H_jk = Re J_j^H J_k, P = s^H x,
        // Q_j = J_j^H x
        float Ss = 0.f, G1 = 0.f, G2 = 0.f, G1i = 0.f, G2i = 0.f, H11 = 0.f, H12 = 0.f, H22 = 0.f;
        float Pr = 0.f, Pi = 0.f, Q1r = 0.f, Q1i = 0.f, Q2r = 0.f, Q2i = 0.f;
#pragma unroll
        for (int r = 0; r < kPts; r++) {
            Ss = fmaf(c0[r], g0[r], Ss);
            G1 = fmaf(c1[r], g0[r], G1);
            G2 = fmaf(c2[r], g0[r], G2);
            // c0^T Gi c_j = -(c_j^T Gi c0)
            G1i = fmaf(-c1[r], h0[r], G1i);
            G2i = fmaf(-c2[r], h0[r], G2i);
            H11 = fmaf(c1[r], g1[r], H11);
            H12 = fmaf(c1[r], g2[r], H12);
            H22 = fmaf(c2[r], g2[r], H22);
            Pr = fmaf(c0[r], pr[r], Pr);
            Pi = fmaf(c0[r], pi[r], Pi);
            Q1r = fmaf(c1[r], pr[r], Q1r);
            Q1i = fmaf(c1[r], pi[r], Q1i);
            Q2r = fmaf(c2[r], pr[r], Q2r);
            Q2i = fmaf(c2[r], pi[r], Q2i);
        }
        if (!(Ss > 0.f)) break;
        // rho = P / Ss; A_jk = |rho|^2 (H_jk - Re(conj(g_j) g_k) / Ss);
        // b_j = Re(conj(rho) (Q_j - conj(g_j) P / Ss)); delta = A^-1 b
        const float rr = Pr / Ss, ri = Pi / Ss, rho2 = rr * rr + ri * ri;
        const float A11 = rho2 * (H11 - (G1 * G1 + G1i * G1i) / Ss);
        const float A12 = rho2 * (H12 - (G1 * G2 + G1i * G2i) / Ss);
        const float A22 = rho2 * (H22 - (G2 * G2 + G2i * G2i) / Ss);
        // conj(g) P = (gr Pr + gi Pi, gr Pi - gi Pr)
        const float e1r = Q1r - (G1 * Pr + G1i * Pi) / Ss, e1i = Q1i - (G1 * Pi - G1i * Pr) / Ss;
        const float e2r = Q2r - (G2 * Pr + G2i * Pi) / Ss, e2i = Q2i - (G2 * Pi - G2i * Pr) / Ss;
        const float b1 = rr * e1r + ri * e1i, b2 = rr * e2r + ri * e2i;
        const float det = A11 * A22 - A12 * A12;
        if (!(det > 0.f) || !(A11 > 0.f) || !isfinite(det)) break;
        float d1 = (A22 * b1 - A12 * b2) / det, d2 = (A11 * b2 - A12 * b1) / det;
        if (!isfinite(d1) || !isfinite(d2)) break;
        d1 = fminf(fmaxf(d1, -lu), lu);
        d2 = fminf(fmaxf(d2, -lv), lv);
        U = fminf(fmaxf(U + d1, ulo), uhi);
        V = fminf(fmaxf(V + d2, vlo), vhi);
    }
    const float T1 = T1c * expf(U), T2 = T2c * expf(V);
    if (!isfinite(T1) || !isfinite(T2) || !(T2 > 0.f) || !(T1 > T2 * (1.f + 1e-4f))) return;
    float *mp = a.maps + v * a.nmaps;
    mp[0] = T1;
    mp[1] = T2;
    if (a.count) atomicAdd(a.count, 1);
}

}  // namespace rstart
}  // namespace snapmrf

using namespace snapmrf;

extern "C" int snapmrf_refine_start(float *d_maps, int nmaps, const int64_t *d_index, const float *d_atoms,
                                    const float *d_params, int nparams, size_t nreps, size_t NATOMS,
                                    size_t natoms, const float *img, size_t img_stride, size_t nvoxels,
                                    const float *d_b1map, unsigned flags, int *d_count, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_maps || !d_index || !d_atoms || !d_params || !img)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: null pointer");
    if (nmaps < 2 || nparams < 3 || (d_b1map && nparams < 4) || nreps == 0 || natoms == 0 || NATOMS % natoms)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: bad sizes");
    if (flags & ~(SNAPMRF_START_IMAG_ATOMS | SNAPMRF_START_IMAG_ROWS))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: unknown flags");
    if ((flags & SNAPMRF_START_IMAG_ROWS) && !(flags & SNAPMRF_START_IMAG_ATOMS))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: SNAPMRF_START_IMAG_ROWS needs SNAPMRF_START_IMAG_ATOMS");
    if ((reinterpret_cast<uintptr_t>(d_atoms) | reinterpret_cast<uintptr_t>(img)) %
        ((flags & SNAPMRF_START_IMAG_ROWS) ? sizeof(float) : sizeof(float2)))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: atoms and image must be aligned to their elements");
    if (reinterpret_cast<uintptr_t>(img) % sizeof(float2))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: the image must be 8-byte aligned (complex)");
    if (img_stride == 0) img_stride = nreps;
    if (img_stride < nreps) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "refine_start: img_stride < nreps");
    if (nreps > 0x7fffffff || NATOMS > (size_t)1 << 40 || nvoxels > ((size_t)1 << 31) - 1)
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "refine_start: sizes beyond the supported range");
    if (nvoxels == 0) return SNAPMRF_OK;
    rstart::Args a;
    a.maps = d_maps;
    a.nmaps = nmaps;
    a.index = d_index;
    a.atoms = reinterpret_cast<const float2 *>(d_atoms);
    a.atom_stride = (long long)nreps;
    a.params = d_params;
    a.nparams = nparams;
    a.NATOMS = (long long)NATOMS;
    a.natoms = (long long)natoms;
    a.img = reinterpret_cast<const float2 *>(img);
    a.img_stride = (long long)img_stride;
    a.T = (int)nreps;
    a.nvox = (long long)nvoxels;
    a.b1map = d_b1map;
    a.count = d_count;
    a.imag_rows = (flags & SNAPMRF_START_IMAG_ROWS) ? 1 : 0;
    const bool imag = flags & SNAPMRF_START_IMAG_ATOMS;
    DeviceScratch sys;
    SNAPMRF_CUDA(sys.alloc(nvoxels * (imag ? rstart::kSysRows : rstart::kSysRowsComplex) * sizeof(float), st));
    a.sys = sys.as<float>();
    const unsigned grid = (unsigned)((nvoxels + rstart::kWarps - 1) / rstart::kWarps);
    const unsigned grid2 = (unsigned)((nvoxels + 127) / 128);
    // staged samples: per warp kStages x 32 lanes x (3 kPts atom values + the voxel)
    const size_t smem = (size_t)rstart::kWarps * (imag ? rstart::stages<true>() : rstart::stages<false>()) * 32 *
                        (3 * rstart::kPts * (imag ? sizeof(float) : sizeof(float2)) + sizeof(float2));
    if (imag) {
        // staged pairs of samples: per warp kStagesImag2 x 32 lanes x (3 kPts
        // pairs of imaginary parts + two complex voxel samples)
        const size_t smem2 = (size_t)rstart::kWarps * rstart::kStagesImag2 * 32 *
                             (3 * rstart::kPts * sizeof(float2) + sizeof(float4));
        const bool pairs = a.imag_rows && nreps % 2 == 0 && img_stride % 2 == 0 &&
                           reinterpret_cast<uintptr_t>(d_atoms) % 8 == 0 && reinterpret_cast<uintptr_t>(img) % 16 == 0;
        auto kern = pairs ? rstart::accumulate_imag_kernel<true> : rstart::accumulate_imag_kernel<false>;
        SNAPMRF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
        kern<<<grid, rstart::kWarps * 32, smem2, st>>>(a);
        SNAPMRF_LAUNCH_CHECK();
        rstart::solve_kernel<true><<<grid2, 128, 0, st>>>(a);
    } else {
        SNAPMRF_CUDA(cudaFuncSetAttribute(rstart::accumulate_kernel<false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        rstart::accumulate_kernel<false><<<grid, rstart::kWarps * 32, smem, st>>>(a);
        SNAPMRF_LAUNCH_CHECK();
        rstart::solve_kernel<false><<<grid2, 128, 0, st>>>(a);
    }
    SNAPMRF_LAUNCH_CHECK();
    return SNAPMRF_OK;
}

