/*
 * snapMRF oracle: CPU restatement of the reference's dictionary generation
 * (EPG / ROA) and maximum-inner-product matching.
 *
 * TEST INFRASTRUCTURE ONLY.  Built into oracle/liboracle.so and loaded by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker.  The product (snapmrf_b200/) never links or calls it.
 *
 * Two variants are exported from one source (oracle_core.inc):
 *   *_f64  exact math (double) on the reference's float inputs
 *   *_f32  the reference's float operation order, libm sinf/cosf/expf in
 *          place of the device __sincosf/expf
 * Both parallelise over atoms / voxels with OpenMP (nthreads argument).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>

#define ORACLE_ALL_B1_BLOCKS 1u /* non-SSFP echo types: every B1 block, alpha*b1 */
#define ORACLE_NORMALIZE 2u     /* normalise every generated atom */

enum { ECHO_SSFP = 0, ECHO_ROA = 1, ECHO_SR = 2, ECHO_SE = 3, ECHO_TSE = 4, ECHO_FISP = 5 };

/* MRF_dict's schedule preparation (src/functions.cu:1229-1291) and the
 * per-B1-block flip angles.  SSFP reproduces the in-place FA*b1 then
 * FA*(1/b1) drift across blocks (src/functions.cu:969-973, 1011-1013). */
static void oracle_prepare_schedule(float *mrf, float *alpha, const float *params,
                                    const float *h_mrf, size_t nreps, size_t NREPS,
                                    size_t NATOMS, size_t natoms, int nparams, int echo,
                                    unsigned flags)
{
    size_t nblocks = NATOMS / natoms;
    for (int r = 0; r < 4; r++)
        for (size_t t = 0; t < nreps; t++) mrf[r * nreps + t] = h_mrf[r * NREPS + t];
    if (echo == ECHO_SSFP || echo == ECHO_ROA) {
        const float nominal_flip = 60.f, TR_base = 16.f, TE_base = 3.5f;
        const float fa_scale = (float)(nominal_flip * M_PI / 180.f);
        const float ph_scale = (float)(M_PI / 180.f);
        for (size_t t = 0; t < nreps; t++) {
            mrf[t] *= fa_scale;
            mrf[nreps + t] *= ph_scale;
            mrf[2 * nreps + t] += TR_base;
            mrf[3 * nreps + t] += TE_base;
        }
    }
    if (echo == ECHO_SSFP) {
        float *fa = (float *)malloc(nreps * sizeof(float));
        memcpy(fa, mrf, nreps * sizeof(float));
        for (size_t j = 0; j < nblocks; j++) {
            float b1 = params[j * natoms * nparams + 3];
            for (size_t t = 0; t < nreps; t++) fa[t] *= b1;
            memcpy(alpha + j * nreps, fa, nreps * sizeof(float));
            float inv = 1.f / b1;
            for (size_t t = 0; t < nreps; t++) fa[t] *= inv;
        }
        free(fa);
    } else {
        for (size_t j = 0; j < nblocks; j++) {
            float b1 = params[j * natoms * nparams + 3];
            for (size_t t = 0; t < nreps; t++)
                alpha[j * nreps + t] = (flags & ORACLE_ALL_B1_BLOCKS) ? mrf[t] * b1 : mrf[t];
        }
    }
}

#define REAL double
#define SUFFIX _f64
#define ORACLE_IS_F32 0
#include "oracle_core.inc"
#undef REAL
#undef SUFFIX
#undef ORACLE_IS_F32

#define REAL float
#define SUFFIX _f32
#define ORACLE_IS_F32 1
#include "oracle_core.inc"

/* Number of OpenMP threads the CPU can run (for the CPU baseline leg). */
int oracle_max_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------
 * FP64 forward mode (one tangent) for the FISP / SR recursion with every RF
 * phase 0 (epg_fisp src/functions.cu:878-933, epg_sr :687-739; RF matrix
 * :483-508 at phi = 0), the form the derivative kernels differentiate:
 * state (f+, f-, z) = (Im F+, Im F-, Re Z) per EPG state, flip angle
 * alpha_t * b1 (the B1 extension of epg_fisp), readout s_t = i f+[0] after
 * relax(TE) (no normalisation).  Each state carries a value and a
 * derivative along one direction (dT1, dT2, dB1, dalpha[t]).
 * mrf is a compact [4][nreps] schedule.
 *
 * Outputs: sig[T] (value of Im s_t) and dsig[T] (its tangent);
 * loss = sum_t |s_t - y_t|^2 and dloss, its derivative along the direction,
 * with y[2T] interleaved complex targets (NULL: no loss).
 * ---------------------------------------------------------------------- */
typedef struct { double v, d; } dual;

static inline dual dmk(double v, double d) { dual r; r.v = v; r.d = d; return r; }
static inline dual dadd(dual a, dual b) { return dmk(a.v + b.v, a.d + b.d); }
static inline dual dmul(dual a, dual b) { return dmk(a.v * b.v, a.d * b.v + a.v * b.d); }
static inline dual dexp(dual a) { double e = exp(a.v); return dmk(e, e * a.d); }
static inline dual dsin(dual a) { return dmk(sin(a.v), cos(a.v) * a.d); }
static inline dual dcos(dual a) { return dmk(cos(a.v), -sin(a.v) * a.d); }
static inline dual ddiv(dual a, dual b) { return dmk(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }

int oracle_fisp_jvp_f64(double *sig, double *dsig, double *loss, double *dloss, double T1, double T2, double B1,
                        double dT1, double dT2, double dB1, const float *mrf, const double *dalpha, size_t nreps,
                        int nstates, int shift, const double *y)
{
    int w = nstates;
    dual *fp = (dual *)calloc(3 * (size_t)w, sizeof(dual));
    if (!fp) return -3;
    dual *fm = fp + w, *z = fm + w;
    const float *alpha = mrf, *TR = mrf + 2 * nreps, *TE = mrf + 3 * nreps;
    z[0] = dmk(1, 0);
    dual t1 = dmk(T1, dT1), t2 = dmk(T2, dT2), b1 = dmk(B1, dB1);
    dual L = dmk(0, 0);
    for (size_t i = 0; i < nreps; i++) {
        dual a = dmul(dmk(alpha[i], dalpha ? dalpha[i] : 0), b1);
        dual sa = dsin(a), ca = dcos(a);
        dual c2 = dmul(dadd(dmk(1, 0), ca), dmk(0.5, 0)), s2 = dmul(dadd(dmk(1, 0), dmk(-ca.v, -ca.d)), dmk(0.5, 0));
        dual hs = dmul(sa, dmk(0.5, 0));
        for (int k = 0; k < w; k++) {
            dual p = fp[k], m = fm[k], q = z[k];
            fp[k] = dadd(dadd(dmul(c2, p), dmul(s2, m)), dmul(dmk(-sa.v, -sa.d), q));
            fm[k] = dadd(dadd(dmul(s2, p), dmul(c2, m)), dmul(sa, q));
            z[k] = dadd(dadd(dmul(hs, p), dmul(dmk(-hs.v, -hs.d), m)), dmul(ca, q));
        }
        double ta = (double)TE[i], tb = (double)TR[i] - (double)TE[i];
        for (int pass = 0; pass < 2; pass++) {
            double t = pass == 0 ? ta : tb;
            dual E1 = dexp(ddiv(dmk(-t, 0), t1)), E2 = dexp(ddiv(dmk(-t, 0), t2));
            for (int k = 0; k < w; k++) {
                fp[k] = dmul(fp[k], E2);
                fm[k] = dmul(fm[k], E2);
                z[k] = dmul(z[k], E1);
            }
            z[0] = dadd(z[0], dmk(1 - E1.v, -E1.d));
            if (pass == 0) {
                sig[i] = fp[0].v;
                dsig[i] = fp[0].d;
                if (y) {
                    double re = -(double)y[2 * i], im = fp[0].v - y[2 * i + 1];
                    L.v += re * re + im * im;
                    L.d += 2 * im * fp[0].d;
                }
                if (shift) {
                    for (int k = w - 1; k >= 1; k--) fp[k] = fp[k - 1];
                    dual f0 = fm[0];
                    for (int k = 0; k <= w - 2; k++) fm[k] = fm[k + 1];
                    fp[0] = dmk(-(w == 1 ? f0.v : fm[0].v), -(w == 1 ? f0.d : fm[0].d));
                    fm[w - 1] = dmk(0, 0);
                }
            }
        }
    }
    if (loss) *loss = L.v;
    if (dloss) *dloss = L.d;
    free(fp);
    return 0;
}

/* ------------------------------------------------------------------------
 * FP64 forward mode (one tangent) for the complex bSSFP recursion of
 * epg_ssfp (src/functions.cu:935-1019): inversion by init_rf_pulse with
 * alpha = 180 deg, phi = 0 and delay TI (:456-481, 965-966); per step the RF
 * matrix of fill_transition_matrix (:483-508) at flip alpha_t * B1 and phase
 * phi_t, relaxation over TE (:530-583), B0 precession exp(+-i 2 pi B0 t /
 * 1000) over TE (:585-607), readout F+[0] (:609-617), B0 precession over
 * TR - TE, the dephasing shift (:619-668), relaxation over TR - TE.  The
 * atoms are not normalised.  mrf is the converted compact [4][nreps]
 * schedule (flip rad, phase rad, TR ms, TE ms).  Each quantity carries a
 * value and a derivative along (dT1, dT2, dB0, dB1).
 * Outputs: sig[2T] and dsig[2T], interleaved complex.
 * ---------------------------------------------------------------------- */
typedef struct { dual re, im; } cdual;

static inline cdual cdmk(dual re, dual im) { cdual r; r.re = re; r.im = im; return r; }
static inline cdual cdadd(cdual a, cdual b) { return cdmk(dadd(a.re, b.re), dadd(a.im, b.im)); }
static inline cdual cdmul(cdual a, cdual b)
{
    return cdmk(dadd(dmul(a.re, b.re), dmul(dmk(-a.im.v, -a.im.d), b.im)),
                dadd(dmul(a.re, b.im), dmul(a.im, b.re)));
}
static inline cdual cdscale(cdual a, dual s) { return cdmk(dmul(a.re, s), dmul(a.im, s)); }
static inline cdual cdconj(cdual a) { return cdmk(a.re, dmk(-a.im.v, -a.im.d)); }
static inline cdual cdzero(void) { return cdmk(dmk(0, 0), dmk(0, 0)); }

int oracle_ssfp_jvp_f64(double *sig, double *dsig, double T1, double T2, double B0, double B1, double dT1,
                        double dT2, double dB0, double dB1, const float *mrf, size_t nreps, int nstates, double TI)
{
    int w = nstates;
    cdual *fp = (cdual *)calloc(3 * (size_t)w, sizeof(cdual));
    if (!fp) return -3;
    cdual *fm = fp + w, *z = fm + w;
    for (int k = 0; k < 3 * w; k++) fp[k] = cdzero();
    const float *alpha = mrf, *phi = mrf + nreps, *TR = mrf + 2 * nreps, *TE = mrf + 3 * nreps;
    dual t1 = dmk(T1, dT1), t2 = dmk(T2, dT2), b0 = dmk(B0, dB0), b1 = dmk(B1, dB1);
    /* inversion: F+0 = conj(q), F-0 = q with q = E2(TI) sin(a0) (sin p0 + i cos p0),
     * Z0 = E1(TI) cos(a0) + 1 - E1(TI), a0 = pi, p0 = 0 */
    {
        dual e1 = dexp(ddiv(dmk(-TI, 0), t1)), e2 = dexp(ddiv(dmk(-TI, 0), t2));
        double a0 = M_PI, p0 = 0.0;
        cdual q = cdscale(cdmk(dmk(sin(p0), 0), dmk(cos(p0), 0)), dmul(e2, dmk(sin(a0), 0)));
        fp[0] = cdconj(q);
        fm[0] = q;
        z[0] = cdmk(dadd(dmul(e1, dmk(cos(a0), 0)), dmk(1 - e1.v, -e1.d)), dmk(0, 0));
    }
    for (size_t i = 0; i < nreps; i++) {
        dual a = dmul(dmk(alpha[i], 0), b1);
        dual sa = dsin(a), ca = dcos(a);
        dual sa2 = dmul(dadd(dmk(1, 0), dmk(-ca.v, -ca.d)), dmk(0.5, 0));
        dual ca2 = dmul(dadd(dmk(1, 0), ca), dmk(0.5, 0));
        cdual zz = cdmk(dmk(cos((double)phi[i]), 0), dmk(sin((double)phi[i]), 0)), zi = cdconj(zz);
        cdual I = cdmk(dmk(0, 0), dmk(1, 0)), mI = cdmk(dmk(0, 0), dmk(-1, 0));
        cdual M[9];
        M[0] = cdmk(ca2, dmk(0, 0));
        M[1] = cdscale(cdmul(zz, zz), sa2);
        M[2] = cdscale(cdmul(mI, zz), sa);
        M[3] = cdscale(cdmul(zi, zi), sa2);
        M[4] = cdmk(ca2, dmk(0, 0));
        M[5] = cdscale(cdmul(I, zi), sa);
        M[6] = cdscale(cdmul(mI, zi), dmul(sa, dmk(0.5, 0)));
        M[7] = cdscale(cdmul(I, zz), dmul(sa, dmk(0.5, 0)));
        M[8] = cdmk(ca, dmk(0, 0));
        for (int k = 0; k < w; k++) {
            cdual p = fp[k], m = fm[k], q = z[k];
            fp[k] = cdadd(cdadd(cdmul(M[0], p), cdmul(M[1], m)), cdmul(M[2], q));
            fm[k] = cdadd(cdadd(cdmul(M[3], p), cdmul(M[4], m)), cdmul(M[5], q));
            z[k] = cdadd(cdadd(cdmul(M[6], p), cdmul(M[7], m)), cdmul(M[8], q));
        }
        double ta = (double)TE[i], tb = (double)TR[i] - (double)TE[i];
        for (int pass = 0; pass < 2; pass++) {
            double t = pass == 0 ? ta : tb;
            if (pass == 1) {
                dual th = dmul(b0, dmk(2 * M_PI * t / 1000.0, 0));
                cdual e = cdmk(dcos(th), dsin(th)), ec = cdconj(e);
                for (int k = 0; k < w; k++) {
                    fp[k] = cdmul(e, fp[k]);
                    fm[k] = cdmul(ec, fm[k]);
                }
                for (int k = w - 1; k >= 1; k--) fp[k] = fp[k - 1];
                cdual f0 = fm[0];
                for (int k = 0; k <= w - 2; k++) fm[k] = fm[k + 1];
                fp[0] = cdconj(w == 1 ? f0 : fm[0]);
                fm[w - 1] = cdzero();
            }
            dual E1 = dexp(ddiv(dmk(-t, 0), t1)), E2 = dexp(ddiv(dmk(-t, 0), t2));
            for (int k = 0; k < w; k++) {
                fp[k] = cdscale(fp[k], E2);
                fm[k] = cdscale(fm[k], E2);
                z[k] = cdscale(z[k], E1);
            }
            z[0].re = dadd(z[0].re, dmk(1 - E1.v, -E1.d));
            if (pass == 0) {
                dual th = dmul(b0, dmk(2 * M_PI * t / 1000.0, 0));
                cdual e = cdmk(dcos(th), dsin(th)), ec = cdconj(e);
                for (int k = 0; k < w; k++) {
                    fp[k] = cdmul(e, fp[k]);
                    fm[k] = cdmul(ec, fm[k]);
                }
                sig[2 * i] = fp[0].re.v;
                sig[2 * i + 1] = fp[0].im.v;
                dsig[2 * i] = fp[0].re.d;
                dsig[2 * i + 1] = fp[0].im.d;
            }
        }
    }
    free(fp);
    return 0;
}
