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
