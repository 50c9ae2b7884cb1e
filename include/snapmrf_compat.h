/*
 * snapmrf_compat.h -- the reference's host-function surface, implemented by
 * libsnapmrf_compat.so on top of the C ABI (snapmrf.h).
 *
 * The reference's drivers (src/mrf.cu, src/test.cu) call C++ functions
 * declared in its src/functions.h:33-56, 108-144 and the RA functions of
 * src/ra.h:60-74.  This header declares the same functions with the same
 * parameter types, so the symbols (C++ mangled names; C names for the RA
 * functions) are the ones those drivers link against: a driver built
 * against the reference's own header links unchanged against
 * libsnapmrf_compat.so.  Behaviour follows the reference's, with its
 * exit-on-error convention (message on stderr, then exit) but without the
 * wait on stdin; MRF_dict and MRF_match return after the device work ends.
 */
#ifndef SNAPMRF_COMPAT_H
#define SNAPMRF_COMPAT_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

/* the schedule row of the reference's unit tests (src/functions.h:22-28) */
typedef struct ImagingParams {
    float alpha;
    float phi;
    float TR;
    float TE;
} IP;

/* launch-shape and stream globals the reference's drivers declare extern
 * (src/functions.cu:29-33); the shape is accepted and ignored */
extern int blocksize;
extern int gridsize;
extern cudaStream_t stream[2];

void gpuAssert(cudaError_t code, const char *file, int line);
void *mallocAssert(size_t n, const char *file, int line);
void freeAssert(void *p, const char *file, int line);
void print_usage();
size_t csv_dim(const char *filepath);
void csv_read(float *h_mrf, size_t nreps, const char *filepath);
void save_rafile(float2 *h_atoms, const char *atoms_path, size_t dim0, size_t dim1);
void save_rafile(float *h_params, const char *p_path, size_t dim0, size_t dim1);
void parse_range(const char *str, float *min, float *step, float *max, size_t *len);
size_t parse_length(const char *str);
void linspace(float *h_p, float min, float step, size_t len);
void parse_params(float *h_p, const char *str, size_t LEN);
void logspace(float *h_p, float min, float max, size_t len);
void trans_params(float *h_params, float *h_t1, float *h_t2, float *h_b0, float *h_b1, size_t l_t1,
                  size_t l_t2, size_t l_b0, size_t l_b1, size_t NATOMS, int nparams);
size_t compute_natoms(float *h_t1, float *h_t2, size_t l_t1, size_t l_t2, size_t l_b0, size_t l_b1);
void MRF_dict(float2 *d_atoms, float *d_params, float *h_mrf, size_t nreps, size_t NREPS, size_t NATOMS,
              size_t natoms, int nparams, int nstates, const char *echo_type);
void epg_sr(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates);
void epg_se(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates);
void epg_tse(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates);
void epg_fisp(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams,
              int nstates);
void epg_ssfp(float2 *d_atoms, float *d_params, float *d_mrf, float TI, size_t nreps, size_t NATOMS, size_t natoms,
              int nparams, int nstates);
void roa_ssfp(float2 *d_atoms, float *d_mrf, float *d_params, size_t nreps, size_t natoms, int nparams);
#ifdef __CUDACC__
/* the reference's kernel (src/functions.h:87): callers launch it with
 * normalize<<<grid, block>>>(...) from code compiled without relocatable
 * device code and linked with the shared CUDA runtime (nvcc -cudart
 * shared), the runtime this library uses: the launch configuration the
 * caller's <<<...>>> sets is read by the library's kernel stub */
__global__ void normalize(float2 *d_atoms, size_t nreps, size_t NATOMS);
#endif
void MRF_minimatch(float *d_maps, float2 *d_img, float2 *d_atoms, float2 *d_mat, float *d_params, size_t nreps,
                   size_t NATOMS, size_t nminivoxels, int nparams, int nmaps);
void compute_nsplits(size_t *nsplits, size_t *nminivoxels, size_t nvoxels, size_t NATOMS, int type);
void MRF_match(float *d_maps, float2 *h_img, float2 *d_atoms, float *d_params, size_t NREPS, size_t nreps,
               size_t NATOMS, size_t natoms, size_t nvoxels, int nparams, int nmaps, const char *in_b1map);
void generate_echo(float *h_echo, size_t nreps, IP ip);
void compare(int *pass, int *fail, float2 *d_atoms, size_t nreps, size_t NATOMS, const char *echo_type);
void unittest_dictionary(int *pass, int *fail, float *h_echo, size_t nreps, size_t NREPS, int nparams,
                         int nstates, const char *T1, const char *T2, const char *B0, const char *B1,
                         const char *echo_type);
void unittest_matching(int *pass, int *fail, const char *atoms_path, const char *params_path, int nparams,
                       int nmaps, int ntests);

/* RA files with the reference's struct and C names (src/ra.h:20-74) */
typedef struct {
    uint64_t flags;
    uint64_t eltype;
    uint64_t elbyte;
    uint64_t size;
    uint64_t ndims;
    uint64_t *dims;
    uint8_t *data;
} ra_t;

extern "C" {
int ra_read(ra_t *a, const char *path);
void ra_query(const char *path);
int ra_write(ra_t *a, const char *path);
void ra_free(ra_t *a);
}

#endif /* SNAPMRF_COMPAT_H */
