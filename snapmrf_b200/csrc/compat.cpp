// libsnapmrf_compat.so: the reference's host-function surface
// (src/functions.h, src/ra.h) on top of the C ABI, so that drivers written
// for the reference (its src/mrf.cu and src/test.cu included) link against
// this library unchanged.  Each function cites the reference function whose
// behaviour it keeps; every computation goes through libsnapmrf.so.
//
// Environment: SNAPMRF_PRECISION = fp32 (default) | bf16 | fp16 | fp8 selects the
// matching form used by MRF_match.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <err.h>
#include <sysexits.h>

#include <cuda_runtime.h>

#include "snapmrf.h"
#include "snapmrf_compat.h"

int blocksize = 64;
int gridsize = 128;
cudaStream_t stream[2];

static int env_precision();

static void die(int status, const char *what) {
    fprintf(stderr, "%s: %s\n", what, snapmrf_last_error());
    exit(status == SNAPMRF_ERR_ECHO_TYPE ? EX_USAGE : EXIT_FAILURE);
}

// gpuAssert (src/functions.cu:38-48) without the wait on stdin.
void gpuAssert(cudaError_t code, const char *file, int line) {
    if (code != cudaSuccess) {
        fprintf(stderr, "GPUassert: %s %s %d\n", cudaGetErrorString(code), file, line);
        exit(code);
    }
}

void *mallocAssert(size_t n, const char *file, int line) {
    void *p = malloc(n);
    if (p == NULL) {
        printf("Malloc failed from %s:%d", file, line);
        abort();
    }
    return p;
}

// freeAssert (src/functions.cu:66-74) checks for NULL and then frees (the
// reference only checks).
void freeAssert(void *p, const char *file, int line) {
    if (p == NULL) {
        printf("Free failed from %s:%d", file, line);
        abort();
    }
    free(p);
}

void print_usage() {
    fprintf(stderr, "MR fingerprinting dictionary generator and image reconstructor\n");
    fprintf(stderr, "Usage: mrf [OPTION] <rfpulse.csv> <imgstack.ra>\n");
    fprintf(stderr, "\t-M, --b1map <rafile>\t\t B1 map input RA file\n");
    fprintf(stderr, "\t-N <n>\t\t\t\t number of atoms (hard-coded logspace grids)\n");
    fprintf(stderr, "\t-a, --atoms <rafile>\t\t dictionary atoms output RA file\n");
    fprintf(stderr, "\t-m, --map, --maps <rafile>\t parameter map output RA file\n");
    fprintf(stderr, "\t-p, --params <rafile>\t\t dictionary parameters output RA file\n");
    fprintf(stderr, "\t-t, --T1 start:step:end\t\t T1 grid\n");
    fprintf(stderr, "\t-s, --T2 start:step:end\t\t T2 grid\n");
    fprintf(stderr, "\t-b, --B0 start:step:end\t\t B0 grid\n");
    fprintf(stderr, "\t-r, --B1 start:step:end\t\t B1 grid\n");
    fprintf(stderr, "\t-w, --nstates, --states n\t number of EPG states\n");
    fprintf(stderr, "\t-e, --echo_type name\t\t echo type\n");
    fprintf(stderr, "\t-T, --nreps, --timepoints n\t number of time points\n");
    fprintf(stderr, "\t-G, --gridsize n\t\t accepted for compatibility\n");
    fprintf(stderr, "\t-B, --blocksize n\t\t accepted for compatibility\n");
    fprintf(stderr, "\t-h, --help\t\t\t show this help\n");
}

// csv_dim / csv_read (src/functions.cu:100-158): the reference exits when
// the file cannot be opened.
size_t csv_dim(const char *filepath) {
    size_t n = snapmrf_csv_dim(filepath);
    if (n == (size_t)-1) {
        printf("Unable to open file %s\n", filepath);
        exit(1);
    }
    return n;
}

void csv_read(float *h_mrf, size_t nreps, const char *filepath) {
    int rc = snapmrf_csv_read(h_mrf, nreps, filepath);
    if (rc == SNAPMRF_ERR_IO) {
        printf("Unable to open file %s\n", filepath);
        exit(1);
    }
    if (rc) die(rc, "csv_read");
}

static void write_ra(void *data, uint64_t eltype, uint64_t elbyte, const char *path, size_t dim0, size_t dim1) {
    uint64_t dims[2] = {dim0, dim1};
    snapmrf_ra a;
    a.flags = 0;
    a.eltype = eltype;
    a.elbyte = elbyte;
    a.size = dim0 * dim1 * elbyte;
    a.ndims = 2;
    a.dims = dims;
    a.data = (uint8_t *)data;
    int rc = snapmrf_ra_write(&a, path);
    if (rc) err(errno ? errno : 1, "unable to open %s for writing", path);
}

// save_rafile (src/functions.cu:160-194): complex atoms / float params.
void save_rafile(float2 *h_atoms, const char *atoms_path, size_t dim0, size_t dim1) {
    write_ra(h_atoms, 4, sizeof(float2), atoms_path, dim0, dim1);
}

void save_rafile(float *h_params, const char *p_path, size_t dim0, size_t dim1) {
    write_ra(h_params, 3, sizeof(float), p_path, dim0, dim1);
}

// parse_range / parse_length / parse_params (src/functions.cu:197-353):
// the reference asserts on a bad grid.
void parse_range(const char *str, float *min, float *step, float *max, size_t *len) {
    int rc = snapmrf_parse_range(str, min, step, max, len);
    if (rc) die(rc, "parse_range");
}

size_t parse_length(const char *str) {
    size_t n = snapmrf_parse_length(str);
    if (n == 0) die(SNAPMRF_ERR_FORMAT, "parse_length");
    return n;
}

void linspace(float *h_p, float min, float step, size_t len) { snapmrf_linspace(h_p, min, step, len); }

void parse_params(float *h_p, const char *str, size_t LEN) {
    int rc = snapmrf_parse_params(h_p, str, LEN);
    if (rc) die(rc, "parse_params");
}

void logspace(float *h_p, float min, float max, size_t len) { snapmrf_logspace(h_p, min, max, len); }

void trans_params(float *h_params, float *h_t1, float *h_t2, float *h_b0, float *h_b1, size_t l_t1, size_t l_t2,
                  size_t l_b0, size_t l_b1, size_t NATOMS, int nparams) {
    int rc = snapmrf_trans_params(h_params, h_t1, h_t2, h_b0, h_b1, l_t1, l_t2, l_b0, l_b1, NATOMS, nparams);
    if (rc) die(rc, "trans_params");
}

size_t compute_natoms(float *h_t1, float *h_t2, size_t l_t1, size_t l_t2, size_t l_b0, size_t l_b1) {
    return snapmrf_compute_natoms(h_t1, h_t2, l_t1, l_t2, l_b0, l_b1);
}

// MRF_dict (src/functions.cu:1224-1315); returns after the device work.
// The reference's two relaxations per step are kept (bit-identical FISP / SR
// atoms, as its drivers' golden checks expect).
void MRF_dict(float2 *d_atoms, float *d_params, float *h_mrf, size_t nreps, size_t NREPS, size_t NATOMS,
              size_t natoms, int nparams, int nstates, const char *echo_type) {
    printf("Constructing dictionary...\n");
    snapmrf_dict_opts o;
    memset(&o, 0, sizeof o);
    o.flags = SNAPMRF_DICT_SEPARATE_RELAX;
    int rc = snapmrf_mrf_dict(reinterpret_cast<float *>(d_atoms), d_params, h_mrf, nreps, NREPS, NATOMS, natoms,
                              nparams, nstates, echo_type, &o, stream[0]);
    if (rc == SNAPMRF_ERR_ECHO_TYPE) errx(EX_USAGE, "Please put in correct echo types.");
    if (rc) die(rc, "MRF_dict");
    gpuAssert(cudaStreamSynchronize(stream[0]), __FILE__, __LINE__);
}

// The echo-type engines (src/functions.h:89-113): the schedule d_mrf is
// already converted and on the device; the atoms are left as the recursion
// produces them (MRF_dict normalises epg_ssfp / roa_ssfp afterwards).  They
// return after the device work, as the reference's do.  The non-SSFP
// engines fill natoms atoms of block 0; epg_ssfp fills every block.
static void engine(const char *echo, float2 *d_atoms, float *d_params, float *d_mrf, float ti, size_t nreps,
                   size_t NATOMS, size_t natoms, int nparams, int nstates) {
    snapmrf_dict_opts o;
    memset(&o, 0, sizeof o);
    o.flags = SNAPMRF_DICT_SEPARATE_RELAX;
    o.n_iso = 1;
    int rc = snapmrf_dict_engine(reinterpret_cast<float *>(d_atoms), d_params, d_mrf, ti, nreps, NATOMS, natoms,
                                 nparams, nstates, echo, &o, stream[0]);
    if (rc) die(rc, echo);
    gpuAssert(cudaStreamSynchronize(stream[0]), __FILE__, __LINE__);
}

// epg_sr (src/functions.cu:687-739)
void epg_sr(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates) {
    engine("epg_sr", d_atoms, d_params, d_mrf, 0.f, nreps, natoms, natoms, nparams, nstates);
}

// epg_se (src/functions.cu:741-807)
void epg_se(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates) {
    engine("epg_se", d_atoms, d_params, d_mrf, 0.f, nreps, natoms, natoms, nparams, nstates);
}

// epg_tse (src/functions.cu:809-876)
void epg_tse(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams, int nstates) {
    engine("epg_tse1", d_atoms, d_params, d_mrf, 0.f, nreps, natoms, natoms, nparams, nstates);
}

// epg_fisp (src/functions.cu:878-933)
void epg_fisp(float2 *d_atoms, float *d_params, float *d_mrf, size_t nreps, size_t natoms, int nparams,
              int nstates) {
    engine("epg_fisp", d_atoms, d_params, d_mrf, 0.f, nreps, natoms, natoms, nparams, nstates);
}

// epg_ssfp (src/functions.cu:935-1019): every B1 block, inversion with delay TI
void epg_ssfp(float2 *d_atoms, float *d_params, float *d_mrf, float TI, size_t nreps, size_t NATOMS, size_t natoms,
              int nparams, int nstates) {
    engine("epg_ssfp", d_atoms, d_params, d_mrf, TI, nreps, NATOMS, natoms, nparams, nstates);
}

// roa_ssfp (src/functions.cu:1155-1222): one isochromat, block 0
void roa_ssfp(float2 *d_atoms, float *d_mrf, float *d_params, size_t nreps, size_t natoms, int nparams) {
    engine("roa_ssfp", d_atoms, d_params, d_mrf, 0.f, nreps, natoms, natoms, nparams, 1);
}

// normalize (src/functions.cu:670-685), the reference's kernel, launched by
// the caller with any grid and block: atoms are walked grid-stride, one
// thread per atom, the squared moduli summed in time order.
__global__ void normalize(float2 *d_atoms, size_t nreps, size_t NATOMS) {
    for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < NATOMS;
         id += (size_t)blockDim.x * gridDim.x) {
        float2 *a = d_atoms + id * nreps;
        float sum = 0.f;
        for (size_t i = 0; i < nreps; i++) {
            const float n2 = a[i].x * a[i].x + a[i].y * a[i].y;
            sum += n2;
        }
        if (sum > 0.f) sum = 1.f / sqrtf(sum);
        for (size_t i = 0; i < nreps; i++) a[i] = make_float2(a[i].x * sum, a[i].y * sum);
    }
}

// MRF_minimatch (src/functions.cu:1464-1491): the first argmax of |<atom,
// voxel>| over all NATOMS atoms for nminivoxels device voxels, maps written
// as generate_maps does.  The matching never forms the score matrix, so
// d_mat (the reference's cuBLAS output) is not written.
void MRF_minimatch(float *d_maps, float2 *d_img, float2 *d_atoms, float2 *d_mat, float *d_params, size_t nreps,
                   size_t NATOMS, size_t nminivoxels, int nparams, int nmaps) {
    (void)d_mat;
    snapmrf_match_opts o;
    memset(&o, 0, sizeof o);
    o.precision = env_precision();
    int rc = snapmrf_mrf_match(d_maps, reinterpret_cast<const float *>(d_img), 0,
                               reinterpret_cast<const float *>(d_atoms), d_params, nreps, NATOMS, NATOMS,
                               nminivoxels, nparams, nmaps, &o, stream[0]);
    if (rc) die(rc, "MRF_minimatch");
    gpuAssert(cudaStreamSynchronize(stream[0]), __FILE__, __LINE__);
}

// compute_nsplits (src/functions.cu:1418-1462): voxel splits that fit the
// free device memory.  Matching here needs no split; kept for callers.
// When no even split fits, one voxel per split is returned (the reference
// leaves the outputs unset).
void compute_nsplits(size_t *nsplits, size_t *nminivoxels, size_t nvoxels, size_t NATOMS, int type) {
    size_t free_mem = 0, total = 0;
    cudaMemGetInfo(&free_mem, &total);
    printf("Available GPU memory = %lu MB\n", (unsigned long)(free_mem / 1024 / 1024));
    size_t max_float2 = (size_t)(free_mem / sizeof(float2) / 1.01);
    if (type == 1) {
        *nminivoxels = NATOMS ? (max_float2 / NATOMS < nvoxels ? max_float2 / NATOMS : nvoxels) : nvoxels;
        if (*nminivoxels == 0) *nminivoxels = 1;
        *nsplits = nvoxels / *nminivoxels;
    } else if (type == 0) {
        if (NATOMS * nvoxels > max_float2) {
            *nsplits = nvoxels;
            *nminivoxels = 1;
            for (size_t i = 2; i < nvoxels / 2 + 1; i++)
                if (nvoxels % i == 0 && NATOMS * (nvoxels / i) < max_float2) {
                    *nsplits = i;
                    *nminivoxels = nvoxels / i;
                    break;
                }
        } else {
            *nminivoxels = nvoxels;
            *nsplits = 1;
        }
    } else {
        printf("Please put in 0 or 1\n");
    }
}

static int env_precision() {
    const char *p = getenv("SNAPMRF_PRECISION");
    if (!p || !strcmp(p, "fp32")) return SNAPMRF_PREC_FP32;
    if (!strcmp(p, "bf16")) return SNAPMRF_PREC_BF16;
    if (!strcmp(p, "fp16")) return SNAPMRF_PREC_FP16;
    if (!strcmp(p, "fp8")) return SNAPMRF_PREC_FP8;
    fprintf(stderr, "SNAPMRF_PRECISION must be fp32, bf16, fp16 or fp8\n");
    exit(EX_USAGE);
}

// MRF_match (src/functions.cu:1493-1584).  NREPS is the dictionary's time
// points per atom (the reference's caller passes them first) and nreps the
// image's; the first min(NREPS, nreps) are matched with each array's own
// stride.  The B1 map is read from an RA file as in the reference.
void MRF_match(float *d_maps, float2 *h_img, float2 *d_atoms, float *d_params, size_t NREPS, size_t nreps,
               size_t NATOMS, size_t natoms, size_t nvoxels, int nparams, int nmaps, const char *in_b1map) {
    snapmrf_match_opts o;
    memset(&o, 0, sizeof o);
    o.precision = env_precision();
    o.img_stride = nreps;
    o.atom_stride = NREPS;
    snapmrf_ra b1;
    memset(&b1, 0, sizeof b1);
    printf("Matching...\n");
    if (in_b1map) {
        printf("Input B1 map: %s\n", in_b1map);
        int rc = snapmrf_ra_read(&b1, in_b1map, 1);
        if (rc) err(errno ? errno : 1, "unable to open %s for reading", in_b1map);
        if (b1.eltype != 3 || b1.elbyte != 4 || b1.size < nvoxels * sizeof(float))
            errx(EX_DATAERR, "%s: B1 map must hold %zu float values", in_b1map, nvoxels);
        o.b1map = reinterpret_cast<const float *>(b1.data);
        o.b1map_on_host = 1;
    }
    size_t k = NREPS < nreps ? NREPS : nreps;
    int rc = snapmrf_mrf_match(d_maps, reinterpret_cast<const float *>(h_img), 1,
                               reinterpret_cast<const float *>(d_atoms), d_params, k, NATOMS, natoms, nvoxels,
                               nparams, nmaps, &o, stream[0]);
    if (rc) die(rc, "MRF_match");
    gpuAssert(cudaStreamSynchronize(stream[0]), __FILE__, __LINE__);
    if (in_b1map) snapmrf_ra_free(&b1);
}

// generate_echo (src/functions.cu:1588-1598)
void generate_echo(float *h_echo, size_t nreps, IP ip) {
    for (size_t i = 0; i < nreps; i++) {
        h_echo[0 * nreps + i] = ip.alpha;
        h_echo[1 * nreps + i] = ip.phi;
        h_echo[2 * nreps + i] = ip.TR;
        h_echo[3 * nreps + i] = ip.TE;
    }
}

// compare (src/functions.cu:1600-1649): sum of |atom - golden| over the
// dictionary against ../data/atoms_<echo>.ra, pass below 1e-6.
void compare(int *pass, int *fail, float2 *d_atoms, size_t nreps, size_t NATOMS, const char *echo_type) {
    char path[1024];
    snprintf(path, sizeof path, "../data/atoms_%s.ra", echo_type);
    ra_t gt;
    ra_read(&gt, path);
    const float2 *g = reinterpret_cast<const float2 *>(gt.data);
    float2 *h = static_cast<float2 *>(mallocAssert(nreps * NATOMS * sizeof(float2), __FILE__, __LINE__));
    gpuAssert(cudaMemcpy(h, d_atoms, nreps * NATOMS * sizeof(float2), cudaMemcpyDeviceToHost), __FILE__,
              __LINE__);
    float diff = 0.f;
    for (size_t i = 0; i < NATOMS; i++) {
        printf("The %zu th atom\n", i + 1);
        for (size_t j = 0; j < nreps; j++) {
            const float2 a = h[i * nreps + j], b = g[i * nreps + j];
            printf("atoms_%s[%zu] = %f + %fim, atoms_gt[%zu] = %f + %fim\n", echo_type, j, a.x, a.y, j, b.x, b.y);
            diff += hypotf(a.x - b.x, a.y - b.y);
        }
    }
    if (diff < 1E-6) {
        printf("%s unit test passed!\n\n", echo_type);
        (*pass)++;
    } else {
        printf("%s unit test failed!\n\n", echo_type);
        (*fail)++;
    }
    ra_free(&gt);
    free(h);
}

// unittest_dictionary (src/functions.cu:1651-1718)
void unittest_dictionary(int *pass, int *fail, float *h_echo, size_t nreps, size_t NREPS, int nparams, int nstates,
                         const char *T1, const char *T2, const char *B0, const char *B1, const char *echo_type) {
    const char *grids[4] = {T1, T2, B0, B1};
    size_t len[4];
    float *vals[4];
    for (int i = 0; i < 4; i++) {
        len[i] = parse_length(grids[i]);
        vals[i] = static_cast<float *>(mallocAssert(len[i] * sizeof(float), __FILE__, __LINE__));
        parse_params(vals[i], grids[i], len[i]);
    }
    size_t NATOMS = compute_natoms(vals[0], vals[1], len[0], len[1], len[2], len[3]);
    size_t natoms = NATOMS / len[3];
    float *h_params = static_cast<float *>(mallocAssert(NATOMS * nparams * sizeof(float), __FILE__, __LINE__));
    trans_params(h_params, vals[0], vals[1], vals[2], vals[3], len[0], len[1], len[2], len[3], NATOMS, nparams);
    float *d_params;
    float2 *d_atoms;
    gpuAssert(cudaMalloc((void **)&d_params, nparams * NATOMS * sizeof(float)), __FILE__, __LINE__);
    gpuAssert(cudaMemcpy(d_params, h_params, nparams * NATOMS * sizeof(float), cudaMemcpyHostToDevice), __FILE__,
              __LINE__);
    gpuAssert(cudaMalloc((void **)&d_atoms, nreps * NATOMS * sizeof(float2)), __FILE__, __LINE__);
    printf("Begin unit test for %s\n", echo_type);
    printf("T1 = %s\nT2 = %s\nB0 = %s\nB1 = %s\n", T1, T2, B0, B1);
    printf("l_t1: %zu, l_t2: %zu, l_b0: %zu, l_b1: %zu\n", len[0], len[1], len[2], len[3]);
    printf("nreps: %zu, NATOMS: %zu, natoms: %zu\n", nreps, NATOMS, natoms);
    MRF_dict(d_atoms, d_params, h_echo, nreps, NREPS, NATOMS, natoms, nparams, nstates, echo_type);
    compare(pass, fail, d_atoms, nreps, NATOMS, echo_type);
    cudaFree(d_atoms);
    cudaFree(d_params);
    for (int i = 0; i < 4; i++) free(vals[i]);
    free(h_params);
}

// unittest_matching (src/functions.cu:1720-1824): ntests atoms chosen with
// rand() % NATOMS are matched back against the dictionary.
void unittest_matching(int *pass, int *fail, const char *atoms_path, const char *params_path, int nparams, int nmaps,
                       int ntests) {
    ra_t ra_atoms, ra_params;
    printf("Reading %s\n", atoms_path);
    ra_read(&ra_atoms, atoms_path);
    printf("Reading %s\n", params_path);
    ra_read(&ra_params, params_path);
    const float2 *h_atoms = reinterpret_cast<const float2 *>(ra_atoms.data);
    const float *h_params = reinterpret_cast<const float *>(ra_params.data);
    size_t NREPS = ra_atoms.dims[0], NATOMS = ra_atoms.dims[1];
    printf("NREPS: %zu, NATOMS: %zu\n", NREPS, NATOMS);
    float2 *d_atoms;
    float *d_params, *d_maps;
    gpuAssert(cudaMalloc((void **)&d_atoms, NREPS * NATOMS * sizeof(float2)), __FILE__, __LINE__);
    gpuAssert(cudaMemcpy(d_atoms, h_atoms, NREPS * NATOMS * sizeof(float2), cudaMemcpyHostToDevice), __FILE__,
              __LINE__);
    gpuAssert(cudaMalloc((void **)&d_params, nparams * NATOMS * sizeof(float)), __FILE__, __LINE__);
    gpuAssert(cudaMemcpy(d_params, h_params, nparams * NATOMS * sizeof(float), cudaMemcpyHostToDevice), __FILE__,
              __LINE__);
    float2 *h_img = static_cast<float2 *>(mallocAssert(NREPS * ntests * sizeof(float2), __FILE__, __LINE__));
    int *index = static_cast<int *>(mallocAssert(ntests * sizeof(int), __FILE__, __LINE__));
    for (int i = 0; i < ntests; i++) {
        index[i] = rand() % (int)NATOMS;
        memcpy(h_img + (size_t)i * NREPS, h_atoms + (size_t)index[i] * NREPS, NREPS * sizeof(float2));
    }
    gpuAssert(cudaMalloc((void **)&d_maps, nmaps * ntests * sizeof(float)), __FILE__, __LINE__);
    MRF_match(d_maps, h_img, d_atoms, d_params, NREPS, NREPS, NATOMS, NATOMS, ntests, nparams, nmaps, NULL);
    float *h_maps = static_cast<float *>(mallocAssert(nmaps * ntests * sizeof(float), __FILE__, __LINE__));
    gpuAssert(cudaMemcpy(h_maps, d_maps, nmaps * ntests * sizeof(float), cudaMemcpyDeviceToHost), __FILE__,
              __LINE__);
    float diff = 0.f;
    for (int i = 0; i < ntests; i++) {
        printf("The %dth voxel\n", i + 1);
        const char *names[4] = {"T1", "T2", "B0", "B1"};
        for (int m = 0; m < 4; m++) {
            float got = h_maps[i * nmaps + m], gt = h_params[index[i] * nparams + m];
            printf("%s_test[%d] = %.2f, %s_gt[%d] = %.2f\n", names[m], i, got, names[m], i, gt);
            diff += fabsf(got - gt);
        }
    }
    if (diff < 1E-6) {
        printf("Matching unit test passed!\n\n");
        (*pass)++;
    } else {
        printf("Matching unit test failed!\n\n");
        (*fail)++;
    }
    ra_free(&ra_atoms);
    ra_free(&ra_params);
    free(h_maps);
    free(h_img);
    free(index);
    cudaFree(d_atoms);
    cudaFree(d_params);
    cudaFree(d_maps);
}

// RA files (src/ra.cu:23-104): data in page-locked memory, as the reference
// builds with -DCUDA_HOST_MALLOC; exits when the file cannot be read.
extern "C" int ra_read(ra_t *a, const char *path) {
    snapmrf_ra r;
    int rc = snapmrf_ra_read(&r, path, 1);
    if (rc) err(errno ? errno : 1, "unable to open %s for reading (%s)", path, snapmrf_last_error());
    a->flags = r.flags & ~(1ull << 63);
    a->eltype = r.eltype;
    a->elbyte = r.elbyte;
    a->size = r.size;
    a->ndims = r.ndims;
    a->dims = r.dims;
    a->data = r.data;
    return 0;
}

extern "C" void ra_query(const char *path) {
    snapmrf_ra r;
    if (snapmrf_ra_read(&r, path, 0)) {
        fprintf(stderr, "%s\n", snapmrf_last_error());
        return;
    }
    static const char *names[] = {"user", "int", "uint", "float", "complex"};
    printf("---\nname: %s\nendian: %s\ntype: %s%llu\nsize: %llu\ndimension: %llu\nshape:\n", path,
           (r.flags & 1) ? "big" : "little", r.eltype < 5 ? names[r.eltype] : "?",
           (unsigned long long)(r.elbyte * 8), (unsigned long long)r.size, (unsigned long long)r.ndims);
    for (uint64_t i = 0; i < r.ndims; i++) printf("  - %llu\n", (unsigned long long)r.dims[i]);
    printf("...\n");
    snapmrf_ra_free(&r);
}

extern "C" int ra_write(ra_t *a, const char *path) {
    snapmrf_ra r;
    r.flags = a->flags;
    r.eltype = a->eltype;
    r.elbyte = a->elbyte;
    r.size = a->size;
    r.ndims = a->ndims;
    r.dims = a->dims;
    r.data = a->data;
    int rc = snapmrf_ra_write(&r, path);
    if (rc) err(errno ? errno : 1, "unable to open %s for writing", path);
    return 0;
}

extern "C" void ra_free(ra_t *a) {
    cudaFreeHost(a->data);
    free(a->dims);
}
