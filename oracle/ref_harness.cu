/*
 * Reference harness: a small driver linked against the reference's own
 * src/functions.cu and src/ra.cu (compiled from the reference tree by
 * oracle/Makefile into oracle/_ref/).  TEST INFRASTRUCTURE ONLY: it produces
 * known answers from the reference implementation for the oracle and the
 * parity tests; the product never links it.
 *
 * Subcommands (all binary outputs are raw little-endian arrays):
 *   grid   T1 T2 B0 B1 out.f32        params via parse_length/parse_params/
 *                                     compute_natoms/trans_params; prints
 *                                     "l_t1 l_t2 l_b0 l_b1 NATOMS natoms"
 *   gridN  N out.f32                  the -N hard-coded logspace grids
 *                                     (src/mrf.cu:179-203)
 *   logspace min max len out.f32
 *   csv    path out.f32               csv_dim + csv_read; prints NREPS
 *   dict   echo params.f32 mrf.f32 nreps NREPS NATOMS natoms nstates out.c64
 *   match  img.c64 atoms.c64 params.f32 NREPS nreps NATOMS natoms nvox
 *          b1map.ra|- out.f32
 *   normalize in.c64 nreps natoms out.c64   the reference's normalize kernel
 *                                     (GPU subcommands need a device)
 * Run with stdin from /dev/null: the reference's gpuAssert waits on getchar().
 */
#include "functions.h"

extern int gridsize;
extern int blocksize;

static void *read_file(const char *path, size_t *n)
{
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    fseek(f, 0, SEEK_END);
    *n = (size_t)ftell(f);
    fseek(f, 0, SEEK_SET);
    void *p = malloc(*n ? *n : 1);
    if (fread(p, 1, *n, f) != *n) { fprintf(stderr, "short read %s\n", path); exit(2); }
    fclose(f);
    return p;
}

static void write_file(const char *path, const void *p, size_t n)
{
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(p, 1, n, f) != n) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
    fclose(f);
}

static float *grid_of(const char *s, size_t *len)
{
    *len = parse_length(s);
    float *p = (float *)malloc(*len * sizeof(float));
    parse_params(p, s, *len);
    return p;
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const char *cmd = argv[1];
    if (!strcmp(cmd, "grid") && argc == 7) {
        size_t l1, l2, l0, lb;
        float *t1 = grid_of(argv[2], &l1), *t2 = grid_of(argv[3], &l2);
        float *b0 = grid_of(argv[4], &l0), *b1 = grid_of(argv[5], &lb);
        size_t N = compute_natoms(t1, t2, l1, l2, l0, lb);
        float *p = (float *)malloc((N ? N : 1) * 4 * sizeof(float));
        if (N) trans_params(p, t1, t2, b0, b1, l1, l2, l0, lb, N, 4);
        printf("%zu %zu %zu %zu %zu %zu\n", l1, l2, l0, lb, N, lb ? N / lb : 0);
        write_file(argv[6], p, N * 4 * sizeof(float));
        return 0;
    }
    if (!strcmp(cmd, "gridN") && argc == 4) {
        size_t NATOMS = (size_t)atoi(argv[2]);
        size_t l_b1 = 11, l_b0 = 21;
        size_t l_t1 = roundf(sqrtf(NATOMS / l_b0 / l_b1));
        if (l_t1 == 0) l_t1 = 1;
        size_t l_t2 = l_t1;
        float *t1 = (float *)calloc(l_t1 + 2, sizeof(float)), *t2 = (float *)calloc(l_t2 + 2, sizeof(float));
        float *b0 = (float *)calloc(l_b0 + 2, sizeof(float)), *b1 = (float *)calloc(l_b1 + 2, sizeof(float));
        logspace(t1, 100.f, 3000.f, l_t1);
        logspace(t2, 20.f, 1000.f, l_t2);
        logspace(b0, -150.f, 150.f, l_b0);
        logspace(b1, 0.5, 1.5, l_b1);
        size_t N = compute_natoms(t1, t2, l_t1, l_t2, l_b0, l_b1);
        float *p = (float *)malloc((N ? N : 1) * 4 * sizeof(float));
        if (N) trans_params(p, t1, t2, b0, b1, l_t1, l_t2, l_b0, l_b1, N, 4);
        printf("%zu %zu %zu %zu %zu %zu\n", l_t1, l_t2, l_b0, l_b1, N, N / l_b1);
        write_file(argv[3], p, N * 4 * sizeof(float));
        return 0;
    }
    if (!strcmp(cmd, "logspace") && argc == 6) {
        size_t len = (size_t)atoi(argv[4]);
        float *p = (float *)calloc(len + 2, sizeof(float)); /* the reference writes past len */
        logspace(p, (float)atof(argv[2]), (float)atof(argv[3]), len);
        write_file(argv[5], p, len * sizeof(float));
        return 0;
    }
    if (!strcmp(cmd, "csv") && argc == 4) {
        size_t NREPS = csv_dim(argv[2]) - 1;
        float *m = (float *)calloc(NREPS * 4 + 1, sizeof(float));
        csv_read(m, NREPS, argv[2]);
        printf("%zu\n", NREPS);
        write_file(argv[3], m, NREPS * 4 * sizeof(float));
        return 0;
    }
    if (!strcmp(cmd, "dict") && argc == 11) {
        size_t np_, nm;
        float *h_params = (float *)read_file(argv[3], &np_);
        float *h_mrf = (float *)read_file(argv[4], &nm);
        size_t nreps = strtoull(argv[5], 0, 10), NREPS = strtoull(argv[6], 0, 10);
        size_t NATOMS = strtoull(argv[7], 0, 10), natoms = strtoull(argv[8], 0, 10);
        int nstates = atoi(argv[9]);
        float *d_params;
        float2 *d_atoms;
        cuTry(cudaMalloc((void **)&d_params, np_));
        cuTry(cudaMemcpy(d_params, h_params, np_, cudaMemcpyHostToDevice));
        cuTry(cudaMalloc((void **)&d_atoms, nreps * NATOMS * sizeof(float2)));
        cuTry(cudaMemset(d_atoms, 0, nreps * NATOMS * sizeof(float2)));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        MRF_dict(d_atoms, d_params, h_mrf, nreps, NREPS, NATOMS, natoms, 4, nstates, argv[2]);
        cudaEventRecord(e1);
        cuTry(cudaDeviceSynchronize());
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        float2 *h = (float2 *)malloc(nreps * NATOMS * sizeof(float2));
        cuTry(cudaMemcpy(h, d_atoms, nreps * NATOMS * sizeof(float2), cudaMemcpyDeviceToHost));
        write_file(argv[10], h, nreps * NATOMS * sizeof(float2));
        fprintf(stderr, "REF_DICT_MS %.3f\n", ms);
        return 0;
    }
    if (!strcmp(cmd, "match") && argc == 12) {
        size_t ni, na, np_;
        float2 *h_img = (float2 *)read_file(argv[2], &ni);
        float2 *h_atoms = (float2 *)read_file(argv[3], &na);
        float *h_params = (float *)read_file(argv[4], &np_);
        size_t NREPS = strtoull(argv[5], 0, 10), nreps = strtoull(argv[6], 0, 10);
        size_t NATOMS = strtoull(argv[7], 0, 10), natoms = strtoull(argv[8], 0, 10);
        size_t nvox = strtoull(argv[9], 0, 10);
        const char *b1path = strcmp(argv[10], "-") ? argv[10] : NULL;
        float *d_params, *d_maps;
        float2 *d_atoms;
        cuTry(cudaMalloc((void **)&d_params, np_));
        cuTry(cudaMemcpy(d_params, h_params, np_, cudaMemcpyHostToDevice));
        cuTry(cudaMalloc((void **)&d_atoms, na));
        cuTry(cudaMemcpy(d_atoms, h_atoms, na, cudaMemcpyHostToDevice));
        cuTry(cudaMalloc((void **)&d_maps, 5 * nvox * sizeof(float)));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        MRF_match(d_maps, h_img, d_atoms, d_params, NREPS, nreps, NATOMS, natoms, nvox, 4, 5,
                  b1path);
        cudaEventRecord(e1);
        cuTry(cudaDeviceSynchronize());
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        float *h = (float *)malloc(5 * nvox * sizeof(float));
        cuTry(cudaMemcpy(h, d_maps, 5 * nvox * sizeof(float), cudaMemcpyDeviceToHost));
        write_file(argv[11], h, 5 * nvox * sizeof(float));
        fprintf(stderr, "REF_MATCH_MS %.3f\n", ms);
        (void)ni;
        return 0;
    }
    if (!strcmp(cmd, "normalize") && argc == 6) {
        size_t n;
        float2 *h = (float2 *)read_file(argv[2], &n);
        size_t nreps = strtoull(argv[3], 0, 10), natoms = strtoull(argv[4], 0, 10);
        float2 *d;
        cuTry(cudaMalloc((void **)&d, n));
        cuTry(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice));
        normalize<<<gridsize, blocksize>>>(d, nreps, natoms);
        cuTry(cudaDeviceSynchronize());
        cuTry(cudaMemcpy(h, d, n, cudaMemcpyDeviceToHost));
        write_file(argv[5], h, n);
        return 0;
    }
    fprintf(stderr, "bad arguments\n");
    return 2;
}
