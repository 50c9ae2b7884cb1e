/*
 * Engine-level driver: calls the reference's echo-type engines, its
 * normalize kernel and MRF_minimatch directly (src/functions.h:87-134), the
 * way a caller that bypasses MRF_dict / MRF_match would.  TEST
 * INFRASTRUCTURE ONLY: oracle/Makefile links it twice, against the
 * reference's own functions.o (_ref/engine_ref) and against
 * libsnapmrf_compat.so (_ref/engine_on_snapmrf); the GPU tests compare the
 * two outputs.
 *
 * Usage: engine_driver <out_prefix>; writes <prefix>_<engine>.c64 (atoms,
 * [NATOMS][T] complex), <prefix>_norm.c64 (the FISP atoms after normalize)
 * and <prefix>_maps.f32 (MRF_minimatch maps, [nvox][5]).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "functions.h"

extern int gridsize;
extern int blocksize;

static void save(const char *prefix, const char *name, const void *d, size_t bytes) {
    char path[512];
    snprintf(path, sizeof path, "%s_%s", prefix, name);
    void *h = malloc(bytes);
    cuTry(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost));
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(h, 1, bytes, f) != bytes) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
    fclose(f);
    free(h);
}

int main(int argc, char **argv) {
    if (argc != 2) return 2;
    const char *prefix = argv[1];
    const size_t T = 60;
    const int nstates = 24, nparams = 4;
    // grid: T1 x T2 (T1 > T2) x B0 x B1, the reference's own parameter table
    const char *s1 = "200:300:2000", *s2 = "20:40:300", *s0 = "-20:25:30", *sb = "0.9:0.2:1.1";
    size_t l1 = parse_length(s1), l2 = parse_length(s2), l0 = parse_length(s0), lb = parse_length(sb);
    float *t1 = (float *)malloc(l1 * 4), *t2 = (float *)malloc(l2 * 4), *b0 = (float *)malloc(l0 * 4),
          *b1 = (float *)malloc(lb * 4);
    parse_params(t1, s1, l1);
    parse_params(t2, s2, l2);
    parse_params(b0, s0, l0);
    parse_params(b1, sb, lb);
    const size_t NATOMS = compute_natoms(t1, t2, l1, l2, l0, lb), natoms = NATOMS / lb;
    float *h_params = (float *)malloc(NATOMS * nparams * 4);
    trans_params(h_params, t1, t2, b0, b1, l1, l2, l0, lb, NATOMS, nparams);
    // raw schedule (radians, ms) for the EPG engines; converted bSSFP form
    // (flip in radians, RF phase alternating 0 / pi) for epg_ssfp / roa_ssfp
    float *h_raw = (float *)malloc(4 * T * 4), *h_ssfp = (float *)malloc(4 * T * 4);
    for (size_t t = 0; t < T; t++) {
        h_raw[t] = 0.2f + 0.5f * fabsf(sinf(3.14159265f * t / 25.f));
        h_raw[T + t] = 0.f;
        h_raw[2 * T + t] = 12.f + (t % 3);
        h_raw[3 * T + t] = 6.f;
        h_ssfp[t] = 0.1f + 0.9f * fabsf(sinf(3.14159265f * t / 20.f));
        h_ssfp[T + t] = (t % 2) ? 3.14159265f : 0.f;
        h_ssfp[2 * T + t] = 14.f + (t % 2);
        h_ssfp[3 * T + t] = 7.f;
    }
    float *d_params, *d_raw, *d_ssfp;
    float2 *d_atoms;
    cuTry(cudaMalloc((void **)&d_params, NATOMS * nparams * 4));
    cuTry(cudaMemcpy(d_params, h_params, NATOMS * nparams * 4, cudaMemcpyHostToDevice));
    cuTry(cudaMalloc((void **)&d_raw, 4 * T * 4));
    cuTry(cudaMemcpy(d_raw, h_raw, 4 * T * 4, cudaMemcpyHostToDevice));
    cuTry(cudaMalloc((void **)&d_ssfp, 4 * T * 4));
    cuTry(cudaMemcpy(d_ssfp, h_ssfp, 4 * T * 4, cudaMemcpyHostToDevice));
    cuTry(cudaMalloc((void **)&d_atoms, NATOMS * T * sizeof(float2)));
    const size_t blk0 = natoms * T * sizeof(float2);

    cuTry(cudaMemset(d_atoms, 0, NATOMS * T * sizeof(float2)));
    epg_sr(d_atoms, d_params, d_raw, T, natoms, nparams, nstates);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "sr.c64", d_atoms, blk0);
    epg_se(d_atoms, d_params, d_raw, T, natoms, nparams, nstates);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "se.c64", d_atoms, blk0);
    epg_tse(d_atoms, d_params, d_raw, T, natoms, nparams, nstates);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "tse.c64", d_atoms, blk0);
    epg_ssfp(d_atoms, d_params, d_ssfp, 40.f, T, NATOMS, natoms, nparams, nstates);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "ssfp.c64", d_atoms, NATOMS * T * sizeof(float2));
    roa_ssfp(d_atoms, d_ssfp, d_params, T, natoms, nparams);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "roa.c64", d_atoms, blk0);
    epg_fisp(d_atoms, d_params, d_raw, T, natoms, nparams, nstates);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "fisp.c64", d_atoms, blk0);
    normalize<<<gridsize, blocksize>>>(d_atoms, T, natoms);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "norm.c64", d_atoms, blk0);

    // minimatch: voxels = normalised atoms 3, 17, 40 and a scaled mix
    const size_t nvox = 4;
    float2 *h_norm = (float2 *)malloc(blk0);
    cuTry(cudaMemcpy(h_norm, d_atoms, blk0, cudaMemcpyDeviceToHost));
    float2 *h_img = (float2 *)malloc(nvox * T * sizeof(float2));
    const size_t pick[3] = {3, 17, 40 % natoms};
    for (size_t v = 0; v < 3; v++)
        for (size_t t = 0; t < T; t++) h_img[v * T + t] = h_norm[pick[v] * T + t];
    for (size_t t = 0; t < T; t++)
        h_img[3 * T + t] = make_float2(0.7f * h_norm[5 * T + t].x - 0.2f * h_norm[5 * T + t].y,
                                       0.7f * h_norm[5 * T + t].y + 0.2f * h_norm[5 * T + t].x);
    float2 *d_img, *d_mat;
    float *d_maps;
    cuTry(cudaMalloc((void **)&d_img, nvox * T * sizeof(float2)));
    cuTry(cudaMemcpy(d_img, h_img, nvox * T * sizeof(float2), cudaMemcpyHostToDevice));
    cuTry(cudaMalloc((void **)&d_mat, nvox * natoms * sizeof(float2)));
    cuTry(cudaMalloc((void **)&d_maps, nvox * 5 * 4));
    MRF_minimatch(d_maps, d_img, d_atoms, d_mat, d_params, T, natoms, nvox, nparams, 5);
    cuTry(cudaDeviceSynchronize());
    save(prefix, "maps.f32", d_maps, nvox * 5 * 4);
    printf("engine driver: %zu atoms (%zu per block), T %zu\n", NATOMS, natoms, T);
    return 0;
}
