// mrf: the command-line driver of the reference (src/mrf.cu:34-386) on the
// C ABI.  Same flags, positional arguments, defaults and outputs:
//
//   mrf [OPTION] <rfpulse.csv> <imgstack.ra>
//     -M/--b1map RA   -N n (logspace grids)   -a/--atoms RA   -m/--map RA
//     -p/--params RA  -t/--T1 -s/--T2 -b/--B0 -r/--B1 grids
//     -w/--nstates n  -e/--echo_type name     -T/--nreps n
//     -G/--gridsize, -B/--blocksize (accepted, unused)  -h/--help
// The usage text's spellings --maps, --states and --timepoints are accepted
// too.  Additive options: --precision fp32|bf16|fp16|fp8, --topk 8|16,
// --all-b1-blocks (non-SSFP echo types over every B1 block), --normalize,
// --load-atoms / --load-params, --refine n, and --compress sfrac (with
// --max-rank, --out-basis, --out-compressed) for matching in the
// SVD-compressed space of each B1 block.
// Times are wall-clock (CUDA events), not the reference's CPU clock().
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <err.h>
#include <getopt.h>
#include <sysexits.h>
#include <vector>

#include <cuda_runtime.h>

#include "snapmrf.h"

static void check(int rc, const char *what) {
    if (rc) errx(rc == SNAPMRF_ERR_ECHO_TYPE ? EX_USAGE : EX_SOFTWARE, "%s: %s", what, snapmrf_last_error());
}

static void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) errx(EX_SOFTWARE, "%s: %s", what, cudaGetErrorString(e));
}

static void usage() {
    fprintf(stderr,
            "MR fingerprinting dictionary generator and image reconstructor\n"
            "Usage: mrf [OPTION] <rfpulse.csv> <imgstack.ra>\n"
            "\t-M, --b1map <rafile>\t\t B1 map input RA file\n"
            "\t-N n\t\t\t\t number of atoms (hard-coded logspace grids)\n"
            "\t-a, --atoms <rafile>\t\t dictionary atoms output RA file\n"
            "\t-m, --map, --maps <rafile>\t parameter map output RA file\n"
            "\t-p, --params <rafile>\t\t dictionary parameters output RA file\n"
            "\t-t, --T1 start:step:end\t\t T1 grid\n"
            "\t-s, --T2 start:step:end\t\t T2 grid\n"
            "\t-b, --B0 start:step:end\t\t B0 grid\n"
            "\t-r, --B1 start:step:end\t\t B1 grid\n"
            "\t-w, --nstates, --states n\t number of EPG states\n"
            "\t-e, --echo_type name\t\t echo type (epg_ssfp, roa_ssfp, epg_sr, epg_se,\n"
            "\t\t\t\t\t epg_tse1, epg_tse2, epg_fisp)\n"
            "\t-T, --nreps, --timepoints n\t number of time points\n"
            "\t-G, --gridsize n, -B, --blocksize n  accepted, unused\n"
            "\t    --precision fp32|bf16|fp16|fp8 matching form (default fp32)\n"
            "\t    --topk 4|8|16\t\t candidates rescored in FP32 (tensor-core forms)\n"
            "\t    --all-b1-blocks\t\t generate every B1 block for non-SSFP echo types\n"
            "\t    --normalize\t\t\t unit-norm every atom\n"
            "\t    --load-atoms <rafile>\t match against a saved dictionary (with --load-params)\n"
            "\t    --load-params <rafile>\t its parameter table; no dictionary is generated\n"
            "\t    --compress sfrac\t\t match in the SVD-compressed space of each B1 block,\n"
            "\t\t\t\t\t keeping the energy fraction sfrac of block 0\n"
            "\t\t\t\t\t (McGivney et al.; matlab/MRF_dict_B1.m input.reduce)\n"
            "\t    --max-rank r\t\t largest rank --compress may keep (default 64)\n"
            "\t    --out-basis <rafile>\t the bases U_r, complex (nreps, r x B1 blocks)\n"
            "\t    --out-compressed <rafile>\t the compressed atoms, complex (r, NATOMS)\n"
            "\t    --refine n\t\t\t Gauss-Newton refinement after matching, at most n\n"
            "\t\t\t\t\t iterations per voxel, from a sub-grid start taken\n"
            "\t\t\t\t\t from the dictionary (epg_fisp / epg_sr with every\n"
            "\t\t\t\t\t RF phase 0, flip angle x B1 as --all-b1-blocks:\n"
            "\t\t\t\t\t T1, T2; epg_ssfp: also B0 and B1)\n"
            "\t-h, --help\t\t\t show this help\n");
}

static std::vector<float> grid_values(const char *s) {
    size_t n = snapmrf_parse_length(s);
    if (n == 0) errx(EX_USAGE, "bad grid '%s': %s", s, snapmrf_last_error());
    std::vector<float> v(n);
    check(snapmrf_parse_params(v.data(), s, n), "parse_params");
    return v;
}

static void save_ra(const void *data, uint64_t eltype, uint64_t elbyte, const char *path, uint64_t d0, uint64_t d1) {
    uint64_t dims[2] = {d0, d1};
    snapmrf_ra a;
    a.flags = 0;
    a.eltype = eltype;
    a.elbyte = elbyte;
    a.size = d0 * d1 * elbyte;
    a.ndims = 2;
    a.dims = dims;
    a.data = (uint8_t *)data;
    check(snapmrf_ra_write(&a, path), "ra_write");
}

int main(int argc, char **argv) {
    const char *in_mrf = "../data/MRF001.csv", *in_img = NULL, *in_b1map = NULL;
    const char *out_maps = NULL, *out_atoms = NULL, *out_params = NULL;
    const char *T1 = "20:20:3000", *T2 = "20:10:1000", *B0 = "0", *B1 = "1", *echo_type = "epg_ssfp";
    int nparams = 4, nmaps = 5, nstates = 101;
    size_t nreps = 1500, NATOMS_req = 0;
    int precision = SNAPMRF_PREC_FP32, topk = 0, refine = 0, max_rank = 64;
    double compress = 0.0;
    const char *out_basis = NULL, *out_compressed = NULL;
    unsigned dict_flags = 0;
    enum { OPT_PREC = 1000, OPT_TOPK, OPT_ALLB1, OPT_NORM, OPT_REFINE, OPT_LOADA, OPT_LOADP, OPT_COMP, OPT_MAXR,
           OPT_OBAS, OPT_OCMP };
    const char *load_atoms = NULL, *load_params = NULL;
    static struct option longopts[] = {
        {"b1map", 1, NULL, 'M'},      {"atoms", 1, NULL, 'a'},       {"map", 1, NULL, 'm'},
        {"maps", 1, NULL, 'm'},       {"params", 1, NULL, 'p'},      {"T1", 1, NULL, 't'},
        {"T2", 1, NULL, 's'},         {"B0", 1, NULL, 'b'},          {"B1", 1, NULL, 'r'},
        {"nstates", 1, NULL, 'w'},    {"states", 1, NULL, 'w'},      {"echo_type", 1, NULL, 'e'},
        {"nreps", 1, NULL, 'T'},      {"timepoints", 1, NULL, 'T'},  {"gridsize", 1, NULL, 'G'},
        {"blocksize", 1, NULL, 'B'},  {"NATOMS", 1, NULL, 'N'},      {"help", 0, NULL, 'h'},
        {"precision", 1, NULL, OPT_PREC}, {"topk", 1, NULL, OPT_TOPK},
        {"all-b1-blocks", 0, NULL, OPT_ALLB1}, {"normalize", 0, NULL, OPT_NORM},
        {"refine", 1, NULL, OPT_REFINE},  {"load-atoms", 1, NULL, OPT_LOADA},
        {"load-params", 1, NULL, OPT_LOADP}, {"compress", 1, NULL, OPT_COMP},
        {"max-rank", 1, NULL, OPT_MAXR},      {"out-basis", 1, NULL, OPT_OBAS},
        {"out-compressed", 1, NULL, OPT_OCMP}, {NULL, 0, NULL, 0}};
    opterr = 0;
    int c;
    while ((c = getopt_long(argc, argv, "M:N:a:m:p:t:s:b:r:w:e:T:G:B:h", longopts, NULL)) != -1) {
        switch (c) {
        case 'M': in_b1map = optarg; break;
        case 'N': NATOMS_req = (size_t)atoi(optarg); break;
        case 'a': out_atoms = optarg; break;
        case 'm': out_maps = optarg; break;
        case 'p': out_params = optarg; break;
        case 't': T1 = optarg; break;
        case 's': T2 = optarg; break;
        case 'b': B0 = optarg; break;
        case 'r': B1 = optarg; break;
        case 'w': nstates = atoi(optarg); break;
        case 'e': echo_type = optarg; break;
        case 'T': nreps = (size_t)atoi(optarg); break;
        case 'G': case 'B': break;
        case OPT_PREC:
            if (!strcmp(optarg, "fp32")) precision = SNAPMRF_PREC_FP32;
            else if (!strcmp(optarg, "bf16")) precision = SNAPMRF_PREC_BF16;
            else if (!strcmp(optarg, "fp16")) precision = SNAPMRF_PREC_FP16;
            else if (!strcmp(optarg, "fp8")) precision = SNAPMRF_PREC_FP8;
            else errx(EX_USAGE, "--precision must be fp32, bf16, fp16 or fp8");
            break;
        case OPT_TOPK: topk = atoi(optarg); break;
        case OPT_ALLB1: dict_flags |= SNAPMRF_DICT_ALL_B1_BLOCKS; break;
        case OPT_NORM: dict_flags |= SNAPMRF_DICT_NORMALIZE; break;
        case OPT_REFINE: refine = atoi(optarg); break;
        case OPT_LOADA: load_atoms = optarg; break;
        case OPT_LOADP: load_params = optarg; break;
        case OPT_COMP: compress = atof(optarg); break;
        case OPT_MAXR: max_rank = atoi(optarg); break;
        case OPT_OBAS: out_basis = optarg; break;
        case OPT_OCMP: out_compressed = optarg; break;
        case 'h':
        default: usage(); return 1;
        }
    }
    // positional: the first *.ra is the image stack, the first *.csv the schedule
    bool have_ra = false, have_csv = false;
    for (int i = optind; i < argc && !(have_ra && have_csv); i++) {
        if (!have_ra && strstr(argv[i], ".ra")) { in_img = argv[i]; have_ra = true; }
        if (!have_csv && strstr(argv[i], ".csv")) { in_mrf = argv[i]; have_csv = true; }
    }
    printf("\nnstates : %d\nEcho : %s\n\n", nstates, echo_type);

    if ((load_atoms != NULL) != (load_params != NULL)) errx(EX_USAGE, "--load-atoms and --load-params go together");
    const bool loading = load_atoms != NULL;
    // parameter grids (src/mrf.cu:168-232), or a saved parameter table
    std::vector<float> t1, t2, b0, b1;
    snapmrf_ra ra_atoms, ra_params;
    memset(&ra_atoms, 0, sizeof ra_atoms);
    memset(&ra_params, 0, sizeof ra_params);
    if (loading) {
        printf("Loading dictionary...\nAtoms : %s\nParams : %s\n", load_atoms, load_params);
        check(snapmrf_ra_read(&ra_params, load_params, 0), "ra_read");
        check(snapmrf_ra_read(&ra_atoms, load_atoms, 0), "ra_read");
        if (ra_params.eltype != 3 || ra_params.elbyte != 4 || ra_params.ndims < 2 || ra_params.dims[0] != 4)
            errx(EX_DATAERR, "%s: expected a float (4, NATOMS) parameter table", load_params);
        if (ra_atoms.eltype != 4 || ra_atoms.elbyte != 8 || ra_atoms.ndims < 2 || ra_atoms.dims[1] != ra_params.dims[1])
            errx(EX_DATAERR, "%s: expected complex (T, %llu) atoms", load_atoms,
                 (unsigned long long)ra_params.dims[1]);
    } else if (NATOMS_req != 0) {
        printf("Hard coding for parameters...\n");
        size_t l_b1 = 11, l_b0 = 21;
        size_t l_t = (size_t)roundf(sqrtf((float)(NATOMS_req / l_b0 / l_b1)));
        if (l_t == 0) l_t = 1;
        t1.resize(l_t); t2.resize(l_t); b0.resize(l_b0); b1.resize(l_b1);
        snapmrf_logspace(t1.data(), 100.f, 3000.f, l_t);
        snapmrf_logspace(t2.data(), 20.f, 1000.f, l_t);
        snapmrf_logspace(b0.data(), -150.f, 150.f, l_b0);
        snapmrf_logspace(b1.data(), 0.5f, 1.5f, l_b1);
    } else {
        printf("Parsing parameters...\nT1 : %s\nT2 : %s\nB0 : %s\nB1 : %s\n", T1, T2, B0, B1);
        t1 = grid_values(T1); t2 = grid_values(T2); b0 = grid_values(B0); b1 = grid_values(B1);
    }
    size_t NATOMS, natoms;
    std::vector<float> h_params;
    if (loading) {
        NATOMS = (size_t)ra_params.dims[1];
        const float *pr = reinterpret_cast<const float *>(ra_params.data);
        h_params.assign(pr, pr + NATOMS * nparams);
        // B1 blocks: the table's leading run of one B1 value (trans_params order)
        natoms = 1;
        while (natoms < NATOMS && pr[natoms * nparams + 3] == pr[3]) natoms++;
        if (NATOMS % natoms != 0) errx(EX_DATAERR, "%s: B1 blocks of unequal size", load_params);
        printf("NATOMS: %zu, natoms: %zu\n", NATOMS, natoms);
    } else {
        NATOMS = snapmrf_compute_natoms(t1.data(), t2.data(), t1.size(), t2.size(), b0.size(), b1.size());
        natoms = NATOMS / b1.size();
        printf("l_t1: %zu, l_t2: %zu, l_b0: %zu, l_b1: %zu\nNATOMS: %zu, natoms: %zu\n", t1.size(), t2.size(),
               b0.size(), b1.size(), NATOMS, natoms);
        if (NATOMS == 0) errx(EX_SOFTWARE, "Number of atoms is 0!");
        h_params.resize(NATOMS * nparams);
        check(snapmrf_trans_params(h_params.data(), t1.data(), t2.data(), b0.data(), b1.data(), t1.size(),
                                   t2.size(), b0.size(), b1.size(), NATOMS, nparams),
              "trans_params");
    }

    // schedule (src/mrf.cu:260-276)
    printf("Input mrf: %s\n", in_mrf);
    size_t lines = snapmrf_csv_dim(in_mrf);
    if (lines == (size_t)-1 || lines < 2) errx(EX_NOINPUT, "cannot read schedule %s", in_mrf);
    size_t NREPS = lines - 1;
    if (nreps > NREPS) nreps = NREPS;
    if (loading) {
        if ((size_t)ra_atoms.dims[0] > NREPS) errx(EX_DATAERR, "%s: more time points than the schedule", load_atoms);
        nreps = (size_t)ra_atoms.dims[0];
    }
    printf("NREPS: %zu, nreps: %zu\n\n", NREPS, nreps);
    std::vector<float> h_mrf(NREPS * 4);
    check(snapmrf_csv_read(h_mrf.data(), NREPS, in_mrf), "csv_read");

    cuda_check(cudaSetDevice(0), "cudaSetDevice");
    cudaStream_t st;
    cuda_check(cudaStreamCreate(&st), "cudaStreamCreate");
    float *d_params;
    float *d_atoms;
    cuda_check(cudaMalloc((void **)&d_params, h_params.size() * sizeof(float)), "cudaMalloc");
    cuda_check(cudaMemcpyAsync(d_params, h_params.data(), h_params.size() * sizeof(float), cudaMemcpyHostToDevice, st),
               "cudaMemcpy");
    cuda_check(cudaMalloc((void **)&d_atoms, nreps * NATOMS * 2 * sizeof(float)), "cudaMalloc");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);

    float ms = 0;
    if (loading) {
        cuda_check(cudaMemcpyAsync(d_atoms, ra_atoms.data, nreps * NATOMS * 2 * sizeof(float), cudaMemcpyHostToDevice,
                                   st), "cudaMemcpy");
        cuda_check(cudaStreamSynchronize(st), "dictionary upload");
        snapmrf_ra_free(&ra_atoms);
        snapmrf_ra_free(&ra_params);
    } else {
        snapmrf_dict_opts dopt;
        memset(&dopt, 0, sizeof dopt);
        dopt.flags = dict_flags;
        dopt.n_iso = 1;
        printf("Constructing dictionary...\n");
        cudaEventRecord(e0, st);
        check(snapmrf_mrf_dict(d_atoms, d_params, h_mrf.data(), nreps, NREPS, NATOMS, natoms, nparams, nstates,
                               echo_type, &dopt, st), "MRF_dict");
        cudaEventRecord(e1, st);
        cuda_check(cudaStreamSynchronize(st), "dictionary");
        cudaEventElapsedTime(&ms, e0, e1);
        printf("Elapsed dictionary time: %.4f s\n\n", ms / 1e3);
    }

    // low-rank compression per B1 block (the MATLAB code's input.reduce)
    float *d_basis = NULL, *d_coeffs = NULL;
    int svd_rank = 0;
    if (compress > 0.0) {
        const size_t nb = NATOMS / natoms;
        cuda_check(cudaMalloc((void **)&d_basis, nb * max_rank * nreps * 2 * sizeof(float)), "cudaMalloc");
        cuda_check(cudaMalloc((void **)&d_coeffs, NATOMS * max_rank * 2 * sizeof(float)), "cudaMalloc");
        snapmrf_svd_opts so;
        memset(&so, 0, sizeof so);
        so.sfrac = compress;
        printf("Compressing dictionary (SVD per B1 block, sfrac %g)...\n", compress);
        cudaEventRecord(e0, st);
        check(snapmrf_svd_compress(d_atoms, nreps, NATOMS, natoms, max_rank, d_basis, nreps, d_coeffs,
                                   (size_t)max_rank, &svd_rank, NULL, &so, st), "svd_compress");
        cudaEventRecord(e1, st);
        cuda_check(cudaStreamSynchronize(st), "compression");
        cudaEventElapsedTime(&ms, e0, e1);
        printf("Rank: %d\nElapsed compression time: %.4f s\n\n", svd_rank, ms / 1e3);
        if (out_basis) {
            // MATLAB's U_r: the blocks' r vectors side by side, (nreps, r * nb)
            printf("Output basis: %s\n", out_basis);
            std::vector<float> h(nb * max_rank * nreps * 2), o(nb * svd_rank * nreps * 2);
            cuda_check(cudaMemcpy(h.data(), d_basis, h.size() * sizeof(float), cudaMemcpyDeviceToHost), "cudaMemcpy");
            for (size_t b = 0; b < nb; b++)
                memcpy(&o[b * svd_rank * nreps * 2], &h[b * max_rank * nreps * 2], svd_rank * nreps * 2 * sizeof(float));
            save_ra(o.data(), 4, 8, out_basis, nreps, nb * svd_rank);
        }
        if (out_compressed) {
            // MATLAB's dict_compress: (r, NATOMS)
            printf("Output compressed atoms: %s\n", out_compressed);
            std::vector<float> h(NATOMS * max_rank * 2), o(NATOMS * svd_rank * 2);
            cuda_check(cudaMemcpy(h.data(), d_coeffs, h.size() * sizeof(float), cudaMemcpyDeviceToHost), "cudaMemcpy");
            for (size_t j = 0; j < NATOMS; j++)
                memcpy(&o[j * svd_rank * 2], &h[j * max_rank * 2], svd_rank * 2 * sizeof(float));
            save_ra(o.data(), 4, 8, out_compressed, svd_rank, NATOMS);
        }
    }

    if (!in_img && out_maps) printf("NO data specified! Abort matching!\n");
    if (in_img) {
        printf("Input img: %s\n", in_img);
        snapmrf_ra img;
        check(snapmrf_ra_read(&img, in_img, 1), "ra_read");
        if (img.eltype != 4 || img.elbyte != 8 || img.ndims < 2)
            errx(EX_DATAERR, "%s: expected a complex (nt, nx[, ny]) RA image", in_img);
        size_t nt = img.dims[0];
        size_t nvoxels = img.dims[1] * (img.ndims > 2 ? img.dims[2] : 1);
        printf("nt: %zu, voxels: %zu\n\n", nt, nvoxels);
        std::vector<float> h_b1;
        snapmrf_match_opts mopt;
        memset(&mopt, 0, sizeof mopt);
        mopt.precision = precision;
        mopt.img_stride = nt;
        mopt.atom_stride = nreps;
        mopt.topk = topk;
        if (d_basis) {
            mopt.basis = d_basis;
            mopt.basis_rows = (size_t)max_rank;
            mopt.basis_stride = nreps;
            mopt.coeffs = d_coeffs;
            mopt.coeff_stride = (size_t)max_rank;
            mopt.rank = svd_rank;
        }
        snapmrf_ra b1ra;
        memset(&b1ra, 0, sizeof b1ra);
        if (in_b1map) {
            printf("Input B1 map: %s\n", in_b1map);
            check(snapmrf_ra_read(&b1ra, in_b1map, 1), "ra_read");
            if (b1ra.eltype != 3 || b1ra.elbyte != 4 || b1ra.size < nvoxels * sizeof(float))
                errx(EX_DATAERR, "%s: B1 map must hold %zu float values", in_b1map, nvoxels);
            mopt.b1map = reinterpret_cast<const float *>(b1ra.data);
            mopt.b1map_on_host = 1;
        }
        float *d_maps;
        cuda_check(cudaMalloc((void **)&d_maps, nmaps * nvoxels * sizeof(float)), "cudaMalloc");
        // the refinement starts from the matched atom's neighbourhood of the
        // dictionary, which needs the match's atom index
        int64_t *d_index = NULL;
        if (refine > 0) {
            cuda_check(cudaMalloc((void **)&d_index, nvoxels * sizeof(int64_t)), "cudaMalloc");
            mopt.d_index = d_index;
        }
        printf("Matching...\n");
        cudaEventRecord(e0, st);
        check(snapmrf_mrf_match(d_maps, reinterpret_cast<const float *>(img.data), 1, d_atoms, d_params,
                                nreps < nt ? nreps : nt, NATOMS, natoms, nvoxels, nparams, nmaps, &mopt, st),
              "MRF_match");
        cudaEventRecord(e1, st);
        cuda_check(cudaStreamSynchronize(st), "matching");
        cudaEventElapsedTime(&ms, e0, e1);
        printf("Elapsed matching time: %.4f s\n\n", ms / 1e3);
        if (refine > 0) {
            // the voxels and the B1 map on the device, then Gauss-Newton in place
            float *d_img = NULL, *d_b1 = NULL;
            const size_t m = nreps < nt ? nreps : nt;
            cuda_check(cudaMalloc((void **)&d_img, nvoxels * nt * 2 * sizeof(float)), "cudaMalloc");
            cuda_check(cudaMemcpyAsync(d_img, img.data, nvoxels * nt * 2 * sizeof(float), cudaMemcpyHostToDevice,
                                       st), "cudaMemcpy");
            if (in_b1map) {
                cuda_check(cudaMalloc((void **)&d_b1, nvoxels * sizeof(float)), "cudaMalloc");
                cuda_check(cudaMemcpyAsync(d_b1, b1ra.data, nvoxels * sizeof(float), cudaMemcpyHostToDevice, st),
                           "cudaMemcpy");
            }
            printf("Refining (sub-grid start from the dictionary, then Gauss-Newton, at most %d iterations)...\n",
                   refine);
            cudaEventRecord(e0, st);
            check(snapmrf_refine_start(d_maps, nmaps, d_index, d_atoms, d_params, nparams, nreps, NATOMS, natoms,
                                       d_img, nt, nvoxels, d_b1, 0, NULL, st),
                  "refine_start");
            check(snapmrf_refine_gn(d_maps, nmaps, d_img, nt, d_b1, h_mrf.data(), m, NREPS, nvoxels, nstates,
                                    echo_type, refine, 0.2f, 1e-4f, NULL, st),
                  "refine_gn");
            cudaEventRecord(e1, st);
            cuda_check(cudaStreamSynchronize(st), "refinement");
            cudaEventElapsedTime(&ms, e0, e1);
            printf("Elapsed refinement time: %.4f s\n\n", ms / 1e3);
            cudaFree(d_img);
            if (d_b1) cudaFree(d_b1);
            cudaFree(d_index);
        }
        if (!out_maps) out_maps = "../result/maps.ra";
        printf("Output maps: %s\n", out_maps);
        std::vector<float> h_maps(nmaps * nvoxels);
        cuda_check(cudaMemcpy(h_maps.data(), d_maps, h_maps.size() * sizeof(float), cudaMemcpyDeviceToHost),
                   "cudaMemcpy");
        save_ra(h_maps.data(), 3, 4, out_maps, nmaps, nvoxels);
        cudaFree(d_maps);
        snapmrf_ra_free(&img);
        if (in_b1map) snapmrf_ra_free(&b1ra);
    }
    if (out_atoms) {
        printf("Output atoms: %s\n", out_atoms);
        std::vector<float> h(nreps * NATOMS * 2);
        cuda_check(cudaMemcpy(h.data(), d_atoms, h.size() * sizeof(float), cudaMemcpyDeviceToHost), "cudaMemcpy");
        save_ra(h.data(), 4, 8, out_atoms, nreps, NATOMS);
    }
    if (out_params) {
        printf("Output params: %s\n", out_params);
        save_ra(h_params.data(), 3, 4, out_params, nparams, NATOMS);
    }
    cudaFree(d_atoms);
    cudaFree(d_params);
    if (d_basis) cudaFree(d_basis);
    if (d_coeffs) cudaFree(d_coeffs);
    cudaStreamDestroy(st);
    return 0;
}
