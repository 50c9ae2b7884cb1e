// RA file format (replaces src/ra.cu:23-104; layout of src/ra.h:20-51).
// Header: six little-endian u64 (magic, flags, eltype, elbyte, size, ndims),
// then ndims u64 dims, then `size` data bytes, dims[0] fastest.
// Unlike the reference, reads check the magic, the endianness flag and the
// byte counts, and failures return a status instead of exiting.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime_api.h>

#include "common.h"

static const uint64_t kRaMagic = 0x7961727261776172ULL;
static const uint64_t kRaBigEndian = 1ULL;

extern "C" int snapmrf_ra_read(snapmrf_ra *a, const char *path, int pinned) {
    if (!a || !path) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "ra_read: null argument");
    memset(a, 0, sizeof *a);
    FILE *f = fopen(path, "rb");
    if (!f) SNAPMRF_FAIL(SNAPMRF_ERR_IO, "unable to open %s for reading: %s", path, strerror(errno));
    uint64_t hdr[6];
    if (fread(hdr, sizeof(uint64_t), 6, f) != 6) {
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: truncated RA header", path);
    }
    if (hdr[0] != kRaMagic) {
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: not an RA file (bad magic)", path);
    }
    if (hdr[1] & kRaBigEndian) {
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_UNSUPPORTED, "%s: big-endian RA files are not supported", path);
    }
    uint64_t ndims = hdr[5];
    if (ndims == 0 || ndims > 64) {
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: bad ndims %llu", path, (unsigned long long)ndims);
    }
    uint64_t *dims = (uint64_t *)malloc(ndims * sizeof(uint64_t));
    if (!dims || fread(dims, sizeof(uint64_t), ndims, f) != ndims) {
        free(dims);
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: truncated RA dims", path);
    }
    uint64_t size = hdr[4];
    uint8_t *data = nullptr;
    if (pinned) {
        if (cudaMallocHost((void **)&data, size ? size : 1) != cudaSuccess) data = nullptr;
    } else {
        data = (uint8_t *)malloc(size ? size : 1);
    }
    if (!data) {
        free(dims);
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_ALLOC, "%s: cannot allocate %llu bytes", path, (unsigned long long)size);
    }
    if (size && fread(data, 1, size, f) != size) {
        if (pinned) cudaFreeHost(data); else free(data);
        free(dims);
        fclose(f);
        SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: file holds fewer than %llu data bytes", path,
                     (unsigned long long)size);
    }
    fclose(f);
    a->flags = hdr[1] | (pinned ? (1ULL << 63) : 0);  // bit 63 records pinned storage
    a->eltype = hdr[2];
    a->elbyte = hdr[3];
    a->size = size;
    a->ndims = ndims;
    a->dims = dims;
    a->data = data;
    return SNAPMRF_OK;
}

extern "C" int snapmrf_ra_write(const snapmrf_ra *a, const char *path) {
    if (!a || !path || (a->ndims && !a->dims) || (a->size && !a->data))
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "ra_write: bad argument");
    FILE *f = fopen(path, "wb");
    if (!f) SNAPMRF_FAIL(SNAPMRF_ERR_IO, "unable to open %s for writing: %s", path, strerror(errno));
    uint64_t hdr[6] = {kRaMagic, a->flags & ~(1ULL << 63), a->eltype, a->elbyte, a->size, a->ndims};
    bool ok = fwrite(hdr, sizeof(uint64_t), 6, f) == 6 &&
              fwrite(a->dims, sizeof(uint64_t), a->ndims, f) == a->ndims &&
              (a->size == 0 || fwrite(a->data, 1, a->size, f) == a->size);
    ok = (fclose(f) == 0) && ok;
    if (!ok) SNAPMRF_FAIL(SNAPMRF_ERR_IO, "short write to %s", path);
    return SNAPMRF_OK;
}

extern "C" void snapmrf_ra_free(snapmrf_ra *a) {
    if (!a) return;
    if (a->data) {
        if (a->flags & (1ULL << 63)) cudaFreeHost(a->data); else free(a->data);
    }
    free(a->dims);
    a->data = nullptr;
    a->dims = nullptr;
}
