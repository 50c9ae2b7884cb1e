// Host side of the snapMRF path: error reporting, the schedule CSV reader,
// the grid-string parser and the parameter table.  Each function keeps the
// float arithmetic of the reference function it replaces, so the parameter
// values (and therefore atom order and map values) are bit-identical; the
// differences are that failures return a status instead of asserting or
// crashing.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <map>
#include <mutex>

#include <cuda_runtime.h>

#include "common.h"

namespace snapmrf {

// Page-locked staging slots of this thread per device, used in turn.  A slot
// is reused only after the copy that read it has run (its event), so the
// host blocks only when it is kStageSlots calls ahead of the device.
constexpr int kStageSlots = 4;

struct StageSlot {
    void *p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
};

struct Stage {
    StageSlot slot[kStageSlots];
    int cur = 0;
};

static thread_local std::map<int, Stage> g_stage;

void *stage_acquire(size_t bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    Stage &st = g_stage[dev];
    st.cur = (st.cur + 1) % kStageSlots;
    StageSlot &s = st.slot[st.cur];
    if (s.ev) cudaEventSynchronize(s.ev);
    if (s.cap < bytes) {
        if (s.p) cudaFreeHost(s.p);
        s.cap = 0;
        size_t want = bytes < 65536 ? 65536 : bytes;
        if (cudaHostAlloc(&s.p, want, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
            s.p = nullptr;
            return nullptr;
        }
        s.cap = want;
    }
    return s.p;
}

// Reads the staged words straight from page-locked host memory (mapped into
// the device's address space), so the upload does not queue on the copy
// engine behind large transfers of other streams.
__global__ void stage_copy_kernel(uint32_t *dst, const uint32_t *src, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

cudaError_t stage_upload(void *d_dst, const void *h_stage, size_t bytes, cudaStream_t st) {
    // the slot's address in the device's address space; without one (memory
    // not mapped), an ordinary copy
    void *src = nullptr;
    if (bytes % 4 != 0 || cudaHostGetDevicePointer(&src, const_cast<void *>(h_stage), 0) != cudaSuccess || !src) {
        cudaGetLastError();
        return cudaMemcpyAsync(d_dst, h_stage, bytes, cudaMemcpyHostToDevice, st);
    }
    const long long n = (long long)(bytes / 4);
    const unsigned blocks = (unsigned)std::min<long long>(64, (n + 255) / 256);
    stage_copy_kernel<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(static_cast<uint32_t *>(d_dst),
                                                               static_cast<const uint32_t *>(src), n);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t stage_release(cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    StageSlot &s = g_stage[dev].slot[g_stage[dev].cur];
    if (!s.ev) {
        e = cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaEventRecord(s.ev, st);
}

static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

cudaError_t device_pool(cudaMemPool_t *pool) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) {
        *pool = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p;
    e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t threshold = ~0ull;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold);
    if (e != cudaSuccess) return e;
    g_pools[dev] = p;
    *pool = p;
    return cudaSuccess;
}

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

static std::atomic<uint64_t> g_launches{0};

void note_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static std::atomic<uint64_t> g_scratch_allocs{0};

void note_scratch_alloc() { g_scratch_allocs.fetch_add(1, std::memory_order_relaxed); }

}  // namespace snapmrf

using snapmrf::set_error;

extern "C" const char *snapmrf_last_error(void) { return snapmrf::g_last_error.c_str(); }

extern "C" const char *snapmrf_version(void) { return "snapmrf-b200 0.1 (sm_100a)"; }

extern "C" uint64_t snapmrf_kernel_launches(void) { return snapmrf::g_launches.load(); }

extern "C" uint64_t snapmrf_scratch_allocations(void) { return snapmrf::g_scratch_allocs.load(); }

// Returns the scratch memory cached by the library's pool on the current
// device to the driver (after the device finishes its pending work).
extern "C" int snapmrf_release_scratch(void) {
    cudaMemPool_t pool;
    cudaError_t e = snapmrf::device_pool(&pool);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    if (e != cudaSuccess)
        return set_error(SNAPMRF_ERR_CUDA, "release_scratch: %s", cudaGetErrorString(e));
    return SNAPMRF_OK;
}

// csv_dim (src/functions.cu:100-120): counts '\n'.  The reference reads with
// a signed char compared against EOF, so a 0xFF byte also ends the count.
extern "C" size_t snapmrf_csv_dim(const char *path) {
    FILE *f = path ? fopen(path, "r") : nullptr;
    if (!f) {
        set_error(SNAPMRF_ERR_IO, "unable to open file %s", path ? path : "(null)");
        return (size_t)-1;
    }
    size_t rows = 0;
    for (int c = getc(f); c != EOF && c != 0xFF; c = getc(f))
        if (c == '\n') rows++;
    fclose(f);
    return rows;
}

// csv_read (src/functions.cu:122-158): fgets in 100-byte chunks, the first
// two chunks are skipped, then up to nreps rows of four comma-separated
// columns into h_mrf[4][nreps].
extern "C" int snapmrf_csv_read(float *h_mrf, size_t nreps, const char *path) {
    if (!h_mrf || !path) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "csv_read: null argument");
    FILE *f = fopen(path, "r");
    if (!f) SNAPMRF_FAIL(SNAPMRF_ERR_IO, "unable to open file %s", path);
    char buffer[100];
    size_t index = 0;
    int count = 0;
    while (fgets(buffer, 100, f) && index < nreps) {
        if (count > 1) {
            char *tok[4];
            tok[0] = strtok(buffer, ",");
            for (int c = 1; c < 4; c++) tok[c] = tok[c - 1] ? strtok(nullptr, ",") : nullptr;
            for (int c = 0; c < 4; c++) {
                if (!tok[c]) {
                    fclose(f);
                    SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "%s: row %zu has fewer than 4 columns", path,
                                 index + 1);
                }
                h_mrf[c * nreps + index] = (float)atof(tok[c]);
            }
            index++;
        }
        count++;
    }
    fclose(f);
    return SNAPMRF_OK;
}

// parse_range (src/functions.cu:197-237).  The reference asserts max >= min;
// a zero or negative step with three fields has no defined length there.
extern "C" int snapmrf_parse_range(const char *str, float *min, float *step, float *max,
                                   size_t *len) {
    if (!str || !min || !step || !max || !len)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "parse_range: null argument");
    float tmp = (float)atof(str);
    *min = tmp;
    const char *p = strchr(str, ':');
    if (!p) {
        *step = 0;
        *max = tmp;
        *len = 1;
        return SNAPMRF_OK;
    }
    p = p + 1;
    tmp = (float)atof(p);
    *step = tmp;
    p = strchr(p, ':');
    if (!p) {
        *step = 1;
        *max = tmp;
        if (!(*max >= *min)) SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "grid '%s': max < min", str);
        *len = (size_t)(((*max - *min) / 1) + 1);
        return SNAPMRF_OK;
    }
    p = p + 1;
    tmp = (float)atof(p);
    *max = tmp;
    if (!(*max >= *min)) SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "grid '%s': max < min", str);
    if (!(*step > 0)) SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "grid '%s': step must be > 0", str);
    float n = ((*max - *min) / *step) + 1;
    if (!(n < 1e9f)) SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "grid '%s': too many values", str);
    *len = (size_t)n;
    return SNAPMRF_OK;
}

// Shared walk over the '+'-joined ranges of parse_length / parse_params
// (src/functions.cu:239-269, 315-353).  A range whose start equals the
// running end value (|tmp - min| < 1e-7) drops its first value; the running
// value after a later range is min + len*step, as in the reference.
static int walk_ranges(const char *str, float *h_p, size_t cap, size_t *total) {
    if (!str) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "grid string is null");
    size_t n = strlen(str);
    if (n >= 1024) SNAPMRF_FAIL(SNAPMRF_ERR_FORMAT, "grid string longer than 1023 characters");
    char str_cpy[1024];
    memcpy(str_cpy, str, n + 1);
    size_t stride = 0;
    int count = 0;
    float tmp = 0.f;
    char *save = nullptr;
    for (char *range = strtok_r(str_cpy, "+", &save); range; range = strtok_r(nullptr, "+", &save)) {
        count++;
        float mn, st, mx;
        size_t len;
        int rc = snapmrf_parse_range(range, &mn, &st, &mx, &len);
        if (rc) return rc;
        float start = mn;
        if (count == 1) {
            tmp = mn + (len - 1) * st;
        } else {
            if (std::fabs(tmp - mn) < 1E-7) {
                len = len - 1;
                start = mn + st;
            }
            tmp = mn + len * st;
        }
        if (h_p) {
            if (stride + len > cap) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "grid '%s' longer than %zu", str, cap);
            snapmrf_linspace(h_p + stride, start, st, len);
        }
        stride += len;
    }
    *total = stride;
    return SNAPMRF_OK;
}

extern "C" size_t snapmrf_parse_length(const char *str) {
    size_t total = 0;
    if (walk_ranges(str, nullptr, 0, &total)) return 0;
    return total;
}

extern "C" int snapmrf_parse_params(float *h_p, const char *str, size_t LEN) {
    if (!h_p) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "parse_params: null output");
    size_t total = 0;
    int rc = walk_ranges(str, h_p, LEN, &total);
    if (rc) return rc;
    if (total != LEN) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "grid '%s' has %zu values, not %zu", str, total, LEN);
    return SNAPMRF_OK;
}

// linspace (src/functions.cu:271-276)
extern "C" void snapmrf_linspace(float *h_p, float min, float step, size_t len) {
    for (int i = 0; i < (int)len; i++) h_p[i] = min + i * step;
}

// logspace (src/functions.cu:278-313).  The negative branch builds a
// symmetric grid -10^((len/2-i)*s) .. 0 .. 10^((i+1)*s); the reference's
// second loop writes one or two entries past len, which are not written here.
extern "C" void snapmrf_logspace(float *h_p, float min, float max, size_t len) {
    if (len == 0) return;
    if (min > max) {
        float t = min;
        min = max;
        max = t;
    }
    if (len == 1) {
        h_p[0] = (min + max) / 2.f;
        return;
    }
    if (min > 0.f) {
        float logmin = std::log10(min), logmax = std::log10(max);
        float logstep = (logmax - logmin) / (len - 1);
        for (int i = 0; i < (int)len; i++) h_p[i] = std::pow(10.f, logmin + i * logstep);
    } else {
        float logmax = std::log10(max);
        float logstep = logmax / (len / 2);
        for (int i = 0; i < (int)(len / 2 + 1); i++) h_p[i] = -std::pow(10.f, (len / 2 - i) * logstep);
        h_p[len / 2] = 0.f;
        for (int i = 0; i < (int)(len / 2 + 1); i++)
            if (i + len / 2 + 1 < len) h_p[i + len / 2 + 1] = std::pow(10.f, (i + 1) * logstep);
    }
}

// compute_natoms (src/functions.cu:393-414)
extern "C" size_t snapmrf_compute_natoms(const float *h_t1, const float *h_t2, size_t l_t1,
                                         size_t l_t2, size_t l_b0, size_t l_b1) {
    size_t n = 0;
    for (size_t i = 0; i < l_t1; i++)
        for (size_t j = 0; j < l_t2; j++)
            if (h_t1[i] > h_t2[j]) n++;
    return n * l_b0 * l_b1;
}

// trans_params (src/functions.cu:355-391): B1 outermost, then B0, T2, T1.
extern "C" int snapmrf_trans_params(float *h_params, const float *h_t1, const float *h_t2,
                                    const float *h_b0, const float *h_b1, size_t l_t1,
                                    size_t l_t2, size_t l_b0, size_t l_b1, size_t NATOMS,
                                    int nparams) {
    if (!h_params || nparams < 4) SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "trans_params: bad arguments");
    size_t count = 0;
    for (size_t h = 0; h < l_b1; h++)
        for (size_t i = 0; i < l_b0; i++)
            for (size_t j = 0; j < l_t2; j++)
                for (size_t k = 0; k < l_t1; k++) {
                    float T1 = h_t1[k], T2 = h_t2[j];
                    if (T1 > T2) {
                        if (count >= NATOMS)
                            SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "trans_params: more than %zu atoms", NATOMS);
                        float *p = h_params + count * nparams;
                        p[0] = T1;
                        p[1] = T2;
                        p[2] = h_b0[i];
                        p[3] = h_b1[h];
                        count++;
                    }
                }
    if (count != NATOMS)
        SNAPMRF_FAIL(SNAPMRF_ERR_INVALID, "trans_params: %zu atoms, expected %zu", count, NATOMS);
    return SNAPMRF_OK;
}
