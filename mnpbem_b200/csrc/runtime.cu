// Error state, launch accounting and the host-side near-pair classification.
#include "common.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace mnpb {

static thread_local std::string t_err;
std::atomic<int64_t> g_launches{0};

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_err = buf;
}

void clear_error() { t_err.clear(); }

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return MNPB_ECUDA;
    }
    return MNPB_OK;
}

// ---- per-device kernel attributes ------------------------------------------
// cudaFuncSetAttribute acts on the current device only, so the raised
// dynamic shared-memory limit is remembered per (kernel, device) pair; the
// table is guarded by one lock (callers on several host threads are safe).
namespace {
struct SmemKey {
    const void *fn;
    int dev;
    int bytes;
};
std::mutex g_attr_mu;
std::vector<SmemKey> g_attr;
std::mutex g_sms_mu;
int g_sms[64] = {};
}  // namespace

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    return dev;
}

int smem_opt_in(const void *fn, int bytes, const char *what) {
    const int dev = current_device();
    if (dev < 0) {
        set_error("%s: cudaGetDevice failed", what);
        return MNPB_ECUDA;
    }
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (auto &k : g_attr)
        if (k.fn == fn && k.dev == dev && k.bytes >= bytes) return MNPB_OK;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) {
        set_error("%s: cannot reserve %d bytes of shared memory on device %d: %s", what, bytes,
                  dev, cudaGetErrorString(e));
        return MNPB_ECUDA;
    }
    for (auto &k : g_attr)
        if (k.fn == fn && k.dev == dev) {
            k.bytes = bytes;
            return MNPB_OK;
        }
    g_attr.push_back({fn, dev, bytes});
    return MNPB_OK;
}

int device_sms() {
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lk(g_sms_mu);
    if (g_sms[dev] == 0) {
        int v = 0;
        g_sms[dev] = (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) ==
                          cudaSuccess &&
                      v > 0)
                         ? v
                         : 148;
    }
    return g_sms[dev];
}

int check_stream_device(cudaStream_t s, const char *what) {
    if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) return MNPB_OK;
    int sd = -1;
    const int dev = current_device();
    cudaError_t e = cudaStreamGetDevice(s, &sd);
    if (e != cudaSuccess) {
        set_error("%s: cudaStreamGetDevice failed: %s", what, cudaGetErrorString(e));
        return MNPB_ECUDA;
    }
    if (sd != dev) {
        set_error("%s: the stream belongs to device %d but device %d is current", what, sd, dev);
        return MNPB_EINVAL;
    }
    return MNPB_OK;
}

// ---- event profiler ---------------------------------------------------------
// Events come from a pool; records are appended to a shared list under one
// lock; each host thread keeps its own open record (launches nest only
// within one thread's call sequence).
namespace {
struct Rec {
    cudaEvent_t a, b;
    int cls;
    double work;
    char tag[64];
};
bool g_prof = false;
std::mutex g_prof_mu;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
thread_local bool t_has_open = false;
thread_local Rec t_open;

cudaEvent_t take_event() {   // caller holds g_prof_mu
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

bool prof_on() { return g_prof; }

void prof_record(cudaStream_t s, int cls, double work, bool start) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (start) {
        t_open.a = take_event();
        t_open.cls = cls;
        t_open.work = work;
        t_open.tag[0] = 0;
        cudaEventRecord(t_open.a, s);
        t_has_open = true;
    } else if (t_has_open) {
        t_open.b = take_event();
        cudaEventRecord(t_open.b, s);
        g_recs.push_back(t_open);
        t_has_open = false;
    }
}

void prof_tag(const char *fmt, ...) {
    if (!g_prof || !t_has_open) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_open.tag, sizeof(t_open.tag), fmt, ap);
    va_end(ap);
}

}  // namespace mnpb

using namespace mnpb;

static std::vector<Rec> g_last;   // records of the last mnpb_prof_end (for mnpb_prof_dump)

// Start recording CUDA events around the library's launches (host thread
// that issues the launches; single-threaded use).
extern "C" int mnpb_prof_begin(void) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_recs.clear();
    g_prof = true;
    return MNPB_OK;
}

// Stop recording; synchronise and return per class the summed device time
// (ms), the summed algorithmic work and the launch count.
extern "C" int mnpb_prof_end(int ncls, double *ms, double *work, int64_t *count) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof = false;
    for (int c = 0; c < ncls; ++c) {
        ms[c] = 0.0;
        work[c] = 0.0;
        count[c] = 0;
    }
    for (auto &r : g_recs) {
        if (cudaEventSynchronize(r.b) != cudaSuccess) {
            set_error("prof_end: event synchronize failed");
            return MNPB_ECUDA;
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        if (r.cls >= 0 && r.cls < ncls) {
            ms[r.cls] += t;
            work[r.cls] += r.work;
            count[r.cls] += 1;
        }
    }
    g_last = g_recs;
    for (auto &r : g_recs) {
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_recs.clear();
    return MNPB_OK;
}

// Write the launches of the last profiled interval as CSV (class, ms, work,
// gap_ms = device time from the previous record's end to this record's start,
// i.e. idle time plus work launched outside the library, tag).
extern "C" int mnpb_prof_dump(const char *path) {
    clear_error();
    FILE *f = fopen(path, "w");
    if (!f) {
        set_error("prof_dump: cannot open %s", path);
        return MNPB_EINVAL;
    }
    fprintf(f, "class,ms,work,gap_ms,tag\n");
    for (size_t i = 0; i < g_last.size(); ++i) {
        const Rec &r = g_last[i];
        float t = 0.f, g = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        if (i > 0) cudaEventElapsedTime(&g, g_last[i - 1].b, r.a);
        fprintf(f, "%d,%.6f,%.6g,%.6f,%s\n", r.cls, t, r.work, g, r.tag);
    }
    fclose(f);
    return MNPB_OK;
}

extern "C" int mnpb_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" const char *mnpb_last_error(void) { return t_err.c_str(); }

extern "C" int64_t mnpb_launch_count(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------
// Near/self classification (mnpbem/greenfun/refine_utils.py:12-158).
//
// d = sqrt(|p1|^2 + |p2|^2 - 2 p1.p2) with d^2 < 1e-10 -> 0; kind 2 where
// d == 0, kind 1 where (d - rad2_j < abs_cutoff) or ((d - rad2_j)/rad1_i <
// rel_cutoff); rad1 == NULL divides by rad2_j instead (sources without a
// boundary radius, such as points).  The norms are summed x, y, z in order; the cross term is the
// 3-term dot product summed in the same order.  This file is compiled without
// floating-point contraction so no fused multiply-add changes the rounding.
// ---------------------------------------------------------------------------
extern "C" int mnpb_refinematrix(int64_t n1, int64_t n2, const double *pos1, const double *pos2,
                                 const double *rad1, const double *rad2, double abs_cutoff,
                                 double rel_cutoff, int64_t cap, int64_t *nnz, int64_t *row_ptr,
                                 int32_t *cols, int8_t *kinds) {
    clear_error();
    MNPB_REQUIRE(n1 >= 0 && n2 >= 0, "refinematrix: negative size");
    MNPB_REQUIRE(pos1 && pos2 && rad2 && nnz && row_ptr, "refinematrix: null pointer");
    std::vector<double> sq2(n2);
    for (int64_t j = 0; j < n2; ++j) {
        const double *q = pos2 + 3 * j;
        double s = q[0] * q[0];
        s = s + q[1] * q[1];
        s = s + q[2] * q[2];
        sq2[j] = s;
    }
    int64_t count = 0;
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n1; ++i) {
        const double *p = pos1 + 3 * i;
        double s1 = p[0] * p[0];
        s1 = s1 + p[1] * p[1];
        s1 = s1 + p[2] * p[2];
        for (int64_t j = 0; j < n2; ++j) {
            const double *q = pos2 + 3 * j;
            double dot = p[0] * q[0];
            dot = dot + p[1] * q[1];
            dot = dot + p[2] * q[2];
            double d2 = (s1 + sq2[j]) - 2.0 * dot;
            if (d2 < 1e-10) d2 = 0.0;
            double d = std::sqrt(d2);
            int8_t kind = 0;
            if (d == 0.0) {
                kind = 2;
            } else {
                double dd = d - rad2[j];
                double idr = dd / (rad1 ? rad1[i] : rad2[j]);
                if (dd < abs_cutoff || idr < rel_cutoff) kind = 1;
            }
            if (kind) {
                if (count < cap && cols && kinds) {
                    cols[count] = (int32_t)j;
                    kinds[count] = kind;
                }
                ++count;
            }
        }
        row_ptr[i + 1] = count;
    }
    *nnz = count;
    if (count > cap) {
        set_error("refinematrix: %lld pairs exceed capacity %lld", (long long)count, (long long)cap);
        return MNPB_ENOMEM;
    }
    return MNPB_OK;
}
