// Drop-in implementation of the OpenCL-wrapper entry points BigDFT's Fortran
// host calls (bigdft/src/OpenCL/OpenCL_wrappers.h), on CUDA streams.
//
// Handles: a context is a device index, a command queue an in-order CUDA
// stream plus a small FP64 reduction workspace, a cl_mem a (device pointer,
// size) pair.  The caller owns every buffer, as in the reference.  Where the
// reference calls exit(1) (oclErrorCheck, OpenCL_wrappers.h:89) this layer
// records a sticky error on the queue and in wvlh_get_last_error().
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <ctime>
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_plain.h"

// A cl_mem is device memory (cudaMalloc, host == nullptr) or host memory the
// caller handed over (host != nullptr: the reference's CL_MEM_USE_HOST_PTR
// buffers and pinned regions), page-locked so that copies from and to it run
// as DMA without staging.  Under unified addressing the locked range is
// addressable from kernels at its host address.
struct wvlh_mem {
    void *ptr;
    size_t size;
    void *host = nullptr;
    uintptr_t pin_lo = 0, pin_hi = 0;  // the page range this handle holds locked (0, 0: none)
};
struct wvlh_ocl_context {
    int device;
};
struct wvlh_ocl_queue {
    wvlh_ocl_context *ctx;
    cudaStream_t stream;
    double *d_work;   // kDotParts partials + 64 result slots
    double *h_stage;  // 64 pinned result slots
    int next_slot;
    std::vector<std::pair<double *, int>> pending;  // (host destination, slot) resolved at ocl_finish
    int error;
};

// page-locked host ranges (see pin_acquire)
struct PinRange {
    uintptr_t end;
    int refs;
};
static std::mutex g_pin_mu;
static std::map<uintptr_t, PinRange> g_pins;
static std::vector<wvlh_ocl_queue *> g_queues;  // every live queue, for the wait before unlocking

namespace wvlh {
static int g_last_error = 0;
void set_last_error(int code) { g_last_error = code; }
}  // namespace wvlh

using namespace wvlh;

extern "C" int wvlh_get_last_error(void)
{
    const int e = g_last_error;
    g_last_error = 0;
    return e;
}
extern "C" const char *wvlh_error_string(int code)
{
    switch (code) {
    case WVLH_OK: return "success";
    case WVLH_ERR_CUDA: return "CUDA runtime error";
    case WVLH_ERR_ARG: return "invalid argument";
    case WVLH_ERR_KEYS: return "invalid segment keys";
    case WVLH_ERR_NOMEM: return "device allocation failed";
    case WVLH_ERR_UNSUPPORTED: return "unsupported (k-points / spinors)";
    case WVLH_ERR_TOO_LARGE: return "box too large for this path";
    case WVLH_ERR_STALE: return "batch tables replaced by a newer orbital batch";
    default: return "unknown error";
    }
}
extern "C" void *wvlh_mem_ptr(cl_mem m) { return m ? m->ptr : nullptr; }

static void qerr(bigdft_command_queue q, int code, const char *what)
{
    if (q) q->error = code;
    g_last_error = code;
    fprintf(stderr, "wvlh: error %d (%s) in %s\n", code, wvlh_error_string(code), what);
}
#define QCK(q, x)                                                                    \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            fprintf(stderr, "wvlh: %s: %s\n", __func__, cudaGetErrorString(e_));     \
            qerr((q), WVLH_ERR_CUDA, __func__);                                      \
            return;                                                                  \
        }                                                                            \
    } while (0)

static inline double *D(cl_mem *m) { return (double *)(*m)->ptr; }
static inline uint32_t *U(cl_mem *m) { return (uint32_t *)(*m)->ptr; }

// ---------------------------------------------------------------- lifecycle
extern "C" void ocl_create_gpu_context_(bigdft_context *context, cl_uint *device_number)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        *context = nullptr;
        qerr(nullptr, WVLH_ERR_CUDA, "ocl_create_gpu_context");
        return;
    }
    wvlh_ocl_context *c = new wvlh_ocl_context();
    c->device = 0;
    *context = c;
    if (device_number) *device_number = (cl_uint)n;
}

extern "C" void ocl_create_context_(bigdft_context *context, const char *platform, const char *devices,
                                    cl_int *device_type, cl_uint *device_number)
{
    (void)platform;
    (void)devices;
    (void)device_type;
    ocl_create_gpu_context_(context, device_number);
}

// real-time clock in nanoseconds since the epoch (OpenCL_wrappers.h:305-306),
// the host's timer (memguess.f90:2164, MPIfake.f90:419)
extern "C" void nanosec_(unsigned long long *t)
{
    timespec ts;
    clock_gettime(CLOCK_REALTIME, &ts);
    *t = (unsigned long long)ts.tv_sec * 1000000000ull + (unsigned long long)ts.tv_nsec;
}

extern "C" void ocl_build_programs_(bigdft_context *context) { (void)context; }
extern "C" void init_event_list_(bigdft_context *context) { (void)context; }
extern "C" void print_event_list_(bigdft_context *context) { (void)context; }

extern "C" void ocl_create_command_queue_id_(bigdft_command_queue *command_queue, bigdft_context *context,
                                             cl_uint *index)
{
    wvlh_ocl_queue *q = new wvlh_ocl_queue();
    q->ctx = *context;
    q->error = 0;
    q->next_slot = 0;
    int n = 1;
    cudaGetDeviceCount(&n);
    const int dev = (index && n > 0) ? (int)(*index % (cl_uint)n) : 0;
    if (q->ctx) q->ctx->device = dev;
    *command_queue = q;
    QCK(q, cudaSetDevice(dev));
    QCK(q, cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking));
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        g_queues.push_back(q);
    }
    QCK(q, cudaMalloc(&q->d_work, sizeof(double) * (kDotParts + 64)));
    QCK(q, cudaMallocHost(&q->h_stage, sizeof(double) * 64));
}

extern "C" void ocl_create_command_queue_(bigdft_command_queue *command_queue, bigdft_context *context)
{
    cl_uint z = 0;
    ocl_create_command_queue_id_(command_queue, context, &z);
}

static void create_buffer(cl_uint *size, cl_mem *buff_ptr)
{
    wvlh_mem *m = new wvlh_mem();
    m->size = *size;
    m->ptr = nullptr;
    if (m->size && cudaMalloc(&m->ptr, m->size) != cudaSuccess) {
        qerr(nullptr, WVLH_ERR_NOMEM, "ocl_create_buffer");
        m->ptr = nullptr;
    }
    *buff_ptr = m;
}
extern "C" void ocl_create_read_buffer_(bigdft_context *, cl_uint *size, cl_mem *b) { create_buffer(size, b); }
extern "C" void ocl_create_write_buffer_(bigdft_context *, cl_uint *size, cl_mem *b) { create_buffer(size, b); }
extern "C" void ocl_create_read_write_buffer_(bigdft_context *, cl_uint *size, cl_mem *b) { create_buffer(size, b); }
extern "C" void ocl_create_read_buffer_and_copy_(bigdft_context *, cl_uint *size, void *host_ptr, cl_mem *b)
{
    create_buffer(size, b);
    if ((*b)->ptr && cudaMemcpy((*b)->ptr, host_ptr, *size, cudaMemcpyHostToDevice) != cudaSuccess)
        qerr(nullptr, WVLH_ERR_CUDA, "ocl_create_read_buffer_and_copy");
}
// Page-locked host ranges, process-wide (cudaHostRegister is): page-aligned
// [begin, end) ranges that never overlap, each with the number of live handles
// inside it.  A copy must stay inside one registration, so a handle's pages
// always lie in exactly one range: a request inside a range takes a reference
// on it, a request that overlaps none is registered as a new range, and a
// request that straddles ranges (two arrays sharing a page, or one array
// pinned piece by piece) merges them with it into one range after waiting for
// every queue, since the old ranges must be unlocked first.  Releasing a
// handle drops its reference; a range left without references stays locked
// until the next ocl_finish, which waits for every queue (copies queued before
// or after the release may still use the pages) and then unlocks it.
static inline uintptr_t page_down(uintptr_t a) { return a & ~(uintptr_t)4095; }
static inline uintptr_t page_up(uintptr_t a) { return (a + 4095) & ~(uintptr_t)4095; }

static void pin_acquire(wvlh_mem *m)
{
    const uintptr_t a = page_down((uintptr_t)m->host), b = page_up((uintptr_t)m->host + m->size);
    m->pin_lo = a;
    m->pin_hi = b;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto first = g_pins.upper_bound(a);
    if (first != g_pins.begin() && std::prev(first)->second.end > a) --first;
    auto last = first;
    int n = 0;
    while (last != g_pins.end() && last->first < b) {
        ++last;
        ++n;
    }
    if (n == 1 && first->first <= a && first->second.end >= b) {
        ++first->second.refs;  // inside one locked range
        return;
    }
    uintptr_t lo = a, hi = b;
    int refs = 0;
    if (n > 0) {
        // straddles locked ranges: unlock them once no queue can be using them
        lo = std::min(lo, first->first);
        for (auto it = first; it != last; ++it) {
            hi = std::max(hi, it->second.end);
            refs += it->second.refs;
        }
        for (wvlh_ocl_queue *q : g_queues) cudaStreamSynchronize(q->stream);
        for (auto it = first; it != last; ++it) cudaHostUnregister((void *)it->first);
        g_pins.erase(first, last);
    }
    const cudaError_t e = cudaHostRegister((void *)lo, hi - lo, cudaHostRegisterMapped | cudaHostRegisterPortable);
    if (e == cudaSuccess) {
        g_pins[lo] = PinRange{hi, refs + 1};
    } else {
        cudaGetLastError();  // pages locked by someone else (e.g. cudaMallocHost) or not lockable: copies stage
        m->pin_lo = m->pin_hi = 0;
    }
}

static void pin_release(wvlh_mem *m)
{
    if (m->pin_hi == 0) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pins.upper_bound(m->pin_lo);
    if (it != g_pins.begin()) {
        --it;
        if (it->first <= m->pin_lo && it->second.end >= m->pin_hi) --it->second.refs;
    }
    m->pin_lo = m->pin_hi = 0;
}

// unlock the ranges no handle references, after every queue has drained
static void pin_reap()
{
    std::unique_lock<std::mutex> lk(g_pin_mu);
    bool idle = false;
    for (auto &e : g_pins) idle |= e.second.refs == 0;
    if (!idle) return;
    for (wvlh_ocl_queue *q : g_queues) cudaStreamSynchronize(q->stream);
    for (auto it = g_pins.begin(); it != g_pins.end();) {
        if (it->second.refs == 0) {
            cudaHostUnregister((void *)it->first);
            it = g_pins.erase(it);
        } else {
            ++it;
        }
    }
}

extern "C" void ocl_release_mem_object_(cl_mem *buff_ptr)
{
    if (!buff_ptr || !*buff_ptr) return;
    wvlh_mem *m = *buff_ptr;
    if (!m->host) {
        if (m->ptr) cudaFree(m->ptr);
    } else {
        pin_release(m);
    }
    delete m;
    *buff_ptr = nullptr;
}

// A buffer over caller host memory (CL_MEM_USE_HOST_PTR): the range is
// page-locked, so queued copies between it and device buffers are DMA
// transfers, and kernels may read it at its (unified) address.
static void create_host_buffer(bigdft_context *context, cl_uint *size, void *host_ptr, cl_mem *buff_ptr)
{
    (void)context;
    wvlh_mem *m = new wvlh_mem();
    m->size = *size;
    m->host = host_ptr;
    m->ptr = host_ptr;
    *buff_ptr = m;
    if (host_ptr && m->size) pin_acquire(m);
}
extern "C" void ocl_create_read_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr, cl_mem *b)
{
    create_host_buffer(context, size, host_ptr, b);
}
extern "C" void ocl_create_write_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr, cl_mem *b)
{
    create_host_buffer(context, size, host_ptr, b);
}
extern "C" void ocl_create_read_write_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr,
                                                   cl_mem *b)
{
    create_host_buffer(context, size, host_ptr, b);
}

// Mapping a buffer makes its contents visible to the host once the commands
// queued before it are done.  A host buffer is the host memory itself, so a
// map orders nothing beyond the queue: the blocking forms wait for the queue,
// the asynchronous ones are queue-ordered no-ops, as is unmapping.
static void map_buffer(bigdft_command_queue *command_queue, bool blocking)
{
    bigdft_command_queue q = command_queue ? *command_queue : nullptr;
    if (q && blocking) QCK(q, cudaStreamSynchronize(q->stream));
}
extern "C" void ocl_map_read_buffer_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *) { map_buffer(q, true); }
extern "C" void ocl_map_write_buffer_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *) { map_buffer(q, true); }
extern "C" void ocl_map_read_write_buffer_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *)
{
    map_buffer(q, true);
}
extern "C" void ocl_map_read_buffer_async_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *)
{
    map_buffer(q, false);
}
extern "C" void ocl_map_write_buffer_async_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *)
{
    map_buffer(q, false);
}
extern "C" void ocl_map_read_write_buffer_async_(bigdft_command_queue *q, cl_mem *, cl_uint *, cl_uint *)
{
    map_buffer(q, false);
}
extern "C" void ocl_unmap_mem_object_(bigdft_command_queue *q, cl_mem *, void *) { map_buffer(q, false); }

// pin = a host buffer over the range, then a map (OpenCL_wrappers.c:424-505)
static void pin_buffer(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size, void *host_ptr,
                       cl_mem *buff_ptr, bool blocking)
{
    create_host_buffer(context, size, host_ptr, buff_ptr);
    map_buffer(command_queue, blocking);
}
extern "C" void ocl_pin_read_write_buffer_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h,
                                           cl_mem *b)
{
    pin_buffer(c, q, size, h, b, true);
}
extern "C" void ocl_pin_write_buffer_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h, cl_mem *b)
{
    pin_buffer(c, q, size, h, b, true);
}
extern "C" void ocl_pin_read_buffer_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h, cl_mem *b)
{
    pin_buffer(c, q, size, h, b, true);
}
extern "C" void ocl_pin_read_write_buffer_async_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h,
                                                 cl_mem *b)
{
    pin_buffer(c, q, size, h, b, false);
}
extern "C" void ocl_pin_write_buffer_async_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h,
                                            cl_mem *b)
{
    pin_buffer(c, q, size, h, b, false);
}
extern "C" void ocl_pin_read_buffer_async_(bigdft_context *c, bigdft_command_queue *q, cl_uint *size, void *h,
                                           cl_mem *b)
{
    pin_buffer(c, q, size, h, b, false);
}

static void resolve_pending(bigdft_command_queue q)
{
    for (auto &pr : q->pending) *pr.first = q->h_stage[pr.second];
    q->pending.clear();
    q->next_slot = 0;
}

extern "C" void ocl_finish_(bigdft_command_queue *command_queue)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaStreamSynchronize(q->stream));
    resolve_pending(q);
    pin_reap();
}
extern "C" void ocl_enqueue_barrier_(bigdft_command_queue *command_queue) { (void)command_queue; }

extern "C" void ocl_enqueue_write_buffer_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                          const void *host_ptr)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaMemcpyAsync((*buffer)->ptr, host_ptr, *size, cudaMemcpyDefault, q->stream));
    QCK(q, cudaStreamSynchronize(q->stream));
}
extern "C" void ocl_enqueue_write_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                                const void *host_ptr)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaMemcpyAsync((*buffer)->ptr, host_ptr, *size, cudaMemcpyDefault, q->stream));
}
extern "C" void ocl_enqueue_read_buffer_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                         void *host_ptr)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaMemcpyAsync(host_ptr, (*buffer)->ptr, *size, cudaMemcpyDefault, q->stream));
    QCK(q, cudaStreamSynchronize(q->stream));
    resolve_pending(q);
}
extern "C" void ocl_enqueue_read_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                               void *host_ptr)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaMemcpyAsync(host_ptr, (*buffer)->ptr, *size, cudaMemcpyDefault, q->stream));
}

extern "C" void ocl_clean_command_queue_(bigdft_command_queue *command_queue)
{
    bigdft_command_queue q = *command_queue;
    if (!q) return;
    cudaStreamSynchronize(q->stream);
    resolve_pending(q);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        g_queues.erase(std::remove(g_queues.begin(), g_queues.end(), q), g_queues.end());
    }
    cudaFree(q->d_work);
    cudaFreeHost(q->h_stage);
    cudaStreamDestroy(q->stream);
    delete q;
    *command_queue = nullptr;
}
extern "C" void ocl_clean_(bigdft_context *context)
{
    if (context && *context) {
        pin_reap();
        delete *context;
        *context = nullptr;
    }
}

// ---------------------------------------------------------------- reductions
// result of a device reduction: blocking copy to *out, or deferred to ocl_finish
static void reduce_out(bigdft_command_queue q, double *out, bool async)
{
    const int slot = q->next_slot;
    if (slot >= 64) {  // staging full: drain
        cudaStreamSynchronize(q->stream);
        resolve_pending(q);
    }
    const int s = q->next_slot++;
    double *dres = q->d_work + kDotParts + s;
    QCK(q, cudaMemcpyAsync(q->h_stage + s, dres, sizeof(double), cudaMemcpyDeviceToHost, q->stream));
    q->pending.push_back({out, s});
    if (!async) {
        QCK(q, cudaStreamSynchronize(q->stream));
        resolve_pending(q);
    }
}
static double *next_result(bigdft_command_queue q)
{
    if (q->next_slot >= 64) {
        cudaStreamSynchronize(q->stream);
        resolve_pending(q);
    }
    return q->d_work + kDotParts + q->next_slot;
}

static void dot_impl(bigdft_command_queue q, cl_uint n, const double *x, const double *y, double *out, bool async)
{
    if (n == 0) {
        *out = 0.0;
        return;
    }
    QCK(q, plain_dot(n, x, y, q->d_work, next_result(q), q->stream));
    reduce_out(q, out, async);
}

extern "C" void dot_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y, cl_mem *, cl_mem *,
                       cl_double *out)
{
    dot_impl(*command_queue, *n, D(x), D(y), out, false);
}
extern "C" void dot_d_async_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y, cl_mem *,
                             cl_mem *, cl_double *out)
{
    dot_impl(*command_queue, *n, D(x), D(y), out, true);
}
extern "C" void nrm2sq_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *in, cl_mem *, cl_mem *,
                          cl_double *out)
{
    dot_impl(*command_queue, *n, D(in), D(in), out, false);
}
extern "C" void axpy_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x, cl_mem *y,
                        cl_mem *z)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, plain_axpy(*n, *alpha, D(x), D(y), D(z), q->stream));
}
extern "C" void axpy_self_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x,
                             cl_mem *y)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, plain_axpy(*n, *alpha, D(x), D(y), D(y), q->stream));
}
extern "C" void scal_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x, cl_mem *y)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, plain_scal(*n, *alpha, D(x), D(y), q->stream));
}
extern "C" void scal_self_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, plain_scal(*n, *alpha, D(x), D(x), q->stream));
}
extern "C" void copy_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, cudaMemcpyAsync(D(y), D(x), sizeof(double) * (size_t)*n, cudaMemcpyDeviceToDevice, q->stream));
}
extern "C" void set_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *value, cl_mem *x)
{
    bigdft_command_queue q = *command_queue;
    QCK(q, plain_set(*n, *value, D(x), q->stream));
}

// ---------------------------------------------------------------- (un)compress
static void prec_scal(const double *h, double c, double *scal)
{
    // GPUscal0..7 of OpenCL/Uncompress.c:380-470, h = hgrid/2
    double hh[3];
    for (int d = 0; d < 3; ++d) hh[d] = 0.125 / (h[d] * h[d]);
    for (int k = 0; k < 8; ++k) {
        double s = c;
        s += ((k & 1) ? WVL_B2 : WVL_A2) * hh[0];
        s += ((k & 2) ? WVL_B2 : WVL_A2) * hh[1];
        s += ((k & 4) ? WVL_B2 : WVL_A2) * hh[2];
        scal[k] = 1.0 / sqrt(s);
    }
}

static void uncompress_impl(bigdft_command_queue q, int dir, cl_uint *dimensions, cl_uint *nseg_c, cl_uint *nvctr_c,
                            cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                            cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psig, const double *scal)
{
    const int dims[3] = {(int)dimensions[0], (int)dimensions[1], (int)dimensions[2]};
    const int nvf = (int)*nvctr_f;
    QCK(q, plain_uncompress(dir, dims, (int)*nseg_c, (int)*nvctr_c, U(keyg_c), U(keyv_c), (int)*nseg_f, nvf,
                            nvf ? U(keyg_f) : nullptr, nvf ? U(keyv_f) : nullptr, D(psi_c), nvf ? D(psi_f) : nullptr,
                            D(psig), scal, 1, 0, 0, 0, q->stream));
}

extern "C" void uncompress_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *nseg_c, cl_uint *nvctr_c,
                              cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                              cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi_out)
{
    uncompress_impl(*cq, 0, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c,
                    psi_f, psi_out, nullptr);
}
extern "C" void compress_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *nseg_c, cl_uint *nvctr_c,
                            cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                            cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi)
{
    uncompress_impl(*cq, 1, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c,
                    psi_f, psi, nullptr);
}
extern "C" void uncompress_scale_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_double *h, cl_double *c,
                                    cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c,
                                    cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f,
                                    cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi_out)
{
    double s[8];
    prec_scal(h, *c, s);
    uncompress_impl(*cq, 0, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c,
                    psi_f, psi_out, s);
}
extern "C" void compress_scale_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_double *h, cl_double *c,
                                  cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                                  cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                                  cl_mem *psi)
{
    double s[8];
    prec_scal(h, *c, s);
    uncompress_impl(*cq, 1, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c,
                    psi_f, psi, s);
}

extern "C" void scale_psi_d_(bigdft_command_queue *cq, cl_uint *nvctr_c, cl_uint *nvctr_f, cl_double *h,
                             cl_double *c, cl_mem *psi_c, cl_mem *psi_f)
{
    bigdft_command_queue q = *cq;
    double s[8];
    prec_scal(h, *c, s);
    QCK(q, plain_scal(*nvctr_c, s[0], D(psi_c), D(psi_c), q->stream));
    if (*nvctr_f) QCK(q, plain_scale7(*nvctr_f, s + 1, D(psi_f), q->stream));
}

// ---------------------------------------------------------------- 1D passes
extern "C" void syn1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_syn1d(*n, *ndat, 1, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void syngrow1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_syn1d(*n, *ndat, 0, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void ana1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_ana1d(*n, *ndat, 1, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void anashrink1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_ana1d(*n, *ndat, 0, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void magicfilter1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_mf1d(0, *n, *ndat, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void magicfiltergrow1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_mf1d(2, *n, *ndat, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void magicfilter1d_t_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out)
{
    QCK(*cq, plain_mf1d(1, *n, *ndat, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
extern "C" void magicfiltershrink1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi,
                                       cl_mem *out)
{
    QCK(*cq, plain_mf1d(3, *n, *ndat, D(psi), D(out), 1, 0, 0, (*cq)->stream));
}
// MF pass followed by multiplication with the potential (rotated output)
extern "C" void magicfilter1d_pot_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *pot,
                                     cl_mem *out)
{
    bigdft_command_queue q = *cq;
    QCK(q, plain_mf1d(0, *n, *ndat, D(psi), D(out), 1, 0, 0, q->stream));
    QCK(q, plain_potential((size_t)*n * *ndat, D(pot), D(out), q->d_work, 64, nullptr, q->stream));
}
extern "C" void kinetic1d_d_(bigdft_command_queue *cq, cl_uint *n, cl_uint *ndat, cl_double *h, cl_double *c,
                             cl_mem *x, cl_mem *y, cl_mem *workx, cl_mem *worky, cl_double *ekin)
{
    // Kinetic.c:288-294: worky = c*x, then y = worky + scale*K x (rotated), ekin = 0
    bigdft_command_queue q = *cq;
    const size_t ng = (size_t)*n * *ndat;
    QCK(q, plain_scal(ng, *c, D(x), D(worky), q->stream));
    QCK(q, plain_kin1d(*n, *ndat, 1, -0.5 / (*h * *h), D(x), D(workx), D(worky), D(y), 1, 0, 0, q->stream));
    *ekin = 0.0;
}

// ---------------------------------------------------------------- 3D operators
struct Dim3 {
    int N[3], per[3], F[3], I[3];
};
static Dim3 dims3(const cl_uint *dimensions, const cl_uint *periodic)
{
    Dim3 d;
    for (int k = 0; k < 3; ++k) {
        d.N[k] = (int)dimensions[k];
        d.per[k] = periodic ? (periodic[k] ? 1 : 0) : 1;
        d.F[k] = fine_len(d.N[k], d.per[k]);
        d.I[k] = isf_len(d.N[k], d.per[k]);
    }
    return d;
}

// MF over z, y, x: in -> t1 -> t2 -> out (MagicFilter.c:396-424)
static cudaError_t mf3(const Dim3 &d, const double *in, double *t1, double *t2, double *out, cudaStream_t st)
{
    cudaError_t e;
    if ((e = plain_mf1d(d.per[2] ? 0 : 2, d.F[2], d.F[0] * d.F[1], in, t1, 1, 0, 0, st))) return e;
    if ((e = plain_mf1d(d.per[1] ? 0 : 2, d.F[1], d.F[0] * d.I[2], t1, t2, 1, 0, 0, st))) return e;
    return plain_mf1d(d.per[0] ? 0 : 2, d.F[0], d.I[2] * d.I[1], t2, out, 1, 0, 0, st);
}
// MF^T over z, y, x: in -> t1 -> t2 -> out
static cudaError_t mft3(const Dim3 &d, const double *in, double *t1, double *t2, double *out, cudaStream_t st)
{
    cudaError_t e;
    if ((e = plain_mf1d(d.per[2] ? 1 : 3, d.F[2], d.I[0] * d.I[1], in, t1, 1, 0, 0, st))) return e;
    if ((e = plain_mf1d(d.per[1] ? 1 : 3, d.F[1], d.I[0] * d.F[2], t1, t2, 1, 0, 0, st))) return e;
    return plain_mf1d(d.per[0] ? 1 : 3, d.F[0], d.F[2] * d.F[1], t2, out, 1, 0, 0, st);
}

extern "C" void syn_self_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_mem *psi,
                                    cl_mem *out)
{
    // z: psi -> out, y: out -> psi, x: psi -> out
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, plain_syn1d(d.N[2], 4 * d.N[0] * d.N[1], d.per[2], D(psi), D(out), 1, 0, 0, q->stream));
    QCK(q, plain_syn1d(d.N[1], 2 * d.N[0] * d.F[2], d.per[1], D(out), D(psi), 1, 0, 0, q->stream));
    QCK(q, plain_syn1d(d.N[0], d.F[2] * d.F[1], d.per[0], D(psi), D(out), 1, 0, 0, q->stream));
}
extern "C" void syn_self_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_mem *psi, cl_mem *out)
{
    syn_self_d_generic_(cq, dimensions, nullptr, psi, out);
}
extern "C" void syn_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_mem *tmp,
                               cl_mem *psi, cl_mem *out)
{
    // z: psi -> out, y: out -> tmp, x: tmp -> out (psi preserved)
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, plain_syn1d(d.N[2], 4 * d.N[0] * d.N[1], d.per[2], D(psi), D(out), 1, 0, 0, q->stream));
    QCK(q, plain_syn1d(d.N[1], 2 * d.N[0] * d.F[2], d.per[1], D(out), D(tmp), 1, 0, 0, q->stream));
    QCK(q, plain_syn1d(d.N[0], d.F[2] * d.F[1], d.per[0], D(tmp), D(out), 1, 0, 0, q->stream));
}
extern "C" void ana_self_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_mem *psi,
                                    cl_mem *out)
{
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, plain_ana1d(d.N[2], d.F[0] * d.F[1], d.per[2], D(psi), D(out), 1, 0, 0, q->stream));
    QCK(q, plain_ana1d(d.N[1], d.F[0] * 2 * d.N[2], d.per[1], D(out), D(psi), 1, 0, 0, q->stream));
    QCK(q, plain_ana1d(d.N[0], 4 * d.N[2] * d.N[1], d.per[0], D(psi), D(out), 1, 0, 0, q->stream));
}
extern "C" void ana_self_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_mem *psi, cl_mem *out)
{
    ana_self_d_generic_(cq, dimensions, nullptr, psi, out);
}
extern "C" void ana_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_mem *tmp,
                               cl_mem *psi, cl_mem *out)
{
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, plain_ana1d(d.N[2], d.F[0] * d.F[1], d.per[2], D(psi), D(out), 1, 0, 0, q->stream));
    QCK(q, plain_ana1d(d.N[1], d.F[0] * 2 * d.N[2], d.per[1], D(out), D(tmp), 1, 0, 0, q->stream));
    QCK(q, plain_ana1d(d.N[0], 4 * d.N[2] * d.N[1], d.per[0], D(tmp), D(out), 1, 0, 0, q->stream));
}
extern "C" void magic_filter_3d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                         cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out)
{
    const Dim3 d = dims3(dimensions, periodic);
    QCK(*cq, mf3(d, D(psi), D(tmp), D(tmp_dot), D(out), (*cq)->stream));
}
extern "C" void magic_filter_t_3d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                           cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out)
{
    const Dim3 d = dims3(dimensions, periodic);
    QCK(*cq, mft3(d, D(psi), D(tmp), D(tmp_dot), D(out), (*cq)->stream));
}
extern "C" void potential_application_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                                 cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out, cl_mem *pot,
                                                 cl_double *epot)
{
    // MF: psi -> tmp -> out -> tmp; V: tmp; MF^T: tmp -> out -> tmp -> out;
    // epot = <psi|out> (MagicFilter.c:327-383)
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, mf3(d, D(psi), D(tmp), D(out), D(tmp), q->stream));
    const size_t ni = (size_t)d.I[0] * d.I[1] * d.I[2];
    QCK(q, plain_potential(ni, D(pot), D(tmp), q->d_work, 64, nullptr, q->stream));
    QCK(q, mft3(d, D(tmp), D(out), D(tmp_dot), D(out), q->stream));
    dot_impl(q, (cl_uint)((size_t)d.F[0] * d.F[1] * d.F[2]), D(psi), D(out), epot, true);
}
extern "C" void kinetic_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_double *h,
                                   cl_mem *x, cl_mem *y, cl_mem *work_x, cl_mem *work_y)
{
    // Kinetic.c:240-270: (x,y) -> (work_x,work_y) -> (x,y) -> (work_x,work_y)
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    const int F1 = d.F[0], F2 = d.F[1], F3 = d.F[2];
    QCK(q, plain_kin1d(F3, F1 * F2, d.per[2], -0.5 / (h[2] * h[2]), D(x), D(work_x), D(y), D(work_y), 1, 0, 0,
                       q->stream));
    QCK(q, plain_kin1d(F2, F1 * F3, d.per[1], -0.5 / (h[1] * h[1]), D(work_x), D(x), D(work_y), D(y), 1, 0, 0,
                       q->stream));
    QCK(q, plain_kin1d(F1, F2 * F3, d.per[0], -0.5 / (h[0] * h[0]), D(x), D(work_x), D(y), D(work_y), 1, 0, 0,
                       q->stream));
}
extern "C" void kinetic_d_(bigdft_command_queue *cq, cl_uint *dimensions, cl_double *h, cl_mem *x, cl_mem *y,
                           cl_mem *work_x, cl_mem *work_y)
{
    kinetic_d_generic_(cq, dimensions, nullptr, h, x, y, work_x, work_y);
}
extern "C" void magicfilter_den_d_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                           cl_mem *tmp, cl_mem *psi, cl_mem *out)
{
    // MF: psi -> out -> tmp -> out, then squared (MagicFilter.c:209-245)
    const Dim3 d = dims3(dimensions, periodic);
    bigdft_command_queue q = *cq;
    QCK(q, mf3(d, D(psi), D(out), D(tmp), D(out), q->stream));
    const size_t ni = (size_t)d.I[0] * d.I[1] * d.I[2];
    QCK(q, plain_square(ni, D(out), q->stream));
}

// ---------------------------------------------------------------- compositions
extern "C" void ocl_fulllocham_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                        cl_double *h, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c,
                                        cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                                        cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *pot, cl_mem *psi,
                                        cl_mem *out, cl_mem *work, cl_mem *kinres, cl_double *epot,
                                        cl_double *ekinpot)
{
    // Hamiltonian.c:41-72
    uncompress_d_(cq, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c, psi_f,
                  out);
    syn_self_d_generic_(cq, dimensions, periodic, out, psi);
    potential_application_d_generic_(cq, dimensions, periodic, work, kinres, psi, out, pot, epot);
    kinetic_d_generic_(cq, dimensions, periodic, h, psi, out, work, kinres);
    const Dim3 d = dims3(dimensions, periodic);
    cl_uint ndat = (cl_uint)((size_t)d.F[0] * d.F[1] * d.F[2]);
    dot_d_async_(cq, &ndat, work, kinres, psi, out, ekinpot);
    ana_self_d_generic_(cq, dimensions, periodic, kinres, psi);
    compress_d_(cq, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c, psi_f, psi);
}

extern "C" void ocl_fulllocham_generic_k_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                          cl_double *h, cl_double *k, cl_uint *nseg_c, cl_uint *nvctr_c,
                                          cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f,
                                          cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c_r, cl_mem *psi_f_r,
                                          cl_mem *psi_c_i, cl_mem *psi_f_i, cl_mem *pot, cl_mem *psi_r,
                                          cl_mem *out_r, cl_mem *work_r, cl_mem *psi_i, cl_mem *out_i,
                                          cl_mem *work_i, cl_mem *kinres_r, cl_mem *kinres_i, cl_uint *nspinor,
                                          cl_double *epot, cl_double *ekinpot)
{
    // Hamiltonian.c:105-172, Gamma point only
    (void)k;
    (void)psi_c_i;
    (void)psi_f_i;
    (void)psi_i;
    (void)out_i;
    (void)work_i;
    (void)kinres_i;
    if (*nspinor != 1) {
        qerr(*cq, WVLH_ERR_UNSUPPORTED, "ocl_fulllocham_generic_k");
        return;
    }
    epot[1] = 0.0;
    ekinpot[1] = 0.0;
    ocl_fulllocham_generic_(cq, dimensions, periodic, h, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f,
                            keyv_f, psi_c_r, psi_f_r, pot, psi_r, out_r, work_r, kinres_r, &epot[0], &ekinpot[0]);
}

extern "C" void ocl_daub_to_isf_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_uint *nseg_c,
                                 cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f,
                                 cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi,
                                 cl_mem *out, cl_mem *work, cl_mem *kinres)
{
    // Hamiltonian.c:89-103
    uncompress_d_(cq, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c, psi_f,
                  out);
    syn_self_d_generic_(cq, dimensions, periodic, out, psi);
    magic_filter_3d_generic_(cq, dimensions, periodic, work, kinres, psi, out);
}

extern "C" void ocl_isf_to_daub_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_uint *nseg_c,
                                 cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f,
                                 cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi,
                                 cl_mem *out, cl_mem *work, cl_mem *kinres)
{
    // Hamiltonian.c:74-87
    magic_filter_t_3d_generic_(cq, dimensions, periodic, work, kinres, psi, out);
    ana_self_d_generic_(cq, dimensions, periodic, out, psi);
    compress_d_(cq, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c, psi_f, psi);
}

extern "C" void ocl_locden_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                    cl_double *hfac, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c,
                                    cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                                    cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi, cl_mem *out,
                                    cl_mem *work, cl_mem *pot)
{
    // Density.c:37-55: pot (the density) += hfac * (MF^3 syn^3 psi)^2
    uncompress_d_(cq, dimensions, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f, psi_c, psi_f,
                  out);
    syn_self_d_generic_(cq, dimensions, periodic, out, psi);
    magicfilter_den_d_generic_(cq, dimensions, periodic, work, psi, out);
    const Dim3 d = dims3(dimensions, periodic);
    cl_uint ndat = (cl_uint)((size_t)d.I[0] * d.I[1] * d.I[2]);
    axpy_self_d_(cq, &ndat, hfac, out, pot);
}

static void apply_hp_generic(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, double *h, double *c,
                             cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                             cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                             cl_mem *psi_c_out, cl_mem *psi_f_out, cl_mem *psi, cl_mem *out, cl_mem *work,
                             cl_mem *kinres)
{
    // Preconditioner.c:98-128
    uncompress_scale_d_(cq, dimensions, h, c, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f,
                        psi_c, psi_f, out);
    syn_self_d_generic_(cq, dimensions, periodic, out, psi);
    const Dim3 d = dims3(dimensions, periodic);
    cl_uint n = (cl_uint)((size_t)d.F[0] * d.F[1] * d.F[2]);
    scal_d_(cq, &n, c, psi, out);
    kinetic_d_generic_(cq, dimensions, periodic, h, psi, out, work, kinres);
    ana_self_d_generic_(cq, dimensions, periodic, kinres, out);
    compress_scale_d_(cq, dimensions, h, c, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f,
                      psi_c_out, psi_f_out, out);
}

static void precond_cg(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, double *h, double *c,
                       cl_uint *ncong, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c,
                       cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c,
                       cl_mem *psi_f, cl_mem *psi_c_r, cl_mem *psi_f_r, cl_mem *psi_c_b, cl_mem *psi_f_b,
                       cl_mem *psi_c_d, cl_mem *psi_f_d, cl_mem *work1, cl_mem *work2, cl_mem *work3, cl_mem *work4,
                       double *norm_sq_cf)
{
    // Preconditioner.c:130-195 (CG on the scaled system, x0 = psi)
    cl_uint nvctr_f_7 = (*nvctr_f) * 7;
    apply_hp_generic(cq, dimensions, periodic, h, c, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f,
                     psi_c, psi_f, psi_c_d, psi_f_d, work1, work2, work3, work4);
    double alpha, beta, val = -1.0;
    axpy_d_(cq, nvctr_c, &val, psi_c_d, psi_c_b, psi_c_r);
    axpy_d_(cq, &nvctr_f_7, &val, psi_f_d, psi_f_b, psi_f_r);
    copy_d_(cq, nvctr_c, psi_c_r, psi_c_d);
    copy_d_(cq, &nvctr_f_7, psi_f_r, psi_f_d);
    double nc = 0.0, nf = 0.0;
    nrm2sq_d_(cq, nvctr_c, psi_c_r, work1, work2, &nc);
    nrm2sq_d_(cq, &nvctr_f_7, psi_f_r, work1, work2, &nf);
    double norm_sq = nc + nf;
    for (cl_uint i = 0; i < *ncong; ++i) {
        apply_hp_generic(cq, dimensions, periodic, h, c, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f,
                         keyv_f, psi_c_d, psi_f_d, psi_c_b, psi_f_b, work1, work2, work3, work4);
        dot_d_(cq, nvctr_c, psi_c_d, psi_c_b, work1, work2, &nc);
        dot_d_(cq, &nvctr_f_7, psi_f_d, psi_f_b, work1, work2, &nf);
        alpha = norm_sq / (nc + nf);
        val = alpha;
        axpy_self_d_(cq, nvctr_c, &val, psi_c_d, psi_c);
        axpy_self_d_(cq, &nvctr_f_7, &val, psi_f_d, psi_f);
        if (i != *ncong - 1) {
            val = -alpha;
            axpy_self_d_(cq, nvctr_c, &val, psi_c_b, psi_c_r);
            axpy_self_d_(cq, &nvctr_f_7, &val, psi_f_b, psi_f_r);
            nrm2sq_d_(cq, nvctr_c, psi_c_r, work1, work2, &nc);
            nrm2sq_d_(cq, &nvctr_f_7, psi_f_r, work1, work2, &nf);
            beta = (nc + nf) / norm_sq;
            val = beta;
            axpy_d_(cq, nvctr_c, &val, psi_c_d, psi_c_r, psi_c_d);
            axpy_d_(cq, &nvctr_f_7, &val, psi_f_d, psi_f_r, psi_f_d);
            norm_sq = nc + nf;
        }
    }
    if (norm_sq_cf) {
        norm_sq_cf[0] = nc;
        norm_sq_cf[1] = nf;
    }
    scale_psi_d_(cq, nvctr_c, nvctr_f, h, c, psi_c, psi_f);
}

extern "C" void ocl_preconditioner_generic_(bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic,
                                            cl_double *h, cl_double *c, cl_uint *ncong, cl_uint *nseg_c,
                                            cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                                            cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c,
                                            cl_mem *psi_f, cl_mem *psi_c_r, cl_mem *psi_f_r, cl_mem *psi_c_b,
                                            cl_mem *psi_f_b, cl_mem *psi_c_d, cl_mem *psi_f_d, cl_mem *work1,
                                            cl_mem *work2, cl_mem *work3, cl_mem *work4)
{
    precond_cg(cq, dimensions, periodic, h, c, ncong, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f,
               psi_c, psi_f, psi_c_r, psi_f_r, psi_c_b, psi_f_b, psi_c_d, psi_f_d, work1, work2, work3, work4,
               nullptr);
}

extern "C" void ocl_preconditioner_generic_k_(
    bigdft_command_queue *cq, cl_uint *dimensions, cl_uint *periodic, cl_double *h, cl_double *k, cl_double *c,
    cl_uint *ncong, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
    cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c_r, cl_mem *psi_f_r, cl_mem *psi_c_i,
    cl_mem *psi_f_i, cl_mem *psi_c_r_r, cl_mem *psi_f_r_r, cl_mem *psi_c_r_i, cl_mem *psi_f_r_i, cl_mem *psi_c_b_r,
    cl_mem *psi_f_b_r, cl_mem *psi_c_b_i, cl_mem *psi_f_b_i, cl_mem *psi_c_d_r, cl_mem *psi_f_d_r, cl_mem *psi_c_d_i,
    cl_mem *psi_f_d_i, cl_mem *work1_r, cl_mem *work2_r, cl_mem *work3_r, cl_mem *work4_r, cl_mem *work1_i,
    cl_mem *work2_i, cl_mem *work3_i, cl_mem *work4_i, cl_uint *nspinor, cl_double *norm_sq_cf)
{
    // Preconditioner.c:247-360, Gamma point only
    (void)k;
    (void)psi_c_i, (void)psi_f_i, (void)psi_c_r_i, (void)psi_f_r_i, (void)psi_c_b_i, (void)psi_f_b_i;
    (void)psi_c_d_i, (void)psi_f_d_i, (void)work1_i, (void)work2_i, (void)work3_i, (void)work4_i;
    if (*nspinor != 1) {
        qerr(*cq, WVLH_ERR_UNSUPPORTED, "ocl_preconditioner_generic_k");
        return;
    }
    precond_cg(cq, dimensions, periodic, h, c, ncong, nseg_c, nvctr_c, keyg_c, keyv_c, nseg_f, nvctr_f, keyg_f, keyv_f,
               psi_c_r, psi_f_r, psi_c_r_r, psi_f_r_r, psi_c_b_r, psi_f_b_r, psi_c_d_r, psi_f_d_r, work1_r, work2_r,
               work3_r, work4_r, norm_sq_cf);
}
