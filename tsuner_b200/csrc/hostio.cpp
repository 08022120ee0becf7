// Host worker pool and pinned staging pipelines for the C ABI's bulk copies
// (declarations and rationale in hostio.h).
#include "hostio.h"

#include <cstdio>

#include <pthread.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "tsuner_b200.h"

// solver.cu: detail text returned by tsu_last_error() on this thread
void tsu_set_error_detail(const char *text);

namespace tsu {
namespace {

// ------------------------------------------------------------------ pool
// One job at a time.  A worker joins a job when it sees a new generation,
// counts itself active under the lock and takes indices from `next` until
// they run out; the caller sets up the next job only when no worker is
// active, so a worker never mixes two jobs' indices.
class Pool {
   public:
    explicit Pool(int nthreads) {
        for (int i = 0; i < nthreads - 1; i++) std::thread([this] { worker(); }).detach();
        size_ = nthreads;
    }
    int size() const { return size_; }

    void run(int n, const std::function<void(int)> &fn) {
        std::lock_guard<std::mutex> call(call_m_);
        {
            std::unique_lock<std::mutex> lk(m_);
            done_cv_.wait(lk, [&] { return active_ == 0; });
            job_ = &fn;
            njobs_ = n;
            next_.store(0);
            remaining_.store(n);
            gen_++;
        }
        cv_.notify_all();
        drain(&fn, n);
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [&] { return remaining_.load() == 0 && active_ == 0; });
        job_ = nullptr;
    }

   private:
    void drain(const std::function<void(int)> *fn, int n) {
        for (int i; (i = next_.fetch_add(1)) < n;) {
            (*fn)(i);
            if (remaining_.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> lk(m_);
                done_cv_.notify_all();
            }
        }
    }

    void worker() {
        unsigned seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen && job_ != nullptr; });
            seen = gen_;
            const std::function<void(int)> *fn = job_;
            int n = njobs_;
            active_++;
            lk.unlock();
            drain(fn, n);
            lk.lock();
            if (--active_ == 0) done_cv_.notify_all();
        }
    }

    std::mutex call_m_, m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int njobs_ = 0, active_ = 0, size_ = 1;
    unsigned gen_ = 0;
    std::atomic<int> next_{0}, remaining_{0};
};

std::mutex g_pool_m;
Pool *g_pool = nullptr;  // never destroyed: detached workers may outlive static destructors

// A forked child has none of the parent's worker threads (nor a usable CUDA
// context); it drops the pointer so that it builds its own pool.  The pool
// mutex is held across fork() so the child never inherits it locked by a
// thread it does not have.
void before_fork() { g_pool_m.lock(); }
void after_fork_parent() { g_pool_m.unlock(); }
void after_fork_child() {
    g_pool = nullptr;
    g_pool_m.unlock();
}

int want_threads() {
    if (const char *e = getenv("TSU_HOST_THREADS")) {
        int n = atoi(e);
        if (n >= 1) return std::min(n, 256);
    }
    unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hw ? hw : 1u, 16u));
}

Pool &pool() {
    static const int registered = pthread_atfork(before_fork, after_fork_parent, after_fork_child);
    (void)registered;
    std::lock_guard<std::mutex> lk(g_pool_m);
    if (!g_pool) g_pool = new Pool(want_threads());
    return *g_pool;
}

// ------------------------------------------------------------------ staging
constexpr size_t kChunk = 16u << 20;  // bytes per pinned chunk
constexpr int kBufs = 4;              // chunks in flight
constexpr size_t kDirect = 1u << 20;  // smaller copies go straight to the driver
constexpr size_t kPart = 256u << 10;  // least bytes a worker is handed

std::mutex g_stage_m;  // one staged copy at a time (the chunks are shared)
unsigned char *g_pin[kBufs] = {};
bool g_pin_failed = false;

bool staging_ready() {
    if (g_pin[0]) return true;
    if (g_pin_failed) return false;
    for (int b = 0; b < kBufs; b++) {
        if (cudaHostAlloc((void **)&g_pin[b], kChunk, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            for (int k = 0; k < b; k++) cudaFreeHost(g_pin[k]);
            for (int k = 0; k < kBufs; k++) g_pin[k] = nullptr;
            g_pin_failed = true;  // keep using the driver's own pageable path
            return false;
        }
    }
    return true;
}

bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Copies nr rows between a packed buffer (rows of `width` bytes) and a
// pitched one, split over the pool.  to_packed: pitched -> packed.
void rows_copy(unsigned char *packed, unsigned char *pitched, size_t pitch, size_t width, size_t nr,
               bool to_packed) {
    const size_t bytes = width * nr;
    if (pitch == width) {  // one flat range: split by bytes
        int parts = (int)std::min<size_t>((size_t)pool().size(), std::max<size_t>(1, bytes / kPart));
        host_parallel(parts, [&](int p) {
            size_t a = bytes * p / parts, b = bytes * (p + 1) / parts;
            if (to_packed)
                memcpy(packed + a, pitched + a, b - a);
            else
                memcpy(pitched + a, packed + a, b - a);
        });
        return;
    }
    int parts = (int)std::min<size_t>({(size_t)pool().size(), nr, std::max<size_t>(1, bytes / kPart)});
    host_parallel(parts, [&](int p) {
        size_t a = nr * p / parts, b = nr * (p + 1) / parts;
        for (size_t r = a; r < b; r++) {
            if (to_packed)
                memcpy(packed + r * width, pitched + r * pitch, width);
            else
                memcpy(pitched + r * pitch, packed + r * width, width);
        }
    });
}

struct Events {
    cudaEvent_t ev[kBufs] = {};
    cudaError_t make() {
        for (int b = 0; b < kBufs; b++) {
            cudaError_t e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    ~Events() {
        for (int b = 0; b < kBufs; b++)
            if (ev[b]) cudaEventDestroy(ev[b]);
    }
};

// Ends a staged copy: whatever happened, no DMA may still target the shared
// chunks when the next copy starts.
cudaError_t finish(cudaError_t e, cudaStream_t st) {
    cudaError_t s = cudaStreamSynchronize(st);
    return e != cudaSuccess ? e : s;
}

}  // namespace

int host_threads() { return pool().size(); }

void host_parallel(int n, const std::function<void(int)> &fn) {
    if (n <= 0) return;
    if (n == 1) {
        fn(0);
        return;
    }
    pool().run(n, fn);
}

cudaError_t planes_h2d(int nplanes, void *const *dev, size_t dpitch, const void *const *host, size_t hpitch,
                       size_t width, size_t rows, cudaStream_t st, const RowFill &fill) {
    if (nplanes <= 0 || rows == 0 || width == 0) return cudaSuccess;
    const size_t total = width * rows * nplanes;
    bool direct = !fill && (total < kDirect || width > kChunk);
    if (!direct && !fill) {
        direct = true;  // every source plane already pinned: the DMA engine reads them itself
        for (int p = 0; p < nplanes && direct; p++) direct = is_pinned(host[p]);
    }
    if (direct) {
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < nplanes && e == cudaSuccess; p++)
            e = cudaMemcpy2DAsync(dev[p], dpitch, host[p], hpitch, width, rows, cudaMemcpyHostToDevice, st);
        return finish(e, st);
    }
    std::lock_guard<std::mutex> lk(g_stage_m);
    if (!staging_ready() || width > kChunk) {
        if (fill) {  // no staging chunks: fill a temporary buffer plane by plane
            std::vector<unsigned char> tmp;
            try {
                tmp.resize(width * rows);
            } catch (...) {
                return cudaErrorMemoryAllocation;
            }
            cudaError_t e = cudaSuccess;
            for (int p = 0; p < nplanes && e == cudaSuccess; p++) {
                fill(p, 0, rows, tmp.data());
                e = cudaMemcpy2DAsync(dev[p], dpitch, tmp.data(), width, width, rows, cudaMemcpyHostToDevice, st);
                e = finish(e, st);
            }
            return e;
        }
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < nplanes && e == cudaSuccess; p++)
            e = cudaMemcpy2DAsync(dev[p], dpitch, host[p], hpitch, width, rows, cudaMemcpyHostToDevice, st);
        return finish(e, st);
    }
    Events ev;
    cudaError_t e = ev.make();
    if (e != cudaSuccess) return e;
    const size_t R = std::max<size_t>(1, kChunk / width);
    const size_t per = (rows + R - 1) / R;
    const size_t nchunks = per * nplanes;
    for (size_t c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int p = (int)(c / per), b = (int)(c % kBufs);
        const size_t r0 = (c % per) * R, nr = std::min(R, rows - r0);
        if (c >= (size_t)kBufs && (e = cudaEventSynchronize(ev.ev[b])) != cudaSuccess) break;
        if (fill) {
            int parts = (int)std::min<size_t>({(size_t)pool().size(), nr, std::max<size_t>(1, width * nr / kPart)});
            host_parallel(parts, [&](int q) {
                size_t a = nr * q / parts, z = nr * (q + 1) / parts;
                if (z > a) fill(p, r0 + a, z - a, g_pin[b] + a * width);
            });
        } else {
            rows_copy(g_pin[b], (unsigned char *)host[p] + r0 * hpitch, hpitch, width, nr, true);
        }
        e = cudaMemcpy2DAsync((unsigned char *)dev[p] + r0 * dpitch, dpitch, g_pin[b], width, width, nr,
                              cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev.ev[b], st);
    }
    return finish(e, st);
}

cudaError_t planes_d2h(int nplanes, void *const *host, size_t hpitch, const void *const *dev, size_t dpitch,
                       size_t width, size_t rows, cudaStream_t st) {
    if (nplanes <= 0 || rows == 0 || width == 0) return cudaSuccess;
    const size_t total = width * rows * nplanes;
    bool direct = total < kDirect || width > kChunk;
    if (!direct) {
        direct = true;  // every destination plane already pinned
        for (int p = 0; p < nplanes && direct; p++) direct = is_pinned(host[p]);
    }
    std::unique_lock<std::mutex> lk(g_stage_m, std::defer_lock);
    if (!direct) {
        lk.lock();
        direct = !staging_ready();
    }
    if (direct) {
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < nplanes && e == cudaSuccess; p++)
            e = cudaMemcpy2DAsync(host[p], hpitch, dev[p], dpitch, width, rows, cudaMemcpyDeviceToHost, st);
        return finish(e, st);
    }
    Events ev;
    cudaError_t e = ev.make();
    if (e != cudaSuccess) return e;
    const size_t R = std::max<size_t>(1, kChunk / width);
    const size_t per = (rows + R - 1) / R;
    const size_t nchunks = per * nplanes;
    auto issue = [&](size_t c) {
        const int p = (int)(c / per), b = (int)(c % kBufs);
        const size_t r0 = (c % per) * R, nr = std::min(R, rows - r0);
        cudaError_t r = cudaMemcpy2DAsync(g_pin[b], width, (const unsigned char *)dev[p] + r0 * dpitch, dpitch,
                                          width, nr, cudaMemcpyDeviceToHost, st);
        return r == cudaSuccess ? cudaEventRecord(ev.ev[b], st) : r;
    };
    for (size_t c = 0; c < std::min<size_t>(kBufs, nchunks) && e == cudaSuccess; c++) e = issue(c);
    for (size_t c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int p = (int)(c / per), b = (int)(c % kBufs);
        const size_t r0 = (c % per) * R, nr = std::min(R, rows - r0);
        if ((e = cudaEventSynchronize(ev.ev[b])) != cudaSuccess) break;
        rows_copy(g_pin[b], (unsigned char *)host[p] + r0 * hpitch, hpitch, width, nr, false);
        if (c + kBufs < nchunks) e = issue(c + kBufs);
    }
    return finish(e, st);
}

// A flat range is moved as rows of kRow bytes plus a short tail.
static constexpr size_t kRow = 64u << 10;

cudaError_t bytes_h2d(void *dev, const void *host, size_t bytes, cudaStream_t st) {
    const size_t rows = bytes / kRow, tail = bytes - rows * kRow;
    cudaError_t e = cudaSuccess;
    if (rows) {
        void *d[1] = {dev};
        const void *h[1] = {host};
        e = planes_h2d(1, d, kRow, h, kRow, kRow, rows, st);
    }
    if (e == cudaSuccess && tail)
        e = finish(cudaMemcpyAsync((unsigned char *)dev + rows * kRow, (const unsigned char *)host + rows * kRow, tail,
                                   cudaMemcpyHostToDevice, st),
                   st);
    return e;
}

cudaError_t bytes_d2h(void *host, const void *dev, size_t bytes, cudaStream_t st) {
    const size_t rows = bytes / kRow, tail = bytes - rows * kRow;
    cudaError_t e = cudaSuccess;
    if (rows) {
        void *h[1] = {host};
        const void *d[1] = {dev};
        e = planes_d2h(1, h, kRow, d, kRow, kRow, rows, st);
    }
    if (e == cudaSuccess && tail)
        e = finish(cudaMemcpyAsync((unsigned char *)host + rows * kRow, (const unsigned char *)dev + rows * kRow, tail,
                                   cudaMemcpyDeviceToHost, st),
                   st);
    return e;
}

}  // namespace tsu

// ------------------------------------------------------------------ C ABI
namespace {

int copy_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return TSU_OK;
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    tsu_set_error_detail(buf);
    if (e == cudaErrorMemoryAllocation) return TSU_ERR_HOST_OOM;
    if (e == cudaErrorInvalidDevice || e == cudaErrorNoDevice) return TSU_ERR_NO_DEVICE;
    return TSU_ERR_CUDA;
}

int check_planes(int nplanes, const void *const *a, const void *const *b, size_t apitch, size_t bpitch,
                 size_t width) {
    if (nplanes < 0 || (nplanes > 0 && (!a || !b)) || width > apitch || width > bpitch) return TSU_ERR_INVALID;
    for (int k = 0; k < nplanes; k++)
        if (!a[k] || !b[k]) return TSU_ERR_INVALID;
    return TSU_OK;
}

}  // namespace

extern "C" int tsu_copy_planes_to_device(int device, int nplanes, void *const *dev, size_t dpitch,
                                         const void *const *host, size_t hpitch, size_t width, size_t rows) {
    if (int r = check_planes(nplanes, (const void *const *)dev, host, dpitch, hpitch, width)) return r;
    if (cudaError_t e = cudaSetDevice(device)) return copy_status(e, "cudaSetDevice");
    return copy_status(tsu::planes_h2d(nplanes, dev, dpitch, host, hpitch, width, rows, 0), "copy to device");
}

extern "C" int tsu_copy_planes_to_host(int device, int nplanes, void *const *host, size_t hpitch,
                                       const void *const *dev, size_t dpitch, size_t width, size_t rows) {
    if (int r = check_planes(nplanes, (const void *const *)host, dev, hpitch, dpitch, width)) return r;
    if (cudaError_t e = cudaSetDevice(device)) return copy_status(e, "cudaSetDevice");
    return copy_status(tsu::planes_d2h(nplanes, host, hpitch, dev, dpitch, width, rows, 0), "copy to host");
}

extern "C" int tsu_copy_bytes_to_device(int device, void *dev, const void *host, size_t bytes) {
    if (bytes && (!dev || !host)) return TSU_ERR_INVALID;
    if (cudaError_t e = cudaSetDevice(device)) return copy_status(e, "cudaSetDevice");
    return copy_status(tsu::bytes_h2d(dev, host, bytes, 0), "copy to device");
}

extern "C" int tsu_copy_bytes_to_host(int device, void *host, const void *dev, size_t bytes) {
    if (bytes && (!dev || !host)) return TSU_ERR_INVALID;
    if (cudaError_t e = cudaSetDevice(device)) return copy_status(e, "cudaSetDevice");
    return copy_status(tsu::bytes_d2h(host, dev, bytes, 0), "copy to host");
}

extern "C" int tsu_host_threads(void) { return tsu::host_threads(); }
