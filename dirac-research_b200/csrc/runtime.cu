// Library-wide runtime pieces: version, device check, last-error record and the
// per-device scratch buffer used when callers pass no scratch.

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "dgpu_internal.cuh"

namespace dgpu {

namespace {
std::mutex g_err_mu;
char g_last_error[512] = "";

constexpr int kMaxDevices = 64;
// One scratch buffer per (device, stream).  A buffer outgrown by a later call is retired, not
// freed: a call on another host thread may still hold its pointer or have kernels queued on it,
// so retired buffers live until process exit (growth is geometric, so they add up to less than
// the live buffer).
struct Scratch {
    int dev;
    void* stream;
    void* p;
    size_t bytes;
};
std::mutex g_scratch_mu;
std::vector<Scratch> g_scratch;
std::vector<void*> g_retired;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
}

int library_scratch(size_t bytes, void* stream, void** out) {
    int dev = 0;
    DGPU_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return DGPU_ERR_DEVICE;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    Scratch* s = nullptr;
    for (Scratch& e : g_scratch)
        if (e.dev == dev && e.stream == stream) s = &e;
    if (!s) {
        g_scratch.push_back(Scratch{dev, stream, nullptr, 0});
        s = &g_scratch.back();
    }
    if (s->bytes < bytes) {
        const size_t want = align_up(std::max(bytes, 2 * s->bytes), 1 << 20);
        void* p = nullptr;
        if (cudaMalloc(&p, want) != cudaSuccess) {
            cudaGetLastError();
            return DGPU_ERR_NOMEM;
        }
        if (s->p) g_retired.push_back(s->p);
        s->p = p;
        s->bytes = want;
    }
    *out = s->p;
    return DGPU_OK;
}

namespace {

// Host worker threads shared by every caller of parallel_for (several host threads may submit
// at once: each waits only for its own chunks).
class HostPool {
   public:
    explicit HostPool(int n) {
        for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    int size() const { return (int)workers_.size(); }
    void submit(std::function<void()> f) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(f));
        }
        cv_.notify_one();
    }

   private:
    void loop() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                f = std::move(q_.front());
                q_.pop_front();
            }
            f();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> q_;
    bool stop_ = false;
};

// Workers of the host pool: DGPU_HOST_THREADS when set (1..256, read once, when the pool is
// first used), else one fewer than the hardware threads, at most 15.
int host_pool_size() {
    if (const char* v = std::getenv("DGPU_HOST_THREADS")) {
        const int n = std::atoi(v);
        if (n >= 1 && n <= 256) return n;
    }
    return std::max(1, std::min(15, (int)std::thread::hardware_concurrency() - 1));
}

HostPool& host_pool() {
    static HostPool pool(host_pool_size());
    return pool;
}

}  // namespace

// Wait mode (dgpu_set_blocking_waits): 0 (default) polls the stream; 1 sleeps on an event
// created with cudaEventBlockingSync; 2 polls and yields the core between polls.  Modes 1 and
// 2 leave the host cores to other threads while many streams wait at once, mode 1 at the cost
// of a later wake-up.
std::atomic<int> g_blocking_waits{0};

namespace {

// One blocking-sync event per device for each host thread, destroyed when the thread ends.
struct WaitEvents {
    std::vector<cudaEvent_t> ev;
    ~WaitEvents() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

}  // namespace

cudaError_t host_wait(cudaStream_t st) {
    const int mode = g_blocking_waits.load(std::memory_order_relaxed);
    if (mode == 0) return cudaStreamSynchronize(st);
    if (mode == 2) {
        // poll, handing the core to any other runnable thread between polls
        for (;;) {
            const cudaError_t q = cudaStreamQuery(st);
            if (q != cudaErrorNotReady) return q;
            std::this_thread::yield();
        }
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    thread_local WaitEvents T;
    if ((int)T.ev.size() <= dev) T.ev.resize((size_t)dev + 1, nullptr);
    if (!T.ev[dev]) {
        e = cudaEventCreateWithFlags(&T.ev[dev], cudaEventDisableTiming | cudaEventBlockingSync);
        if (e != cudaSuccess) {
            T.ev[dev] = nullptr;
            return e;
        }
    }
    if (cudaEventRecord(T.ev[dev], st) != cudaSuccess) {
        // a stream of another device than the current one: wait on the stream itself
        cudaGetLastError();
        return cudaStreamSynchronize(st);
    }
    return cudaEventSynchronize(T.ev[dev]);
}

void parallel_for(int n, int grain, const std::function<void(int, int)>& body) {
    if (n <= 0) return;
    grain = std::max(1, grain);
    HostPool& pool = host_pool();
    const int chunks = std::min(pool.size() + 1, (n + grain - 1) / grain);
    if (chunks <= 1) {
        body(0, n);
        return;
    }
    const int per = (n + chunks - 1) / chunks;
    std::mutex m;
    std::condition_variable done;
    int left = chunks - 1;
    for (int c = 1; c < chunks; ++c) {
        const int b = c * per, e = std::min(n, b + per);
        pool.submit([&, b, e] {
            if (b < e) body(b, e);
            std::lock_guard<std::mutex> lk(m);
            if (--left == 0) done.notify_all();
        });
    }
    body(0, std::min(n, per));
    std::unique_lock<std::mutex> lk(m);
    done.wait(lk, [&] { return left == 0; });
}

}  // namespace dgpu

extern "C" const char* dgpu_version(void) { return "dirac-b200 0.1 (sm_100a)"; }

extern "C" int dgpu_set_blocking_waits(int on) {
    if (on < 0 || on > 2) return DGPU_ERR_ARG;
    dgpu::g_blocking_waits.store(on);
    return DGPU_OK;
}

extern "C" const char* dgpu_last_error(void) { return dgpu::g_last_error; }

extern "C" unsigned long long dgpu_launch_count(void) { return dgpu::g_launches.load(); }

extern "C" int dgpu_device_check(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return DGPU_ERR_DEVICE;
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return DGPU_ERR_DEVICE;
    if (p.major != 10) return DGPU_ERR_DEVICE;
    return p.major * 10 + p.minor;
}
