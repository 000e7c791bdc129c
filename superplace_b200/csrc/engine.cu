// Host side of the sm_100a GP engine and the C ABI of include/spgpu.h.
//
// The host code here plays the role of the reference's EPlace / BinGrid drivers
// (src/gp/eplace.cpp, src/gp/bin_grid.cpp): it builds the stage-static data (bin grid
// dimension, terminal and base density, local-smoothing footprints, optimisation set,
// clamp boxes) once per stage, then launches the device-resident iteration. It never
// computes an iteration quantity itself: every schedule scalar lives in DevState and is
// updated by control kernels. Per iteration it reads a 16-byte status to learn whether
// to launch a backtracking re-evaluation or the next iteration.
#include <cuda_runtime.h>
#include <pthread.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "poisson.h"

namespace spg {

std::atomic<int64_t> g_launches{0};

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("SPG_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

thread_local cudaStream_t t_alloc_stream = nullptr;

namespace {
// The opt cells' WA pass 2 runs on the WA stream ahead of the assembly (wl_cells_kernel);
// SPG_WL_AHEAD=0 leaves it inside the assembly. Same sums either way.
bool wl_ahead() {
    static const bool on = [] {
        const char* e = std::getenv("SPG_WL_AHEAD");
        return !(e && e[0] == '0');
    }();
    return on;
}

cudaMemPool_t library_pool(int dev) {
    static std::mutex mu;
    static std::vector<std::pair<int, cudaMemPool_t>> pools;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& e : pools)
        if (e.first == dev) return e.second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    SPG_CUDA(cudaMemPoolCreate(&pool, &props));
    // keep freed memory in the pool for the next context instead of returning it at every sync
    uint64_t keep = ~0ull;
    SPG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    // Reuse memory freed on another stream only once that free has completed: never make one
    // context's stream wait on another's (which the pool would do to hand out memory freed
    // ahead in another stream, serializing independent placements).
    int off = 0, on = 1;
    SPG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseFollowEventDependencies, &off));
    SPG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off));
    SPG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &on));
    pools.emplace_back(dev, pool);
    return pool;
}
}  // namespace

// Waits on the host for the work queued on `s` so far, sleeping instead of spinning: a
// thread-local event created with cudaEventBlockingSync. Many host threads (one per context
// of a placement server) then wait without taking the CPU from threads with host work.
cudaError_t host_wait(cudaStream_t s) {
    struct Ev {
        int dev = -1;
        cudaEvent_t ev = nullptr;
        ~Ev() {
            if (ev) cudaEventDestroy(ev);
        }
    };
    static thread_local Ev e;
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) return r;
    if (!e.ev || e.dev != dev) {
        if (e.ev) cudaEventDestroy(e.ev);
        e.ev = nullptr;
        r = cudaEventCreateWithFlags(&e.ev, cudaEventBlockingSync | cudaEventDisableTiming);
        if (r != cudaSuccess) return r;
        e.dev = dev;
    }
    r = cudaEventRecord(e.ev, s);
    return r == cudaSuccess ? cudaEventSynchronize(e.ev) : r;
}

void* dev_alloc(size_t bytes, cudaStream_t* owner) {
    void* p = nullptr;
    const cudaStream_t s = t_alloc_stream;
    *owner = s;
    if (!s) {
        SPG_CUDA(cudaMalloc(&p, bytes));
        return p;
    }
    int dev = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    SPG_CUDA(cudaMallocFromPoolAsync(&p, bytes, library_pool(dev), s));
    // complete before return: callers copy into it from the host or use it on other streams
    SPG_CUDA(host_wait(s));
    return p;
}

void dev_free(void* p, cudaStream_t owner) {
    if (!p) return;
    if (owner) cudaFreeAsync(p, owner);
    else cudaFree(p);
}

int launch_priority(bool high) {
    static const std::pair<int, int> range = [] {
        int l = 0, h = 0;
        if (cudaDeviceGetStreamPriorityRange(&l, &h) != cudaSuccess) l = h = 0;
        return std::make_pair(l, h);
    }();
    return high ? range.second : range.first;
}

int wave_grid(const void* kernel, int threads, int cap) {
    struct Entry {
        const void* kernel;
        int device, threads, blocks;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int dev = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    int blocks = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (const Entry& e : cache)
            if (e.kernel == kernel && e.device == dev && e.threads == threads) blocks = e.blocks;
    }
    if (blocks == 0) {
        int sms = 0, per_sm = 0;
        SPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        SPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
        blocks = std::max(1, sms) * std::max(1, per_sm);
        std::lock_guard<std::mutex> lock(mu);
        cache.push_back(Entry{kernel, dev, threads, blocks});
    }
    if (blocks <= cap) return blocks;
    int sms = 0;
    SPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // whole blocks per SM under the cap, so the wave stays even
    return sms > 0 && cap >= sms ? (cap / sms) * sms : cap;
}

// optimizer.cu entry points not declared in engine.h
void launch_ctl_lambda_init(const DevPtrs& p, cudaStream_t s);
void launch_ctl_step(const DevPtrs& p, int reduce_fresh, cudaStream_t s);
void launch_init_norms(const DevPtrs& p, cudaStream_t s);
void launch_ctl_init_scale(const DevPtrs& p, float init_perturb, cudaStream_t s);
void launch_init_diff(const DevPtrs& p, cudaStream_t s);
void launch_ctl_init_finish(const DevPtrs& p, cudaStream_t s);
void launch_clamp_role(const DevPtrs& p, int role, cudaStream_t s);
void launch_stage_clock(const DevPtrs& p, cudaStream_t s);
void launch_check_geometry(const DevPtrs& p, float lx, float ly, float hx, float hy, const float* w,
                           const float* h, cudaStream_t s);

namespace {

thread_local std::string g_last_error;

constexpr int kMaxBinDim = 1024;      // bin_grid.cpp:18
constexpr float kBoundaryEps = 1e-3f;  // eplace.cpp:38

}  // namespace

// A process-wide pool of host worker threads for run_parts and PartsTask. The host passes of a
// stage run as parts at once (grid statics, the footprint scan, large copies); a pool spares
// each part a thread start. Any number of callers (contexts on threads of their own) may submit
// at once, and a waiting caller runs parts of its own batch as well, so its wait completes even
// when every worker is busy elsewhere. Every access to a batch is under the pool's lock, and
// wait returns only after the last part of its batch has been accounted for there, so no worker
// touches a batch after its wait ends. The pool is never destroyed (its workers idle until the
// process exits); a forked child, which has none of the parent's workers, starts a pool of its
// own on first use.
class HostPool {
public:
    static HostPool& get() {
        HostPool* p = g_pool.load(std::memory_order_acquire);
        if (p) return *p;
        std::lock_guard<std::mutex> lock(*g_pool_mu);
        p = g_pool.load(std::memory_order_relaxed);
        if (!p) {
            static const int registered = pthread_atfork(nullptr, nullptr, [] {
                g_pool_mu = new (g_pool_mu_store) std::mutex();  // the child's first and only thread
                g_pool.store(nullptr, std::memory_order_relaxed);
            });
            (void)registered;
            p = new HostPool();
            g_pool.store(p, std::memory_order_release);
        }
        return *p;
    }

    // One submission: fn(t) for t = 0..n-1. It must stay in place (and fn alive) from submit
    // to the end of wait.
    struct Batch {
        std::function<void(int)> fn;
        int n = 0, next = 0, finished = 0;
        std::exception_ptr err;
    };

    void submit(Batch& b) {
        if (b.n <= 0) return;
        {
            std::lock_guard<std::mutex> lock(mu_);
            queue_.push_back(&b);
        }
        work_.notify_all();
    }

    // Runs the batch's unclaimed parts on the calling thread, waits for the others, then
    // rethrows the first exception a part raised.
    void wait(Batch& b) {
        if (b.n <= 0) return;
        for (;;) {
            int t;
            {
                std::lock_guard<std::mutex> lock(mu_);
                if (!claim(&b, &t)) break;
            }
            execute(&b, t);
        }
        std::unique_lock<std::mutex> lock(mu_);
        done_.wait(lock, [&] { return b.finished == b.n; });
        lock.unlock();
        if (b.err) std::rethrow_exception(b.err);
    }

    template <typename F>
    void run(int n, F& fn) {
        Batch b;
        b.fn = [&fn](int t) { fn(t); };
        b.n = n;
        submit(b);
        wait(b);
    }

private:
    HostPool() {
        const unsigned hc = std::thread::hardware_concurrency();
        const int workers = static_cast<int>(std::min(15u, hc > 1 ? hc - 1 : 0u));
        for (int i = 0; i < workers; ++i) std::thread([this] { loop(); }).detach();
    }

    // under mu_: the next unclaimed part of b (the batch leaves the queue with its last part)
    bool claim(Batch* b, int* t) {
        if (b->next >= b->n) return false;
        *t = b->next++;
        if (b->next == b->n) queue_.erase(std::find(queue_.begin(), queue_.end(), b));
        return true;
    }

    void execute(Batch* b, int t) {
        std::exception_ptr err;
        try {
            b->fn(t);
        } catch (...) {
            err = std::current_exception();
        }
        std::lock_guard<std::mutex> lock(mu_);
        if (err && !b->err) b->err = err;
        if (++b->finished == b->n) done_.notify_all();
    }

    void loop() {
        for (;;) {
            Batch* b;
            int t;
            {
                std::unique_lock<std::mutex> lock(mu_);
                work_.wait(lock, [&] { return !queue_.empty(); });
                b = queue_.front();
                claim(b, &t);
            }
            execute(b, t);
        }
    }

    std::mutex mu_;
    std::condition_variable work_, done_;
    std::vector<Batch*> queue_;

    static std::atomic<HostPool*> g_pool;
    alignas(std::mutex) static unsigned char g_pool_mu_store[sizeof(std::mutex)];
    static std::mutex* g_pool_mu;
};
std::atomic<HostPool*> HostPool::g_pool{nullptr};
alignas(std::mutex) unsigned char HostPool::g_pool_mu_store[sizeof(std::mutex)];
std::mutex* HostPool::g_pool_mu = new (HostPool::g_pool_mu_store) std::mutex();

// Runs fn(t) for t = 0..n-1 at once on the host pool and the calling thread; returns once all
// have finished. Used for host passes whose parts write disjoint data.
template <typename F>
void run_parts(int n, F&& fn) {
    HostPool::get().run(n, fn);
}

// run_parts in the background: the parts start on the pool at construction, and wait() runs
// what is left on the calling thread and waits for the rest (the destructor does the same on an
// exception's way out, dropping the parts' own errors). fn must outlive the task.
class PartsTask {
public:
    template <typename F>
    PartsTask(int n, F& fn) {
        b_.fn = [&fn](int t) { fn(t); };
        b_.n = n;
        HostPool::get().submit(b_);
    }
    PartsTask(const PartsTask&) = delete;
    PartsTask& operator=(const PartsTask&) = delete;
    void wait() {
        waited_ = true;
        HostPool::get().wait(b_);
    }
    ~PartsTask() {
        if (waited_) return;
        try {
            HostPool::get().wait(b_);
        } catch (...) {
        }
    }

private:
    HostPool::Batch b_;
    bool waited_ = false;
};

// memcpy of a large host buffer split over four threads (a single thread copies a few GB/s,
// well below what the host link and the host's memory sustain).
void host_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kSplit = size_t(4) << 20;
    if (bytes < kSplit) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes / 4 + 4095) & ~size_t(4095);
    run_parts(4, [&](int t) {
        const size_t b0 = std::min(bytes, part * t), b1 = std::min(bytes, part * (t + 1));
        if (b1 > b0) std::memcpy(static_cast<char*>(dst) + b0, static_cast<const char*>(src) + b0, b1 - b0);
    });
}

// Pinned staging memory for the host <-> device copies of one context: a copy from pageable
// memory is staged by the driver through a shared buffer (serialized across threads and
// synchronous), one from pinned memory is a plain DMA on the context's stream. Regions are
// handed out in order and recycled after the stream has been synchronized.
struct Staging {
    char* buf = nullptr;
    size_t cap = 0, used = 0;
    cudaStream_t s = nullptr;
    Staging() = default;
    Staging(const Staging&) = delete;
    Staging& operator=(const Staging&) = delete;
    ~Staging() {
        if (buf) cudaFreeHost(buf);
    }
    void* reserve(size_t bytes) {
        const size_t need = (bytes + 255) & ~static_cast<size_t>(255);
        if (used + need > cap) {
            SPG_CUDA(host_wait(s));  // every earlier region has been consumed
            used = 0;
            if (need > cap) {
                if (buf) cudaFreeHost(buf);
                buf = nullptr;
                cap = 0;
                const size_t grown = std::max(need, static_cast<size_t>(8) << 20);
                SPG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&buf), grown, cudaHostAllocDefault));
                cap = grown;
            }
        }
        void* d = buf + used;
        used += need;
        return d;
    }
};
// The staging memory of the context the calling thread is working on (see CtxScope).
thread_local Staging* t_staging = nullptr;

void upload_bytes(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    if (t_staging && t_staging->s == s) {
        void* d = t_staging->reserve(bytes);
        host_copy(d, src, bytes);
        src = d;
    }
    SPG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}

// Whether [p, p + bytes) lies in page-locked host memory (cudaHostAlloc'd or registered), which
// the copy engines read and write directly: a caller's array there needs no staging.
bool host_pinned(const void* p, size_t bytes) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();  // pageable memory on an older driver reports an error
        return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
    const char* last = static_cast<const char*>(p) + bytes - 1;
    if (cudaPointerGetAttributes(&a, last) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Two host -> device copies of `bytes` each from a caller's arrays, which are free again once
// this returns: from page-locked arrays, direct DMA on `s` and one wait for both; from
// pageable ones, copies into the context's staging memory (no wait).
void upload_pair(void* dst0, const void* src0, void* dst1, const void* src1, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    if (host_pinned(src0, bytes) && host_pinned(src1, bytes)) {
        SPG_CUDA(cudaMemcpyAsync(dst0, src0, bytes, cudaMemcpyHostToDevice, s));
        SPG_CUDA(cudaMemcpyAsync(dst1, src1, bytes, cudaMemcpyHostToDevice, s));
        SPG_CUDA(host_wait(s));
        return;
    }
    upload_bytes(dst0, src0, bytes, s);
    upload_bytes(dst1, src1, bytes, s);
}

// Two device -> host copies of `bytes` each, complete on return, with one wait.
void download_pair(void* dst0, const void* src0, void* dst1, const void* src1, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    if (t_staging && t_staging->s == s && !(host_pinned(dst0, bytes) && host_pinned(dst1, bytes))) {
        // one region for both (a second reservation could recycle the first's memory)
        const size_t half = (bytes + 255) & ~static_cast<size_t>(255);
        char* d0 = static_cast<char*>(t_staging->reserve(2 * half));
        char* d1 = d0 + half;
        SPG_CUDA(cudaMemcpyAsync(d0, src0, bytes, cudaMemcpyDeviceToHost, s));
        SPG_CUDA(cudaMemcpyAsync(d1, src1, bytes, cudaMemcpyDeviceToHost, s));
        SPG_CUDA(host_wait(s));
        host_copy(dst0, d0, bytes);
        host_copy(dst1, d1, bytes);
        return;
    }
    SPG_CUDA(cudaMemcpyAsync(dst0, src0, bytes, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(cudaMemcpyAsync(dst1, src1, bytes, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(host_wait(s));
}

// Device -> host copy, complete on return.
void download_bytes(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    if (t_staging && t_staging->s == s) {
        void* d = t_staging->reserve(bytes);
        SPG_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToHost, s));
        SPG_CUDA(host_wait(s));
        host_copy(dst, d, bytes);
        return;
    }
    SPG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(host_wait(s));
}

namespace {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    cudaStream_t owner = nullptr;  // the stream its free is ordered on
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void reset() {
        dev_free(p, owner);
        p = nullptr;
        n = cap = 0;
    }
    // Size the buffer for `count` elements. An allocation with enough capacity is kept, so
    // repeated stage runs, and a context reloaded with another netlist of no larger size,
    // reuse their device memory and keep their addresses; a larger size grows it by half.
    void alloc(size_t count) {
        if (count == 0) count = 1;
        if (p && count <= cap) {
            n = count;
            return;
        }
        const size_t grown = p ? std::max(count, cap + cap / 2) : count;
        reset();
        p = static_cast<T*>(dev_alloc(grown * sizeof(T), &owner));
        n = count;
        cap = grown;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count);
        upload_bytes(p, h, count * sizeof(T), s);
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void zero(cudaStream_t s) { SPG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
};

int clampi_h(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
float hmin(float a, float b) { return (b < a) ? b : a; }
float hmax(float a, float b) { return (a < b) ? b : a; }
float overlap_area(float alx, float aly, float ahx, float ahy, float blx, float bly, float bhx,
                   float bhy) {
    const float dx = hmin(ahx, bhx) - hmax(alx, blx);
    const float dy = hmin(ahy, bhy) - hmax(aly, bly);
    return (dx > 0.f && dy > 0.f) ? dx * dy : 0.f;
}

}  // namespace

// ---------------------------------------------------------------------------------------
struct LoopGraph;

// The context's streams live in a base class: the members' device buffers are freed (in
// order on `stream`) before the streams are destroyed.
struct ContextStreams {
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // WA pass 1 overlaps the density -> Poisson chain
    ~ContextStreams() {
        if (stream) host_wait(stream);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct Context : ContextStreams {
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // the stage loop's timing events
    spg_params prm{};
    // host copy of the db (flags and sizes change with mLG; positions live on the device)
    int num_movable = 0, num_nodes = 0, num_fillers = 0, total = 0, num_pins = 0, num_nets = 0, num_slots = 0;
    std::vector<float> w, h;
    std::vector<uint8_t> flags;
    std::vector<int> node_start;
    std::vector<float> row_ly, row_hgt, row_lx, row_step;
    std::vector<int> row_sites;
    float core_lx = 0, core_ly = 0, core_hx = 0, core_hy = 0;

    DevBuf<float> x, y, dw, dh, hw, hh, wgt;
    DevBuf<uint8_t> kind;
    DevBuf<float> pox, poy, gpx, gpy;
    DevBuf<int> pin2node, pin2net, net_start, net_pins, node_start_d, node_pins, net_order;
    DevBuf<int> slot_start, net_slot, wa_start;
    DevBuf<int2> wa_node_slot;
    DevBuf<float2> wa_off;
    WaClasses wa_classes{};
    // grid
    bool grid_ready = false;
    GridGeom geom{};
    double movable_area_scaled = 0.0;
    DevBuf<unsigned long long> node_fix, filler_fix;
    DevBuf<float> terminal, base, rho, phi, ex, ey, node_map, filler_map;
    std::unique_ptr<PoissonPlan> plan;                      // the current grid's Poisson plan
    std::vector<std::unique_ptr<PoissonPlan>> spare_plans;  // other grid sizes seen (reused)
    DevBuf<int> dens_large;
    int n_dens_small = 0, n_dens_large = 0;
    std::vector<int> dens_large_h;  // host copy (ascending), for the per-stage lists
    bool fillers_alike = false;     // every filler has the same size and degree and no pin slots
    DevBuf<int> rest_small, rest_large;
    int n_rest_small = 0, n_rest_large = 0;
    // stage
    int n_opt = 0;
    DevBuf<int> opt_idx, opt_large, opt_cells;
    std::vector<int> opt_cells_h;  // the stage's opt cells (host), ascending
    DevBuf<float4> opt_geom;
    DevBuf<int4> opt_meta;
    // the fillers' shared attributes (see DevPtrs::filler_k0)
    int filler_k0 = 0;
    float4 filler_geom{};
    int4 filler_meta{};
    double filler_area = 0.0;
    float filler_lo_x = 0.f, filler_hi_x = 0.f, filler_lo_y = 0.f, filler_hi_y = 0.f;
    DevBuf<uint8_t> flags_d;  // the node flags the current grid was built with
    std::vector<int> slot_start_h;         // node-order pin slots (see DevPtrs::slot_start)

    // host copy of the node positions as last uploaded, while the device copy is unchanged
    std::vector<float> x_mirror, y_mirror;  // host copy of the non-filler positions (fixed nodes' terminal density)
    bool mirror_valid = false;
    DevBuf<float> opt_lo, opt_hi, force, wlg, pool;
    // the fillers' spatial reorder (filler_order.cu): active for the stage when the fillers
    // share their attributes and are numerous; the loop pauses at the listed iterations
    bool fo_active = false;
    std::vector<int> fo_pauses;
    // the iteration callback (spg_set_iter_callback) and the evaluation-point snapshots
    spg_iter_fn iter_fn = nullptr;
    void* iter_user = nullptr;
    int iter_stride = 0;
    spg_iter_fn mid_fn = nullptr;  // spg_set_stagnation_callback
    void* mid_user = nullptr;
    bool have_eval = false;  // a stage ran: its last evaluation point is on the device
    int eval_role = 0, eval_prev_role = 0;  // the roles that hold it and the point before it
    DevBuf<float> frame_x, frame_y;
    std::vector<float> frame_hx, frame_hy;
    DevBuf<int> fo_key, fo_tmp, fo_perm, fo_fid, fo_fid_tmp, fo_count, fo_offset, fo_cursor, fo_skip;
    DevBuf<float> fo_scratch;
    DevBuf<double> opt_area;
    int n_opt_large = 0;
    size_t vec_stride = 0;
    DevBuf<double> partials;
    DevBuf<DevState> st;
    DevBuf<spg_iter_metrics> metrics;
    DevBuf<double> scratch_d;
    int metrics_rows = 0;
    DevState* hst = nullptr;  // pinned host mirror
    Staging staging;          // pinned staging of this context's host <-> device copies
    float step_x_gamma = 1.f;
    // the iteration loop as a conditional CUDA graph (engine.cu: build_loop_graph), one per
    // Poisson plan held (the kernel sequence differs between grid sizes); the host-driven
    // loop runs instead where the driver refuses conditional nodes
    bool use_graph = true;
    bool last_run_graph = false;
    double last_graph_build_ms = 0.0;
    std::vector<std::pair<const PoissonPlan*, std::shared_ptr<LoopGraph>>> loop_graphs;
    FillerOrderBufs filler_order_bufs() {
        return FillerOrderBufs{fo_key.p, fo_tmp.p, fo_perm.p, fo_fid.p, fo_fid_tmp.p, fo_count.p, fo_offset.p,
                               fo_cursor.p, fo_skip.p, fo_scratch.p, opt_idx.p};
    }
    void drop_loop_graph(const PoissonPlan* pl) {
        for (auto it = loop_graphs.begin(); it != loop_graphs.end(); ++it)
            if (it->first == pl) {
                loop_graphs.erase(it);
                return;
            }
    }

    ~Context() {
        if (side) host_wait(side);
        if (stream) host_wait(stream);
        loop_graphs.clear();
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_t0) cudaEventDestroy(ev_t0);
        if (ev_t1) cudaEventDestroy(ev_t1);
        if (plan) poisson_plan_destroy(*plan);
        for (auto& q : spare_plans) poisson_plan_destroy(*q);
        if (hst) cudaFreeHost(hst);
    }

    DevPtrs ptrs() const {
        DevPtrs p;
        std::memset(&p, 0, sizeof(p));  // padding too: graphs are keyed on the bytes
        p.num_movable = num_movable;
        p.num_nodes = num_nodes;
        p.num_fillers = num_fillers;
        p.total = total;
        p.num_pins = num_pins;
        p.num_nets = num_nets;
        p.x = x.p;
        p.y = y.p;
        p.hw = hw.p;
        p.hh = hh.p;
        p.wgt = wgt.p;
        p.kind = kind.p;
        p.pox = pox.p;
        p.poy = poy.p;
        p.pin2node = pin2node.p;
        p.pin2net = pin2net.p;
        p.net_start = net_start.p;
        p.net_pins = net_pins.p;
        p.node_start = node_start_d.p;
        p.node_pins = node_pins.p;
        p.net_order = net_order.p;
        p.gpx = gpx.p;
        p.gpy = gpy.p;
        p.slot_start = slot_start.p;
        p.net_slot = net_slot.p;
        p.wa_start = wa_start.p;
        p.wa_node_slot = wa_node_slot.p;
        p.wa_off = wa_off.p;
        p.geom = geom;
        p.node_fix = node_fix.p;
        p.filler_fix = filler_fix.p;
        p.terminal = terminal.p;
        p.base = base.p;
        p.rho = rho.p;
        p.phi = phi.p;
        p.ex = ex.p;
        p.ey = ey.p;
        p.node_map = node_map.p;
        p.filler_map = filler_map.p;
        p.movable_area_scaled = movable_area_scaled;
        p.n_opt = n_opt;
        p.opt_idx = opt_idx.p;
        p.opt_geom = opt_geom.p;
        p.opt_meta = opt_meta.p;
        p.filler_k0 = filler_k0;
        p.filler_node0 = num_nodes - filler_k0;
        p.filler_geom = filler_geom;
        p.filler_meta = filler_meta;
        p.filler_area = filler_area;
        p.filler_lo_x = filler_lo_x;
        p.filler_hi_x = filler_hi_x;
        p.filler_lo_y = filler_lo_y;
        p.filler_hi_y = filler_hi_y;
        p.opt_lo = opt_lo.p;
        p.opt_hi = opt_hi.p;
        p.opt_area = opt_area.p;
        p.force = force.p;
        p.wlg = wl_ahead() ? wlg.p : nullptr;
        p.pool = pool.p;
        p.vec_stride = vec_stride;
        p.dens_large = dens_large.p;
        p.n_dens_small = n_dens_small;
        p.n_dens_large = n_dens_large;
        p.rest_small = rest_small.p;
        p.rest_large = rest_large.p;
        p.n_rest_small = n_rest_small;
        p.n_rest_large = n_rest_large;
        p.opt_large = opt_large.p;
        p.n_opt_large = n_opt_large;
        p.partials = partials.p;
        p.st = st.p;
        p.metrics = metrics.p;
        p.ignore_net_degree = prm.ignore_net_degree;
        p.use_bb = prm.use_bb;
        p.backtrack = prm.gp_backtrack;
        p.max_backtrack = prm.max_backtrack;
        p.min_gain = std::min(std::max(prm.gp_stagnation_min_gain, 0.f), 0.5f);
        p.stagnation_window = prm.gp_stagnation_window;
        p.freeze_lambda = prm.freeze_lambda != 0;
        p.freeze_gamma = prm.freeze_gamma != 0;
        p.step_x_gamma = step_x_gamma;
        return p;
    }

    bool fixed(int i) const { return (flags[i] & SPG_F_FIXED) != 0; }
    bool ni(int i) const { return (flags[i] & SPG_F_NI) != 0; }
    bool macro(int i) const { return (flags[i] & SPG_F_MACRO) != 0; }
    bool filler(int i) const { return (flags[i] & SPG_F_FILLER) != 0; }
};

namespace {

// BinGrid::initialize (src/gp/bin_grid.cpp:64-189) for the current flags, plus the
// per-node footprint data the density kernels read and the fixed-point scale.
// SPG_HOST_TIMING=1: stage_run (and grid_init) print the host time of their phases to stderr.
struct HostTimer {
    bool on;
    std::chrono::steady_clock::time_point t0;
    std::string line;
    const char* tag;
    explicit HostTimer(const char* t = "") : tag(t) {
        const char* e = std::getenv("SPG_HOST_TIMING");
        on = e && e[0] == '1';
        t0 = std::chrono::steady_clock::now();
    }
    void mark(const char* name) {
        if (!on) return;
        const auto t = std::chrono::steady_clock::now();
        line += std::string(" ") + name + "=" +
                std::to_string(std::chrono::duration<double, std::milli>(t - t0).count()).substr(0, 6);
        t0 = t;
    }
    ~HostTimer() {
        if (on) std::fprintf(stderr, "[spg host ms%s]%s\n", tag, line.c_str());
    }
};

// footprintOf + chargeWeight (bin_grid.cpp:22-62) of one node: half extents after local
// smoothing (a node narrower or shorter than a bin is widened to it, with scale w/step), the
// charge weight (the scale, times the target density for macros) and the kernel class
// (density node, filler, large: a footprint of more than 16 bins). footprint_kernel writes
// the same values for every node with the same single and double operations.
struct NodeFootprint {
    float hw, hh, wgt;
    uint8_t kind;
};

NodeFootprint node_footprint(const Context& c, const GridGeom& g, float target, int i) {
    const float w = c.w[i], h = c.h[i];
    NodeFootprint r{0.5f * w, 0.5f * h, 0.f, 0};
    float sx = 1.f, sy = 1.f;
    if (w < g.step_x) {
        sx = w / g.step_x;
        r.hw = 0.5f * g.step_x;
    }
    if (h < g.step_y) {
        sy = h / g.step_y;
        r.hh = 0.5f * g.step_y;
    }
    const float scale = sx * sy;
    r.wgt = c.filler(i) ? scale : (c.macro(i) ? scale * target : scale);
    if (!(c.fixed(i) || c.ni(i))) {
        r.kind = K_DENSITY;
        if (c.filler(i)) r.kind |= K_FILLER;
        const double bins = (std::floor(2.0 * r.hw / g.step_x) + 2.0) * (std::floor(2.0 * r.hh / g.step_y) + 2.0);
        if (bins > 16.0) r.kind |= K_LARGE;
    }
    return r;
}

struct FootprintArgs {
    const float *w, *h;
    const uint8_t* flags;
    int total;
    float step_x, step_y, target;
    float *hw, *hh, *wgt;
    uint8_t* kind;
};

__global__ void footprint_kernel(FootprintArgs a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.total; i += gridDim.x * blockDim.x) {
        const float w = a.w[i], h = a.h[i];
        const uint8_t f = a.flags[i];
        float sx = 1.f, sy = 1.f, hw = fmul(0.5f, w), hh = fmul(0.5f, h);
        if (w < a.step_x) {
            sx = fdiv(w, a.step_x);
            hw = fmul(0.5f, a.step_x);
        }
        if (h < a.step_y) {
            sy = fdiv(h, a.step_y);
            hh = fmul(0.5f, a.step_y);
        }
        const float scale = fmul(sx, sy);
        const bool filler = (f & SPG_F_FILLER) != 0;
        a.wgt[i] = filler ? scale : ((f & SPG_F_MACRO) ? fmul(scale, a.target) : scale);
        a.hw[i] = hw;
        a.hh[i] = hh;
        uint8_t k = 0;
        if (!(f & (SPG_F_FIXED | SPG_F_NI))) {
            k = K_DENSITY | (filler ? K_FILLER : 0);
            const double bx = floor(__ddiv_rn(__dmul_rn(2.0, static_cast<double>(hw)), static_cast<double>(a.step_x)));
            const double by = floor(__ddiv_rn(__dmul_rn(2.0, static_cast<double>(hh)), static_cast<double>(a.step_y)));
            if (__dmul_rn(__dadd_rn(bx, 2.0), __dadd_rn(by, 2.0)) > 16.0) k |= K_LARGE;
        }
        a.kind[i] = k;
    }
}

// BinGrid::initialize (bin_grid.cpp:64-189) for the context's nodes at hx_pos / hy_pos: the
// grid, its static maps, the footprints and the fixed-point scale. `meanwhile` (optional) runs
// on the calling thread after the device set-up and before the static maps are uploaded, while
// the pool still builds them; it may enqueue work that needs no static map.
void grid_init(Context& c, float target, int bin_dim, const std::vector<float>& hx_pos,
               const std::vector<float>& hy_pos, const std::function<void()>& meanwhile = nullptr) {
    HostTimer ht(" grid");
    double cell_area = 0.0, macro_area = 0.0;
    for (int i = 0; i < c.num_movable; ++i) {
        if (c.fixed(i) || c.ni(i)) continue;
        const double a = static_cast<double>(c.w[i]) * static_cast<double>(c.h[i]);
        if (c.macro(i)) macro_area += a;
        else cell_area += a;
    }
    c.movable_area_scaled = cell_area + macro_area * static_cast<double>(target);
    int dim;
    if (bin_dim > 0) {
        dim = std::min(bin_dim, kMaxBinDim);
    } else {
        const double avg = (c.num_movable > 0) ? (cell_area + macro_area) / c.num_movable : 1.0;
        const double ideal_bin = std::max(avg / target, 1e-9);
        const float cw = c.core_hx - c.core_lx, ch = c.core_hy - c.core_ly;
        const double ideal = static_cast<double>(cw) * static_cast<double>(ch) / ideal_bin;
        dim = 4;
        while (dim * 2 <= kMaxBinDim && static_cast<double>(dim * 2) * (dim * 2) <= ideal) dim *= 2;
    }
    GridGeom& g = c.geom;
    g.dim = dim;
    g.origin_x = c.core_lx;
    g.origin_y = c.core_ly;
    g.step_x = (c.core_hx - c.core_lx) / static_cast<float>(dim);
    g.step_y = (c.core_hy - c.core_ly) / static_cast<float>(dim);
    g.inv_step_x = 1.0 / static_cast<double>(g.step_x);
    g.inv_step_y = 1.0 / static_cast<double>(g.step_y);
    g.target_density = target;
    c.step_x_gamma = g.step_x;
    const size_t n = static_cast<size_t>(dim) * dim;

    // terminal density (bin_grid.cpp:120-137): every bin adds its fixed nodes' overlaps in
    // node order; thread `part` of the pass below takes the bin columns bx = part (mod kParts)
    constexpr int kParts = 4;
    std::vector<int> fixed_nodes;
    for (int i = 0; i < c.num_nodes; ++i)
        if (c.fixed(i) && !c.ni(i)) fixed_nodes.push_back(i);
    std::vector<float> term(n, 0.f), base(n, 0.f);
    auto terminal_part = [&](int part) {
        for (int i : fixed_nodes) {
            const float lx = hx_pos[i] - 0.5f * c.w[i], hx = hx_pos[i] + 0.5f * c.w[i];
            const float ly = hy_pos[i] - 0.5f * c.h[i], hy = hy_pos[i] + 0.5f * c.h[i];
            const int bx0 = clampi_h(static_cast<int>((lx - g.origin_x) / g.step_x), 0, dim - 1);
            const int bx1 = clampi_h(static_cast<int>((hx - g.origin_x) / g.step_x), 0, dim - 1);
            const int by0 = clampi_h(static_cast<int>((ly - g.origin_y) / g.step_y), 0, dim - 1);
            const int by1 = clampi_h(static_cast<int>((hy - g.origin_y) / g.step_y), 0, dim - 1);
            for (int bx = bx0 + ((part - bx0) % kParts + kParts) % kParts; bx <= bx1; bx += kParts) {
                const float blx = g.origin_x + bx * g.step_x;
                for (int by = by0; by <= by1; ++by) {
                    const float bly = g.origin_y + by * g.step_y;
                    term[static_cast<size_t>(bx) * dim + by] +=
                        target * overlap_area(blx, bly, blx + g.step_x, bly + g.step_y, lx, ly, hx, hy);
                }
            }
        }
    };
    // base density: non-row area of each bin (bin_grid.cpp:144-173)
    const int nr = static_cast<int>(c.row_ly.size());
    std::vector<int> order(nr);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return c.row_ly[a] < c.row_ly[b]; });
    std::vector<float> rly(nr), rhy(nr), rlx(nr), rhx(nr);
    for (int t = 0; t < nr; ++t) {
        const int r = order[t];
        rly[t] = c.row_ly[r];
        rhy[t] = c.row_ly[r] + c.row_hgt[r];
        rlx[t] = c.row_lx[r];
        rhx[t] = c.row_lx[r] + c.row_step[r] * static_cast<float>(c.row_sites[r]);
    }
    // footprint data (half extents after local smoothing, charge weight, kernel class) is
    // written on the device by footprint_kernel; the host keeps the fixed-point bound, the
    // large nodes (only nodes at least a bin wide or tall can be) and the small-node count
    std::vector<int>& dlarge = c.dens_large_h;
    dlarge.clear();
    // bound partials: node i adds into acc[i % 4], in ascending i; thread t owns partial t (the
    // same sums in the same order as one pass), its large nodes and its small-node count
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int small_t[4] = {0, 0, 0, 0};
    std::vector<int> large_t[4];
    auto footprint_part = [&](int t) {
        double a = 0.0;
        int ns = 0;
        std::vector<int>& lg = large_t[t];
        for (int i = t; i < c.total; i += 4) {
            if (c.fixed(i) || c.ni(i)) continue;
            const float w = c.w[i], h = c.h[i];
            a += static_cast<double>(w) * static_cast<double>(h);
            const bool large = !(w < g.step_x && h < g.step_y) && (node_footprint(c, g, target, i).kind & K_LARGE);
            if (large) lg.push_back(i);
            else ++ns;
        }
        acc[t] = a;
        small_t[t] = ns;
    };
    // The statics run in the background on the pool: four parts, each its terminal columns,
    // then one contiguous block of bin rows of the base map (so no two threads write into one
    // cache line; bin rows are independent). Meanwhile the footprint scan's four partials run,
    // then the device set-up and the caller's `meanwhile` work, which need no static map.
    auto statics_part = [&](int part) {
        terminal_part(part);
        const int by_end = (part + 1) * dim / kParts;
        for (int by = part * dim / kParts; by < by_end; ++by) {
            const float bly = g.origin_y + by * g.step_y;
            const float bhy = bly + g.step_y;
            size_t lo = 0, hi = static_cast<size_t>(nr);
            while (lo < hi) {
                const size_t mid = (lo + hi) / 2;
                if (rhy[mid] <= bly) lo = mid + 1;
                else hi = mid;
            }
            for (int bx = 0; bx < dim; ++bx) {
                const float blx = g.origin_x + bx * g.step_x;
                const float bhx = blx + g.step_x;
                float covered = 0.f;
                for (size_t t = lo; t < static_cast<size_t>(nr); ++t) {
                    if (rly[t] >= bhy) break;
                    covered += overlap_area(blx, bly, bhx, bhy, rlx[t], rly[t], rhx[t], rhy[t]);
                }
                const float area = (bhx - blx) * (bhy - bly);
                base[static_cast<size_t>(bx) * dim + by] = target * hmax(0.f, area - covered);
            }
        }
    };
    PartsTask statics(kParts, statics_part);
    run_parts(4, footprint_part);
    ht.mark("footprints");
    const int n_small = (small_t[0] + small_t[1]) + (small_t[2] + small_t[3]);
    for (const std::vector<int>& lg : large_t) dlarge.insert(dlarge.end(), lg.begin(), lg.end());
    std::sort(dlarge.begin(), dlarge.end());
    double bound = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    // fixed-point scale: largest s <= 40 with (total charge bound) * 2^s < 2^62
    bound *= target > 1.f ? static_cast<double>(target) : 1.0;
    int s = 40;
    if (bound > 0.0) {
        int e = 0;
        std::frexp(bound, &e);
        s = std::min(40, 62 - e);
    }
    g.shift = s;
    g.scale = std::ldexp(1.0, s);
    g.scale_f = s >= 0 ? std::ldexp(1.0f, s) : 0.f;
    g.inv_scale = std::ldexp(1.0, -s);

    cudaStream_t st = c.stream;
    c.flags_d.upload(c.flags, st);
    c.hw.alloc(c.total);
    c.hh.alloc(c.total);
    c.wgt.alloc(c.total);
    c.kind.alloc(c.total);
    if (c.total > 0) {
        FootprintArgs fa{c.dw.p, c.dh.p, c.flags_d.p, c.total, g.step_x, g.step_y, target,
                         c.hw.p, c.hh.p, c.wgt.p, c.kind.p};
        footprint_kernel<<<work_grid(reinterpret_cast<const void*>(footprint_kernel), c.total, RED_THREADS),
                           RED_THREADS, 0, st>>>(fa);
        count_launch();
        SPG_CHECK_LAUNCH();
    }
    c.dens_large.upload(dlarge, st);
    c.n_dens_small = n_small;
    c.n_dens_large = static_cast<int>(dlarge.size());
    c.node_fix.alloc(n);
    c.filler_fix.alloc(n);
    c.node_fix.zero(st);
    c.filler_fix.zero(st);
    for (DevBuf<float>* b : {&c.rho, &c.phi, &c.ex, &c.ey, &c.node_map, &c.filler_map}) {
        b->alloc(n);
        b->zero(st);
    }
    ht.mark("uploads");
    // a plan per grid size and precision is kept; new bin steps only rewrite its tables
    auto fits = [&](const std::unique_ptr<PoissonPlan>& q) {
        return q && q->nx == dim && q->ny == dim && q->precision == c.prm.poisson_precision;
    };
    if (!fits(c.plan)) {
        auto it = std::find_if(c.spare_plans.begin(), c.spare_plans.end(), fits);
        std::unique_ptr<PoissonPlan> next;
        if (it != c.spare_plans.end()) {
            next = std::move(*it);
            c.spare_plans.erase(it);
        } else {
            next = std::make_unique<PoissonPlan>();
            poisson_plan_create(*next, dim, dim, g.step_x, g.step_y, c.prm.poisson_precision, 1);
        }
        if (c.plan) c.spare_plans.push_back(std::move(c.plan));
        c.plan = std::move(next);
        constexpr size_t kSparePlans = 4;
        while (c.spare_plans.size() > kSparePlans) {
            c.drop_loop_graph(c.spare_plans.front().get());
            poisson_plan_destroy(*c.spare_plans.front());
            c.spare_plans.erase(c.spare_plans.begin());
        }
    }
    poisson_plan_set_steps(*c.plan, g.step_x, g.step_y);
    c.plan->single_launch = c.prm.poisson_single_launch != 0;
    ht.mark("plan");
    c.partials.alloc(static_cast<size_t>(RED_SLOTS) * RED_CAP);
    c.partials.zero(st);
    if (meanwhile) {
        meanwhile();
        ht.mark("meanwhile");
    }
    statics.wait();
    ht.mark("statics");
    c.terminal.upload(term, st);
    c.base.upload(base, st);
    c.grid_ready = true;
}

// Per-opt-node arrays of a stage, built on the device from the node arrays already there:
// opt k is node cells[k] (k < k0) or filler num_nodes + (k - k0). Clamp box, degree, area,
// footprint and slot range use the same IEEE single and double operations as the reference
// (eplace.cpp:117-133,176-178), so every value equals a host computation bit for bit.
struct StageOptArgs {
    const int* cells;
    int k0, n, num_nodes, num_movable;
    const float *w, *h, *hw, *hh, *wgt;
    const int *node_start, *slot_start;
    const uint8_t* kind;
    float core_lx, core_ly, core_hx, core_hy;
    int* opt_idx;
    float *lo, *hi;
    double* area;
    float4* geom;
    int4* meta;
};

__device__ __forceinline__ float dmax_f(float a, float b) { return (a < b) ? b : a; }

__global__ void stage_opt_kernel(StageOptArgs a) {
    const int n = a.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = k < a.k0 ? a.cells[k] : a.num_nodes + (k - a.k0);
        a.opt_idx[k] = i;
        const float w = a.w[i], h = a.h[i];
        const float hw = fmul(0.5f, w), hh = fmul(0.5f, h);
        const float xlo = fadd(fadd(a.core_lx, hw), kBoundaryEps);
        const float ylo = fadd(fadd(a.core_ly, hh), kBoundaryEps);
        a.lo[k] = xlo;
        a.hi[k] = dmax_f(xlo, fsub(fsub(a.core_hx, hw), kBoundaryEps));
        a.lo[n + k] = ylo;
        a.hi[n + k] = dmax_f(ylo, fsub(fsub(a.core_hy, hh), kBoundaryEps));
        const int d = a.node_start[i + 1] - a.node_start[i];
        a.area[k] = __dmul_rn(static_cast<double>(w), static_cast<double>(h));
        a.geom[k] = make_float4(a.hw[i], a.hh[i], a.wgt[i], 0.f);
        const bool has_wl = i < a.num_movable;
        a.meta[k] = make_int4(a.slot_start[i], has_wl ? a.slot_start[i + 1] : a.slot_start[i], d,
                              static_cast<int>(a.kind[i]) | (has_wl ? OPT_HAS_WL : 0));
    }
}

__global__ void iota_kernel(int* a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

// EPlace::Impl::buildOptSet (eplace.cpp:82-94) and the per-opt-node clamp boxes
// (eplace.cpp:117-133), degrees and areas (eplace.cpp:176-178). The host picks the opt cells,
// checks whether the fillers share every attribute and lists the large opt nodes; the
// per-node arrays are written by stage_opt_kernel.
void stage_setup(Context& c, int stage) {
    std::vector<int>& cells = c.opt_cells_h;
    cells.clear();
    if (stage != SPG_STAGE_FILLER_ONLY) {
        for (int i = 0; i < c.num_movable; ++i) {
            if (c.fixed(i) || c.ni(i)) continue;
            if (stage == SPG_STAGE_CGP && c.macro(i)) continue;
            cells.push_back(i);
        }
    }
    const int k0 = static_cast<int>(cells.size());
    const int nf = c.total - c.num_nodes;
    const int n = k0 + nf;
    c.n_opt = n;
    // opt k's clamp box (eplace.cpp:117-133), for the filler constants
    auto box = [&](int i, float& xlo, float& xhi, float& ylo, float& yhi) {
        const float hw = 0.5f * c.w[i], hh = 0.5f * c.h[i];
        xlo = c.core_lx + hw + kBoundaryEps;
        xhi = hmax(xlo, c.core_hx - hw - kBoundaryEps);
        ylo = c.core_ly + hh + kBoundaryEps;
        yhi = hmax(ylo, c.core_hy - hh - kBoundaryEps);
    };
    // the large opt nodes: the large density nodes (ascending) matched against the opt cells
    // (ascending) and the filler run
    std::vector<int> olarge;
    {
        size_t q = 0;
        for (int i : c.dens_large_h) {
            if (i >= c.num_nodes) {
                olarge.push_back(k0 + (i - c.num_nodes));
                continue;
            }
            while (q < cells.size() && cells[q] < i) ++q;
            if (q < cells.size() && cells[q] == i) olarge.push_back(static_cast<int>(q));
        }
    }
    // the fillers close the opt set (nodes num_nodes..total-1); when they all share every
    // attribute the kernels read (size and flags, so clamp box, area, footprint and kind;
    // degree; no pin slots), pass those once instead of per node
    bool same = nf > 0;
    {
        const int f0 = c.num_nodes;
        same = same && c.fillers_alike;  // sizes, degrees and pin slots: fixed per netlist
        // all flags equal: the run equals itself shifted by one
        same = same && (c.total - f0 < 2 ||
                        std::memcmp(c.flags.data() + f0, c.flags.data() + f0 + 1, c.total - f0 - 1) == 0);
        if (same) {
            const NodeFootprint fp = node_footprint(c, c.geom, c.geom.target_density, f0);
            c.filler_k0 = k0;
            c.filler_geom = make_float4(fp.hw, fp.hh, fp.wgt, 0.f);
            c.filler_meta = make_int4(0, 0, c.node_start[f0 + 1] - c.node_start[f0], static_cast<int>(fp.kind));
            c.filler_area = static_cast<double>(c.w[f0]) * static_cast<double>(c.h[f0]);
            box(f0, c.filler_lo_x, c.filler_hi_x, c.filler_lo_y, c.filler_hi_y);
        } else {
            c.filler_k0 = n;
        }
    }
    cudaStream_t s = c.stream;
    c.opt_cells.upload(cells, s);
    const size_t nn = static_cast<size_t>(std::max(n, 1));
    c.opt_idx.alloc(nn);
    c.opt_lo.alloc(2 * nn);
    c.opt_hi.alloc(2 * nn);
    c.opt_area.alloc(nn);
    c.opt_geom.alloc(nn);
    c.opt_meta.alloc(nn);
    if (n > 0) {
        StageOptArgs a{c.opt_cells.p, k0, n, c.num_nodes, c.num_movable, c.dw.p, c.dh.p, c.hw.p, c.hh.p,
                       c.wgt.p, c.node_start_d.p, c.slot_start.p, c.kind.p, c.core_lx, c.core_ly, c.core_hx,
                       c.core_hy, c.opt_idx.p, c.opt_lo.p, c.opt_hi.p, c.opt_area.p, c.opt_geom.p,
                       c.opt_meta.p};
        stage_opt_kernel<<<work_grid(reinterpret_cast<const void*>(stage_opt_kernel), n, RED_THREADS),
                           RED_THREADS, 0, s>>>(a);
        count_launch();
        SPG_CHECK_LAUNCH();
    }
    // density nodes the loop's step kernel does not rasterize: small ones outside the opt
    // set (the cells of FILLERONLY, the macros of cGP) and every large node. Every density
    // node is movable (or a filler, always in the opt set).
    {
        std::vector<int> rs;
        const GridGeom& g = c.geom;
        for (int i = 0; i < c.num_nodes; ++i) {  // fillers are always in the opt set
            if (c.fixed(i) || c.ni(i)) continue;  // not a density node
            const bool in_opt = i < c.num_movable && stage != SPG_STAGE_FILLER_ONLY &&
                                !(stage == SPG_STAGE_CGP && c.macro(i));
            if (in_opt) continue;
            const bool large = !(c.w[i] < g.step_x && c.h[i] < g.step_y) &&
                               (node_footprint(c, g, g.target_density, i).kind & K_LARGE);
            if (!large) rs.push_back(i);
        }
        c.rest_small.upload(rs, s);
        c.n_rest_small = static_cast<int>(rs.size());
        c.rest_large.upload(c.dens_large_h, s);
        c.n_rest_large = static_cast<int>(c.dens_large_h.size());
    }
    c.opt_large.upload(olarge, s);
    c.n_opt_large = static_cast<int>(olarge.size());
    c.force.alloc(2 * static_cast<size_t>(std::max(n, 1)));
    if (wl_ahead()) c.wlg.alloc(2 * static_cast<size_t>(std::max(n, 1)));
    // vectors padded to 64 floats so every role starts 256-byte aligned
    c.vec_stride = (2 * static_cast<size_t>(std::max(n, 1)) + 63) / 64 * 64;
    c.pool.alloc(c.vec_stride * (NUM_ROLES + SNAP_MAX));
    c.pool.zero(s);
    // the fillers' spatial reorder (filler_order.cu): fillers sharing their attributes, none
    // large, at least 4096 of them, grids up to 1024 (the tile key's range). SPG_FILLER_ORDER
    // lists the pause iterations ("8" by default; "0" turns the reorder off). One reorder at
    // iteration 8 measured best at 211k cells: 6292 iter/s against 6236 at 12, 6066 with a
    // second pause at 40 (each pause costs a host round trip) and 6059 without the reorder.
    {
        static const std::vector<int> pauses = [] {
            std::vector<int> v;
            const char* e = std::getenv("SPG_FILLER_ORDER");
            std::string str = e ? e : "8";
            size_t at = 0;
            while (at < str.size()) {
                const size_t comma = str.find(',', at);
                const int it = std::atoi(str.substr(at, comma - at).c_str());
                if (it > 0) v.push_back(it);
                if (comma == std::string::npos) break;
                at = comma + 1;
            }
            std::sort(v.begin(), v.end());
            return v;
        }();
        const int nf = n - c.filler_k0;
        c.fo_active = !pauses.empty() && c.filler_k0 < n && !(c.filler_meta.w & K_LARGE) && nf >= 4096 &&
                      c.geom.dim <= 1024;
        c.fo_pauses = pauses;
        if (c.fo_active) {
            const size_t nfs = static_cast<size_t>(nf);
            const size_t keys = static_cast<size_t>(filler_order_keys(c.geom.dim));
            for (DevBuf<int>* b : {&c.fo_key, &c.fo_tmp, &c.fo_perm, &c.fo_fid, &c.fo_fid_tmp}) b->alloc(nfs);
            for (DevBuf<int>* b : {&c.fo_count, &c.fo_offset, &c.fo_cursor}) b->alloc(keys);
            c.fo_skip.alloc(1);
            c.fo_scratch.alloc(2 * nfs * static_cast<size_t>(filler_order_vectors()));
            iota_kernel<<<work_grid(reinterpret_cast<const void*>(iota_kernel), nf, RED_THREADS), RED_THREADS, 0, s>>>(
                c.fo_fid.p, nf);
            count_launch();
            SPG_CHECK_LAUNCH();
        }
    }
    c.metrics_rows = 0;
    c.metrics.alloc(static_cast<size_t>(std::max(c.prm.gp_max_iter, c.prm.filler_only_iters) + 1));
    if (!c.st.p) c.st.alloc(1);
    if (!c.hst) SPG_CUDA(cudaMallocHost(&c.hst, sizeof(DevState)));
    if (!c.scratch_d.p) c.scratch_d.alloc(16);
}

// One objAndGrad evaluation at the positions of `pos_role`, gradient into `grad_role`
// (eplace.cpp:136-203).
// One objAndGrad evaluation (eplace.cpp:136-203) at the current node positions (scattered
// by the update kernels; pos_role >= 0 scatters that role first), gradient into grad_role.
// The WA pass 1 depends only on the positions, so it runs on a side stream, overlapping
// the density -> Poisson chain; the assembly joins both.
// `stepped`: the step kernel already added the opt nodes' charge (loop evaluations).
// rho and tau partials from the fixed-point maps (clearing them); with a tensor-core plan
// the same launch also writes the solve's first operand. Returns whether it did.
bool rho_and_split(Context& c, const DevPtrs& p, cudaStream_t s) {
    RhoOperand op{};
    if (tc_rho_operand(*c.plan, &op)) {
        launch_rho_prep(p, op.planes, op.plane_stride, op.ld, op.sums, s);
        return true;
    }
    launch_rho_overflow(p, 0, 1, s);
    return false;
}

bool wa_serial() {
    static const bool on = [] {
        const char* e = std::getenv("SPG_WA_SERIAL");
        return e && e[0] == '1';
    }();
    return on;
}

// The WA pass of an evaluation on the side stream, after the work queued on the main stream
// so far (it reads the cells' node positions); the assembly joins it.
void fork_wa(Context& c, const DevPtrs& p) {
    SPG_CUDA(cudaEventRecord(c.ev_fork, c.stream));
    SPG_CUDA(cudaStreamWaitEvent(c.side, c.ev_fork, 0));
    launch_wa_nets(p, c.wa_classes, &p.st->gamma, 0.f, 1, c.side);
    launch_wl_cells(p, c.side);
    SPG_CUDA(cudaEventRecord(c.ev_join, c.side));
}

// wa_forked: the loop's step already forked the WA pass (after the cells' step launch).
void evaluate(Context& c, const DevPtrs& p, int pos_role, int grad_role, int count, bool fused_reduce = false,
              bool stepped = false, cudaGraphConditionalHandle loop_cond = 0, bool wa_forked = false) {
    cudaStream_t s = c.stream;
    if (pos_role >= 0) launch_scatter(p, pos_role, s);
    if (wa_serial()) {
        launch_wa_nets(p, c.wa_classes, &p.st->gamma, 0.f, 1, s);
        launch_wl_cells(p, s);
    } else if (!wa_forked) {
        fork_wa(c, p);
    }
    if (stepped) launch_density_rest(p, s);
    else launch_density_accumulate(p, s);
    const bool fused = rho_and_split(c, p, s);
    poisson_solve(*c.plan, 1, c.rho.p, c.phi.p, c.ex.p, c.ey.p, s, fused);
    launch_gather_opt_large(p, s);
    if (!wa_serial()) SPG_CUDA(cudaStreamWaitEvent(s, c.ev_join, 0));
    if (fused_reduce) launch_assemble_reduce(p, s, loop_cond);
    else launch_assemble(p, pos_role >= 0 ? pos_role : R_U, grad_role, count, s);
}

// A tensor-core Poisson solve that gave up a bounded pipeline wait leaves its code in the
// plan's flag; it becomes the stage's error, so the state read below raises it.
__global__ void fold_error_kernel(DevState* st, const int* flag) {
    const int e = *flag;
    if (e) atomicCAS(&st->error, 0, e);
}

void read_state(Context& c) {
    if (c.plan) {
        if (const int* f = tc_error_flag(*c.plan)) {
            fold_error_kernel<<<1, 1, 0, c.stream>>>(c.st.p, f);
            count_launch();
            SPG_CHECK_LAUNCH();
        }
    }
    SPG_CUDA(cudaMemcpyAsync(c.hst, c.st.p, sizeof(DevState), cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(host_wait(c.stream));
    if (c.hst->error) {
        const int e = c.hst->error;
        throw Error(e, e == SPG_E_NON_FINITE ? "GP/evaluate: non-finite coordinate, gradient or metric"
                     : e == SPG_E_OUT_OF_CORE ? "GP: node outside core"
                     : e == SPG_E_CAPACITY ? "GP: stagnation snapshot capacity exceeded"
                     : e == SPG_E_CUDA ? "GP: a tensor-core Poisson solve gave up a bounded pipeline wait"
                                           : "GP: device error");
    }
}

// hpwlReference (src/gp/lambda_schedule.h:11-20)
double hpwl_reference(const spg_params& p, double initial, bool filler_only) {
    const bool rel = p.lambda_schedule_relative != 0 && !filler_only;
    const double ref = rel ? initial * p.delta_hpwl_relative : static_cast<double>(p.delta_hpwl_ref);
    if (initial == 0.0 && rel) return p.delta_hpwl_ref;
    if (!(ref > 0.0) || !std::isfinite(ref)) throw Error(SPG_E_INVALID, "invalid effective HPWL reference");
    return ref;
}

__global__ void gather_pos_kernel(DevPtrs p) {
    float* pos = p.pool + static_cast<size_t>(p.st->role[R_POS]) * p.vec_stride;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < p.n_opt; k += gridDim.x * blockDim.x) {
        const int i = p.opt_idx[k];
        pos[k] = p.x[i];
        pos[p.n_opt + k] = p.y[i];
    }
}

__global__ void init_state_kernel(DevPtrs p, int stage, int max_iter, float target_tau) {
    DevState* st = p.st;
    memset(st, 0, sizeof(DevState));
    for (int r = 0; r < NUM_ROLES; ++r) st->role[r] = r;
    st->stage = stage;
    st->max_iter = max_iter;
    st->target_tau = target_tau;
    st->lambda = 1.f;
    st->a = 1.f;
    st->alpha = 1.f;
    st->alpha0 = 1.f;
    st->tries = 1;
    st->best_tau = INFINITY;
    st->ref_tau = INFINITY;
    st->snap_copy_to = -1;
    st->rollback_iter = -1;
    st->deliver = 0;
    st->pause_iter = INT_MAX;
    st->pause_row = INT_MAX;
    st->diag_mid = 0;
    st->diag_mid_hit = 0;
}

__global__ void gamma_init_kernel(DevPtrs p) {
    // computeGamma(1.f, stepX) (eplace.cpp:248): tau = 1 lies in the pow branch
    float g = __fmul_rn(8.0f, p.step_x_gamma);
    g = __fmul_rn(g, powf(10.0f, __fsub_rn(__fmul_rn(20.0f / 9.0f, __fsub_rn(1.0f, 0.1f)), 1.0f)));
    p.st->gamma = fmaxf(g, 1e-4f);
    p.st->lambda = 1.f;
}

__global__ void set_hpwl_ref_kernel(DevPtrs p, double ref) { p.st->hpwl_ref = ref; }

__global__ void set_pause_kernel(DevState* st, int at_iter, int at_row, int diag_mid) {
    st->pause_iter = at_iter;
    st->pause_row = at_row;
    st->diag_mid = diag_mid;
}

// The opt nodes' positions at the evaluation point held by `role` (R_U: the last evaluated
// point) written over a copy of the node arrays (whose filler entries are only rewritten when
// the stage ends): every node's position at that point.
__global__ void eval_positions_opt_kernel(DevPtrs p, int role, float* out_x, float* out_y) {
    const float* u = role_ptr(p, role);
    const int n = p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = p.opt_idx[k];
        out_x[i] = u[k];
        out_y[i] = u[n + k];
    }
}

// Every node's position at the evaluation point of `role` into the host arrays x, y (total
// entries each); complete on return.
void download_eval_positions(Context& c, const DevPtrs& p, int role, float* x, float* y) {
    const size_t n = static_cast<size_t>(c.total);
    if (n == 0) return;
    cudaStream_t s = c.stream;
    c.frame_x.alloc(n);
    c.frame_y.alloc(n);
    SPG_CUDA(cudaMemcpyAsync(c.frame_x.p, c.x.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    SPG_CUDA(cudaMemcpyAsync(c.frame_y.p, c.y.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if (p.n_opt > 0) {
        eval_positions_opt_kernel<<<work_grid(reinterpret_cast<const void*>(eval_positions_opt_kernel), p.n_opt,
                                              RED_THREADS),
                                    RED_THREADS, 0, s>>>(p, role, c.frame_x.p, c.frame_y.p);
        count_launch();
        SPG_CHECK_LAUNCH();
    }
    download_pair(x, c.frame_x.p, y, c.frame_y.p, n * sizeof(float), s);
}

// Final metrics at the delivered positions: overflow and HPWL (eplace.cpp:484-488).
__global__ void final_metrics_kernel(DevPtrs p, double* out) {
    double over = 0.0, hp = 0.0;
    for (int j = threadIdx.x; j < RED_CAP; j += blockDim.x) {
        over += p.partials[SLOT_OVERFLOW * RED_CAP + j];
        hp += p.partials[SLOT_HPWL * RED_CAP + j];
    }
    __shared__ double so[256], sh[256];
    so[threadIdx.x] = over;
    sh[threadIdx.x] = hp;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            so[threadIdx.x] += so[threadIdx.x + w];
            sh[threadIdx.x] += sh[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = p.movable_area_scaled > 0.0 ? static_cast<double>(static_cast<float>(so[0] / p.movable_area_scaled)) : 0.0;
        out[1] = sh[0];
    }
}

void final_metrics(Context& c, const DevPtrs& p, float* overflow, double* hpwl) {
    cudaStream_t s = c.stream;
    launch_scatter(p, R_POS, s);
    launch_density_accumulate(p, s);
    launch_rho_overflow(p, 0, 1, s);
    launch_wa_nets(p, c.wa_classes, &p.st->gamma, 0.f, 1, s);
    final_metrics_kernel<<<1, 256, 0, s>>>(p, c.scratch_d.p);
    count_launch();
    SPG_CHECK_LAUNCH();
    double out[2];
    SPG_CUDA(cudaMemcpyAsync(out, c.scratch_d.p, sizeof(out), cudaMemcpyDeviceToHost, s));
    SPG_CUDA(host_wait(s));
    *overflow = static_cast<float>(out[0]);
    *hpwl = out[1];
}

// One loop pass: the step the last decisions asked for (the next Nesterov step, or a
// redoIfOvershot re-evaluation step, nesterov.cpp:97-119,158-166), the evaluation at the new
// u, and the redo test / next decisions. A re-evaluation takes a pass of its own, so the loop
// body is the same for both.
// One loop pass; in a captured body the assembly's last block also sets the WHILE node's
// condition (loop_cond), so the body needs no kernel of its own for it.
void enqueue_iteration(Context& c, const DevPtrs& p, cudaGraphConditionalHandle loop_cond = 0) {
    cudaStream_t s = c.stream;
    // The cells' step, the WA pass forked after it (WA reads only cell positions), then the
    // fillers' step beside WA: WA then overlaps the fillers' step instead of holding the SMs
    // that the density -> Poisson chain needs (the chain started up to 22 us late behind it).
    // 6426-6491 iter/s at 211k cells against 6212-6368 as one launch. SPG_SPLIT_STEP=0: one launch.
    static const bool split = [] {
        const char* e = std::getenv("SPG_SPLIT_STEP");
        return !(e && e[0] == '0');
    }();
    if (split && !wa_serial() && p.filler_k0 > 0 && p.filler_k0 < p.n_opt) {
        launch_update_range(p, 0, p.filler_k0, s);
        fork_wa(c, p);
        launch_update_range(p, p.filler_k0, p.n_opt, s);
        evaluate(c, p, -1, R_G, 1, true, true, loop_cond, true);
        return;
    }
    launch_update(p, s);
    evaluate(c, p, -1, R_G, 1, true, true, loop_cond);
}

// Host-driven loop: one state read per pass.
void host_loop(Context& c, const DevPtrs& p, int max_iter) {
    read_state(c);
    // the device sets `done` by max_iter; this bound guards the host loop itself
    const int64_t pass_bound = static_cast<int64_t>(max_iter + 2) * std::max(c.prm.max_backtrack, 1);
    int64_t passes = 0;
    while (!c.hst->done && c.hst->iter < c.hst->pause_iter && c.hst->rows <= c.hst->pause_row &&
           !(c.hst->diag_mid && c.hst->diag_mid_hit)) {
        if (++passes > pass_bound) throw Error(SPG_E_STATE, "GP loop exceeded its iteration bound");
        enqueue_iteration(c, p);
        read_state(c);
    }
}

}  // namespace

// Binds the calling thread's device allocations and host copies to one context: buffers come
// from the pool on its stream and copies go through its pinned staging memory. The
// context's earlier work is waited for first, so the staging memory can be reused.
struct CtxScope {
    AllocScope alloc;
    Staging* prev;
    explicit CtxScope(Context& c) : alloc(c.stream), prev(t_staging) {
        SPG_CUDA(host_wait(c.stream));
        c.staging.s = c.stream;
        c.staging.used = 0;
        t_staging = &c.staging;
    }
    ~CtxScope() { t_staging = prev; }
    CtxScope(const CtxScope&) = delete;
    CtxScope& operator=(const CtxScope&) = delete;
};

struct LoopGraph {
    cudaGraph_t graph = nullptr;  // the template the executable was made from (kept with it)
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle loop_h{};
    std::vector<cudaGraphNode_t> body_nodes;  // the WHILE body's kernel nodes, in launch order
    bool patchable = true;                    // the last patch attempt worked (or none was made)
    DevPtrs sig{};
    const void* plan = nullptr;
    int64_t body_kernels = 0;
    ~LoopGraph() { reset(); }
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        body_nodes.clear();
        patchable = true;
    }
};

namespace {

// The whole iteration loop as one CUDA graph:
//   WHILE (!done) {                      loop_h, set by the assembly's last block
//     step (Nesterov or re-evaluation); evaluate; norms, decisions and loop_h in the assembly
//   }
// Built once per context and stage layout, relaunched on later runs with the same buffers.
// SPG_GRAPH_STATS=1: print a body graph's node and edge counts, and how many edges are
// programmatic (PDL) ones, to stderr.
void graph_stats(const char* name, cudaGraph_t g) {
    static const bool on = [] {
        const char* e = std::getenv("SPG_GRAPH_STATS");
        return e && e[0] == '1';
    }();
    if (!on || !g) return;
    size_t nodes = 0, edges = 0;
    cudaGraphGetNodes(g, nullptr, &nodes);
    cudaGraphGetEdges_v2(g, nullptr, nullptr, nullptr, &edges);
    std::vector<cudaGraphNode_t> from(edges), to(edges);
    std::vector<cudaGraphEdgeData> data(edges);
    size_t n = edges;
    int prog = 0;
    if (edges && cudaGraphGetEdges_v2(g, from.data(), to.data(), data.data(), &n) == cudaSuccess)
        for (size_t i = 0; i < n; ++i) prog += data[i].type == cudaGraphDependencyTypeProgrammatic;
    std::fprintf(stderr, "[spg graph] %s: %zu nodes, %zu edges, %d programmatic\n", name, nodes, edges, prog);
}

void graph_note(const char* what) {
    static const bool on = [] {
        const char* e = std::getenv("SPG_GRAPH_STATS");
        return e && e[0] == '1';
    }();
    if (on) std::fprintf(stderr, "[spg graph] %s\n", what);
}

// The kernel nodes of a graph in creation (launch) order, or false when it holds any other
// kind of node.
bool kernel_nodes(cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return false;
    out.resize(n);
    if (n && cudaGraphGetNodes(g, out.data(), &n) != cudaSuccess) return false;
    for (cudaGraphNode_t nd : out) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) return false;
    }
    return true;
}

// A new netlist's loop with the same kernel sequence: capture the body alone (a plain graph,
// cheap to build and to destroy) and write its kernel arguments and launch shapes into the
// executable's body nodes. Keeping the template avoids destroying a graph that holds a
// conditional node per request, which is slow and stalls other threads' CUDA calls.
// Returns false (the executable is then rebuilt) when the sequences differ in length,
// kernels or dependency counts.
bool patch_loop_graph(Context& c, const DevPtrs& p, LoopGraph& lg) {
    cudaStream_t s = c.stream;
    const int64_t launches0 = g_launches;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    bool fine = true;
    try {
        enqueue_iteration(c, p, lg.loop_h);
    } catch (const Error&) {
        fine = false;
    }
    cudaGraph_t nb = nullptr;
    const bool ended = cudaStreamEndCapture(s, &nb) == cudaSuccess;
    g_launches = launches0;
    struct Drop {
        cudaGraph_t g;
        ~Drop() {
            if (g) cudaGraphDestroy(g);
        }
    } drop{nb};
    std::vector<cudaGraphNode_t> nodes;
    if (!fine || !ended || !nb || !kernel_nodes(nb, nodes) || nodes.size() != lg.body_nodes.size()) {
        cudaGetLastError();
        return false;
    }
    std::vector<cudaKernelNodeParams> kp(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        cudaKernelNodeParams old{};
        size_t da = 0, db = 0;
        if (cudaGraphKernelNodeGetParams(nodes[i], &kp[i]) != cudaSuccess ||
            cudaGraphKernelNodeGetParams(lg.body_nodes[i], &old) != cudaSuccess || kp[i].func != old.func ||
            cudaGraphNodeGetDependencies(nodes[i], nullptr, &da) != cudaSuccess ||
            cudaGraphNodeGetDependencies(lg.body_nodes[i], nullptr, &db) != cudaSuccess || da != db) {
            cudaGetLastError();
            return false;
        }
    }
    for (size_t i = 0; i < nodes.size(); ++i)
        if (cudaGraphExecKernelNodeSetParams(lg.exec, lg.body_nodes[i], &kp[i]) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
    return true;
}

bool build_loop_graph(Context& c, const DevPtrs& p, LoopGraph& lg) {
    const CallClock clk_all("build_loop_graph (capture, update or instantiate, destroy)", __LINE__);
    if (lg.exec && lg.patchable && !lg.body_nodes.empty()) {
        if (patch_loop_graph(c, p, lg)) {
            graph_note("loop graph patched in place");
            lg.sig = p;
            lg.plan = c.plan.get();
            return true;
        }
        lg.patchable = false;
    }
    // an executable graph of an earlier netlist is updated in place when the new capture
    // allows it (same topology, new kernel arguments), which costs far less than a new
    // instantiation; otherwise it is replaced
    cudaGraphExec_t old_exec = lg.exec;
    cudaGraph_t old_graph = lg.graph;
    lg.exec = nullptr;
    lg.graph = nullptr;
    struct DropOld {
        cudaGraphExec_t& e;
        cudaGraph_t& g;
        ~DropOld() {
            const CallClock clk_("cudaGraphExecDestroy / cudaGraphDestroy", __LINE__);
            if (e) cudaGraphExecDestroy(e);
            if (g) cudaGraphDestroy(g);
        }
    } drop_old{old_exec, old_graph};
    cudaStream_t s = c.stream;
    const int64_t launches0 = g_launches;
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    cudaGraph_t g = nullptr;
    if (!ok(cudaGraphCreate(&g, 0))) return false;
    lg.graph = g;
    cudaGraphConditionalHandle loop_h;
    if (!ok(cudaGraphConditionalHandleCreate(&loop_h, g, 1, cudaGraphCondAssignDefault))) return false;
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = loop_h;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    if (!ok(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp))) return false;
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    lg.loop_h = loop_h;
    if (!ok(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)))
        return false;
    bool fine = true;
    try {
        const int64_t k0 = g_launches;
        enqueue_iteration(c, p, loop_h);
        lg.body_kernels = g_launches - k0;
    } catch (const Error&) {
        fine = false;
    }
    cudaGraph_t out = nullptr;
    const bool ended = ok(cudaStreamEndCapture(s, &out));
    g_launches = launches0;  // executions are counted after each launch
    if (!fine || !ended) {
        cudaGetLastError();
        return false;
    }
    graph_stats("loop body", body);
    bool updated_in_place = false;
    if (old_exec) {
        cudaGraphExecUpdateResultInfo info{};
        cudaError_t ue;
        {
            const CallClock clk_("cudaGraphExecUpdate", __LINE__);
            ue = cudaGraphExecUpdate(old_exec, g, &info);
        }
        if (ue == cudaSuccess) {
            lg.exec = old_exec;
            old_exec = nullptr;
            updated_in_place = true;
        } else {
            cudaGetLastError();
        }
        graph_note(lg.exec ? "loop graph updated in place" : "loop graph re-instantiated");
    }
    if (!lg.exec && !ok(cudaGraphInstantiate(&lg.exec, g, 0))) {
        cudaGetLastError();
        return false;
    }
    // node-level patches address the nodes of the graph the executable was instantiated
    // from: not this template after an update in place
    lg.patchable = !updated_in_place && kernel_nodes(body, lg.body_nodes);
    if (!lg.patchable) lg.body_nodes.clear();
    cudaGetLastError();
    lg.sig = p;
    lg.plan = c.plan.get();
    return true;
}

bool graph_loop(Context& c, const DevPtrs& p) {
    std::shared_ptr<LoopGraph> lgp;
    for (auto& e : c.loop_graphs)
        if (e.first == c.plan.get()) lgp = e.second;
    if (!lgp) {
        lgp = std::make_shared<LoopGraph>();
        c.loop_graphs.emplace_back(c.plan.get(), lgp);
    }
    LoopGraph& lg = *lgp;
    const bool same = lg.exec && lg.plan == c.plan.get() && std::memcmp(&lg.sig, &p, sizeof(DevPtrs)) == 0;
    const auto tb = std::chrono::steady_clock::now();
    const bool built = !same && build_loop_graph(c, p, lg);
    if (!same) c.last_graph_build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
    if (!same && !built) {
        lg.reset();
        c.use_graph = false;  // this device/driver refused the conditional graph: host loop
        return false;
    }
    const int64_t before = static_cast<int64_t>(c.hst->iter) + c.hst->redos;
    SPG_CUDA(cudaGraphLaunch(lg.exec, c.stream));
    read_state(c);
    // one body per pass: per applied update and per re-evaluation
    g_launches += (static_cast<int64_t>(c.hst->iter) + c.hst->redos - before) * lg.body_kernels;
    return true;
}

// What constructing EPlace and buildOptSet do for a stage (gp_stage.cpp:175-177,
// eplace.cpp:82-133): the grid rebuilt with the current flags, then the stage's opt set.
void prepare_stage(Context& c, int stage, HostTimer* ht) {
    if (!c.mirror_valid) {
        c.x_mirror.resize(c.num_nodes);
        c.y_mirror.resize(c.num_nodes);
        download_bytes(c.x_mirror.data(), c.x.p, c.num_nodes * sizeof(float), c.stream);
        download_bytes(c.y_mirror.data(), c.y.p, c.num_nodes * sizeof(float), c.stream);
    }
    // the opt set is built while the pool builds the grid's static maps
    grid_init(c, c.prm.target_density, c.prm.gp_bin_dim, c.x_mirror, c.y_mirror, [&] { stage_setup(c, stage); });
    c.mirror_valid = false;  // the stage moves the positions
    if (ht) ht->mark("grid_init+stage_setup");
}

// EPlace::run (eplace.cpp:223-526) for one stage, device-resident.
void stage_run(Context& c, int stage, spg_result* res) {
    SPG_REQUIRE(stage >= SPG_STAGE_MGP && stage <= SPG_STAGE_CGP, SPG_E_INVALID, "unknown stage");
    HostTimer ht;
    std::memset(res, 0, sizeof(*res));
    res->rollback_iter = -1;
    cudaStream_t s = c.stream;
    c.have_eval = false;
    prepare_stage(c, stage, &ht);
    if (c.n_opt == 0) return;  // "no nodes to optimise" (eplace.cpp:232-236)
    const bool filler_only = stage == SPG_STAGE_FILLER_ONLY;
    const float target_tau = stage == SPG_STAGE_CGP ? c.prm.cgp_target_overflow : c.prm.target_overflow;
    const int max_iter = filler_only ? c.prm.filler_only_iters : c.prm.gp_max_iter;
    DevPtrs p = c.ptrs();
    init_state_kernel<<<1, 1, 0, s>>>(p, stage, max_iter, target_tau);
    gather_pos_kernel<<<work_grid(reinterpret_cast<const void*>(gather_pos_kernel), p.n_opt, RED_THREADS),
                        RED_THREADS, 0, s>>>(p);
    count_launch(2);
    SPG_CHECK_LAUNCH();
    launch_clamp_role(p, R_POS, s);
    // lambda_0 probe (eplace.cpp:248-259)
    gamma_init_kernel<<<1, 1, 0, s>>>(p);
    count_launch();
    evaluate(c, p, R_POS, R_GA, 0);
    launch_ctl_lambda_init(p, s);
    read_state(c);
    const double ref = hpwl_reference(c.prm, c.hst->hpwl, filler_only);
    res->initial_hpwl = c.hst->hpwl;
    res->initial_overflow = c.hst->tau;
    res->initial_lambda = c.hst->lambda;
    set_hpwl_ref_kernel<<<1, 1, 0, s>>>(p, ref);
    count_launch();
    ht.mark("lambda_probe");

    if (!filler_only && c.hst->tau < target_tau) {
        // already converged: take no step (eplace.cpp:278-296)
        c.have_eval = true;
        c.eval_role = c.eval_prev_role = R_POS;
        final_metrics(c, p, &res->overflow, &res->hpwl);
        res->converged = 1;
        return;
    }

    cudaEvent_t e0 = c.ev_t0, e1 = c.ev_t1;
    SPG_CUDA(cudaEventRecord(e0, s));
    launch_stage_clock(p, s);
    // optimizer init: u = v = uPrev = vPrev = pos, g = gPrevTmp = 0 (nesterov.cpp:174-185)
    for (int r : {R_U, R_V, R_UPREV, R_VPREV}) launch_copy_role(p, r, R_POS, s);
    // estimateInitialStep (nesterov.cpp:190-218): two uncounted evaluations
    evaluate(c, p, R_U, R_GA, 0);
    launch_init_norms(p, s);
    launch_ctl_init_scale(p, 0.1f, s);
    launch_init_perturb(p, s);
    evaluate(c, p, R_PROBE, R_GB, 0);
    launch_init_diff(p, s);
    launch_ctl_init_finish(p, s);

    // first evaluation of iteration 0, its norms, and the redo test (a no-op at iteration 0)
    evaluate(c, p, R_U, R_G, 1, true);
    ht.mark("init_enqueue");
    c.last_run_graph = false;
    c.last_graph_build_ms = 0.0;
    if (max_iter > 0) {
        // the loop runs in segments: it pauses at the filler-reorder iterations (the fillers are
        // reordered, filler_order.cu) and after the metrics rows of the iteration callback's
        // iterations (the callback runs at that evaluation point), and resumes where it stopped
        size_t next = 0;
        const bool callback = c.iter_fn && c.iter_stride > 0;
        int next_row = callback ? 0 : INT_MAX;
        bool mid_pending = c.mid_fn && stage != SPG_STAGE_FILLER_ONLY && c.prm.gp_stagnation_window > 0;
        auto arm = [&] {
            const int at = (c.fo_active && next < c.fo_pauses.size()) ? c.fo_pauses[next] : INT_MAX;
            set_pause_kernel<<<1, 1, 0, s>>>(c.st.p, at, next_row, mid_pending ? 1 : 0);
            count_launch();
            SPG_CHECK_LAUNCH();
        };
        // every node's position at the evaluation point u, with the metrics rows so far readable
        auto frame = [&] {
            c.metrics_rows = std::min(c.hst->rows, max_iter);
            c.have_eval = true;  // spg_eval_positions inside the callback: u and the point before
            c.eval_role = R_U;
            c.eval_prev_role = R_UPREV;
            c.frame_hx.resize(c.total);
            c.frame_hy.resize(c.total);
            download_eval_positions(c, p, R_U, c.frame_hx.data(), c.frame_hy.data());
        };
        // the callbacks due at the current state (the loop has paused right after their row)
        auto service = [&] {
            bool any = false;
            if (callback && c.hst->rows > next_row && !c.hst->error) {
                // the row of iteration next_row is written and u is its evaluation point
                frame();
                c.iter_fn(c.iter_user, stage, next_row, c.frame_hx.data(), c.frame_hy.data());
                next_row = next_row > INT_MAX - c.iter_stride ? INT_MAX : next_row + c.iter_stride;
                any = true;
            }
            if (mid_pending && c.hst->diag_mid_hit && !c.hst->error) {
                // the stagnation counter reached half the window at iteration rows - 1
                frame();
                c.mid_fn(c.mid_user, stage, c.hst->rows - 1, c.frame_hx.data(), c.frame_hy.data());
                mid_pending = false;
                any = true;
            }
            return any;
        };
        arm();
        read_state(c);  // the state the first segment starts from: iteration 0 evaluated, its row written
        if (service() && !c.hst->done) arm();
        c.last_run_graph = c.use_graph;
        for (;;) {
            if (c.hst->done || c.hst->error) break;
            if (c.last_run_graph) c.last_run_graph = graph_loop(c, p);
            if (!c.last_run_graph) host_loop(c, p, max_iter);
            bool resume = service();
            if (c.hst->done || c.hst->error) break;
            if (c.fo_active && next < c.fo_pauses.size() && c.hst->iter >= c.fo_pauses[next]) {
                launch_filler_order(p, c.filler_order_bufs(), s);
                ++next;
                resume = true;
            }
            if (!resume) break;
            arm();
        }
    }
    // the last evaluation point: u, unless the loop ran to max_iter, which takes the last step
    // (v is delivered) and evaluates its u once more without counting it: then the point is
    // uPrev and the one before it was rotated into the spare slot uNew
    c.have_eval = true;
    const bool ran_out = max_iter > 0 && !c.hst->converged && !c.hst->stagnated;
    c.eval_role = ran_out ? R_UPREV : R_U;
    c.eval_prev_role = ran_out ? R_UNEW : R_UPREV;
    ht.mark("loop");
    if (ht.on) ht.line += " (graph_build=" + std::to_string(c.last_graph_build_ms).substr(0, 6) + ")";
    SPG_CUDA(cudaEventRecord(e1, s));
    launch_deliver(p, s);
    final_metrics(c, p, &res->overflow, &res->hpwl);
    launch_check_geometry(p, c.core_lx, c.core_ly, c.core_hx, c.core_hy, c.dw.p, c.dh.p, s);
    read_state(c);
    ht.mark("final");
    float ms = 0.f;
    SPG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const DevState& h = *c.hst;
    res->iterations = h.rows;
    res->converged = h.converged;
    res->stagnated = h.stagnated;
    res->rollback_iter = h.stagnated ? h.rollback_iter : -1;
    res->evaluations = h.evals;
    res->elapsed_ms = ms;
    c.metrics_rows = std::min(h.rows, max_iter);
    if (res->converged && !(res->overflow < target_tau))
        throw Error(SPG_E_CONVERGENCE, "delivered overflow disagrees with convergence");
    if (res->stagnated) {
        spg_iter_metrics row{};
        SPG_CUDA(cudaMemcpy(&row, c.metrics.p + res->rollback_iter, sizeof(row), cudaMemcpyDeviceToHost));
        if (!(std::fabs(double(res->overflow) - row.overflow) <= 1e-7 + 1e-6 * std::fabs(row.overflow) &&
              std::fabs(res->hpwl - row.hpwl) <= 1e-6 + 1e-10 * std::fabs(row.hpwl)))
            throw Error(SPG_E_ROLLBACK, "delivered metrics disagree with rollback point");
    }
}

// lambda and gamma of an evaluation outside the loop; `done` set, so the loop body's step
// kernel applies no step (it rasterizes the current u) and its decisions are skipped.
__global__ void set_eval_kernel(DevState* st, float lambda, float gamma) {
    st->lambda = lambda;
    st->gamma = gamma;
    st->done = 1;
}

// EPlace::Impl::objAndGrad (eplace.cpp:136-203) at opt-set positions pos (x then y, the opt
// order of buildOptSet) for the given lambda and gamma, through the GP loop body's own kernels
// (enqueue_iteration): the step kernel's fixed-point scatter of u, the WA pass 1 with HPWL,
// WA pass 2 of the cells, the rest-list scatter, rho and tau, the Poisson solve, the large
// nodes' gather, and the fused assembly (cell gather, preconditioned gradient). grad gets
// 2*nOpt floats; out[0..4] = WA value, tau, HPWL, sum|grad WL|, sum|q xi|; *n_opt the opt-set
// size. With pos = NULL only *n_opt is set. The grid and opt set are rebuilt for `stage` from
// the context's positions and flags first, as constructing EPlace does.
void eval_grad(Context& c, int stage, float lambda, float gamma, const float* pos, float* grad, double* out,
               int* n_opt) {
    SPG_REQUIRE(stage >= SPG_STAGE_MGP && stage <= SPG_STAGE_CGP, SPG_E_INVALID, "unknown stage");
    prepare_stage(c, stage, nullptr);
    *n_opt = c.n_opt;
    if (!pos || c.n_opt == 0) return;
    SPG_REQUIRE(grad && out, SPG_E_INVALID, "eval_grad: null output");
    cudaStream_t s = c.stream;
    DevPtrs p = c.ptrs();
    init_state_kernel<<<1, 1, 0, s>>>(p, stage, 1, 0.f);
    set_eval_kernel<<<1, 1, 0, s>>>(p.st, lambda, gamma);
    count_launch(2);
    SPG_CHECK_LAUNCH();
    const size_t n2 = 2 * static_cast<size_t>(c.n_opt);
    // the roles start as the identity, so role R_U is pool slot R_U
    upload_bytes(c.pool.p + static_cast<size_t>(R_U) * c.vec_stride, pos, n2 * sizeof(float), s);
    launch_scatter(p, R_U, s);  // node positions for the WA pass and the large nodes
    enqueue_iteration(c, p);
    read_state(c);
    download_bytes(grad, c.pool.p + static_cast<size_t>(c.hst->role[R_G]) * c.vec_stride, n2 * sizeof(float), s);
    const DevState& h = *c.hst;
    out[0] = h.wl_obj;
    out[1] = h.tau;
    out[2] = h.hpwl;
    out[3] = h.sum_wl;
    out[4] = h.sum_den;
}

__global__ void set_alpha0_kernel(DevState* st, float a) { st->alpha0 = a; }

// NesterovOptimizer::step called `steps` times (src/numeric/cpu/nesterov.cpp:51-122) on the
// quadratic test objective of quad_eval_kernel, with the GP loop's own step kernel, redo test
// and step decisions: the optimizer vectors in the role pool, estimateInitialStep's two
// uncounted evaluations (or alpha0 = init_step when positive), then one counted evaluation
// per pass. n coordinates (even: the pool holds them as n/2 x-y pairs); no constraint, as in
// the reference's optimizer tests. pos: the start in, the current solution v out.
// out[0..3] = objective of the last counted evaluation, evaluations, step size, re-evaluations.
void nesterov_quadratic(int n, const float* coef, const float* target, float* pos, int steps, int use_bb,
                        int backtrack, int max_backtrack, float init_step, double* out) {
    SPG_REQUIRE(n >= 2 && n % 2 == 0 && steps >= 0 && max_backtrack >= 1, SPG_E_INVALID,
                "nesterov_quadratic: n must be even and >= 2, steps >= 0, max_backtrack >= 1");
    SPG_REQUIRE(coef && target && pos && out, SPG_E_INVALID, "nesterov_quadratic: null pointer");
    cudaStream_t s = nullptr;
    SPG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            host_wait(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    const size_t nn = static_cast<size_t>(n);
    const size_t stride = (nn + 63) / 64 * 64;
    DevBuf<float> pool, lo, hi, c, t;
    DevBuf<DevState> st;
    DevBuf<double> partials;
    pool.alloc(stride * NUM_ROLES);
    pool.zero(s);
    lo.upload(std::vector<float>(nn, -INFINITY), s);
    hi.upload(std::vector<float>(nn, INFINITY), s);
    c.upload(coef, nn, s);
    t.upload(target, nn, s);
    st.alloc(1);
    partials.alloc(static_cast<size_t>(RED_SLOTS) * RED_CAP);
    partials.zero(s);
    DevPtrs p{};
    p.n_opt = n / 2;
    p.pool = pool.p;
    p.vec_stride = stride;
    p.st = st.p;
    p.partials = partials.p;
    p.opt_lo = lo.p;
    p.opt_hi = hi.p;
    p.filler_k0 = p.n_opt;
    p.use_bb = use_bb;
    p.backtrack = backtrack;
    p.max_backtrack = max_backtrack;
    init_state_kernel<<<1, 1, 0, s>>>(p, SPG_STAGE_MGP, steps, 0.f);
    count_launch();
    SPG_CHECK_LAUNCH();
    upload_bytes(pool.p + static_cast<size_t>(R_POS) * stride, pos, nn * sizeof(float), s);
    DevState h{};
    auto read = [&] {
        SPG_CUDA(cudaMemcpyAsync(&h, st.p, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        SPG_CUDA(host_wait(s));
        if (h.error) throw Error(h.error, "nesterov_quadratic: non-finite coordinate or gradient");
    };
    if (steps > 0) {
        // NesterovOptimizer::init (nesterov.cpp:173-186)
        for (int r : {R_U, R_V, R_UPREV, R_VPREV}) launch_copy_role(p, r, R_POS, s);
        if (init_step > 0.f) {
            set_alpha0_kernel<<<1, 1, 0, s>>>(st.p, init_step);
            count_launch();
            SPG_CHECK_LAUNCH();
        } else {
            launch_quad_eval(p, c.p, t.p, R_U, R_GA, 0, s);
            launch_init_norms(p, s);
            launch_ctl_init_scale(p, 0.1f, s);
            launch_init_perturb(p, s);
            launch_quad_eval(p, c.p, t.p, R_PROBE, R_GB, 0, s);
            launch_init_diff(p, s);
            launch_ctl_init_finish(p, s);
        }
        launch_quad_eval(p, c.p, t.p, R_U, R_G, 1, s);
        read();
        // each pass is a step or a re-evaluation: at most max_backtrack per step
        const int64_t bound = static_cast<int64_t>(steps + 1) * max_backtrack + 2;
        int64_t passes = 0;
        while (!h.done) {
            SPG_REQUIRE(++passes <= bound, SPG_E_STATE, "nesterov_quadratic: pass bound exceeded");
            launch_quad_step(p, s);
            launch_quad_eval(p, c.p, t.p, R_U, R_G, 1, s);
            read();
        }
        download_bytes(pos, pool.p + static_cast<size_t>(h.role[R_V]) * stride, nn * sizeof(float), s);
    }
    out[0] = h.wl_obj;
    out[1] = static_cast<double>(h.evals);
    out[2] = steps > 0 ? h.alpha : 0.0;
    out[3] = static_cast<double>(h.redos);
}

int fail(const std::exception& e) {
    g_last_error = e.what();
    if (auto* se = dynamic_cast<const Error*>(&e)) return se->code;
    return SPG_E_INVALID;
}

bool device_ok() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return false;
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return false;
    return prop.major == 10;
}

}  // namespace

// Records the calling thread's last error for spg_last_error() and returns its status.
int record_error(const std::exception& e) { return fail(e); }

struct PoissonHandle {
    PoissonPlan plan;
    DevBuf<float> io;
    cudaStream_t stream = nullptr;
    ~PoissonHandle() {
        // the buffers' frees are ordered on `stream`, so it goes last
        if (stream) host_wait(stream);
        poisson_plan_destroy(plan);
        io.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace spg

using spg::Context;
using spg::Error;

struct spg_ctx {
    Context c;
};
struct spg_poisson {
    spg::PoissonHandle h;
};

namespace spg {

// Uploads a netlist into the context, replacing any earlier one (spg_ctx_create and
// spg_ctx_load): host copies, device arrays, the degree-ordered net classes of the WA kernel
// and the node-order pin slots. Device buffers with enough capacity are reused. The grid
// and the stage state are rebuilt by the next stage run.
void load_netlist(Context& c, const spg_db_view* v, const spg_params* prm) {
    HostTimer ht(" load");
    SPG_REQUIRE(v->num_movable >= 0 && v->num_nodes >= v->num_movable && v->num_fillers >= 0 &&
                    v->num_pins >= 0 && v->num_nets >= 0,
                SPG_E_INVALID, "inconsistent db counts");
    c.prm = *prm;
    c.have_eval = false;
    c.grid_ready = false;
    c.metrics_rows = 0;
    c.num_movable = v->num_movable;
    c.num_nodes = v->num_nodes;
    c.num_fillers = v->num_fillers;
    c.total = v->num_nodes + v->num_fillers;
    c.num_pins = v->num_pins;
    c.num_nets = v->num_nets;
    const size_t T = static_cast<size_t>(c.total);
    c.w.assign(v->node_w, v->node_w + T);
    c.h.assign(v->node_h, v->node_h + T);
    c.flags.assign(v->node_flags, v->node_flags + T);
    c.node_start.assign(v->node2pin_start, v->node2pin_start + T + 1);
    c.row_ly.assign(v->row_ly, v->row_ly + v->num_rows);
    c.row_hgt.assign(v->row_height, v->row_height + v->num_rows);
    c.row_lx.assign(v->row_lx, v->row_lx + v->num_rows);
    c.row_step.assign(v->row_step, v->row_step + v->num_rows);
    c.row_sites.assign(v->row_num_sites, v->row_num_sites + v->num_rows);
    c.core_lx = v->core_lx;
    c.core_ly = v->core_ly;
    c.core_hx = v->core_hx;
    c.core_hy = v->core_hy;
    for (int p = 0; p < c.num_pins; ++p)
        SPG_REQUIRE(v->pin2node[p] >= 0 && v->pin2node[p] < c.total, SPG_E_INVALID, "pin2node out of range");
    for (int k = 0; k < c.num_nets; ++k)
        SPG_REQUIRE(v->net2pin_start[k] <= v->net2pin_start[k + 1], SPG_E_INVALID, "net CSR not monotone");
    for (size_t i = 0; i < T; ++i)
        SPG_REQUIRE(c.node_start[i] <= c.node_start[i + 1], SPG_E_INVALID, "node CSR not monotone");
    SPG_REQUIRE(v->net2pin_start[0] == 0 && c.node_start[0] == 0 &&
                    v->net2pin_start[c.num_nets] == c.num_pins && c.node_start[T] == c.num_pins,
                SPG_E_INVALID, "CSR sizes disagree with num_pins");
    for (int p = 0; p < c.num_pins; ++p) {
        SPG_REQUIRE(v->flat_net2pin[p] >= 0 && v->flat_net2pin[p] < c.num_pins, SPG_E_INVALID,
                    "flat_net2pin out of range");
        SPG_REQUIRE(v->flat_node2pin[p] >= 0 && v->flat_node2pin[p] < c.num_pins, SPG_E_INVALID,
                    "flat_node2pin out of range");
        SPG_REQUIRE(v->pin2net[p] < c.num_nets, SPG_E_INVALID, "pin2net out of range");
    }
    ht.mark("validate");
    cudaStream_t s = c.stream;
    c.x.upload(v->node_x, T, s);
    c.y.upload(v->node_y, T, s);
    c.x_mirror.assign(v->node_x, v->node_x + v->num_nodes);
    c.y_mirror.assign(v->node_y, v->node_y + v->num_nodes);
    c.mirror_valid = true;
    c.dw.upload(v->node_w, T, s);
    c.dh.upload(v->node_h, T, s);
    c.pox.upload(v->pin_offset_x, c.num_pins, s);
    c.poy.upload(v->pin_offset_y, c.num_pins, s);
    c.pin2node.upload(v->pin2node, c.num_pins, s);
    c.pin2net.upload(v->pin2net, c.num_pins, s);
    c.net_start.upload(v->net2pin_start, c.num_nets + 1, s);
    c.net_pins.upload(v->flat_net2pin, c.num_pins, s);
    c.node_start_d.upload(v->node2pin_start, T + 1, s);
    c.node_pins.upload(v->flat_node2pin, c.num_pins, s);
    // nets in ascending degree (stable), cut into classes of one degree each: a net of degree
    // d <= kWaThreadNetDegree is owned by one thread, a larger one by a lane group of the next
    // power of two >= d, and the nets above 32 pins by one warp each that loops over its pins
    // (wirelength.cu)
    ht.mark("uploads");
    std::vector<int> order(c.num_nets);
    std::iota(order.begin(), order.end(), 0);
    auto deg = [&](int k) { return v->net2pin_start[k + 1] - v->net2pin_start[k]; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return deg(a) < deg(b); });
    c.net_order.upload(order, s);
    {
        WaClasses& wc = c.wa_classes;
        wc = WaClasses{};
        int thread_deg = kWaThreadNetDegree;
        if (const char* e = std::getenv("SPG_WA_THREAD_DEGREE")) thread_deg = std::atoi(e);
        SPG_REQUIRE(thread_deg >= 0 && thread_deg <= kWaThreadNetDegree, SPG_E_INVALID,
                    "SPG_WA_THREAD_DEGREE out of range");
        int warps = 0, pins = 0;
        auto add = [&](int g, int d, int begin, int end) {
            SPG_REQUIRE(wc.n < WA_MAX_CLASSES, SPG_E_INVALID, "too many WA degree classes");
            const int i = wc.n++;
            wc.group[i] = g;
            wc.shift[i] = g > 0 ? __builtin_ctz(g) : 0;
            wc.deg[i] = d;
            wc.net_begin[i] = begin;
            wc.net_end[i] = end;
            wc.pin_begin[i] = pins;
            wc.warp_begin[i] = warps;
            warps += g ? ceil_div(end - begin, 32 / g) : (end - begin);
        };
        for (int t = 0; t < c.num_nets;) {
            const int d = deg(order[t]);
            if (d > 32) {  // the sorted tail: every remaining net is above 32 pins
                add(0, -1, t, c.num_nets);
                break;
            }
            int e = t;
            while (e < c.num_nets && deg(order[e]) == d) ++e;
            if (d > 0) {
                int g = 1;
                if (d > thread_deg)
                    while (g < d || g < 2) g <<= 1;
                add(g, d, t, e);
            }
            pins += d * (e - t);
            t = e;
        }
        wc.warp_begin[wc.n] = warps;
    }
    ht.mark("classes");
    // node-order slots of the pins that belong to a net; the last slot is never read
    {
        for (int k = 0; k < c.num_nets; ++k)
            for (int q = v->net2pin_start[k]; q < v->net2pin_start[k + 1]; ++q)
                SPG_REQUIRE(v->pin2net[v->flat_net2pin[q]] == k, SPG_E_INVALID,
                            "pin2net disagrees with the net CSR");
        std::vector<int> slot_of_pin(c.num_pins, -1), slot_start(T + 1);
        int slots = 0;
        for (size_t i = 0; i < T; ++i) {
            slot_start[i] = slots;
            for (int t = c.node_start[i]; t < c.node_start[i + 1]; ++t) {
                const int pin = v->flat_node2pin[t];
                if (v->pin2net[pin] >= 0) slot_of_pin[pin] = slots++;
            }
        }
        slot_start[T] = slots;
        std::vector<int> net_slot(c.num_pins);
        for (int q = 0; q < c.num_pins; ++q) {
            const int sl = slot_of_pin[v->flat_net2pin[q]];
            net_slot[q] = sl >= 0 ? sl : slots;
        }
        c.slot_start.upload(slot_start, s);
        c.slot_start_h = slot_start;
        c.net_slot.upload(net_slot, s);
        c.num_slots = slots;
        // the WA pass-1 copy of each pin's data, in the degree-sorted net order
        std::vector<int> wa_start(c.num_nets + 1);
        std::vector<int2> node_slot(c.num_pins);
        std::vector<float2> off(c.num_pins);
        int q = 0;
        for (int t = 0; t < c.num_nets; ++t) {
            const int k = order[t];
            wa_start[t] = q;
            for (int e = v->net2pin_start[k]; e < v->net2pin_start[k + 1]; ++e, ++q) {
                const int pin = v->flat_net2pin[e];
                node_slot[q] = make_int2(v->pin2node[pin], net_slot[e]);
                off[q] = make_float2(v->pin_offset_x[pin], v->pin_offset_y[pin]);
            }
        }
        wa_start[c.num_nets] = q;
        c.wa_start.upload(wa_start, s);
        c.wa_node_slot.upload(node_slot, s);
        c.wa_off.upload(off, s);
    }
    ht.mark("slots");
    {
        const int f0 = c.num_nodes;
        bool alike = c.total > f0;
        for (int i = f0; alike && i < c.total; ++i)
            alike = c.w[i] == c.w[f0] && c.h[i] == c.h[f0] &&
                    c.node_start[i + 1] - c.node_start[i] == c.node_start[f0 + 1] - c.node_start[f0] &&
                    c.slot_start_h[i] == c.slot_start_h[i + 1];
        c.fillers_alike = alike;
    }
    c.gpx.alloc(c.num_slots + 1);
    c.gpy.alloc(c.num_slots + 1);
    c.gpx.zero(s);
    c.gpy.zero(s);
    c.st.alloc(1);
    if (!c.hst) SPG_CUDA(cudaMallocHost(&c.hst, sizeof(DevState)));
    c.scratch_d.alloc(16);
    ht.mark("alloc");
}

}  // namespace spg

#define API_TRY try {
#define API_CATCH \
    }             \
    catch (const std::exception& e) { return spg::fail(e); }

extern "C" {

int spg_abi_version(void) { return SPG_ABI_VERSION; }
const char* spg_last_error(void) { return spg::g_last_error.c_str(); }
int spg_device_check(void) {
    if (!spg::device_ok()) {
        spg::g_last_error = "no usable sm_100 device";
        return SPG_E_NO_DEVICE;
    }
    return SPG_OK;
}

int spg_host_alloc(size_t bytes, void** out) {
    API_TRY
    SPG_REQUIRE(out, SPG_E_INVALID, "null argument");
    *out = nullptr;
    SPG_CUDA(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
    return SPG_OK;
    API_CATCH
}

int spg_host_free(void* p) {
    API_TRY
    if (p) SPG_CUDA(cudaFreeHost(p));
    return SPG_OK;
    API_CATCH
}

int spg_bin_index_check(float step, const float* a, int32_t n, int32_t* q_div, int32_t* q_mul) {
    API_TRY
    SPG_REQUIRE(a && q_div && q_mul && n >= 0 && step > 0.f, SPG_E_INVALID, "bad argument");
    SPG_REQUIRE(spg::device_ok(), SPG_E_NO_DEVICE, "no usable sm_100 device");
    if (n == 0) return SPG_OK;
    const size_t bytes = static_cast<size_t>(n) * 4;
    float* da = nullptr;
    int *dq = nullptr, *dm = nullptr;
    SPG_CUDA(cudaMalloc(&da, bytes));
    SPG_CUDA(cudaMalloc(&dq, bytes));
    SPG_CUDA(cudaMalloc(&dm, bytes));
    SPG_CUDA(cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice));
    // the same double reciprocal as grid_init's
    spg::launch_bin_index_check(da, n, step, 1.0 / static_cast<double>(step), dq, dm, nullptr);
    SPG_CUDA(cudaGetLastError());
    SPG_CUDA(cudaMemcpy(q_div, dq, bytes, cudaMemcpyDeviceToHost));
    SPG_CUDA(cudaMemcpy(q_mul, dm, bytes, cudaMemcpyDeviceToHost));
    cudaFree(da);
    cudaFree(dq);
    cudaFree(dm);
    return SPG_OK;
    API_CATCH
}

void spg_params_default(spg_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->target_density = 1.0f;
    p->target_overflow = 0.10f;
    p->cgp_target_overflow = 0.10f;
    p->gp_max_iter = 2000;
    p->ignore_net_degree = 100;
    p->gp_bin_dim = 0;
    p->filler_only_iters = 20;
    p->delta_hpwl_ref = 3.5e5f;
    p->lambda_schedule_relative = 0;
    p->delta_hpwl_relative = 0.01;
    p->use_bb = 1;
    p->gp_backtrack = 1;
    p->max_backtrack = 10;
    p->gp_stagnation_window = 200;
    p->gp_stagnation_min_gain = 0.02f;
    p->random_seed = 1002;
    p->poisson_precision = SPG_POISSON_FP32;
    p->verbose = 0;
    p->freeze_lambda = 0;
    p->freeze_gamma = 0;
    p->poisson_single_launch = 0;
}

// ------------------------------------------------------------------ Poisson
int spg_poisson_create_batched(int nx, int ny, float sx, float sy, int precision, int batch_cap,
                               spg_poisson** out) {
    API_TRY
    SPG_REQUIRE(out, SPG_E_INVALID, "null output");
    *out = nullptr;
    if (!spg::device_ok()) throw Error(SPG_E_NO_DEVICE, "no usable sm_100 device");
    auto h = std::make_unique<spg_poisson>();
    SPG_CUDA(cudaStreamCreateWithFlags(&h->h.stream, cudaStreamNonBlocking));
    spg::AllocScope alloc_scope(h->h.stream);
    spg::poisson_plan_create(h->h.plan, nx, ny, sx, sy, precision, batch_cap);
    h->h.io.alloc(4 * static_cast<size_t>(nx) * ny);
    *out = h.release();
    return SPG_OK;
    API_CATCH
}

int spg_poisson_create(int nx, int ny, float sx, float sy, int precision, spg_poisson** out) {
    return spg_poisson_create_batched(nx, ny, sx, sy, precision, 1, out);
}

int spg_poisson_solve(spg_poisson* h, const float* rho, float* phi, float* fx, float* fy) {
    API_TRY
    SPG_REQUIRE(h && rho && phi && fx && fy, SPG_E_INVALID, "null argument");
    const size_t n = static_cast<size_t>(h->h.plan.nx) * h->h.plan.ny;
    float* d = h->h.io.p;
    cudaStream_t s = h->h.stream;
    SPG_CUDA(cudaMemcpyAsync(d, rho, n * 4, cudaMemcpyHostToDevice, s));
    spg::poisson_solve(h->h.plan, 1, d, d + n, d + 2 * n, d + 3 * n, s);
    SPG_CUDA(cudaMemcpyAsync(phi, d + n, n * 4, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(cudaMemcpyAsync(fx, d + 2 * n, n * 4, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(cudaMemcpyAsync(fy, d + 3 * n, n * 4, cudaMemcpyDeviceToHost, s));
    SPG_CUDA(spg::host_wait(s));
    if (const int* f = spg::tc_error_flag(h->h.plan)) {
        int e = 0;
        SPG_CUDA(cudaMemcpyAsync(&e, f, sizeof(e), cudaMemcpyDeviceToHost, s));
        SPG_CUDA(spg::host_wait(s));
        if (e) throw spg::Error(e, "Poisson tensor-core solve gave up a bounded pipeline wait");
    }
    return SPG_OK;
    API_CATCH
}

int spg_poisson_solve_batch_device(spg_poisson* h, int batch, const float* rho, float* phi,
                                   float* fx, float* fy, void* stream) {
    API_TRY
    SPG_REQUIRE(h && rho && phi && fx && fy, SPG_E_INVALID, "null argument");
    spg::poisson_solve(h->h.plan, batch, rho, phi, fx, fy, static_cast<cudaStream_t>(stream));
    return SPG_OK;
    API_CATCH
}

int spg_poisson_solve_device(spg_poisson* h, const float* rho, float* phi, float* fx, float* fy,
                             void* stream) {
    return spg_poisson_solve_batch_device(h, 1, rho, phi, fx, fy, stream);
}

const char* spg_poisson_name(const spg_poisson* h) { return h ? h->h.plan.name.c_str() : "none"; }

int spg_poisson_set_single_launch(spg_poisson* h, int on) {
    if (!h) return spg::fail(Error(SPG_E_INVALID, "null argument"));
    h->h.plan.single_launch = on != 0;
    return SPG_OK;
}

int spg_poisson_destroy(spg_poisson* h) {
    delete h;
    return SPG_OK;
}

// ------------------------------------------------------------------ fillers (host)
int spg_fillers_plan(const spg_db_view* db, float target, spg_filler_info* out) {
    API_TRY
    SPG_REQUIRE(db && out, SPG_E_INVALID, "null argument");
    // initializeFillers (src/gp/filler.cpp:47-120)
    spg_filler_info info{};
    double overlap = 0.0;
    for (int i = db->num_movable; i < db->num_nodes; ++i) {
        if (db->node_flags[i] & SPG_F_NI) continue;
        const float blx = db->node_x[i] - 0.5f * db->node_w[i], bhx = db->node_x[i] + 0.5f * db->node_w[i];
        const float bly = db->node_y[i] - 0.5f * db->node_h[i], bhy = db->node_y[i] + 0.5f * db->node_h[i];
        for (int r = 0; r < db->num_rows; ++r) {
            const float rly = db->row_ly[r], rhy = db->row_ly[r] + db->row_height[r];
            if (rly >= bhy) break;
            if (rhy <= bly) continue;
            const float rlx = db->row_lx[r], rhx = db->row_lx[r] + db->row_step[r] * static_cast<float>(db->row_num_sites[r]);
            overlap += static_cast<double>(spg::overlap_area(blx, bly, bhx, bhy, rlx, rly, rhx, rhy));
        }
    }
    info.whitespace_area = std::max(0.0, db->total_row_area - overlap);
    double cell = 0.0, macro = 0.0;
    for (int i = 0; i < db->num_movable; ++i) {
        const double a = static_cast<double>(db->node_w[i]) * static_cast<double>(db->node_h[i]);
        if (db->node_flags[i] & SPG_F_MACRO) macro += a;
        else cell += a;
    }
    info.node_area_scaled = cell + macro * static_cast<double>(target);
    info.total_filler_area = info.whitespace_area * static_cast<double>(target) - info.node_area_scaled;
    if (db->num_movable == 0) {
        *out = info;
        return SPG_OK;
    }
    std::vector<double> areas(static_cast<size_t>(db->num_movable));
    for (int i = 0; i < db->num_movable; ++i)
        areas[i] = static_cast<double>(db->node_w[i]) * static_cast<double>(db->node_h[i]);
    std::sort(areas.begin(), areas.end());
    const int lo = static_cast<int>(0.10 * db->num_movable), hi = static_cast<int>(0.90 * db->num_movable);
    double avg = 0.0;
    if (hi > lo) {
        for (int i = lo; i < hi; ++i) avg += areas[i];
        avg /= (hi - lo);
    } else {
        avg = areas[db->num_movable / 2];
    }
    info.height = db->row_height_mode > 0.f ? db->row_height_mode : 1.f;
    info.width = static_cast<float>(avg) / info.height;
    if (!(info.width > 0.f)) info.width = 1.f;
    const double single = static_cast<double>(info.width) * info.height;
    const double raw = info.total_filler_area / std::max(single, 1e-9);
    info.count = std::max(0, static_cast<int>(raw + 0.5));
    *out = info;
    return SPG_OK;
    API_CATCH
}

int spg_fillers_scatter(const spg_db_view* db, int32_t count, float width, float height,
                        uint64_t seed, float* x, float* y) {
    API_TRY
    SPG_REQUIRE(db && (count == 0 || (x && y)), SPG_E_INVALID, "null argument");
    // scatterFillers (src/gp/filler.cpp:33-45): mt19937 seeded with the config seed,
    // uniform_real_distribution<float> per coordinate, x then y per filler.
    std::mt19937 eng(static_cast<std::mt19937::result_type>(seed));
    const float hw = 0.5f * width, hh = 0.5f * height;
    const float lo_x = db->core_lx + hw, hi_x = db->core_hx - hw;
    const float lo_y = db->core_ly + hh, hi_y = db->core_hy - hh;
    const float cx = 0.5f * (db->core_lx + db->core_hx), cy = 0.5f * (db->core_ly + db->core_hy);
    for (int i = 0; i < count; ++i) {
        if (hi_x > lo_x) {
            std::uniform_real_distribution<float> d(lo_x, hi_x);
            x[i] = d(eng);
        } else {
            x[i] = cx;
        }
        if (hi_y > lo_y) {
            std::uniform_real_distribution<float> d(lo_y, hi_y);
            y[i] = d(eng);
        } else {
            y[i] = cy;
        }
    }
    return SPG_OK;
    API_CATCH
}

// ------------------------------------------------------------------ context
int spg_ctx_create(const spg_db_view* v, const spg_params* prm, spg_ctx** out) {
    API_TRY
    SPG_REQUIRE(v && prm && out, SPG_E_INVALID, "null argument");
    *out = nullptr;
    if (!spg::device_ok()) throw Error(SPG_E_NO_DEVICE, "no usable sm_100 device");
    auto h = std::make_unique<spg_ctx>();
    Context& c = h->c;
    // SPG_HOST_LOOP=1 selects the host-driven iteration loop (one state read per iteration)
    // instead of the conditional CUDA graph; both run the same kernels in the same order.
    c.use_graph = std::getenv("SPG_HOST_LOOP") == nullptr;
    // The main stream carries the latency-bound chain (scatter -> rho -> Poisson -> assembly)
    // at the highest priority; the WA pass on the side stream is throughput work that fills
    // whatever SMs the chain leaves free.
    int prio_low = 0, prio_high = 0;
    SPG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    SPG_CUDA(cudaStreamCreateWithPriority(&c.stream, cudaStreamNonBlocking, prio_high));
    SPG_CUDA(cudaStreamCreateWithPriority(&c.side, cudaStreamNonBlocking, prio_low));
    SPG_CUDA(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
    SPG_CUDA(cudaEventCreateWithFlags(&c.ev_join, cudaEventDisableTiming));
    SPG_CUDA(cudaEventCreate(&c.ev_t0));
    SPG_CUDA(cudaEventCreate(&c.ev_t1));
    spg::CtxScope scope(c);
    spg::load_netlist(c, v, prm);
    SPG_CUDA(spg::host_wait(c.stream));
    *out = h.release();
    return SPG_OK;
    API_CATCH
}

int spg_ctx_load(spg_ctx* ctx, const spg_db_view* v, const spg_params* prm) {
    API_TRY
    SPG_REQUIRE(ctx && v && prm, SPG_E_INVALID, "null argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    if (c.side) SPG_CUDA(spg::host_wait(c.side));
    spg::load_netlist(c, v, prm);
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_ctx_destroy(spg_ctx* ctx) {
    delete ctx;
    return SPG_OK;
}

int spg_positions_h2d(spg_ctx* ctx, const float* x, const float* y) {
    API_TRY
    SPG_REQUIRE(ctx && x && y, SPG_E_INVALID, "null argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    // the caller's arrays are free once this returns: page-locked ones are copied by DMA and
    // waited for, pageable ones are staged and their copies run ahead of the context's next work
    spg::upload_pair(c.x.p, x, c.y.p, y, c.total * sizeof(float), c.stream);
    c.x_mirror.assign(x, x + c.num_nodes);
    c.y_mirror.assign(y, y + c.num_nodes);
    c.mirror_valid = true;
    return SPG_OK;
    API_CATCH
}

int spg_positions_d2h(spg_ctx* ctx, float* x, float* y) {
    API_TRY
    SPG_REQUIRE(ctx && x && y, SPG_E_INVALID, "null argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::download_pair(x, c.x.p, y, c.y.p, c.total * sizeof(float), c.stream);
    return SPG_OK;
    API_CATCH
}

int spg_flags_h2d(spg_ctx* ctx, const uint8_t* flags) {
    API_TRY
    SPG_REQUIRE(ctx && flags, SPG_E_INVALID, "null argument");
    ctx->c.flags.assign(flags, flags + ctx->c.total);
    ctx->c.grid_ready = false;
    return SPG_OK;
    API_CATCH
}

int spg_grid_init(spg_ctx* ctx, float target, int bin_dim) {
    API_TRY
    SPG_REQUIRE(ctx && target > 0.f, SPG_E_INVALID, "bad argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    std::vector<float> hx(c.total), hy(c.total);
    spg::download_bytes(hx.data(), c.x.p, c.total * sizeof(float), c.stream);
    spg::download_bytes(hy.data(), c.y.p, c.total * sizeof(float), c.stream);
    spg::grid_init(c, target, bin_dim, hx, hy);
    // parity hooks evaluate over every node: an opt set of all density nodes is not needed
    return SPG_OK;
    API_CATCH
}

int spg_grid_info(const spg_ctx* ctx, int* dim, float* sx, float* sy, float* ox, float* oy,
                  double* den) {
    API_TRY
    SPG_REQUIRE(ctx && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    const Context& c = ctx->c;
    if (dim) *dim = c.geom.dim;
    if (sx) *sx = c.geom.step_x;
    if (sy) *sy = c.geom.step_y;
    if (ox) *ox = c.geom.origin_x;
    if (oy) *oy = c.geom.origin_y;
    if (den) *den = c.movable_area_scaled;
    return SPG_OK;
    API_CATCH
}

int spg_grid_read(const spg_ctx* ctx, int which, float* out) {
    API_TRY
    SPG_REQUIRE(ctx && out && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    const Context& c = ctx->c;
    const spg::DevBuf<float>* b[] = {&c.node_map, &c.filler_map, &c.terminal, &c.base,
                                     &c.rho, &c.phi, &c.ex, &c.ey};
    SPG_REQUIRE(which >= 0 && which < 8, SPG_E_INVALID, "unknown map");
    const size_t n = static_cast<size_t>(c.geom.dim) * c.geom.dim;
    SPG_CUDA(cudaMemcpyAsync(out, b[which]->p, n * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_grid_write(spg_ctx* ctx, int which, const float* in) {
    API_TRY
    SPG_REQUIRE(ctx && in && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevBuf<float>* b[] = {&c.node_map, &c.filler_map, &c.terminal, &c.base,
                               &c.rho, &c.phi, &c.ex, &c.ey};
    SPG_REQUIRE(which >= 4 && which < 8, SPG_E_INVALID, "only rho, phi, xi_x, xi_y are writable");
    const size_t n = static_cast<size_t>(c.geom.dim) * c.geom.dim;
    SPG_CUDA(cudaMemcpyAsync(b[which]->p, in, n * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_grid_read_fixed(const spg_ctx* ctx, int64_t* node, int64_t* filler, int* shift) {
    API_TRY
    SPG_REQUIRE(ctx && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    const Context& c = ctx->c;
    const size_t n = static_cast<size_t>(c.geom.dim) * c.geom.dim;
    if (node) SPG_CUDA(cudaMemcpyAsync(node, c.node_fix.p, n * 8, cudaMemcpyDeviceToHost, c.stream));
    if (filler) SPG_CUDA(cudaMemcpyAsync(filler, c.filler_fix.p, n * 8, cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    if (shift) *shift = c.geom.shift;
    return SPG_OK;
    API_CATCH
}

int spg_density_accumulate(spg_ctx* ctx) {
    API_TRY
    SPG_REQUIRE(ctx && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevPtrs p = c.ptrs();
    c.node_fix.zero(c.stream);
    c.filler_fix.zero(c.stream);
    spg::launch_density_accumulate(p, c.stream);
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_overflow(spg_ctx* ctx, float* tau) {
    API_TRY
    SPG_REQUIRE(ctx && tau && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevPtrs p = c.ptrs();
    // rho, the float maps and tau from the current fixed-point maps (kept for read_fixed)
    spg::launch_rho_overflow(p, 1, 0, c.stream);
    double over = 0.0;
    spg::launch_finalize_slots(p, spg::SLOT_OVERFLOW, 1, c.scratch_d.p, c.stream);
    SPG_CUDA(cudaMemcpyAsync(&over, c.scratch_d.p, 8, cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    *tau = c.movable_area_scaled > 0.0 ? static_cast<float>(over / c.movable_area_scaled) : 0.f;
    return SPG_OK;
    API_CATCH
}

int spg_solve_field(spg_ctx* ctx) {
    API_TRY
    SPG_REQUIRE(ctx && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::poisson_solve(*c.plan, 1, c.rho.p, c.phi.p, c.ex.p, c.ey.p, c.stream);
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_gather_force(spg_ctx* ctx, float* force) {
    API_TRY
    SPG_REQUIRE(ctx && force && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevPtrs p = c.ptrs();
    spg::DevBuf<float> out;
    out.alloc(2 * static_cast<size_t>(c.total));
    out.zero(c.stream);
    spg::launch_gather_all(p, out.p, c.stream);
    SPG_CUDA(cudaMemcpyAsync(force, out.p, 2 * c.total * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_total_charge(spg_ctx* ctx, double* charge) {
    API_TRY
    SPG_REQUIRE(ctx && charge && ctx->c.grid_ready, SPG_E_STATE, "grid not initialised");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    const size_t n = static_cast<size_t>(c.geom.dim) * c.geom.dim;
    std::vector<long long> a(n), b(n);
    SPG_CUDA(cudaMemcpyAsync(a.data(), c.node_fix.p, n * 8, cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(cudaMemcpyAsync(b.data(), c.filler_fix.p, n * 8, cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    long long s = 0;
    for (size_t i = 0; i < n; ++i) s += a[i] + b[i];
    *charge = static_cast<double>(s) * c.geom.inv_scale;
    return SPG_OK;
    API_CATCH
}

int spg_wa_wirelength(spg_ctx* ctx, float gamma, int ignore, double* wl, float* grad) {
    API_TRY
    SPG_REQUIRE(ctx, SPG_E_INVALID, "null context");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevPtrs p = c.ptrs();
    p.ignore_net_degree = ignore;
    if (!c.partials.p) {
        c.partials.alloc(static_cast<size_t>(spg::RED_SLOTS) * spg::RED_CAP);
        c.partials.zero(c.stream);
        p.partials = c.partials.p;
    }
    spg::launch_wa_nets(p, c.wa_classes, nullptr, gamma, 0, c.stream);
    spg::DevBuf<float> g;
    g.alloc(2 * static_cast<size_t>(std::max(c.num_movable, 1)));
    spg::launch_wa_node_grad(p, g.p, c.stream);
    spg::launch_finalize_slots(p, spg::SLOT_WL, 1, c.scratch_d.p, c.stream);
    double v = 0.0;
    SPG_CUDA(cudaMemcpyAsync(&v, c.scratch_d.p, 8, cudaMemcpyDeviceToHost, c.stream));
    if (grad)
        SPG_CUDA(cudaMemcpyAsync(grad, g.p, 2 * c.num_movable * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    if (wl) *wl = v;
    return SPG_OK;
    API_CATCH
}

int spg_hpwl(spg_ctx* ctx, double* hpwl) {
    API_TRY
    SPG_REQUIRE(ctx && hpwl, SPG_E_INVALID, "null argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    spg::DevPtrs p = c.ptrs();
    if (!c.partials.p) {
        c.partials.alloc(static_cast<size_t>(spg::RED_SLOTS) * spg::RED_CAP);
        c.partials.zero(c.stream);
        p.partials = c.partials.p;
    }
    spg::launch_wa_nets(p, c.wa_classes, nullptr, 1.f, 0, c.stream);
    spg::launch_finalize_slots(p, spg::SLOT_HPWL, 1, c.scratch_d.p, c.stream);
    SPG_CUDA(cudaMemcpyAsync(hpwl, c.scratch_d.p, 8, cudaMemcpyDeviceToHost, c.stream));
    SPG_CUDA(spg::host_wait(c.stream));
    return SPG_OK;
    API_CATCH
}

int spg_stage_run(spg_ctx* ctx, int stage, spg_result* result) {
    API_TRY
    SPG_REQUIRE(ctx && result, SPG_E_INVALID, "null argument");
    spg::CtxScope scope(ctx->c);
    spg::stage_run(ctx->c, stage, result);
    return SPG_OK;
    API_CATCH
}

int spg_set_iter_callback(spg_ctx* ctx, spg_iter_fn fn, void* user, int32_t stride) {
    API_TRY
    SPG_REQUIRE(ctx, SPG_E_INVALID, "null argument");
    spg::Context& c = ctx->c;
    c.iter_fn = stride > 0 ? fn : nullptr;
    c.iter_user = user;
    c.iter_stride = fn ? stride : 0;
    return SPG_OK;
    API_CATCH
}

int spg_set_stagnation_callback(spg_ctx* ctx, spg_iter_fn fn, void* user) {
    API_TRY
    SPG_REQUIRE(ctx, SPG_E_INVALID, "null argument");
    ctx->c.mid_fn = fn;
    ctx->c.mid_user = user;
    return SPG_OK;
    API_CATCH
}

int spg_eval_positions(spg_ctx* ctx, int32_t which, float* x, float* y) {
    API_TRY
    SPG_REQUIRE(ctx && x && y && (which == 0 || which == 1), SPG_E_INVALID, "bad argument");
    spg::Context& c = ctx->c;
    SPG_REQUIRE(c.have_eval, SPG_E_STATE, "no stage has evaluated a point yet");
    spg::CtxScope scope(c);
    spg::download_eval_positions(c, c.ptrs(), which == 0 ? c.eval_role : c.eval_prev_role, x, y);
    return SPG_OK;
    API_CATCH
}

int spg_metrics_d2h(const spg_ctx* ctx, spg_iter_metrics* rows, int cap, int* n_rows) {
    API_TRY
    SPG_REQUIRE(ctx && n_rows, SPG_E_INVALID, "null argument");
    const Context& c = ctx->c;
    const int n = std::min(cap, c.metrics_rows);
    if (n > 0 && rows)
        SPG_CUDA(cudaMemcpy(rows, c.metrics.p, n * sizeof(spg_iter_metrics), cudaMemcpyDeviceToHost));
    *n_rows = n;
    return SPG_OK;
    API_CATCH
}

int64_t spg_ctx_launch_count(const spg_ctx* ctx) {
    (void)ctx;
    return spg::g_launches;
}

void* spg_ctx_stream(const spg_ctx* ctx) { return ctx ? static_cast<void*>(ctx->c.stream) : nullptr; }

int spg_ctx_graph_loop(const spg_ctx* ctx) { return ctx && ctx->c.last_run_graph ? 1 : 0; }

int spg_eval_grad(spg_ctx* ctx, int stage, float lambda, float gamma, const float* pos, float* grad, double* out,
                  int32_t* n_opt) {
    API_TRY
    SPG_REQUIRE(ctx && n_opt, SPG_E_INVALID, "null argument");
    spg::CtxScope scope(ctx->c);
    spg::eval_grad(ctx->c, stage, lambda, gamma, pos, grad, out, n_opt);
    return SPG_OK;
    API_CATCH
}

int spg_nesterov_quadratic(int32_t n, const float* coef, const float* target, float* pos, int32_t steps,
                           int32_t use_bb, int32_t backtrack, int32_t max_backtrack, float init_step,
                           double* out) {
    try {
        if (!spg::device_ok()) return spg::fail(Error(SPG_E_NO_DEVICE, "no sm_100 device"));
        spg::nesterov_quadratic(n, coef, target, pos, steps, use_bb, backtrack, max_backtrack, init_step, out);
        return SPG_OK;
    } catch (const std::exception& e) {
        return spg::fail(e);
    }
}

int spg_ctx_profile(spg_ctx* ctx, int reps, double* us, int n) {
    API_TRY
    SPG_REQUIRE(ctx && us && reps > 0, SPG_E_INVALID, "bad argument");
    Context& c = ctx->c;
    spg::CtxScope scope(c);
    SPG_REQUIRE(c.grid_ready && c.n_opt > 0 && c.plan, SPG_E_STATE, "run a stage before profiling");
    c.mirror_valid = false;  // the parts below write the node positions
    cudaStream_t s = c.stream;
    const spg::DevPtrs p = c.ptrs();
    // keep the stage's state; profiling runs with decisions off (done) except for the update
    spg::DevState saved;
    SPG_CUDA(cudaMemcpyAsync(&saved, c.st.p, sizeof(saved), cudaMemcpyDeviceToHost, s));
    SPG_CUDA(spg::host_wait(s));
    spg::DevState probe = saved;
    probe.done = 1;
    probe.redo = 0;
    probe.snap_copy_to = -1;
    probe.error = 0;
    probe.tk_update = probe.tk_assemble = probe.tk_reduce = 0;
    auto set_state = [&](const spg::DevState& st) {
        SPG_CUDA(cudaMemcpyAsync(c.st.p, &st, sizeof(st), cudaMemcpyHostToDevice, s));
        SPG_CUDA(spg::host_wait(s));
    };
    cudaEvent_t e0, e1;
    SPG_CUDA(cudaEventCreate(&e0));
    SPG_CUDA(cudaEventCreate(&e1));
    const int64_t launches0 = spg::g_launches;
    auto time = [&](auto&& body, auto&& before) {
        double total = 0.0;
        for (int r = 0; r < reps + 2; ++r) {  // two untimed warm-up launches
            before();
            SPG_CUDA(cudaEventRecord(e0, s));
            body();
            SPG_CUDA(cudaEventRecord(e1, s));
            SPG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            SPG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r >= 2) total += ms;
        }
        return total * 1e3 / reps;
    };
    auto nothing = [] {};
    auto zero_maps = [&] {
        c.node_fix.zero(s);
        c.filler_fix.zero(s);
    };
    double t[8] = {};
    spg::DevState upd = probe;
    upd.done = 0;
    upd.last = 0;
    set_state(upd);
    // the step carries the density scatter of the opt nodes (part 2 is the rest list only)
    t[0] = time([&] { spg::launch_update(p, s); }, zero_maps);
    set_state(probe);
    spg::launch_scatter(p, spg::R_POS, s);  // the delivered positions again
    t[1] = time([&] {
        spg::launch_wa_nets(p, c.wa_classes, &p.st->gamma, 0.f, 1, s);
        spg::launch_wl_cells(p, s);
    }, nothing);
    t[2] = (c.n_rest_small + c.n_rest_large) > 0 ? time([&] { spg::launch_density_rest(p, s); }, zero_maps) : 0.0;
    bool fused = false;
    t[3] = time([&] { fused = spg::rho_and_split(c, p, s); }, [&] { spg::launch_density_accumulate(p, s); });
    t[4] = time([&] { spg::poisson_solve(*c.plan, 1, c.rho.p, c.phi.p, c.ex.p, c.ey.p, s, fused); }, nothing);
    // the loop's assembly carries the norms and decisions of the reduce step (part 6 = 0)
    t[5] = time([&] {
        spg::launch_gather_opt_large(p, s);
        spg::launch_assemble_reduce(p, s);
    }, nothing);
    t[6] = 0.0;
    t[7] = time([&] { spg::evaluate(c, p, -1, spg::R_G, 1, true, true); }, nothing);
    spg::g_launches = launches0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // restore: state, delivered positions, and the evaluation at them
    set_state(saved);
    spg::launch_scatter(p, spg::R_POS, s);
    SPG_CUDA(spg::host_wait(s));
    spg::g_launches = launches0;
    for (int i = 0; i < n && i < 8; ++i) us[i] = t[i];
    return SPG_OK;
    API_CATCH
}

}  // extern "C"
