// Continuous-batching FFT server (C++), and a Poisson load generator for it.
//
// Requests (type C2C or R2C, length n, `rows` transforms, host or device
// buffers) arrive at any time.  A scheduler thread keeps one resident plan
// per (type, length, direction) sized for the largest batch, and a set of
// lanes (CUDA streams, each with resident device staging buffers).  Whenever
// a lane is free it forms a batch from the oldest pending request's class,
// adding later requests of the same class up to the lane's row capacity, as
// long as the bytes in flight stay within the workspace budget; it copies the
// inputs in (one cudaMemcpyAsync per request), runs the plan re-targeted to
// the batch's row count, copies each request's rows out and records an event.
// Requests in device memory of 8 MB or more skip the staging copies: the plan
// runs on their own buffers, on the lane's stream and workspace.
// Batches on different lanes run concurrently, so requests that arrive while
// others are on the GPU are admitted as soon as a lane and budget free up.
// Per-request latency is measured from submission to the host observing the
// batch's completion event.
//
// The reference has no serving layer; this sits above the same planner and
// kernels as the asdFft* entry points.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <random>
#include <thread>

#include "../../include/asdsip_fft_ext.h"
#include "sipfft_internal.h"

namespace sipfft {

namespace {

using Clock = std::chrono::steady_clock;

double now_s()
{
    return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

struct Req {
    int64_t id = 0;
    int type = 0x10;
    int dir = 0x10;
    int64_t n = 0;
    int64_t rows = 0;
    const void *in = nullptr;
    void *out = nullptr;
    double t_submit = 0.0;
    double t_done = 0.0;
};

struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    char *d_in = nullptr;
    char *d_out = nullptr;
    char *d_ws = nullptr;
    size_t bytes_in = 0, bytes_out = 0, bytes_ws = 0;
    std::vector<Req> batch;
    size_t batch_bytes = 0;
    bool busy = false;
};

int64_t in_bytes(const Req &r) { return r.type == 0x12 ? r.rows * r.n * 4 : r.rows * r.n * 8; }
// device-memory requests at least this large run on their own buffers
constexpr int64_t kDirectBytes = int64_t(8) << 20;
int64_t out_bytes(const Req &r) { return r.type == 0x12 ? r.rows * (r.n / 2 + 1) * 8 : r.rows * r.n * 8; }

}  // namespace

class Server {
public:
    Server(int64_t budget, int lanes, int64_t max_rows, bool device_io, int device)
        : budget_(budget), max_rows_(max_rows), device_io_(device_io), device_(device), lanes_(lanes)
    {
        for (Lane &l : lanes_) {
            cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking);
            cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming);
        }
        worker_ = std::thread([this] { loop(); });
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        worker_.join();
        for (Lane &l : lanes_) {
            cudaStreamSynchronize(l.stream);
            cudaFree(l.d_in);
            cudaFree(l.d_out);
            cudaFree(l.d_ws);
            cudaEventDestroy(l.done);
            cudaStreamDestroy(l.stream);
        }
        cudaGetLastError();
    }

    // Creates the resident plan of a request class ahead of traffic and
    // grows every lane's staging buffers to that class's largest batch, so no
    // allocation happens while requests are timed.
    std::string warm(int type, int dir, int64_t n)
    {
        Plan *p = nullptr;
        {
            std::lock_guard<std::mutex> lock(plan_mu_);
            p = plan_for(type, dir, n);
            if (!p) return last_err_;
        }
        Req probe;
        probe.type = type;
        probe.n = n;
        probe.rows = max_rows_;
        std::lock_guard<std::mutex> lock(lane_mu_);
        for (Lane &l : lanes_) {
            if (l.busy) continue;
            if (!grow(l.d_in, l.bytes_in, static_cast<size_t>(in_bytes(probe))) ||
                !grow(l.d_out, l.bytes_out, static_cast<size_t>(out_bytes(probe))) ||
                !grow(l.d_ws, l.bytes_ws, std::max<size_t>(p->ws_bytes, 256)))
                return "out of device memory";
        }
        return std::string();
    }

    // While held, pending requests are queued but not admitted (operators can
    // drain lanes; tests use it to make batching deterministic).
    void hold(bool on)
    {
        std::lock_guard<std::mutex> lock(mu_);
        hold_ = on;
        cv_.notify_all();
    }

    int64_t submit(Req r)
    {
        if (r.rows > max_rows_) return -1;  // larger than a lane: refused, never queued
        std::lock_guard<std::mutex> lock(mu_);
        r.id = next_id_++;
        r.t_submit = now_s();
        pending_.push_back(r);
        cv_.notify_all();
        return r.id;
    }

    // Blocks until every submitted request has completed; returns them.
    std::vector<Req> drain()
    {
        std::unique_lock<std::mutex> lock(mu_);
        cv_done_.wait(lock, [this] { return pending_.empty() && inflight_ == 0; });
        std::vector<Req> out;
        out.swap(completed_);
        return out;
    }

    // Arithmetic of the resident plans (asdFftSetPrecision modes); only
    // before the first plan exists, so every request class uses one form.
    bool set_precision(int mode)
    {
        std::lock_guard<std::mutex> lock(plan_mu_);
        if (!plans_.empty()) return false;
        precision_ = mode;
        return true;
    }

    int64_t batches() const { return batches_.load(); }
    int64_t failures() const { return failures_.load(); }

private:
    Plan *plan_for(int type, int dir, int64_t n)
    {
        auto key = std::make_tuple(type, dir, n);
        auto it = plans_.find(key);
        if (it != plans_.end()) return it->second.get();
        auto p = std::make_unique<Plan>();
        p->fft_type = type;
        p->direction = dir;
        p->sizes = {n};
        p->strides = {1};
        p->batch = max_rows_;
        p->device = device_;
        p->precision = precision_;
        std::string e = build_plan_1d(*p);
        if (!e.empty()) {
            last_err_ = e;
            return nullptr;
        }
        p->initialized = true;
        Plan *raw = p.get();
        plans_.emplace(key, std::move(p));
        return raw;
    }

    static bool grow(char *&ptr, size_t &have, size_t need)
    {
        if (have >= need) return true;
        cudaFree(ptr);
        ptr = nullptr;
        have = 0;
        if (cudaMalloc(&ptr, need) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        have = need;
        return true;
    }

    void finish_lane(Lane &l, double t)
    {
        std::lock_guard<std::mutex> lock(mu_);
        for (Req &r : l.batch) {
            r.t_done = t;
            completed_.push_back(r);
        }
        inflight_bytes_ -= static_cast<int64_t>(l.batch_bytes);
        inflight_ -= static_cast<int64_t>(l.batch.size());
        l.batch.clear();
        l.batch_bytes = 0;
        l.busy = false;
        cv_done_.notify_all();
    }

    // Takes the oldest pending request's class and as many same-class
    // requests as fit the lane and the budget (caller holds mu_).
    bool form_batch(std::vector<Req> &batch, int64_t &bytes)
    {
        if (pending_.empty() || hold_) return false;
        const Req head = pending_.front();
        int64_t rows = 0;
        bytes = 0;
        for (auto it = pending_.begin(); it != pending_.end();) {
            const bool same = it->type == head.type && it->dir == head.dir && it->n == head.n;
            const int64_t b = in_bytes(*it) + out_bytes(*it);
            // the head request is admitted on its own when nothing is in flight, so a
            // request larger than the budget cannot stall the queue
            const bool fits = inflight_bytes_ + bytes + b <= budget_ || (batch.empty() && inflight_bytes_ == 0);
            if (same && rows + it->rows <= max_rows_ && fits) {
                rows += it->rows;
                bytes += b;
                batch.push_back(*it);
                it = pending_.erase(it);
            } else {
                ++it;
            }
        }
        return !batch.empty();
    }

    bool launch(Lane &l)
    {
        const Req &h = l.batch.front();
        Plan *p = nullptr;
        {
            std::lock_guard<std::mutex> lock(plan_mu_);
            p = plan_for(h.type, h.dir, h.n);
        }
        if (!p) return false;
        if (!grow(l.d_ws, l.bytes_ws, std::max<size_t>(p->ws_bytes, 256))) return false;
        // Requests in device memory of at least kDirectBytes run the plan on their
        // own buffers (a staged copy in and out would double their HBM traffic);
        // smaller ones, and every request in host memory, are copied into the
        // lane's staging buffers and run as one batch.
        std::vector<const Req *> staged;
        int64_t rows = 0;
        for (const Req &r : l.batch) {
            const uintptr_t i0 = reinterpret_cast<uintptr_t>(r.in), o0 = reinterpret_cast<uintptr_t>(r.out);
            const bool aligned = (i0 | o0) % 16 == 0;
            // a request whose output overlaps its input keeps the staged path
            const bool disjoint = i0 + static_cast<uintptr_t>(in_bytes(r)) <= o0 ||
                                  o0 + static_cast<uintptr_t>(out_bytes(r)) <= i0;
            if (device_io_ && aligned && disjoint && in_bytes(r) >= kDirectBytes) {
                std::vector<Step> steps;
                if (!scale_steps_to_rows(*p, r.rows, steps)) return false;
                if (execute_steps(*p, steps, r.in, r.out, l.d_ws, l.stream) != cudaSuccess) return false;
            } else {
                staged.push_back(&r);
                rows += r.rows;
            }
        }
        if (!staged.empty()) {
            std::vector<Step> steps;
            if (!scale_steps_to_rows(*p, rows, steps)) return false;
            const size_t ib = static_cast<size_t>(in_bytes(h) / h.rows * max_rows_);
            const size_t ob = static_cast<size_t>(out_bytes(h) / h.rows * max_rows_);
            if (!grow(l.d_in, l.bytes_in, ib) || !grow(l.d_out, l.bytes_out, ob)) return false;
            const cudaMemcpyKind kin = device_io_ ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            const cudaMemcpyKind kout = device_io_ ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
            size_t off = 0;
            for (const Req *r : staged) {
                const size_t b = static_cast<size_t>(in_bytes(*r));
                if (cudaMemcpyAsync(l.d_in + off, r->in, b, kin, l.stream) != cudaSuccess) return false;
                off += b;
            }
            if (execute_steps(*p, steps, l.d_in, l.d_out, l.d_ws, l.stream) != cudaSuccess) return false;
            off = 0;
            for (const Req *r : staged) {
                const size_t b = static_cast<size_t>(out_bytes(*r));
                if (cudaMemcpyAsync(r->out, l.d_out + off, b, kout, l.stream) != cudaSuccess) return false;
                off += b;
            }
        }
        return cudaEventRecord(l.done, l.stream) == cudaSuccess;
    }

    void loop()
    {
        cudaSetDevice(device_);
        for (;;) {
            // completions
            for (Lane &l : lanes_) {
                if (l.busy && cudaEventQuery(l.done) == cudaSuccess) finish_lane(l, now_s());
            }
            // admissions
            bool launched = false;
            {
            std::lock_guard<std::mutex> lanes_lock(lane_mu_);
            for (Lane &l : lanes_) {
                if (l.busy) continue;
                std::vector<Req> batch;
                int64_t bytes = 0;
                {
                    std::lock_guard<std::mutex> lock(mu_);
                    if (!form_batch(batch, bytes)) break;
                    inflight_bytes_ += bytes;
                    inflight_ += static_cast<int64_t>(batch.size());
                }
                l.batch = std::move(batch);
                l.batch_bytes = static_cast<size_t>(bytes);
                l.busy = true;
                batches_++;
                if (!launch(l)) {
                    failures_++;
                    cudaGetLastError();
                    cudaStreamSynchronize(l.stream);
                    finish_lane(l, -1.0);  // reported with a negative completion time
                }
                launched = true;
            }
            }
            {
                std::unique_lock<std::mutex> lock(mu_);
                if (stop_) {
                    bool any = false;
                    for (Lane &l : lanes_) any = any || l.busy;
                    if (!any && pending_.empty()) return;
                }
                bool any_busy = false;
                for (Lane &l : lanes_) any_busy = any_busy || l.busy;
                if (!launched) {
                    if (any_busy)
                        cv_.wait_for(lock, std::chrono::microseconds(20));
                    else
                        cv_.wait_for(lock, std::chrono::milliseconds(2),
                                     [this] { return stop_ || !pending_.empty(); });
                }
            }
        }
    }

    int64_t budget_, max_rows_;
    bool device_io_;
    int device_;
    std::vector<Lane> lanes_;
    std::map<std::tuple<int, int, int64_t>, std::unique_ptr<Plan>> plans_;
    int precision_ = 0;
    std::mutex plan_mu_;
    std::string last_err_;
    std::mutex mu_;
    std::condition_variable cv_, cv_done_;
    std::deque<Req> pending_;
    std::vector<Req> completed_;
    int64_t inflight_bytes_ = 0;
    int64_t inflight_ = 0;
    int64_t next_id_ = 0;
    bool stop_ = false;
    bool hold_ = false;
    std::mutex lane_mu_;
    std::atomic<int64_t> batches_{0}, failures_{0};
    std::thread worker_;
};

}  // namespace sipfft

namespace {
std::mutex g_srv_mu;
std::map<void *, std::unique_ptr<sipfft::Server>> g_servers;

sipfft::Server *find_server(void *h)
{
    std::lock_guard<std::mutex> lock(g_srv_mu);
    auto it = g_servers.find(h);
    return it == g_servers.end() ? nullptr : it->second.get();
}

bool valid_class(int type, int dir, int64_t n)
{
    return (type == 0x10 || type == 0x12) && (dir == 0x10 || dir == 0x11) && n > 0 && n <= (int64_t(1) << 27) &&
           (type != 0x12 || n % 2 == 0);
}
}  // namespace

extern "C" {

int32_t asdFftServerCreate(void **server, int64_t budget_bytes, int32_t lanes, int64_t max_rows, int32_t device_io)
{
    if (!server || budget_bytes <= 0 || lanes <= 0 || lanes > 64 || max_rows <= 0) return AsdSip::ACL_ERROR_INVALID_PARAM;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || sipfft::configure_kernels(dev) != cudaSuccess) {
        cudaGetLastError();
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    try {
        auto s = std::make_unique<sipfft::Server>(budget_bytes, lanes, max_rows, device_io != 0, dev);
        void *h = s.get();
        std::lock_guard<std::mutex> lock(g_srv_mu);
        g_servers.emplace(h, std::move(s));
        *server = h;
        return AsdSip::ACL_SUCCESS;
    } catch (...) {
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
}

int32_t asdFftServerSetPrecision(void *server, int32_t mode)
{
    sipfft::Server *s = find_server(server);
    if (!s || mode < 0 || mode > 2) return AsdSip::ACL_ERROR_INVALID_PARAM;
    return s->set_precision(mode) ? AsdSip::ACL_SUCCESS : AsdSip::ACL_ERROR_INVALID_PARAM;
}

int32_t asdFftServerWarm(void *server, int32_t type, int32_t direction, int64_t n)
{
    sipfft::Server *s = find_server(server);
    if (!s || !valid_class(type, direction, n)) return AsdSip::ACL_ERROR_INVALID_PARAM;
    return s->warm(type, direction, n).empty() ? AsdSip::ACL_SUCCESS : AsdSip::ACL_ERROR_API_NOT_SUPPORT;
}

int64_t asdFftServerSubmit(void *server, int32_t type, int32_t direction, int64_t n, int64_t rows, const void *input,
                           void *output)
{
    sipfft::Server *s = find_server(server);
    if (!s || !valid_class(type, direction, n) || rows <= 0 || !input || !output) return -1;
    sipfft::Req r;
    r.type = type;
    r.dir = direction;
    r.n = n;
    r.rows = rows;
    r.in = input;
    r.out = output;
    return s->submit(r);
}

// Waits for all submitted requests; fills up to `cap` completions
// (id, latency seconds; latency < 0 marks a failed request).
int64_t asdFftServerDrain(void *server, int64_t *ids, double *latency_s, int64_t cap)
{
    sipfft::Server *s = find_server(server);
    if (!s) return -1;
    std::vector<sipfft::Req> done = s->drain();
    const int64_t n = std::min<int64_t>(cap, static_cast<int64_t>(done.size()));
    for (int64_t i = 0; i < n; i++) {
        if (ids) ids[i] = done[i].id;
        if (latency_s) latency_s[i] = done[i].t_done < 0 ? -1.0 : done[i].t_done - done[i].t_submit;
    }
    return static_cast<int64_t>(done.size());
}

int32_t asdFftServerHold(void *server, int32_t hold)
{
    sipfft::Server *s = find_server(server);
    if (!s) return AsdSip::ACL_ERROR_INVALID_PARAM;
    s->hold(hold != 0);
    return AsdSip::ACL_SUCCESS;
}

int64_t asdFftServerBatches(void *server)
{
    sipfft::Server *s = find_server(server);
    return s ? s->batches() : -1;
}

int32_t asdFftServerDestroy(void *server)
{
    std::unique_ptr<sipfft::Server> victim;
    {
        std::lock_guard<std::mutex> lock(g_srv_mu);
        auto it = g_servers.find(server);
        if (it == g_servers.end()) return AsdSip::ACL_ERROR_INVALID_PARAM;
        victim = std::move(it->second);
        g_servers.erase(it);
    }
    victim.reset();
    return AsdSip::ACL_SUCCESS;
}

// Poisson load generator: `count` requests at `rate` req/s drawn from the
// classes (types[i], sizes[i]) with rows uniform in [rows_min, rows_max];
// inputs come from per-class pools (pool_in[i], at least rows_max rows) and
// outputs go to per-class pools (pool_out[i]).  Fills per-request latency
// (seconds) and returns the wall time from the first arrival to the last
// completion.
double asdFftServeRun(void *server, double rate, int64_t count, uint64_t seed, int32_t nclasses, const int32_t *types,
                      const int64_t *sizes, const void *const *pool_in, void *const *pool_out, int64_t rows_min,
                      int64_t rows_max, int32_t direction, double *latency_s, int64_t *rows_out, int32_t *class_out)
{
    sipfft::Server *s = find_server(server);
    if (!s || rate <= 0 || count <= 0 || nclasses <= 0 || rows_min <= 0 || rows_max < rows_min) return -1.0;
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate);
    std::uniform_int_distribution<int> pick(0, nclasses - 1);
    std::uniform_int_distribution<int64_t> rows_d(rows_min, rows_max);
    std::vector<int64_t> id_of(count);
    const auto t0 = std::chrono::steady_clock::now();
    double t_arrive = 0.0;
    for (int64_t i = 0; i < count; i++) {
        t_arrive += gap(rng);
        const int c = pick(rng);
        const int64_t rows = rows_d(rng);
        std::this_thread::sleep_until(t0 + std::chrono::duration<double>(t_arrive));
        id_of[i] = asdFftServerSubmit(server, types[c], direction, sizes[c], rows, pool_in[c], pool_out[c]);
        if (rows_out) rows_out[i] = rows;
        if (class_out) class_out[i] = c;
    }
    std::vector<int64_t> ids(count);
    std::vector<double> lat(count);
    const int64_t got = asdFftServerDrain(server, ids.data(), lat.data(), count);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::map<int64_t, double> by_id;
    for (int64_t i = 0; i < got && i < count; i++) by_id[ids[i]] = lat[i];
    for (int64_t i = 0; i < count; i++) {
        auto it = by_id.find(id_of[i]);
        latency_s[i] = it == by_id.end() ? -1.0 : it->second;
    }
    return wall;
}

}  // extern "C"
