// oceanlib-b200: the serving loop (ocean_server_*).
//
// Many sessions - each an ocean and optionally an iWave interaction field -
// live on one GPU; clients submit update and height-query requests from any
// thread as they arrive. A dispatcher thread does continuous batching: while
// up to `max_inflight` batches run on the GPU it gathers what has arrived
// since, and launches it as one batch:
//
//   one H2D copy    every per-batch table (ocean pointer tables and times,
//                   resolved sources, per-substep field lists, query jobs
//                   and points) from one pinned block;
//   ocean frames    one persistent frame kernel per ocean size over every
//                   session updating in this batch (pointer-table form);
//   interaction     one source-mean launch for all sources, then per field
//                   kind and substep one batched source-stamp and one batched
//                   stencil launch over every session stepping, one finalize;
//   queries         one launch for every height request of the batch;
//   D2H copy        all heights, and the frame kernel's error word.
//
// Per session, requests keep their submission order: a batch takes at most
// one update of a session and then only queries that follow it, so a query
// sees exactly the updates submitted before it. Batches run in order on one
// stream. Each session's arithmetic is the single-session arithmetic (same
// kernels, same per-cell order), so a result is the same alone and in any
// mix. Session memory comes from a stream-ordered pool: a session is
// admitted when its bytes fit in the budget (FIFO), and a closed session's
// memory is released behind the last batch that used it.

#include "../../include/ocean_b200.h"
#include "host_util.h"
#include "iwave.h"
#include "iwave_host.h"
#include "ocean_host.h"
#include "serve.h"
#include "spectrum.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace ocean_b200 {
namespace {

using Clock = std::chrono::steady_clock;
constexpr double kInvTwoPi = 0.159154943091895335769;
constexpr uint64_t kDefaultBudget = 120000000000ull;  // 120 GB
constexpr size_t kAlign = 256;

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void server_desc_defaults(ocean_server_desc* d)
{
    std::memset(d, 0, sizeof(*d));
    d->struct_size = sizeof(ocean_server_desc);
    d->hbm_budget = kDefaultBudget;
    d->max_inflight = 2;
    d->max_batch_requests = 4096;
    d->max_batch_points = 1u << 20;
    d->max_query_points = 65536;
    d->fft_form = OCEAN_FFT_EXACT;
}

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Nearest-rank percentile (q in (0, 1]).
double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    size_t rank = static_cast<size_t>(std::ceil(q * static_cast<double>(v.size())));
    rank = std::min(std::max<size_t>(rank, 1), v.size());
    std::nth_element(v.begin(), v.begin() + static_cast<ptrdiff_t>(rank - 1), v.end());
    return v[rank - 1];
}

// Field kinds share the fitted stencil and damping tables.
bool same_field_kind(const ocean_interaction_desc& a, const ocean_interaction_desc& b)
{
    return a.size == b.size && a.extent == b.extent && a.kernel_radius == b.kernel_radius &&
           a.damping == b.damping && a.absorb_cells == b.absorb_cells && a.fixed_dt == b.fixed_dt &&
           a.max_substeps == b.max_substeps && a.max_sources == b.max_sources && a.gravity == b.gravity &&
           a.water_depth == b.water_depth && a.obstruction == b.obstruction;
}

// Byte layout of one session's single allocation.
struct SessionLayout {
    size_t h0 = 0, geom = 0, kvec = 0, disp = 0, normal = 0, vel = 0;
    size_t plane0 = 0, plane1 = 0, field_out = 0;
    size_t total = 0;
};

SessionLayout session_layout(const ocean_desc& od, const ocean_interaction_desc* fd)
{
    SessionLayout l;
    const size_t cells = static_cast<size_t>(od.size) * od.size;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += round_up(bytes, kAlign);
        return at;
    };
    l.h0 = take(cells * sizeof(float2));
    l.geom = take(cells * sizeof(float2));
    l.kvec = take(od.size * sizeof(float));
    l.disp = take(cells * sizeof(float4));
    l.normal = take(cells * sizeof(float4));
    if (od.compute_velocity) l.vel = take(cells * sizeof(float4));
    if (fd != nullptr) {
        const size_t n = fd->size, p = fd->kernel_radius;
        const size_t stride = (n + 2 * p + 15u) & ~size_t(15);
        const size_t plane = (n + 2 * p) * stride * sizeof(float);
        l.plane0 = take(plane);
        l.plane1 = take(plane);
        l.field_out = take(n * n * sizeof(float4));
    }
    l.total = off;
    return l;
}

enum class Kind { Update, Query, Close };

struct Session;

struct Request {
    uint64_t ticket = 0;
    Kind kind = Kind::Update;
    Session* session = nullptr;
    Clock::time_point submitted;
    double time = 0.0;
    float dt = 0.0f;
    std::vector<ocean_disturbance> sources;
    std::vector<float2> xz;
    float* out = nullptr;
    size_t out_offset = 0;  // float index into the batch's height block
};

// Ocean sessions of one (N, velocity) share the frame kernel's twiddles,
// intermediate ring and work-queue counters.
struct OceanKind {
    uint32_t n = 0;
    bool velocity = false;
    int log_n = 0, nf = 4;
    int grid = 0;
    DevBuf<float2> tw, inter;
    unsigned* queue = nullptr;  // pool allocation, 1 + 2 * queue_cap
    size_t queue_cap = 0;
    size_t bytes = 0;
};

struct FieldKind {
    ocean_interaction_desc desc{};
    IWaveSetup setup;
    DevBuf<float> c1, c2;
    bool ready = false;     // tables on the device (dispatcher thread)
    bool reserved = false;  // their bytes counted in the budget (under the lock)
    size_t bytes = 0;
};

struct Session {
    uint64_t id = 0;
    ocean_session_state state = OCEAN_SESSION_WAITING;
    ocean_desc od{};
    bool has_field = false;
    ocean_interaction_desc fd{};
    SessionLayout layout;
    size_t bytes = 0;
    OceanKind* ok = nullptr;
    FieldKind* fk = nullptr;
    std::deque<Request*> queue;
    bool in_ready = false;
    bool closing = false;
    uint64_t last_ticket = 0;
    // The reference's constructor evaluates t = 0 (src/ocean.cpp:275-277):
    // an internal update (ticket 0) at the head of the queue does the same.
    std::unique_ptr<Request> init;
    // device state
    unsigned char* block = nullptr;
    OceanSlot slot{};
    float* plane[2] = {nullptr, nullptr};
    float4* field_out = nullptr;
    int cur = 0;  // which plane holds h^n
    IWaveClock clock;
    IWaveQueue sources;
};

// One batch in flight: its staging blocks, events and requests.
struct BatchCtx {
    HostBuf<unsigned char> host_in;
    size_t host_in_cap = 0;
    unsigned char* dev = nullptr;  // pool allocation: inputs, then heights
    size_t dev_cap = 0;
    HostBuf<float> host_out;       // heights + the error word
    size_t host_out_cap = 0;       // floats
    cudaEvent_t start = nullptr, done = nullptr;
    std::vector<Request*> requests;
    std::vector<Session*> closes;
    uint64_t points = 0;
    uint32_t kernels = 0;
    float gpu_ms = 0.0f;
    bool complete = false;
    bool failed = false;
    void* server = nullptr;
};

struct Layout {
    size_t size = 0;
    size_t add(size_t bytes)
    {
        const size_t at = size;
        size = round_up(size + bytes, 16);
        return at;
    }
};

}  // namespace

class Server {
public:
    explicit Server(const ocean_server_desc& d) : desc_(d)
    {
        if (desc_.max_inflight == 0) desc_.max_inflight = 1;
        if (desc_.max_batch_requests == 0) throw std::invalid_argument("max_batch_requests");
        if (desc_.max_batch_points == 0 || desc_.max_query_points == 0) throw std::invalid_argument("points");
        if (desc_.fft_form != OCEAN_FFT_EXACT && desc_.fft_form != OCEAN_FFT_FAST &&
            desc_.fft_form != OCEAN_FFT_TENSOR && desc_.fft_form != OCEAN_FFT_PRECISE)
            throw std::invalid_argument("fft_form");
        check(cudaGetDevice(&device_), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "SM count");
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device_;
        check(cudaMemPoolCreate(&pool_, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // keep freed memory cached in the pool
        check(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep), "pool attribute");
        error_ = DevBuf<unsigned>(1);
        mix_ticket_ = DevBuf<unsigned>(1);
        check(cudaMemsetAsync(error_.p, 0, sizeof(unsigned), stream_), "memset");
        ctxs_.resize(desc_.max_inflight);
        // Staging for a full batch of query points plus the tables and sources
        // of a few thousand updates, reserved now so that a backlog never
        // waits on pinned-memory allocation.
        const size_t in_reserve = static_cast<size_t>(desc_.max_batch_points) * sizeof(float2) + (4u << 20);
        const size_t out_reserve = static_cast<size_t>(desc_.max_batch_points) + 4;
        for (auto& c : ctxs_) {
            c = std::make_unique<BatchCtx>();
            check(cudaEventCreate(&c->start), "event");
            check(cudaEventCreate(&c->done), "event");
            c->server = this;
            ensure_host(c.get(), in_reserve, out_reserve);
            free_ctx_.push_back(c.get());
        }
        staging_growths_ = 0;
        stats_t0_ = Clock::now();
        thread_ = std::thread([this] { run(); });
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (thread_.joinable()) thread_.join();
        cudaStreamSynchronize(stream_);
        for (auto& kv : sessions_)
            if (kv.second->block) cudaFreeAsync(kv.second->block, stream_);
        for (auto& k : ocean_kinds_)
            if (k->queue) cudaFreeAsync(k->queue, stream_);
        for (auto& c : ctxs_) {
            if (c->dev) cudaFreeAsync(c->dev, stream_);
            if (c->start) cudaEventDestroy(c->start);
            if (c->done) cudaEventDestroy(c->done);
        }
        cudaStreamSynchronize(stream_);
        ocean_kinds_.clear();
        field_kinds_.clear();
        if (pool_) cudaMemPoolDestroy(pool_);
        cudaStreamDestroy(stream_);
    }

    static uint64_t session_bytes(const ocean_desc& od, const ocean_interaction_desc* fd)
    {
        return session_layout(od, fd).total;
    }

    uint64_t open(const ocean_desc& od_in, const ocean_interaction_desc* fd_in)
    {
        ocean_desc od = od_in;
        validate(od);
        // The dispatcher batches sessions into persistent frame launches.
        if (od.size > kMaxPersistentSize) throw std::invalid_argument("session size above 1024");
        if (desc_.fft_form == OCEAN_FFT_TENSOR && (od.size < 64 || od.size > 512))
            throw std::invalid_argument("the tensor-core form needs N = 64 to 512");
        ocean_interaction_desc fd{};
        if (fd_in != nullptr) {
            fd = *fd_in;
            validate_interaction(fd);
        }
        const SessionLayout layout = session_layout(od, fd_in ? &fd : nullptr);
        if (layout.total > desc_.hbm_budget) throw std::length_error("session larger than the budget");
        // The field kind's stencil fit (host work, milliseconds) happens here,
        // on the caller's thread, so the dispatcher never stalls on it.
        FieldKind* fk = nullptr;
        if (fd_in != nullptr) fk = field_kind(fd);
        std::lock_guard<std::mutex> lk(mu_);
        auto s = std::make_unique<Session>();
        s->id = next_session_++;
        s->od = od;
        s->has_field = fd_in != nullptr;
        s->fd = fd;
        s->layout = layout;
        s->bytes = layout.total;
        s->fk = fk;
        if (fk) s->sources.reset(fd.max_sources);
        s->init = std::make_unique<Request>();
        s->init->kind = Kind::Update;
        s->init->session = s.get();
        s->init->submitted = Clock::now();
        s->queue.push_back(s->init.get());
        Session* raw = s.get();
        sessions_[raw->id] = std::move(s);
        waiting_.push_back(raw);
        cv_.notify_all();
        return raw->id;
    }

    ocean_session_state state(uint64_t id)
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = sessions_.find(id);
        return it == sessions_.end() ? OCEAN_SESSION_CLOSED : it->second->state;
    }

    uint64_t submit(uint64_t id, std::unique_ptr<Request> r)
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = sessions_.find(id);
        if (it == sessions_.end() || it->second->closing || it->second->state == OCEAN_SESSION_CLOSED)
            throw std::invalid_argument("session");
        Session* s = it->second.get();
        r->ticket = next_ticket_++;
        r->session = s;
        r->submitted = Clock::now();
        if (r->kind == Kind::Close) s->closing = true;
        s->last_ticket = r->ticket;
        Request* raw = r.get();
        pending_[raw->ticket] = std::move(r);
        s->queue.push_back(raw);
        if (s->state == OCEAN_SESSION_ACTIVE && !s->in_ready) {
            s->in_ready = true;
            ready_.push_back(s);
        }
        ++submitted_;
        cv_.notify_all();
        return raw->ticket;
    }

    ocean_status wait(uint64_t ticket, uint32_t timeout_ms)
    {
        std::unique_lock<std::mutex> lk(mu_);
        if (ticket == 0 || ticket >= next_ticket_) return OCEAN_ERROR_INVALID_ARG;
        const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms);
        while (pending_.count(ticket) != 0) {
            if (done_cv_.wait_until(lk, deadline) == std::cv_status::timeout && pending_.count(ticket) != 0)
                return OCEAN_ERROR_TIMEOUT;
        }
        return failed_.count(ticket) ? OCEAN_ERROR_DEVICE : OCEAN_OK;
    }

    ocean_status drain(uint32_t timeout_ms)
    {
        std::unique_lock<std::mutex> lk(mu_);
        const uint64_t last = next_ticket_;
        const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms);
        auto done = [&] {
            for (const auto& kv : pending_)
                if (kv.first < last) return false;
            return true;
        };
        while (!done()) {
            if (done_cv_.wait_until(lk, deadline) == std::cv_status::timeout && !done()) return OCEAN_ERROR_TIMEOUT;
        }
        return OCEAN_OK;
    }

    void read_session(uint64_t id, float* disp, float* normal, float* field)
    {
        uint64_t last = 0;
        Session* s = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = sessions_.find(id);
            if (it == sessions_.end() || it->second->state == OCEAN_SESSION_CLOSED)
                throw std::invalid_argument("session");
            s = it->second.get();
            last = s->last_ticket;
        }
        if (last != 0) {
            const ocean_status st = wait(last, 600000);
            if (st == OCEAN_ERROR_TIMEOUT) throw TimeoutError();
        }
        {
            // Admission and the t = 0 frame happen on the dispatcher thread.
            std::unique_lock<std::mutex> lk(mu_);
            done_cv_.wait_for(lk, std::chrono::seconds(600),
                              [&] { return s->state != OCEAN_SESSION_WAITING && s->init == nullptr; });
            if (s->state != OCEAN_SESSION_ACTIVE) throw std::invalid_argument("session not admitted");
            if (s->init != nullptr) throw TimeoutError();
        }
        const size_t cells = static_cast<size_t>(s->od.size) * s->od.size;
        if (disp) check(cudaMemcpy(disp, s->slot.disp, cells * sizeof(float4), cudaMemcpyDeviceToHost), "read");
        if (normal) check(cudaMemcpy(normal, s->slot.normal, cells * sizeof(float4), cudaMemcpyDeviceToHost), "read");
        if (field && s->has_field) {
            const size_t fc = static_cast<size_t>(s->fd.size) * s->fd.size;
            check(cudaMemcpy(field, s->field_out, fc * sizeof(float4), cudaMemcpyDeviceToHost), "read");
        }
    }

    void stats(ocean_server_stats* o)
    {
        std::vector<double> all, up, qu;
        std::memset(o, 0, sizeof(*o));
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (const auto& kv : sessions_) {
                const Session& s = *kv.second;
                if (s.state == OCEAN_SESSION_ACTIVE) ++o->sessions_active;
                else if (s.state == OCEAN_SESSION_WAITING) ++o->sessions_waiting;
                else ++o->sessions_closed;
            }
            o->bytes_in_use = in_use_;
            o->hbm_budget = desc_.hbm_budget;
            o->requests_submitted = submitted_;
            o->requests_completed = completed_;
            o->requests_failed = failed_count_;
            o->updates_completed = updates_done_;
            o->queries_completed = queries_done_;
            o->query_points_completed = points_done_;
            o->batches = batches_;
            o->kernel_launches = kernels_;
            o->bytes_staging = staging_bytes_;
            o->mean_batch_requests = batches_ ? static_cast<double>(batched_requests_) / batches_ : 0.0;
            o->gpu_busy_ms = gpu_ms_;
            o->wall_ms = ms_between(stats_t0_, Clock::now());
            o->dispatch_max_ms = dispatch_max_ms_;
            o->staging_growths = staging_growths_;
            up = lat_update_;
            qu = lat_query_;
        }
        all = up;
        all.insert(all.end(), qu.begin(), qu.end());
        o->latency_p50_ms = percentile(all, 0.50);
        o->latency_p99_ms = percentile(all, 0.99);
        o->latency_max_ms = all.empty() ? 0.0 : *std::max_element(all.begin(), all.end());
        o->update_p50_ms = percentile(up, 0.50);
        o->update_p99_ms = percentile(up, 0.99);
        o->query_p50_ms = percentile(qu, 0.50);
        o->query_p99_ms = percentile(qu, 0.99);
    }

    void reset_stats()
    {
        std::lock_guard<std::mutex> lk(mu_);
        submitted_ = completed_ = failed_count_ = updates_done_ = queries_done_ = points_done_ = 0;
        batches_ = kernels_ = batched_requests_ = 0;
        gpu_ms_ = 0.0;
        dispatch_max_ms_ = 0.0;
        staging_growths_ = 0;
        lat_update_.clear();
        lat_query_.clear();
        samples_.clear();
        stats_t0_ = Clock::now();
    }

    uint64_t samples(double* submit_ms, double* latency_ms, int32_t* kind, uint64_t capacity)
    {
        std::lock_guard<std::mutex> lk(mu_);
        const uint64_t n = std::min<uint64_t>(capacity, samples_.size());
        for (uint64_t i = 0; i < n; ++i) {
            if (submit_ms) submit_ms[i] = samples_[i].submit_ms;
            if (latency_ms) latency_ms[i] = samples_[i].latency_ms;
            if (kind) kind[i] = samples_[i].kind;
        }
        return samples_.size();
    }

    const ocean_server_desc& desc() const { return desc_; }

private:
    // ---- kinds --------------------------------------------------------------
    FieldKind* field_kind(const ocean_interaction_desc& d)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto& k : field_kinds_)
                if (same_field_kind(k->desc, d)) return k.get();
        }
        auto k = std::make_unique<FieldKind>();
        k->desc = d;
        k->setup = iwave_setup(d);  // throws for an unstable stencil
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& e : field_kinds_)
            if (same_field_kind(e->desc, d)) return e.get();
        field_kinds_.push_back(std::move(k));
        return field_kinds_.back().get();
    }

    // Bytes a new ocean / field kind would add (shared tables).
    size_t ocean_kind_bytes(const ocean_desc& od) const
    {
        const size_t cells = static_cast<size_t>(od.size) * od.size;
        const int nf = od.compute_velocity ? 6 : 4;
        return round_up((od.size - 1) * sizeof(float2), kAlign) + round_up(3 * cells * nf * sizeof(float2), kAlign);
    }

    OceanKind* find_ocean_kind(const ocean_desc& od)
    {
        for (auto& k : ocean_kinds_)
            if (k->n == od.size && k->velocity == (od.compute_velocity != 0)) return k.get();
        return nullptr;
    }

    // Dispatcher thread only.
    OceanKind* make_ocean_kind(const ocean_desc& od)
    {
        auto k = std::make_unique<OceanKind>();
        k->n = od.size;
        k->velocity = od.compute_velocity != 0;
        k->log_n = ilog2u(k->n);
        k->nf = k->velocity ? 6 : 4;
        const size_t cells = static_cast<size_t>(k->n) * k->n;
        k->tw = DevBuf<float2>(k->n - 1);
        k->inter = DevBuf<float2>(3 * cells * k->nf);
        const std::vector<float2> tw = stage_twiddles(k->n);
        check(cudaMemcpyAsync(k->tw.p, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, stream_),
              "twiddles");
        const int per_sm = frame_blocks_per_sm(k->log_n, k->nf, desc_.fft_form, false);
        if (per_sm <= 0) throw DeviceError(cudaErrorInvalidConfiguration, "frame occupancy");
        k->grid = per_sm * sms_;
        k->bytes = ocean_kind_bytes(od);
        check(cudaStreamSynchronize(stream_), "twiddles");
        ocean_kinds_.push_back(std::move(k));
        return ocean_kinds_.back().get();
    }

    void ensure_field_tables(FieldKind* k)
    {
        if (k->ready) return;
        std::vector<float> c1, c2;
        iwave_damping(k->desc, k->setup, c1, c2);
        k->c1 = DevBuf<float>(c1.size());
        k->c2 = DevBuf<float>(c2.size());
        check(cudaMemcpyAsync(k->c1.p, c1.data(), c1.size() * sizeof(float), cudaMemcpyHostToDevice, stream_),
              "damping");
        check(cudaMemcpyAsync(k->c2.p, c2.data(), c2.size() * sizeof(float), cudaMemcpyHostToDevice, stream_),
              "damping");
        check(cudaStreamSynchronize(stream_), "damping");
        k->bytes = 2 * round_up(c1.size() * sizeof(float), kAlign);
        k->ready = true;
    }

    // ---- admission (dispatcher thread) ---------------------------------------
    // Under the lock: pick the waiting sessions (FIFO) whose bytes, plus any
    // shared table a first session of its kind brings, fit in the budget.
    std::vector<Session*> pick_admissions_locked()
    {
        std::vector<Session*> out;
        while (!waiting_.empty()) {
            Session* s = waiting_.front();
            const size_t cost = admission_cost_locked(s);
            if (in_use_ + cost > desc_.hbm_budget) break;
            waiting_.pop_front();
            in_use_ += cost;
            ocean_kind_keys_.insert(ocean_key(s->od));
            if (s->fk) s->fk->reserved = true;
            out.push_back(s);
        }
        return out;
    }

    static uint64_t ocean_key(const ocean_desc& od)
    {
        return (static_cast<uint64_t>(od.size) << 1) | (od.compute_velocity ? 1u : 0u);
    }

    // Session bytes plus the shared tables a first session of its kinds brings.
    size_t admission_cost_locked(const Session* s) const
    {
        size_t cost = s->bytes;
        if (ocean_kind_keys_.count(ocean_key(s->od)) == 0) cost += ocean_kind_bytes(s->od);
        if (s->fk && !s->fk->reserved)
            cost += 2 * round_up(static_cast<size_t>(s->fd.size) * s->fd.size * sizeof(float), kAlign);
        return cost;
    }

    // Outside the lock: allocate and build each admitted session.
    void admit(Session* s)
    {
        OceanKind* k = find_ocean_kind(s->od);
        if (!k) k = make_ocean_kind(s->od);
        s->ok = k;
        if (s->fk) ensure_field_tables(s->fk);
        check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s->block), s->bytes, pool_, stream_),
              "session allocation");
        const SessionLayout& l = s->layout;
        unsigned char* b = s->block;
        s->slot.h0 = reinterpret_cast<const float2*>(b + l.h0);
        s->slot.omega_kinv = reinterpret_cast<const float2*>(b + l.geom);
        s->slot.kvec = reinterpret_cast<const float*>(b + l.kvec);
        s->slot.disp = reinterpret_cast<float4*>(b + l.disp);
        s->slot.normal = reinterpret_cast<float4*>(b + l.normal);
        s->slot.velocity = s->od.compute_velocity ? reinterpret_cast<float4*>(b + l.vel) : nullptr;
        s->slot.cst.lambda = s->od.choppiness;
        s->slot.cst.foam_threshold = s->od.foam_threshold;
        // src/core/evolve.cpp:251-252
        s->slot.cst.inv_threshold = (s->od.foam_threshold > 1e-6f) ? (1.0f / s->od.foam_threshold) : 0.0f;
        s->slot.cst.geom = 0;
        const SpectrumParams sp = spectrum_params(s->od);
        check(launch_geometry(sp, reinterpret_cast<float2*>(b + l.geom), reinterpret_cast<float*>(b + l.kvec), stream_),
              "geometry kernel");
        check(launch_h0(sp, reinterpret_cast<float2*>(b + l.h0), stream_), "h0 kernel");
        const size_t cells = static_cast<size_t>(s->od.size) * s->od.size;
        // Before the first update the outputs read as an ocean at rest.
        check(cudaMemsetAsync(b + l.disp, 0, cells * sizeof(float4), stream_), "memset");
        check(cudaMemsetAsync(b + l.normal, 0, cells * sizeof(float4), stream_), "memset");
        if (s->has_field) {
            const IWaveSetup& g = s->fk->setup;
            const size_t plane = static_cast<size_t>(g.rows) * g.stride;
            s->plane[0] = reinterpret_cast<float*>(b + l.plane0);
            s->plane[1] = reinterpret_cast<float*>(b + l.plane1);
            s->field_out = reinterpret_cast<float4*>(b + l.field_out);
            check(cudaMemsetAsync(s->plane[0], 0, plane * sizeof(float), stream_), "memset");
            check(cudaMemsetAsync(s->plane[1], 0, plane * sizeof(float), stream_), "memset");
            // finalize of an all-zero field is all zero (src/interaction.cpp:497)
            check(cudaMemsetAsync(s->field_out, 0, g.cells * sizeof(float4), stream_), "memset");
            s->cur = 0;
        }
    }

    IWaveField field_of(const Session& s, int cur) const
    {
        const IWaveSetup& g = s.fk->setup;
        const size_t off = static_cast<size_t>(g.p) * g.stride + g.p;
        IWaveField f;
        f.cur = s.plane[cur] + off;
        f.old = s.plane[cur ^ 1] + off;
        f.c1 = s.fk->c1.p;
        f.c2 = s.fk->c2.p;
        f.out = s.field_out;
        f.n = static_cast<int32_t>(g.n);
        f.stride = g.stride;
        f.gdt2 = s.fd.gravity * g.dt * g.dt;
        f.inv_two_cell = 0.5f / g.cell;
        f.inv_dt = 1.0f / g.dt;
        f.inv_dt_d = 1.0 / static_cast<double>(g.dt);
        return f;
    }

    // ---- batch building (under the lock) ---------------------------------------
    struct FieldWork {
        Session* s;
        uint32_t steps;
        int cur0;
        std::vector<uint32_t> first;  // absolute offsets into Plan::sources
    };
    struct Plan {
        std::map<OceanKind*, std::vector<std::pair<Session*, double>>> frames;
        std::map<FieldKind*, std::vector<FieldWork>> fields;
        std::vector<IWaveSource> sources;
        std::vector<Request*> queries;
        uint64_t points = 0;
    };

    bool build_locked(BatchCtx* c, Plan& plan)
    {
        c->requests.clear();
        c->closes.clear();
        const size_t rounds = ready_.size();
        bool full = false;
        for (size_t i = 0; i < rounds && !full; ++i) {
            Session* s = ready_.front();
            ready_.pop_front();
            bool took_any = false;
            while (!s->queue.empty()) {
                Request* r = s->queue.front();
                if (c->requests.size() >= desc_.max_batch_requests) {
                    full = true;
                    break;
                }
                if (r->kind == Kind::Update) {
                    if (took_any) break;
                    take_update(s, r, plan);
                } else if (r->kind == Kind::Query) {
                    if (plan.points + r->xz.size() > desc_.max_batch_points || plan.queries.size() >= 65535) {
                        full = true;
                        break;
                    }
                    r->out_offset = plan.points;
                    plan.points += r->xz.size();
                    plan.queries.push_back(r);
                } else {
                    c->closes.push_back(s);
                }
                took_any = true;
                s->queue.pop_front();
                c->requests.push_back(r);
                if (r->kind == Kind::Close) break;
            }
            if (!s->queue.empty() && !closed_in(c, s)) {
                ready_.push_back(s);
            } else {
                s->in_ready = false;
            }
        }
        return !c->requests.empty();
    }

    static bool closed_in(const BatchCtx* c, const Session* s)
    {
        return std::find(c->closes.begin(), c->closes.end(), s) != c->closes.end();
    }

    // Host side of one session update: the ocean frame's time, and the field's
    // accumulator, source queue and substep plan (InteractionField::update,
    // src/interaction.cpp:531-587).
    void take_update(Session* s, Request* r, Plan& plan)
    {
        plan.frames[s->ok].emplace_back(s, r->time);
        if (!s->has_field) return;
        for (const ocean_disturbance& d : r->sources) s->sources.add(d);
        const IWaveSetup& g = s->fk->setup;
        const uint32_t steps = s->clock.advance(r->dt, g.dt, s->fd.max_substeps);
        if (steps == 0) {
            s->sources.keep_impulses();
            return;
        }
        FieldWork w;
        w.s = s;
        w.steps = steps;
        w.cur0 = s->cur;
        s->sources.resolve_all(steps, g, 0, 0, plan.sources, w.first);
        plan.fields[s->fk].push_back(std::move(w));
        s->cur = (s->cur + static_cast<int>(steps)) & 1;
    }

    // ---- staging and launch (dispatcher thread, outside the lock) ----------------
    void ensure_host(BatchCtx* c, size_t in_bytes, size_t out_floats)
    {
        // Growth past the size reserved at creation pins new host memory (slow,
        // and freeing the old block synchronises the device): rare by design.
        if (in_bytes > c->host_in_cap) {
            const size_t cap = std::max(in_bytes, c->host_in_cap * 2);
            c->host_in = HostBuf<unsigned char>(cap, false);
            c->host_in_cap = cap;
            ++staging_growths_;
        }
        if (out_floats > c->host_out_cap) {
            const size_t cap = std::max(out_floats, c->host_out_cap * 2);
            c->host_out = HostBuf<float>(cap, false);
            c->host_out_cap = cap;
            ++staging_growths_;
        }
        const size_t dev_bytes = in_bytes + round_up(out_floats * sizeof(float), 16);
        if (dev_bytes > c->dev_cap) {
            const size_t cap = std::max(dev_bytes, c->dev_cap * 2);
            if (c->dev) check(cudaFreeAsync(c->dev, stream_), "free staging");
            c->dev = nullptr;
            check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&c->dev), cap, pool_, stream_), "staging");
            std::lock_guard<std::mutex> lk(mu_);
            staging_bytes_ += cap - c->dev_cap;  // reported, not part of the session budget
            c->dev_cap = cap;
        }
    }

    void ensure_queue(OceanKind* k, size_t count)
    {
        if (count <= k->queue_cap) return;
        const size_t cap = std::max(count, k->queue_cap * 2);
        if (k->queue) check(cudaFreeAsync(k->queue, stream_), "free queue");
        k->queue = nullptr;
        check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&k->queue), (1 + 2 * cap) * sizeof(unsigned), pool_,
                                      stream_), "queue");
        k->queue_cap = cap;
    }

    void launch(BatchCtx* c, Plan& plan)
    {
        // Layout of the input block.
        Layout L;
        struct OceanPart { OceanKind* k; size_t slots, top, count; };
        std::vector<OceanPart> oparts;
        for (auto& kv : plan.frames) {
            OceanPart p{kv.first, 0, 0, kv.second.size()};
            p.slots = L.add(p.count * sizeof(OceanSlot));
            p.top = L.add(p.count * sizeof(double));
            oparts.push_back(p);
        }
        const size_t src_off = L.add(plan.sources.size() * sizeof(IWaveSource));
        struct StepPart { size_t fields, ranges, count; bool any_sources; };
        struct FieldPart { FieldKind* k; std::vector<StepPart> steps; size_t fin, fin_count; };
        std::vector<FieldPart> fparts;
        for (auto& kv : plan.fields) {
            FieldPart fp;
            fp.k = kv.first;
            uint32_t max_steps = 0;
            for (const FieldWork& w : kv.second) max_steps = std::max(max_steps, w.steps);
            for (uint32_t st = 0; st < max_steps; ++st) {
                StepPart sp{0, 0, 0, false};
                for (const FieldWork& w : kv.second)
                    if (w.steps > st) ++sp.count;
                sp.fields = L.add(sp.count * sizeof(IWaveField));
                sp.ranges = L.add(sp.count * sizeof(int2));
                fp.steps.push_back(sp);
            }
            fp.fin_count = kv.second.size();
            fp.fin = L.add(fp.fin_count * sizeof(IWaveField));
            fparts.push_back(std::move(fp));
        }
        const size_t jobs_off = L.add(plan.queries.size() * sizeof(QueryJob));
        const size_t pts_off = L.add(plan.points * sizeof(float2));
        const size_t in_bytes = L.size;
        const size_t out_floats = plan.points + 4;  // heights, then the error word
        ensure_host(c, in_bytes, out_floats);
        for (auto& p : oparts) ensure_queue(p.k, p.count);

        unsigned char* h = c->host_in.p;
        unsigned char* d = c->dev;
        float* dev_heights = reinterpret_cast<float*>(d + in_bytes);

        // Fill the block.
        for (size_t i = 0; i < oparts.size(); ++i) {
            const auto& list = plan.frames[oparts[i].k];
            OceanSlot* slots = reinterpret_cast<OceanSlot*>(h + oparts[i].slots);
            double* top = reinterpret_cast<double*>(h + oparts[i].top);
            for (size_t j = 0; j < list.size(); ++j) {
                slots[j] = list[j].first->slot;
                top[j] = list[j].second * kInvTwoPi;  // hoisted as src/core/evolve.cpp:33
            }
        }
        if (!plan.sources.empty())
            std::memcpy(h + src_off, plan.sources.data(), plan.sources.size() * sizeof(IWaveSource));
        size_t fi = 0;
        for (auto& kv : plan.fields) {
            FieldPart& fp = fparts[fi++];
            for (size_t st = 0; st < fp.steps.size(); ++st) {
                StepPart& sp = fp.steps[st];
                IWaveField* fl = reinterpret_cast<IWaveField*>(h + sp.fields);
                int2* rg = reinterpret_cast<int2*>(h + sp.ranges);
                size_t k = 0;
                for (const FieldWork& w : kv.second) {
                    if (w.steps <= st) continue;
                    fl[k] = field_of(*w.s, (w.cur0 + static_cast<int>(st)) & 1);
                    const int first = static_cast<int>(w.first[st]);
                    const int count = static_cast<int>(w.first[st + 1] - w.first[st]);
                    rg[k] = make_int2(first, count);
                    if (count > 0) sp.any_sources = true;
                    ++k;
                }
            }
            IWaveField* fin = reinterpret_cast<IWaveField*>(h + fp.fin);
            size_t k = 0;
            for (const FieldWork& w : kv.second)
                fin[k++] = field_of(*w.s, (w.cur0 + static_cast<int>(w.steps)) & 1);
        }
        QueryJob* jobs = reinterpret_cast<QueryJob*>(h + jobs_off);
        float2* pts = reinterpret_cast<float2*>(h + pts_off);
        uint32_t max_points = 0;
        for (size_t q = 0; q < plan.queries.size(); ++q) {
            Request* r = plan.queries[q];
            const Session& s = *r->session;
            QueryJob j;
            std::memset(&j, 0, sizeof(j));
            j.disp = s.slot.disp;
            j.normal = s.slot.normal;
            j.xz = reinterpret_cast<const float2*>(d + pts_off) + r->out_offset;
            j.out = dev_heights + r->out_offset;
            j.n = static_cast<int32_t>(s.od.size);
            j.inv_cell = static_cast<float>(s.od.size) / s.od.patch_length;
            if (s.has_field) {
                j.field = s.field_out;
                j.fn = static_cast<int32_t>(s.fd.size);
                j.cell = s.fk->setup.cell;
                j.origin_x = 0.0f;
                j.origin_z = 0.0f;
            }
            j.count = static_cast<uint32_t>(r->xz.size());
            max_points = std::max(max_points, j.count);
            jobs[q] = j;
            std::memcpy(pts + r->out_offset, r->xz.data(), r->xz.size() * sizeof(float2));
        }

        // Launch.
        uint32_t kernels = 0;
        check(cudaEventRecord(c->start, stream_), "event");
        if (in_bytes > 0) check(cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, stream_), "batch upload");
        // The batch's oceans: one launch for every size when the sizes allow
        // it (mixed_frame_kernel: N up to 1024, one field count, an FP32
        // form), else one persistent launch per size.
        bool one_launch = oparts.size() > 1 && oparts.size() <= static_cast<size_t>(kMaxMixedGroups) &&
                          desc_.fft_form != OCEAN_FFT_TENSOR;
        for (const OceanPart& p : oparts)
            one_launch = one_launch && mixed_size_ok(p.k->log_n) && p.k->nf == oparts[0].k->nf;
        MixedArgs m{};
        for (const OceanPart& p : oparts) {
            OceanKind* k = p.k;
            const int count = static_cast<int>(p.count);
            check(cudaMemsetAsync(k->queue, 0, (1 + 2 * p.count) * sizeof(unsigned), stream_), "queue reset");
            FrameArgs a{};
            a.twiddles = k->tw.p;
            a.t_over_2pi = reinterpret_cast<const double*>(d + p.top);
            a.inter = k->inter.p;
            a.table = reinterpret_cast<const OceanSlot*>(d + p.slots);
            a.ocean_base = 0;
            a.chunk = count;
            if (one_launch) {
                MixedGroup& g = m.g[m.groups++];
                g.a = a;
                g.rows_done = k->queue + 1;
                g.cols_done = k->queue + 1 + p.count;
                g.count = count;
                g.slots = std::min(count, 3);
                g.log_n = k->log_n;
                continue;
            }
            QueueArgs q;
            q.ticket = k->queue;
            q.rows_done = k->queue + 1;
            q.cols_done = k->queue + 1 + p.count;
            q.error = error_.p;
            q.count = count;
            q.slots = std::min(count, 3);
            q.wait_ns = 1000000000ull;
            q.defer = k->nf == 6 ? 1 : 0;
            const int grid = static_cast<int>(std::min<uint64_t>(k->grid, uint64_t(count) * k->n));
            check(launch_frame(k->log_n, k->nf, desc_.fft_form, false, a, q, grid, stream_), "frame kernel");
            ++kernels;
        }
        if (one_launch) {
            // Largest sizes first, so the short tasks fill the wave's tail.
            std::sort(m.g, m.g + m.groups, [](const MixedGroup& x, const MixedGroup& y) { return x.log_n > y.log_n; });
            uint32_t first = 0;
            for (int i = 0; i < m.groups; ++i) {
                m.g[i].first = first;
                first += mixed_tasks(m.g[i].log_n, m.g[i].count);
            }
            m.total = first;
            m.ticket = mix_ticket_.p;
            m.error = error_.p;
            m.wait_ns = 1000000000ull;
            const int nf = oparts[0].k->nf;
            m.defer = nf == 6 ? 1 : 0;
            const int ar = arith_of_form(desc_.fft_form);
            int& grid = mix_grid_[nf == 6 ? 1 : 0];
            if (grid == 0) {
                const int per_sm = mixed_blocks_per_sm(nf, ar);
                if (per_sm <= 0) throw DeviceError(cudaErrorInvalidConfiguration, "mixed frame occupancy");
                grid = per_sm * sms_;
            }
            check(cudaMemsetAsync(mix_ticket_.p, 0, sizeof(unsigned), stream_), "ticket reset");
            check(launch_mixed_frame(nf, ar, m, static_cast<int>(std::min<uint64_t>(grid, first)), stream_),
                  "mixed frame kernel");
            ++kernels;
        }
        const IWaveSource* dev_src = reinterpret_cast<const IWaveSource*>(d + src_off);
        if (!plan.sources.empty()) {
            check(launch_source_mean(const_cast<IWaveSource*>(dev_src), static_cast<int>(plan.sources.size()), stream_),
                  "source mean");
            ++kernels;
        }
        for (const FieldPart& fp : fparts) {
            const IWaveSetup& g = fp.k->setup;
            for (const StepPart& sp : fp.steps) {
                const IWaveField* fl = reinterpret_cast<const IWaveField*>(d + sp.fields);
                if (sp.any_sources) {
                    check(launch_source_apply_batch(fl, reinterpret_cast<const int2*>(d + sp.ranges), dev_src,
                                                    static_cast<int>(sp.count), static_cast<int>(g.n), stream_),
                          "sources");
                    ++kernels;
                }
                check(launch_iwave_step(static_cast<int>(g.p), fl, static_cast<int>(sp.count), static_cast<int>(g.n),
                                        g.taps, stream_), "iwave step");
                ++kernels;
            }
            check(launch_iwave_finalize(reinterpret_cast<const IWaveField*>(d + fp.fin), static_cast<int>(fp.fin_count),
                                        static_cast<int>(g.n), stream_), "finalize");
            ++kernels;
        }
        if (!plan.queries.empty()) {
            check(launch_serve_queries(reinterpret_cast<const QueryJob*>(d + jobs_off),
                                       static_cast<int>(plan.queries.size()), max_points, stream_), "queries");
            ++kernels;
        }
        if (plan.points > 0)
            check(cudaMemcpyAsync(c->host_out.p, dev_heights, plan.points * sizeof(float), cudaMemcpyDeviceToHost,
                                  stream_), "heights");
        check(cudaMemcpyAsync(c->host_out.p + plan.points, error_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_),
              "error word");
        check(cudaMemsetAsync(error_.p, 0, sizeof(unsigned), stream_), "error word");
        check(cudaEventRecord(c->done, stream_), "event");
        // Closed sessions: their memory is released behind this batch.
        for (Session* s : c->closes) {
            if (s->block) check(cudaFreeAsync(s->block, stream_), "free session");
            s->block = nullptr;
        }
        check(cudaLaunchHostFunc(stream_, &Server::on_done, c), "host callback");
        c->points = plan.points;
        c->kernels = kernels;
    }

    static void CUDART_CB on_done(void* p)
    {
        BatchCtx* c = static_cast<BatchCtx*>(p);
        Server* s = static_cast<Server*>(c->server);
        {
            std::lock_guard<std::mutex> lk(s->mu_);
            c->complete = true;
        }
        s->cv_.notify_all();
    }

    // Outside the lock: results to the callers' buffers.
    void finish(BatchCtx* c)
    {
        unsigned err = 0;
        std::memcpy(&err, c->host_out.p + c->points, sizeof(unsigned));
        c->failed = c->failed || err != 0;
        if (!c->failed)
            for (Request* r : c->requests)
                if (r->kind == Kind::Query && r->out)
                    std::memcpy(r->out, c->host_out.p + r->out_offset, r->xz.size() * sizeof(float));
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, c->start, c->done) == cudaSuccess) c->gpu_ms = ms;
    }

    void complete_locked(BatchCtx* c)
    {
        const auto now = Clock::now();
        gpu_ms_ += c->gpu_ms;
        for (Request* r : c->requests) {
            if (r->ticket == 0) {  // a session's internal t = 0 frame
                r->session->init.reset();
                continue;
            }
            const double lat = ms_between(r->submitted, now);
            if (c->failed) {
                failed_.insert(r->ticket);
                ++failed_count_;
            } else if (r->kind == Kind::Update) {
                lat_update_.push_back(lat);
                samples_.push_back({ms_between(stats_t0_, r->submitted), lat, 0});
                ++updates_done_;
            } else if (r->kind == Kind::Query) {
                lat_query_.push_back(lat);
                samples_.push_back({ms_between(stats_t0_, r->submitted), lat, 1});
                ++queries_done_;
                points_done_ += r->xz.size();
            }
            ++completed_;
            pending_.erase(r->ticket);  // frees the request
        }
        for (Session* s : c->closes) {
            s->state = OCEAN_SESSION_CLOSED;
            in_use_ -= s->bytes;
        }
        c->requests.clear();
        c->closes.clear();
        c->complete = false;
        c->failed = false;
        c->gpu_ms = 0.0f;
    }

    void fail_locked(BatchCtx* c)
    {
        c->failed = true;
        complete_locked(c);
    }

    // ---- the dispatcher -------------------------------------------------------
    void run()
    {
        cudaSetDevice(device_);  // the dispatcher issues every launch on the server's device
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            // 1. Completed batches, in launch order.
            while (!inflight_.empty() && inflight_.front()->complete) {
                BatchCtx* c = inflight_.front();
                inflight_.pop_front();
                lk.unlock();
                const auto t_finish = Clock::now();
                finish(c);
                const double host_ms = ms_between(t_finish, Clock::now());
                lk.lock();
                dispatch_max_ms_ = std::max(dispatch_max_ms_, host_ms);
                complete_locked(c);
                free_ctx_.push_back(c);
                done_cv_.notify_all();
            }
            // 2. Admissions.
            std::vector<Session*> admits = pick_admissions_locked();
            if (!admits.empty()) {
                lk.unlock();
                std::vector<bool> ok(admits.size(), true);
                for (size_t i = 0; i < admits.size(); ++i) {
                    try {
                        admit(admits[i]);
                    } catch (const std::exception&) {
                        ok[i] = false;
                    }
                }
                lk.lock();
                for (size_t i = 0; i < admits.size(); ++i) {
                    Session* s = admits[i];
                    if (!ok[i]) {
                        in_use_ -= s->bytes;
                        s->state = OCEAN_SESSION_CLOSED;
                        fail_queue_locked(s);
                        continue;
                    }
                    s->state = OCEAN_SESSION_ACTIVE;
                    if (!s->queue.empty() && !s->in_ready) {
                        s->in_ready = true;
                        ready_.push_back(s);
                    }
                }
                done_cv_.notify_all();
            }
            // 3. A new batch.
            if (!free_ctx_.empty() && !ready_.empty()) {
                BatchCtx* c = free_ctx_.front();
                Plan plan;
                if (build_locked(c, plan)) {
                    free_ctx_.pop_front();
                    lk.unlock();
                    bool launched = true;
                    const auto t_launch = Clock::now();
                    try {
                        launch(c, plan);
                    } catch (const std::exception&) {
                        launched = false;
                    }
                    const double host_ms = ms_between(t_launch, Clock::now());
                    lk.lock();
                    dispatch_max_ms_ = std::max(dispatch_max_ms_, host_ms);
                    if (launched) {
                        ++batches_;
                        kernels_ += c->kernels;
                        batched_requests_ += c->requests.size();
                        inflight_.push_back(c);
                    } else {
                        fail_locked(c);
                        free_ctx_.push_back(c);
                        done_cv_.notify_all();
                    }
                    continue;
                }
            }
            if (stop_ && inflight_.empty() && ready_.empty()) {
                if (!can_admit_locked()) break;  // nothing left to free for those waiting
            }
            cv_.wait_for(lk, std::chrono::milliseconds(50), [&] {
                if (!inflight_.empty() && inflight_.front()->complete) return true;
                if (!free_ctx_.empty() && !ready_.empty()) return true;
                if (can_admit_locked()) return true;
                return stop_;
            });
        }
        // Sessions never admitted: their requests fail.
        for (Session* s : waiting_) {
            s->state = OCEAN_SESSION_CLOSED;
            fail_queue_locked(s);
        }
        waiting_.clear();
        done_cv_.notify_all();
    }

    bool can_admit_locked() const
    {
        return !waiting_.empty() && in_use_ + admission_cost_locked(waiting_.front()) <= desc_.hbm_budget;
    }

    void fail_queue_locked(Session* s)
    {
        for (Request* r : s->queue) {
            if (r->ticket == 0) continue;
            failed_.insert(r->ticket);
            ++failed_count_;
            ++completed_;
            pending_.erase(r->ticket);
        }
        s->queue.clear();
    }

    ocean_server_desc desc_;
    int device_ = 0, sms_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaMemPool_t pool_ = nullptr;
    DevBuf<unsigned> error_;
    DevBuf<unsigned> mix_ticket_;  // the one-launch frame's ticket
    int mix_grid_[2] = {0, 0};     // its resident grid, by field count (4, 6)
    std::vector<std::unique_ptr<BatchCtx>> ctxs_;
    std::deque<BatchCtx*> free_ctx_, inflight_;
    std::vector<std::unique_ptr<OceanKind>> ocean_kinds_;
    std::vector<std::unique_ptr<FieldKind>> field_kinds_;

    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::thread thread_;
    bool stop_ = false;
    std::unordered_map<uint64_t, std::unique_ptr<Session>> sessions_;
    std::deque<Session*> waiting_, ready_;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> pending_;
    std::unordered_set<uint64_t> failed_;
    std::unordered_set<uint64_t> ocean_kind_keys_;  // ocean kinds whose tables are in the budget
    uint64_t next_session_ = 1, next_ticket_ = 1;
    size_t in_use_ = 0;        // sessions and their shared tables (the budgeted bytes)
    size_t staging_bytes_ = 0; // per-batch device staging
    uint64_t staging_growths_ = 0;
    double dispatch_max_ms_ = 0.0;  // longest host step of the dispatcher (launch or finish)
    // statistics
    uint64_t submitted_ = 0, completed_ = 0, failed_count_ = 0;
    uint64_t updates_done_ = 0, queries_done_ = 0, points_done_ = 0;
    uint64_t batches_ = 0, kernels_ = 0, batched_requests_ = 0;
    double gpu_ms_ = 0.0;
    std::vector<double> lat_update_, lat_query_;
    struct Sample {
        double submit_ms, latency_ms;
        int32_t kind;
    };
    std::vector<Sample> samples_;
    Clock::time_point stats_t0_;
};

}  // namespace ocean_b200

struct ocean_server {
    ocean_b200::Server impl;
    explicit ocean_server(const ocean_server_desc& d) : impl(d) {}
};

using ocean_b200::guarded;

extern "C" {

void ocean_server_desc_init(ocean_server_desc* desc)
{
    if (desc != nullptr) ocean_b200::server_desc_defaults(desc);
}

ocean_server* ocean_server_create(const ocean_server_desc* desc, ocean_status* out_status)
{
    ocean_server* s = nullptr;
    ocean_status st = OCEAN_OK;
    ocean_server_desc d;
    ocean_b200::server_desc_defaults(&d);
    if (desc == nullptr || desc->struct_size == 0 || desc->struct_size > sizeof(ocean_server_desc)) {
        st = OCEAN_ERROR_INVALID_ARG;
    } else {
        std::memcpy(&d, desc, desc->struct_size);
        d.struct_size = sizeof(ocean_server_desc);
        st = guarded([&] { s = new ocean_server(d); });
    }
    if (out_status != nullptr) *out_status = st;
    return st == OCEAN_OK ? s : nullptr;
}

void ocean_server_destroy(ocean_server* server) { delete server; }

uint64_t ocean_server_session_bytes(const ocean_desc* ocean, const ocean_interaction_desc* field)
{
    ocean_desc od;
    if (!ocean_b200::copy_desc(ocean, od)) return 0;
    ocean_interaction_desc fd;
    if (field != nullptr && !ocean_b200::copy_interaction_desc(field, fd)) return 0;
    return ocean_b200::Server::session_bytes(od, field ? &fd : nullptr);
}

ocean_status ocean_server_open_session(ocean_server* server, const ocean_desc* ocean,
                                       const ocean_interaction_desc* field, uint64_t* out_session)
{
    if (server == nullptr || out_session == nullptr) return OCEAN_ERROR_INVALID_ARG;
    ocean_desc od;
    if (!ocean_b200::copy_desc(ocean, od)) return OCEAN_ERROR_INVALID_ARG;
    ocean_interaction_desc fd;
    if (field != nullptr && !ocean_b200::copy_interaction_desc(field, fd)) return OCEAN_ERROR_INVALID_ARG;
    try {
        *out_session = server->impl.open(od, field ? &fd : nullptr);
        return OCEAN_OK;
    } catch (const std::length_error&) {
        return OCEAN_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return guarded([] { throw; });
    }
}

ocean_status ocean_server_close_session(ocean_server* server, uint64_t session)
{
    if (server == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] {
        auto r = std::make_unique<ocean_b200::Request>();
        r->kind = ocean_b200::Kind::Close;
        server->impl.submit(session, std::move(r));
    });
}

ocean_session_state ocean_server_session_state(ocean_server* server, uint64_t session)
{
    if (server == nullptr) return OCEAN_SESSION_CLOSED;
    return server->impl.state(session);
}

ocean_status ocean_server_submit_update(ocean_server* server, uint64_t session, double time, float dt,
                                        const ocean_disturbance* sources, uint32_t count, uint64_t* out_ticket)
{
    if (server == nullptr || (count > 0 && sources == nullptr)) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] {
        auto r = std::make_unique<ocean_b200::Request>();
        r->kind = ocean_b200::Kind::Update;
        r->time = time;
        r->dt = dt;
        r->sources.assign(sources, sources + count);
        const uint64_t t = server->impl.submit(session, std::move(r));
        if (out_ticket) *out_ticket = t;
    });
}

ocean_status ocean_server_submit_query(ocean_server* server, uint64_t session, const float* xz, uint32_t count,
                                       float* heights, uint64_t* out_ticket)
{
    if (server == nullptr || (count > 0 && (xz == nullptr || heights == nullptr))) return OCEAN_ERROR_INVALID_ARG;
    if (count > server->impl.desc().max_query_points || count > server->impl.desc().max_batch_points)
        return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] {
        auto r = std::make_unique<ocean_b200::Request>();
        r->kind = ocean_b200::Kind::Query;
        r->xz.resize(count);
        std::memcpy(r->xz.data(), xz, static_cast<size_t>(count) * sizeof(float2));
        r->out = heights;
        const uint64_t t = server->impl.submit(session, std::move(r));
        if (out_ticket) *out_ticket = t;
    });
}

ocean_status ocean_server_wait(ocean_server* server, uint64_t ticket, uint32_t timeout_ms)
{
    if (server == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return server->impl.wait(ticket, timeout_ms);
}

ocean_status ocean_server_drain(ocean_server* server, uint32_t timeout_ms)
{
    if (server == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return server->impl.drain(timeout_ms);
}

ocean_status ocean_server_read_session(ocean_server* server, uint64_t session, float* displacement, float* normal,
                                       float* field)
{
    if (server == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] { server->impl.read_session(session, displacement, normal, field); });
}

ocean_status ocean_server_get_stats(ocean_server* server, ocean_server_stats* out)
{
    if (server == nullptr || out == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] { server->impl.stats(out); });
}

uint64_t ocean_server_latency_samples(ocean_server* server, double* submit_ms, double* latency_ms, int32_t* kind,
                                      uint64_t capacity)
{
    if (server == nullptr) return 0;
    return server->impl.samples(submit_ms, latency_ms, kind, capacity);
}

ocean_status ocean_server_reset_stats(ocean_server* server)
{
    if (server == nullptr) return OCEAN_ERROR_INVALID_ARG;
    server->impl.reset_stats();
    return OCEAN_OK;
}

}  // extern "C"
