// oceanlib-b200: iWave interaction field - host layer and C ABI.
//
// The reference's InteractionField (src/interaction.cpp) with its state on the
// GPU. Host-side work is what the reference does once, not per substep: the
// stencil fit, the damping tables, the obstruction BFS (per set_obstruction),
// and resolving each queued disturbance to grid units (a few floats per
// source per substep). Sources, obstruction, the stencil step and finalize
// run as device kernels (csrc/iwave.cu).

#include "../../include/ocean_b200.h"
#include "host_util.h"
#include "iwave.h"
#include "iwave_host.h"
#include "iwave_stencil.h"
#include "spectrum.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace ocean_b200 {

class Interaction {
public:
    explicit Interaction(const ocean_interaction_desc& d) : desc_(d), setup_(iwave_setup(d))
    {
        n_ = setup_.n;
        p_ = setup_.p;
        cell_ = setup_.cell;
        cells_ = setup_.cells;
        stride_ = setup_.stride;
        rows_ = setup_.rows;
        dt_limit_ = setup_.dt_limit;
        dt_ = setup_.dt;

        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        const size_t plane = static_cast<size_t>(rows_) * stride_;
        for (auto& b : planes_) {
            b = DevBuf<float>(plane);
            check(cudaMemsetAsync(b.p, 0, plane * sizeof(float), stream_), "memset");
        }
        cur_ = 0;
        old_ = 1;
        c1_ = DevBuf<float>(cells_);
        c2_ = DevBuf<float>(cells_);
        out_ = DevBuf<float4>(cells_);
        out_host_ = HostBuf<float>(cells_ * 4);
        fields_ = DevBuf<IWaveField>(4);
        sources_dev_ = DevBuf<IWaveSource>(static_cast<size_t>(d.max_sources) * d.max_substeps);
        sources_host_ = HostBuf<IWaveSource>(static_cast<size_t>(d.max_sources) * d.max_substeps);
        queue_.reset(d.max_sources);
        solid_dev_ = DevBuf<uint32_t>(cells_);
        nearest_dev_ = DevBuf<uint32_t>(cells_);
        mask_dev_ = DevBuf<uint8_t>(cells_);
        mask_.assign(cells_, 0);
        const std::vector<float>& taps = setup_.stencil.taps;
        taps_dev_ = DevBuf<float>(taps.size());
        check(cudaMemcpyAsync(taps_dev_.p, taps.data(), taps.size() * sizeof(float),
                              cudaMemcpyHostToDevice, stream_), "taps");
        build_damping();
        upload_fields();
        q_in_ = DevBuf<float2>(1);
        q_out_ = DevBuf<float4>(1);
        q_host_in_ = HostBuf<float2>(1);
        q_host_out_ = HostBuf<float4>(1);
        finalize();  // a valid all-zero output (src/interaction.cpp:497)
        refresh_host();
    }

    ~Interaction()
    {
        if (stream_) {
            cudaStreamSynchronize(stream_);
            cudaStreamDestroy(stream_);
        }
    }

    void add(const ocean_disturbance& d) { queue_.add(d); }

    // InteractionField::update (src/interaction.cpp:531-587).
    void update(float dt)
    {
        moved_ = false;
        const uint32_t steps = clock_.advance(dt, dt_, desc_.max_substeps);
        if (steps == 0) {
            queue_.keep_impulses();
            return;
        }
        // Resolve every substep's sources first (one upload), then run.
        std::vector<uint32_t>& first = first_;
        resolved_.clear();
        queue_.resolve_all(steps, setup_, origin_x_, origin_z_, resolved_, first);
        const uint32_t total = first[steps];
        std::copy(resolved_.begin(), resolved_.end(), sources_host_.p);
        if (total > 0)
            check(cudaMemcpyAsync(sources_dev_.p, sources_host_.p, total * sizeof(IWaveSource),
                                  cudaMemcpyHostToDevice, stream_), "sources");
        for (uint32_t s = 0; s < steps; ++s) {
            const int count = static_cast<int>(first[s + 1] - first[s]);
            if (count > 0) {
                check(launch_source_mean(sources_dev_.p + first[s], count, stream_), "source mean");
                check(launch_source_apply(field(), sources_dev_.p + first[s], count, stream_), "sources");
            }
            substep();
        }
        finalize();
        refresh_host();
    }

    // InteractionField::recenter (src/interaction.cpp:601-705).
    bool recenter(float world_x, float world_z)
    {
        const float half = 0.5f * desc_.extent;
        const int32_t tx = static_cast<int32_t>(std::lround((world_x - half) / cell_));
        const int32_t tz = static_cast<int32_t>(std::lround((world_z - half) / cell_));
        const int32_t dx = tx - origin_x_;
        const int32_t dz = tz - origin_z_;
        shift_x_ = dx;
        shift_z_ = dz;
        if (dx == 0 && dz == 0) {
            moved_ = false;
            return false;
        }
        moved_ = true;
        origin_x_ = tx;
        origin_z_ = tz;
        const int32_t n = static_cast<int32_t>(n_);
        if (std::abs(dx) >= n || std::abs(dz) >= n) {
            const size_t plane = static_cast<size_t>(rows_) * stride_;
            for (auto& b : planes_) check(cudaMemsetAsync(b.p, 0, plane * sizeof(float), stream_), "memset");
            std::fill(mask_.begin(), mask_.end(), 0);
        } else {
            // Both levels move together, out of place into the spare planes.
            int spare[2], k = 0;
            for (int b = 0; b < 4 && k < 2; ++b)
                if (b != cur_ && b != old_) spare[k++] = b;
            check(launch_shift(interior(cur_), interior(spare[0]), n, stride_, dx, dz, stream_), "shift");
            check(launch_shift(interior(old_), interior(spare[1]), n, stride_, dx, dz, stream_), "shift");
            cur_ = spare[0];
            old_ = spare[1];
            if (has_mask_) {
                std::vector<uint8_t> moved(cells_, 0);
                for (int32_t z = 0; z < n; ++z)
                    for (int32_t x = 0; x < n; ++x) {
                        const int32_t sx = x + dx, sz = z + dz;
                        if (sx >= 0 && sx < n && sz >= 0 && sz < n)
                            moved[static_cast<size_t>(z) * n + x] = mask_[static_cast<size_t>(sz) * n + sx];
                    }
                mask_.swap(moved);
            }
        }
        rebuild_mask_tables();
        upload_fields();
        finalize();
        refresh_host();
        return true;
    }

    // InteractionField::set_obstruction (src/interaction.cpp:709-723).
    void set_obstruction(const uint8_t* m)
    {
        if (m == nullptr) {
            std::fill(mask_.begin(), mask_.end(), 0);
            has_mask_ = false;
            solid_count_ = 0;
            return;
        }
        std::memcpy(mask_.data(), m, cells_);
        has_mask_ = true;
        rebuild_mask_tables();
    }

    // The tables as the device holds them (host arrays of cells entries).
    void read_tables(uint32_t* solid, uint32_t* nearest, uint32_t* count)
    {
        *count = has_mask_ ? solid_count_ : 0;
        if (has_mask_ && solid != nullptr && solid_count_ > 0)
            check(cudaMemcpyAsync(solid, solid_dev_.p, solid_count_ * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  stream_), "tables");
        if (has_mask_ && nearest != nullptr)
            check(cudaMemcpyAsync(nearest, nearest_dev_.p, cells_ * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  stream_), "tables");
        check(cudaStreamSynchronize(stream_), "tables");
    }

    void sample(float x, float z, ocean_interaction_sample* out)
    {
        std::lock_guard<std::mutex> lock(query_mutex_);
        q_host_in_.p[0] = make_float2(x, z);
        check(cudaMemcpyAsync(q_in_.p, q_host_in_.p, sizeof(float2), cudaMemcpyHostToDevice, stream_), "query");
        check(launch_interaction_sample(out_.p, static_cast<int>(n_), cell_, origin_wx(), origin_wz(), q_in_.p, 1,
                                        q_out_.p, stream_), "query kernel");
        check(cudaMemcpyAsync(q_host_out_.p, q_out_.p, sizeof(float4), cudaMemcpyDeviceToHost, stream_), "query");
        check(cudaStreamSynchronize(stream_), "query");
        std::memcpy(out, q_host_out_.p, sizeof(float4));
    }

    // Device-resident queries (xz, res on the device), on the field's stream.
    void sample_device(const float2* xz, uint64_t count, float4* res)
    {
        check(launch_interaction_sample(out_.p, static_cast<int>(n_), cell_, origin_wx(), origin_wz(), xz,
                                        count, res, stream_), "query kernel");
    }

    double energy()
    {
        DevBuf<double> kin(n_), pot(n_);
        check(launch_energy_rows(field(), taps_dev_.p, static_cast<int>(p_), kin.p, pot.p, stream_), "energy");
        std::vector<double> hk(n_), hp(n_);
        check(cudaMemcpyAsync(hk.data(), kin.p, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "energy");
        check(cudaMemcpyAsync(hp.data(), pot.p, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "energy");
        check(cudaStreamSynchronize(stream_), "energy");
        double k = 0.0, pt = 0.0;
        for (uint32_t i = 0; i < n_; ++i) {
            k += hk[i];
            pt += hp[i];
        }
        return 0.5 * (k + static_cast<double>(desc_.gravity) * pt);
    }

    void get_state(float* cur, float* old)
    {
        copy_plane_out(cur_, cur);
        copy_plane_out(old_, old);
        check(cudaStreamSynchronize(stream_), "state");
    }

    void set_state(const float* cur, const float* old)
    {
        copy_plane_in(cur_, cur);
        copy_plane_in(old_, old);
        finalize();
        refresh_host();
    }

    const float* host_field() const { return out_host_.p; }
    const float4* device_field() const { return out_.p; }
    cudaStream_t stream() const { return stream_; }
    uint32_t size() const { return n_; }
    float cell() const { return cell_; }
    const ocean_interaction_desc& desc() const { return desc_; }
    float origin_wx() const { return static_cast<float>(origin_x_) * cell_; }
    float origin_wz() const { return static_cast<float>(origin_z_) * cell_; }
    float fixed_dt() const { return dt_; }
    float dt_limit() const { return dt_limit_; }
    float dispersion_error() const { return static_cast<float>(setup_.stencil.peak_relative_error); }
    uint64_t dropped() const { return queue_.dropped; }
    uint32_t last_substeps() const { return clock_.last_steps; }
    bool last_clamped() const { return clock_.clamped; }
    bool moved() const { return moved_; }
    int32_t shift_x() const { return shift_x_; }
    int32_t shift_z() const { return shift_z_; }
    const std::vector<float>& taps() const { return setup_.stencil.taps; }

private:
    float* interior(int b) const { return planes_[b].p + static_cast<size_t>(p_) * stride_ + p_; }

    IWaveField field() const
    {
        IWaveField f;
        f.cur = interior(cur_);
        f.old = interior(old_);
        f.c1 = c1_.p;
        f.c2 = c2_.p;
        f.out = out_.p;
        f.n = static_cast<int32_t>(n_);
        f.stride = stride_;
        f.gdt2 = desc_.gravity * dt_ * dt_;
        f.inv_two_cell = 0.5f / cell_;
        f.inv_dt = 1.0f / dt_;
        f.inv_dt_d = 1.0 / static_cast<double>(dt_);
        return f;
    }

    // Device copies of the field descriptor for both (cur, old) orders, so a
    // substep only picks one (no upload per substep).
    void upload_fields()
    {
        IWaveField fs[2];
        fs[0] = field();
        fs[1] = fs[0];
        std::swap(fs[1].cur, fs[1].old);
        check(cudaMemcpyAsync(fields_.p, fs, sizeof(fs), cudaMemcpyHostToDevice, stream_), "fields");
        check(cudaStreamSynchronize(stream_), "fields");
        which_ = 0;
    }

    void substep()
    {
        if (has_mask_ && solid_count_ > 0)
            check(launch_obstruction(field(), solid_dev_.p, nearest_dev_.p, solid_count_,
                                     desc_.obstruction == OCEAN_OBSTRUCTION_DIRICHLET, stream_), "obstruction");
        check(launch_iwave_step(static_cast<int>(p_), fields_.p + which_, 1, static_cast<int>(n_), setup_.taps, stream_),
              "iwave step");
        std::swap(cur_, old_);
        which_ ^= 1;
    }

    void finalize()
    {
        const IWaveField f = field();
        check(cudaMemcpyAsync(fields_.p + 2, &f, sizeof(f), cudaMemcpyHostToDevice, stream_), "fields");
        check(launch_iwave_finalize(fields_.p + 2, 1, static_cast<int>(n_), stream_), "finalize");
        check(cudaStreamSynchronize(stream_), "finalize");
    }

    void refresh_host()
    {
        check(cudaMemcpyAsync(out_host_.p, out_.p, cells_ * sizeof(float4), cudaMemcpyDeviceToHost, stream_),
              "mirror");
        check(cudaStreamSynchronize(stream_), "mirror");
    }

    // The absorbing sponge (src/interaction.cpp:212-241), float arithmetic
    // as the reference.
    void build_damping()
    {
        std::vector<float> c1, c2;
        iwave_damping(desc_, setup_, c1, c2);
        check(cudaMemcpyAsync(c1_.p, c1.data(), cells_ * sizeof(float), cudaMemcpyHostToDevice, stream_), "damping");
        check(cudaMemcpyAsync(c2_.p, c2.data(), cells_ * sizeof(float), cudaMemcpyHostToDevice, stream_), "damping");
        check(cudaStreamSynchronize(stream_), "damping");
    }

    // The obstruction tables (src/interaction.cpp:255-292), built on the
    // device from the mask by a level-synchronous BFS that reproduces the
    // reference's queue order (obstruction.cu).
    void rebuild_mask_tables()
    {
        solid_count_ = 0;
        if (!has_mask_) return;
        check(cudaMemcpyAsync(mask_dev_.p, mask_.data(), cells_, cudaMemcpyHostToDevice, stream_), "mask");
        uint32_t count = 0;
        check(build_obstruction_tables(mask_dev_.p, static_cast<int>(n_), solid_dev_.p, nearest_dev_.p, &count,
                                       stream_),
              "obstruction tables");
        solid_count_ = count;
    }

    void copy_plane_out(int b, float* dst)
    {
        check(cudaMemcpy2DAsync(dst, n_ * sizeof(float), interior(b), stride_ * sizeof(float), n_ * sizeof(float),
                                n_, cudaMemcpyDeviceToHost, stream_), "state");
    }

    void copy_plane_in(int b, const float* src)
    {
        check(cudaMemcpy2DAsync(interior(b), stride_ * sizeof(float), src, n_ * sizeof(float), n_ * sizeof(float),
                                n_, cudaMemcpyHostToDevice, stream_), "state");
        check(cudaStreamSynchronize(stream_), "state");
    }

    ocean_interaction_desc desc_;
    IWaveSetup setup_;
    uint32_t n_ = 0, p_ = 0, rows_ = 0;
    int stride_ = 0;
    size_t cells_ = 0;
    float cell_ = 0.0f, dt_ = 0.0f, dt_limit_ = 0.0f;
    cudaStream_t stream_ = nullptr;
    DevBuf<float> planes_[4];
    int cur_ = 0, old_ = 1, which_ = 0;
    DevBuf<float> c1_, c2_, taps_dev_;
    DevBuf<float4> out_;
    HostBuf<float> out_host_;
    DevBuf<IWaveField> fields_;
    DevBuf<IWaveSource> sources_dev_;
    HostBuf<IWaveSource> sources_host_;
    IWaveQueue queue_;
    IWaveClock clock_;
    std::vector<IWaveSource> resolved_;
    std::vector<uint32_t> first_;
    int32_t origin_x_ = 0, origin_z_ = 0, shift_x_ = 0, shift_z_ = 0;
    bool moved_ = false;
    std::vector<uint8_t> mask_;
    bool has_mask_ = false;
    uint32_t solid_count_ = 0;
    DevBuf<uint32_t> solid_dev_, nearest_dev_;
    DevBuf<uint8_t> mask_dev_;
    std::mutex query_mutex_;
    DevBuf<float2> q_in_;
    DevBuf<float4> q_out_;
    HostBuf<float2> q_host_in_;
    HostBuf<float4> q_host_out_;
};

}  // namespace ocean_b200

struct ocean_interaction {
    ocean_b200::Interaction impl;
    explicit ocean_interaction(const ocean_interaction_desc& d) : impl(d) {}
};

using ocean_b200::guarded;

extern "C" {

void ocean_interaction_desc_init(ocean_interaction_desc* desc)
{
    if (desc != nullptr) ocean_b200::interaction_desc_defaults(desc);
}

ocean_interaction* ocean_interaction_create(const ocean_interaction_desc* desc, ocean_status* out_status)
{
    ocean_interaction* f = nullptr;
    ocean_interaction_desc resolved;
    ocean_status st = OCEAN_OK;
    if (!ocean_b200::copy_interaction_desc(desc, resolved)) {
        st = OCEAN_ERROR_INVALID_ARG;
    } else {
        st = guarded([&] { f = new ocean_interaction(resolved); });
    }
    if (out_status != nullptr) *out_status = st;
    return st == OCEAN_OK ? f : nullptr;
}

void ocean_interaction_destroy(ocean_interaction* field) { delete field; }

void ocean_interaction_add(ocean_interaction* field, const ocean_disturbance* d)
{
    if (field == nullptr || d == nullptr) return;
    field->impl.add(*d);
}

uint64_t ocean_interaction_dropped(const ocean_interaction* field)
{
    return field == nullptr ? 0u : field->impl.dropped();
}

void ocean_interaction_update(ocean_interaction* field, float dt)
{
    if (field == nullptr) return;
    guarded([&] { field->impl.update(dt); });
}

int32_t ocean_interaction_recenter(ocean_interaction* field, float world_x, float world_z)
{
    if (field == nullptr) return 0;
    bool moved = false;
    guarded([&] { moved = field->impl.recenter(world_x, world_z); });
    return moved ? 1 : 0;
}

void ocean_interaction_last_shift(const ocean_interaction* field, int32_t* dx, int32_t* dz)
{
    // InteractionField::recentered / last_shift_x / last_shift_z
    // (src/interaction.cpp:707-709): zero for a NULL handle.
    if (dx != nullptr) *dx = field == nullptr ? 0 : field->impl.shift_x();
    if (dz != nullptr) *dz = field == nullptr ? 0 : field->impl.shift_z();
}

ocean_status ocean_interaction_obstruction_tables(const ocean_interaction* field, uint32_t* solid,
                                                  uint32_t* nearest, uint32_t* solid_count)
{
    if (field == nullptr || solid_count == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] { const_cast<ocean_interaction*>(field)->impl.read_tables(solid, nearest, solid_count); });
}

void ocean_interaction_set_obstruction(ocean_interaction* field, const uint8_t* mask)
{
    if (field == nullptr) return;
    guarded([&] { field->impl.set_obstruction(mask); });
}

ocean_interaction_buffers ocean_interaction_get_buffers(const ocean_interaction* field)
{
    ocean_interaction_buffers b;
    std::memset(&b, 0, sizeof(b));
    if (field == nullptr) return b;
    b.field = field->impl.host_field();
    b.size = field->impl.size();
    b.extent = field->impl.desc().extent;
    b.origin_x = field->impl.origin_wx();
    b.origin_z = field->impl.origin_wz();
    return b;
}

void ocean_interaction_sample_at(const ocean_interaction* field, float world_x, float world_z,
                                 ocean_interaction_sample* out)
{
    if (out == nullptr) return;
    std::memset(out, 0, sizeof(*out));
    if (field == nullptr) return;
    ocean_interaction_sample s{};
    if (guarded([&] { const_cast<ocean_interaction*>(field)->impl.sample(world_x, world_z, &s); }) == OCEAN_OK)
        *out = s;
}

float ocean_interaction_height_at(const ocean_interaction* field, float world_x, float world_z)
{
    ocean_interaction_sample s;
    ocean_interaction_sample_at(field, world_x, world_z, &s);
    return s.height;
}

float ocean_interaction_fixed_dt(const ocean_interaction* field)
{
    return field == nullptr ? 0.0f : field->impl.fixed_dt();
}

float ocean_interaction_dt_limit(const ocean_interaction* field)
{
    return field == nullptr ? 0.0f : field->impl.dt_limit();
}

float ocean_interaction_dispersion_error(const ocean_interaction* field)
{
    return field == nullptr ? 0.0f : field->impl.dispersion_error();
}

const float* ocean_interaction_device_field(const ocean_interaction* field)
{
    return field == nullptr ? nullptr : reinterpret_cast<const float*>(field->impl.device_field());
}

uint32_t ocean_interaction_last_substeps(const ocean_interaction* field)
{
    return field == nullptr ? 0u : field->impl.last_substeps();
}

int32_t ocean_interaction_last_clamped(const ocean_interaction* field)
{
    return (field != nullptr && field->impl.last_clamped()) ? 1 : 0;
}

double ocean_interaction_energy(const ocean_interaction* field)
{
    if (field == nullptr) return 0.0;
    double e = 0.0;
    guarded([&] { e = const_cast<ocean_interaction*>(field)->impl.energy(); });
    return e;
}

ocean_status ocean_interaction_get_state(const ocean_interaction* field, float* cur, float* old)
{
    if (field == nullptr || cur == nullptr || old == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] { const_cast<ocean_interaction*>(field)->impl.get_state(cur, old); });
}

ocean_status ocean_interaction_set_state(ocean_interaction* field, const float* cur, const float* old)
{
    if (field == nullptr || cur == nullptr || old == nullptr) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] { field->impl.set_state(cur, old); });
}

ocean_status ocean_interaction_kernel_taps(const ocean_interaction* field, float* taps)
{
    if (field == nullptr || taps == nullptr) return OCEAN_ERROR_INVALID_ARG;
    const auto& t = field->impl.taps();
    std::memcpy(taps, t.data(), t.size() * sizeof(float));
    return OCEAN_OK;
}

ocean_status ocean_interaction_sample_many(const ocean_interaction* field, const float* xz, uint64_t count,
                                           ocean_interaction_sample* out)
{
    if (field == nullptr || (count > 0 && (xz == nullptr || out == nullptr))) return OCEAN_ERROR_INVALID_ARG;
    if (count == 0) return OCEAN_OK;
    return guarded([&] {
        auto& f = const_cast<ocean_interaction*>(field)->impl;
        ocean_b200::DevBuf<float2> in(count);
        ocean_b200::DevBuf<float4> res(count);
        ocean_b200::check(cudaMemcpyAsync(in.p, xz, count * sizeof(float2), cudaMemcpyHostToDevice, f.stream()),
                          "query");
        f.sample_device(in.p, count, res.p);
        ocean_b200::check(cudaMemcpyAsync(out, res.p, count * sizeof(float4), cudaMemcpyDeviceToHost, f.stream()),
                          "query");
        ocean_b200::check(cudaStreamSynchronize(f.stream()), "query");
    });
}

ocean_status ocean_sample_combined_many(const ocean_sim* sim, const ocean_interaction* field, const float* xz,
                                        uint64_t count, ocean_surface_ex* out)
{
    if (sim == nullptr || field == nullptr || (count > 0 && (xz == nullptr || out == nullptr)))
        return OCEAN_ERROR_INVALID_ARG;
    if (count == 0) return OCEAN_OK;
    ocean_device_buffers db;
    if (ocean_get_device_buffers(sim, &db) != OCEAN_OK) return OCEAN_ERROR_INVALID_ARG;
    return guarded([&] {
        auto& f = const_cast<ocean_interaction*>(field)->impl;
        cudaStream_t st = f.stream();
        ocean_b200::DevBuf<float2> in(count);
        ocean_b200::DevBuf<float4> e(count);
        ocean_b200::DevBuf<ocean_b200::SurfaceEx> s(count);
        ocean_b200::check(cudaMemcpyAsync(in.p, xz, count * sizeof(float2), cudaMemcpyHostToDevice, st), "query");
        // The ocean's frame may still be running on its own stream.
        ocean_b200::check(cudaDeviceSynchronize(), "query");
        const float inv_cell = static_cast<float>(db.size) / db.patch_length;
        ocean_b200::check(ocean_b200::launch_sample(static_cast<int>(db.size), inv_cell,
                                                    reinterpret_cast<const float4*>(db.displacement),
                                                    reinterpret_cast<const float4*>(db.normal),
                                                    reinterpret_cast<const float4*>(db.velocity), in.p, count, s.p,
                                                    st),
                          "ocean query");
        f.sample_device(in.p, count, e.p);
        ocean_b200::check(ocean_b200::launch_combine(s.p, e.p, count, s.p, st), "combine");
        ocean_b200::check(cudaMemcpyAsync(out, s.p, count * sizeof(ocean_b200::SurfaceEx), cudaMemcpyDeviceToHost,
                                          st),
                          "query");
        ocean_b200::check(cudaStreamSynchronize(st), "query");
    });
}

void ocean_sample_combined(const ocean_sim* sim, const ocean_interaction* field, float world_x, float world_z,
                           ocean_surface_ex* out)
{
    // include/ocean/ocean.h:413 (src/c_api.cpp:478-506)
    if (out == nullptr) return;
    if (field == nullptr) {
        ocean_sample_ex(sim, world_x, world_z, out);
        return;
    }
    if (sim == nullptr) {
        std::memset(out, 0, sizeof(*out));
        out->normal_y = 1.0f;
        ocean_interaction_sample e;
        ocean_interaction_sample_at(field, world_x, world_z, &e);
        out->height = e.height;
        out->velocity_y = e.velocity_y;
        return;
    }
    const float xz[2] = {world_x, world_z};
    if (ocean_sample_combined_many(sim, field, xz, 1, out) != OCEAN_OK) {
        std::memset(out, 0, sizeof(*out));
        out->normal_y = 1.0f;
    }
}

}  // extern "C"
