// A C++ program written against the reference's public C++ API
// (include/ocean/ocean.hpp, foam.hpp, cascade.hpp, interaction.hpp) and
// linked against libocean_b200.so: the relink check of the drop-in boundary.
// tests/test_gpu_cxx_api.py builds it, runs it on the GPU and compares the
// arrays it writes with the oracle and with the reference's golden records.
//
//   ocean_api_check OUT_DIR
//
// Inputs read from OUT_DIR: xz.bin (query points, float pairs),
// cascade_xz.bin. Outputs written there: raw float32 arrays and report.txt
// (key = value lines).
#include "ocean/cascade.hpp"
#include "ocean/foam.hpp"
#include "ocean/interaction.hpp"
#include "ocean/ocean.hpp"
#include "ocean/ocean.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

std::string g_dir;
std::ofstream g_report;

std::vector<float> read_floats(const std::string& name)
{
    std::ifstream f(g_dir + "/" + name, std::ios::binary);
    std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<float> v(bytes.size() / sizeof(float));
    std::memcpy(v.data(), bytes.data(), v.size() * sizeof(float));
    return v;
}

void write_floats(const std::string& name, const float* p, size_t count)
{
    std::ofstream f(g_dir + "/" + name, std::ios::binary);
    f.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(count * sizeof(float)));
}

void write_surfaces(const std::string& name, const std::vector<ocean::Surface>& s)
{
    static_assert(sizeof(ocean::Surface) == 10 * sizeof(float), "Surface is 10 floats");
    write_floats(name, reinterpret_cast<const float*>(s.data()), s.size() * 10);
}

template <class T>
void report(const char* key, const T& value)
{
    g_report << key << " = " << value << "\n";
}

// A blocking parallel_for that counts its calls (the reference's hook contract).
unsigned g_dispatches = 0;
void serial_for(void*, ocean::TaskFn task, void* ctx, std::uint32_t count)
{
    ++g_dispatches;
    for (std::uint32_t i = 0; i < count; ++i) task(ctx, i);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    g_dir = argv[1];
    g_report.open(g_dir + "/report.txt");

    // --- Ocean: one frame, buffers, queries ------------------------------
    ocean::OceanDesc d;
    d.size = 64;
    d.patch_length = 80.0f;
    d.spectrum.wind_speed = 14.0f;
    d.spectrum.wind_direction = 0.7f;
    d.choppiness = 1.3f;
    d.seed = 4242;
    d.compute_velocity = true;
    ocean::Ocean oc(d);
    report("time_after_construction", oc.time());
    oc.update(3.25);
    report("time", oc.time());
    const ocean::Buffers b = oc.buffers();
    const size_t cells = size_t(b.size) * b.size;
    write_floats("ocean_disp.bin", b.displacement, cells * 4);
    write_floats("ocean_normal.bin", b.normal, cells * 4);
    write_floats("ocean_vel.bin", b.velocity, cells * 4);
    const std::vector<float> xz = read_floats("xz.bin");
    std::vector<ocean::Surface> q;
    bool height_matches = true;
    for (size_t i = 0; i + 1 < xz.size(); i += 2) {
        q.push_back(oc.sample_at(xz[i], xz[i + 1]));
        height_matches = height_matches && oc.height_at(xz[i], xz[i + 1]) == q.back().height;
    }
    write_surfaces("ocean_queries.bin", q);
    report("height_at_matches_sample_at", height_matches ? 1 : 0);

    // Move keeps the buffers (the handle is the object).
    ocean::Ocean moved(std::move(oc));
    report("move_keeps_buffers", moved.buffers().displacement == b.displacement ? 1 : 0);

    // The C handle behind it answers the C ABI the same way.
    const ocean_buffers cb = ocean_get_buffers(static_cast<const ocean_sim*>(moved.c_handle()));
    report("c_handle_buffers_match", cb.displacement == b.displacement ? 1 : 0);

    // Malformed descriptors throw std::invalid_argument, as the reference does.
    int threw = 0;
    try {
        ocean::OceanDesc bad;
        bad.size = 100;
        ocean::Ocean x(bad);
    } catch (const std::invalid_argument&) {
        threw = 1;
    }
    report("invalid_size_throws", threw);

    // A parallel_for hook is called four times per update.
    ocean::OceanDesc hooked = d;
    hooked.compute_velocity = false;
    hooked.parallel_for = &serial_for;
    ocean::Ocean oh(hooked);
    g_dispatches = 0;
    oh.update(1.0);
    report("hook_dispatches_per_update", g_dispatches);

    // --- FoamField: 30 frames at 60 Hz on the moved ocean -----------------
    {
        ocean::FoamDesc fd;
        ocean::FoamField foam(moved, fd);
        for (int k = 1; k <= 30; ++k) {
            moved.update(k / 60.0);
            foam.update(1.0f / 60.0f);
        }
        write_floats("foam.bin", foam.data(), cells);
        report("foam_size", foam.size());
        report("foam_last_substeps", foam.last_substeps());
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.17g", foam.coverage());
        report("foam_coverage", buf);
        std::vector<float> at;
        for (size_t i = 0; i + 1 < xz.size(); i += 2) at.push_back(foam.foam_at(xz[i], xz[i + 1]));
        write_floats("foam_at.bin", at.data(), at.size());
        ocean::FoamField moved_foam(std::move(foam));
        moved_foam.clear();
        report("foam_cleared_coverage", moved_foam.coverage());
        int refused = 0;
        try {
            ocean::FoamField nf(oh, fd);  // no velocity
        } catch (const std::invalid_argument&) {
            refused = 1;
        }
        report("foam_without_velocity_throws", refused);
    }

    // --- CascadeStack: the reference's three-level case at t = 10 ---------
    {
        std::vector<ocean::CascadeLevel> levels(3);
        const float lengths[3] = {800.0f, 150.0f, 25.0f};
        for (int i = 0; i < 3; ++i) {
            levels[i].size = 256;
            levels[i].patch_length = lengths[i];
            levels[i].spectrum.wind_speed = 15.0f;
            levels[i].spectrum.depth = 30.0f;
            levels[i].seed = static_cast<std::uint64_t>(i + 1);
            levels[i].compute_velocity = true;
        }
        ocean::CascadeStack cs{std::span<const ocean::CascadeLevel>(levels)};
        cs.update(10.0);
        report("cascade_levels", cs.level_count());
        report("cascade_time", cs.time());
        report("cascade_level_time", cs.level(1).time());
        const std::vector<float> cxz = read_floats("cascade_xz.bin");
        std::vector<ocean::Surface> cq;
        for (size_t i = 0; i + 1 < cxz.size(); i += 2) cq.push_back(cs.sample_at(cxz[i], cxz[i + 1]));
        write_surfaces("cascade_queries.bin", cq);
        const ocean::Buffers lb = cs.buffers(2);
        write_floats("cascade_level2_disp.bin", lb.displacement, size_t(lb.size) * lb.size * 4);
        std::vector<ocean::Surface> lq;
        for (size_t i = 0; i + 1 < xz.size(); i += 2) lq.push_back(cs.level(2).sample_at(xz[i], xz[i + 1]));
        write_surfaces("cascade_level2_queries.bin", lq);

        // --- InteractionField and WaterSurface -----------------------------
        ocean::InteractionDesc idesc;
        idesc.size = 64;
        idesc.extent = 16.0f;
        ocean::InteractionField field(idesc);
        ocean::Disturbance dist;
        dist.world_x = 8.0f;
        dist.world_z = 8.0f;
        dist.radius = 0.5f;
        dist.velocity_y = -1.0f;
        field.add(dist);
        for (int i = 0; i < 10; ++i) field.update(1.0f / 60.0f);
        report("interaction_crater", field.sample_at(8.0f, 8.0f).height < 0.0f ? 1 : 0);
        report("interaction_dt_ok", field.stable_dt_limit() > field.fixed_dt() ? 1 : 0);
        field.recenter(30.0f, 8.0f);
        report("interaction_recentered", field.recentered() ? 1 : 0);
        report("interaction_shift_x", field.last_shift_x());
        report("interaction_shift_z", field.last_shift_z());
        const ocean::InteractionBuffers ib = field.buffers();
        report("interaction_buffers_size", ib.size);

        const ocean::WaterSurface ws(moved, field);
        ocean_surface_ex ex;
        bool combined_same = true, height_same = true;
        for (size_t i = 0; i + 1 < xz.size(); i += 2) {
            const ocean::Surface s = ws.sample_at(xz[i], xz[i + 1]);
            ocean_sample_combined(static_cast<const ocean_sim*>(moved.c_handle()),
                                  static_cast<const ocean_interaction*>(field.c_handle()), xz[i], xz[i + 1], &ex);
            combined_same = combined_same && std::memcmp(&s, &ex, sizeof(ex)) == 0;
            height_same = height_same &&
                          ws.height_at(xz[i], xz[i + 1]) ==
                              moved.height_at(xz[i], xz[i + 1]) + field.height_at(xz[i], xz[i + 1]);
        }
        report("water_surface_matches_c_combined", combined_same ? 1 : 0);
        report("water_surface_height_is_sum", height_same ? 1 : 0);
        const ocean::WaterSurface wc(cs, field);
        std::vector<ocean::Surface> wq;
        for (size_t i = 0; i + 1 < xz.size(); i += 2) wq.push_back(wc.sample_at(xz[i], xz[i + 1]));
        write_surfaces("water_cascade_queries.bin", wq);
        std::vector<float> iq;
        for (size_t i = 0; i + 1 < xz.size(); i += 2) {
            const ocean::InteractionSample e = wc.interaction_at(xz[i], xz[i + 1]);
            iq.insert(iq.end(), {e.height, e.slope_x, e.slope_z, e.velocity_y});
        }
        write_floats("water_cascade_interaction.bin", iq.data(), iq.size());
    }
    report("done", 1);
    return 0;
}
