/* Compiled as C (C99, -pedantic): the reference's C header path
 * "ocean/ocean.h" must be plain C, and the C ABI must link from a C object.
 * Written against the reference's C API only. main() runs a small session
 * and returns 0, or a code naming the first check that failed; the GPU test
 * runs it, the CPU test only compiles and links it. */
#include "ocean/ocean.h"

#include <stdio.h>

static unsigned g_calls = 0;

/* A blocking scheduler hook written in C. */
static void serial_for(void* user, ocean_task_fn task, void* ctx, uint32_t count)
{
    uint32_t i;
    (void)user;
    ++g_calls;
    for (i = 0; i < count; ++i) task(ctx, i);
}

int main(void)
{
    ocean_desc desc;
    ocean_status status = OCEAN_ERROR_UNKNOWN;
    ocean_sim* sim;
    ocean_buffers buf;
    ocean_surface s;
    ocean_surface_ex ex;
    ocean_interaction_desc idesc;
    ocean_interaction* field;
    ocean_interaction_sample is;
    ocean_disturbance dist;
    uint32_t major = 0, minor = 0, patch = 0;
    int i;

    ocean_desc_init(&desc);
    if (desc.struct_size != sizeof(ocean_desc)) return 1;
    desc.size = 32;
    desc.seed = 777u;
    desc.parallel_for = &serial_for;
    sim = ocean_create(&desc, &status);
    if (sim == NULL || status != OCEAN_OK) return 2;
    g_calls = 0;
    ocean_update(sim, 1.5);
    if (g_calls != 4u) return 3;
    if (ocean_get_time(sim) != 1.5) return 4;
    buf = ocean_get_buffers(sim);
    if (buf.displacement == NULL || buf.normal == NULL || buf.size != 32u) return 5;
    s = ocean_sample_at(sim, 2.0f, 5.0f);
    if (s.height != ocean_height_at(sim, 2.0f, 5.0f)) return 6;
    ocean_sample_ex(sim, 2.0f, 5.0f, &ex);
    if (ex.height != s.height) return 7;
    if (ocean_get_velocity(sim) != NULL) return 8;
    ocean_version(&major, &minor, &patch);
    if (major != 1u) return 9;
    if (ocean_simd_level() == NULL || ocean_status_string(OCEAN_OK) == NULL) return 10;

    ocean_interaction_desc_init(&idesc);
    idesc.size = 64;
    idesc.extent = 16.0f;
    field = ocean_interaction_create(&idesc, &status);
    if (field == NULL || status != OCEAN_OK) return 11;
    dist.world_x = 8.0f;
    dist.world_z = 8.0f;
    dist.radius = 0.5f;
    dist.strength = 0.25f;
    dist.velocity_y = -1.0f;
    dist.velocity_x = 0.0f;
    dist.velocity_z = 0.0f;
    dist.kind = OCEAN_SOURCE_IMPULSE;
    ocean_interaction_add(field, &dist);
    for (i = 0; i < 10; ++i) ocean_interaction_update(field, 1.0f / 60.0f);
    ocean_interaction_sample_at(field, 8.0f, 8.0f, &is);
    if (!(is.height < 0.0f)) return 12;
    ocean_sample_combined(sim, field, 8.0f, 8.0f, &ex);
    ocean_interaction_destroy(field);
    ocean_interaction_destroy(NULL);
    ocean_destroy(sim);
    ocean_destroy(NULL);
    printf("c header check ok\n");
    return 0;
}
