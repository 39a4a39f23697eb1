// scene_loader.h -- TOML scene files (the reference's examples/*.toml schema)
// turned into an arp_scene.
#pragma once

#include <string>
#include <vector>

#include "../../include/arphys.h"

namespace arp {

struct LoadedScene {
    std::vector<arp_particle> particles, boundary;
    std::vector<arp_material> materials;
    std::vector<arp_interaction> interactions;
    std::vector<uint8_t> given;
    arp_aabb bounds{};
    float h = 1.0f / 64.0f, dt = 0.01f, gravity = 1.0f, alpha = 50.0f;
    uint32_t subticks = 1;
    int integrator = ARP_INT_VERLET;
    std::string name;
    // objects marked "on_click": seeded, not part of the initial scene; a host
    // passes them to add_particles (with an offset when `relative`)
    struct Addition {
        std::string name;
        std::vector<arp_particle> particles;
        arp_material material{};
        bool relative = false;
    };
    std::vector<Addition> on_click;
    // renderer settings of the file (examples/test_mods/config.rs:302-323)
    std::vector<float> colors;  // 12 per material: color, color_low_density, color_high_density
    bool lighting = false;
    float render_h = 1.0f / 64.0f;
    float light_pos[3] = {-3, 3, -3}, light_color[3] = {1, 1, 1};
    float ambient = 1.0f, diffuse = 10.0f, specular = 0.0f;
    double view_pos[2] = {0, 0}, view_scale = 1.0, view_angle = 0.0;

    arp_scene as_scene() const {
        arp_scene s{};
        s.particles = particles.data();
        s.n_particles = (uint32_t)particles.size();
        s.boundary = boundary.data();
        s.n_boundary = (uint32_t)boundary.size();
        s.materials = materials.data();
        s.n_materials = (uint32_t)materials.size();
        s.interactions = interactions.empty() ? nullptr : interactions.data();
        s.interaction_given = given.empty() ? nullptr : given.data();
        s.bounds = bounds;
        s.kernel_radius = h;
        s.integrator = integrator;
        s.timestep = dt;
        s.subticks = subticks;
        s.gravity = gravity;
        s.artificial_viscocity = alpha;
        return s;
    }
};

// Parse `path` and seed its regions.  Returns ARP_OK or an error code with a
// message in `err`.
arp_status load_scene_toml(const char* path, LoadedScene& out, std::string& err);

}  // namespace arp
