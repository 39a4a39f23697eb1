// scene_loader.cpp -- TOML scene loader (placeholder until the parser lands).
#include "scene_loader.h"

namespace arp {

arp_status load_scene_toml(const char* path, LoadedScene& out, std::string& err) {
    (void)path;
    (void)out;
    err = "TOML scene loading is not implemented in this build";
    return ARP_ERR_UNSUPPORTED;
}

}  // namespace arp
