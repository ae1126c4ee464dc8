// plugin_host.cpp -- the reference's modifier-plugin ABI on the host side.
//
// A reference plugin is a shared library exporting biocore_plugin_init (returns the
// number of functions it registered, > 0) and optionally biocore_plugin_desc (a JSON
// descriptor); its init registers CPU functions through the host's
// register_modifier_current / register_modulator_release (extern "C",
// modifier_interface.h:38-39) or register_user_modifier / register_user_modulator
// (C++ linkage, plugin_manager.h:98-99).  The reference loads it with
// dlopen(RTLD_LAZY | RTLD_GLOBAL), keeps the handle for the process's life and puts the
// functions in its CPU dispatch tables, for IDs 0-127 (plugin_manager.cpp:36-60,
// 208-258).
//
// This backend exports the same four registration functions with the same names and
// linkage, so an unmodified plugin binds to it, and records which IDs a plugin
// registered.  The functions are CPU code: they never run here.  A network that uses
// an ID registered this way is refused at load unless device code is registered for
// it (biocore_gpu_register_device_modifier), because the reference would run the
// plugin's function on its CPU path, and this backend has no CPU fallback.
#include <dirent.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#define BNC_PLUGIN_HOST_IMPL
#include "common.h"

// The reference's types, by name only: the registration functions with C++ linkage
// mangle them (register_user_modifier(unsigned char, double (*)(Modifier*, Segment*,
// float))), so these declarations give the reference's symbol names.
struct Modifier;
struct Segment;
typedef double (*ModifierFunc)(Modifier* mod, Segment* seg, float dt);
typedef float (*ReleaseModulatorFunc)(Modifier* mod, float* cleft_nt, float dt);

namespace bnc {
namespace {
constexpr int kTableSize = 128;   // MOD_TABLE_SIZE (modifier_interface.h:16)
std::atomic<ModifierFunc> g_current[kTableSize];
std::atomic<ReleaseModulatorFunc> g_release[kTableSize];

struct LoadedPlugin {
    std::string path, name, version;
    std::vector<uint8_t> ids;   // from the descriptor
    int registered = 0;
};
std::mutex g_mu;
std::vector<LoadedPlugin> g_plugins;

// Value of "key": <string> after `from`, or empty.
std::string json_str(const char* from, const char* key) {
    const char* p = std::strstr(from, key);
    if (!p) return std::string();
    p = std::strchr(p + std::strlen(key), ':');
    if (!p) return std::string();
    p = std::strchr(p, '"');
    if (!p) return std::string();
    const char* e = std::strchr(p + 1, '"');
    return e ? std::string(p + 1, e) : std::string();
}

// The descriptor's fields the reference reads (plugin_manager.cpp:120-206): name,
// version and the "id" of each object in the "modifiers" array.
void parse_descriptor(const char* json, LoadedPlugin* pl) {
    if (!json) return;
    pl->name = json_str(json, "\"name\"");
    pl->version = json_str(json, "\"version\"");
    const char* m = std::strstr(json, "\"modifiers\"");
    if (!m) return;
    m = std::strchr(m, '[');
    if (!m) return;
    const char* end = std::strchr(m, ']');
    for (const char* p = m; (p = std::strstr(p, "\"id\"")) != nullptr && (!end || p < end); p++) {
        const char* c = std::strchr(p + 4, ':');
        if (!c) break;
        pl->ids.push_back((uint8_t)std::strtol(c + 1, nullptr, 10));
    }
}
}  // namespace

bool host_plugin_registered(uint8_t type) {
    return type < kTableSize && (g_current[type].load() != nullptr || g_release[type].load() != nullptr);
}
}  // namespace bnc

extern "C" void register_modifier_current(uint8_t type, ModifierFunc func) {
    if (type < bnc::kTableSize) bnc::g_current[type].store(func);
}

extern "C" void register_modulator_release(uint8_t type, ReleaseModulatorFunc func) {
    if (type < bnc::kTableSize) bnc::g_release[type].store(func);
}

void register_user_modifier(uint8_t type, ModifierFunc func) { register_modifier_current(type, func); }

void register_user_modulator(uint8_t type, ReleaseModulatorFunc func) { register_modulator_release(type, func); }

extern "C" {

int bnc_plugin_load(const char* so_path) {
    using namespace bnc;
    if (!so_path) { set_error("bnc_plugin_load: null path"); return -1; }
    // The plugin resolves register_* against the global scope; a host that loaded this
    // library with RTLD_LOCAL (a Python ctypes load, say) has it outside that scope, so
    // it is promoted first.
    Dl_info self;
    if (dladdr(reinterpret_cast<void*>(&register_modifier_current), &self) && self.dli_fname)
        dlopen(self.dli_fname, RTLD_NOW | RTLD_NOLOAD | RTLD_GLOBAL);
    void* h = dlopen(so_path, RTLD_LAZY | RTLD_GLOBAL);
    if (!h) {
        const char* e = dlerror();
        set_error("bnc_plugin_load: dlopen %s: %s", so_path, e ? e : "failed");
        return -1;
    }
    typedef int (*InitFunc)();
    typedef const char* (*DescFunc)();
    InitFunc init = reinterpret_cast<InitFunc>(dlsym(h, "biocore_plugin_init"));
    if (!init) {
        set_error("bnc_plugin_load: %s has no biocore_plugin_init", so_path);
        dlclose(h);
        return -2;
    }
    DescFunc desc = reinterpret_cast<DescFunc>(dlsym(h, "biocore_plugin_desc"));
    LoadedPlugin pl;
    pl.path = so_path;
    if (desc) parse_descriptor(desc(), &pl);
    const int registered = init();
    if (registered <= 0) {
        set_error("bnc_plugin_load: biocore_plugin_init of %s returned %d", so_path, registered);
        dlclose(h);
        return -3;
    }
    pl.registered = registered;
    std::lock_guard<std::mutex> lock(g_mu);
    g_plugins.push_back(pl);
    return registered;   // the handle stays open for the process, as in the reference
}

int bnc_plugin_load_directory(const char* dir_path) {
    using namespace bnc;
    if (!dir_path) { set_error("bnc_plugin_load_directory: null path"); return 0; }
    std::string dir(dir_path);
    while (dir.size() > 1 && dir.back() == '/') dir.pop_back();
    DIR* d = opendir(dir.c_str());
    if (!d) { set_error("bnc_plugin_load_directory: cannot open %s", dir.c_str()); return 0; }
    std::vector<std::string> files;
    while (struct dirent* e = readdir(d)) {
        const size_t len = std::strlen(e->d_name);
        if (len < 4 || std::strcmp(e->d_name + len - 3, ".so") != 0) continue;
        const std::string full = dir + "/" + e->d_name;
        struct stat st;
        if (stat(full.c_str(), &st) == 0 && S_ISREG(st.st_mode)) files.push_back(full);
    }
    closedir(d);
    int total = 0;
    for (const auto& f : files) {
        const int n = bnc_plugin_load(f.c_str());
        if (n > 0) total += n;
    }
    return total;
}

int bnc_plugin_registered(uint8_t type_id) {
    if (type_id >= bnc::kTableSize) return 0;
    return (bnc::g_current[type_id].load() ? 1 : 0) | (bnc::g_release[type_id].load() ? 2 : 0);
}

int bnc_plugin_count(void) {
    std::lock_guard<std::mutex> lock(bnc::g_mu);
    return (int)bnc::g_plugins.size();
}

void bnc_plugin_unregister_all(void) {
    for (int t = 0; t < bnc::kTableSize; t++) {
        bnc::g_current[t].store(nullptr);
        bnc::g_release[t].store(nullptr);
    }
}

}  // extern "C"
