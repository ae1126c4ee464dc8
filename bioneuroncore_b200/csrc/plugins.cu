// plugins.cu -- user modifiers on the device: registration, compilation, launch.
//
// The reference's plugins register host functions for modifier IDs 0-127
// (register_modifier_current, modifier_interface.h:38) that override the built-in
// model of that ID on the CPU path (kernel_dispatch.h:336-343); its device path has
// no plugins and returns 0 for unknown IDs (kernel_dispatch.h:564-568).  Here a user
// modifier is CUDA C++ source (include/bnc_device_modifier.h describes what it
// sees), compiled once by NVRTC for sm_100a, loaded with the runtime's library API
// on each device that runs it, and launched by the modifier pass on the user
// type's items of every phase.  NVRTC is opened with dlopen on first use, so the
// library loads on machines without it and reports its absence only when a user
// modifier is registered.
#include <dlfcn.h>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "net.h"
#include "bnc_device_modifier.h"

namespace bnc {

static_assert(sizeof(BncSegmentState) == sizeof(SegRec), "user segment view matches SegRec");
static_assert(offsetof(BncSegmentState, itot) == offsetof(SegRec, itot), "itot offset");
static_assert(offsetof(BncSegmentState, vol) == offsetof(SegRec, vol), "vol offset");
static_assert(offsetof(BncSegmentState, area) == offsetof(SegRec, area), "area offset");

namespace {

// The interface header handed to NVRTC under its include name.
const char* const kDeviceModifierHeader =
#include "bnc_device_modifier_h.inc"
    ;

// NVRTC entry points (nvrtc.h), resolved from libnvrtc at run time.
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
    bool tried = false, ok = false;
    std::string why;
    const char* (*GetErrorString)(nvrtcResult_t) = nullptr;
    nvrtcResult_t (*CreateProgram)(nvrtcProgram_t*, const char*, const char*, int, const char* const*,
                                   const char* const*) = nullptr;
    nvrtcResult_t (*CompileProgram)(nvrtcProgram_t, int, const char* const*) = nullptr;
    nvrtcResult_t (*GetProgramLogSize)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*GetProgramLog)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*GetCUBINSize)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*GetCUBIN)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*DestroyProgram)(nvrtcProgram_t*) = nullptr;
};

Nvrtc g_nvrtc;

bool load_nvrtc() {
    if (g_nvrtc.tried) return g_nvrtc.ok;
    g_nvrtc.tried = true;
    void* h = nullptr;
    for (const char* name : {"libnvrtc.so.12", "libnvrtc.so"}) {
        h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
        if (h) break;
    }
    if (!h) { g_nvrtc.why = "libnvrtc.so.12 not found"; return false; }
    bool ok = true;
    auto sym = [&](const char* n) { void* p = dlsym(h, n); if (!p) ok = false; return p; };
    g_nvrtc.GetErrorString = (const char* (*)(nvrtcResult_t))sym("nvrtcGetErrorString");
    g_nvrtc.CreateProgram = (decltype(g_nvrtc.CreateProgram))sym("nvrtcCreateProgram");
    g_nvrtc.CompileProgram = (decltype(g_nvrtc.CompileProgram))sym("nvrtcCompileProgram");
    g_nvrtc.GetProgramLogSize = (decltype(g_nvrtc.GetProgramLogSize))sym("nvrtcGetProgramLogSize");
    g_nvrtc.GetProgramLog = (decltype(g_nvrtc.GetProgramLog))sym("nvrtcGetProgramLog");
    g_nvrtc.GetCUBINSize = (decltype(g_nvrtc.GetCUBINSize))sym("nvrtcGetCUBINSize");
    g_nvrtc.GetCUBIN = (decltype(g_nvrtc.GetCUBIN))sym("nvrtcGetCUBIN");
    g_nvrtc.DestroyProgram = (decltype(g_nvrtc.DestroyProgram))sym("nvrtcDestroyProgram");
    if (!ok) { g_nvrtc.why = "libnvrtc lacks an expected entry point"; return false; }
    g_nvrtc.ok = true;
    return true;
}

struct DeviceModifier {
    std::string entry;
    std::vector<char> cubin;
    cudaLibrary_t lib = nullptr;   // loaded on first use on a device (context-independent)
    cudaKernel_t kernel = nullptr;
};

std::mutex g_mu;
// Registered modifiers.  Entries are never freed: a network built with one keeps
// its kernel handle (the reference keeps plugin handles open the same way,
// plugin_manager.cpp:214,255).
DeviceModifier* g_mods[128] = {};

int compile(uint8_t type_id, const char* source, const char* entry, std::vector<char>* cubin) {
    if (!load_nvrtc()) { set_error("device modifier %u: NVRTC unavailable (%s)", type_id, g_nvrtc.why.c_str()); return BNC_ERR_UNSUPPORTED; }
    nvrtcProgram_t prog = nullptr;
    const char* hdr_src[1] = {kDeviceModifierHeader};
    const char* hdr_name[1] = {"bnc_device_modifier.h"};
    char name[64];
    snprintf(name, sizeof(name), "device_modifier_%u.cu", type_id);
    nvrtcResult_t r = g_nvrtc.CreateProgram(&prog, source, name, 1, hdr_src, hdr_name);
    if (r != 0) { set_error("device modifier %u: %s", type_id, g_nvrtc.GetErrorString(r)); return BNC_ERR_ARG; }
    const char* opts[] = {"--gpu-architecture=sm_100a", "--fmad=false", "--std=c++17"};
    r = g_nvrtc.CompileProgram(prog, 3, opts);
    if (r != 0) {
        size_t n = 0;
        g_nvrtc.GetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        if (n) g_nvrtc.GetProgramLog(prog, &log[0]);
        g_nvrtc.DestroyProgram(&prog);
        set_error("device modifier %u does not compile: %s", type_id, log.c_str());
        return BNC_ERR_ARG;
    }
    size_t n = 0;
    g_nvrtc.GetCUBINSize(prog, &n);
    cubin->assign(n, 0);
    if (n) g_nvrtc.GetCUBIN(prog, cubin->data());
    g_nvrtc.DestroyProgram(&prog);
    if (n == 0) { set_error("device modifier %u: empty compilation result", type_id); return BNC_ERR_ARG; }
    // the entry must exist in the source as an extern "C" kernel
    std::string needle = std::string(entry);
    if (std::strstr(source, needle.c_str()) == nullptr) {
        set_error("device modifier %u: entry '%s' not found in the source", type_id, entry);
        return BNC_ERR_ARG;
    }
    return BNC_OK;
}

}  // namespace

bool device_modifier_registered(uint8_t type) {
    if (type >= 128) return false;
    std::lock_guard<std::mutex> lock(g_mu);
    return g_mods[type] != nullptr;
}

int device_modifier_kernel(uint8_t type, const void** kernel) {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceModifier* m = type < 128 ? g_mods[type] : nullptr;
    if (!m) { set_error("modifier type %u has no registered device implementation", type); return BNC_ERR_UNSUPPORTED; }
    if (!m->kernel) {
        cudaError_t e = cudaLibraryLoadData(&m->lib, m->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
        if (e != cudaSuccess) { set_error("device modifier %u: loading failed: %s", type, cudaGetErrorString(e)); return BNC_ERR_CUDA; }
        e = cudaLibraryGetKernel(&m->kernel, m->lib, m->entry.c_str());
        if (e != cudaSuccess) {
            set_error("device modifier %u: kernel '%s' not found (declare it extern \"C\" __global__): %s", type,
                      m->entry.c_str(), cudaGetErrorString(e));
            m->kernel = nullptr;
            return BNC_ERR_ARG;
        }
    }
    *kernel = (const void*)m->kernel;
    return BNC_OK;
}

cudaError_t launch_device_modifier(const void* kernel, const NetDev& d, uint8_t type, uint32_t b, uint32_t e, float dt,
                                   cudaStream_t stream) {
    BncDeviceModifierArgs a;
    a.seg = reinterpret_cast<BncSegmentState*>(d.rec);
    a.item_seg = d.it_seg;
    a.density = d.it_den;
    a.state = d.it_st;
    a.nt = d.nt;
    a.n_items = d.n_items;
    a.n_seg = d.n_seg;
    a.begin = b;
    a.end = e;
    a.dt = dt;
    a.type = type;
    void* args[1] = {&a};
    return cudaLaunchKernel(kernel, dim3((e - b + 255) / 256), dim3(256), args, 0, stream);
}

}  // namespace bnc

using namespace bnc;

extern "C" {

int bnc_register_device_modifier(uint8_t type_id, const char* source, const char* entry) {
    if (!source || !entry || !*entry) { set_error("bnc_register_device_modifier: null argument"); return BNC_ERR_ARG; }
    if (type_id >= 128) {
        set_error("device modifier IDs are the reference's plugin range 0-127 (got %u)", type_id);
        return BNC_ERR_ARG;
    }
    std::unique_ptr<DeviceModifier> m(new DeviceModifier());
    m->entry = entry;
    int rc = compile(type_id, source, entry, &m->cubin);
    if (rc != BNC_OK) return rc;
    std::lock_guard<std::mutex> lock(g_mu);
    g_mods[type_id] = m.release();   // a previous entry stays alive for networks built with it
    return BNC_OK;
}

int biocore_gpu_register_device_modifier(uint8_t type_id, const char* cu_path, const char* entry) {
    if (!cu_path) { set_error("biocore_gpu_register_device_modifier: null path"); return BNC_ERR_ARG; }
    FILE* f = fopen(cu_path, "rb");
    if (!f) { set_error("cannot open %s", cu_path); return BNC_BION_ERR_FILE_OPEN; }
    std::string src;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) src.append(buf, n);
    fclose(f);
    return bnc_register_device_modifier(type_id, src.c_str(), entry);
}

int bnc_device_modifier_registered(uint8_t type_id) { return device_modifier_registered(type_id) ? 1 : 0; }

}  // extern "C"
