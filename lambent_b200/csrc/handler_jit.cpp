// handler_jit.cpp - run-time compilation of intersection handlers (RayTracer::set_intersection_handler,
// src/lib.rs:291-295: the reference links the handler's WESL into its ray-query shader when the
// pipeline is created).  NVRTC compiles the handler's CUDA source to LTO intermediate code, nvJitLink
// links it with the procedural traversal kernels embedded in this library (procedural.cu), and the
// CUDA library API loads the result.  NVRTC and nvJitLink are opened on first use, so the library
// itself does not depend on them.
#include <dlfcn.h>
#include <nvJitLink.h>
#include <nvrtc.h>

#include <mutex>
#include <string>
#include <vector>

#include "scene.h"
#include "tracer.h"

extern "C" const char _binary_procedural_fatbin_start[], _binary_procedural_fatbin_end[];
extern "C" const char _binary_lambent_handler_h_start[], _binary_lambent_handler_h_end[];

namespace lam {

namespace {

struct JitApi {
    bool ok = false;
    std::string why;
    nvrtcResult (*createProgram)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compileProgram)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*getProgramLogSize)(nvrtcProgram, size_t*);
    nvrtcResult (*getProgramLog)(nvrtcProgram, char*);
    nvrtcResult (*getLTOIRSize)(nvrtcProgram, size_t*);
    nvrtcResult (*getLTOIR)(nvrtcProgram, char*);
    nvrtcResult (*destroyProgram)(nvrtcProgram*);
    nvJitLinkResult (*linkCreate)(nvJitLinkHandle*, uint32_t, const char**);
    nvJitLinkResult (*linkAddData)(nvJitLinkHandle, nvJitLinkInputType, const void*, size_t, const char*);
    nvJitLinkResult (*linkComplete)(nvJitLinkHandle);
    nvJitLinkResult (*linkCubinSize)(nvJitLinkHandle, size_t*);
    nvJitLinkResult (*linkCubin)(nvJitLinkHandle, void*);
    nvJitLinkResult (*linkErrorLogSize)(nvJitLinkHandle, size_t*);
    nvJitLinkResult (*linkErrorLog)(nvJitLinkHandle, char*);
    nvJitLinkResult (*linkDestroy)(nvJitLinkHandle*);
};

void* open_first(const char* const* names) {
    for (const char* const* n = names; *n; ++n)
        if (void* h = dlopen(*n, RTLD_NOW | RTLD_LOCAL)) return h;
    return nullptr;
}

template <class F>
bool sym(void* lib, const char* name, F& out) {
    out = reinterpret_cast<F>(dlsym(lib, name));
    return out != nullptr;
}

JitApi load_api() {
    JitApi a;
    // The toolkit's copies first: a process may already hold older ones under the same names (Python
    // frameworks bundle their own), and the embedded kernels need the linker of the CUDA that built them.
    static const char* rtc_names[] = {"/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12", "libnvrtc.so", nullptr};
    static const char* jl_names[] = {"/usr/local/cuda/lib64/libnvJitLink.so.12", "libnvJitLink.so.12", "libnvJitLink.so",
                                     nullptr};
    void* rtc = open_first(rtc_names);
    void* jl = open_first(jl_names);
    if (!rtc || !jl) {
        a.why = "NVRTC or nvJitLink (CUDA 12) not found";
        return a;
    }
    bool ok = sym(rtc, "nvrtcCreateProgram", a.createProgram) && sym(rtc, "nvrtcCompileProgram", a.compileProgram) &&
              sym(rtc, "nvrtcGetProgramLogSize", a.getProgramLogSize) && sym(rtc, "nvrtcGetProgramLog", a.getProgramLog) &&
              sym(rtc, "nvrtcGetLTOIRSize", a.getLTOIRSize) && sym(rtc, "nvrtcGetLTOIR", a.getLTOIR) &&
              sym(rtc, "nvrtcDestroyProgram", a.destroyProgram) && sym(jl, "__nvJitLinkCreate_12_9", a.linkCreate) &&
              sym(jl, "__nvJitLinkAddData_12_9", a.linkAddData) && sym(jl, "__nvJitLinkComplete_12_9", a.linkComplete) &&
              sym(jl, "__nvJitLinkGetLinkedCubinSize_12_9", a.linkCubinSize) &&
              sym(jl, "__nvJitLinkGetLinkedCubin_12_9", a.linkCubin) &&
              sym(jl, "__nvJitLinkGetErrorLogSize_12_9", a.linkErrorLogSize) &&
              sym(jl, "__nvJitLinkGetErrorLog_12_9", a.linkErrorLog) && sym(jl, "__nvJitLinkDestroy_12_9", a.linkDestroy);
    if (!ok) {
        a.why = "NVRTC / nvJitLink lack a required entry point (CUDA 12.9 or later needed)";
        return a;
    }
    a.ok = true;
    return a;
}

const JitApi& api() {
    static std::once_flag once;
    static JitApi a;
    std::call_once(once, [] { a = load_api(); });
    return a;
}

}  // namespace

// Compiles `source` (which defines intersect()) and links it with the procedural kernels into a
// cubin; the log of a failed step is returned in *log.
int compile_handler_cubin(const std::string& source, std::vector<char>* cubin, std::string* log) {
    const JitApi& a = api();
    if (!a.ok) {
        *log = a.why;
        return LAM_ERR_UNSUPPORTED;
    }
    const std::string header(_binary_lambent_handler_h_start, _binary_lambent_handler_h_end);
    const std::string program = "#include \"lambent_handler.h\"\n" + source +
                                "\nextern \"C\" __device__ lam_aabb_intersection lam_user_intersect(const lam_ray_intersection& i) {\n"
                                "    return intersect(i);\n}\n";
    const char* hdr_src[] = {header.c_str()};
    const char* hdr_name[] = {"lambent_handler.h"};
    nvrtcProgram prog = nullptr;
    if (a.createProgram(&prog, program.c_str(), "intersection_handler.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS) {
        *log = "nvrtcCreateProgram failed";
        return LAM_ERR_COMPILE;
    }
    const char* opts[] = {"-arch=sm_100a", "-dlto", "-rdc=true", "-std=c++17"};
    const nvrtcResult rc = a.compileProgram(prog, 4, opts);
    size_t n = 0;
    a.getProgramLogSize(prog, &n);
    std::string clog(n, '\0');
    if (n) a.getProgramLog(prog, &clog[0]);
    if (rc != NVRTC_SUCCESS) {
        *log = "handler does not compile:\n" + clog;
        a.destroyProgram(&prog);
        return LAM_ERR_COMPILE;
    }
    a.getLTOIRSize(prog, &n);
    std::vector<char> ir(n);
    a.getLTOIR(prog, ir.data());
    a.destroyProgram(&prog);

    nvJitLinkHandle h = nullptr;
    const char* lopts[] = {"-arch=sm_100a", "-lto", "-O3"};
    if (a.linkCreate(&h, 3, lopts) != NVJITLINK_SUCCESS) {
        *log = "nvJitLinkCreate failed";
        return LAM_ERR_COMPILE;
    }
    auto fail = [&](const char* what) {
        size_t m = 0;
        a.linkErrorLogSize(h, &m);
        std::string el(m, '\0');
        if (m) a.linkErrorLog(h, &el[0]);
        *log = std::string(what) + ":\n" + el;
        a.linkDestroy(&h);
        return LAM_ERR_COMPILE;
    };
    const size_t fb = (size_t)(_binary_procedural_fatbin_end - _binary_procedural_fatbin_start);
    if (a.linkAddData(h, NVJITLINK_INPUT_FATBIN, _binary_procedural_fatbin_start, fb, "procedural") != NVJITLINK_SUCCESS)
        return fail("linking the procedural kernels");
    if (a.linkAddData(h, NVJITLINK_INPUT_LTOIR, ir.data(), ir.size(), "handler") != NVJITLINK_SUCCESS)
        return fail("linking the handler");
    if (a.linkComplete(h) != NVJITLINK_SUCCESS) return fail("linking the handler into the traversal");
    size_t cs = 0;
    a.linkCubinSize(h, &cs);
    cubin->resize(cs);
    a.linkCubin(h, cubin->data());
    a.linkDestroy(&h);
    return LAM_OK;
}

int load_handler_module(const std::vector<char>& cubin, HandlerModule* m) {
    cudaError_t e = cudaLibraryLoadData(&m->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&m->extend, m->lib, "lam_proc_extend");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&m->trace_closest, m->lib, "lam_proc_trace_closest");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&m->trace_any, m->lib, "lam_proc_trace_any");
    if (e != cudaSuccess) return cuda_error(e, "loading the linked intersection handler");
    return LAM_OK;
}

void free_handler_module(HandlerModule* m) {
    if (!m) return;
    if (m->lib) cudaLibraryUnload(m->lib);
    delete m;
}

}  // namespace lam
