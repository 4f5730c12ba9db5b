// Device functions in place of teal's host Compute callbacks (src/equations.h:27-41): the custom
// boundary condition (src/equations/boundary.c:27-33) and the source term
// (src/equations/derivative.c:242-266). A caller registers CUDA C source defining
//
//   __device__ void <name>(double *out, const double *property, const double *center, double time,
//                          const double *context)
//
// with teal's Compute arguments; the registry wraps it in a kernel over the boundary's faces or
// the inner cells, compiles it with NVRTC for sm_100a (loaded at run time: the library does not
// link NVRTC) and loads the code with the runtime's context-independent library API on first use.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cctype>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "functions.h"

namespace tg {
namespace {

struct Nvrtc {
    void *handle = nullptr;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

void load_nvrtc(Nvrtc &n)
{
    const char *paths[] = {"/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12", "libnvrtc.so"};
    for (const char *p : paths) {
        n.handle = dlopen(p, RTLD_NOW | RTLD_LOCAL);
        if (n.handle) break;
    }
    if (!n.handle) return;
    n.create = (decltype(n.create))dlsym(n.handle, "nvrtcCreateProgram");
    n.compile = (decltype(n.compile))dlsym(n.handle, "nvrtcCompileProgram");
    n.log_size = (decltype(n.log_size))dlsym(n.handle, "nvrtcGetProgramLogSize");
    n.log = (decltype(n.log))dlsym(n.handle, "nvrtcGetProgramLog");
    n.cubin_size = (decltype(n.cubin_size))dlsym(n.handle, "nvrtcGetCUBINSize");
    n.cubin = (decltype(n.cubin))dlsym(n.handle, "nvrtcGetCUBIN");
    n.destroy = (decltype(n.destroy))dlsym(n.handle, "nvrtcDestroyProgram");
    if (!n.create || !n.compile || !n.log_size || !n.log || !n.cubin_size || !n.cubin || !n.destroy) {
        dlclose(n.handle);
        n.handle = nullptr;
    }
}

// NVRTC of the CUDA installation, else whichever libnvrtc the loader finds (looked up once)
const Nvrtc *nvrtc()
{
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] { load_nvrtc(n); });
    return n.handle ? &n : nullptr;
}

struct Entry {
    int kind = 0;
    std::vector<char> cubin;
    cudaLibrary_t library = nullptr;
    cudaKernel_t kernel = nullptr;
};

std::mutex registry_mutex;
std::map<std::string, Entry> &registry()
{
    static std::map<std::string, Entry> r;
    return r;
}

bool valid_name(const char *name)
{
    if (!name || !(std::isalpha((unsigned char)name[0]) || name[0] == '_')) return false;
    size_t n = std::strlen(name);
    if (n > 64) return false;
    for (size_t i = 0; i < n; i++) {
        if (!(std::isalnum((unsigned char)name[i]) || name[i] == '_')) return false;
    }
    return std::strncmp(name, "tg_", 3) != 0;  // the wrapper's own names
}

// The wrapper kernels (the user's source comes first). Boundary: for the faces [f0, f0 + n) of one
// boundary, outer = the ghost row as it stands (teal's Compute writes into it in place), context =
// the inner cell's primitive state, center = the ghost cell's centre. Source: S[v][c] for every
// inner cell, from a zeroed source vector; its context is the cell's state followed by the Prepare
// pass's volume average (avg; zeros without one). The stage time is time[0] + coef * step[0] on the
// device inside step sequences, else host_time. A stopped instance (active[0] == 0) is left as it is.
const char *boundary_wrapper = R"(
extern "C" __global__ void tg_function_kernel(int n, int f0, const int *lr, const double *center, double *q,
                                              long N, const double *property, const double *time,
                                              const double *step, double coef, double host_time,
                                              const int *active)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (active && !active[0])) {
        return;
    }
    const int f = f0 + i;
    const long l = lr[2 * (long)f], r = lr[2 * (long)f + 1];
    double inner[5], outer[5];
    for (int v = 0; v < 5; v++) {
        inner[v] = q[v * N + l];
        outer[v] = q[v * N + r];
    }
    const double t = time ? time[0] + coef * step[0] : host_time;
    TG_USER_FUNCTION(outer, property, center + 3 * (long)i, t, inner);
    for (int v = 0; v < 5; v++) {
        q[v * N + r] = outer[v];
    }
}
)";

const char *source_wrapper = R"(
extern "C" __global__ void tg_function_kernel(int C, const double *center, const double *q, long N,
                                              const double *property, const double *time,
                                              const double *step, double coef, double host_time,
                                              double *S, const double *avg)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    double state[10], s[5] = {0, 0, 0, 0, 0};
    for (int v = 0; v < 5; v++) {
        state[v] = q[v * N + c];
        state[5 + v] = avg ? avg[v] : 0.0;
    }
    const double t = time ? time[0] + coef * step[0] : host_time;
    TG_USER_FUNCTION(s, property, center + 3 * (long)c, t, state);
    for (int v = 0; v < 5; v++) {
        S[(long)v * C + c] = s[v];
    }
}
)";

void put_log(char *log, long log_size, const std::string &text)
{
    if (log && log_size > 0) {
        size_t n = std::min((size_t)log_size - 1, text.size());
        std::memcpy(log, text.data(), n);
        log[n] = 0;
    }
}

}  // namespace

int function_register(const char *name, int kind, const char *source, char *log, long log_size,
                      std::string &error)
{
    put_log(log, log_size, "");
    if (!valid_name(name)) {
        error = "a device function name is a C identifier of at most 64 characters not starting with tg_";
        return 1;
    }
    if (kind != FUNCTION_BOUNDARY && kind != FUNCTION_SOURCE) {
        error = "device function kind must be boundary (1) or source (2)";
        return 1;
    }
    if (!source) {
        error = "null device function source";
        return 1;
    }
    const Nvrtc *rt = nvrtc();
    if (!rt) {
        error = "NVRTC (libnvrtc.so.12) could not be loaded";
        return 2;
    }
    std::string text = std::string("#define TG_USER_FUNCTION ") + name + "\n#line 1 \"" + name + "\"\n" + source +
                       "\n" + (kind == FUNCTION_BOUNDARY ? boundary_wrapper : source_wrapper);
    nvrtcProgram prog = nullptr;
    if (rt->create(&prog, text.c_str(), name, 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        error = "NVRTC could not create the program";
        return 2;
    }
    // no contraction of products into FMAs: host C callbacks (teal's ISO C build) round each step
    const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false", "-default-device"};
    nvrtcResult rc = rt->compile(prog, 4, opts);
    size_t ls = 0;
    rt->log_size(prog, &ls);
    std::string text_log(ls ? ls : 1, '\0');
    if (ls) rt->log(prog, &text_log[0]);
    put_log(log, log_size, text_log.c_str());
    if (rc != NVRTC_SUCCESS) {
        rt->destroy(&prog);
        error = std::string("device function ") + name + " does not compile (see the log)";
        return 1;
    }
    size_t cs = 0;
    rt->cubin_size(prog, &cs);
    Entry e;
    e.kind = kind;
    e.cubin.resize(cs);
    rt->cubin(prog, e.cubin.data());
    rt->destroy(&prog);
    std::lock_guard<std::mutex> lock(registry_mutex);
    // a replaced function's code stays loaded: contexts bound to it keep launching its kernel
    registry()[name] = std::move(e);
    return 0;
}

int function_kernel(const char *name, int kind, const void **kernel, std::string &error)
{
    std::lock_guard<std::mutex> lock(registry_mutex);
    auto &r = registry();
    auto it = r.find(name ? name : "");
    if (it == r.end()) {
        error = std::string("no device function registered as ") + (name ? name : "(null)");
        return 1;
    }
    Entry &e = it->second;
    if (e.kind != kind) {
        error = std::string("device function ") + name + " has another kind";
        return 1;
    }
    if (!e.kernel) {
        cudaError_t c = cudaLibraryLoadData(&e.library, e.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
        if (c == cudaSuccess) c = cudaLibraryGetKernel(&e.kernel, e.library, "tg_function_kernel");
        if (c != cudaSuccess) {
            error = std::string("loading device function ") + name + ": " + cudaGetErrorString(c);
            e.kernel = nullptr;
            return 2;
        }
    }
    *kernel = reinterpret_cast<const void *>(e.kernel);
    return 0;
}

}  // namespace tg
