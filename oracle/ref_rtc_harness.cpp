// Test infrastructure only: runs the reference's run-time-compiled BM3D kernel
// (bm3dcuda_rtc, rtc_source/kernel.hpp) the way its plugin does, as the
// checker of this engine's block-distance and transform variants. Nothing in
// the product links this file.
//
// The reference header is #included unchanged; it holds the kernel source as
// two strings (kernel_header_template, kernel_source_template). The plugin's
// compile() (rtc_source/source.cpp:191-296) prepends the chosen transforms and
// distance as #defines and every parameter as a `__device__ static const`,
// compiles the text with NVRTC (-use_fast_math, -std=c++17) for the device's
// architecture and launches the `bm3d` kernel with (d_res, d_src) on a grid of
// ceil(width / (4 block_step)) x ceil(height / block_step) warps
// (rtc_source/source.cpp:357-376). refrtc_window does the same for one
// window; compiled modules are cached per program text.
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdio>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>

#include BM3D_REF_RTC_SOURCE

namespace {

thread_local std::string g_err;
std::mutex g_lock;
std::map<std::string, CUfunction> g_cache;

int fail(const std::string &msg) {
    g_err = msg;
    return 1;
}

const char *bm_name(int m) {
    static const char *names[] = {"ssd", "sad", "zssd", "zsad", "ssd_norm"};
    return (m >= 0 && m <= 4) ? names[m] : nullptr;
}

const char *tx_name(int t) {
    static const char *names[] = {"dct", "haar", "wht", "bior1_5"};
    return (t >= 0 && t <= 3) ? names[t] : nullptr;
}

// The program text of the plugin's compile() for one configuration.
std::string program_text(int width, int height, int stride, float sigma, int block_step,
                         int bm_range, int radius, int ps_num, int ps_range, bool chroma,
                         float sigma_u, float sigma_v, bool final_, const char *bm_error,
                         const char *t2d, const char *t1d, float extractor) {
    std::ostringstream o;
    o << kernel_header_template << "#define transform_2d " << t2d << "\n"
      << "#define transform_1d " << t1d << "\n"
      << "#define bm_error " << bm_error << "\n"
      << std::hexfloat << std::boolalpha;
    auto i = [&](const char *n, int v) { o << "__device__ static const int " << n << " = " << v << ";\n"; };
    auto f = [&](const char *n, float v) { o << "__device__ static const float " << n << " = " << v << ";\n"; };
    auto b = [&](const char *n, bool v) { o << "__device__ static const bool " << n << " = " << v << ";\n"; };
    i("width", width);
    i("height", height);
    i("stride", stride);
    f("sigma_y", sigma);
    i("block_step", block_step);
    i("bm_range", bm_range);
    i("_radius", radius);
    i("ps_num", ps_num);
    i("ps_range", ps_range);
    f("sigma_u", sigma_u);
    f("sigma_v", sigma_v);
    b("temporal", radius > 0);
    b("chroma", chroma);
    b("final_", final_);
    f("extractor", extractor);
    f("FLT_MAX", std::numeric_limits<float>::max());
    f("FLT_EPSILON", std::numeric_limits<float>::epsilon());
    o << kernel_source_template;
    return o.str();
}

int compile(const std::string &text, CUfunction *fn) {
    std::lock_guard<std::mutex> lk(g_lock);
    auto it = g_cache.find(text);
    if (it != g_cache.end()) {
        *fn = it->second;
        return 0;
    }
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess)
        return fail("no CUDA device");
    const std::string arch = "-arch=sm_" + std::to_string(major * 10 + minor);
    const char *opts[] = {arch.c_str(), "-use_fast_math", "-std=c++17",
                          "-modify-stack-limit=false"};
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, text.c_str(), nullptr, 0, nullptr, nullptr) != NVRTC_SUCCESS)
        return fail("nvrtcCreateProgram failed");
    if (nvrtcCompileProgram(prog, 4, opts) != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        nvrtcGetProgramLog(prog, log.data());
        nvrtcDestroyProgram(&prog);
        return fail("NVRTC: " + log);
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    std::unique_ptr<char[]> image(new char[n]);
    nvrtcGetCUBIN(prog, image.get());
    nvrtcDestroyProgram(&prog);
    cudaFree(nullptr);  // the runtime's primary context is current from here on
    CUmodule mod;
    if (cuModuleLoadData(&mod, image.get()) != CUDA_SUCCESS) return fail("cuModuleLoadData failed");
    if (cuModuleGetFunction(fn, mod, "bm3d") != CUDA_SUCCESS) return fail("no bm3d kernel");
    g_cache.emplace(text, *fn);
    return 0;
}

}  // namespace

extern "C" {

const char *refrtc_last_error(void) { return g_err.c_str(); }

// One BM3D window through the reference's run-time-compiled kernel: zeroes
// d_res and runs the kernel on `stream`. Buffers in the reference layouts
// (d_src [(final_ ? 2 : 1)][planes][2r+1][height][stride], d_res
// [planes][2r+1][2][height][stride]); sigma values already scaled;
// bm_error 0-4 (ssd, sad, zssd, zsad, ssd/norm), transforms 0-3 (dct, haar,
// wht, bior1.5).
int refrtc_window(float *d_res, const float *d_src, int width, int height, int stride,
                  float sigma, int block_step, int bm_range, int radius, int ps_num,
                  int ps_range, int chroma, float sigma_u, float sigma_v, int final_,
                  float extractor, int bm_error, int transform_2d, int transform_1d,
                  void *stream) {
    const char *be = bm_name(bm_error), *t2 = tx_name(transform_2d), *t1 = tx_name(transform_1d);
    if (!be || !t2 || !t1) return fail("invalid variant");
    CUfunction fn;
    if (int rc = compile(program_text(width, height, stride, sigma, block_step, bm_range, radius,
                                      ps_num, ps_range, chroma != 0, sigma_u, sigma_v,
                                      final_ != 0, be, t2, t1, extractor),
                         &fn))
        return rc;
    const size_t rows = (size_t)(chroma ? 3 : 1) * (2 * radius + 1) * 2 * height;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(d_res, 0, rows * stride * sizeof(float), s) != cudaSuccess)
        return fail("cudaMemsetAsync failed");
    void *args[] = {&d_res, &d_src};
    if (cuLaunchKernel(fn, (unsigned)((width + 4 * block_step - 1) / (4 * block_step)),
                       (unsigned)((height + block_step - 1) / block_step), 1, 32, 1, 1, 0,
                       (CUstream)s, args, nullptr) != CUDA_SUCCESS)
        return fail("cuLaunchKernel failed");
    return 0;
}

}  // extern "C"
