// Consumer narrow phases: the traversal kernels recompiled at run time with
// NVRTC around the caller's `sq_narrow` device function.
//
// The reference's `gpu` feature takes the consumer's narrow phase as WGSL
// source and splices it into its shader (GpuGeometry::narrow_wgsl,
// crates/spatial-query/src/gpu/mod.rs:69-99). Here the consumer hands CUDA
// source: it is compiled for sm_100a together with the library's own
// traversal headers (embedded at build time), with --fmad=false like the
// built-in kernels, and the nearest / all-hits instantiations are loaded as a
// CUDA library whose kernel handles launch through the same runtime calls as
// the built-in kernels.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "sq_internal.cuh"
#include "rtc_sources.h"  // generated by build.py: kRtcMath, kRtcTraverse

namespace sqi {

namespace {

struct Entry {
  cudaLibrary_t lib = nullptr;
  sq::KernelSet ks{};
};

std::mutex g_mu;
std::map<std::string, Entry> g_cache;

const char* const kNames[6] = {
    "&sq::query_kernel<3, 4, 0, false, false, false>",  // ray nearest, near-first
    "&sq::query_kernel<3, 4, 0, false, true, false>",   // ... with counters
    "&sq::query_kernel<3, 4, 0, true, false, false>",   // ray nearest, reference order
    "&sq::query_kernel<3, 4, 0, true, true, false>",    // ... with counters
    "&sq::query_kernel<3, 4, 1, true, false, false>",   // all hits
    "&sq::query_kernel<3, 4, 1, true, true, false>",    // ... with counters
};

}  // namespace

int32_t rtc_kernel_set(uint32_t stride, const char* src, sq::KernelSet* out, std::string* log) {
  const std::string key = std::to_string(stride) + '\n' + src;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *out = it->second.ks;
    return SQ_OK;
  }
  // A source that defines sq_narrow_crossings also serves raycast_crossings
  // with every crossing it emits.
  const bool crossings = std::strstr(src, "sq_narrow_crossings") != nullptr;
  const std::string prog_src = "#define SQ_RTC_CUSTOM 1\n#define SQ_CUSTOM_STRIDE " + std::to_string(stride) +
                               (crossings ? "\n#define SQ_RTC_CROSSINGS 1" : "") +
                               "\n#include \"traverse.cuh\"\nnamespace sq {\n#line 1 \"narrow\"\n" + src +
                               "\n}  // namespace sq\n";
  const char* headers[2] = {kRtcMath, kRtcTraverse};
  const char* header_names[2] = {"sq_math.cuh", "traverse.cuh"};
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, prog_src.c_str(), "consumer_narrow.cu", 2, headers, header_names) !=
      NVRTC_SUCCESS) {
    *log = "nvrtcCreateProgram failed";
    return SQ_ERR_COMPILE;
  }
  for (const char* n : kNames) nvrtcAddNameExpression(prog, n);
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-lineinfo",
                        "-diag-suppress=549"};
  const nvrtcResult cr = nvrtcCompileProgram(prog, 5, opts);
  if (cr != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string l(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &l[0]);
    *log = std::string("consumer narrow phase did not compile: ") + nvrtcGetErrorString(cr) + "\n" + l;
    nvrtcDestroyProgram(&prog);
    return SQ_ERR_COMPILE;
  }
  size_t cubin_size = 0;
  nvrtcGetCUBINSize(prog, &cubin_size);
  std::vector<char> cubin(cubin_size);
  nvrtcGetCUBIN(prog, cubin.data());
  std::string lowered[6];
  for (int i = 0; i < 6; ++i) {
    const char* ln = nullptr;
    nvrtcGetLoweredName(prog, kNames[i], &ln);
    lowered[i] = ln ? ln : "";
  }
  nvrtcDestroyProgram(&prog);

  Entry e;
  cudaError_t ce = cudaLibraryLoadData(&e.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (ce != cudaSuccess) {
    *log = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(ce);
    return SQ_ERR_CUDA;
  }
  cudaKernel_t k[6];
  for (int i = 0; i < 6; ++i) {
    ce = lowered[i].empty() ? cudaErrorSymbolNotFound : cudaLibraryGetKernel(&k[i], e.lib, lowered[i].c_str());
    if (ce != cudaSuccess) {
      *log = std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(ce);
      cudaLibraryUnload(e.lib);
      return SQ_ERR_CUDA;
    }
  }
  e.ks = sq::KernelSet{};
  e.ks.ray_nearest[0][0] = reinterpret_cast<const void*>(k[0]);
  e.ks.ray_nearest[0][1] = reinterpret_cast<const void*>(k[1]);
  e.ks.ray_nearest[1][0] = reinterpret_cast<const void*>(k[2]);
  e.ks.ray_nearest[1][1] = reinterpret_cast<const void*>(k[3]);
  e.ks.ray_all[0] = reinterpret_cast<const void*>(k[4]);
  e.ks.ray_all[1] = reinterpret_cast<const void*>(k[5]);
  g_cache[key] = e;
  *out = e.ks;
  return SQ_OK;
}

}  // namespace sqi
