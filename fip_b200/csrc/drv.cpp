#include "drv.h"

#include <cuda_runtime.h>

#include <mutex>

namespace fip {
namespace drv {

PFN_cuTensorMapEncodeTiled_v12000 TensorMapEncodeTiled = nullptr;
PFN_cuModuleLoadData_v2000 ModuleLoadData = nullptr;
PFN_cuModuleGetFunction_v2000 ModuleGetFunction = nullptr;
PFN_cuModuleUnload_v2000 ModuleUnload = nullptr;
PFN_cuLaunchKernel_v4000 LaunchKernel = nullptr;
PFN_cuGetErrorString_v6000 GetErrorString = nullptr;

namespace {
std::once_flag g_once;
std::string g_err;

template <typename T>
void resolve(const char* name, T* out) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
    if (g_err.empty()) g_err = std::string("driver entry point ") + name + " unavailable: " + cudaGetErrorString(e);
    return;
  }
  *out = reinterpret_cast<T>(p);
}
}  // namespace

bool load(std::string* err) {
  std::call_once(g_once, [] {
    resolve("cuTensorMapEncodeTiled", &TensorMapEncodeTiled);
    resolve("cuModuleLoadData", &ModuleLoadData);
    resolve("cuModuleGetFunction", &ModuleGetFunction);
    resolve("cuModuleUnload", &ModuleUnload);
    resolve("cuLaunchKernel", &LaunchKernel);
    resolve("cuGetErrorString", &GetErrorString);
  });
  if (!g_err.empty()) {
    if (err) *err = g_err;
    return false;
  }
  return true;
}

std::string message(CUresult r, const char* what) {
  const char* s = nullptr;
  if (GetErrorString) GetErrorString(r, &s);
  return std::string(what) + ": " + (s ? s : ("CUresult " + std::to_string((int)r)).c_str());
}

}  // namespace drv
}  // namespace fip
