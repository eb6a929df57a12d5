// Driver-API entry points resolved at run time through the CUDA runtime
// (cudaGetDriverEntryPoint), so libfip_b200.so does not link libcuda.so.1 and loads on a
// machine without a GPU driver (the host-only entry points and the CPU tests need that).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <string>

namespace fip {
namespace drv {

extern PFN_cuTensorMapEncodeTiled_v12000 TensorMapEncodeTiled;
extern PFN_cuModuleLoadData_v2000 ModuleLoadData;
extern PFN_cuModuleGetFunction_v2000 ModuleGetFunction;
extern PFN_cuModuleUnload_v2000 ModuleUnload;
extern PFN_cuLaunchKernel_v4000 LaunchKernel;
extern PFN_cuGetErrorString_v6000 GetErrorString;

// Resolves every pointer once (thread-safe); false with a message when a symbol is missing.
bool load(std::string* err);

// "name: message" of a driver result
std::string message(CUresult r, const char* what);

}  // namespace drv
}  // namespace fip
