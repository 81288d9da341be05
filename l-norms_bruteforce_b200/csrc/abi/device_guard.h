// Keeps a caller's current CUDA context across an entry point of the library.
//
// Every entry point selects the device it is asked for (cudaSetDevice), which
// makes that device's primary context current on the calling thread.  A
// caller that drives several GPUs from one thread, or a framework such as
// torch that relies on the thread's current device, must find the thread as
// it left it.  The guard records the thread's current driver context on entry
// and makes it current again on exit, including "no context" (restoring
// through cudaSetDevice instead would create a primary context on a device
// the caller never used).  The two driver calls are looked up through the
// runtime, so the library does not link libcuda itself.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace ldsolve {

class ContextRestore {
 public:
  ContextRestore() {
    if (fns().ok && fns().get(&prev_) == CUDA_SUCCESS) armed_ = true;
  }
  ~ContextRestore() {
    if (!armed_) return;
    CUcontext cur = nullptr;
    if (fns().get(&cur) == CUDA_SUCCESS && cur != prev_) fns().set(prev_);
  }
  ContextRestore(const ContextRestore&) = delete;
  ContextRestore& operator=(const ContextRestore&) = delete;

 private:
  struct Fns {
    CUresult (*get)(CUcontext*) = nullptr;
    CUresult (*set)(CUcontext) = nullptr;
    bool ok = false;
  };
  static const Fns& fns() {
    static const Fns f = [] {
      Fns r;
      void* g = nullptr;
      void* s = nullptr;
      cudaDriverEntryPointQueryResult qg, qs;
      if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &g, cudaEnableDefault, &qg) == cudaSuccess &&
          cudaGetDriverEntryPoint("cuCtxSetCurrent", &s, cudaEnableDefault, &qs) == cudaSuccess &&
          qg == cudaDriverEntryPointSuccess && qs == cudaDriverEntryPointSuccess && g && s) {
        r.get = reinterpret_cast<CUresult (*)(CUcontext*)>(g);
        r.set = reinterpret_cast<CUresult (*)(CUcontext)>(s);
        r.ok = true;
      }
      cudaGetLastError();   // a failed lookup (no driver) leaves no sticky error
      return r;
    }();
    return f;
  }
  CUcontext prev_ = nullptr;
  bool armed_ = false;
};

}  // namespace ldsolve
