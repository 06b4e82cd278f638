// ref_stubs.cpp -- host-side stand-ins for the two CUDA stream calls that the reference's
// LeCoGPU<T> constructor and destructor make (api/G-LeCo.cuh:103-113).  With
// GLC_REF_CPU_ONLY=1 they succeed without a driver, so the reference's host-only code
// (directRandomAccessCPU, the CPU partitioner) can run in a container without a GPU; otherwise
// they forward to the CUDA runtime.  TEST INFRASTRUCTURE ONLY (linked into _ref/ref_harness).
#include <dlfcn.h>
#include <cstdlib>

typedef int cuda_status;           // cudaError_t; 0 == cudaSuccess
typedef struct CUstream_st* cuda_stream;

static bool cpu_only() {
  const char* e = getenv("GLC_REF_CPU_ONLY");
  return e && e[0] == '1';
}

extern "C" cuda_status cudaStreamCreate(cuda_stream* s) {
  if (cpu_only()) { *s = nullptr; return 0; }
  typedef cuda_status (*fn_t)(cuda_stream*);
  static fn_t real = (fn_t)dlsym(RTLD_NEXT, "cudaStreamCreate");
  return real ? real(s) : 1;
}

extern "C" cuda_status cudaStreamDestroy(cuda_stream s) {
  if (cpu_only()) return 0;
  typedef cuda_status (*fn_t)(cuda_stream);
  static fn_t real = (fn_t)dlsym(RTLD_NEXT, "cudaStreamDestroy");
  return real ? real(s) : 1;
}
