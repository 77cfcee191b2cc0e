// Host stand-ins for the CUDA runtime calls that the host code of csr.cu and
// precond.cu makes, so that code runs under AddressSanitizer and UBSan on a
// machine without a GPU: device memory is host memory, copies are memcpy,
// launches, graphs and streams do nothing (the fuzz drivers read no kernel
// output).  Test infrastructure only; never linked into the library.
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
extern "C" {
void** __cudaRegisterFatBinary(void*) { static void* h = nullptr; return &h; }
void __cudaRegisterFatBinaryEnd(void**) {}
void __cudaUnregisterFatBinary(void**) {}
void __cudaRegisterFunction(void**, const char*, char*, const char*, int, uint3*, uint3*, dim3*,
                            dim3*, int*) {}
char __cudaInitModule(void**) { return 0; }
unsigned __cudaPushCallConfiguration(dim3, dim3, size_t, void*) { return 0; }
cudaError_t __cudaPopCallConfiguration(dim3*, dim3*, size_t*, void*) { return cudaSuccess; }
cudaError_t cudaLaunchKernel(const void*, dim3, dim3, void**, size_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaMalloc(void** p, size_t n) { *p = malloc(n ? n : 1); return cudaSuccess; }
cudaError_t cudaFree(void* p) { free(p); return cudaSuccess; }
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { memcpy(d, s, n); return cudaSuccess; }
cudaError_t cudaMemset(void* d, int v, size_t n) { memset(d, v, n); return cudaSuccess; }
cudaError_t cudaPointerGetAttributes(cudaPointerAttributes*, const void*) { return cudaErrorInvalidValue; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaEventDestroy(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
}
// the library's own helpers that a driver's source file may not define
// (weak: a definition in the file under test wins)
struct sb2_csr;
namespace sb2 {
__attribute__((weak)) int current_device() { return 0; }
__attribute__((weak)) int map_cuda_error(cudaError_t) { return -3; }
__attribute__((weak)) int num_sms(int) { return 148; }
__attribute__((weak)) int ensure_diag(const sb2_csr*) { return 0; }
}
extern "C" {
cudaError_t cudaGraphDestroy(cudaGraph_t) { return cudaSuccess; }
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t) { return cudaSuccess; }
cudaError_t cudaGraphInstantiate(cudaGraphExec_t* e, cudaGraph_t, unsigned long long) {
  *e = nullptr;
  return cudaSuccess;
}
cudaError_t cudaGraphLaunch(cudaGraphExec_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) {
  memcpy(d, s, n);
  return cudaSuccess;
}
cudaError_t cudaMemsetAsync(void* d, int v, size_t n, cudaStream_t) { memset(d, v, n); return cudaSuccess; }
cudaError_t cudaStreamBeginCapture(cudaStream_t, cudaStreamCaptureMode) { return cudaSuccess; }
cudaError_t cudaStreamEndCapture(cudaStream_t, cudaGraph_t* g) { *g = nullptr; return cudaSuccess; }
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned) { *s = nullptr; return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
}

extern "C" {
cudaError_t cudaEventCreate(cudaEvent_t* e) { *e = nullptr; return cudaSuccess; }
cudaError_t cudaFuncSetAttribute(const void*, cudaFuncAttribute, int) { return cudaSuccess; }
cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) { *ms = 1.0f; return cudaSuccess; }
cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(int* n, const void*, int, size_t,
                                                                   unsigned) {
  *n = 1;
  return cudaSuccess;
}
cudaError_t cudaOccupancyMaxActiveClusters(int* n, const void*, const cudaLaunchConfig_t*) {
  *n = 1;
  return cudaSuccess;
}
cudaError_t cudaLaunchKernelExC(const cudaLaunchConfig_t*, const void*, void**) { return cudaSuccess; }
}
