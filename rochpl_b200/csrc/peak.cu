// FP64 throughput probes: the roofline denominators for the DGEMM.
//
// dmma_peak_kernel keeps every warp issuing independent m16n8k8 f64 MMAs on
// register operands (8 accumulator chains per warp), dfma_peak_kernel does the
// same with scalar DFMA.  Neither touches memory inside the timed loop, so the
// rate is the FP64 tensor / FP64 vector issue ceiling at the clocks the GPU
// runs under that load.
#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

__global__ void __launch_bounds__(256) dmma_peak_kernel(int iters, double seed, double* out) {
  double a[4], b[2], d[8][4];
#pragma unroll
  for(int q = 0; q < 4; ++q) a[q] = seed * (threadIdx.x + q + 1);
  b[0] = seed * 0.5;
  b[1] = seed * 0.25;
#pragma unroll
  for(int c = 0; c < 8; ++c)
#pragma unroll
    for(int q = 0; q < 4; ++q) d[c][q] = 0.0;
  for(int it = 0; it < iters; ++it) {
#pragma unroll
    for(int c = 0; c < 8; ++c)
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
          "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
          : "+d"(d[c][0]), "+d"(d[c][1]), "+d"(d[c][2]), "+d"(d[c][3])
          : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
  }
  double s = 0.0;
#pragma unroll
  for(int c = 0; c < 8; ++c) s += d[c][0] + d[c][1] + d[c][2] + d[c][3];
  if(s == 12345.678) out[0] = s;  // keeps the chains alive; never true for the probe input
}

__global__ void __launch_bounds__(256) dfma_peak_kernel(int iters, double seed, double* out) {
  double x[16];
  const double y = seed * 0.999, z = seed * 1e-3;
#pragma unroll
  for(int c = 0; c < 16; ++c) x[c] = seed * (threadIdx.x + c);
  for(int it = 0; it < iters; ++it)
#pragma unroll
    for(int c = 0; c < 16; ++c) x[c] = fma(x[c], y, z);
  double s = 0.0;
#pragma unroll
  for(int c = 0; c < 16; ++c) s += x[c];
  if(s == 12345.678) out[0] = s;
}

// Waits on a flag nothing sets, with the library's bounded-wait pattern and a
// caller-chosen budget: the host sees ST_TIMEOUT and the context stays usable.
__global__ void wait_selftest_kernel(const int* flag, int* status, unsigned long long budget_ns) {
  if(threadIdx.x != 0) return;
  const unsigned long long t0 = globaltimer();
  while(ld_acquire_gpu(flag) == 0) {
    if(globaltimer() - t0 > budget_ns) {
      atomicCAS(status + ST_TIMEOUT, 0, 99);
      return;
    }
    __nanosleep(1000);
  }
}

}  // namespace

cudaError_t launch_wait_selftest(const int* flag, int* status, unsigned long long budget_ns,
                                 cudaStream_t stream) {
  wait_selftest_kernel<<<1, 32, 0, stream>>>(flag, status, budget_ns);
  return cudaGetLastError();
}

cudaError_t fp64_peak(int num_sms, int iters, double* dmma_tflops, double* dfma_tflops,
                      cudaStream_t stream) {
  double* scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, 64);
  if(e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = num_sms * 4, threads = 256;
  float     ms = 0.f;
  // Warm-up, then timed runs.
  dmma_peak_kernel<<<blocks, threads, 0, stream>>>(iters / 8 + 1, 1.0, scratch);
  cudaEventRecord(e0, stream);
  dmma_peak_kernel<<<blocks, threads, 0, stream>>>(iters, 1.0, scratch);
  cudaEventRecord(e1, stream);
  e = cudaEventSynchronize(e1);
  if(e == cudaSuccess) {
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 16 * 8 * 8 * 8.0 * iters * (double)blocks * (threads / 32);
    *dmma_tflops       = flops / (ms * 1e-3) / 1e12;
  }
  dfma_peak_kernel<<<blocks, threads, 0, stream>>>(iters / 8 + 1, 1.0, scratch);
  cudaEventRecord(e0, stream);
  dfma_peak_kernel<<<blocks, threads, 0, stream>>>(iters, 1.0, scratch);
  cudaEventRecord(e1, stream);
  if(e == cudaSuccess) e = cudaEventSynchronize(e1);
  if(e == cudaSuccess) {
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 16 * (double)iters * blocks * threads;
    *dfma_tflops       = flops / (ms * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if(e == cudaSuccess) e = cudaGetLastError();
  return e;
}

}  // namespace hplb
