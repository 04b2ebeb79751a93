// Shared host/device helpers of the PDLP library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "pdlp_b200.h"

namespace pdlp {

// Thread-local message behind pdlp_last_error().
void set_error(const std::string& msg);
const std::string& get_error();

// Kernel launches made by the library (pdlp_launch_count()).
void count_launches(long long n);

inline int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

inline int cuda_fail(cudaError_t e, const char* what) {
  return fail(PDLP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PDLP_CUDA(call)                                        \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return ::pdlp::cuda_fail(e_, #call);\
  } while (0)

// ---- device helpers ------------------------------------------------------

// Loads of data that other blocks write during the launch: L2 only, so a
// stale L1 line can never be read after a grid barrier.
__device__ __forceinline__ double ld_mut(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ld_mut(const int* p) { return __ldcg(p); }
__device__ __forceinline__ long long ld_mut(const long long* p) { return __ldcg(p); }

// Loads of data that is immutable for the whole launch.
// Gathers of a vector that was written before the last grid barrier and is
// not written again until the next one: L1-cached.  The barrier's acquire
// (ld.acquire.gpu, then bar.sync) orders those writes before these loads, so
// no stale L1 line can be returned.
__device__ __forceinline__ double ld_gather(const double* p) { return __ldca(p); }
__device__ __forceinline__ float ld_gather(const float* p) { return __ldca(p); }
__device__ __forceinline__ double ld_ro(const double* p) { return __ldg(p); }
__device__ __forceinline__ int ld_ro(const int* p) { return __ldg(p); }

// Acquire-release atomic add at GPU scope: publishes this thread's earlier
// writes (and, through a preceding bar.sync, its block's) and, for the thread
// that reads the final count, makes the other arrivers' writes visible.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// numpy.clip semantics: minimum(maximum(v, lo), hi).
__device__ __forceinline__ double clip(double v, double lo, double hi) {
  double t = v < lo ? lo : v;
  return t > hi ? hi : t;
}

// exp2(rint(log2(s))) for finite s > 0 (1.0 otherwise), computed exactly:
// with s = f * 2^e, f in [0.5, 1), log2(s) rounds down to e - 1 exactly when
// f < 2^-1/2, i.e. when f*f - 1/2 < 0, whose sign one fused multiply-add
// gives exactly (the boundary itself is irrational and never met).
__device__ __forceinline__ double pow2_round(double s) {
  if (!(s > 0.0) || !isfinite(s)) return 1.0;
  int e;
  double f = frexp(s, &e);
  int k = (fma(f, f, -0.5) < 0.0) ? e - 1 : e;
  return ldexp(1.0, k);
}

}  // namespace pdlp
