// Arithmetic-throughput probe of this GPU's CUDA cores: the compute ceiling
// that the particle kernel's floating-point work is measured against (the
// particle step of shape order 3 does ~1.5 kflop per particle, more than the
// HBM traffic of its ~60 bytes can keep up with).
#include "pxr_common.cuh"

namespace {

constexpr int PROBE_CHAINS = 8;   // independent FMA chains per thread

typedef unsigned long long f2r;

__device__ __forceinline__ f2r pfma(f2r a, f2r b, f2r c) {
  f2r d;
  asm volatile("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// kind 0: FP32 fma; 1: packed f32x2 fma (two FP32 FMAs per instruction);
// 2: FP64 fma.  Each thread runs PROBE_CHAINS chains a <- a*b + c for `iters`
// rounds and writes the sum of its chains to sink[thread].
template <int KIND>
__global__ void k_fma_probe(float* __restrict__ sink, int iters, float b, float c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float out = 0.f;
  if (KIND == 0) {
    float a[PROBE_CHAINS];
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) a[i] = (float)i;
    for (int r = 0; r < iters; ++r) {
#pragma unroll
      for (int i = 0; i < PROBE_CHAINS; ++i) a[i] = fmaf(a[i], b, c);
    }
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) out += a[i];
  } else if (KIND == 1) {
    f2r a[PROBE_CHAINS], bb, cc;
    asm("mov.b64 %0, {%1, %1};" : "=l"(bb) : "f"(b));
    asm("mov.b64 %0, {%1, %1};" : "=l"(cc) : "f"(c));
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) {
      const float lo = (float)(2 * i), hi = (float)(2 * i + 1);
      asm("mov.b64 %0, {%1, %2};" : "=l"(a[i]) : "f"(lo), "f"(hi));
    }
    for (int r = 0; r < iters; ++r) {
#pragma unroll
      for (int i = 0; i < PROBE_CHAINS; ++i) a[i] = pfma(a[i], bb, cc);
    }
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) {
      float lo, hi;
      asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[i]));
      out += lo + hi;
    }
  } else {
    double a[PROBE_CHAINS];
    const double bd = b, cd = c;
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) a[i] = (double)i;
    for (int r = 0; r < iters; ++r) {
#pragma unroll
      for (int i = 0; i < PROBE_CHAINS; ++i) a[i] = fma(a[i], bd, cd);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; ++i) s += a[i];
    out = (float)s;
  }
  sink[t] = out;
}

}  // namespace

extern "C" {

int64_t pxrb_fma_probe_flops(int32_t kind, int32_t blocks, int32_t threads, int32_t iters) {
  if (kind < 0 || kind > 2 || blocks < 1 || threads < 1 || iters < 0) return -1;
  return (int64_t)blocks * threads * iters * PROBE_CHAINS * 2 * (kind == 1 ? 2 : 1);
}

int pxrb_fma_probe(int32_t kind, int32_t blocks, int32_t threads, int32_t iters, float b,
                   float c, float* sink, void* stream) {
  if (!sink || blocks < 1 || threads < 32 || threads > 1024 || threads % 32 || iters < 0)
    return PXRB_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  if (kind == 0) k_fma_probe<0><<<blocks, threads, 0, s>>>(sink, iters, b, c);
  else if (kind == 1) k_fma_probe<1><<<blocks, threads, 0, s>>>(sink, iters, b, c);
  else if (kind == 2) k_fma_probe<2><<<blocks, threads, 0, s>>>(sink, iters, b, c);
  else return PXRB_EINVAL;
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"
