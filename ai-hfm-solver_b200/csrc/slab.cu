// Vector updates of the Z-slab conjugate-gradient solve: every slab of the decomposed grid is
// one instance (n interior cells at base + inst * stride); the CG coefficient is a ratio of two
// float64 sums that are already reduced over all slabs (and all ranks) on the device.
#include "hfm_internal.cuh"

namespace hfm {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float ratio(const double *num, const double *den) {
  if (!den) return 0.f;
  const double d = *den;
  return d != 0.0 ? (float)(*num / d) : 0.f;
}

// V = 4 moves float4 vectors (every pointer 16-byte aligned, n and stride multiples of 4).
template <int V>
__global__ void __launch_bounds__(kThreads)
    k_update_xr(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                const float *__restrict__ q, const double *__restrict__ num,
                const double *__restrict__ den, int64_t n, int64_t stride) {
  const float a = ratio(num, den);
  const int64_t off = (int64_t)blockIdx.y * stride;
  const int64_t nv = n / V;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (V == 4) {
      float4 *xv = reinterpret_cast<float4 *>(x + off) + i;
      float4 *rv = reinterpret_cast<float4 *>(r + off) + i;
      const float4 pv = __ldg(reinterpret_cast<const float4 *>(p + off) + i);
      const float4 qv = __ldg(reinterpret_cast<const float4 *>(q + off) + i);
      float4 xa = *xv, ra = *rv;
      xa.x = fmaf(a, pv.x, xa.x); xa.y = fmaf(a, pv.y, xa.y);
      xa.z = fmaf(a, pv.z, xa.z); xa.w = fmaf(a, pv.w, xa.w);
      ra.x = fmaf(-a, qv.x, ra.x); ra.y = fmaf(-a, qv.y, ra.y);
      ra.z = fmaf(-a, qv.z, ra.z); ra.w = fmaf(-a, qv.w, ra.w);
      *xv = xa;
      *rv = ra;
    } else {
      const int64_t j = off + i;
      x[j] = fmaf(a, p[j], x[j]);
      r[j] = fmaf(-a, q[j], r[j]);
    }
  }
}

template <int V>
__global__ void __launch_bounds__(kThreads)
    k_update_p(float *__restrict__ p, const float *__restrict__ z, const double *__restrict__ num,
               const double *__restrict__ den, int64_t n, int64_t stride) {
  const float b = ratio(num, den);
  const int64_t off = (int64_t)blockIdx.y * stride;
  const int64_t nv = n / V;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (V == 4) {
      float4 *pv = reinterpret_cast<float4 *>(p + off) + i;
      const float4 zv = __ldg(reinterpret_cast<const float4 *>(z + off) + i);
      float4 pa = *pv;
      // b == 0 on the first iteration, where p holds whatever the buffer held: select z
      // instead of multiplying, so a stale NaN in p cannot leak in
      if (b == 0.f) {
        pa = zv;
      } else {
        pa.x = fmaf(b, pa.x, zv.x); pa.y = fmaf(b, pa.y, zv.y);
        pa.z = fmaf(b, pa.z, zv.z); pa.w = fmaf(b, pa.w, zv.w);
      }
      *pv = pa;
    } else {
      const int64_t j = off + i;
      p[j] = b == 0.f ? z[j] : fmaf(b, p[j], z[j]);
    }
  }
}

bool aligned16(const void *ptr) { return ((uintptr_t)ptr & 15u) == 0; }

dim3 grid_for(int64_t n, int B) {
  int64_t nb = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)sm_count() * 8 / (B < 8 ? B : 8);
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  return dim3((unsigned)nb, (unsigned)B);
}

}  // namespace
}  // namespace hfm

using namespace hfm;

extern "C" int hfm_cg_update_xr(float *x, float *r, const float *p, const float *q,
                                const double *num, const double *den, int64_t n, int B,
                                int64_t stride, hfm_stream_t stream) {
  if (!x || !r || !p || !q || !num || !den || n <= 0 || B <= 0 || (B > 1 && stride < n))
    return fail(HFM_ERR_BAD_ARG, "hfm_cg_update_xr: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  const bool v4 = n % 4 == 0 && stride % 4 == 0 && aligned16(x) && aligned16(r) &&
                  aligned16(p) && aligned16(q);
  if (v4) {
    k_update_xr<4><<<grid_for(n / 4, B), kThreads, 0, s>>>(x, r, p, q, num, den, n, stride);
  } else {
    k_update_xr<1><<<grid_for(n, B), kThreads, 0, s>>>(x, r, p, q, num, den, n, stride);
  }
  HFM_CHECK_LAUNCH("k_update_xr");
  return HFM_OK;
}

extern "C" int hfm_cg_update_p(float *p, const float *z, const double *num, const double *den,
                               int64_t n, int B, int64_t stride, hfm_stream_t stream) {
  if (!p || !z || (den && !num) || n <= 0 || B <= 0 || (B > 1 && stride < n))
    return fail(HFM_ERR_BAD_ARG, "hfm_cg_update_p: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  const bool v4 = n % 4 == 0 && stride % 4 == 0 && aligned16(p) && aligned16(z);
  if (v4) {
    k_update_p<4><<<grid_for(n / 4, B), kThreads, 0, s>>>(p, z, num, den, n, stride);
  } else {
    k_update_p<1><<<grid_for(n, B), kThreads, 0, s>>>(p, z, num, den, n, stride);
  }
  HFM_CHECK_LAUNCH("k_update_p");
  return HFM_OK;
}
