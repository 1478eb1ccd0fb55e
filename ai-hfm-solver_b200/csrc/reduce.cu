// Per-instance reductions with a fixed summation order, dtype conversions.
#include <mutex>
#include <vector>

#include "hfm_internal.cuh"

namespace hfm {

// Block partial sums for hfm_norm2_f64_noalloc.  Every GPU that loads the library holds
// this array (HFM_NORM2_NOALLOC_SCRATCH_BYTES) until the process exits.
static __device__ __align__(256) double g_norm2_noalloc_scratch[HFM_NORM2_NOALLOC_SCRATCH_BYTES /
                                                                sizeof(double)];

namespace {
constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_sumsq(const T *__restrict__ x, int64_t n, int64_t stride, double *__restrict__ partials,
            const int *__restrict__ active) {
  __shared__ double sh[kThreads / 32];
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const T *xi = x + inst * stride;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v = St<T>::ld(xi + i);
    acc += v * v;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kThreads / 32 ? sh[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = v;
  }
}

// partials[inst][block] = sum of x*y over the block's cells of instance inst (float64).
__global__ void __launch_bounds__(kThreads)
    k_dot(const float *__restrict__ x, const float *__restrict__ y, int64_t n, int64_t stride,
          double *__restrict__ partials) {
  __shared__ double sh[kThreads / 32];
  const int64_t inst = blockIdx.y;
  const float *xi = x + inst * stride;
  const float *yi = y + inst * stride;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc += (double)__ldg(xi + i) * (double)__ldg(yi + i);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kThreads / 32 ? sh[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = v;
  }
}

// out[inst] = sum of partials[inst][0..nblk) in a fixed tree order.
__global__ void k_finalize_sum(const double *__restrict__ partials, int nblk,
                               double *__restrict__ out) {
  __shared__ double sh[32];
  const int64_t inst = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += partials[inst * nblk + i];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) out[inst] = v;
  }
}

__global__ void k_sqrt_inplace(double *v, int B) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B) v[i] = sqrt(v[i]);
}

__global__ void __launch_bounds__(kThreads)
    k_maxabs(const float *__restrict__ x, int64_t n, float *__restrict__ partials) {
  __shared__ float sh[kThreads / 32];
  const int64_t inst = blockIdx.y;
  const float *xi = x + inst * n;
  float m = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v = fabsf(__ldg(xi + i));
    m = (v > m || v != v) ? v : m;  // keeps NaN visible
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < kThreads / 32 ? sh[threadIdx.x] : 0.f;
    v = warp_max(v);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void k_finalize_max(const float *__restrict__ partials, int nblk,
                               float *__restrict__ out) {
  const int64_t inst = blockIdx.x;
  float m = 0.f;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    float v = partials[inst * nblk + i];
    m = (v > m || v != v) ? v : m;
  }
  m = warp_max(m);
  __shared__ float sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.f;
    v = warp_max(v);
    if (threadIdx.x == 0) out[inst] = v;
  }
}

template <class T>
__global__ void k_convert_in(const void *__restrict__ src, int src_dtype, T *__restrict__ dst,
                             int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v;
    if (src_dtype == HFM_F64) v = (float)((const double *)src)[i];
    else v = ((const float *)src)[i];
    dst[i] = St<T>::from(v);
  }
}

template <class T>
__global__ void k_convert_out(const T *__restrict__ src, float *__restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = St<T>::to(src[i]);
}

}  // namespace

int reduce_blocks_for(int64_t n) {
  int64_t b = (n + kThreads * 8 - 1) / (kThreads * 8);
  int64_t cap = (int64_t)sm_count() * 2;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

template <class T>
int launch_sumsq_partials(const T *x, int64_t n, int64_t stride, int B, double *partials,
                          int *nblk_out, const int *active, cudaStream_t s) {
  int nb = reduce_blocks_for(n);
  if (nblk_out) *nblk_out = nb;
  k_sumsq<T><<<dim3(nb, B), kThreads, 0, s>>>(x, n, stride, partials, active);
  HFM_CHECK_LAUNCH("k_sumsq");
  return HFM_OK;
}

int launch_finalize_sum(const double *partials, int nblk, int B, double *out_sum,
                        cudaStream_t s) {
  k_finalize_sum<<<B, 256, 0, s>>>(partials, nblk, out_sum);
  HFM_CHECK_LAUNCH("k_finalize_sum");
  return HFM_OK;
}

template <class T>
int launch_convert(const void *src, int src_dtype, T *dst, int64_t n, cudaStream_t s) {
  int nb = (int)((n + 255) / 256);
  if (nb > sm_count() * 8) nb = sm_count() * 8;
  if (nb < 1) nb = 1;
  k_convert_in<T><<<nb, 256, 0, s>>>(src, src_dtype, dst, n);
  HFM_CHECK_LAUNCH("k_convert_in");
  return HFM_OK;
}

template <class T>
int launch_convert_out(const T *src, float *dst, int64_t n, cudaStream_t s) {
  int nb = (int)((n + 255) / 256);
  if (nb > sm_count() * 8) nb = sm_count() * 8;
  if (nb < 1) nb = 1;
  k_convert_out<T><<<nb, 256, 0, s>>>(src, dst, n);
  HFM_CHECK_LAUNCH("k_convert_out");
  return HFM_OK;
}

#define HFM_RED_INST(T)                                                                    \
  template int launch_sumsq_partials<T>(const T *, int64_t, int64_t, int, double *, int *, \
                                        const int *, cudaStream_t);                        \
  template int launch_convert<T>(const void *, int, T *, int64_t, cudaStream_t);           \
  template int launch_convert_out<T>(const T *, float *, int64_t, cudaStream_t);
HFM_RED_INST(float)
HFM_RED_INST(__nv_bfloat16)
HFM_RED_INST(__half)

}  // namespace hfm

// ------------------------------------------------------------------------- C ABI
using namespace hfm;

// The per-instance reductions launch one grid row per instance (gridDim.y = B), so B is
// limited to the grid's y extent.
constexpr int kMaxInstances = 65535;

extern "C" size_t hfm_reduce_scratch_bytes(int64_t n, int B) {
  if (n <= 0 || B <= 0 || B > kMaxInstances) return 0;
  return (size_t)reduce_blocks_for(n) * (size_t)B * sizeof(double);
}

extern "C" int hfm_norm2_f64(const float *x, int64_t n, int B, double *out, void *scratch,
                             hfm_stream_t stream) {
  if (!x || !out || !scratch || n <= 0 || B <= 0) return fail(HFM_ERR_BAD_ARG, "hfm_norm2_f64: bad argument");
  if (B > kMaxInstances) return fail(HFM_ERR_BAD_ARG, "hfm_norm2_f64: at most 65535 instances");
  cudaStream_t s = (cudaStream_t)stream;
  int nb = 0;
  int st = launch_sumsq_partials<float>(x, n, n, B, (double *)scratch, &nb, nullptr, s);
  if (st) return st;
  if ((st = launch_finalize_sum((double *)scratch, nb, B, out, s))) return st;
  k_sqrt_inplace<<<(B + 127) / 128, 128, 0, s>>>(out, B);
  HFM_CHECK_LAUNCH("k_sqrt_inplace");
  return HFM_OK;
}

namespace {

// Device address of g_norm2_noalloc_scratch on the current device.  In host code the
// array's name only stands for the symbol, so the address is looked up with
// cudaGetSymbolAddress once per device (with that device current) and cached.
int noalloc_scratch(double **out) {
  static std::mutex mu;
  static std::vector<double *> ptrs;
  int dev = 0;
  HFM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if ((int)ptrs.size() <= dev) ptrs.resize(dev + 1, nullptr);
  if (!ptrs[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_norm2_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_status(e, "cudaGetSymbolAddress(norm2 scratch)");
    ptrs[dev] = (double *)p;
  }
  *out = ptrs[dev];
  return HFM_OK;
}

}  // namespace

// Same kernels and summation order as hfm_norm2_f64, with the block partial sums kept in
// the library's static device array instead of caller memory.
extern "C" int hfm_norm2_f64_noalloc(const float *x, int64_t n, int B, double *out,
                                     hfm_stream_t stream) {
  if (!x || !out || n <= 0 || B <= 0) return fail(HFM_ERR_BAD_ARG, "hfm_norm2_f64_noalloc: bad argument");
  if (B > kMaxInstances) return fail(HFM_ERR_BAD_ARG, "hfm_norm2_f64_noalloc: at most 65535 instances");
  const size_t need = hfm_reduce_scratch_bytes(n, B);
  if (need > HFM_NORM2_NOALLOC_SCRATCH_BYTES)
    return fail(HFM_ERR_BAD_ARG,
                "hfm_norm2_f64_noalloc: needs " + std::to_string(need) +
                    " bytes of partial sums (B x blocks x 8), more than the library's static " +
                    std::to_string((size_t)HFM_NORM2_NOALLOC_SCRATCH_BYTES) +
                    "-byte array; use hfm_norm2_f64 with caller scratch");
  double *scratch = nullptr;
  int st = noalloc_scratch(&scratch);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = 0;
  // every partial the finalize step reads is written by this call's first kernel, so the
  // array needs no clearing between calls
  if ((st = launch_sumsq_partials<float>(x, n, n, B, scratch, &nb, nullptr, s))) return st;
  if ((st = launch_finalize_sum(scratch, nb, B, out, s))) return st;
  k_sqrt_inplace<<<(B + 127) / 128, 128, 0, s>>>(out, B);
  HFM_CHECK_LAUNCH("k_sqrt_inplace");
  return HFM_OK;
}

extern "C" int hfm_dot_f64(const float *x, const float *y, int64_t n, int B, int64_t stride,
                           double *out, void *scratch, hfm_stream_t stream) {
  if (!x || !y || !out || !scratch || n <= 0 || B <= 0 || (B > 1 && stride < n))
    return fail(HFM_ERR_BAD_ARG, "hfm_dot_f64: bad argument");
  if (B > kMaxInstances) return fail(HFM_ERR_BAD_ARG, "hfm_dot_f64: at most 65535 instances");
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = reduce_blocks_for(n);
  k_dot<<<dim3(nb, B), kThreads, 0, s>>>(x, y, n, stride, (double *)scratch);
  HFM_CHECK_LAUNCH("k_dot");
  return launch_finalize_sum((double *)scratch, nb, B, out, s);
}

extern "C" int hfm_max_abs(const float *x, int64_t n, int B, float *out, void *scratch,
                           hfm_stream_t stream) {
  if (!x || !out || !scratch || n <= 0 || B <= 0) return fail(HFM_ERR_BAD_ARG, "hfm_max_abs: bad argument");
  if (B > kMaxInstances) return fail(HFM_ERR_BAD_ARG, "hfm_max_abs: at most 65535 instances");
  cudaStream_t s = (cudaStream_t)stream;
  int nb = reduce_blocks_for(n);
  k_maxabs<<<dim3(nb, B), kThreads, 0, s>>>(x, n, (float *)scratch);
  HFM_CHECK_LAUNCH("k_maxabs");
  k_finalize_max<<<B, 256, 0, s>>>((float *)scratch, nb, out);
  HFM_CHECK_LAUNCH("k_finalize_max");
  return HFM_OK;
}
