// Generic stencil / transfer kernels: one thread per output cell, any grid extent.
//
// These kernels serve every extent (odd sizes, the 1^3 / 2^3 / 5x1x1 coarse levels of the
// reference cycles, X not a multiple of 4).  Fine levels with X % 4 == 0 are served by the
// plane-marching kernels in ops_fast.cu.
#include "hfm_internal.cuh"

namespace hfm {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

int blocks_for(int64_t n, int B) {
  // Enough blocks per instance to fill the GPU about four times over, capped by the work.
  int64_t want = (int64_t)sm_count() * 8 / (B > 0 ? B : 1);
  if (want < 1) want = 1;
  int64_t need = (n + kThreads - 1) / kThreads;
  int64_t b = need < want ? need : want;
  return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

template <int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    k_smooth(DevOp op, PhiSrc<T> phi, const T *__restrict__ rhs, int64_t rhs_stride,
             T *__restrict__ out, int64_t out_stride, int Z, int Y, int X, float omega,
             unsigned flags, const int *__restrict__ active, double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int64_t n = (int64_t)Z * Y * X;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % X);
    int64_t t = i / X;
    int y = (int)(t % Y);
    int z = (int)(t / Y);
    // boundary_condition_top: plane 0 receives the smoothed value of plane 1.
    if ((flags & HFM_FLAG_TOP_COPY) && z == 0 && Z > 1) z = 1;
    float diag;
    float ax = op_apply_at<KIND, T>(op, phi, inst, z, y, x, Z, Y, X, &diag);
    float pc = phi(inst, z, y, x, Y, X);
    float f = rhs ? St<T>::ld(rhs + inst * rhs_stride + ((int64_t)z * Y + y) * X + x) : 0.f;
    const float v = pc + omega * (f - ax) / diag;
    out[inst * out_stride + i] = St<T>::from(v);
    acc += (double)v * f;
  }
  if (partials) {
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = acc;
  }
}

template <int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    k_residual(DevOp op, PhiSrc<T> phi, const T *__restrict__ b, int64_t b_stride,
               T *__restrict__ r, int64_t r_stride, int Z, int Y, int X, unsigned flags,
               const int *__restrict__ active, double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int64_t n = (int64_t)Z * Y * X;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % X);
    int64_t t = i / X;
    int y = (int)(t % Y);
    int z = (int)(t / Y);
    float diag;
    float v = op_apply_at<KIND, T>(op, phi, inst, z, y, x, Z, Y, X, &diag);
    if (b) v -= St<T>::ld(b + inst * b_stride + i);
    if ((flags & HFM_FLAG_ZERO_XEND) && x == X - 1) v = 0.f;
    if (r) r[inst * r_stride + i] = St<T>::from(v);
    acc += (double)v * (double)((flags & HFM_INT_DOT_PHI) ? phi(inst, z, y, x, Y, X) : v);
  }
  if (partials) {
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = acc;
  }
}

// One thread per coarse cell: residual of its 2x2x2 fine block, averaged.
template <int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    k_residual_restrict(DevOp op, PhiSrc<T> phi, const T *__restrict__ b, int64_t b_stride,
                        T *__restrict__ rf, int64_t rf_stride, T *__restrict__ rc,
                        int64_t rc_stride, int Z, int Y, int X, unsigned flags,
                        const int *__restrict__ active, double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int Zc = Z >> 1, Yc = Y >> 1, Xc = X >> 1;
  const int64_t nc = (int64_t)Zc * Yc * Xc;
  double acc = 0.0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nc;
       j += (int64_t)gridDim.x * blockDim.x) {
    int xc = (int)(j % Xc);
    int64_t t = j / Xc;
    int yc = (int)(t % Yc);
    int zc = (int)(t / Yc);
    float sum = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          int z = 2 * zc + a, y = 2 * yc + bb, x = 2 * xc + c;
          int64_t i = ((int64_t)z * Y + y) * X + x;
          float diag;
          float v = op_apply_at<KIND, T>(op, phi, inst, z, y, x, Z, Y, X, &diag);
          if (b) v -= St<T>::ld(b + inst * b_stride + i);
          if ((flags & HFM_FLAG_ZERO_XEND) && x == X - 1) v = 0.f;
          if (rf) rf[inst * rf_stride + i] = St<T>::from(v);
          acc += (double)v * (double)v;
          sum += 0.125f * v;
        }
    rc[inst * rc_stride + j] = St<T>::from(sum);
  }
  if (partials) {
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[inst * gridDim.x + blockIdx.x] = acc;
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_restrict(const T *__restrict__ f, int64_t fs, T *__restrict__ c, int64_t cs, int Z, int Y,
               int X, const int *__restrict__ active) {
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int Zc = Z >> 1, Yc = Y >> 1, Xc = X >> 1;
  const int64_t nc = (int64_t)Zc * Yc * Xc;
  const T *fi = f + inst * fs;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nc;
       j += (int64_t)gridDim.x * blockDim.x) {
    int xc = (int)(j % Xc);
    int64_t t = j / Xc;
    int yc = (int)(t % Yc);
    int zc = (int)(t / Yc);
    float sum = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
          sum += 0.125f * St<T>::ld(fi + ((int64_t)(2 * zc + a) * Y + 2 * yc + bb) * X + 2 * xc + cc);
    c[inst * cs + j] = St<T>::from(sum);
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_prolong(const T *__restrict__ c, int64_t cs, T *__restrict__ f, int64_t fs, int Zc,
              int Yc, int Xc, const int *__restrict__ active) {
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int Y = 2 * Yc, X = 2 * Xc;
  const int64_t n = (int64_t)8 * Zc * Yc * Xc;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % X);
    int64_t t = i / X;
    int y = (int)(t % Y);
    int z = (int)(t / Y);
    f[inst * fs + i] = c[inst * cs + ((int64_t)(z >> 1) * Yc + (y >> 1)) * Xc + (x >> 1)];
  }
}

// The same transfers with 16-byte accesses for rows of a multiple of VEC = 16 / sizeof(T)
// fine values (16-byte aligned fine pointer and stride, 8-byte aligned coarse ones): a thread
// owns HC = VEC / 2 consecutive coarse cells of one coarse row.  Restriction loads VEC fine
// values from each of its four fine rows (two y, two z) and sums in the order of k_restrict
// (z, then y, then x), so both give the same bits; prolongation loads HC coarse values and
// stores VEC fine values into each of the four rows.
template <class T> struct Vec16 {
  static constexpr int VEC = 16 / (int)sizeof(T), HC = VEC / 2;
  static __device__ __forceinline__ void ld(const T *p, float (&v)[VEC]) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    if constexpr (sizeof(T) == 4) {
      v[0] = __uint_as_float(u.x); v[1] = __uint_as_float(u.y);
      v[2] = __uint_as_float(u.z); v[3] = __uint_as_float(u.w);
    } else {
      const T *h = reinterpret_cast<const T *>(&u);
#pragma unroll
      for (int k = 0; k < VEC; ++k) v[k] = St<T>::to(h[k]);
    }
  }
};

// One instance's vector restriction, the block's share of the grid-stride loop.
template <class T>
__device__ __forceinline__ void restrict_v_instance(const T *__restrict__ fi, T *__restrict__ ci,
                                                    int Z, int Y, int X) {
  constexpr int VEC = Vec16<T>::VEC, HC = Vec16<T>::HC;
  const int Zc = Z >> 1, Yc = Y >> 1, Xc = X >> 1, Xv = Xc / HC;
  const int64_t nv = (int64_t)Zc * Yc * Xv;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nv;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int xv = (int)(j % Xv);
    const int64_t t = j / Xv;
    const int yc = (int)(t % Yc), zc = (int)(t / Yc);
    float sum[HC];
#pragma unroll
    for (int k = 0; k < HC; ++k) sum[k] = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        float v[VEC];
        Vec16<T>::ld(fi + ((int64_t)(2 * zc + a) * Y + 2 * yc + bb) * X + (int64_t)VEC * xv, v);
#pragma unroll
        for (int k = 0; k < HC; ++k) {
          sum[k] += 0.125f * v[2 * k];
          sum[k] += 0.125f * v[2 * k + 1];
        }
      }
    alignas(8) T out[HC];
#pragma unroll
    for (int k = 0; k < HC; ++k) out[k] = St<T>::from(sum[k]);
    *reinterpret_cast<uint2 *>(ci + ((int64_t)zc * Yc + yc) * Xc + (int64_t)HC * xv) =
        *reinterpret_cast<const uint2 *>(out);
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_restrict_v(const T *__restrict__ f, int64_t fs, T *__restrict__ c, int64_t cs, int Z, int Y,
                 int X, const int *__restrict__ active) {
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  restrict_v_instance<T>(f + inst * fs, c + inst * cs, Z, Y, X);
}

// Three arrays of the same shape restricted in one launch (blockIdx.z picks the array): the
// conductivity hierarchy of a slot.
template <class T> struct Arr3 {
  const T *f[3];
  T *c[3];
};
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_restrict3_v(Arr3<T> a, int64_t fs, int64_t cs, int Z, int Y, int X) {
  const int64_t inst = blockIdx.y;
  restrict_v_instance<T>(a.f[blockIdx.z] + inst * fs, a.c[blockIdx.z] + inst * cs, Z, Y, X);
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_prolong_v(const T *__restrict__ c, int64_t cs, T *__restrict__ f, int64_t fs, int Zc,
                int Yc, int Xc, const int *__restrict__ active) {
  constexpr int VEC = Vec16<T>::VEC, HC = Vec16<T>::HC;
  const int64_t inst = blockIdx.y;
  if (active && !active[inst]) return;
  const int Y = 2 * Yc, X = 2 * Xc, Xv = Xc / HC;
  const int64_t nv = (int64_t)Zc * Yc * Xv;
  const T *ci = c + inst * cs;
  T *fi = f + inst * fs;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nv;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int xv = (int)(j % Xv);
    const int64_t t = j / Xv;
    const int yc = (int)(t % Yc), zc = (int)(t / Yc);
    const uint2 u = *reinterpret_cast<const uint2 *>(ci + ((int64_t)zc * Yc + yc) * Xc + (int64_t)HC * xv);
    const T *h = reinterpret_cast<const T *>(&u);
    alignas(16) T w[VEC];
#pragma unroll
    for (int k = 0; k < VEC; ++k) w[k] = h[k >> 1];
    const uint4 o = *reinterpret_cast<const uint4 *>(w);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
        *reinterpret_cast<uint4 *>(fi + ((int64_t)(2 * zc + a) * Y + 2 * yc + bb) * X + (int64_t)VEC * xv) = o;
  }
}

// The vector transfers apply: X (fine) a multiple of VEC, fine pointer and instance stride
// 16-byte aligned, coarse ones 8-byte aligned.
template <class T>
bool transfer_vec_ok(const T *fine, int64_t f_stride, const T *coarse, int64_t c_stride, int X, int B) {
  constexpr int VEC = Vec16<T>::VEC;
  const int64_t es = (int64_t)sizeof(T);
  if (X % VEC) return false;
  if ((uintptr_t)fine % 16 || (uintptr_t)coarse % 8) return false;
  if (B > 1 && ((f_stride * es) % 16 || (c_stride * es) % 8)) return false;
  return true;
}

// Small-grid Jacobi: the level lives in shared memory, one block per instance.
template <int KIND, class T>
__global__ void k_coarse_jacobi(DevOp op, const T *__restrict__ rhs, int64_t rhs_stride,
                                const T *__restrict__ phi0, T *__restrict__ out,
                                int64_t stride, int Z, int Y, int X, float omega, int sweeps,
                                const int *__restrict__ active) {
  extern __shared__ float sm[];
  const int64_t inst = blockIdx.x;
  if (active && !active[inst]) return;
  const int n = Z * Y * X;
  float *a = sm, *bnew = sm + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    a[i] = phi0 ? St<T>::ld(phi0 + inst * stride + i) : 0.f;
  __syncthreads();
  struct SmemPhi {
    const float *p;
    __device__ float operator()(int64_t, int z, int y, int x, int Y, int X) const {
      return p[(z * Y + y) * X + x];
    }
  };
  for (int s = 0; s < sweeps; ++s) {
    SmemPhi ph{a};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int x = i % X, y = (i / X) % Y, z = i / (X * Y);
      float diag;
      float ax = op_apply_at<KIND, T>(op, ph, inst, z, y, x, Z, Y, X, &diag);
      float f = St<T>::ld(rhs + inst * rhs_stride + i);
      bnew[i] = a[i] + omega * (f - ax) / diag;
    }
    __syncthreads();
    float *tmp = a;
    a = bnew;
    bnew = tmp;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[inst * stride + i] = St<T>::from(a[i]);
}

}  // namespace

int coarse_smem_limit() { return 4096; }

int64_t max_partial_blocks(Grid3 g, int B) {
  // generic kernels: blocks_for() <= 8 per SM; fast kernels: plane tiles x z chunks
  const int64_t tiles = ((int64_t)g.Y * (g.X / 4) + 255) / 256 + 1;
  const int64_t chunks = (g.Z + 3) / 4 + 1;
  int64_t v = tiles * chunks;
  const int64_t tma_tiles = ((int64_t)(g.X + 63) / 64) * ((g.Y + 7) / 8);
  if (tma_tiles * chunks > v) v = tma_tiles * chunks;
  int64_t gen = (int64_t)sm_count() * 8;
  return v > gen ? v : gen;
}

#define HFM_DISPATCH_KIND(kind, ...)                                          \
  switch (kind) {                                                             \
    case HFM_OP_CONST7: { constexpr int K_ = HFM_OP_CONST7; __VA_ARGS__; break; } \
    case HFM_OP_SIGMA7: { constexpr int K_ = HFM_OP_SIGMA7; __VA_ARGS__; break; } \
    case HFM_OP_DIR7: { constexpr int K_ = HFM_OP_DIR7; __VA_ARGS__; break; }     \
    case HFM_OP_K27: { constexpr int K_ = HFM_OP_K27; __VA_ARGS__; break; }       \
    case HFM_OP_FACE7: { constexpr int K_ = HFM_OP_FACE7; __VA_ARGS__; break; }   \
    default: return fail(HFM_ERR_BAD_ARG, "unknown operator kind");          \
  }

template <class T>
int launch_smooth(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                  int64_t rhs_stride, T *out, int64_t out_stride, int B, Grid3 g, float omega,
                  unsigned flags, const int *active, cudaStream_t s, double *partials,
                  int *nblk_out) {
  if (!(flags & HFM_INT_DOT_RHS)) partials = nullptr;
  if ((!phi.base || phi.base_stride == out_stride) && (phi.base || phi.corr || rhs) &&
      (!rhs || rhs_stride == out_stride) &&
      tma_eligible(kind, g, FAST_SMOOTH, phi.corr, phi.corr_coarse, (int)sizeof(T)) &&
      face_tma_ok<T>(kind, phi, flags) &&
      vec_aligned<T>(kind, op, phi, rhs, out, nullptr, out_stride, 16))
    return tma_launch<T>(kind, FAST_SMOOTH, op, phi, rhs, out, nullptr, out_stride, 0, B, g,
                         omega, flags, active, partials, nblk_out, s);
  if (fast_eligible(kind, g, false) && (!rhs || rhs_stride == out_stride) &&
      (!phi.base || phi.base_stride == out_stride) && (!phi.corr || phi.corr_coarse || phi.corr_stride == out_stride) &&
      vec_aligned<T>(kind, op, phi, rhs, out, nullptr, out_stride, 4 * (int64_t)sizeof(T)))
    return fast_launch<T>(kind, FAST_SMOOTH, op, phi, rhs, out, nullptr, out_stride, 0, B, g,
                          omega, flags, active, partials, nblk_out, s);
  const int nb = blocks_for(g.n(), B);
  if (nblk_out) *nblk_out = nb;
  dim3 grid(nb, B);
  HFM_DISPATCH_KIND(kind, (k_smooth<K_, T><<<grid, kThreads, 0, s>>>(
                              op, phi, rhs, rhs_stride, out, out_stride, g.Z, g.Y, g.X, omega,
                              flags, active, partials)));
  HFM_CHECK_LAUNCH("k_smooth");
  return HFM_OK;
}

template <class T>
int launch_residual(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *b,
                    int64_t b_stride, T *r, int64_t r_stride, int B, Grid3 g, unsigned flags,
                    const int *active, double *partials, int *nblk_out, cudaStream_t s) {
  if (phi.base && !phi.corr && !phi.zero_xend && r && phi.base_stride == r_stride &&
      (!b || b_stride == r_stride) && tma_eligible(kind, g, FAST_RESID, nullptr, 0, (int)sizeof(T)) &&
      face_tma_ok<T>(kind, phi, flags) &&
      vec_aligned<T>(kind, op, phi, b, r, nullptr, r_stride, 16))
    return tma_launch<T>(kind, FAST_RESID, op, phi, b, r, nullptr, r_stride, 0, B, g, 0.f,
                         flags, active, partials, nblk_out, s);
  if (fast_eligible(kind, g, false) && !phi.corr && !phi.zero_xend && r &&
      (!b || b_stride == r_stride) && (!phi.base || phi.base_stride == r_stride) &&
      vec_aligned<T>(kind, op, phi, b, r, nullptr, r_stride, 4 * (int64_t)sizeof(T)))
    return fast_launch<T>(kind, FAST_RESID, op, phi, b, r, nullptr, r_stride, 0, B, g, 0.f,
                          flags, active, partials, nblk_out, s);
  int nb = blocks_for(g.n(), B);
  if (nblk_out) *nblk_out = nb;
  dim3 grid(nb, B);
  HFM_DISPATCH_KIND(kind, (k_residual<K_, T><<<grid, kThreads, 0, s>>>(
                              op, phi, b, b_stride, r, r_stride, g.Z, g.Y, g.X, flags, active,
                              partials)));
  HFM_CHECK_LAUNCH("k_residual");
  return HFM_OK;
}

template <class T>
int launch_apply(int kind, const DevOp &op, const PhiSrc<T> &phi, T *out, int64_t out_stride,
                 int B, Grid3 g, const int *active, cudaStream_t s) {
  return launch_residual<T>(kind, op, phi, nullptr, 0, out, out_stride, B, g, 0u, active,
                            nullptr, nullptr, s);
}

template <class T>
int launch_residual_restrict(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *b,
                             int64_t b_stride, T *r_fine, int64_t rf_stride, T *r_coarse,
                             int64_t rc_stride, int B, Grid3 g, unsigned flags,
                             const int *active, double *partials, int *nblk_out,
                             cudaStream_t s) {
  if ((g.Z | g.Y | g.X) & 1) return fail(HFM_ERR_BAD_ARG, "residual_restrict needs even extents");
  if (phi.base && !phi.corr && !phi.zero_xend && b && phi.base_stride == b_stride &&
      (!r_fine || rf_stride == b_stride) && rc_stride == b_stride / 8 &&
      tma_eligible(kind, g, FAST_RESTRICT, nullptr, 0, (int)sizeof(T)) &&
      face_tma_ok<T>(kind, phi, flags) &&
      vec_aligned<T>(kind, op, phi, b, r_fine, nullptr, b_stride, 16))
    return tma_launch<T>(kind, FAST_RESTRICT, op, phi, b, r_fine, r_coarse, b_stride, rc_stride,
                         B, g, 0.f, flags, active, partials, nblk_out, s);
  if (fast_eligible(kind, g, true) && !phi.corr && !phi.zero_xend && b &&
      (!r_fine || rf_stride == b_stride) && (!phi.base || phi.base_stride == b_stride) &&
      rc_stride == b_stride / 8 &&
      vec_aligned<T>(kind, op, phi, b, r_fine, r_coarse, b_stride, 4 * (int64_t)sizeof(T)))
    return fast_launch<T>(kind, FAST_RESTRICT, op, phi, b, r_fine, r_coarse, b_stride, rc_stride,
                          B, g, 0.f, flags, active, partials, nblk_out, s);
  int64_t nc = g.n() / 8;
  int nb = blocks_for(nc, B);
  if (nblk_out) *nblk_out = nb;
  dim3 grid(nb, B);
  HFM_DISPATCH_KIND(kind, (k_residual_restrict<K_, T><<<grid, kThreads, 0, s>>>(
                              op, phi, b, b_stride, r_fine, rf_stride, r_coarse, rc_stride,
                              g.Z, g.Y, g.X, flags, active, partials)));
  HFM_CHECK_LAUNCH("k_residual_restrict");
  return HFM_OK;
}

template <class T>
int launch_restrict(const T *fine, int64_t f_stride, T *coarse, int64_t c_stride, int B,
                    Grid3 g, const int *active, cudaStream_t s) {
  int64_t nc = (int64_t)(g.Z / 2) * (g.Y / 2) * (g.X / 2);
  if (nc == 0) return HFM_OK;
  if (transfer_vec_ok<T>(fine, f_stride, coarse, c_stride, g.X, B)) {
    dim3 grid(blocks_for(nc / Vec16<T>::HC, B), B);
    k_restrict_v<T><<<grid, kThreads, 0, s>>>(fine, f_stride, coarse, c_stride, g.Z, g.Y, g.X,
                                              active);
    HFM_CHECK_LAUNCH("k_restrict_v");
    return HFM_OK;
  }
  dim3 grid(blocks_for(nc, B), B);
  k_restrict<T><<<grid, kThreads, 0, s>>>(fine, f_stride, coarse, c_stride, g.Z, g.Y, g.X,
                                          active);
  HFM_CHECK_LAUNCH("k_restrict");
  return HFM_OK;
}

template <class T>
int launch_restrict3(const T *const fine[3], int64_t f_stride, T *const coarse[3], int64_t c_stride,
                     int B, Grid3 g, cudaStream_t s) {
  const int64_t nc = (int64_t)(g.Z / 2) * (g.Y / 2) * (g.X / 2);
  if (nc == 0) return HFM_OK;
  bool vec = true;
  for (int a = 0; a < 3; ++a) vec = vec && transfer_vec_ok<T>(fine[a], f_stride, coarse[a], c_stride, g.X, B);
  if (!vec) {
    for (int a = 0; a < 3; ++a) {
      int st = launch_restrict<T>(fine[a], f_stride, coarse[a], c_stride, B, g, nullptr, s);
      if (st) return st;
    }
    return HFM_OK;
  }
  Arr3<T> arr;
  for (int a = 0; a < 3; ++a) {
    arr.f[a] = fine[a];
    arr.c[a] = coarse[a];
  }
  dim3 grid(blocks_for(nc / Vec16<T>::HC, B * 3), B, 3);
  k_restrict3_v<T><<<grid, kThreads, 0, s>>>(arr, f_stride, c_stride, g.Z, g.Y, g.X);
  HFM_CHECK_LAUNCH("k_restrict3_v");
  return HFM_OK;
}

template <class T>
int launch_prolong(const T *coarse, int64_t c_stride, T *fine, int64_t f_stride, int B,
                   Grid3 gc, const int *active, cudaStream_t s) {
  if (transfer_vec_ok<T>(fine, f_stride, coarse, c_stride, 2 * gc.X, B)) {
    dim3 grid(blocks_for(gc.n() / Vec16<T>::HC, B), B);
    k_prolong_v<T><<<grid, kThreads, 0, s>>>(coarse, c_stride, fine, f_stride, gc.Z, gc.Y,
                                             gc.X, active);
    HFM_CHECK_LAUNCH("k_prolong_v");
    return HFM_OK;
  }
  dim3 grid(blocks_for(gc.n() * 8, B), B);
  k_prolong<T><<<grid, kThreads, 0, s>>>(coarse, c_stride, fine, f_stride, gc.Z, gc.Y, gc.X,
                                         active);
  HFM_CHECK_LAUNCH("k_prolong");
  return HFM_OK;
}

template <class T>
int launch_coarse_jacobi(int kind, const DevOp &op, const T *rhs, int64_t rhs_stride,
                         const T *phi0, T *out, int64_t stride, int B, Grid3 g, float omega,
                         int sweeps, const int *active, cudaStream_t s) {
  int n = (int)g.n();
  if (n > coarse_smem_limit()) return fail(HFM_ERR_BAD_ARG, "coarsest level too large for in-block solve");
  size_t smem = (size_t)2 * n * sizeof(float);
  int threads = n < 256 ? ((n + 31) / 32) * 32 : 256;
  HFM_DISPATCH_KIND(kind, (k_coarse_jacobi<K_, T><<<B, threads, smem, s>>>(
                              op, rhs, rhs_stride, phi0, out, stride, g.Z, g.Y, g.X, omega,
                              sweeps, active)));
  HFM_CHECK_LAUNCH("k_coarse_jacobi");
  return HFM_OK;
}

#define HFM_INST(T)                                                                         \
  template int launch_smooth<T>(int, const DevOp &, const PhiSrc<T> &, const T *, int64_t,  \
                                T *, int64_t, int, Grid3, float, unsigned, const int *,     \
                                cudaStream_t, double *, int *);                             \
  template int launch_residual<T>(int, const DevOp &, const PhiSrc<T> &, const T *,         \
                                  int64_t, T *, int64_t, int, Grid3, unsigned, const int *, \
                                  double *, int *, cudaStream_t);                           \
  template int launch_apply<T>(int, const DevOp &, const PhiSrc<T> &, T *, int64_t, int,    \
                               Grid3, const int *, cudaStream_t);                           \
  template int launch_residual_restrict<T>(int, const DevOp &, const PhiSrc<T> &, const T *, \
                                           int64_t, T *, int64_t, T *, int64_t, int, Grid3,  \
                                           unsigned, const int *, double *, int *,           \
                                           cudaStream_t);                                    \
  template int launch_restrict3<T>(const T *const[3], int64_t, T *const[3], int64_t, int, Grid3,   \
                                   cudaStream_t);                                           \
  template int launch_restrict<T>(const T *, int64_t, T *, int64_t, int, Grid3, const int *, \
                                  cudaStream_t);                                             \
  template int launch_prolong<T>(const T *, int64_t, T *, int64_t, int, Grid3, const int *,  \
                                 cudaStream_t);                                              \
  template int launch_coarse_jacobi<T>(int, const DevOp &, const T *, int64_t, const T *,    \
                                       T *, int64_t, int, Grid3, float, int, const int *,    \
                                       cudaStream_t);

HFM_INST(float)
HFM_INST(__nv_bfloat16)
HFM_INST(__half)

}  // namespace hfm
