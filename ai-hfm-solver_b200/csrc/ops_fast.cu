// Plane-marching stencil kernels for grids with X % 4 == 0 (the fine and most coarse
// levels).  Layout and semantics are those of ops_generic.cu; these kernels differ only in
// how they move data:
//   * a thread owns 4 consecutive x (one 16-byte float32 / 8-byte 16-bit load) on R rows and
//     marches along z through a chunk of planes, so z neighbours, the z-face coefficient and
//     27-point partial sums stay in registers;
//   * x neighbours come from the adjacent lanes by warp shuffle (lanes hold consecutive
//     vectors of the flattened (row, x-vector) index); only lanes 0 / 31 load them;
//   * y neighbours are vector loads served mostly by L1 (the rows belong to the same block).
// Modes: SMOOTH (weighted Jacobi), RESID (A phi - b, optional norm partials), RESTRICT
// (residual of R = 2 rows x 2 planes x 2 columns averaged into the coarse grid).
#include <map>
#include <mutex>

#include "hfm_internal.cuh"

namespace hfm {

namespace {

constexpr int kFastThreads = 256;

enum { M_SMOOTH = FAST_SMOOTH, M_RESID = FAST_RESID, M_RESTRICT = FAST_RESTRICT };
enum { C_NONE = 0, C_COARSE = 1, C_SAME = 2 };

struct F4 {
  float v[4];
};

template <class T> __device__ __forceinline__ F4 ld4(const T *p);
template <> __device__ __forceinline__ F4 ld4<float>(const float *p) {
  float4 a = __ldg(reinterpret_cast<const float4 *>(p));
  return F4{{a.x, a.y, a.z, a.w}};
}
template <> __device__ __forceinline__ F4 ld4<__nv_bfloat16>(const __nv_bfloat16 *p) {
  uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
  __nv_bfloat162 a = *reinterpret_cast<__nv_bfloat162 *>(&u.x);
  __nv_bfloat162 b = *reinterpret_cast<__nv_bfloat162 *>(&u.y);
  float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
  return F4{{fa.x, fa.y, fb.x, fb.y}};
}
template <> __device__ __forceinline__ F4 ld4<__half>(const __half *p) {
  uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
  __half2 a = *reinterpret_cast<__half2 *>(&u.x);
  __half2 b = *reinterpret_cast<__half2 *>(&u.y);
  float2 fa = __half22float2(a), fb = __half22float2(b);
  return F4{{fa.x, fa.y, fb.x, fb.y}};
}

template <class T> __device__ __forceinline__ float2 ld2(const T *p);
template <> __device__ __forceinline__ float2 ld2<float>(const float *p) {
  return __ldg(reinterpret_cast<const float2 *>(p));
}
template <> __device__ __forceinline__ float2 ld2<__nv_bfloat16>(const __nv_bfloat16 *p) {
  unsigned u = __ldg(reinterpret_cast<const unsigned *>(p));
  return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&u));
}
template <> __device__ __forceinline__ float2 ld2<__half>(const __half *p) {
  unsigned u = __ldg(reinterpret_cast<const unsigned *>(p));
  return __half22float2(*reinterpret_cast<__half2 *>(&u));
}

template <class T> __device__ __forceinline__ void st4(T *p, const F4 &v);
template <> __device__ __forceinline__ void st4<float>(float *p, const F4 &v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
template <> __device__ __forceinline__ void st4<__nv_bfloat16>(__nv_bfloat16 *p, const F4 &v) {
  __nv_bfloat162 a = __floats2bfloat162_rn(v.v[0], v.v[1]);
  __nv_bfloat162 b = __floats2bfloat162_rn(v.v[2], v.v[3]);
  uint2 u;
  u.x = *reinterpret_cast<unsigned *>(&a);
  u.y = *reinterpret_cast<unsigned *>(&b);
  *reinterpret_cast<uint2 *>(p) = u;
}
template <> __device__ __forceinline__ void st4<__half>(__half *p, const F4 &v) {
  __half2 a = __floats2half2_rn(fminf(fmaxf(v.v[0], -65504.f), 65504.f), fminf(fmaxf(v.v[1], -65504.f), 65504.f));
  __half2 b = __floats2half2_rn(fminf(fmaxf(v.v[2], -65504.f), 65504.f), fminf(fmaxf(v.v[3], -65504.f), 65504.f));
  uint2 u;
  u.x = *reinterpret_cast<unsigned *>(&a);
  u.y = *reinterpret_cast<unsigned *>(&b);
  *reinterpret_cast<uint2 *>(p) = u;
}

template <class T> struct FastArgs {
  DevOp op;
  const T *base;      // phi (nullable = zero)
  const T *corr;      // correction (nullable)
  const T *rhs;       // b / f (nullable = zero)
  T *out;             // smoothed phi / residual (nullable in RESTRICT mode)
  T *coarse;          // RESTRICT output
  double *partials;   // [inst][blocks] squared-residual partial sums (nullable)
  const int *active;
  int64_t stride, corr_stride, coarse_stride;
  int Z, Y, X, zc;    // extents, planes per z-chunk
  float omega, corr_sign;
  int zero_xend;      // input: phi' = 0 on x = X-1 (NS correction before the sweep)
  int zero_xend_out;  // output: residual = 0 on x = X-1 (NS residual)
  int top_copy;
  int dot_phi;        // partials of res * phi instead of res^2 (RESID)
  int dot_rhs;        // partials of out * rhs (SMOOTH)
};

template <class T, int CORR>
__device__ __forceinline__ float phi_scalar(const FastArgs<T> &a, int64_t ib, int64_t ic, int z,
                                            int y, int x) {
  float v = a.base ? St<T>::ld(a.base + ib + ((int64_t)z * a.Y + y) * a.X + x) : 0.f;
  if (CORR == C_COARSE)
    v += a.corr_sign *
         St<T>::ld(a.corr + ic + ((int64_t)(z >> 1) * (a.Y >> 1) + (y >> 1)) * (a.X >> 1) + (x >> 1));
  else if (CORR == C_SAME)
    v += a.corr_sign * St<T>::ld(a.corr + ic + ((int64_t)z * a.Y + y) * a.X + x);
  if (a.zero_xend && x == a.X - 1) v = 0.f;
  return v;
}

// Load phi' (4-vector) at (z, y, x0); zero outside the grid.  `inb` must be warp-uniform
// only for the shuffle that follows; loads are guarded per lane.
template <class T, int CORR>
__device__ __forceinline__ F4 phi_vec(const FastArgs<T> &a, int64_t ib, int64_t ic, int z, int y,
                                      int x0, bool inb) {
  F4 v{{0.f, 0.f, 0.f, 0.f}};
  if (!inb) return v;
  if (a.base) v = ld4<T>(a.base + ib + ((int64_t)z * a.Y + y) * a.X + x0);
  if (CORR == C_COARSE) {
    float2 c = ld2<T>(a.corr + ic + ((int64_t)(z >> 1) * (a.Y >> 1) + (y >> 1)) * (a.X >> 1) + (x0 >> 1));
    v.v[0] += a.corr_sign * c.x;
    v.v[1] += a.corr_sign * c.x;
    v.v[2] += a.corr_sign * c.y;
    v.v[3] += a.corr_sign * c.y;
  } else if (CORR == C_SAME) {
    F4 c = ld4<T>(a.corr + ic + ((int64_t)z * a.Y + y) * a.X + x0);
#pragma unroll
    for (int e = 0; e < 4; ++e) v.v[e] += a.corr_sign * c.v[e];
  }
  if (a.zero_xend && x0 + 4 == a.X) v.v[3] = 0.f;
  return v;
}

// Neighbours across the vector boundary by shuffle (all lanes must call).
template <class T, int CORR>
__device__ __forceinline__ void halo_x(const FastArgs<T> &a, int64_t ib, int64_t ic, int z, int y,
                                       int x0, bool inb, const F4 &c, float &l, float &r) {
  const int lane = threadIdx.x & 31;
  float sl = __shfl_up_sync(0xffffffffu, c.v[3], 1);
  float sr = __shfl_down_sync(0xffffffffu, c.v[0], 1);
  l = 0.f;
  r = 0.f;
  if (inb) {
    if (x0 > 0) l = lane > 0 ? sl : phi_scalar<T, CORR>(a, ib, ic, z, y, x0 - 1);
    if (x0 + 4 < a.X) r = lane < 31 ? sr : phi_scalar<T, CORR>(a, ib, ic, z, y, x0 + 4);
  }
}

template <class T>
__device__ __forceinline__ void coef_halo_x(const T *s, int64_t base_off, int x0, int X, bool inb,
                                            const F4 &c, float &l, float &r) {
  const int lane = threadIdx.x & 31;
  float sl = __shfl_up_sync(0xffffffffu, c.v[3], 1);
  float sr = __shfl_down_sync(0xffffffffu, c.v[0], 1);
  l = c.v[0];  // wall: ghost sigma = interior sigma
  r = c.v[3];
  if (inb) {
    if (x0 > 0) l = lane > 0 ? sl : St<T>::ld(s + base_off - 1);
    if (x0 + 4 < X) r = lane < 31 ? sr : St<T>::ld(s + base_off + 4);
  }
}

__device__ __forceinline__ double block_reduce(double v) {
  __shared__ double sh[kFastThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

// ---------------------------------------------------------------------------------------
// 7-point forms (CONST7, SIGMA7).  R rows per thread.
// ---------------------------------------------------------------------------------------
template <int KIND, class T, int MODE, int CORR, int R>
__global__ void __launch_bounds__(kFastThreads, R == 1 ? 4 : 2)
    k_fast7(FastArgs<T> a) {
  const int64_t inst = blockIdx.z;
  if (a.active && !a.active[inst]) return;
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int nvx = X >> 2;
  const int ngroups = (Y + R - 1) / R;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < ngroups * nvx;
  const int g = valid ? i / nvx : 0;
  const int x0 = valid ? (i - g * nvx) * 4 : 0;
  const int64_t ib = inst * a.stride, ic = inst * a.corr_stride;
  const int64_t plane = (int64_t)Y * X;
  const int z0 = blockIdx.y * a.zc;
  const int z1 = min(Z, z0 + a.zc);

  // coefficient setup
  float kx = 0.f, ky = 0.f, kz = 0.f, dconst = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
  const T *sx = nullptr, *sy = nullptr, *sz = nullptr;
  if (KIND == HFM_OP_CONST7) {
    kz = a.op.k[0];
    ky = a.op.k[1];
    kx = a.op.k[2];
    dconst = 2.f * (kx + ky + kz);
  } else {
    const float s = a.op.scale;
    cz = a.op.c[0] * s;
    cy = a.op.c[1] * s;
    cx = a.op.c[2] * s;
    if (KIND == HFM_OP_FACE7) {  // instance strides follow from the extents
      sx = (const T *)a.op.coef[0] + inst * face7_nx(Z, Y, X);
      sy = (const T *)a.op.coef[1] + inst * face7_ny(Z, Y, X);
      sz = (const T *)a.op.coef[2] + inst * face7_nz(Z, Y, X);
    } else {
      sx = (const T *)a.op.coef[0] + inst * a.op.coef_stride;
      sy = (const T *)a.op.coef[1] + inst * a.op.coef_stride;
      sz = (const T *)a.op.coef[2] + inst * a.op.coef_stride;
    }
  }

  // per-row z queue: phi' at z-1, z, z+1; for SIGMA7 also sigma_z at z and the z- face
  F4 pm[R], pc[R], pp[R], szc[R], azlo[R];
  bool rin[R];
  int yr[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    yr[r] = g * R + r;
    rin[r] = valid && yr[r] < Y;
    pm[r] = (z0 > 0) ? phi_vec<T, CORR>(a, ib, ic, z0 - 1, yr[r], x0, rin[r]) : F4{{0.f, 0.f, 0.f, 0.f}};
    pc[r] = phi_vec<T, CORR>(a, ib, ic, z0, yr[r], x0, rin[r]);
    if (KIND == HFM_OP_SIGMA7) {
      const int64_t off = (int64_t)z0 * plane + (int64_t)yr[r] * X + x0;
      szc[r] = rin[r] ? ld4<T>(sz + off) : F4{{1.f, 1.f, 1.f, 1.f}};
      if (z0 > 0 && rin[r]) {
        F4 sm = ld4<T>(sz + off - plane);
#pragma unroll
        for (int e = 0; e < 4; ++e) azlo[r].v[e] = cz * 0.5f * (szc[r].v[e] + sm.v[e]);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) azlo[r].v[e] = cz * szc[r].v[e];
      }
    } else if (KIND == HFM_OP_FACE7) {
      // the z face below plane z0 (wall faces included in the array), times the scale
      const float s = a.op.scale;
      const F4 fz = rin[r] ? ld4<T>(sz + (int64_t)z0 * plane + (int64_t)yr[r] * X + x0) : F4{{0.f, 0.f, 0.f, 0.f}};
#pragma unroll
      for (int e = 0; e < 4; ++e) azlo[r].v[e] = s * fz.v[e];
    }
  }
  double acc = 0.0;
  float cpart[2] = {0.f, 0.f};  // RESTRICT: the two coarse cells of this vector, summed over planes

  for (int z = z0; z < z1; ++z) {
    F4 res[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int y = yr[r];
      const bool in = rin[r];
      pp[r] = (z + 1 < Z) ? phi_vec<T, CORR>(a, ib, ic, z + 1, y, x0, in) : F4{{0.f, 0.f, 0.f, 0.f}};
      float pl, pr;
      halo_x<T, CORR>(a, ib, ic, z, y, x0, in, pc[r], pl, pr);
      F4 pym = phi_vec<T, CORR>(a, ib, ic, z, y - 1, x0, in && y > 0);
      F4 pyp = phi_vec<T, CORR>(a, ib, ic, z, y + 1, x0, in && y + 1 < Y);
      const int64_t off = (int64_t)z * plane + (int64_t)y * X + x0;
      F4 Ax, dg;
      if (KIND == HFM_OP_CONST7) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          float xm = e == 0 ? pl : pc[r].v[e - 1];
          float xp = e == 3 ? pr : pc[r].v[e + 1];
          Ax.v[e] = dconst * pc[r].v[e] - kz * (pm[r].v[e] + pp[r].v[e]) -
                    ky * (pym.v[e] + pyp.v[e]) - kx * (xm + xp);
          dg.v[e] = dconst;
        }
      } else if (KIND == HFM_OP_FACE7) {
        // stored faces (scale applied here): the x faces of the 4 cells and the one right of
        // the last, the y faces below and above, the z face above (the one below is carried)
        const float s = a.op.scale;
        const int64_t rx = ((int64_t)z * Y + y) * (X + 8) + x0;
        const int64_t ry = ((int64_t)z * (Y + 1) + y) * X + x0;
        const F4 zero4{{0.f, 0.f, 0.f, 0.f}};
        const F4 fx = in ? ld4<T>(sx + rx) : zero4;
        const float fx4 = in ? St<T>::ld(sx + rx + 4) : 0.f;
        const F4 fyl = in ? ld4<T>(sy + ry) : zero4;
        const F4 fyh = in ? ld4<T>(sy + ry + X) : zero4;
        const F4 fzh = in ? ld4<T>(sz + off + plane) : zero4;
        F4 azhi;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float axm = s * fx.v[e], axp = s * (e == 3 ? fx4 : fx.v[e + 1]);
          const float aym = s * fyl.v[e], ayp = s * fyh.v[e];
          azhi.v[e] = s * fzh.v[e];
          const float xm = e == 0 ? pl : pc[r].v[e - 1];
          const float xp = e == 3 ? pr : pc[r].v[e + 1];
          const float p = pc[r].v[e];
          Ax.v[e] = axm * (p - xm) + axp * (p - xp) + aym * (p - pym.v[e]) + ayp * (p - pyp.v[e]) +
                    azlo[r].v[e] * (p - pm[r].v[e]) + azhi.v[e] * (p - pp[r].v[e]);
          dg.v[e] = ((axm + axp) + (aym + ayp)) + (azlo[r].v[e] + azhi.v[e]);
        }
        azlo[r] = azhi;
      } else {
        F4 sxc = in ? ld4<T>(sx + off) : F4{{1.f, 1.f, 1.f, 1.f}};
        float sxl, sxr;
        coef_halo_x<T>(sx, off, x0, X, in, sxc, sxl, sxr);
        F4 syc = in ? ld4<T>(sy + off) : F4{{1.f, 1.f, 1.f, 1.f}};
        F4 sym = (in && y > 0) ? ld4<T>(sy + off - X) : syc;
        F4 syp = (in && y + 1 < Y) ? ld4<T>(sy + off + X) : syc;
        F4 szp = (in && z + 1 < Z) ? ld4<T>(sz + off + plane) : szc[r];
        F4 azhi;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float sxe = sxc.v[e];
          const float sxm = e == 0 ? sxl : sxc.v[e - 1];
          const float sxp = e == 3 ? sxr : sxc.v[e + 1];
          // wall faces use the interior sigma (sxl / sxr already do at x = 0 / X-1)
          const float axm = cx * 0.5f * (sxe + sxm);
          const float axp = cx * 0.5f * (sxe + sxp);
          const float aym = cy * 0.5f * (syc.v[e] + sym.v[e]);
          const float ayp = cy * 0.5f * (syc.v[e] + syp.v[e]);
          azhi.v[e] = cz * 0.5f * (szc[r].v[e] + szp.v[e]);
          const float xm = e == 0 ? pl : pc[r].v[e - 1];
          const float xp = e == 3 ? pr : pc[r].v[e + 1];
          const float p = pc[r].v[e];
          Ax.v[e] = axm * (p - xm) + axp * (p - xp) + aym * (p - pym.v[e]) + ayp * (p - pyp.v[e]) +
                    azlo[r].v[e] * (p - pm[r].v[e]) + azhi.v[e] * (p - pp[r].v[e]);
          dg.v[e] = axm + axp + aym + ayp + azlo[r].v[e] + azhi.v[e];
        }
        azlo[r] = azhi;
        szc[r] = szp;
      }
      F4 f{{0.f, 0.f, 0.f, 0.f}};
      if (a.rhs && in) f = ld4<T>(a.rhs + ib + off);
      if (MODE == M_SMOOTH) {
#pragma unroll
        for (int e = 0; e < 4; ++e) res[r].v[e] = pc[r].v[e] + a.omega * __fdividef(f.v[e] - Ax.v[e], dg.v[e]);
        if (a.dot_rhs && in) {
#pragma unroll
          for (int e = 0; e < 4; ++e) acc += (double)res[r].v[e] * f.v[e];
        }
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) res[r].v[e] = Ax.v[e] - f.v[e];
        if (a.zero_xend_out && x0 + 4 == X) res[r].v[3] = 0.f;
        if (in) {
#pragma unroll
          for (int e = 0; e < 4; ++e) acc += (double)res[r].v[e] * (a.dot_phi ? pc[r].v[e] : res[r].v[e]);
        }
      }
      if (in && a.out) {
        if (MODE == M_SMOOTH && a.top_copy && z == 1) st4<T>(a.out + ib + y * X + x0, res[r]);
        if (!(MODE == M_SMOOTH && a.top_copy && z == 0 && Z > 1)) st4<T>(a.out + ib + off, res[r]);
      }
      pm[r] = pc[r];
      pc[r] = pp[r];
    }
    if (MODE == M_RESTRICT) {
      // x-pairs within the vector, y-pairs across the thread's two rows, z-pairs over planes
      cpart[0] += 0.125f * ((res[0].v[0] + res[0].v[1]) + (res[R - 1].v[0] + res[R - 1].v[1]));
      cpart[1] += 0.125f * ((res[0].v[2] + res[0].v[3]) + (res[R - 1].v[2] + res[R - 1].v[3]));
      if (z & 1) {
        if (valid) {
          const int Yc = Y >> 1, Xc = X >> 1;
          T *cp = a.coarse + inst * a.coarse_stride + ((int64_t)(z >> 1) * Yc + g) * Xc + (x0 >> 1);
          if (sizeof(T) == 4) {
            *reinterpret_cast<float2 *>(cp) = make_float2(cpart[0], cpart[1]);
          } else {
            cp[0] = St<T>::from(cpart[0]);
            cp[1] = St<T>::from(cpart[1]);
          }
        }
        cpart[0] = cpart[1] = 0.f;
      }
    }
  }
  if ((MODE != M_SMOOTH || a.dot_rhs) && a.partials) {
    double t = block_reduce(acc);
    if (threadIdx.x == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------------------------------
// 27-point form (K27): per-plane partial sums into three pending outputs.
// ---------------------------------------------------------------------------------------
template <class T, int MODE, int CORR>
__global__ void __launch_bounds__(kFastThreads)
    k_fast27(FastArgs<T> a) {
  const int64_t inst = blockIdx.z;
  if (a.active && !a.active[inst]) return;
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int nvx = X >> 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < Y * nvx;
  const int y = valid ? i / nvx : 0;
  const int x0 = valid ? (i - y * nvx) * 4 : 0;
  const int64_t ib = inst * a.stride, ic = inst * a.corr_stride;
  const int64_t plane = (int64_t)Y * X;
  const int z0 = blockIdx.y * a.zc;
  const int z1 = min(Z, z0 + a.zc);
  const float *K = a.op.k;

  // s[a] of plane p = sum_{b,c} K[a][b][c] phi'(p, y+b-1, x+c-1)
  auto plane_sums = [&](int p, F4 &s0, F4 &s1, F4 &s2, F4 &centre) {
    F4 rows[3];
    float ls[3], rs[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int yy = y + b - 1;
      const bool in = valid && p >= 0 && p < Z && yy >= 0 && yy < Y;
      rows[b] = phi_vec<T, CORR>(a, ib, ic, p, yy, x0, in);
      halo_x<T, CORR>(a, ib, ic, p, yy, x0, in, rows[b], ls[b], rs[b]);
    }
    centre = rows[1];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float t0 = 0.f, t1 = 0.f, t2 = 0.f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float xm = e == 0 ? ls[b] : rows[b].v[e - 1];
        const float xc = rows[b].v[e];
        const float xp = e == 3 ? rs[b] : rows[b].v[e + 1];
        t0 += K[3 * b + 0] * xm + K[3 * b + 1] * xc + K[3 * b + 2] * xp;
        t1 += K[9 + 3 * b + 0] * xm + K[9 + 3 * b + 1] * xc + K[9 + 3 * b + 2] * xp;
        t2 += K[18 + 3 * b + 0] * xm + K[18 + 3 * b + 1] * xc + K[18 + 3 * b + 2] * xp;
      }
      s0.v[e] = t0;
      s1.v[e] = t1;
      s2.v[e] = t2;
    }
  };

  // pending: out(z) = s0(z-1) + s1(z) + s2(z+1)
  F4 acc_cur, acc_next, cen_cur, cen_next, d0, d1, d2, dc;
  plane_sums(z0 - 1, d0, d1, d2, dc);
  F4 s0, s1, s2;
  plane_sums(z0, s0, s1, s2, cen_cur);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    acc_cur.v[e] = d0.v[e] + s1.v[e];
    acc_next.v[e] = s0.v[e];
  }
  const float diag = K[13];
  double acc2 = 0.0;
  for (int z = z0; z < z1; ++z) {
    F4 n0, n1, n2;
    plane_sums(z + 1, n0, n1, n2, cen_next);
    F4 Ax, res;
#pragma unroll
    for (int e = 0; e < 4; ++e) Ax.v[e] = acc_cur.v[e] + n2.v[e];
    const int64_t off = (int64_t)z * plane + (int64_t)y * X + x0;
    F4 f{{0.f, 0.f, 0.f, 0.f}};
    if (a.rhs && valid) f = ld4<T>(a.rhs + ib + off);
    if (MODE == M_SMOOTH) {
#pragma unroll
      for (int e = 0; e < 4; ++e) res.v[e] = cen_cur.v[e] + a.omega * __fdividef(f.v[e] - Ax.v[e], diag);
      if (a.dot_rhs && valid) {
#pragma unroll
        for (int e = 0; e < 4; ++e) acc2 += (double)res.v[e] * f.v[e];
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) res.v[e] = Ax.v[e] - f.v[e];
      if (a.zero_xend_out && x0 + 4 == X) res.v[3] = 0.f;
      if (valid) {
#pragma unroll
        for (int e = 0; e < 4; ++e) acc2 += (double)res.v[e] * (a.dot_phi ? cen_cur.v[e] : res.v[e]);
      }
    }
    if (valid && a.out) {
      if (MODE == M_SMOOTH && a.top_copy && z == 1) st4<T>(a.out + ib + y * X + x0, res);
      if (!(MODE == M_SMOOTH && a.top_copy && z == 0 && Z > 1)) st4<T>(a.out + ib + off, res);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      acc_cur.v[e] = acc_next.v[e] + n1.v[e];
      acc_next.v[e] = n0.v[e];
    }
    cen_cur = cen_next;
  }
  if ((MODE != M_SMOOTH || a.dot_rhs) && a.partials) {
    double t = block_reduce(acc2);
    if (threadIdx.x == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

// Resident blocks per SM of a kernel (its registers decide: 2-3 blocks of 256 threads),
// looked up once per kernel.
int resident_blocks(const void *kernel) {
  static std::mutex mu;
  static std::map<const void *, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kFastThreads, 0) != cudaSuccess || nb < 1)
    nb = 2;
  cache[kernel] = nb;
  return nb;
}

// Grid shape: (plane tiles, z chunks, instances); z chunks sized so that the launch fills the
// GPU's resident blocks once (a second, partly filled wave doubled the time of the small
// levels: 64 instances of 32^3 made 512 blocks against 444 resident), at least 4 planes each
// (even for the restriction).
template <class T>
dim3 fast_grid(FastArgs<T> &a, int B, int rows, bool even_chunks, int per_sm) {
  const int nvx = a.X >> 2;
  const int64_t vecs = (int64_t)((a.Y + rows - 1) / rows) * nvx;
  const int tiles = (int)((vecs + kFastThreads - 1) / kFastThreads);
  const int64_t target = (int64_t)sm_count() * per_sm;
  int64_t chunks = std::max<int64_t>(1, target / ((int64_t)tiles * B));
  int zc = (int)((a.Z + chunks - 1) / chunks);
  if (zc < 4) zc = 4;
  if (even_chunks && (zc & 1)) ++zc;
  if (zc > a.Z) zc = a.Z;
  a.zc = zc;
  return dim3(tiles, (a.Z + zc - 1) / zc, B);
}

}  // namespace

bool fast_eligible(int kind, Grid3 g, bool restrict_mode) {
  if (kind != HFM_OP_CONST7 && kind != HFM_OP_SIGMA7 && kind != HFM_OP_K27 && kind != HFM_OP_FACE7)
    return false;
  if ((g.X & 3) || g.X < 4) return false;
  if (restrict_mode) {
    if (kind == HFM_OP_K27) return false;
    if ((g.Y & 1) || (g.Z & 1)) return false;
  }
  return true;
}

template <class T>
int fast_launch(int kind, int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                T *out, T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g,
                float omega, unsigned flags, const int *active, double *partials,
                int *nblk_out, cudaStream_t s) {
  FastArgs<T> a;
  a.op = op;
  a.base = phi.base;
  a.corr = phi.corr;
  a.rhs = rhs;
  a.out = out;
  a.coarse = coarse;
  a.partials = partials;
  a.active = active;
  a.stride = stride;
  a.corr_stride = phi.corr_stride;
  a.coarse_stride = coarse_stride;
  a.Z = g.Z;
  a.Y = g.Y;
  a.X = g.X;
  a.omega = omega;
  a.corr_sign = phi.corr_sign;
  a.zero_xend = phi.zero_xend ? 1 : 0;
  a.zero_xend_out = (mode != M_SMOOTH && (flags & HFM_FLAG_ZERO_XEND)) ? 1 : 0;
  a.top_copy = (mode == M_SMOOTH && (flags & HFM_FLAG_TOP_COPY)) ? 1 : 0;
  a.dot_phi = (mode == M_RESID && (flags & HFM_INT_DOT_PHI)) ? 1 : 0;
  a.dot_rhs = (mode == M_SMOOTH && (flags & HFM_INT_DOT_RHS) && partials) ? 1 : 0;
  a.zc = 0;
  if (phi.base && phi.base_stride != stride) return fail(HFM_ERR_BAD_ARG, "fast path: stride mismatch");
  const int corr = phi.corr ? (phi.corr_coarse ? C_COARSE : C_SAME) : C_NONE;
  const int rows = (mode == M_RESTRICT) ? 2 : 1;
#define HFM_FAST_GO(KER)                                                                       \
  do {                                                                                         \
    const dim3 grid = fast_grid<T>(a, B, rows, mode == M_RESTRICT,                             \
                                   resident_blocks((const void *)KER));                        \
    if (nblk_out) *nblk_out = grid.x * grid.y;                                                 \
    KER<<<grid, kFastThreads, 0, s>>>(a);                                                      \
  } while (0)
  // dispatch
  if (kind == HFM_OP_K27) {
    if (mode == M_SMOOTH) {
      if (corr == C_NONE) HFM_FAST_GO((k_fast27<T, M_SMOOTH, C_NONE>));
      else if (corr == C_COARSE) HFM_FAST_GO((k_fast27<T, M_SMOOTH, C_COARSE>));
      else HFM_FAST_GO((k_fast27<T, M_SMOOTH, C_SAME>));
    } else {
      if (corr != C_NONE) return fail(HFM_ERR_UNSUPPORTED, "fast path: corrected residual");
      HFM_FAST_GO((k_fast27<T, M_RESID, C_NONE>));
    }
  } else {
#define HFM_FAST7(KIND)                                                                        \
  if (mode == M_SMOOTH) {                                                                      \
    if (corr == C_NONE) HFM_FAST_GO((k_fast7<KIND, T, M_SMOOTH, C_NONE, 1>));                  \
    else if (corr == C_COARSE) HFM_FAST_GO((k_fast7<KIND, T, M_SMOOTH, C_COARSE, 1>));         \
    else HFM_FAST_GO((k_fast7<KIND, T, M_SMOOTH, C_SAME, 1>));                                 \
  } else if (mode == M_RESID) {                                                                \
    if (corr != C_NONE) return fail(HFM_ERR_UNSUPPORTED, "fast path: corrected residual");     \
    HFM_FAST_GO((k_fast7<KIND, T, M_RESID, C_NONE, 1>));                                       \
  } else {                                                                                     \
    if (corr != C_NONE) return fail(HFM_ERR_UNSUPPORTED, "fast path: corrected residual");     \
    HFM_FAST_GO((k_fast7<KIND, T, M_RESTRICT, C_NONE, 2>));                                    \
  }
    if (kind == HFM_OP_CONST7) {
      HFM_FAST7(HFM_OP_CONST7)
    } else if (kind == HFM_OP_FACE7) {
      HFM_FAST7(HFM_OP_FACE7)
    } else {
      HFM_FAST7(HFM_OP_SIGMA7)
    }
#undef HFM_FAST7
  }
#undef HFM_FAST_GO
  HFM_CHECK_LAUNCH("fast stencil kernel");
  return HFM_OK;
}

#define HFM_FAST_INST(T)                                                                       \
  template int fast_launch<T>(int, int, const DevOp &, const PhiSrc<T> &, const T *, T *, T *, \
                              int64_t, int64_t, int, Grid3, float, unsigned, const int *,      \
                              double *, int *, cudaStream_t);
HFM_FAST_INST(float)
HFM_FAST_INST(__nv_bfloat16)
HFM_FAST_INST(__half)

}  // namespace hfm
