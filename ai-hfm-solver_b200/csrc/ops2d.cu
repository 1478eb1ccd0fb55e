// Two-dimensional operators: the reference's Conv2D form of the multigrid
// (Unstructured Mesh/Multigrid_2D.ipynb: 3x3 SAME convolution #c7, 2x2 VALID averaging
// restriction with weight 0.25 #c9, UpSampling2D #c11, sawtooth cycle #c18) with zero or
// periodic padding, in float32 or bf16 storage with float32 arithmetic, and the kernels of the
// doubly periodic Kolmogorov-flow stepper (two-stage momentum with sin(k y) forcing,
// divergence, pressure-gradient projection).
//
// Layout: (B, Y, X) float32 / bf16, x fastest.  The fields of this path are small (512^2 cells,
// 1 MB per float32 field) and stay in L2 across the kernels of a step, so these kernels map one
// thread to one output cell and are launched from captured CUDA graphs.
#include <cooperative_groups.h>
#include <cstdint>

#include "hfm_internal.cuh"

namespace hfm {

namespace {

constexpr int kT2 = 256;

struct W9 {
  float w[9];  // w[3a + b]: weight of phi[y + a - 1][x + b - 1]
};

// phi' = base + sign * coarse[y/2][x/2] at (y, x) of instance b, or 0 outside a zero-padded grid
template <class T> struct Src2 {
  const T *base;
  const T *coarse;
  float sign;
  int64_t stride, cstride;
  int Y, X, Xc;
  int periodic;
  int cshift;  // 1: coarse is the next coarser level (nearest upsampling); 0: same level
  __device__ __forceinline__ float operator()(int64_t b, int y, int x) const {
    if (periodic) {
      y = y < 0 ? y + Y : (y >= Y ? y - Y : y);
      x = x < 0 ? x + X : (x >= X ? x - X : x);
    } else if (y < 0 || y >= Y || x < 0 || x >= X) {
      return 0.f;
    }
    float v = base ? St<T>::ld(base + b * stride + (int64_t)y * X + x) : 0.f;
    if (coarse) v += sign * St<T>::ld(coarse + b * cstride + (int64_t)(y >> cshift) * Xc + (x >> cshift));
    return v;
  }
};

// The first Jacobi sweep from a zero iterate at (y, x), as hfm_jacobi2d stores it: 0 + omega
// f / w[4] rounded to T (0 outside a zero-padded grid); the source of the second sweep of a
// fused pair.
template <class T> struct Sweep1Src {
  const T *f;
  float omega, diag;
  int64_t stride;
  int Y, X;
  int periodic;
  __device__ __forceinline__ float operator()(int64_t b, int y, int x) const {
    if (periodic) {
      y = y < 0 ? y + Y : (y >= Y ? y - Y : y);
      x = x < 0 ? x + X : (x >= X ? x - X : x);
    } else if (y < 0 || y >= Y || x < 0 || x >= X) {
      return 0.f;
    }
    const float fv = St<T>::ld(f + b * stride + (int64_t)y * X + x);
    return St<T>::to(St<T>::from(0.f + omega * fv / diag));
  }
};

template <class S>
__device__ __forceinline__ float conv9(const W9 &w, const S &s, int64_t b, int y, int x,
                                       float *centre) {
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float v = s(b, y + a - 1, x + c - 1);
      if (a == 1 && c == 1) *centre = v;
      acc += w.w[3 * a + c] * v;
    }
  return acc;
}

// MODE 0: out = A phi; 1: out = A phi - f; 2: out = phi + omega (f - A phi) / w[4]
template <class T, int MODE>
__global__ void __launch_bounds__(kT2) k2_stencil(W9 w, Src2<T> s, const T *__restrict__ f,
                                                  T *__restrict__ out, float omega) {
  const int64_t b = blockIdx.y;
  const int64_t n = (int64_t)s.Y * s.X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / s.X), x = (int)(i % s.X);
    float pc;
    const float ax = conv9(w, s, b, y, x, &pc);
    const float fv = f ? St<T>::ld(f + b * s.stride + i) : 0.f;
    float r;
    if (MODE == 0) r = ax;
    else if (MODE == 1) r = ax - fv;
    else r = pc + omega * (fv - ax) / w.w[4];
    out[b * s.stride + i] = St<T>::from(r);
  }
}

// Two Jacobi sweeps from a zero iterate in one pass: out = phi1 + omega (f - A phi1) / w[4]
// with phi1 the first sweep (Sweep1Src), recomputed at each neighbour; the bits of two
// hfm_jacobi2d launches.
template <class T>
__global__ void __launch_bounds__(kT2) k2_two_sweeps(W9 w, Sweep1Src<T> s, T *__restrict__ out) {
  const int64_t b = blockIdx.y;
  const int64_t n = (int64_t)s.Y * s.X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / s.X), x = (int)(i % s.X);
    float pc;
    const float ax = conv9(w, s, b, y, x, &pc);
    const float fv = St<T>::ld(s.f + b * s.stride + i);
    out[b * s.stride + i] = St<T>::from(pc + s.omega * (fv - ax) / w.w[4]);
  }
}

// Two Jacobi sweeps in one pass from phi = base + sign P(coarse) (Src2): a 32 x 8 tile of
// the first sweep and its one-cell ring in shared memory (each value computed as the
// one-sweep launch computes it and rounded to T as it stores it), then the second sweep from
// there; the bits of two hfm_jacobi2d launches.
constexpr int kTwoTX = 32, kTwoTY = 8;
static_assert(kTwoTX * kTwoTY == kT2, "one thread per output cell of a tile");
template <class T>
__global__ void __launch_bounds__(kT2) k2_two_sweeps_tile(W9 w, Src2<T> s, const T *__restrict__ f,
                                                          T *__restrict__ out, float omega) {
  __shared__ float mid[kTwoTY + 2][kTwoTX + 2];
  const int64_t b = blockIdx.z;
  const int x0 = blockIdx.x * kTwoTX, y0 = blockIdx.y * kTwoTY;
  for (int k = threadIdx.x; k < (kTwoTY + 2) * (kTwoTX + 2); k += blockDim.x) {
    const int ty = k / (kTwoTX + 2), tx = k - ty * (kTwoTX + 2);
    int y = y0 + ty - 1, x = x0 + tx - 1;  // -1 <= y <= y0 + kTwoTY, likewise x
    float v = 0.f;
    // cells past row Y / column X neighbour no cell of the grid: left at 0
    bool live = y <= s.Y && x <= s.X;
    if (s.periodic) {
      y = y < 0 ? y + s.Y : (y >= s.Y ? y - s.Y : y);
      x = x < 0 ? x + s.X : (x >= s.X ? x - s.X : x);
    } else {
      live = live && y >= 0 && y < s.Y && x >= 0 && x < s.X;
    }
    if (live) {
      float pc;
      const float ax = conv9(w, s, b, y, x, &pc);
      const float fv = St<T>::ld(f + b * s.stride + (int64_t)y * s.X + x);
      v = St<T>::to(St<T>::from(pc + omega * (fv - ax) / w.w[4]));
    }
    mid[ty][tx] = v;
  }
  __syncthreads();
  const int tx = threadIdx.x % kTwoTX, ty = threadIdx.x / kTwoTX;
  const int y = y0 + ty, x = x0 + tx;
  if (y < s.Y && x < s.X) {
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc += w.w[3 * a + c] * mid[ty + a][tx + c];
    const float pc = mid[ty + 1][tx + 1];
    const int64_t i = b * s.stride + (int64_t)y * s.X + x;
    out[i] = St<T>::from(pc + omega * (St<T>::ld(f + i) - acc) / w.w[4]);
  }
}

// The down leg of a level with two pre-sweeps in one pass: phi = two Jacobi sweeps from zero
// and the coarse rhs 0.25 * sum over 2 x 2 cells of (A phi - f).  A 32 x 8 tile holds the
// first sweep on a two-cell ring, the second on a one-cell ring (each value computed and
// rounded to T as the one-sweep launches store it) and the tile's residuals in shared memory;
// the bits of hfm_jacobi2d (HFM_FLAG_TWO_SWEEPS) followed by hfm_residual_restrict2d.
// Even extents: the tile's coarse cells lie inside the grid or wholly outside it.
template <class T>
__global__ void __launch_bounds__(kT2) k2_pre2_restrict(W9 w, Sweep1Src<T> s, T *__restrict__ phi,
                                                        T *__restrict__ coarse) {
  __shared__ float s1[kTwoTY + 4][kTwoTX + 4];
  __shared__ float s2[kTwoTY + 2][kTwoTX + 2];
  __shared__ float rr[kTwoTY][kTwoTX];
  const int64_t b = blockIdx.z;
  const int Y = s.Y, X = s.X;
  const int x0 = blockIdx.x * kTwoTX, y0 = blockIdx.y * kTwoTY;
  // first sweep on the tile and a two-cell ring (s(b, y, x) wraps or pads, -2 <= y - y0 <= 9)
  for (int k = threadIdx.x; k < (kTwoTY + 4) * (kTwoTX + 4); k += blockDim.x) {
    const int ty = k / (kTwoTX + 4), tx = k - ty * (kTwoTX + 4);
    int y = y0 + ty - 2, x = x0 + tx - 2;
    if (s.periodic) {  // a ring cell may lie more than one period out on a grid of 1 row
      y = ((y % Y) + Y) % Y;
      x = ((x % X) + X) % X;
    }
    s1[ty][tx] = s(b, y, x);
  }
  __syncthreads();
  // second sweep on the tile and a one-cell ring
  for (int k = threadIdx.x; k < (kTwoTY + 2) * (kTwoTX + 2); k += blockDim.x) {
    const int ty = k / (kTwoTX + 2), tx = k - ty * (kTwoTX + 2);
    int y = y0 + ty - 1, x = x0 + tx - 1;
    bool live = true;
    if (s.periodic) {
      y = ((y % Y) + Y) % Y;
      x = ((x % X) + X) % X;
    } else {
      live = y >= 0 && y < Y && x >= 0 && x < X;
    }
    float v = 0.f;
    if (live) {
      float acc = 0.f;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc += w.w[3 * a + c] * s1[ty + a][tx + c];
      const float pc = s1[ty + 1][tx + 1];
      const float fv = St<T>::ld(s.f + b * s.stride + (int64_t)y * X + x);
      v = St<T>::to(St<T>::from(pc + s.omega * (fv - acc) / w.w[4]));
    }
    s2[ty][tx] = v;
  }
  __syncthreads();
  {
    const int tx = threadIdx.x % kTwoTX, ty = threadIdx.x / kTwoTX;
    const int y = y0 + ty, x = x0 + tx;
    if (y < Y && x < X) {
      float acc = 0.f;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc += w.w[3 * a + c] * s2[ty + a][tx + c];
      const int64_t i = b * s.stride + (int64_t)y * X + x;
      phi[i] = St<T>::from(s2[ty + 1][tx + 1]);
      float r = acc;
      r -= St<T>::ld(s.f + i);
      rr[ty][tx] = r;
    }
  }
  __syncthreads();
  if (threadIdx.x < (kTwoTY / 2) * (kTwoTX / 2)) {
    const int jy = threadIdx.x / (kTwoTX / 2), jx = threadIdx.x - jy * (kTwoTX / 2);
    const int yc = y0 / 2 + jy, xc = x0 / 2 + jx, Yc = Y / 2, Xc = X / 2;
    if (yc < Yc && xc < Xc) {
      float sum = 0.f;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 2; ++c) sum += rr[2 * jy + a][2 * jx + c];
      coarse[b * (int64_t)Yc * Xc + (int64_t)yc * Xc + xc] = St<T>::from(0.25f * sum);
    }
  }
}

// Coarse cell (yc, xc) = 0.25 * sum over its 2x2 fine cells of (A phi - f); float32 phi and f
// may be read while the coarse output is stored in T (TI = input storage).
template <class TI, class TO>
__global__ void __launch_bounds__(kT2) k2_resid_restrict(W9 w, Src2<TI> s, const TI *__restrict__ f,
                                                         TO *__restrict__ rc, int64_t cstride) {
  const int64_t b = blockIdx.y;
  const int Yc = s.Y >> 1, Xc = s.X >> 1;
  const int64_t nc = (int64_t)Yc * Xc;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nc;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int yc = (int)(j / Xc), xc = (int)(j % Xc);
    float sum = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int y = 2 * yc + a, x = 2 * xc + c;
        float pc;
        float v = conv9(w, s, b, y, x, &pc);
        if (f) v -= St<TI>::ld(f + b * s.stride + (int64_t)y * s.X + x);
        sum += v;
      }
    rc[b * cstride + j] = St<TO>::from(0.25f * sum);
  }
}

// Residual A phi - f of float32 phi / f stored in T (the outer defect of a mixed-precision
// solve), with per-block partial sums of its square (float64) when `partials` is given.
template <class TO>
__global__ void __launch_bounds__(kT2) k2_outer_resid(W9 w, Src2<float> s, const float *__restrict__ f,
                                                      TO *__restrict__ r, double *partials) {
  __shared__ double sh[kT2 / 32];
  const int64_t b = blockIdx.y;
  const int64_t n = (int64_t)s.Y * s.X;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / s.X), x = (int)(i % s.X);
    float pc;
    const float v = conv9(w, s, b, y, x, &pc) - f[b * s.stride + i];
    r[b * s.stride + i] = St<TO>::from(v);
    acc += (double)v * v;
  }
  if (!partials) return;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kT2 / 32; ++k) t += sh[k];
    partials[b * gridDim.x + blockIdx.x] = t;
  }
}

template <class T>
__global__ void __launch_bounds__(kT2) k2_restrict(const T *__restrict__ fine, T *__restrict__ coarse,
                                                   int Y, int X) {
  const int64_t b = blockIdx.y;
  const int Yc = Y >> 1, Xc = X >> 1;
  const int64_t nc = (int64_t)Yc * Xc, nf = (int64_t)Y * X;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nc;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int yc = (int)(j / Xc), xc = (int)(j % Xc);
    const T *p = fine + b * nf + (int64_t)(2 * yc) * X + 2 * xc;
    const float s = (St<T>::to(p[0]) + St<T>::to(p[1])) + (St<T>::to(p[X]) + St<T>::to(p[X + 1]));
    coarse[b * nc + j] = St<T>::from(0.25f * s);
  }
}

template <class T>
__global__ void __launch_bounds__(kT2) k2_prolong(const T *__restrict__ coarse, T *__restrict__ fine,
                                                  int Yc, int Xc) {
  const int64_t b = blockIdx.y;
  const int Y = 2 * Yc, X = 2 * Xc;
  const int64_t nf = (int64_t)Y * X, nc = (int64_t)Yc * Xc;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nf;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / X), x = (int)(i % X);
    fine[b * nf + i] = coarse[b * nc + (int64_t)(y >> 1) * Xc + (x >> 1)];
  }
}

// p += sign * w (float32 p, w in T)
template <class T>
__global__ void __launch_bounds__(kT2) k2_update(float *__restrict__ p, const T *__restrict__ w,
                                                 float sign, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] += sign * St<T>::to(w[i]);
}

// `sweeps` Jacobi sweeps from phi = 0 on a small grid held in shared memory, one block per
// instance (the coarsest level of a cycle).
template <class T>
__global__ void __launch_bounds__(kT2) k2_coarse_jacobi(W9 w, const T *__restrict__ f, T *__restrict__ out,
                                                        int Y, int X, float omega, int sweeps,
                                                        int periodic) {
  extern __shared__ float sm2[];
  const int n = Y * X;
  float *a = sm2, *c = sm2 + n, *ff = sm2 + 2 * n;
  const int64_t b = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a[i] = 0.f;
    ff[i] = St<T>::to(f[b * n + i]);
  }
  __syncthreads();
  for (int s = 0; s < sweeps; ++s) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int y = i / X, x = i % X;
      float acc = 0.f;
      for (int aa = 0; aa < 3; ++aa)
        for (int cc = 0; cc < 3; ++cc) {
          int yy = y + aa - 1, xx = x + cc - 1;
          float v;
          if (periodic) {
            yy = (yy + Y) % Y;
            xx = (xx + X) % X;
            v = a[yy * X + xx];
          } else {
            v = (yy < 0 || yy >= Y || xx < 0 || xx >= X) ? 0.f : a[yy * X + xx];
          }
          acc += w.w[3 * aa + cc] * v;
        }
      c[i] = a[i] + omega * (ff[i] - acc) / w.w[4];
    }
    __syncthreads();
    float *t = a;
    a = c;
    c = t;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[b * n + i] = St<T>::from(a[i]);
}

// ------------------------------------------------------------------ fused coarse cycle
// The V-cycle of the levels of at most 4096 cells (64^2 .. 4^2 of a 512^2 grid) in one
// launch: one 1024-thread block per instance, every field of those levels in shared memory
// (float32), sweeps separated by __syncthreads(); a coarsest level of at most 32 cells runs
// on one warp with its iterate in registers (shuffles, no barriers).  The steps and their
// arithmetic are those of the per-level kernels (hfm_jacobi2d, hfm_residual_restrict2d,
// hfm_coarse_jacobi2d): nu_pre sweeps from zero, residual + 2 x 2 averaging restriction
// (0.25 x the sum), recursion, coarse_sweeps sweeps from zero on the coarsest level, then
// the nearest-prolongation correction phi - P w and nu_post sweeps; iterates stay in float32
// between sweeps (the per-level path stores them in the storage type, so float32 storage
// gives the same bits).
constexpr int kSub2Levels = 8;
constexpr int kSub2Threads = 1024;
struct Sub2Args {
  W9 w[kSub2Levels];
  int Y[kSub2Levels], X[kSub2Levels];
  int nlev, periodic, nu_pre, nu_post, coarse_sweeps;
  int smem_floats;  // shared memory of all levels, in floats
  float omega;
};

// This thread's first cell of a Y x X level and the step between its cells, for walks by
// the whole block (thread t visits cells t, t + nt, ...; one division per level visit).
struct Walk2 {
  int y0, x0, sy, sx;
};
__device__ __forceinline__ Walk2 walk2_of(int X) {
  Walk2 w;
  const int t = threadIdx.x, nt = blockDim.x;
  if ((X & (X - 1)) == 0) {  // a power of two: shifts and masks
    const int s = __ffs(X) - 1;
    w.y0 = t >> s;
    w.x0 = t & (X - 1);
    w.sy = nt >> s;
    w.sx = nt & (X - 1);
  } else {
    w.y0 = t / X;
    w.x0 = t - w.y0 * X;
    w.sy = nt / X;
    w.sx = nt - w.sy * X;
  }
  return w;
}
template <class F>
__device__ __forceinline__ void walk2(const Walk2 &w, int Y, int X, F &&f) {
  int y = w.y0, x = w.x0;
  while (y < Y) {
    f(y * X + x, y, x);
    x += w.sx;
    y += w.sy;
    if (x >= X) {
      x -= X;
      ++y;
    }
  }
}

// The iterates of a level live in (Y + 2) x (X + 2) fields (row pitch P = X + 2): the cells
// inside and a one-cell ring that holds zeros (zero padding) or the periodic images of the
// opposite edge, so that a stencil reads nine fixed offsets.  A phi at a cell, in the order
// of conv9 (rows, then columns).
__device__ __forceinline__ float stencil9(const W9 &w, const float *c, int P, float *centre) {
  const float *u = c - P, *d = c + P;
  float acc = 0.f;
  acc += w.w[0] * u[-1];
  acc += w.w[1] * u[0];
  acc += w.w[2] * u[1];
  acc += w.w[3] * c[-1];
  acc += w.w[4] * c[0];
  acc += w.w[5] * c[1];
  acc += w.w[6] * d[-1];
  acc += w.w[7] * d[0];
  acc += w.w[8] * d[1];
  *centre = c[0];
  return acc;
}

// fld(y, x) = v, and on a periodic level also every ring cell that is an image of (y, x)
__device__ __forceinline__ void put2(float *fld, int P, int Y, int X, int y, int x, float v,
                                     int periodic) {
  float *c = fld + (y + 1) * P + x + 1;
  *c = v;
  if (!periodic) return;
  const bool t0 = y == 0, t1 = y == Y - 1;
  if (t0) c[Y * P] = v;
  if (t1) c[-Y * P] = v;
  if (x == 0) {
    c[X] = v;
    if (t0) c[Y * P + X] = v;
    if (t1) c[-Y * P + X] = v;
  }
  if (x == X - 1) {
    c[-X] = v;
    if (t0) c[Y * P - X] = v;
    if (t1) c[-Y * P - X] = v;
  }
}

// out = in + omega (f - A in) / w[4] on level (Y, X), the whole block; in == nullptr: a zero
// iterate
__device__ __forceinline__ void sub2_sweep(const W9 &w, const float *__restrict__ in, const float *__restrict__ f,
                           float *__restrict__ out, int Y, int X, const Walk2 &wk, int periodic,
                           float omega) {
  const int P = X + 2;
  walk2(wk, Y, X, [&](int i, int y, int x) {
    float pc = 0.f, ax = 0.f;
    if (in) ax = stencil9(w, in + (y + 1) * P + x + 1, P, &pc);
    put2(out, P, Y, X, y, x, pc + omega * (f[i] - ax) / w.w[4], periodic);
  });
  __syncthreads();
}

// `sweeps` sweeps from zero on a level of at most 32 cells by warp 0, one cell per lane in a
// register and the neighbours by shuffles; the same operation order as apply9 / sub2_sweep.
// Lanes outside the level carry zeros.  Returns this lane's value.
__device__ __forceinline__ float sub2_coarsest_warp(const W9 &w9, const float *__restrict__ f, int Y, int X,
                                    int periodic, float omega, int sweeps) {
  const int lane = threadIdx.x, n = Y * X;
  const bool live = lane < n;
  const int y = live ? lane / X : 0, x = live ? lane - (lane / X) * X : 0;
  int r[3] = {y - 1, y, y + 1}, c[3] = {x - 1, x, x + 1};
  unsigned ok = 0x1ff;  // bit 3a + b: neighbour (a, b) inside the grid
  if (periodic) {
    r[0] = r[0] < 0 ? Y - 1 : r[0];
    r[2] = r[2] >= Y ? 0 : r[2];
    c[0] = c[0] < 0 ? X - 1 : c[0];
    c[2] = c[2] >= X ? 0 : c[2];
  } else {
    if (r[0] < 0) ok &= ~0x007u;
    if (r[2] >= Y) ok &= ~0x1c0u;
    if (c[0] < 0) ok &= ~0x049u;
    if (c[2] >= X) ok &= ~0x124u;
  }
  if (!live) ok = 0;
  int src[9];
  float w[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    src[k] = (ok >> k) & 1 ? r[k / 3] * X + c[k % 3] : lane;
    w[k] = w9.w[k];
  }
  const float fv = live ? f[lane] : 0.f;
  float ph = 0.f;
  for (int s = 0; s < sweeps; ++s) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float v = __shfl_sync(0xffffffffu, ph, src[k]);
      acc += w[k] * ((ok >> k) & 1 ? v : 0.f);
    }
    const float nv = ph + omega * (fv - acc) / w[4];
    ph = live ? nv : 0.f;
  }
  return ph;
}

// One level of the fused cycle: extents, row pitch of the padded iterates P = X + 2, their
// size np = (Y + 2) P, the level's offset in shared memory (two iterates, then the rhs of
// Y X floats) and its weights, held in registers while the level runs.
struct Lv2 {
  int Y, X, P, np, off;
  W9 w;
};

// pre-sweeps from zero, then the coarse rhs 0.25 * sum over the 2 x 2 cells of (A phi - f);
// the iterate ends in buffer (nu_pre - 1) & 1
__device__ __forceinline__ void sub2_down(float *sm, const Lv2 &L, const Lv2 &Lc,
                                          const Sub2Args &a) {
  float *const b0 = sm + L.off, *const b1 = b0 + L.np;
  auto buf = [&](int k) { return k ? b1 : b0; };  // selects: no local-memory array
  const float *f = sm + L.off + 2 * L.np;
  const Walk2 wk = walk2_of(L.X);
  int c = 0;
  sub2_sweep(L.w, nullptr, f, buf(0), L.Y, L.X, wk, a.periodic, a.omega);
  for (int k = 1; k < a.nu_pre; ++k) {
    sub2_sweep(L.w, buf(c), f, buf(c ^ 1), L.Y, L.X, wk, a.periodic, a.omega);
    c ^= 1;
  }
  const float *ph = buf(c);
  float *fc = sm + Lc.off + 2 * Lc.np;
  const int P = L.P, X = L.X;
  walk2(walk2_of(Lc.X), Lc.Y, Lc.X, [&](int j, int yc, int xc) {
    float sum = 0.f;
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int y = 2 * yc + p, x = 2 * xc + q;
        float pc;
        sum += stencil9(L.w, ph + (y + 1) * P + x + 1, P, &pc) - f[y * X + x];
      }
    fc[j] = 0.25f * sum;
  });
  __syncthreads();
}

// coarse_sweeps sweeps from zero on the coarsest level; returns the buffer holding the result
__device__ __forceinline__ int sub2_coarsest(float *sm, const Lv2 &L, const Sub2Args &a) {
  float *const b0 = sm + L.off, *const b1 = b0 + L.np;
  auto buf = [&](int k) { return k ? b1 : b0; };  // selects: no local-memory array
  const float *f = sm + L.off + 2 * L.np;
  const int n = L.Y * L.X;
  if (n <= 32) {
    if (threadIdx.x < 32) {
      const float v = sub2_coarsest_warp(L.w, f, L.Y, L.X, a.periodic, a.omega, a.coarse_sweeps);
      const int y = threadIdx.x / L.X, x = threadIdx.x - y * L.X;
      if (threadIdx.x < n) buf(0)[(y + 1) * L.P + x + 1] = v;
    }
    __syncthreads();
    return 0;
  }
  // buf(0) holds zeros (shared memory is cleared at the start)
  const Walk2 wk = walk2_of(L.X);
  int c = 0;
  for (int k = 0; k < a.coarse_sweeps; ++k) {
    sub2_sweep(L.w, buf(c), f, buf(c ^ 1), L.Y, L.X, wk, a.periodic, a.omega);
    c ^= 1;
  }
  return c;
}

// phi - P w (nearest prolongation of the coarser level's result wc), then the post-sweeps;
// the iterate starts in buffer c and the result's buffer is returned
__device__ __forceinline__ int sub2_up(float *sm, const Lv2 &L, const Lv2 &Lc, int c, int cc,
                                       const Sub2Args &a) {
  float *const b0 = sm + L.off, *const b1 = b0 + L.np;
  auto buf = [&](int k) { return k ? b1 : b0; };  // selects: no local-memory array
  const float *f = sm + L.off + 2 * L.np;
  const float *wc = sm + Lc.off + cc * Lc.np;
  const Walk2 wk = walk2_of(L.X);
  const int P = L.P, Pc = Lc.P;
  float *ph = buf(c);
  walk2(wk, L.Y, L.X, [&](int, int y, int x) {
    const float v = ph[(y + 1) * P + x + 1] - wc[((y >> 1) + 1) * Pc + (x >> 1) + 1];
    put2(ph, P, L.Y, L.X, y, x, v, a.periodic);
  });
  __syncthreads();
  sub2_sweep(L.w, buf(c), f, buf(c ^ 1), L.Y, L.X, wk, a.periodic, a.nu_post ? a.omega : 0.f);
  c ^= 1;
  for (int k = 1; k < a.nu_post; ++k) {
    sub2_sweep(L.w, buf(c), f, buf(c ^ 1), L.Y, L.X, wk, a.periodic, a.omega);
    c ^= 1;
  }
  return c;
}

template <class T>
__global__ void __launch_bounds__(kSub2Threads) k2_subcycle(const __grid_constant__ Sub2Args a,
                                                            const T *__restrict__ rhs,
                                                            T *__restrict__ out) {
  extern __shared__ float sm2[];
  __shared__ Lv2 lv[kSub2Levels];
  const int nl = a.nlev;
  if (threadIdx.x < nl) {
    const int l = threadIdx.x;
    int o = 0;
    for (int k = 0; k < l; ++k) o += 2 * (a.Y[k] + 2) * (a.X[k] + 2) + a.Y[k] * a.X[k];
    Lv2 L;
    L.Y = a.Y[l];
    L.X = a.X[l];
    L.P = L.X + 2;
    L.np = (L.Y + 2) * L.P;
    L.off = o;
    L.w = a.w[l];
    lv[l] = L;
  }
  for (int i = threadIdx.x; i < a.smem_floats; i += blockDim.x) sm2[i] = 0.f;
  __syncthreads();  // the zeros land before the rhs below
  const int64_t b = blockIdx.x;
  const int Y0 = a.Y[0], X0 = a.X[0], n0 = Y0 * X0, P0 = X0 + 2;
  float *f0 = sm2 + 2 * (Y0 + 2) * P0;
  for (int i = threadIdx.x; i < n0; i += blockDim.x) f0[i] = St<T>::to(rhs[b * n0 + i]);
  __syncthreads();
  for (int l = 0; l < nl - 1; ++l) {
    const Lv2 L = lv[l], Lc = lv[l + 1];
    sub2_down(sm2, L, Lc, a);
  }
  const int cd = (a.nu_pre - 1) & 1;  // a level's iterate after its pre-sweeps
  int cc;
  {
    const Lv2 L = lv[nl - 1];
    cc = sub2_coarsest(sm2, L, a);
  }
  for (int l = nl - 2; l >= 0; --l) {
    const Lv2 L = lv[l], Lc = lv[l + 1];
    cc = sub2_up(sm2, L, Lc, cd, cc, a);
  }
  const float *res = sm2 + cc * (Y0 + 2) * P0;
  walk2(walk2_of(X0), Y0, X0, [&](int i, int y, int x) {
    out[b * n0 + i] = St<T>::from(res[(y + 1) * P0 + x + 1]);
  });
}

// Shared-memory bytes of k2_subcycle for nlev levels from Y x X (each coarser level halved)
size_t sub2_smem_bytes(int Y, int X, int nlev) {
  size_t n = 0;
  for (int l = 0; l < nlev; ++l, Y /= 2, X /= 2) n += (size_t)2 * (Y + 2) * (X + 2) + (size_t)Y * X;
  return n * sizeof(float);
}
constexpr size_t kSub2MaxSmem = 200 * 1024;

// Subtract each instance's mean (the constant null space of a periodic operator).  One
// thread-block cluster of kMeanCluster blocks per instance: each block sums its contiguous
// share in a fixed order (thread-strided, warp tree, warps in order), the blocks read the
// cluster's partial sums from each other's shared memory in rank order, and each subtracts
// the mean from its share - a single block per instance spent 89 us on a 512^2 grid.
constexpr int kMeanCluster = 8;
__global__ void __cluster_dims__(kMeanCluster, 1, 1) __launch_bounds__(1024)
    k2_mean_subtract(float *p, int64_t n) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double sh[32];
  __shared__ double part;
  __shared__ float mean;
  const int rank = (int)cl.block_rank();
  float *q = p + (int64_t)(blockIdx.x / kMeanCluster) * n;
  const int64_t lo = n * rank / kMeanCluster, hi = n * (rank + 1) / kMeanCluster;
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += q[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    part = t;
  }
  cl.sync();  // every block's partial sum is in its shared memory
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int r = 0; r < kMeanCluster; ++r) t += *cl.map_shared_rank(&part, r);
    mean = (float)(t / (double)n);
  }
  cl.sync();  // no block leaves while another may still read its partial
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) q[i] -= mean;
}

// ------------------------------------------------------------------ Kolmogorov stepper
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// out = base + c dt (nu L phi - U d/dx phi - V d/dy phi + F) for both velocity components,
// with (U, V) = (phi_u, phi_v), L the 5-point Laplacian, d/dx the central difference and
// F = (famp sin(fk y h), 0); doubly periodic grid of spacing h.
__global__ void __launch_bounds__(kT2) k2_ns_stage(const float *__restrict__ pu, const float *__restrict__ pv,
                                                   const float *__restrict__ bu, const float *__restrict__ bv,
                                                   float *__restrict__ ou, float *__restrict__ ov, int Y,
                                                   int X, float c, float dt, float nu, float h,
                                                   float famp, float fk) {
  const int64_t n = (int64_t)Y * X;
  const float ih = 1.f / h, ih2 = ih * ih, i2h = 0.5f * ih;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / X), x = (int)(i % X);
    const int64_t l = (int64_t)y * X + wrap(x - 1, X), r = (int64_t)y * X + wrap(x + 1, X);
    const int64_t d = (int64_t)wrap(y - 1, Y) * X + x, u = (int64_t)wrap(y + 1, Y) * X + x;
    const float U = pu[i], V = pv[i];
    const float lap_u = (pu[l] + pu[r] + pu[d] + pu[u] - 4.f * U) * ih2;
    const float lap_v = (pv[l] + pv[r] + pv[d] + pv[u] - 4.f * V) * ih2;
    const float ux = (pu[r] - pu[l]) * i2h, uy = (pu[u] - pu[d]) * i2h;
    const float vx = (pv[r] - pv[l]) * i2h, vy = (pv[u] - pv[d]) * i2h;
    const float force = famp * sinf(fk * (float)y * h);
    ou[i] = bu[i] + c * dt * (nu * lap_u - U * ux - V * uy + force);
    ov[i] = bv[i] + c * dt * (nu * lap_v - U * vx - V * vy);
  }
}

// f = -(du/dx + dv/dy) / dt  (right-hand side of -L p = f; central differences)
__global__ void __launch_bounds__(kT2) k2_ns_divergence(const float *__restrict__ u, const float *__restrict__ v,
                                                        float *__restrict__ f, int Y, int X, float h,
                                                        float dt) {
  const int64_t n = (int64_t)Y * X;
  const float i2h = 0.5f / h;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / X), x = (int)(i % X);
    const float div = (u[(int64_t)y * X + wrap(x + 1, X)] - u[(int64_t)y * X + wrap(x - 1, X)]) * i2h +
                      (v[(int64_t)wrap(y + 1, Y) * X + x] - v[(int64_t)wrap(y - 1, Y) * X + x]) * i2h;
    f[i] = -div / dt;
  }
}

// u -= dt dp/dx, v -= dt dp/dy (central differences)
__global__ void __launch_bounds__(kT2) k2_ns_project(float *__restrict__ u, float *__restrict__ v,
                                                     const float *__restrict__ p, int Y, int X, float h,
                                                     float dt) {
  const int64_t n = (int64_t)Y * X;
  const float i2h = 0.5f / h;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / X), x = (int)(i % X);
    u[i] -= dt * (p[(int64_t)y * X + wrap(x + 1, X)] - p[(int64_t)y * X + wrap(x - 1, X)]) * i2h;
    v[i] -= dt * (p[(int64_t)wrap(y + 1, Y) * X + x] - p[(int64_t)wrap(y - 1, Y) * X + x]) * i2h;
  }
}

int blocks2(int64_t n, int B) {
  int64_t want = (int64_t)sm_count() * 8 / (B > 0 ? B : 1);
  if (want < 1) want = 1;
  int64_t need = (n + kT2 - 1) / kT2;
  int64_t b = need < want ? need : want;
  return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

int check2(int B, int Y, int X) {
  if (B < 1 || Y < 1 || X < 1) return fail(HFM_ERR_BAD_ARG, "2D: extents must be >= 1");
  if (B > 65535) return fail(HFM_ERR_BAD_ARG, "2D: at most 65535 instances");
  return HFM_OK;
}

int check_dtype2(int dtype) {
  if (dtype != HFM_F32 && dtype != HFM_BF16) return fail(HFM_ERR_BAD_ARG, "2D: dtype must be F32 or BF16");
  return HFM_OK;
}

W9 w9_of(const float *w) {
  W9 k;
  for (int i = 0; i < 9; ++i) k.w[i] = w[i];
  return k;
}

template <class T>
Src2<T> src2(const void *base, const void *coarse, float sign, int Y, int X, unsigned flags) {
  Src2<T> s;
  s.base = (const T *)base;
  s.coarse = (const T *)coarse;
  s.sign = sign;
  s.cshift = (flags & HFM_FLAG_SAME_LEVEL_CORR) ? 0 : 1;
  s.stride = (int64_t)Y * X;
  s.cstride = (int64_t)(Y >> s.cshift) * (X >> s.cshift);
  s.Y = Y;
  s.X = X;
  s.Xc = X >> s.cshift;
  s.periodic = (flags & HFM_FLAG_PERIODIC) ? 1 : 0;
  return s;
}

}  // namespace
}  // namespace hfm

using namespace hfm;

#define HFM2_DT(dtype, ...)                                  \
  if ((dtype) == HFM_F32) {                                  \
    using T = float;                                         \
    __VA_ARGS__;                                             \
  } else {                                                   \
    using T = __nv_bfloat16;                                 \
    __VA_ARGS__;                                             \
  }

extern "C" {

int hfm_conv2d_k3(const float *x, float *y, int B, int Y, int X, const float *w9_host,
                  unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X))) return st;
  if (!x || !y || !w9_host) return fail(HFM_ERR_BAD_ARG, "hfm_conv2d_k3: NULL argument");
  if (x == y) return fail(HFM_ERR_BAD_ARG, "hfm_conv2d_k3: in-place call");
  const int64_t n = (int64_t)Y * X;
  k2_stencil<float, 0><<<dim3(blocks2(n, B), B), kT2, 0, (cudaStream_t)stream>>>(
      w9_of(w9_host), src2<float>(x, nullptr, 0.f, Y, X, flags), nullptr, y, 0.f);
  HFM_CHECK_LAUNCH("k2_stencil");
  return HFM_OK;
}

int hfm_restrict_avg2d(int dtype, const void *fine, void *coarse, int B, int Y, int X,
                       hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!fine || !coarse) return fail(HFM_ERR_BAD_ARG, "hfm_restrict_avg2d: NULL argument");
  if (Y < 2 || X < 2) return fail(HFM_ERR_BAD_ARG, "hfm_restrict_avg2d: extents must be >= 2");
  const int64_t nc = (int64_t)(Y / 2) * (X / 2);
  HFM2_DT(dtype, (k2_restrict<T><<<dim3(blocks2(nc, B), B), kT2, 0, (cudaStream_t)stream>>>(
                     (const T *)fine, (T *)coarse, Y, X)));
  HFM_CHECK_LAUNCH("k2_restrict");
  return HFM_OK;
}

int hfm_prolong_nearest2d(int dtype, const void *coarse, void *fine, int B, int Yc, int Xc,
                          hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Yc, Xc)) || (st = check_dtype2(dtype))) return st;
  if (!fine || !coarse) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_nearest2d: NULL argument");
  const int64_t nf = (int64_t)4 * Yc * Xc;
  HFM2_DT(dtype, (k2_prolong<T><<<dim3(blocks2(nf, B), B), kT2, 0, (cudaStream_t)stream>>>(
                     (const T *)coarse, (T *)fine, Yc, Xc)));
  HFM_CHECK_LAUNCH("k2_prolong");
  return HFM_OK;
}

int hfm_jacobi2d(int dtype, const float *w9_host, const void *base, const void *coarse,
                 float coarse_sign, const void *rhs, void *out, int B, int Y, int X, float omega,
                 unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_host || !out) return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: NULL argument");
  if (w9_host[4] == 0.f) return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: zero diagonal weight");
  if ((base && base == out) || (coarse && coarse == out))
    return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: out aliases an input");
  if (coarse && !(flags & HFM_FLAG_SAME_LEVEL_CORR) && ((Y | X) & 1))
    return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: coarse correction needs even extents");
  const int64_t n = (int64_t)Y * X;
  if (flags & HFM_FLAG_TWO_SWEEPS) {
    if (!rhs || rhs == out)
      return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: two sweeps need an rhs apart from out");
    if (base || coarse) {
      const dim3 grid((X + kTwoTX - 1) / kTwoTX, (Y + kTwoTY - 1) / kTwoTY, B);
      if (grid.y > 65535) return fail(HFM_ERR_BAD_ARG, "hfm_jacobi2d: two sweeps: Y too large");
      HFM2_DT(dtype, (k2_two_sweeps_tile<T><<<grid, kT2, 0, (cudaStream_t)stream>>>(
                         w9_of(w9_host), src2<T>(base, coarse, coarse_sign, Y, X, flags),
                         (const T *)rhs, (T *)out, omega)));
      HFM_CHECK_LAUNCH("k2_two_sweeps_tile");
      return HFM_OK;
    }
    HFM2_DT(dtype, {
      Sweep1Src<T> s;
      s.f = (const T *)rhs;
      s.omega = omega;
      s.diag = w9_host[4];
      s.stride = n;
      s.Y = Y;
      s.X = X;
      s.periodic = (flags & HFM_FLAG_PERIODIC) ? 1 : 0;
      k2_two_sweeps<T><<<dim3(blocks2(n, B), B), kT2, 0, (cudaStream_t)stream>>>(w9_of(w9_host), s, (T *)out);
    });
    HFM_CHECK_LAUNCH("k2_two_sweeps");
    return HFM_OK;
  }
  HFM2_DT(dtype, (k2_stencil<T, 2><<<dim3(blocks2(n, B), B), kT2, 0, (cudaStream_t)stream>>>(
                     w9_of(w9_host), src2<T>(base, coarse, coarse_sign, Y, X, flags),
                     (const T *)rhs, (T *)out, omega)));
  HFM_CHECK_LAUNCH("k2_stencil");
  return HFM_OK;
}

int hfm_residual2d(int dtype, const float *w9_host, const void *phi, const void *rhs, void *r,
                   int B, int Y, int X, unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_host || !phi || !r) return fail(HFM_ERR_BAD_ARG, "hfm_residual2d: NULL argument");
  if (phi == r) return fail(HFM_ERR_BAD_ARG, "hfm_residual2d: in-place call");
  const int64_t n = (int64_t)Y * X;
  HFM2_DT(dtype, (k2_stencil<T, 1><<<dim3(blocks2(n, B), B), kT2, 0, (cudaStream_t)stream>>>(
                     w9_of(w9_host), src2<T>(phi, nullptr, 0.f, Y, X, flags), (const T *)rhs,
                     (T *)r, 0.f)));
  HFM_CHECK_LAUNCH("k2_stencil");
  return HFM_OK;
}

int hfm_residual_restrict2d(int dtype, const float *w9_host, const void *phi, const void *rhs,
                            void *r_coarse, int B, int Y, int X, unsigned flags,
                            hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_host || !r_coarse) return fail(HFM_ERR_BAD_ARG, "hfm_residual_restrict2d: NULL argument");
  if ((Y | X) & 1) return fail(HFM_ERR_BAD_ARG, "hfm_residual_restrict2d: extents must be even");
  const int64_t nc = (int64_t)(Y / 2) * (X / 2);
  HFM2_DT(dtype, (k2_resid_restrict<T, T><<<dim3(blocks2(nc, B), B), kT2, 0, (cudaStream_t)stream>>>(
                     w9_of(w9_host), src2<T>(phi, nullptr, 0.f, Y, X, flags), (const T *)rhs,
                     (T *)r_coarse, nc)));
  HFM_CHECK_LAUNCH("k2_resid_restrict");
  return HFM_OK;
}

int hfm_pre2_restrict2d(int dtype, const float *w9_host, const void *rhs, void *phi,
                        void *coarse_rhs, int B, int Y, int X, float omega, unsigned flags,
                        hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_host || !rhs || !phi || !coarse_rhs || rhs == phi || rhs == coarse_rhs || phi == coarse_rhs)
    return fail(HFM_ERR_BAD_ARG, "hfm_pre2_restrict2d: NULL or aliased fields");
  if (w9_host[4] == 0.f) return fail(HFM_ERR_BAD_ARG, "hfm_pre2_restrict2d: zero diagonal weight");
  if ((Y | X) & 1) return fail(HFM_ERR_BAD_ARG, "hfm_pre2_restrict2d: extents must be even");
  const dim3 grid((X + kTwoTX - 1) / kTwoTX, (Y + kTwoTY - 1) / kTwoTY, B);
  if (grid.y > 65535) return fail(HFM_ERR_BAD_ARG, "hfm_pre2_restrict2d: Y too large");
  HFM2_DT(dtype, {
    Sweep1Src<T> s;
    s.f = (const T *)rhs;
    s.omega = omega;
    s.diag = w9_host[4];
    s.stride = (int64_t)Y * X;
    s.Y = Y;
    s.X = X;
    s.periodic = (flags & HFM_FLAG_PERIODIC) ? 1 : 0;
    k2_pre2_restrict<T><<<grid, kT2, 0, (cudaStream_t)stream>>>(w9_of(w9_host), s, (T *)phi,
                                                               (T *)coarse_rhs);
  });
  HFM_CHECK_LAUNCH("k2_pre2_restrict");
  return HFM_OK;
}

int hfm_outer_residual2d(const float *w9_host, const float *phi, const float *rhs, int out_dtype,
                         void *r, int B, int Y, int X, unsigned flags, double *partials,
                         int *nblk_out, hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(out_dtype))) return st;
  if (!w9_host || !phi || !rhs || !r) return fail(HFM_ERR_BAD_ARG, "hfm_outer_residual2d: NULL argument");
  const int64_t n = (int64_t)Y * X;
  const int nb = blocks2(n, B);
  if (nblk_out) *nblk_out = nb;
  HFM2_DT(out_dtype, (k2_outer_resid<T><<<dim3(nb, B), kT2, 0, (cudaStream_t)stream>>>(
                         w9_of(w9_host), src2<float>(phi, nullptr, 0.f, Y, X, flags), rhs, (T *)r,
                         partials)));
  HFM_CHECK_LAUNCH("k2_outer_resid");
  return HFM_OK;
}

int hfm_update2d(float *p, int dtype, const void *w, float sign, int64_t n, hfm_stream_t stream) {
  int st;
  if ((st = check_dtype2(dtype))) return st;
  if (!p || !w || n < 1) return fail(HFM_ERR_BAD_ARG, "hfm_update2d: bad argument");
  HFM2_DT(dtype, (k2_update<T><<<blocks2(n, 1), kT2, 0, (cudaStream_t)stream>>>(p, (const T *)w, sign, n)));
  HFM_CHECK_LAUNCH("k2_update");
  return HFM_OK;
}

int hfm_coarse_jacobi2d(int dtype, const float *w9_host, const void *rhs, void *out, int B, int Y,
                        int X, float omega, int sweeps, unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_host || !rhs || !out || sweeps < 0) return fail(HFM_ERR_BAD_ARG, "hfm_coarse_jacobi2d: bad argument");
  if ((int64_t)Y * X > 4096) return fail(HFM_ERR_BAD_ARG, "hfm_coarse_jacobi2d: at most 4096 cells");
  if (w9_host[4] == 0.f) return fail(HFM_ERR_BAD_ARG, "hfm_coarse_jacobi2d: zero diagonal weight");
  const size_t smem = (size_t)3 * Y * X * sizeof(float);
  HFM2_DT(dtype, (k2_coarse_jacobi<T><<<B, kT2, smem, (cudaStream_t)stream>>>(
                     w9_of(w9_host), (const T *)rhs, (T *)out, Y, X, omega, sweeps,
                     (flags & HFM_FLAG_PERIODIC) ? 1 : 0)));
  HFM_CHECK_LAUNCH("k2_coarse_jacobi");
  return HFM_OK;
}

int hfm_subcycle2d(int dtype, const float *w9_levels, const void *rhs, void *out, int B, int Y, int X,
                   int nlev, float omega, int nu_pre, int nu_post, int coarse_sweeps, unsigned flags,
                   hfm_stream_t stream) {
  int st;
  if ((st = check2(B, Y, X)) || (st = check_dtype2(dtype))) return st;
  if (!w9_levels || !rhs || !out || nlev < 1 || nlev > kSub2Levels || nu_pre < 1 || nu_post < 0 ||
      coarse_sweeps < 0)
    return fail(HFM_ERR_BAD_ARG, "hfm_subcycle2d: bad argument");
  if ((int64_t)Y * X > 4096) return fail(HFM_ERR_BAD_ARG, "hfm_subcycle2d: at most 4096 cells on the first level");
  Sub2Args a;
  a.nlev = nlev;
  a.periodic = (flags & HFM_FLAG_PERIODIC) ? 1 : 0;
  a.nu_pre = nu_pre;
  a.nu_post = nu_post;
  a.coarse_sweeps = coarse_sweeps;
  a.omega = omega;
  for (int l = 0; l < nlev; ++l) {
    a.Y[l] = l ? a.Y[l - 1] / 2 : Y;
    a.X[l] = l ? a.X[l - 1] / 2 : X;
    if (a.Y[l] < 1 || a.X[l] < 1) return fail(HFM_ERR_BAD_ARG, "hfm_subcycle2d: too many levels");
    if (l + 1 < nlev && ((a.Y[l] & 1) || (a.X[l] & 1)))
      return fail(HFM_ERR_BAD_ARG, "hfm_subcycle2d: odd extent above the coarsest level");
    if (w9_levels[9 * l + 4] == 0.f) return fail(HFM_ERR_BAD_ARG, "hfm_subcycle2d: zero diagonal weight");
    a.w[l] = w9_of(w9_levels + 9 * l);
  }
  for (int l = nlev; l < kSub2Levels; ++l) a.Y[l] = a.X[l] = 0;
  const size_t smem = sub2_smem_bytes(Y, X, nlev);
  if (smem > kSub2MaxSmem) return fail(HFM_ERR_UNSUPPORTED, "hfm_subcycle2d: levels exceed shared memory");
  a.smem_floats = (int)(smem / sizeof(float));
  HFM2_DT(dtype, {
    if ((st = set_max_dynamic_smem((const void *)k2_subcycle<T>, (int)kSub2MaxSmem,
                                   "cudaFuncSetAttribute(k2_subcycle)")))
      return st;
    k2_subcycle<T><<<B, kSub2Threads, smem, (cudaStream_t)stream>>>(a, (const T *)rhs, (T *)out);
  });
  HFM_CHECK_LAUNCH("k2_subcycle");
  return HFM_OK;
}

int hfm_mean_subtract2d(float *p, int B, int64_t n, hfm_stream_t stream) {
  if (!p || B < 1 || n < 1) return fail(HFM_ERR_BAD_ARG, "hfm_mean_subtract2d: bad argument");
  if ((int64_t)B * kMeanCluster > INT32_MAX) return fail(HFM_ERR_BAD_ARG, "hfm_mean_subtract2d: too many instances");
  k2_mean_subtract<<<B * kMeanCluster, 1024, 0, (cudaStream_t)stream>>>(p, n);
  HFM_CHECK_LAUNCH("k2_mean_subtract");
  return HFM_OK;
}

int hfm_kolmogorov_stage(const float *phi_u, const float *phi_v, const float *base_u,
                         const float *base_v, float *out_u, float *out_v, int Y, int X, float c,
                         float dt, float nu, float h, float famp, float fk, hfm_stream_t stream) {
  int st;
  if ((st = check2(1, Y, X))) return st;
  if (!phi_u || !phi_v || !base_u || !base_v || !out_u || !out_v)
    return fail(HFM_ERR_BAD_ARG, "hfm_kolmogorov_stage: NULL argument");
  if (out_u == phi_u || out_v == phi_v || out_u == phi_v || out_v == phi_u)
    return fail(HFM_ERR_BAD_ARG, "hfm_kolmogorov_stage: outputs alias the differentiated fields");
  const int64_t n = (int64_t)Y * X;
  k2_ns_stage<<<blocks2(n, 1), kT2, 0, (cudaStream_t)stream>>>(phi_u, phi_v, base_u, base_v, out_u,
                                                               out_v, Y, X, c, dt, nu, h, famp, fk);
  HFM_CHECK_LAUNCH("k2_ns_stage");
  return HFM_OK;
}

int hfm_kolmogorov_divergence(const float *u, const float *v, float *f, int Y, int X, float h,
                              float dt, hfm_stream_t stream) {
  int st;
  if ((st = check2(1, Y, X))) return st;
  if (!u || !v || !f) return fail(HFM_ERR_BAD_ARG, "hfm_kolmogorov_divergence: NULL argument");
  const int64_t n = (int64_t)Y * X;
  k2_ns_divergence<<<blocks2(n, 1), kT2, 0, (cudaStream_t)stream>>>(u, v, f, Y, X, h, dt);
  HFM_CHECK_LAUNCH("k2_ns_divergence");
  return HFM_OK;
}

int hfm_kolmogorov_project(float *u, float *v, const float *p, int Y, int X, float h, float dt,
                           hfm_stream_t stream) {
  int st;
  if ((st = check2(1, Y, X))) return st;
  if (!u || !v || !p) return fail(HFM_ERR_BAD_ARG, "hfm_kolmogorov_project: NULL argument");
  const int64_t n = (int64_t)Y * X;
  k2_ns_project<<<blocks2(n, 1), kT2, 0, (cudaStream_t)stream>>>(u, v, p, Y, X, h, dt);
  HFM_CHECK_LAUNCH("k2_ns_project");
  return HFM_OK;
}

}  // extern "C"
