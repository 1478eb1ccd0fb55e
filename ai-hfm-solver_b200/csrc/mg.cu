// Multigrid handle: resident hierarchies for `slots` same-size instances, device-side
// convergence control and CUDA graphs of whole cycles.
//
// Cycle forms (sign convention r = A phi - b, phi -= P w, as in the reference):
//   SAWTOOTH  the reference loop (Anisotropic_3d_Multigrid_7point.ipynb:406-449,
//             BGS_multigrid_v1.ipynb cell 42, naiver_stokes_3D.py:646-703);
//   V / F     textbook cycles with nu_pre / nu_post weighted-Jacobi sweeps and a Jacobi
//             solve on the coarsest level;
//   accel CG  the V / F cycle (symmetric: nu_pre == nu_post) preconditions conjugate
//             gradients on the fine level.
// Every slot carries its own state on the device; a slot whose relative residual falls
// below tol (or that fails, or reaches max_cycles) is switched off by the check kernel and
// every later kernel skips it, so the host only polls between graph launches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <type_traits>
#include <vector>

#include "hfm_internal.cuh"

namespace hfm {

struct SlotState {
  int status;
  int cycles;        // cycles (stationary) or CG iterations (in total, for refinement)
  int sol_buf;
  int inner_cycles;  // CG iterations of the current (inner) solve
  double norm_b;
  double rel;        // last relative residual (outer residual for refinement)
  double rz;
  double pq;
  double rr;         // last ||r||^2 of the CG residual (scales the preconditioner input)
  double inner_norm; // refinement: ||b - A x|| when the current inner solve started
  int outer;         // refinement steps taken
  int first;         // refinement: the next outer step has no correction to add yet
};

namespace {

constexpr int kMaxLevels = 24;

__global__ void k_init_state(SlotState *st, int *active, int slot, const double *sumsq_b,
                             int status_if_zero, int *outer_mask) {
  double nb = sqrt(sumsq_b[0]);
  SlotState s;
  s.status = HFM_OK;
  s.cycles = 0;
  s.sol_buf = 0;

  s.norm_b = nb;
  s.rel = 1.0;
  s.rz = 0.0;
  s.pq = 0.0;
  s.inner_cycles = 0;
  s.rr = sumsq_b[0];
  s.inner_norm = nb;
  s.outer = 0;
  s.first = 1;
  int act = 1;
  if (!(nb > 0.0)) {
    s.rel = 0.0;
    act = 0;
    if (nb != nb) s.status = HFM_ERR_NAN;
    else s.status = status_if_zero;
  }
  st[slot] = s;
  if (outer_mask) {  // refinement starts with an outer step (residual of x0 in float64)
    outer_mask[slot] = act;
    active[slot] = 0;
  } else {
    active[slot] = act;
  }
}

// Sum the residual partials of each slot, update its state, switch it off when done.
// A TMA plane or drain wait expired somewhere on this device since the counters were last
// cleared (wf = the two wait-failure counters): the slot's data may come from an incomplete
// stage, so it ends with HFM_ERR_TIMEOUT instead of a status computed from that data.
__device__ __forceinline__ bool waits_failed(const int *wf) {
  return wf && (*(volatile const int *)&wf[0] | *(volatile const int *)&wf[1]);
}

__global__ void k_check(const double *__restrict__ partials, int nblk, SlotState *st,
                        int *active, double tol, int max_cycles, int which_buf, const int *wf,
                        const double *rz_new = nullptr) {
  const int inst = blockIdx.x;
  if (!active[inst]) return;
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += partials[(int64_t)inst * nblk + i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
    SlotState s = st[inst];
    double rel = sqrt(tot) / s.norm_b;
    s.rel = rel;
    s.rr = tot;
    if (rz_new) s.rz = rz_new[inst];  // CG: this iteration's r . z becomes the current one
    if (waits_failed(wf)) {
      s.status = HFM_ERR_TIMEOUT;
      s.sol_buf = which_buf;
      active[inst] = 0;
    } else if (!(rel == rel) || isinf(rel)) {
      s.status = HFM_ERR_NAN;
      s.sol_buf = which_buf;
      active[inst] = 0;
    } else if (rel < tol) {
      s.status = HFM_OK;
      s.sol_buf = which_buf;
      active[inst] = 0;
    } else if (s.cycles >= max_cycles) {
      s.status = HFM_ERR_NOT_CONVERGED;
      s.sol_buf = which_buf;
      active[inst] = 0;
    } else {
      s.cycles += 1;
      s.inner_cycles += 1;
    }
    st[inst] = s;
  }
}

// End of one inner CG iteration of the refinement: the inner solve stops when its residual
// reaches max(inner_tol * ||r0||, 0.3 tol ||b||) or after inner_max iterations, and hands
// the slot to the outer (float64) step.
__global__ void k_check_inner(const double *__restrict__ partials, int nblk, SlotState *st,
                              int *active, int *outer_mask, double tol, double inner_tol,
                              int inner_max, const int *wf, const double *rz_new) {
  const int inst = blockIdx.x;
  if (!active[inst]) return;
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += partials[(int64_t)inst * nblk + i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
    SlotState s = st[inst];
    s.rr = tot;
    s.rz = rz_new[inst];  // this iteration's r . z becomes the current one
    s.cycles += 1;
    s.inner_cycles += 1;
    const double r = sqrt(tot);
    const double target = fmax(inner_tol * s.inner_norm, 0.3 * tol * s.norm_b);
    if (waits_failed(wf)) {
      s.status = HFM_ERR_TIMEOUT;
      active[inst] = 0;
    } else if (!(r == r) || isinf(r)) {
      s.status = HFM_ERR_NAN;
      active[inst] = 0;
    } else if (r < target || s.inner_cycles >= inner_max) {
      active[inst] = 0;
      outer_mask[inst] = 1;
    }
    st[inst] = s;
  }
}

// Outer step bookkeeping: relative residual of the float64 solution; finish, or start the
// next inner solve from its residual.
__global__ void k_check_outer(const double *__restrict__ partials, int nblk, SlotState *st,
                              int *active, int *outer_mask, double tol, int max_cycles,
                              const int *wf) {
  const int inst = blockIdx.x;
  if (!outer_mask[inst]) return;
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += partials[(int64_t)inst * nblk + i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
    SlotState s = st[inst];
    const double r = sqrt(tot);
    const double rel = r / s.norm_b;
    s.rel = rel;
    s.outer += 1;
    s.first = 0;
    outer_mask[inst] = 0;
    if (waits_failed(wf)) {
      s.status = HFM_ERR_TIMEOUT;
    } else if (!(rel == rel) || isinf(rel)) {
      s.status = HFM_ERR_NAN;
    } else if (rel < tol) {
      s.status = HFM_OK;
    } else if (s.cycles >= max_cycles) {
      s.status = HFM_ERR_NOT_CONVERGED;
    } else {
      s.inner_norm = r;
      s.rr = tot;
      s.rz = 0.0;
      s.inner_cycles = 0;
      active[inst] = 1;
    }
    st[inst] = s;
  }
}

// float64 outer residual r = b - A x (sigma / kernel read as float32), partial sums of r^2.
// Work items of the vector kernels: (slot, chunk) pairs.  A block takes items blockIdx.x,
// blockIdx.x + gridDim.x, ...; chunk c of a slot covers elements [n c / CH, n (c+1) / CH).
// Items of inactive slots are skipped, so however few slots are active the whole grid works
// on them; reductions produce one partial per (slot, chunk), independent of which block
// handled the item, so the summation order is fixed.
struct Items {
  int B, CH;
  int64_t n;
};

__device__ __forceinline__ double block_reduce_sum(double v) {
  __shared__ double sh[32];
  __syncthreads();  // sh is reused across items
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

// When n is a multiple of 4 the chunk bounds are too, so the kernels below can move 16 bytes of
// float32 (8 of 16-bit) per access: v4 loops run i over lo, lo + 4, ... with vector loads.
__host__ __device__ __forceinline__ int64_t item_bound(int64_t n, int ch, int CH) {
  return (n & 3) ? n * ch / CH : 4 * ((n >> 2) * ch / CH);
}
#define HFM_FOR_ITEMS(it, MASK)                                                   \
  for (int w_ = blockIdx.x; w_ < (it).B * (it).CH; w_ += gridDim.x) {            \
    const int slot = w_ / (it).CH, ch = w_ - slot * (it).CH;                     \
    if (!(MASK)) continue;                                                        \
    const int64_t lo = item_bound((it).n, ch, (it).CH), hi = item_bound((it).n, ch + 1, (it).CH); \
    const int64_t base = (int64_t)slot * (it).n;                                  \
    const bool v4 = ((it).n & 3) == 0;                                            \
    (void)base;                                                                   \
    (void)v4;
#define HFM_END_ITEMS }

// Four consecutive values as float4 / stored from float4 (16-byte float32, 8-byte 16-bit).
template <class T> __device__ __forceinline__ float4 ld4v(const T *p);
template <> __device__ __forceinline__ float4 ld4v<float>(const float *p) {
  return *reinterpret_cast<const float4 *>(p);
}
template <> __device__ __forceinline__ float4 ld4v<__nv_bfloat16>(const __nv_bfloat16 *p) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
template <> __device__ __forceinline__ float4 ld4v<__half>(const __half *p) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p);
  const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
template <class T> __device__ __forceinline__ void st4v(T *p, float4 v) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = v;
  } else {
    T a[4] = {St<T>::from(v.x), St<T>::from(v.y), St<T>::from(v.z), St<T>::from(v.w)};
    *reinterpret_cast<uint2 *>(p) = *reinterpret_cast<const uint2 *>(a);
  }
}

// x64 += x_in for slots whose outer step is due (not before the first inner solve).
__global__ void k_ir_update(double *__restrict__ x64, const float *__restrict__ xin, Items it,
                            const SlotState *st, const int *outer_mask) {
  HFM_FOR_ITEMS(it, outer_mask[slot] && !st[slot].first)
  if (v4) {
    for (int64_t i = lo + 4 * threadIdx.x; i < hi; i += 4 * blockDim.x) {
      const float4 v = ld4v<float>(xin + base + i);
      double2 *d = reinterpret_cast<double2 *>(x64 + base + i);
      double2 a = d[0], b = d[1];
      a.x += v.x; a.y += v.y; b.x += v.z; b.y += v.w;
      d[0] = a;
      d[1] = b;
    }
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) x64[base + i] += (double)xin[base + i];
  }
  HFM_END_ITEMS
}

// float64 outer residual r = b - A x (sigma / kernel read as float32), written as the float32
// right-hand side of the next inner solve (and, when `rstore` is given, as the 16-bit copy the
// inner cycle reads), with partial sums of r^2.
template <int KIND, class T>
__global__ void k_residual64(DevOp op, const double *__restrict__ x, const double *__restrict__ b,
                             float *__restrict__ rout, T *__restrict__ rstore, int Z, int Y, int X,
                             Items it, const int *__restrict__ mask, double *__restrict__ partials) {
  HFM_FOR_ITEMS(it, mask[slot])
  const double *xi = x + base;
  auto P = [&](int zz, int yy, int xx) -> double {
    if (zz < 0 || zz >= Z || yy < 0 || yy >= Y || xx < 0 || xx >= X) return 0.0;
    return xi[((int64_t)zz * Y + yy) * X + xx];
  };
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const int xx = (int)(i % X);
    const int64_t t = i / X;
    const int yy = (int)(t % Y), zz = (int)(t / Y);
    double ax;
    if (KIND == HFM_OP_K27) {
      ax = 0.0;
      for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb)
          for (int c = 0; c < 3; ++c) {
            const float wgt = op.k[9 * a + 3 * bb + c];
            if (wgt != 0.f) ax += (double)wgt * P(zz + a - 1, yy + bb - 1, xx + c - 1);
          }
    } else if (KIND == HFM_OP_CONST7) {
      const double kz = op.k[0], ky = op.k[1], kx = op.k[2];
      ax = 2.0 * (kz + ky + kx) * P(zz, yy, xx) - kz * (P(zz - 1, yy, xx) + P(zz + 1, yy, xx)) -
           ky * (P(zz, yy - 1, xx) + P(zz, yy + 1, xx)) - kx * (P(zz, yy, xx - 1) + P(zz, yy, xx + 1));
    } else {
      const float *sx = (const float *)op.coef[0] + (int64_t)slot * op.coef_stride;
      const float *sy = (const float *)op.coef[1] + (int64_t)slot * op.coef_stride;
      const float *sz = (const float *)op.coef[2] + (int64_t)slot * op.coef_stride;
      const double sc = op.scale;
      const double cz = op.c[0] * sc, cy = op.c[1] * sc, cx = op.c[2] * sc;
      const double vx = sx[i], vy = sy[i], vz = sz[i];
      const int64_t PL = (int64_t)X * Y;
      const double axm = cx * (xx > 0 ? 0.5 * (vx + sx[i - 1]) : vx);
      const double axp = cx * (xx < X - 1 ? 0.5 * (vx + sx[i + 1]) : vx);
      const double aym = cy * (yy > 0 ? 0.5 * (vy + sy[i - X]) : vy);
      const double ayp = cy * (yy < Y - 1 ? 0.5 * (vy + sy[i + X]) : vy);
      const double azm = cz * (zz > 0 ? 0.5 * (vz + sz[i - PL]) : vz);
      const double azp = cz * (zz < Z - 1 ? 0.5 * (vz + sz[i + PL]) : vz);
      const double pc = P(zz, yy, xx);
      ax = axm * (pc - P(zz, yy, xx - 1)) + axp * (pc - P(zz, yy, xx + 1)) +
           aym * (pc - P(zz, yy - 1, xx)) + ayp * (pc - P(zz, yy + 1, xx)) +
           azm * (pc - P(zz - 1, yy, xx)) + azp * (pc - P(zz + 1, yy, xx));
    }
    const double r = b[base + i] - ax;
    rout[base + i] = (float)r;
    if (rstore) rstore[base + i] = St<T>::from((float)r);
    acc += r * r;
  }
  const double t = block_reduce_sum(acc);
  if (threadIdx.x == 0) partials[(int64_t)slot * it.CH + ch] = t;
  HFM_END_ITEMS
}

// The same float64 outer residual for SIGMA7 with X % 4 == 0: a thread takes four
// consecutive cells of a row (one index computation, 32-byte loads of x64 / b64 and 16-byte
// loads of the conductivities), rows of a slot indexed in 32 bits (n < 2^31).
template <class T>
__global__ void k_residual64_sigma4(DevOp op, const double *__restrict__ x,
                                    const double *__restrict__ b, float *__restrict__ rout,
                                    T *__restrict__ rstore, int Z, int Y, int X, Items it,
                                    const int *__restrict__ mask, double *__restrict__ partials) {
  HFM_FOR_ITEMS(it, mask[slot])
  const double *xi = x + base;
  const float *sx = (const float *)op.coef[0] + (int64_t)slot * op.coef_stride;
  const float *sy = (const float *)op.coef[1] + (int64_t)slot * op.coef_stride;
  const float *sz = (const float *)op.coef[2] + (int64_t)slot * op.coef_stride;
  const double sc = op.scale;
  const double cz = op.c[0] * sc, cy = op.c[1] * sc, cx = op.c[2] * sc;
  const int PL = X * Y;
  double acc = 0.0;
  for (int64_t i64 = lo + 4 * threadIdx.x; i64 < hi; i64 += 4 * blockDim.x) {
    const int i = (int)i64;
    const int row = i / X, xx = i - row * X;
    const int yy = row % Y, zz = row / Y;
    auto ld4d = [](const double *p, double (&v)[4]) {
      const double2 a = *reinterpret_cast<const double2 *>(p), c = *reinterpret_cast<const double2 *>(p + 2);
      v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y;
    };
    auto ld4f = [](const float *p, double (&v)[4]) {
      const float4 a = *reinterpret_cast<const float4 *>(p);
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    };
    double pc[4], pym[4] = {0, 0, 0, 0}, pyp[4] = {0, 0, 0, 0}, pzm[4] = {0, 0, 0, 0}, pzp[4] = {0, 0, 0, 0};
    double vx[4], vy[4], vz[4], sym[4], syp[4], szm[4], szp[4];
    ld4d(xi + i, pc);
    ld4f(sx + i, vx);
    ld4f(sy + i, vy);
    ld4f(sz + i, vz);
    const bool ylo = yy > 0, yhi = yy < Y - 1, zlo = zz > 0, zhi = zz < Z - 1;
    if (ylo) ld4d(xi + i - X, pym);
    if (yhi) ld4d(xi + i + X, pyp);
    if (zlo) ld4d(xi + i - PL, pzm);
    if (zhi) ld4d(xi + i + PL, pzp);
    ld4f(ylo ? sy + i - X : sy + i, sym);
    ld4f(yhi ? sy + i + X : sy + i, syp);
    ld4f(zlo ? sz + i - PL : sz + i, szm);
    ld4f(zhi ? sz + i + PL : sz + i, szp);
    const double pl = xx > 0 ? xi[i - 1] : 0.0, pr = xx + 4 < X ? xi[i + 4] : 0.0;
    const double sl = xx > 0 ? (double)sx[i - 1] : 0.0, sr = xx + 4 < X ? (double)sx[i + 4] : 0.0;
    double bb[4];
    ld4d(b + base + i, bb);
    float rr[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int xe = xx + e;
      const double vxl = e == 0 ? sl : vx[e - 1], vxr = e == 3 ? sr : vx[e + 1];
      const double axm = cx * (xe > 0 ? 0.5 * (vx[e] + vxl) : vx[e]);
      const double axp = cx * (xe < X - 1 ? 0.5 * (vx[e] + vxr) : vx[e]);
      const double aym = cy * (ylo ? 0.5 * (vy[e] + sym[e]) : vy[e]);
      const double ayp = cy * (yhi ? 0.5 * (vy[e] + syp[e]) : vy[e]);
      const double azm = cz * (zlo ? 0.5 * (vz[e] + szm[e]) : vz[e]);
      const double azp = cz * (zhi ? 0.5 * (vz[e] + szp[e]) : vz[e]);
      const double xl = e == 0 ? pl : pc[e - 1], xr = e == 3 ? pr : pc[e + 1];
      const double ax = axm * (pc[e] - xl) + axp * (pc[e] - xr) + aym * (pc[e] - pym[e]) +
                        ayp * (pc[e] - pyp[e]) + azm * (pc[e] - pzm[e]) + azp * (pc[e] - pzp[e]);
      const double r = bb[e] - ax;
      rr[e] = (float)r;
      acc += r * r;
    }
    *reinterpret_cast<float4 *>(rout + base + i) = make_float4(rr[0], rr[1], rr[2], rr[3]);
    if (rstore) st4v<T>(rstore + base + i, make_float4(rr[0], rr[1], rr[2], rr[3]));
  }
  const double t = block_reduce_sum(acc);
  if (threadIdx.x == 0) partials[(int64_t)slot * it.CH + ch] = t;
  HFM_END_ITEMS
}

template <class T>
__global__ void k_fetch(const T *__restrict__ b0, const T *__restrict__ b1,
                        const float *__restrict__ bx, int64_t n, const SlotState *st,
                        const int *active, int slot, float *__restrict__ out) {
  const int which = active[slot] ? 0 : st[slot].sol_buf;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v;
    if (bx) v = bx[i];
    else v = St<T>::to(which ? b1[i] : b0[i]);
    out[i] = v;
  }
}

__global__ void k_to_f64(const void *__restrict__ src, int dt, double *__restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = dt == HFM_F64 ? ((const double *)src)[i] : (double)((const float *)src)[i];
}

__global__ void k_f64_to_f32(const double *__restrict__ src, float *__restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

__global__ void k_sumsq64(const double *__restrict__ x, int64_t n, double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t inst = blockIdx.y;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[inst * n + i];
    acc += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    partials[inst * gridDim.x + blockIdx.x] = t;
  }
}

// Pack the public per-slot statistics (for the asynchronous query).
__global__ void k_pack_stats(const SlotState *st, const int *active, const int *outer, int B,
                             hfm_slot_stats *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  hfm_slot_stats o;
  o.active = active[i] | (outer ? outer[i] : 0);
  o.status = st[i].status;
  o.cycles = st[i].cycles;
  o.outer = st[i].outer;
  o.norm_b = st[i].norm_b;
  o.rel_resid = st[i].rel;
  out[i] = o;
}

// Geometric mean of a slot's three conductivity arrays (one block per slot).
__global__ void k_log_mean(const void *sx, const void *sy, const void *sz, int dt, int64_t n,
                           int slot0, double *gscale) {
  __shared__ double sh[32];
  const int64_t sl = blockIdx.x;
  const void *arr[3] = {sx, sy, sz};
  double acc = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      const int64_t k = sl * n + i;
      const double v = dt == HFM_F64 ? ((const double *)arr[a])[k] : (double)((const float *)arr[a])[k];
      acc += log(v);
    }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    gscale[slot0 + sl] = exp(t / (3.0 * (double)n));
  }
}

// Admission of a slot's conductivities in one launch: blockIdx.y picks sx / sy / sz; each
// cell is stored in the storage type (divided by the slot's geometric mean when gscale is
// given) and, where the handle keeps one, as a float32 copy for the float32 operator.
template <class T> struct Admit3 {
  const void *src[3];
  T *dst[3];
  float *dst32[3];
};
template <class T>
__global__ void k_admit_convert(Admit3<T> a, int dt, int64_t n, int count, int slot0,
                                const double *gscale) {
  const void *src = a.src[blockIdx.y];
  T *dst = a.dst[blockIdx.y];
  float *d32 = a.dst32[blockIdx.y];
  const int64_t tot = n * count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = dt == HFM_F64 ? ((const double *)src)[i] : (double)((const float *)src)[i];
    dst[i] = St<T>::from(gscale ? (float)(v / gscale[slot0 + i / n]) : (float)v);
    if (d32) d32[i] = (float)v;
  }
}

// 1 / diagonal of every SIGMA7 level of the slots [slot0, slot0 + gridDim.y) in one launch:
// the blocks of blockIdx.x are split over the levels by the prefix sums in first[]; indices
// inside one instance are 32-bit (an instance has fewer than 2^31 cells).
struct InvdLevels {
  const void *sx[kMaxLevels], *sy[kMaxLevels], *sz[kMaxLevels];
  void *out[kMaxLevels];
  float cz[kMaxLevels], cy[kMaxLevels], cx[kMaxLevels];
  int Z[kMaxLevels], Y[kMaxLevels], X[kMaxLevels];
  int first[kMaxLevels + 1];
  int L;
};
template <class T>
__global__ void __launch_bounds__(256) k_invdiag_levels(const InvdLevels d, int slot0) {
  int l = 0;
  while (l + 1 < d.L && (int)blockIdx.x >= d.first[l + 1]) ++l;
  const int Z = d.Z[l], Y = d.Y[l], X = d.X[l], P = X * Y, n = P * Z;
  const int64_t o = (int64_t)(slot0 + blockIdx.y) * n;
  const T *sx = (const T *)d.sx[l] + o, *sy = (const T *)d.sy[l] + o, *sz = (const T *)d.sz[l] + o;
  T *out = (T *)d.out[l] + o;
  const float cz = d.cz[l], cy = d.cy[l], cx = d.cx[l];
  const float hz = 0.5f * cz, hy = 0.5f * cy, hx = 0.5f * cx;
  const int nb = d.first[l + 1] - d.first[l];
  for (int i = ((int)blockIdx.x - d.first[l]) * 256 + (int)threadIdx.x; i < n; i += nb * 256) {
    const int x = i % X, t = i / X, y = t % Y, z = t / Y;
    const float vx = St<T>::to(sx[i]), vy = St<T>::to(sy[i]), vz = St<T>::to(sz[i]);
    const float axm = x > 0 ? hx * (vx + St<T>::to(sx[i - 1])) : cx * vx;
    const float axp = x < X - 1 ? hx * (vx + St<T>::to(sx[i + 1])) : cx * vx;
    const float aym = y > 0 ? hy * (vy + St<T>::to(sy[i - X])) : cy * vy;
    const float ayp = y < Y - 1 ? hy * (vy + St<T>::to(sy[i + X])) : cy * vy;
    const float azm = z > 0 ? hz * (vz + St<T>::to(sz[i - P])) : cz * vz;
    const float azp = z < Z - 1 ? hz * (vz + St<T>::to(sz[i + P])) : cz * vz;
    out[i] = St<T>::from(1.f / (((axm + axp) + (aym + ayp)) + (azm + azp)));
  }
}

template <class T>
__global__ void k_copy_active(const T *__restrict__ src, T *__restrict__ dst, int64_t n,
                              const int *active) {
  const int64_t inst = blockIdx.y;
  if (!active[inst]) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[inst * n + i] = src[inst * n + i];
}

// Initial state of every slot from its ||b||^2 (batched load).
__global__ void k_init_states(SlotState *st, int *active, int B, const double *sumsq_b,
                              int *outer_mask) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  double nb = sqrt(sumsq_b[i]);
  SlotState s;
  s.status = HFM_OK;
  s.cycles = 0;
  s.sol_buf = 0;

  s.norm_b = nb;
  s.rel = 1.0;
  s.rz = 0.0;
  s.pq = 0.0;
  s.inner_cycles = 0;
  s.rr = sumsq_b[i];
  s.inner_norm = nb;
  s.outer = 0;
  s.first = 1;
  int act = 1;
  if (!(nb > 0.0)) {
    s.rel = 0.0;
    act = 0;
    s.status = (nb != nb) ? HFM_ERR_NAN : HFM_OK;
  }
  st[i] = s;
  if (outer_mask) {
    outer_mask[i] = act;
    active[i] = 0;
  } else {
    active[i] = act;
  }
}

template <class T>
__global__ void k_fetch_all(const T *__restrict__ b0, const T *__restrict__ b1,
                            const float *__restrict__ bx, int64_t n, const SlotState *st,
                            const int *active, float *__restrict__ out) {
  const int64_t slot = blockIdx.y;
  const int which = active[slot] ? 0 : st[slot].sol_buf;
  const int64_t o = slot * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[o + i] = bx ? bx[o + i] : St<T>::to(which ? b1[o + i] : b0[o + i]);
}

// ----------------------------------------------------------------- CG vector kernels
// Scale of the preconditioner input for fp16 storage.  scaled = 0: none (float32 / bf16 have
// the exponent range of float32); 2: fp16 - the cycle solves for r / s with s = RMS(r) =
// |r|_2 / sqrt(n), with conductivities divided by their geometric mean g, so
// z = (s / g) M'(r / s).  Entries of r / s are O(1) and at most sqrt(n) (a single spike), well
// inside fp16's range on both sides: normalising by |r|_2 instead pushed typical entries of a
// 256^3 residual (~1 / sqrt(n)) into fp16's subnormal range, and the refinement stalled near
// 1e-9.  pc_in is the divisor of the input, pc_out the factor of the output.
__device__ __forceinline__ float pc_in(const SlotState &s, int64_t n, int scaled) {
  return (scaled == 2 && s.rr > 0.0) ? (float)sqrt(s.rr / (double)n) : 1.f;
}
__device__ __forceinline__ float pc_out(const SlotState &s, int64_t n, int scaled,
                                        const double *gscale, int64_t slot) {
  return scaled == 2 ? (float)(pc_in(s, n, scaled) / gscale[slot]) : 1.f;
}

template <class TZ>
__global__ void k_dot_partials(const float *__restrict__ a, const TZ *__restrict__ b, Items it,
                               double *partials, const int *active, const SlotState *st,
                               int scaled, const double *gscale) {
  HFM_FOR_ITEMS(it, active[slot])
  const double zs = st ? pc_out(st[slot], it.n, scaled, gscale, slot) : 1.0;
  double acc = 0.0;
  if (v4) {
    for (int64_t i = lo + 4 * threadIdx.x; i < hi; i += 4 * blockDim.x) {
      const float4 av = ld4v<float>(a + base + i), bv = ld4v<TZ>(b + base + i);
      acc += (double)av.x * bv.x + (double)av.y * bv.y + (double)av.z * bv.z + (double)av.w * bv.w;
    }
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
      acc += (double)a[base + i] * (double)St<TZ>::ld(b + base + i);
  }
  const double t = block_reduce_sum(acc * zs);
  if (threadIdx.x == 0) partials[(int64_t)slot * it.CH + ch] = t;
  HFM_END_ITEMS
}

// Sum of one slot's nblk partial sums in a fixed order (256 threads: a thread-strided sum, a
// warp tree, then the warps in order), so every block that computes it gets the same value.
__device__ double slot_sum(const double *__restrict__ p, int nblk) {
  __shared__ double sh[32];
  __shared__ double res;
  __syncthreads();  // sh / res are reused across items
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += p[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    res = t;
  }
  __syncthreads();
  return res;
}

// p = z + beta p (beta = rz_new / rz; first iteration p = z).  rz_new = r . z is summed here
// from the slot's nblk_rz partials (every item of the slot sums them in the same order) and
// stored in rz_new[slot] by the slot's first chunk; the check at the end of the iteration
// makes it the current rz.
template <class TZ>
__global__ void k_cg_p(const TZ *__restrict__ z, float *__restrict__ p, Items it, SlotState *st,
                       const double *__restrict__ rz_part, int nblk_rz, double *rz_new,
                       const int *active, int scaled, const double *gscale) {
  HFM_FOR_ITEMS(it, active[slot])
  const double rzn = slot_sum(rz_part + (int64_t)slot * nblk_rz, nblk_rz);
  if (ch == 0 && threadIdx.x == 0) rz_new[slot] = rzn;
  const SlotState s = st[slot];
  const bool first = s.inner_cycles == 0 || s.rz == 0.0;
  const float beta = first ? 0.f : (float)(rzn / s.rz);
  const float zs = pc_out(s, it.n, scaled, gscale, slot);
  if (v4) {
    // two 4-element groups per thread and iteration, their loads issued together: one group
    // (24 bytes in flight per thread) left the kernel latency-bound at 0.7 of the bandwidth
    const int64_t step = 4 * (int64_t)blockDim.x;
    for (int64_t i = lo + 4 * threadIdx.x; i < hi; i += 2 * step) {
      const int64_t j = i + step;
      const bool two = j < hi;
      const float4 zv = ld4v<TZ>(z + base + i);
      const float4 zw = two ? ld4v<TZ>(z + base + j) : make_float4(0.f, 0.f, 0.f, 0.f);
      float4 po = make_float4(0.f, 0.f, 0.f, 0.f), pw = po;
      if (!first) {
        po = ld4v<float>(p + base + i);
        if (two) pw = ld4v<float>(p + base + j);
      }
      float4 pv = make_float4(zs * zv.x, zs * zv.y, zs * zv.z, zs * zv.w);
      float4 px = make_float4(zs * zw.x, zs * zw.y, zs * zw.z, zs * zw.w);
      if (!first) {
        pv.x += beta * po.x;
        pv.y += beta * po.y;
        pv.z += beta * po.z;
        pv.w += beta * po.w;
        px.x += beta * pw.x;
        px.y += beta * pw.y;
        px.z += beta * pw.z;
        px.w += beta * pw.w;
      }
      st4v<float>(p + base + i, pv);
      if (two) st4v<float>(p + base + j, px);
    }
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      const float zv = zs * St<TZ>::ld(z + base + i);
      p[base + i] = first ? zv : zv + beta * p[base + i];
    }
  }
  HFM_END_ITEMS
}

// x += alpha p, r -= alpha q, partial sums of r^2; with `rstore` also the storage-type copy of
// the new r that the next iteration's cycle reads (bf16 refinement: no separate conversion).
// alpha = rz_new / p.q, with p.q summed here from the slot's nblk_pq partials of the operator
// pass (a buffer of its own: this kernel writes its r^2 partials into `partials`).  With
// `fresh` (refinement) the first iteration of an inner solve starts from x = 0: x = alpha p,
// x not read (no separate zeroing pass).
template <class T>
__global__ void k_cg_xr(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                        const float *__restrict__ q, T *__restrict__ rstore, Items it,
                        const double *__restrict__ pq_part, int nblk_pq,
                        const double *__restrict__ rz_new, double *partials, const int *active,
                        const SlotState *st, int fresh) {
  HFM_FOR_ITEMS(it, active[slot])
  const double pq = slot_sum(pq_part + (int64_t)slot * nblk_pq, nblk_pq);
  const float alpha = (pq != 0.0) ? (float)(rz_new[slot] / pq) : 0.f;
  const bool zx = fresh && st[slot].inner_cycles == 0;
  double acc = 0.0;
  if (v4) {
    for (int64_t i = lo + 4 * threadIdx.x; i < hi; i += 4 * blockDim.x) {
      const int64_t k = base + i;
      float4 xv = zx ? make_float4(0.f, 0.f, 0.f, 0.f) : ld4v<float>(x + k), rv = ld4v<float>(r + k);
      const float4 pv = ld4v<float>(p + k), qv = ld4v<float>(q + k);
      xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z; xv.w += alpha * pv.w;
      rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z; rv.w -= alpha * qv.w;
      st4v<float>(x + k, xv);
      st4v<float>(r + k, rv);
      if (rstore) st4v<T>(rstore + k, rv);
      acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
    }
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      const int64_t k = base + i;
      x[k] = (zx ? 0.f : x[k]) + alpha * p[k];
      const float rv = r[k] - alpha * q[k];
      r[k] = rv;
      if (rstore) rstore[k] = St<T>::from(rv);
      acc += (double)rv * rv;
    }
  }
  const double t = block_reduce_sum(acc);
  if (threadIdx.x == 0) partials[(int64_t)slot * it.CH + ch] = t;
  HFM_END_ITEMS
}

// r = b - A x computed as -(A x - b): negate in place.
__global__ void k_negate(float *__restrict__ v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = -v[i];
}

template <class T>
__global__ void k_to_storage(const float *__restrict__ a, T *__restrict__ b, Items it,
                             const int *active, const SlotState *st, int scaled) {
  HFM_FOR_ITEMS(it, active[slot])
  const float inv = 1.f / pc_in(st[slot], it.n, scaled);
  if (v4) {
    for (int64_t i = lo + 4 * threadIdx.x; i < hi; i += 4 * blockDim.x) {
      const float4 v = ld4v<float>(a + base + i);
      st4v<T>(b + base + i, make_float4(v.x * inv, v.y * inv, v.z * inv, v.w * inv));
    }
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
      b[base + i] = St<T>::from(a[base + i] * inv);
  }
  HFM_END_ITEMS
}

// Chunks per slot for the vector kernels (about 4096 elements each) and their grid.
int item_chunks(int64_t n) {
  int64_t c = (n + 4095) / 4096;
  return (int)std::max<int64_t>(1, std::min<int64_t>(c, 4096));
}
int item_blocks(int B, int CH) {
  int64_t want = (int64_t)sm_count() * 8;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)B * CH));
}

int vec_blocks(int64_t n, int B) {
  int64_t want = (int64_t)sm_count() * 8 / std::max(B, 1);
  int64_t need = (n + 255) / 256;
  int64_t b = std::min(std::max<int64_t>(want, 1), need);
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 65535));
}

size_t dtype_size(int dt) { return dt == HFM_F32 ? 4 : 2; }

}  // namespace

struct Level {
  int Z, Y, X;
  int64_t n;
  void *phi = nullptr, *tmp = nullptr, *rhs = nullptr;
  void *coef[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void *invd = nullptr;  // SIGMA7: 1 / diagonal of the level's operator (two-sweep pass)
  DevOp op;
  // 16-bit SIGMA7 levels the plane-marching kernels take: the FACE7 arrays of the level's
  // operator (scale folded in) and that operator, used by every sweep and residual there
  void *face[3] = {nullptr, nullptr, nullptr};
  DevOp fop;
};

// A level of a handle holds FACE7 arrays: 16-bit SIGMA7 storage, the option not set, and a
// grid the face plane-marching kernel takes, or a level of more than 4096 cells the
// register-queue kernels take (the levels between the plane-marching ones and the fused
// coarse cycle, which forms its own faces in shared memory).
static bool face_level(const hfm_mg_config &c, Grid3 g) {
  if (c.op_kind != HFM_OP_SIGMA7 || (c.storage != HFM_BF16 && c.storage != HFM_F16) ||
      (c.options & HFM_OPT_NO_FACES))
    return false;
  return tma_eligible(HFM_OP_FACE7, g, FAST_SMOOTH, nullptr, 0, 2) ||
         (fast_eligible(HFM_OP_FACE7, g, false) && g.n() > 4096);
}

class EngineBase {
 public:
  virtual ~EngineBase() {}
  virtual int emit_cycles(int cycles, cudaStream_t s) = 0;
  virtual int load(int slot, const float *rhs, const float *phi0, cudaStream_t s) = 0;
  virtual int fetch(int slot, float *out, cudaStream_t s) = 0;
  virtual int load_all(const float *rhs, cudaStream_t s) = 0;
  virtual int load64(int slot, const double *rhs, const double *phi0, cudaStream_t s) = 0;
  virtual int fetch64(int slot, double *out, cudaStream_t s) = 0;
  virtual int fetch_all(float *out, cudaStream_t s) = 0;
  virtual int set_operator(int slot, const hfm_operator &op, cudaStream_t s) = 0;
  virtual int read_level(int slot, int level, int which, float *out, cudaStream_t s) = 0;
  virtual bool cycle_flips_parity() const = 0;
};

}  // namespace hfm

struct hfm_mg {
  hfm_mg_config cfg;
  int Z, Y, X, slots, L;
  std::vector<hfm::Level> lv;
  float *cg[4] = {nullptr, nullptr, nullptr, nullptr};  // x, r, p, q (CG) / w, r (sawtooth)
  void *fine_b = nullptr;   // b for CG (rhs[0] holds r in storage type)
  void *saw[2] = {nullptr, nullptr};  // sawtooth: r, w in storage type
  int *active = nullptr;
  int *outer = nullptr;     // refinement: slots whose float64 outer step is due
  double *x64 = nullptr;    // refinement: float64 solution and right-hand side
  double *b64 = nullptr;
  hfm::SlotState *state = nullptr;
  hfm_slot_stats *stats_dev = nullptr;  // packed per-slot statistics for asynchronous queries
  double *partials = nullptr;
  double *partials2 = nullptr;  // CG: the p . q partials (read while `partials` is rewritten)
  int *small_ctr = nullptr;     // persistent small-end kernel: work ticket, per-slot counts
  int64_t partials_per_slot = 0;
  double *scal = nullptr;  // per-slot scratch scalars (rz_new), and ||b||^2 at load
  double *gscale = nullptr;  // fp16 storage: geometric mean of each slot's conductivities
  const int *wait_fail = nullptr;  // the device's TMA wait-failure counters (read by checks)
  hfm_operator fine_desc;
  cudaStream_t cap = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  std::map<int, int64_t> graph_kernels;
  std::vector<void *> allocs;
  std::unique_ptr<hfm::EngineBase> eng;
};

namespace hfm {

template <class T>
class Engine : public EngineBase {
 public:
  explicit Engine(hfm_mg *m) : m_(m) {}

  bool cycle_flips_parity() const override {
    const hfm_mg_config &c = m_->cfg;
    if (c.accel != HFM_ACCEL_NONE) return false;
    if (c.cycle == HFM_CYCLE_SAWTOOTH) return true;
    int post = std::max(c.nu_post, 1);
    return ((c.nu_pre + post) & 1) != 0;
  }

  // ----------------------------------------------------------------- helpers
  T *buf(int l, int which) { return (T *)(which ? m_->lv[l].tmp : m_->lv[l].phi); }
  T *rhs(int l) { return (T *)m_->lv[l].rhs; }
  Grid3 g(int l) { return Grid3{m_->lv[l].Z, m_->lv[l].Y, m_->lv[l].X}; }
  int64_t n(int l) { return m_->lv[l].n; }
  int kind() { return m_->cfg.op_kind; }
  // the operator level l runs: FACE7 where the level holds face arrays
  int lk(int l) { return m_->lv[l].face[0] ? HFM_OP_FACE7 : kind(); }
  const DevOp &lo(int l) { return m_->lv[l].face[0] ? m_->lv[l].fop : m_->lv[l].op; }
  // bf16 refinement: the storage-type copy of the CG residual is written by the kernels that
  // produce r (outer residual, k_cg_xr) instead of a separate conversion pass
  bool fused_rhs() const {
    return std::is_same<T, __nv_bfloat16>::value && m_->cfg.accel == HFM_ACCEL_IR;
  }

  PhiSrc<T> src(const T *base, int64_t stride) {
    PhiSrc<T> p;
    memset(&p, 0, sizeof(p));
    p.base = base;
    p.base_stride = stride;
    return p;
  }
  PhiSrc<T> with_coarse(PhiSrc<T> p, int lc, const T *corr, float sign) {
    p.corr = corr;
    p.corr_stride = n(lc);
    p.corr_coarse = 1;
    p.corr_sign = sign;
    p.Yc = m_->lv[lc].Y;
    p.Xc = m_->lv[lc].X;
    return p;
  }

  int smooth(int l, const PhiSrc<T> &p, const T *f, T *out, float omega, unsigned flags,
             cudaStream_t s, double *partials = nullptr, int *nblk = nullptr) {
    return launch_smooth<T>(lk(l), lo(l), p, f, n(l), out, n(l), m_->slots, g(l),
                            omega, flags, m_->active, s, partials, nblk);
  }

  int check(int nblk, int which, cudaStream_t s, const double *rz_new = nullptr) {
    k_check<<<m_->slots, 256, 0, s>>>(m_->partials, nblk, m_->state, m_->active, m_->cfg.tol,
                                      m_->cfg.max_cycles, which, m_->wait_fail, rz_new);
    HFM_CHECK_LAUNCH("k_check");
    return HFM_OK;
  }

  // ----------------------------------------------------------------- V / F cycles
  int coarse_solve(int l, cudaStream_t s) {
    cur_[l] = 0;
    if (n(l) <= coarse_smem_limit())
      return launch_coarse_jacobi<T>(kind(), m_->lv[l].op, rhs(l), n(l), nullptr, buf(l, 0),
                                     n(l), m_->slots, g(l), m_->cfg.coarse_omega,
                                     m_->cfg.coarse_sweeps, m_->active, s);
    // large coarsest level: global-memory sweeps
    for (int k = 0; k < m_->cfg.coarse_sweeps; ++k) {
      PhiSrc<T> p = src(k == 0 ? nullptr : buf(l, cur_[l]), n(l));
      int st = smooth(l, p, rhs(l), buf(l, cur_[l] ^ 1), m_->cfg.coarse_omega, 0u, s);
      if (st) return st;
      cur_[l] ^= 1;
    }
    return HFM_OK;
  }

  // Approximately solve A_l phi = rhs(l); `zero` says the current iterate is zero.
  // The fused first two sweeps run on the TMA path: SIGMA7 levels the TMA kernels take.
  // Two sweeps per pass (tma_face2.cuh) on FACE7 levels, 16-bit storage.
  bool face2_ok(int l, int pair, bool corr) {
    if (sizeof(T) != 2 || lk(l) != HFM_OP_FACE7 || !(m_->cfg.options & HFM_OPT_TEMPORAL))
      return false;
    if (m_->cfg.flags & (HFM_FLAG_ZERO_XEND | HFM_FLAG_TOP_COPY)) return false;
    if (!face2_eligible(pair, corr, g(l))) return false;
    auto a16 = [](const void *q) { return ((uintptr_t)q & 15) == 0; };
    return a16(buf(l, 0)) && a16(buf(l, 1)) && a16(rhs(l)) && (n(l) % 8) == 0;
  }

  bool pre2_ok(int l) {
    if (kind() != HFM_OP_SIGMA7 || !m_->lv[l].invd || (m_->cfg.options & HFM_OPT_NO_FUSED_PRE))
      return false;
    if (!tma_eligible(lk(l), g(l), FAST_SMOOTH, nullptr, 0, (int)sizeof(T))) return false;
    PhiSrc<T> p = src(rhs(l), n(l));
    return vec_aligned<T>(lk(l), lo(l), p, m_->lv[l].invd, buf(l, 0), nullptr, n(l), 16) &&
           vec_aligned<T>(lk(l), lo(l), p, m_->lv[l].invd, buf(l, 1), nullptr, n(l), 16);
  }

  // First level of the fused coarse V-cycle (subcycle.cu), or -1: the deepest levels of at
  // most 4096 cells of a SIGMA7, CONST7 or K27 hierarchy, at least two of them, below the fine
  // level.
  int fused_first_level() {
    const hfm_mg_config &c = m_->cfg;
    const int k = kind();
    if ((k != HFM_OP_SIGMA7 && k != HFM_OP_CONST7 && k != HFM_OP_K27) ||
        (c.options & HFM_OPT_NO_FUSED_COARSE))
      return -1;
    // one block per instance: with few instances the separate kernels, which spread a level
    // over many SMs, are as fast (measured: a single 64 x 128 x 128 pressure solve)
    if (m_->slots < 8) return -1;
    if (n(m_->L - 1) > coarse_smem_limit()) return -1;
    int l0 = m_->L - 1;
    while (l0 - 1 >= 1 && n(l0 - 1) <= 4096 && m_->L - (l0 - 1) <= kMaxSubLevels) --l0;
    if (l0 >= m_->L - 1) return -1;
    Grid3 gs[kMaxSubLevels];
    for (int l = l0; l < m_->L; ++l) gs[l - l0] = g(l);
    if (subcycle_smem_bytes(gs, m_->L - l0, k == HFM_OP_SIGMA7) > kSubcycleMaxSmem) return -1;
    return l0;
  }

  int fused_vcycle(int l0, cudaStream_t s) {
    SubArgs<T> a = make_sub(l0);
    cur_[l0] = 0;
    return launch_subcycle<T>(kind(), a, m_->slots, s);
  }

  // Arguments of the fused coarse cycle from level l0 down (right-hand side rhs(l0), result
  // in buf(l0, 0)).
  SubArgs<T> make_sub(int l0) {
    const hfm_mg_config &c = m_->cfg;
    SubArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.nlev = m_->L - l0;
    for (int l = l0; l < m_->L; ++l) {
      SubLevel<T> &q = a.lv[l - l0];
      const DevOp &op = m_->lv[l].op;
      q.Z = m_->lv[l].Z;
      q.Y = m_->lv[l].Y;
      q.X = m_->lv[l].X;
      q.n = (int)n(l);
      q.cz = op.c[0] * op.scale;
      q.cy = op.c[1] * op.scale;
      q.cx = op.c[2] * op.scale;
      q.sx = (const T *)op.coef[0];
      q.sy = (const T *)op.coef[1];
      q.sz = (const T *)op.coef[2];
      for (int j = 0; j < 27; ++j) q.k[j] = op.k[j];  // CONST7 / K27 weights, scale applied
    }
    a.rhs = rhs(l0);
    a.out = buf(l0, 0);
    a.active = m_->active;
    a.omega = c.omega;
    a.coarse_omega = c.coarse_omega;
    a.nu_pre = c.nu_pre;
    a.nu_post = c.nu_post;
    a.coarse_sweeps = c.coarse_sweeps;
    return a;
  }

  // The small end as one persistent kernel: level l (which the TMA kernels do not take) and
  // the fused coarse cycle directly below it.
  bool small_ok(int l) {
    const hfm_mg_config &c = m_->cfg;
    if (!(c.options & HFM_OPT_PERSISTENT) || fused_l0_ < 0 || l + 1 != fused_l0_) return false;
    if (lk(l) == HFM_OP_FACE7) return false;
    if (tma_eligible(lk(l), g(l), FAST_SMOOTH, nullptr, 0, (int)sizeof(T))) return false;
    if ((g(l).Z | g(l).Y | g(l).X) & 1) return false;
    if (l == 0 && (c.flags & HFM_FLAG_ZERO_XEND)) return false;
    if (c.nu_pre + std::max(c.nu_post, 1) + 2 > kSmallMaxSteps) return false;
    return true;
  }

  int small_vcycle(int l, cudaStream_t s) {
    const hfm_mg_config &c = m_->cfg;
    const int B = m_->slots;
    SmallArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.sub = make_sub(l + 1);
    a.op = lo(l);
    a.Z = g(l).Z;
    a.Y = g(l).Y;
    a.X = g(l).X;
    a.n = n(l);
    a.f = rhs(l);
    a.invd = (const T *)m_->lv[l].invd;
    a.buf[0] = buf(l, 0);
    a.buf[1] = buf(l, 1);
    a.active = m_->active;
    // z tiles: about two items per SM and step over the instances, an even number of planes
    const int want = std::max(1, (2 * sm_count() + B - 1) / B);
    int zc = (a.Z + want - 1) / want;
    zc += zc & 1;
    zc = std::max(2, std::min(zc, a.Z));
    a.zc = zc;
    a.tiles = (a.Z + zc - 1) / zc;
    const bool dot = want_rz_ && l == 0;
    int ns = 0, cur = 0;
    bool zero = true;
    auto add = [&](int kind, int corr, int dotk, float om) {
      a.kind[ns] = kind;
      a.src[ns] = zero ? -1 : cur;
      a.dst[ns] = cur ^ 1;
      a.corr[ns] = corr;
      a.dot[ns] = dotk;
      a.om[ns] = om;
      ++ns;
    };
    int k0 = 0;
    if (c.nu_pre >= 2 && kind() == HFM_OP_SIGMA7 && a.invd && !(c.options & HFM_OPT_NO_FUSED_PRE)) {
      add(SK_PRE2, 0, 0, c.omega);  // phi1 = omega f / diag formed inside the second sweep
      cur ^= 1;
      zero = false;
      k0 = 2;
    }
    for (int k = k0; k < c.nu_pre; ++k) {
      add(SK_SMOOTH, 0, 0, c.omega);
      cur ^= 1;
      zero = false;
    }
    a.kind[ns] = SK_RESTRICT;
    a.src[ns] = zero ? -1 : cur;
    ++ns;
    a.kind[ns] = SK_SUB;
    ++ns;
    const int post = std::max(c.nu_post, 1);
    for (int k = 0; k < post; ++k) {
      add(SK_SMOOTH, k == 0, dot && k == post - 1, c.nu_post == 0 ? 0.f : c.omega);
      cur ^= 1;
      zero = false;
    }
    a.nsteps = ns;
    int per_inst = 0;
    for (int i = 0; i < ns; ++i) {
      const int cnt = a.kind[i] == SK_SUB ? 1 : a.tiles;
      a.base[i] = B * per_inst;
      a.need[i] = per_inst;
      per_inst += cnt;
    }
    a.base[ns] = B * per_inst;
    a.partials = dot ? m_->partials : nullptr;
    a.ticket = m_->small_ctr;
    a.done = m_->small_ctr + 1;
    a.wait_budget = current_wait_budget();
    a.wait_fail = const_cast<int *>(m_->wait_fail);
    HFM_CUDA(cudaMemsetAsync(m_->small_ctr, 0, (size_t)(B + 1) * sizeof(int), s));
    int st = launch_small<T>(kind(), a, B, s);
    if (st) return st;
    if (dot) nblk_rz_ = a.tiles;
    cur_[l] = cur;
    cur_[l + 1] = 0;
    return HFM_OK;
  }

  int vcycle(int l, bool zero, bool fcycle, int check_level0, cudaStream_t s) {
    const hfm_mg_config &c = m_->cfg;
    int st;
    if (l == m_->L - 1) return coarse_solve(l, s);
    if (zero && !fcycle && !(l == 0 && check_level0) && small_ok(l)) return small_vcycle(l, s);
    if (zero && !fcycle && l > 0 && l == fused_l0_) return fused_vcycle(l, s);
    if (zero) cur_[l] = 0;
    // NS outflow rule on the fine level (as the reference cycle applies it): the iterate is
    // read as zero on x = X-1 and the residual is zero there
    const int xend = (l == 0 && (c.flags & HFM_FLAG_ZERO_XEND)) ? 1 : 0;
    int k0 = 0;
    const bool chk = (l == 0 && check_level0);
    int nblk = 0;
    bool restricted = false;
    if (zero && c.nu_pre >= 2 && !xend && pre2_ok(l)) {
      // the first two sweeps from zero in one pass (phi1 = omega f / diag is pointwise); with
      // nu_pre = 2 on a FACE7 level also the residual and its restriction
      if (c.nu_pre == 2 && face2_ok(l, PAIR_PR, false)) {
        PhiSrc<T> none = src(nullptr, n(l));
        if ((st = tma_launch_face2<T>(PAIR_PR, lo(l), none, rhs(l), (const T *)m_->lv[l].invd,
                                      buf(l, cur_[l] ^ 1), rhs(l + 1), n(l), n(l + 1), m_->slots,
                                      g(l), c.omega, 0u, m_->active,
                                      chk ? m_->partials : nullptr, &nblk, s)))
          return st;
        restricted = true;
      } else if ((st = tma_launch_pre2<T>(lk(l), lo(l), rhs(l), (const T *)m_->lv[l].invd,
                                          buf(l, cur_[l] ^ 1), n(l), m_->slots, g(l), c.omega,
                                          m_->active, s))) {
        return st;
      }
      cur_[l] ^= 1;
      k0 = 2;
    }
    for (int k = k0; k < c.nu_pre; ++k) {
      PhiSrc<T> p = src((zero && k == 0) ? nullptr : buf(l, cur_[l]), n(l));
      p.zero_xend = xend;
      if ((st = smooth(l, p, rhs(l), buf(l, cur_[l] ^ 1), c.omega, 0u, s))) return st;
      cur_[l] ^= 1;
    }
    const bool still_zero = zero && c.nu_pre == 0;
    PhiSrc<T> p = src(still_zero ? nullptr : buf(l, cur_[l]), n(l));
    if (restricted) {
      // done by the two-sweep pass
    } else if (xend) {
      // residual of the iterate with its x = X-1 plane read as zero, zero there, restricted
      T *rf = (T *)m_->saw[0];
      p.zero_xend = 1;
      if ((st = launch_residual<T>(lk(l), lo(l), p, rhs(l), n(l), rf, n(l), m_->slots,
                                   g(l), HFM_FLAG_ZERO_XEND, m_->active,
                                   chk ? m_->partials : nullptr, &nblk, s)))
        return st;
      if ((st = launch_restrict<T>(rf, n(l), rhs(l + 1), n(l + 1), m_->slots, g(l), m_->active, s)))
        return st;
    } else if ((st = launch_residual_restrict<T>(lk(l), lo(l), p, rhs(l), n(l), nullptr, 0,
                                                 rhs(l + 1), n(l + 1), m_->slots, g(l), 0u,
                                                 m_->active, chk ? m_->partials : nullptr, &nblk, s)))
      return st;
    if (chk && (st = check(nblk, cur_[0], s))) return st;
    if (fcycle) {
      if ((st = vcycle(l + 1, true, true, 0, s))) return st;
      if ((st = vcycle(l + 1, false, false, 0, s))) return st;
    } else {
      if ((st = vcycle(l + 1, true, false, 0, s))) return st;
    }
    // correction fused with the first post-smoothing sweep (omega = 0 when nu_post == 0);
    // with nu_post = 2 on a FACE7 level both post-sweeps in one pass
    if (c.nu_post == 2 && !still_zero && !xend && face2_ok(l, PAIR_SS, true)) {
      PhiSrc<T> q = with_coarse(src(buf(l, cur_[l]), n(l)), l + 1, buf(l + 1, cur_[l + 1]), -1.f);
      const bool dot = want_rz_ && l == 0;
      if ((st = tma_launch_face2<T>(PAIR_SS, lo(l), q, rhs(l), nullptr, buf(l, cur_[l] ^ 1),
                                    nullptr, n(l), 0, m_->slots, g(l), c.omega,
                                    dot ? HFM_INT_DOT_RHS : 0u, m_->active,
                                    dot ? m_->partials : nullptr, dot ? &nblk_rz_ : nullptr, s)))
        return st;
      cur_[l] ^= 1;
      return HFM_OK;
    }
    const int post = std::max(c.nu_post, 1);
    for (int k = 0; k < post; ++k) {
      PhiSrc<T> q = src(still_zero && k == 0 ? nullptr : buf(l, cur_[l]), n(l));
      if (k == 0) q = with_coarse(q, l + 1, buf(l + 1, cur_[l + 1]), -1.f);
      q.zero_xend = xend;
      float om = c.nu_post == 0 ? 0.f : c.omega;
      // a CG preconditioner's last fine-level sweep also sums z . r (r is its right-hand side)
      const bool dot = want_rz_ && l == 0 && k == post - 1;
      if ((st = smooth(l, q, rhs(l), buf(l, cur_[l] ^ 1), om, dot ? HFM_INT_DOT_RHS : 0u, s,
                       dot ? m_->partials : nullptr, dot ? &nblk_rz_ : nullptr)))
        return st;
      cur_[l] ^= 1;
    }
    return HFM_OK;
  }

  // ----------------------------------------------------------------- sawtooth
  int sawtooth(cudaStream_t s) {
    const hfm_mg_config &c = m_->cfg;
    const int L = m_->L;
    T *r0 = (T *)m_->saw[0], *w0 = (T *)m_->saw[1];
    int st, nblk = 0;
    const unsigned xend = c.flags & HFM_FLAG_ZERO_XEND;
    // 1. r = A phi - b (NS: r[..., X-1] = 0), residual norm for the stopping test
    if ((st = launch_residual<T>(lk(0), lo(0), src(buf(0, cur_[0]), n(0)), rhs(0), n(0),
                                 r0, n(0), m_->slots, g(0), xend, m_->active, m_->partials,
                                 &nblk, s)))
      return st;
    if ((st = check(nblk, cur_[0], s))) return st;
    // 2. restriction chain r -> r_1 -> ... -> r_{L-1} (coarse rhs buffers)
    for (int l = 1; l < L; ++l) {
      const T *f = l == 1 ? r0 : rhs(l - 1);
      if ((st = launch_restrict<T>(f, n(l - 1), rhs(l), n(l), m_->slots, g(l - 1), m_->active, s)))
        return st;
    }
    // 3. coarsest: one Jacobi sweep from w = 0 (coarse_sweeps of them with
    //    HFM_OPT_SAWTOOTH_COARSE_SWEEPS), the last one landing in buffer 0
    const int ncs = (c.options & HFM_OPT_SAWTOOTH_COARSE_SWEEPS) ? c.coarse_sweeps : 1;
    for (int k = 0; k < ncs; ++k) {
      const int dst = (ncs - 1 - k) & 1;
      PhiSrc<T> p = src(k == 0 ? nullptr : buf(L - 1, dst ^ 1), n(L - 1));
      if ((st = smooth(L - 1, p, rhs(L - 1), buf(L - 1, dst), c.omega, 0u, s))) return st;
    }
    // 4. coarse levels: w = P w; one Jacobi
    for (int l = L - 2; l >= 1; --l) {
      PhiSrc<T> p = with_coarse(src(nullptr, n(l)), l + 1, buf(l + 1, 0), 1.f);
      if ((st = smooth(l, p, rhs(l), buf(l, 0), c.omega, 0u, s))) return st;
    }
    // 5. fine: w = P w (+ one Jacobi against r in the 7-point form)
    if (c.sawtooth_fine_smooth) {
      PhiSrc<T> p = with_coarse(src(nullptr, n(0)), 1, buf(1, 0), 1.f);
      if ((st = smooth(0, p, r0, w0, c.omega, 0u, s))) return st;
    } else {
      if ((st = launch_prolong<T>(buf(1, 0), n(1), w0, n(0), m_->slots, g(1), m_->active, s)))
        return st;
    }
    // 6. phi = J(phi - w) against b (NS: phi[..., X-1] = 0 before the sweep; _BC: top copy)
    PhiSrc<T> p = src(buf(0, cur_[0]), n(0));
    p.corr = w0;
    p.corr_stride = n(0);
    p.corr_sign = -1.f;
    p.zero_xend = xend ? 1 : 0;
    if ((st = smooth(0, p, rhs(0), buf(0, cur_[0] ^ 1), c.omega, c.flags & HFM_FLAG_TOP_COPY, s)))
      return st;
    cur_[0] ^= 1;
    return HFM_OK;
  }

  // ----------------------------------------------------------------- PCG iteration
  // float64 outer step of the refinement for the slots whose inner solve ended:
  // x64 += x_in; r = b - A x64 (float64); finish or restart the inner solve from r.
  int outer_step(cudaStream_t s) {
    const int B = m_->slots;
    const int64_t nf = n(0);
    const Items it{B, item_chunks(nf), nf};
    const int vb = it.CH, ib = item_blocks(B, it.CH);
    k_ir_update<<<ib, 256, 0, s>>>(m_->x64, m_->cg[0], it, m_->state, m_->outer);
    HFM_CHECK_LAUNCH("k_ir_update");
    DevOp d = fine32_;
    T *rs = fused_rhs() ? rhs(0) : nullptr;
    const bool vec4 = (g(0).X % 4) == 0 && nf < ((int64_t)1 << 31);
    switch (kind()) {
      case HFM_OP_SIGMA7:
        if (vec4) {
          k_residual64_sigma4<T><<<ib, 256, 0, s>>>(d, m_->x64, m_->b64, m_->cg[1], rs, g(0).Z,
                                                    g(0).Y, g(0).X, it, m_->outer, m_->partials);
          break;
        }
        k_residual64<HFM_OP_SIGMA7, T><<<ib, 256, 0, s>>>(d, m_->x64, m_->b64, m_->cg[1], rs, g(0).Z,
                                                           g(0).Y, g(0).X, it, m_->outer, m_->partials);
        break;
      case HFM_OP_CONST7:
        k_residual64<HFM_OP_CONST7, T><<<ib, 256, 0, s>>>(d, m_->x64, m_->b64, m_->cg[1], rs, g(0).Z,
                                                           g(0).Y, g(0).X, it, m_->outer, m_->partials);
        break;
      default:
        k_residual64<HFM_OP_K27, T><<<ib, 256, 0, s>>>(d, m_->x64, m_->b64, m_->cg[1], rs, g(0).Z,
                                                        g(0).Y, g(0).X, it, m_->outer, m_->partials);
    }
    HFM_CHECK_LAUNCH("k_residual64");
    k_check_outer<<<B, 256, 0, s>>>(m_->partials, vb, m_->state, m_->active, m_->outer,
                                    m_->cfg.tol, m_->cfg.max_cycles, m_->wait_fail);
    HFM_CHECK_LAUNCH("k_check_outer");
    return HFM_OK;
  }

  int cg_iteration(cudaStream_t s, bool ir) {
    const int B = m_->slots;
    const int64_t nf = n(0);
    float *x = m_->cg[0], *r = m_->cg[1], *p = m_->cg[2], *q = m_->cg[3];
    const Items it{B, item_chunks(nf), nf};
    const int vb = it.CH, ib = item_blocks(B, it.CH);
    const int scaled = std::is_same<T, __half>::value ? 2 : 0;
    int st;
    // z = M r  (rhs(0) holds r / s in the storage type; float32 storage reads r in place; the
    // bf16 refinement path has it written already by the outer residual or the last k_cg_xr)
    if (!std::is_same<T, float>::value && !fused_rhs()) {
      k_to_storage<T><<<ib, 256, 0, s>>>(r, rhs(0), it, m_->active, m_->state, scaled);
      HFM_CHECK_LAUNCH("k_to_storage");
    }
    // r . z comes from the cycle's last fine-level sweep, whose right-hand side is r itself
    // (float32 storage: rhs(0) is the CG residual) or its bf16 copy (bf16 refinement)
    want_rz_ = fused_rhs() || std::is_same<T, float>::value;
    nblk_rz_ = 0;
    st = vcycle(0, true, m_->cfg.cycle == HFM_CYCLE_F, 0, s);
    want_rz_ = false;
    if (st) return st;
    const T *z = buf(0, cur_[0]);
    // rz_new = r . z (summed inside k_cg_p from the last sweep's partials, or from a separate
    // dot pass); p = z + beta p
    const double *rz_part = m_->partials;
    int nblk_rz = nblk_rz_;
    if (nblk_rz_ <= 0) {
      k_dot_partials<T><<<ib, 256, 0, s>>>(r, z, it, m_->partials, m_->active, m_->state, scaled,
                                           m_->gscale);
      HFM_CHECK_LAUNCH("k_dot_partials");
      nblk_rz = vb;
    }
    // k_cg_p writes no per-chunk partials, so it takes chunks four times longer: every chunk
    // re-sums the slot's r . z partials (three block barriers), which at 4096 elements held
    // it near 0.7 of the copy bandwidth
    const Items itp{B, std::max(1, it.CH / 4), nf};
    k_cg_p<T><<<item_blocks(B, itp.CH), 256, 0, s>>>(z, p, itp, m_->state, rz_part, nblk_rz,
                                                     m_->scal, m_->active, scaled, m_->gscale);
    HFM_CHECK_LAUNCH("k_cg_p");
    // q = A p with the partial sums of p . q in the same pass (float32 operator on the fine
    // level), into a partials buffer of their own
    PhiSrc<float> pp;
    memset(&pp, 0, sizeof(pp));
    pp.base = p;
    pp.base_stride = nf;
    int nblk_pq = 0;
    if ((st = launch_residual<float>(kind(), fine32_, pp, nullptr, 0, q, nf, B, g(0), HFM_INT_DOT_PHI,
                                     m_->active, m_->partials2, &nblk_pq, s)))
      return st;
    // x += alpha p ; r -= alpha q ; ||r||  (alpha from rz_new and the p . q partials)
    k_cg_xr<T><<<ib, 256, 0, s>>>(x, r, p, q, fused_rhs() ? rhs(0) : nullptr, it, m_->partials2,
                                  nblk_pq, m_->scal, m_->partials, m_->active, m_->state,
                                  ir ? 1 : 0);
    HFM_CHECK_LAUNCH("k_cg_xr");
    if (!ir) return check(vb, 0, s, m_->scal);
    k_check_inner<<<B, 256, 0, s>>>(m_->partials, vb, m_->state, m_->active, m_->outer,
                                    m_->cfg.tol, m_->cfg.inner_tol, m_->cfg.inner_max_cycles,
                                    m_->wait_fail, m_->scal);
    HFM_CHECK_LAUNCH("k_check_inner");
    return HFM_OK;
  }

  int emit_cycles(int cycles, cudaStream_t s) override {
    int st;
    for (int k = 0; k < kMaxLevels; ++k) cur_[k] = 0;
    fused_l0_ = fused_first_level();
    for (int i = 0; i < cycles; ++i) {
      const hfm_mg_config &c = m_->cfg;
      if (c.accel == HFM_ACCEL_IR) {
        if ((st = outer_step(s))) return st;
        st = cg_iteration(s, true);
      } else if (c.accel == HFM_ACCEL_CG) st = cg_iteration(s, false);
      else if (c.cycle == HFM_CYCLE_SAWTOOTH) st = sawtooth(s);
      else st = vcycle(0, false, c.cycle == HFM_CYCLE_F, 1, s);
      if (st) return st;
    }
    if (m_->cfg.accel == HFM_ACCEL_NONE && cur_[0] != 0) {
      // an odd number of fine-level sweeps: bring the iterate back to the canonical buffer
      // (slots switched off inside this launch keep their solution where the check saw it)
      k_copy_active<T><<<dim3(vec_blocks(n(0), m_->slots), m_->slots), 256, 0, s>>>(
          buf(0, 1), buf(0, 0), n(0), m_->active);
      HFM_CHECK_LAUNCH("k_copy_active");
      cur_[0] = 0;
    }
    return HFM_OK;
  }

  // ----------------------------------------------------------------- slots
  int set_operator(int slot, const hfm_operator &op, cudaStream_t s) override {
    const int k = m_->cfg.op_kind;
    if (op.kind != k) return fail(HFM_ERR_BAD_ARG, "operator kind differs from the handle's");
    m_->fine_desc = op;
    if (k == HFM_OP_CONST7 || k == HFM_OP_K27) {
      float sc = 1.f;
      for (int l = 0; l < m_->L; ++l) {
        hfm_operator o = op;
        o.scale = (op.scale == 0.f ? 1.f : op.scale) * sc;
        m_->lv[l].op = make_devop(o, 0);
        sc *= m_->cfg.coarse_scale;
      }
      fine32_ = m_->lv[0].op;
      return HFM_OK;
    }
    if (k == HFM_OP_DIR7) return set_directional(slot, op, s);
    if (k != HFM_OP_SIGMA7) return fail(HFM_ERR_UNSUPPORTED, "unknown operator kind");
    if (op.coef_dtype != HFM_F32 && op.coef_dtype != HFM_F64)
      return fail(HFM_ERR_BAD_ARG, "coefficients must be float32 or float64");
    // slot < 0: every slot at once (the arrays hold all slots), one launch per level
    const int lo = slot < 0 ? 0 : slot, cnt = slot < 0 ? m_->slots : 1;
    const hfm_operator fine_src = op;  // the caller's conductivities (fine-level faces)
    // fp16 cycles used as a preconditioner store sigma / g (their output is rescaled by 1/g);
    // stationary fp16 cycles keep sigma itself, their iterate is the solution
    const bool normalize = std::is_same<T, __half>::value && m_->cfg.accel != HFM_ACCEL_NONE;
    for (int a = 0; a < 3; ++a)
      if (!op.coef[a]) return fail(HFM_ERR_BAD_ARG, "SIGMA7 needs sx, sy, sz");
    if (normalize) {
      k_log_mean<<<cnt, 256, 0, s>>>(op.coef[0], op.coef[1], op.coef[2], op.coef_dtype, n(0), lo,
                                     m_->gscale);
      HFM_CHECK_LAUNCH("k_log_mean");
    }
    {
      Admit3<T> ad;
      for (int a = 0; a < 3; ++a) {
        ad.src[a] = op.coef[a];
        ad.dst[a] = (T *)m_->lv[0].coef[a] + lo * n(0);
        ad.dst32[a] = fine32_coef_[a] ? fine32_coef_[a] + lo * n(0) : nullptr;
      }
      k_admit_convert<T><<<dim3(vec_blocks(n(0) * cnt, 3), 3), 256, 0, s>>>(
          ad, op.coef_dtype, n(0), cnt, lo, normalize ? m_->gscale : nullptr);
      HFM_CHECK_LAUNCH("k_admit_convert");
    }
    for (int l = 1; l < m_->L; ++l) {
      const T *f3[3];
      T *c3[3];
      for (int a = 0; a < 3; ++a) {
        f3[a] = (const T *)m_->lv[l - 1].coef[a] + lo * n(l - 1);
        c3[a] = (T *)m_->lv[l].coef[a] + lo * n(l);
      }
      if (int st = launch_restrict3<T>(f3, n(l - 1), c3, n(l), cnt, g(l - 1), s)) return st;
    }
    float sc = 1.f;
    for (int l = 0; l < m_->L; ++l) {
      hfm_operator o = op;
      o.scale = (op.scale == 0.f ? 1.f : op.scale) * sc;
      for (int a = 0; a < 3; ++a) o.coef[a] = m_->lv[l].coef[a];
      m_->lv[l].op = make_devop(o, n(l));
      sc *= m_->cfg.coarse_scale;
    }
    fine32_ = m_->lv[0].op;
    if (fine32_coef_[0])
      for (int a = 0; a < 3; ++a) fine32_.coef[a] = fine32_coef_[a];
    // 1 / diagonal of every level, for the fused first two sweeps of a cycle
    {
      InvdLevels d;
      d.L = m_->L;
      d.first[0] = 0;
      for (int l = 0; l < m_->L; ++l) {
        const DevOp &o = m_->lv[l].op;
        d.sx[l] = o.coef[0];
        d.sy[l] = o.coef[1];
        d.sz[l] = o.coef[2];
        d.out[l] = m_->lv[l].invd;
        d.cz[l] = o.c[0] * o.scale;
        d.cy[l] = o.c[1] * o.scale;
        d.cx[l] = o.c[2] * o.scale;
        d.Z[l] = g(l).Z;
        d.Y[l] = g(l).Y;
        d.X[l] = g(l).X;
        d.first[l + 1] = d.first[l] + (int)std::min<int64_t>((n(l) + 1023) / 1024, 1024);
      }
      k_invdiag_levels<T><<<dim3(d.first[m_->L], cnt), 256, 0, s>>>(d, lo);
      HFM_CHECK_LAUNCH("k_invdiag_levels");
    }
    // FACE7 arrays of the levels that hold them: the fine level's faces from the caller's
    // float32 / float64 conductivities (divided by the slot's geometric mean for normalised
    // fp16 cycles), coarse levels' from their restricted conductivities.  bf16 (float32's
    // exponent range) folds the level's scale and c into the faces; fp16 divides them by
    // kappa = scale * max(c) and keeps kappa as the operator's scale, so the stored faces stay
    // in the range of the conductivities (c = 1/h^2 folded in would overflow fp16, and a
    // coarse scale of 2^-l pushed small faces into its subnormals)
    for (int l = 0; l < m_->L; ++l) {
      Level &L_ = m_->lv[l];
      if (!L_.face[0]) continue;
      const DevOp &op = L_.op;
      float s_ = op.scale, kappa = 1.f;
      if (std::is_same<T, __half>::value) {
        kappa = op.scale * std::max(std::fabs(op.c[0]), std::max(std::fabs(op.c[1]), std::fabs(op.c[2])));
        if (!(kappa > 0.f) || !std::isfinite(kappa)) kappa = 1.f;
        s_ = op.scale / kappa;
      }
      const float cz = op.c[0] * s_, cy = op.c[1] * s_, cx = op.c[2] * s_;
      const int64_t nx = face7_nx(g(l).Z, g(l).Y, g(l).X), ny = face7_ny(g(l).Z, g(l).Y, g(l).X),
                    nz = face7_nz(g(l).Z, g(l).Y, g(l).X);
      T *fx = (T *)L_.face[0] + lo * nx, *fy = (T *)L_.face[1] + lo * ny, *fz = (T *)L_.face[2] + lo * nz;
      const double *div = normalize ? m_->gscale : nullptr;
      int st;
      if (l == 0 && fine_src.coef_dtype == HFM_F64)
        st = launch_sigma_faces<double, T>((const double *)fine_src.coef[0], (const double *)fine_src.coef[1],
                                           (const double *)fine_src.coef[2], n(0), cz, cy, cx, div, lo,
                                           fx, fy, fz, cnt, g(0), s);
      else if (l == 0)
        st = launch_sigma_faces<float, T>((const float *)fine_src.coef[0], (const float *)fine_src.coef[1],
                                          (const float *)fine_src.coef[2], n(0), cz, cy, cx, div, lo,
                                          fx, fy, fz, cnt, g(0), s);
      else
        st = launch_sigma_faces<T, T>((const T *)op.coef[0] + lo * n(l), (const T *)op.coef[1] + lo * n(l),
                                      (const T *)op.coef[2] + lo * n(l), n(l), cz, cy, cx, nullptr, 0,
                                      fx, fy, fz, cnt, g(l), s);
      if (st) return st;
      hfm_operator fo;
      memset(&fo, 0, sizeof(fo));
      fo.kind = HFM_OP_FACE7;
      fo.scale = kappa;
      for (int a = 0; a < 3; ++a) fo.coef[a] = L_.face[a];
      L_.fop = make_devop(fo, 0);
      // the fused first two sweeps divide by the diagonal of the stored faces
      if constexpr (sizeof(T) == 2) {
        if (L_.invd && (st = launch_invdiag_faces<T>(fx, fy, fz, kappa, (T *)L_.invd + lo * n(l), n(l),
                                                     cnt, g(l), s)))
          return st;
      }
    }
    return HFM_OK;
  }

  // The directional form of BGS_multigrid_v1.ipynb cells 38-40: six per-cell face
  // coefficient arrays (x-, x+, y-, y+, z-, z+) and their sum (the diagonal A_MAT_TOT); coarse
  // levels restrict all seven with the averaging restriction, without rescaling (cell 38,
  // lines 16-33); coarse_scale^l multiplies level l as for the other forms.
  int set_directional(int slot, const hfm_operator &op, cudaStream_t s) {
    if (op.coef_dtype != HFM_F32 && op.coef_dtype != HFM_F64)
      return fail(HFM_ERR_BAD_ARG, "coefficients must be float32 or float64");
    for (int a = 0; a < 7; ++a)
      if (!op.coef[a]) return fail(HFM_ERR_BAD_ARG, "DIR7 needs seven coefficient arrays");
    const int lo = slot < 0 ? 0 : slot, cnt = slot < 0 ? m_->slots : 1;
    for (int a = 0; a < 7; ++a) {
      int st = launch_convert<T>(op.coef[a], op.coef_dtype, (T *)m_->lv[0].coef[a] + lo * n(0),
                                 n(0) * cnt, s);
      if (st) return st;
      for (int l = 1; l < m_->L; ++l)
        if ((st = launch_restrict<T>((T *)m_->lv[l - 1].coef[a] + lo * n(l - 1), n(l - 1),
                                     (T *)m_->lv[l].coef[a] + lo * n(l), n(l), cnt, g(l - 1),
                                     nullptr, s)))
          return st;
    }
    float sc = 1.f;
    for (int l = 0; l < m_->L; ++l) {
      hfm_operator o = op;
      o.scale = (op.scale == 0.f ? 1.f : op.scale) * sc;
      o.coef_dtype = HFM_F32;
      for (int a = 0; a < 7; ++a) o.coef[a] = m_->lv[l].coef[a];
      m_->lv[l].op = make_devop(o, n(l));
      sc *= m_->cfg.coarse_scale;
    }
    fine32_ = m_->lv[0].op;
    return HFM_OK;
  }

  // Refinement: float64 right-hand side / initial guess (from float32 or float64 input).
  int load_ir(int slot, int count, const void *b, const void *phi0, int dt, cudaStream_t s) {
    const int64_t nf = n(0) * count;
    double *bb = m_->b64 + (int64_t)slot * n(0), *xx = m_->x64 + (int64_t)slot * n(0);
    const int vb = vec_blocks(nf, 1);
    k_to_f64<<<vb, 256, 0, s>>>(b, dt, bb, nf);
    if (phi0) k_to_f64<<<vb, 256, 0, s>>>(phi0, dt, xx, nf);
    else HFM_CUDA(cudaMemsetAsync(xx, 0, nf * 8, s));
    HFM_CHECK_LAUNCH("k_to_f64");
    HFM_CUDA(cudaMemsetAsync(m_->cg[0] + (int64_t)slot * n(0), 0, nf * 4, s));
    const int nb = vec_blocks(n(0), count);
    k_sumsq64<<<dim3(nb, count), 256, 0, s>>>(bb, n(0), m_->partials);
    HFM_CHECK_LAUNCH("k_sumsq64");
    int st;
    if ((st = launch_finalize_sum(m_->partials, nb, count, m_->scal + (count == 1 ? m_->slots : 0), s)))
      return st;
    if (count == 1)
      k_init_state<<<1, 1, 0, s>>>(m_->state, m_->active, slot, m_->scal + m_->slots, HFM_OK, m_->outer);
    else
      k_init_states<<<(count + 127) / 128, 128, 0, s>>>(m_->state, m_->active, count, m_->scal, m_->outer);
    HFM_CHECK_LAUNCH("k_init_state");
    return HFM_OK;
  }

  int load64(int slot, const double *b, const double *phi0, cudaStream_t s) override {
    if (m_->cfg.accel != HFM_ACCEL_IR) return fail(HFM_ERR_UNSUPPORTED, "float64 load needs accel = IR");
    return load_ir(slot, 1, b, phi0, HFM_F64, s);
  }

  int fetch64(int slot, double *out, cudaStream_t s) override {
    if (m_->cfg.accel != HFM_ACCEL_IR) return fail(HFM_ERR_UNSUPPORTED, "float64 fetch needs accel = IR");
    HFM_CUDA(cudaMemcpyAsync(out, m_->x64 + (int64_t)slot * n(0), n(0) * 8, cudaMemcpyDeviceToDevice, s));
    return HFM_OK;
  }

  int load(int slot, const float *b, const float *phi0, cudaStream_t s) override {
    const int64_t nf = n(0);
    int st;
    if (m_->cfg.accel == HFM_ACCEL_IR) return load_ir(slot, 1, b, phi0, HFM_F32, s);
    const bool cg = m_->cfg.accel == HFM_ACCEL_CG;
    if (cg) {
      float *x = m_->cg[0] + slot * nf, *r = m_->cg[1] + slot * nf, *bb = (float *)m_->fine_b + slot * nf;
      HFM_CUDA(cudaMemcpyAsync(bb, b, nf * 4, cudaMemcpyDeviceToDevice, s));
      if (phi0) {
        HFM_CUDA(cudaMemcpyAsync(x, phi0, nf * 4, cudaMemcpyDeviceToDevice, s));
        DevOp d = fine32_;
        for (int a = 0; a < 7; ++a)
          if (d.coef[a]) d.coef[a] = (const char *)d.coef[a] + (size_t)slot * nf * 4;
        PhiSrc<float> p;
        memset(&p, 0, sizeof(p));
        p.base = x;
        p.base_stride = nf;
        if (!std::is_same<T, float>::value && m_->cfg.op_kind == HFM_OP_SIGMA7 && !fine32_coef_[0])
          return fail(HFM_ERR_UNSUPPORTED, "initial guess with reduced-precision CG");
        if ((st = launch_residual<float>(kind(), d, p, bb, nf, r, nf, 1, g(0), 0u, nullptr,
                                         nullptr, nullptr, s)))
          return st;
        k_negate<<<vec_blocks(nf, 1), 256, 0, s>>>(r, nf);
      } else {
        HFM_CUDA(cudaMemsetAsync(x, 0, nf * 4, s));
        HFM_CUDA(cudaMemcpyAsync(r, b, nf * 4, cudaMemcpyDeviceToDevice, s));
      }
      HFM_CUDA(cudaMemsetAsync(m_->cg[2] + slot * nf, 0, nf * 4, s));
    } else {
      if ((st = launch_convert<T>(b, HFM_F32, rhs(0) + slot * nf, nf, s))) return st;
      if (phi0) {
        if ((st = launch_convert<T>(phi0, HFM_F32, buf(0, 0) + slot * nf, nf, s))) return st;
      } else {
        HFM_CUDA(cudaMemsetAsync(buf(0, 0) + slot * nf, 0, nf * sizeof(T), s));
      }
    }
    int nb = 0;
    if ((st = launch_sumsq_partials<float>(b, nf, nf, 1, m_->partials, &nb, nullptr, s))) return st;
    if ((st = launch_finalize_sum(m_->partials, nb, 1, m_->scal + m_->slots, s))) return st;
    k_init_state<<<1, 1, 0, s>>>(m_->state, m_->active, slot, m_->scal + m_->slots, HFM_OK, nullptr);
    HFM_CHECK_LAUNCH("k_init_state");
    return HFM_OK;
  }

  // All slots at once from rhs [slots][n] (zero initial guess): the batched form of load().
  int load_all(const float *b, cudaStream_t s) override {
    const int64_t nf = n(0);
    const int B = m_->slots;
    int st;
    if (m_->cfg.accel == HFM_ACCEL_IR) return load_ir(0, B, b, nullptr, HFM_F32, s);
    if (m_->cfg.accel == HFM_ACCEL_CG) {
      HFM_CUDA(cudaMemcpyAsync(m_->fine_b, b, nf * B * 4, cudaMemcpyDeviceToDevice, s));
      HFM_CUDA(cudaMemsetAsync(m_->cg[0], 0, nf * B * 4, s));
      HFM_CUDA(cudaMemcpyAsync(m_->cg[1], b, nf * B * 4, cudaMemcpyDeviceToDevice, s));
      HFM_CUDA(cudaMemsetAsync(m_->cg[2], 0, nf * B * 4, s));
    } else {
      if ((st = launch_convert<T>(b, HFM_F32, rhs(0), nf * B, s))) return st;
      HFM_CUDA(cudaMemsetAsync(buf(0, 0), 0, nf * B * sizeof(T), s));
    }
    int nb = 0;
    if ((st = launch_sumsq_partials<float>(b, nf, nf, B, m_->partials, &nb, nullptr, s))) return st;
    if ((st = launch_finalize_sum(m_->partials, nb, B, m_->scal, s))) return st;
    k_init_states<<<(B + 127) / 128, 128, 0, s>>>(m_->state, m_->active, B, m_->scal, nullptr);
    HFM_CHECK_LAUNCH("k_init_states");
    return HFM_OK;
  }

  int fetch_all(float *out, cudaStream_t s) override {
    const int64_t nf = n(0);
    if (m_->cfg.accel == HFM_ACCEL_IR) {
      k_f64_to_f32<<<vec_blocks(nf * m_->slots, 1), 256, 0, s>>>(m_->x64, out, nf * m_->slots);
      HFM_CHECK_LAUNCH("k_f64_to_f32");
      return HFM_OK;
    }
    const float *bx = m_->cfg.accel == HFM_ACCEL_CG ? m_->cg[0] : nullptr;
    k_fetch_all<T><<<dim3(vec_blocks(nf, m_->slots), m_->slots), 256, 0, s>>>(
        buf(0, 0), buf(0, 1), bx, nf, m_->state, m_->active, out);
    HFM_CHECK_LAUNCH("k_fetch_all");
    return HFM_OK;
  }

  int fetch(int slot, float *out, cudaStream_t s) override {
    const int64_t nf = n(0);
    if (m_->cfg.accel == HFM_ACCEL_IR) {
      k_f64_to_f32<<<vec_blocks(nf, 1), 256, 0, s>>>(m_->x64 + slot * nf, out, nf);
      HFM_CHECK_LAUNCH("k_f64_to_f32");
      return HFM_OK;
    }
    const float *bx = m_->cfg.accel == HFM_ACCEL_CG ? m_->cg[0] + slot * nf : nullptr;
    k_fetch<T><<<vec_blocks(nf, 1), 256, 0, s>>>(buf(0, 0) + slot * nf, buf(0, 1) + slot * nf,
                                                bx, nf, m_->state, m_->active, slot, out);
    HFM_CHECK_LAUNCH("k_fetch");
    return HFM_OK;
  }

  int read_level(int slot, int level, int which, float *out, cudaStream_t s) override {
    if (level < 0 || level >= m_->L) return fail(HFM_ERR_BAD_ARG, "level out of range");
    const T *src_p;
    if (m_->cfg.cycle == HFM_CYCLE_SAWTOOTH && level == 0 && m_->cfg.accel == HFM_ACCEL_NONE)
      src_p = (const T *)(which ? m_->saw[0] : m_->saw[1]);
    else
      src_p = which ? rhs(level) : buf(level, 0);
    return launch_convert_out<T>(src_p + slot * n(level), out, n(level), s);
  }

  DevOp fine32_;
  float *fine32_coef_[3] = {nullptr, nullptr, nullptr};

 private:
  hfm_mg *m_;
  int cur_[kMaxLevels] = {0};
  int fused_l0_ = -1;  // first level of the fused coarse V-cycle, -1: none
  bool want_rz_ = false;  // the next fine-level post-sweep sums z . r into the partials
  int nblk_rz_ = 0;       // partials per slot it wrote (0: none)
};

}  // namespace hfm

using namespace hfm;

namespace {

void *dalloc(hfm_mg *m, size_t bytes, int *st) {
  if (*st) return nullptr;
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *st = fail(HFM_ERR_OOM, "cudaMalloc failed while creating a multigrid handle");
    return nullptr;
  }
  m->allocs.push_back(p);
  return p;
}

std::vector<Grid3> plan_levels(const hfm_mg_config &c, int Z, int Y, int X) {
  std::vector<Grid3> v{Grid3{Z, Y, X}};
  const int want = c.n_levels > 0 ? c.n_levels : kMaxLevels;
  while ((int)v.size() < want) {
    Grid3 t = v.back();
    bool even = !(t.Z & 1) && !(t.Y & 1) && !(t.X & 1);
    if (c.n_levels > 0) {
      // explicit depth: the reference's VALID restriction floors odd extents
      if (t.Z < 2 && t.Y < 2 && t.X < 2) break;
      v.push_back(Grid3{std::max(t.Z / 2, 1), std::max(t.Y / 2, 1), std::max(t.X / 2, 1)});
      continue;
    }
    if (!even || std::min(t.Z, std::min(t.Y, t.X)) <= c.min_coarse_edge) break;
    v.push_back(Grid3{t.Z / 2, t.Y / 2, t.X / 2});
  }
  return v;
}

int validate_cfg(const hfm_mg_config &c, int Z, int Y, int X, int slots) {
  if (Z <= 0 || Y <= 0 || X <= 0 || slots <= 0 || slots > 65535)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: bad extents or slot count");
  if ((int64_t)Z * Y * X >= ((int64_t)1 << 31))
    return fail(HFM_ERR_UNSUPPORTED, "hfm_mg_create: an instance holds at most 2^31 - 1 cells");
  if (c.op_kind != HFM_OP_CONST7 && c.op_kind != HFM_OP_SIGMA7 && c.op_kind != HFM_OP_K27 &&
      c.op_kind != HFM_OP_DIR7)
    return fail(HFM_ERR_UNSUPPORTED, "hfm_mg_create: unknown operator kind");
  if (c.op_kind == HFM_OP_DIR7 && (c.storage != HFM_F32 || c.accel == HFM_ACCEL_IR))
    return fail(HFM_ERR_UNSUPPORTED, "hfm_mg_create: the directional form runs in float32 storage without refinement");
  if (c.storage != HFM_F32 && c.storage != HFM_BF16 && c.storage != HFM_F16)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: storage must be F32, BF16 or F16");
  if (c.cycle < 0 || c.cycle > 2 || c.accel < 0 || c.accel > 2)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: bad cycle / accel");
  if (c.cycle == HFM_CYCLE_SAWTOOTH && c.accel != HFM_ACCEL_NONE)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: the sawtooth cycle is not symmetric; use V or F with CG");
  if (c.accel != HFM_ACCEL_NONE && (c.flags & HFM_FLAG_ZERO_XEND))
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: the x-end rule is for stationary cycles only");
  if (c.accel != HFM_ACCEL_NONE && c.cycle == HFM_CYCLE_F)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: the F-cycle is not symmetric and cannot precondition CG; use V");
  if (c.accel != HFM_ACCEL_NONE && c.nu_pre != c.nu_post)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: CG needs a symmetric cycle (nu_pre == nu_post)");
  if (c.nu_pre < 0 || c.nu_post < 0 || c.coarse_sweeps < 1 || c.max_cycles < 1)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: bad sweep counts");
  if (!(c.omega > 0.f) || !(c.tol > 0.0)) return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: bad omega / tol");
  return HFM_OK;
}

}  // namespace

extern "C" {

void hfm_mg_config_default(hfm_mg_config *c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->op_kind = HFM_OP_SIGMA7;
  c->cycle = HFM_CYCLE_V;
  c->accel = HFM_ACCEL_NONE;
  c->n_levels = 0;
  c->min_coarse_edge = 4;
  c->nu_pre = 2;
  c->nu_post = 2;
  c->coarse_sweeps = 32;
  c->omega = 2.f / 3.f;
  c->coarse_omega = 2.f / 3.f;
  c->coarse_scale = 0.5f;
  c->sawtooth_fine_smooth = 1;
  c->flags = 0;
  c->storage = HFM_F32;
  c->tol = 1e-6;
  c->max_cycles = 500;
  c->cycles_per_launch = 4;
  c->inner_tol = 1e-6;
  c->inner_max_cycles = 200;
}

size_t hfm_mg_footprint_bytes(const hfm_mg_config *c, int Z, int Y, int X, int slots) {
  if (!c) return 0;
  std::vector<Grid3> lv = plan_levels(*c, Z, Y, X);
  const size_t es = dtype_size(c->storage);
  size_t tot = 0;
  for (size_t l = 0; l < lv.size(); ++l) {
    size_t nl = (size_t)lv[l].n();
    size_t fields = 3 + (c->op_kind == HFM_OP_SIGMA7 ? 4 : 0) + (c->op_kind == HFM_OP_DIR7 ? 7 : 0);
    tot += nl * fields * es;
    if (face_level(*c, lv[l]))
      tot += (size_t)(face7_nx(lv[l].Z, lv[l].Y, lv[l].X) + face7_ny(lv[l].Z, lv[l].Y, lv[l].X) +
                      face7_nz(lv[l].Z, lv[l].Y, lv[l].X)) * es;
  }
  const size_t nf = (size_t)Z * Y * X;
  if (c->accel != HFM_ACCEL_NONE) {
    tot += nf * 5 * 4;  // x r p q b
    if (c->accel == HFM_ACCEL_IR) tot += nf * 2 * 8;  // float64 x, b
    if (c->op_kind == HFM_OP_SIGMA7 && c->storage != HFM_F32) tot += nf * 3 * 4;
  } else if (c->cycle == HFM_CYCLE_SAWTOOTH || (c->flags & HFM_FLAG_ZERO_XEND)) {
    tot += nf * 2 * es;
  }
  tot *= (size_t)slots;
  tot += (size_t)slots * (sizeof(SlotState) + 64) +
         (size_t)slots * 4096 * 8 * (c->accel != HFM_ACCEL_NONE ? 2 : 1);
  return tot;
}

int hfm_mg_create(const hfm_mg_config *cfg, int Z, int Y, int X, int slots, hfm_mg **out) {
  if (!cfg || !out) return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: NULL argument");
  *out = nullptr;
  int st = validate_cfg(*cfg, Z, Y, X, slots);
  if (st) return st;
  std::unique_ptr<hfm_mg> m(new hfm_mg());
  m->cfg = *cfg;
  if (m->cfg.cycles_per_launch < 1) m->cfg.cycles_per_launch = 1;
  m->Z = Z;
  m->Y = Y;
  m->X = X;
  m->slots = slots;
  std::vector<Grid3> lv = plan_levels(*cfg, Z, Y, X);
  m->L = (int)lv.size();
  if (m->L < 2 && cfg->cycle == HFM_CYCLE_SAWTOOTH)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: the sawtooth cycle needs at least two levels");
  if (lv.back().n() > coarse_smem_limit() && cfg->cycle != HFM_CYCLE_SAWTOOTH && m->L > 1 &&
      cfg->coarse_sweeps > 64)
    return fail(HFM_ERR_BAD_ARG, "hfm_mg_create: coarsest level too large");
  const size_t es = dtype_size(cfg->storage);
  m->lv.resize(m->L);
  for (int l = 0; l < m->L; ++l) {
    Level &L = m->lv[l];
    L.Z = lv[l].Z;
    L.Y = lv[l].Y;
    L.X = lv[l].X;
    L.n = lv[l].n();
    const size_t b = (size_t)L.n * slots * es;
    L.phi = dalloc(m.get(), b, &st);
    L.tmp = dalloc(m.get(), b, &st);
    // float32 CG: the fine-level cycle reads the CG residual in place (set below)
    if (!(l == 0 && cfg->accel != HFM_ACCEL_NONE && cfg->storage == HFM_F32))
      L.rhs = dalloc(m.get(), b, &st);
    if (cfg->op_kind == HFM_OP_SIGMA7) {
      for (int a = 0; a < 3; ++a) L.coef[a] = dalloc(m.get(), b, &st);
      L.invd = dalloc(m.get(), b, &st);
    }
    if (face_level(*cfg, lv[l])) {
      L.face[0] = dalloc(m.get(), (size_t)face7_nx(L.Z, L.Y, L.X) * slots * es, &st);
      L.face[1] = dalloc(m.get(), (size_t)face7_ny(L.Z, L.Y, L.X) * slots * es, &st);
      L.face[2] = dalloc(m.get(), (size_t)face7_nz(L.Z, L.Y, L.X) * slots * es, &st);
    }
    if (cfg->op_kind == HFM_OP_DIR7)
      for (int a = 0; a < 7; ++a) L.coef[a] = dalloc(m.get(), b, &st);
  }
  const size_t nf = (size_t)Z * Y * X * slots;
  if (cfg->accel == HFM_ACCEL_IR) {
    m->x64 = (double *)dalloc(m.get(), nf * 8, &st);
    m->b64 = (double *)dalloc(m.get(), nf * 8, &st);
  }
  m->outer = (int *)dalloc(m.get(), (size_t)slots * 4, &st);
  if (cfg->accel != HFM_ACCEL_NONE) {
    for (int i = 0; i < 4; ++i) m->cg[i] = (float *)dalloc(m.get(), nf * 4, &st);
    m->fine_b = dalloc(m.get(), nf * 4, &st);
    if (cfg->storage == HFM_F32) m->lv[0].rhs = m->cg[1];
  } else if (cfg->cycle == HFM_CYCLE_SAWTOOTH || (cfg->flags & HFM_FLAG_ZERO_XEND)) {
    m->saw[0] = dalloc(m.get(), nf * es, &st);
    m->saw[1] = dalloc(m.get(), nf * es, &st);
  }
  m->partials_per_slot = std::max<int64_t>(std::max<int64_t>(4096, max_partial_blocks(lv[0], slots)),
                                          item_chunks(lv[0].n()));
  m->partials = (double *)dalloc(m.get(), (size_t)slots * m->partials_per_slot * 8, &st);
  if (cfg->accel != HFM_ACCEL_NONE)
    m->partials2 = (double *)dalloc(m.get(), (size_t)slots * m->partials_per_slot * 8, &st);
  m->active = (int *)dalloc(m.get(), (size_t)slots * 4, &st);
  m->small_ctr = (int *)dalloc(m.get(), (size_t)(slots + 1) * 4, &st);
  m->state = (SlotState *)dalloc(m.get(), (size_t)slots * sizeof(SlotState), &st);
  m->stats_dev = (hfm_slot_stats *)dalloc(m.get(), (size_t)slots * sizeof(hfm_slot_stats), &st);
  m->scal = (double *)dalloc(m.get(), (size_t)(slots + 1) * 8, &st);
  m->gscale = (double *)dalloc(m.get(), (size_t)slots * 8, &st);
  if (!st) {
    if (cudaMemset(m->active, 0, (size_t)slots * 4) != cudaSuccess ||
        cudaMemset(m->outer, 0, (size_t)slots * 4) != cudaSuccess ||
        cudaMemset(m->state, 0, (size_t)slots * sizeof(SlotState)) != cudaSuccess)
      st = fail(HFM_ERR_CUDA, "cudaMemset failed");
  }
  if (!st) st = wait_fail_counters(&m->wait_fail);
  if (!st && cudaStreamCreateWithFlags(&m->cap, cudaStreamNonBlocking) != cudaSuccess)
    st = fail(HFM_ERR_CUDA, "cudaStreamCreate failed");
  if (!st) {
    switch (cfg->storage) {
      case HFM_F32: m->eng.reset(new Engine<float>(m.get())); break;
      case HFM_BF16: m->eng.reset(new Engine<__nv_bfloat16>(m.get())); break;
      default: m->eng.reset(new Engine<__half>(m.get())); break;
    }
    // CG runs its outer vectors and fine operator in float32: keep float32 conductivities.
    if (cfg->accel != HFM_ACCEL_NONE && cfg->op_kind == HFM_OP_SIGMA7 && cfg->storage != HFM_F32) {
      float **fc = nullptr;
      switch (cfg->storage) {
        case HFM_BF16: fc = ((Engine<__nv_bfloat16> *)m->eng.get())->fine32_coef_; break;
        default: fc = ((Engine<__half> *)m->eng.get())->fine32_coef_; break;
      }
      for (int a = 0; a < 3; ++a) fc[a] = (float *)dalloc(m.get(), nf * 4, &st);
    }
  }
  if (st) {
    for (void *p : m->allocs) cudaFree(p);
    if (m->cap) cudaStreamDestroy(m->cap);
    return st;
  }
  // default constant operator so that CONST7 / K27 handles work after set_operator only
  *out = m.release();
  return HFM_OK;
}

int hfm_mg_destroy(hfm_mg *m) {
  if (!m) return HFM_OK;
  for (auto &kv : m->graphs) cudaGraphExecDestroy(kv.second);
  if (m->cap) {
    cudaStreamSynchronize(m->cap);
    cudaStreamDestroy(m->cap);
  }
  cudaDeviceSynchronize();
  for (void *p : m->allocs) cudaFree(p);
  delete m;
  return HFM_OK;
}

int hfm_mg_num_levels(const hfm_mg *m) { return m ? m->L : 0; }

int hfm_mg_level_shape(const hfm_mg *m, int level, int *Z, int *Y, int *X) {
  if (!m || level < 0 || level >= m->L || !Z || !Y || !X) return fail(HFM_ERR_BAD_ARG, "bad level");
  *Z = m->lv[level].Z;
  *Y = m->lv[level].Y;
  *X = m->lv[level].X;
  return HFM_OK;
}

int hfm_mg_set_operator(hfm_mg *m, int slot, const hfm_operator *op, hfm_stream_t stream) {
  if (!m || !op || slot >= m->slots || slot < -1) return fail(HFM_ERR_BAD_ARG, "hfm_mg_set_operator: bad argument");
  return m->eng->set_operator(slot, *op, (cudaStream_t)stream);
}

int hfm_mg_load(hfm_mg *m, int slot, const float *rhs, const float *phi0, hfm_stream_t stream) {
  if (!m || !rhs || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_load: bad argument");
  return m->eng->load(slot, rhs, phi0, (cudaStream_t)stream);
}

int hfm_mg_run(hfm_mg *m, int cycles, hfm_stream_t stream) {
  if (!m || cycles < 1) return fail(HFM_ERR_BAD_ARG, "hfm_mg_run: bad argument");
  cudaGraphExec_t exec = nullptr;
  auto it = m->graphs.find(cycles);
  if (it != m->graphs.end()) {
    exec = it->second;
  } else {
    cudaGraph_t graph = nullptr;
    HFM_CUDA(cudaStreamBeginCapture(m->cap, cudaStreamCaptureModeRelaxed));
    set_capturing(true);
    int st = m->eng->emit_cycles(cycles, m->cap);
    set_capturing(false);
    cudaError_t e = cudaStreamEndCapture(m->cap, &graph);
    if (st) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    size_t nn = 0;
    int64_t nk = 0;
    if (cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn) {
      std::vector<cudaGraphNode_t> nodes(nn);
      if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
        for (size_t i = 0; i < nn; ++i) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
        }
    }
    m->graph_kernels[cycles] = nk;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
    m->graphs[cycles] = exec;
  }
  HFM_CUDA(cudaGraphLaunch(exec, (cudaStream_t)stream));
  note_graph_launch(m->graph_kernels[cycles]);
  return HFM_OK;
}

int hfm_mg_query(hfm_mg *m, hfm_slot_stats *out, hfm_stream_t stream) {
  if (!m || !out) return fail(HFM_ERR_BAD_ARG, "hfm_mg_query: bad argument");
  std::vector<SlotState> st(m->slots);
  std::vector<int> act(m->slots), outer(m->slots);
  cudaStream_t s = (cudaStream_t)stream;
  HFM_CUDA(cudaMemcpyAsync(st.data(), m->state, m->slots * sizeof(SlotState), cudaMemcpyDeviceToHost, s));
  HFM_CUDA(cudaMemcpyAsync(act.data(), m->active, m->slots * 4, cudaMemcpyDeviceToHost, s));
  HFM_CUDA(cudaMemcpyAsync(outer.data(), m->outer, m->slots * 4, cudaMemcpyDeviceToHost, s));
  HFM_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < m->slots; ++i) {
    out[i].active = act[i] | outer[i];
    out[i].status = st[i].status;
    out[i].cycles = st[i].cycles;
    out[i].outer = st[i].outer;
    out[i].norm_b = st[i].norm_b;
    out[i].rel_resid = st[i].rel;
  }
  return HFM_OK;
}

int hfm_mg_query_async(hfm_mg *m, hfm_slot_stats *stats_host, hfm_stream_t stream) {
  if (!m || !stats_host) return fail(HFM_ERR_BAD_ARG, "hfm_mg_query_async: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  k_pack_stats<<<(m->slots + 127) / 128, 128, 0, s>>>(m->state, m->active, m->outer, m->slots,
                                                      m->stats_dev);
  HFM_CHECK_LAUNCH("k_pack_stats");
  HFM_CUDA(cudaMemcpyAsync(stats_host, m->stats_dev, m->slots * sizeof(hfm_slot_stats),
                           cudaMemcpyDeviceToHost, s));
  return HFM_OK;
}

int hfm_mg_fetch(hfm_mg *m, int slot, float *out, hfm_stream_t stream) {
  if (!m || !out || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_fetch: bad argument");
  return m->eng->fetch(slot, out, (cudaStream_t)stream);
}

int hfm_mg_cancel(hfm_mg *m, int slot, hfm_stream_t stream) {
  if (!m || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_cancel: bad argument");
  HFM_CUDA(cudaMemsetAsync(m->active + slot, 0, 4, (cudaStream_t)stream));
  HFM_CUDA(cudaMemsetAsync(m->outer + slot, 0, 4, (cudaStream_t)stream));
  return HFM_OK;
}

int hfm_mg_load_f64(hfm_mg *m, int slot, const double *rhs, const double *phi0,
                    hfm_stream_t stream) {
  if (!m || !rhs || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_load_f64: bad argument");
  return m->eng->load64(slot, rhs, phi0, (cudaStream_t)stream);
}

int hfm_mg_fetch_f64(hfm_mg *m, int slot, double *phi_out, hfm_stream_t stream) {
  if (!m || !phi_out || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_fetch_f64: bad argument");
  return m->eng->fetch64(slot, phi_out, (cudaStream_t)stream);
}

int hfm_mg_read_level(hfm_mg *m, int slot, int level, int which, float *out, hfm_stream_t stream) {
  if (!m || !out || slot < 0 || slot >= m->slots) return fail(HFM_ERR_BAD_ARG, "hfm_mg_read_level: bad argument");
  return m->eng->read_level(slot, level, which, out, (cudaStream_t)stream);
}

int hfm_mg_solve(hfm_mg *m, const float *rhs, float *phi, hfm_slot_stats *stats_host,
                 hfm_stream_t stream) {
  if (!m || !rhs || !phi) return fail(HFM_ERR_BAD_ARG, "hfm_mg_solve: bad argument");
  int st;
  if ((st = m->eng->load_all(rhs, (cudaStream_t)stream))) return st;
  std::vector<hfm_slot_stats> tmp(m->slots);
  hfm_slot_stats *ss = stats_host ? stats_host : tmp.data();
  const int per = m->cfg.cycles_per_launch;
  for (int done = 0; done <= m->cfg.max_cycles + per; done += per) {
    if ((st = hfm_mg_run(m, per, stream))) return st;
    if ((st = hfm_mg_query(m, ss, stream))) return st;
    bool any = false;
    for (int s = 0; s < m->slots; ++s) any |= ss[s].active != 0;
    if (!any) break;
  }
  if ((st = m->eng->fetch_all(phi, (cudaStream_t)stream))) return st;
  HFM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int worst = HFM_OK;
  for (int s = 0; s < m->slots; ++s)
    if (ss[s].status != HFM_OK) worst = ss[s].status;
  return worst;
}

}  // extern "C"
