// The coarse end of a V-cycle in one kernel: one thread block per instance runs the V-cycle
// of every level from l0 (at most 4096 cells) down to the coarsest and back, with all fields
// of those levels in shared memory.
//
// On the deep levels the stencil kernels are a few microseconds of work behind a launch and a
// dependency each (the 16^3, 8^3, 4^3 levels of 64 instances make ~15 launches per cycle);
// this kernel replaces them with one launch whose sweeps are separated by __syncthreads().
// The sequence is the one the multi-kernel V-cycle runs (nu_pre sweeps from zero, residual +
// 2x2x2 averaging restriction, recursion, coarsest level `coarse_sweeps` sweeps from zero with
// coarse_omega, nearest prolongation + correction fused with the first post-sweep, the
// remaining post-sweeps); iterates stay in float32 between sweeps (the multi-kernel path
// rounds them to the storage type).  Operators as the other kernels evaluate them, ghost
// phi = 0: SIGMA7 face coefficients c_d (s_i + s_j) / 2 (wall face c_d s_i); CONST7 the
// anisotropic 7-point stencil with diagonal 2 (kz + ky + kx); K27 any 3x3x3 kernel, diagonal
// its centre weight.
#include <algorithm>

#include "hfm_internal.cuh"

namespace hfm {

namespace {

constexpr int kSubThreads = 512;

// Shared-memory layout of one level (floats): phi and tmp with a one-cell ghost layer on every
// side, kept zero ((Z+2)(Y+2)(X+2) each), so a stencil reads its neighbours without bounds
// checks; rhs (Z Y X); for SIGMA7 the level's face coefficients Fx [Z][Y][X+1], Fy
// [Z][Y+1][X], Fz [Z+1][Y][X] (c_d (s_i + s_j) / 2, wall faces c_d s_i) and the diagonal
// (Z Y X), formed once per launch from the conductivities in global memory.
__host__ __device__ __forceinline__ int sub_padded(int Z, int Y, int X) { return (Z + 2) * (Y + 2) * (X + 2); }
__host__ __device__ __forceinline__ int sub_faces(int Z, int Y, int X) {
  return Z * Y * (X + 1) + Z * (Y + 1) * X + (Z + 1) * Y * X;
}

// Index of cell (z, y, x) (each may be -1 .. extent) in a padded field.
__device__ __forceinline__ int pix(int z, int y, int x, int Y, int X) {
  return ((z + 1) * (Y + 2) + (y + 1)) * (X + 2) + (x + 1);
}

// A phi at cell (z, y, x), whose padded index is ip, with its diagonal.  ph is a padded field
// (ghosts zero); the face coefficients (SIGMA7) and diagonals come from the level's shared
// arrays.  The products and sums are those the conductivity form evaluates.
template <int KIND, class T>
__device__ __forceinline__ float sub_apply(const SubLevel<T> &L, const float *ph, const float *Fc,
                                           int z, int y, int x, int ip, int i, float *diag) {
  const int X = L.X, Y = L.Y, Z = L.Z;
  const int PX = X + 2, PXY = (X + 2) * (Y + 2);
  if (KIND == HFM_OP_K27) {
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float wgt = L.k[9 * a + 3 * b + c];
          if (wgt != 0.f) acc += wgt * ph[ip + (a - 1) * PXY + (b - 1) * PX + (c - 1)];
        }
    *diag = L.k[13];
    return acc;
  }
  if (KIND == HFM_OP_CONST7) {
    const float kz = L.k[0], ky = L.k[1], kx = L.k[2], d = 2.f * (kz + ky + kx);
    *diag = d;
    return d * ph[ip] - kz * (ph[ip - PXY] + ph[ip + PXY]) - ky * (ph[ip - PX] + ph[ip + PX]) -
           kx * (ph[ip - 1] + ph[ip + 1]);
  }
  const float *fx = Fc, *fy = fx + Z * Y * (X + 1), *fz = fy + Z * (Y + 1) * X, *dg = fz + (Z + 1) * Y * X;
  const int ixf = (z * Y + y) * (X + 1) + x, iyf = (z * (Y + 1) + y) * X + x;
  const float axm = fx[ixf], axp = fx[ixf + 1];
  const float aym = fy[iyf], ayp = fy[iyf + X];
  const float azm = fz[i], azp = fz[i + X * Y];
  const float pc = ph[ip];
  *diag = dg[i];
  return axm * (pc - ph[ip - 1]) + axp * (pc - ph[ip + 1]) + aym * (pc - ph[ip - PX]) +
         ayp * (pc - ph[ip + PX]) + azm * (pc - ph[ip - PXY]) + azp * (pc - ph[ip + PXY]);
}

// Coordinates of the cells a thread visits in a block-strided loop over a Z x Y x X grid: the
// first from one division, the next ones by adding the stride's own coordinates with carries
// (dx < X, dy < Y, so at most one carry each) instead of dividing per cell.
struct Walk {
  int z, y, x, dz, dy, dx;
  __device__ Walk(int i, int stride, int Y, int X) {
    x = i % X;
    const int t = i / X;
    y = t % Y;
    z = t / Y;
    dx = stride % X;
    const int u = stride / X;
    dy = u % Y;
    dz = u / Y;
  }
  __device__ void step(int Y, int X) {
    x += dx;
    int cy = 0;
    if (x >= X) {
      x -= X;
      cy = 1;
    }
    y += dy + cy;
    int cz = 0;
    if (y >= Y) {
      y -= Y;
      cz = 1;
    }
    z += dz + cz;
  }
};

// out = in + om (f - A in) / diag over the level's cells (in may be null: a zero iterate;
// in and out are padded fields, only out's interior is written)
template <int KIND, class T>
__device__ void sub_sweep(const SubLevel<T> &L, const float *in, const float *Fc, const float *f,
                          float *out, float om, const float *zero_pad) {
  // a zero iterate: A in = 0 and the diagonal from zero_pad's call (a zero-filled field)
  const float *ph = in ? in : zero_pad;
  Walk w(threadIdx.x, blockDim.x, L.Y, L.X);
  for (int i = threadIdx.x; i < L.n; i += blockDim.x, w.step(L.Y, L.X)) {
    const int ip = pix(w.z, w.y, w.x, L.Y, L.X);
    float dg;
    float ax = sub_apply<KIND, T>(L, ph, Fc, w.z, w.y, w.x, ip, i, &dg);
    if (!in) ax = 0.f;
    const float pc = in ? in[ip] : 0.f;
    out[ip] = pc + om * __fdividef(f[i] - ax, dg);
  }
  __syncthreads();
}

// phi -= P(coarse) on the level's interior (nearest prolongation; phi identically zero when
// `zero`: phi = -P(coarse)).  Both fields padded.
template <class T>
__device__ void sub_correct(const SubLevel<T> &L, float *ph, const SubLevel<T> &Lc,
                            const float *coarse, bool zero) {
  Walk w(threadIdx.x, blockDim.x, L.Y, L.X);
  for (int i = threadIdx.x; i < L.n; i += blockDim.x, w.step(L.Y, L.X)) {
    const int ip = pix(w.z, w.y, w.x, L.Y, L.X);
    const float c = coarse[pix(w.z >> 1, w.y >> 1, w.x >> 1, Lc.Y, Lc.X)];
    ph[ip] = zero ? -c : ph[ip] - c;
  }
  __syncthreads();
}

// fc = R(A phi - f): 0.125 times the sum over each coarse cell's eight fine residuals (ph
// padded, or null for a zero iterate)
template <int KIND, class T>
__device__ void sub_resid_restrict(const SubLevel<T> &L, const float *ph, const float *Fc,
                                   const float *f, const SubLevel<T> &Lc, float *fc) {
  Walk w(threadIdx.x, blockDim.x, Lc.Y, Lc.X);
  for (int j = threadIdx.x; j < Lc.n; j += blockDim.x, w.step(Lc.Y, Lc.X)) {
    const int xc = w.x, yc = w.y, zc = w.z;
    float sum = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int z = 2 * zc + a, y = 2 * yc + b, x = 2 * xc + c;
          const int i = (z * L.Y + y) * L.X + x;
          float dg;
          const float ax = ph ? sub_apply<KIND, T>(L, ph, Fc, z, y, x, pix(z, y, x, L.Y, L.X), i, &dg) : 0.f;
          sum += ax - f[i];
        }
    fc[j] = 0.125f * sum;
  }
  __syncthreads();
}

// A 16-bit or float32 value read through L2 (ld.global.cg): data another block of the same
// launch may have written (the persistent kernel's restricted residual).
template <class T> __device__ __forceinline__ T ld_l2(const T *p);
template <> __device__ __forceinline__ float ld_l2<float>(const float *p) { return __ldcg(p); }
template <> __device__ __forceinline__ __nv_bfloat16 ld_l2<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __ushort_as_bfloat16(__ldcg(reinterpret_cast<const unsigned short *>(p)));
}
template <> __device__ __forceinline__ __half ld_l2<__half>(const __half *p) {
  return __ushort_as_half(__ldcg(reinterpret_cast<const unsigned short *>(p)));
}

// The face coefficients and diagonals of a SIGMA7 level of instance `inst` into its shared
// arrays, from the conductivities in global memory, as the conductivity form forms them.
template <class T>
__device__ void sub_faces_init(const SubLevel<T> &L, int64_t inst, float *Fc) {
  const int X = L.X, Y = L.Y, Z = L.Z;
  const int64_t g = inst * (int64_t)L.n;
  const T *sx = L.sx + g, *sy = L.sy + g, *sz = L.sz + g;
  float *fx = Fc, *fy = fx + Z * Y * (X + 1), *fz = fy + Z * (Y + 1) * X;
  const int nx = Z * Y * (X + 1), ny = Z * (Y + 1) * X, nz = (Z + 1) * Y * X;
  for (int k = threadIdx.x; k < nx; k += blockDim.x) {
    const int i = k % (X + 1), row = k / (X + 1);
    const float a = i > 0 ? St<T>::to(sx[row * X + i - 1]) : 0.f, b = i < X ? St<T>::to(sx[row * X + i]) : 0.f;
    fx[k] = L.cx * (i == 0 ? b : (i == X ? a : 0.5f * (b + a)));
  }
  for (int k = threadIdx.x; k < ny; k += blockDim.x) {
    const int x = k % X, t = k / X, j = t % (Y + 1), z = t / (Y + 1);
    const int c0 = (z * Y + j) * X + x;
    const float a = j > 0 ? St<T>::to(sy[c0 - X]) : 0.f, b = j < Y ? St<T>::to(sy[c0]) : 0.f;
    fy[k] = L.cy * (j == 0 ? b : (j == Y ? a : 0.5f * (b + a)));
  }
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    const int yx = k % (Y * X), kz = k / (Y * X);
    const float a = kz > 0 ? St<T>::to(sz[(kz - 1) * Y * X + yx]) : 0.f, b = kz < Z ? St<T>::to(sz[kz * Y * X + yx]) : 0.f;
    fz[k] = L.cz * (kz == 0 ? b : (kz == Z ? a : 0.5f * (b + a)));
  }
  __syncthreads();
  float *dg = fz + nz;
  Walk w(threadIdx.x, blockDim.x, Y, X);
  for (int i = threadIdx.x; i < L.n; i += blockDim.x, w.step(Y, X)) {
    const int ixf = (w.z * Y + w.y) * (X + 1) + w.x, iyf = (w.z * (Y + 1) + w.y) * X + w.x;
    dg[i] = fx[ixf] + fx[ixf + 1] + fy[iyf] + fy[iyf + X] + fz[i] + fz[i + X * Y];
  }
}

// The coarse-end V-cycle of one instance with the block's shared memory `sub_smem`.  COH:
// the right-hand side was written by other blocks of the same launch (read through L2).
template <int KIND, class T, bool COH>
__device__ void subcycle_body(const SubArgs<T> &a, int64_t inst, unsigned char *sub_smem) {
  float *F = reinterpret_cast<float *>(sub_smem);
  const int nl = a.nlev;
  // zero every padded field (ghosts stay zero: sweeps write interiors only), faces, rhs
  for (int l = 0; l < nl; ++l) {
    const SubLevel<T> &L = a.lv[l];
    const int np = 2 * sub_padded(L.Z, L.Y, L.X);
    for (int i = threadIdx.x; i < np; i += blockDim.x) F[L.o_phi + i] = 0.f;
    if (KIND == HFM_OP_SIGMA7) sub_faces_init<T>(L, inst, F + L.o_face);
  }
  for (int i = threadIdx.x; i < a.lv[0].n; i += blockDim.x) {
    const T *src = a.rhs + inst * (int64_t)a.lv[0].n + i;
    F[a.lv[0].o_rhs + i] = St<T>::to(COH ? ld_l2<T>(src) : *src);
  }
  __syncthreads();

  int cur[kMaxSubLevels];    // 0: iterate in phi, 1: in tmp
  bool zero[kMaxSubLevels];  // iterate still identically zero (nu_pre == 0)
  // down: pre-smoothing from zero, residual, restriction
  for (int l = 0; l < nl - 1; ++l) {
    const SubLevel<T> &L = a.lv[l];
    float *buf[2] = {F + L.o_phi, F + L.o_tmp};
    const float *f = F + L.o_rhs, *Fc = F + L.o_face;
    int c = 0;
    for (int k = 0; k < a.nu_pre; ++k) {
      sub_sweep<KIND, T>(L, k == 0 ? nullptr : buf[c], Fc, f, buf[c ^ 1], a.omega, buf[c]);
      c ^= 1;
    }
    cur[l] = c;
    zero[l] = a.nu_pre == 0;
    sub_resid_restrict<KIND, T>(L, zero[l] ? nullptr : buf[c], Fc, f, a.lv[l + 1], F + a.lv[l + 1].o_rhs);
  }
  // coarsest: coarse_sweeps sweeps from zero; a level of at most 64 cells (4^3, 3^3) on one
  // warp, two cells a lane with their indices computed once, __syncwarp() between the
  // sweeps instead of a block barrier (the per-cell arithmetic is sub_sweep's)
  {
    const SubLevel<T> &L = a.lv[nl - 1];
    float *buf[2] = {F + L.o_phi, F + L.o_tmp};
    const float *Fc = F + L.o_face;
    int c = 0;
    if (L.n <= 64 && a.coarse_sweeps > 0) {
      if (threadIdx.x < 32) {
        const float *f = F + L.o_rhs;
        int zz[2], yy[2], xx[2], ipp[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int i = threadIdx.x + 32 * q;
          xx[q] = i % L.X;
          const int t = i / L.X;
          yy[q] = t % L.Y;
          zz[q] = t / L.Y;
          ipp[q] = pix(zz[q], yy[q], xx[q], L.Y, L.X);
        }
        for (int k = 0; k < a.coarse_sweeps; ++k) {
          const float *in = k == 0 ? nullptr : buf[c];
          float *out = buf[c ^ 1];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int i = threadIdx.x + 32 * q;
            if (i < L.n) {
              float dg;
              const float ax = sub_apply<KIND, T>(L, in ? in : buf[c], Fc, zz[q], yy[q], xx[q], ipp[q], i, &dg);
              const float axv = in ? ax : 0.f;
              const float pc = in ? in[ipp[q]] : 0.f;
              out[ipp[q]] = pc + a.coarse_omega * __fdividef(f[i] - axv, dg);
            }
          }
          __syncwarp();
          c ^= 1;
        }
      } else {
        c = a.coarse_sweeps & 1;
      }
      __syncthreads();
    } else {
      for (int k = 0; k < a.coarse_sweeps; ++k) {
        sub_sweep<KIND, T>(L, k == 0 ? nullptr : buf[c], Fc, F + L.o_rhs, buf[c ^ 1], a.coarse_omega, buf[c]);
        c ^= 1;
      }
    }
    cur[nl - 1] = c;
  }
  // up: prolongation + correction (in place), then the post-sweeps
  const int post = a.nu_post > 0 ? a.nu_post : 1;
  for (int l = nl - 2; l >= 0; --l) {
    const SubLevel<T> &L = a.lv[l];
    const SubLevel<T> &Lc = a.lv[l + 1];
    float *buf[2] = {F + L.o_phi, F + L.o_tmp};
    const float *coarse = F + (cur[l + 1] ? Lc.o_tmp : Lc.o_phi);
    const float *Fc = F + L.o_face;
    int c = cur[l];
    sub_correct<T>(L, buf[c], Lc, coarse, zero[l]);
    for (int k = 0; k < post; ++k) {
      const float om = a.nu_post == 0 ? 0.f : a.omega;
      sub_sweep<KIND, T>(L, buf[c], Fc, F + L.o_rhs, buf[c ^ 1], om, buf[c]);
      c ^= 1;
    }
    cur[l] = c;
  }
  const SubLevel<T> &L0 = a.lv[0];
  const float *res = F + (cur[0] ? L0.o_tmp : L0.o_phi);
  Walk w(threadIdx.x, blockDim.x, L0.Y, L0.X);
  for (int i = threadIdx.x; i < L0.n; i += blockDim.x, w.step(L0.Y, L0.X))
    a.out[inst * (int64_t)L0.n + i] = St<T>::from(res[pix(w.z, w.y, w.x, L0.Y, L0.X)]);
}

template <int KIND, class T>
__global__ void __launch_bounds__(kSubThreads) k_subcycle(const __grid_constant__ SubArgs<T> a) {
  const int64_t inst = blockIdx.x;
  if (a.active && !a.active[inst]) return;
  extern __shared__ __align__(16) unsigned char sub_smem[];
  subcycle_body<KIND, T, false>(a, inst, sub_smem);
}

}  // namespace

size_t subcycle_smem_bytes(const Grid3 *g, int nlev, bool sigma) {
  size_t f = 0;
  for (int l = 0; l < nlev; ++l) {
    const int Z = g[l].Z, Y = g[l].Y, X = g[l].X, n = Z * Y * X;
    f += (size_t)2 * sub_padded(Z, Y, X) + n;
    if (sigma) f += (size_t)sub_faces(Z, Y, X) + n;
  }
  return ((f * 4 + 15) / 16) * 16;
}

template <int KIND, class T>
int go_subcycle(const SubArgs<T> &a, int B, size_t smem, cudaStream_t s) {
  int st = set_max_dynamic_smem((const void *)k_subcycle<KIND, T>, (int)kSubcycleMaxSmem,
                                "cudaFuncSetAttribute(k_subcycle)");
  if (st) return st;
  k_subcycle<KIND, T><<<B, kSubThreads, smem, s>>>(a);
  HFM_CHECK_LAUNCH("k_subcycle");
  return HFM_OK;
}

// Shared-memory layout of the coarse-end cycle, level after level: phi and tmp (padded), rhs,
// and for SIGMA7 the face arrays and the diagonal.  Returns the bytes, 0 if they exceed the
// limit.
template <class T> size_t layout_sub(int kind, SubArgs<T> &a) {
  Grid3 g[kMaxSubLevels];
  int off = 0;
  for (int l = 0; l < a.nlev; ++l) {
    SubLevel<T> &L = a.lv[l];
    g[l] = Grid3{L.Z, L.Y, L.X};
    const int np = sub_padded(L.Z, L.Y, L.X);
    L.o_phi = off;
    L.o_tmp = off + np;
    L.o_rhs = off + 2 * np;
    L.o_face = L.o_rhs + L.n;
    off = L.o_face + (kind == HFM_OP_SIGMA7 ? sub_faces(L.Z, L.Y, L.X) + L.n : 0);
  }
  const size_t smem = subcycle_smem_bytes(g, a.nlev, kind == HFM_OP_SIGMA7);
  return smem > kSubcycleMaxSmem ? 0 : smem;
}

// ------------------------------------------------------------------ persistent small end
// Level l1 of a V-cycle and the coarse end below it in one launch.  A block takes work items
// in order from a global ticket: (step, instance, z tile) for the sweeps and the residual +
// restriction of level l1, (SUB, instance) for the coarse end, which runs in the block's
// shared memory exactly as k_subcycle does.  Items are numbered step by step, so an item
// only waits for items with smaller numbers - items other running blocks have already taken
// - and the waits always end; each is still bounded (the wait budget), and one that runs out
// is counted in the device's wait-failure counters (the handle then ends its slots with
// HFM_ERR_TIMEOUT) and the item is skipped.  Iterates, the restricted residual and the
// correction written in this launch are read through L2; conductivities, 1 / diag and f are
// read-only here.

// Iterate source of a sweep of the persistent kernel: phi' = (src or 0) - P(wc), or the
// fused first sweep's phi1 = omega f / diag.
template <class T> struct SmallPhi {
  const T *base, *corr, *f, *invd;
  int64_t stride, cstride;
  int Yc, Xc;
  float omega;
  int pre2;
  __device__ __forceinline__ float operator()(int64_t inst, int z, int y, int x, int Y, int X) const {
    const int64_t i = inst * stride + ((int64_t)z * Y + y) * X + x;
    if (pre2) return omega * St<T>::ld(f + i) * St<T>::ld(invd + i);
    float v = base ? St<T>::to(ld_l2<T>(base + i)) : 0.f;
    if (corr) v -= St<T>::to(ld_l2<T>(corr + inst * cstride + ((int64_t)(z >> 1) * Yc + (y >> 1)) * Xc + (x >> 1)));
    return v;
  }
};

template <int KIND, class T>
__device__ void small_sweep(const SmallArgs<T> &a, int sidx, int64_t inst, int tile) {
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int z0 = tile * a.zc, z1 = min(Z, z0 + a.zc);
  SmallPhi<T> ph;
  ph.base = a.src[sidx] >= 0 ? a.buf[a.src[sidx]] : nullptr;
  ph.corr = a.corr[sidx] ? a.sub.out : nullptr;
  ph.f = a.f;
  ph.invd = a.invd;
  ph.stride = a.n;
  ph.cstride = a.sub.lv[0].n;
  ph.Yc = a.sub.lv[0].Y;
  ph.Xc = a.sub.lv[0].X;
  ph.omega = a.om[sidx];
  ph.pre2 = a.kind[sidx] == SK_PRE2;
  T *out = a.buf[a.dst[sidx]] + inst * a.n;
  const float om = a.om[sidx];
  double acc = 0.0;
  const int64_t cells = (int64_t)(z1 - z0) * Y * X;
  for (int64_t k = threadIdx.x; k < cells; k += blockDim.x) {
    const int x = (int)(k % X);
    const int64_t t = k / X;
    const int y = (int)(t % Y), z = z0 + (int)(t / Y);
    float dg;
    const float ax = op_apply_at<KIND, T>(a.op, ph, inst, z, y, x, Z, Y, X, &dg);
    const int64_t i = ((int64_t)z * Y + y) * X + x;
    const float fv = St<T>::ld(a.f + inst * a.n + i);
    const float pc = ph(inst, z, y, x, Y, X);
    const float v = pc + om * __fdividef(fv - ax, dg);
    out[i] = St<T>::from(v);
    if (a.dot[sidx]) acc += (double)v * fv;
  }
  if (a.dot[sidx] && a.partials) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
      a.partials[inst * a.tiles + tile] = tot;
    }
  }
}

// r_c = R(A phi - f) for the coarse planes of z tile `tile` (zc even).
template <int KIND, class T>
__device__ void small_restrict(const SmallArgs<T> &a, int sidx, int64_t inst, int tile) {
  const int X = a.X, Y = a.Y, Z = a.Z;
  const SubLevel<T> &C = a.sub.lv[0];
  SmallPhi<T> ph;
  ph.base = a.src[sidx] >= 0 ? a.buf[a.src[sidx]] : nullptr;
  ph.corr = nullptr;
  ph.f = a.f;
  ph.invd = a.invd;
  ph.stride = a.n;
  ph.pre2 = 0;
  T *fc = const_cast<T *>(a.sub.rhs) + inst * (int64_t)C.n;
  const int c0 = tile * a.zc / 2, c1 = min(C.Z, (tile * a.zc + a.zc) / 2);
  const int64_t cells = (int64_t)(c1 - c0) * C.Y * C.X;
  for (int64_t k = threadIdx.x; k < cells; k += blockDim.x) {
    const int xc = (int)(k % C.X);
    const int64_t t = k / C.X;
    const int yc = (int)(t % C.Y), zcc = c0 + (int)(t / C.Y);
    float sum = 0.f;
#pragma unroll
    for (int aa = 0; aa < 2; ++aa)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int z = 2 * zcc + aa, y = 2 * yc + bb, x = 2 * xc + cc;
          float dg;
          const float ax = op_apply_at<KIND, T>(a.op, ph, inst, z, y, x, Z, Y, X, &dg);
          sum += 0.125f * (ax - St<T>::ld(a.f + inst * a.n + ((int64_t)z * Y + y) * X + x));
        }
    fc[((int64_t)zcc * C.Y + yc) * C.X + xc] = St<T>::from(sum);
  }
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int KIND, class T>
__global__ void __launch_bounds__(kSubThreads) k_small(const __grid_constant__ SmallArgs<T> a) {
  extern __shared__ __align__(16) unsigned char sub_smem[];
  __shared__ int item_sh, ok_sh;
  const int total = a.base[a.nsteps];
  for (;;) {
    if (threadIdx.x == 0) item_sh = atomicAdd(a.ticket, 1);
    __syncthreads();
    const int item = item_sh;
    if (item >= total) break;
    int s = 0;
    while (item >= a.base[s + 1]) ++s;
    const int cnt = a.kind[s] == SK_SUB ? 1 : a.tiles;
    const int local = item - a.base[s];
    const int64_t inst = local / cnt;
    const int tile = local % cnt;
    if (a.active && !a.active[inst]) {
      __syncthreads();  // item_sh is rewritten by the next take
      continue;
    }
    if (threadIdx.x == 0) {
      int ok = 1;
      if (a.need[s] > 0) {
        ok = 0;
        for (int i = 0; i < a.wait_budget; ++i)
          if (ld_acquire(a.done + inst) >= a.need[s]) {
            ok = 1;
            break;
          }
        if (!ok) atomicAdd(a.wait_fail, 1);
      }
      ok_sh = ok;
    }
    __syncthreads();
    if (ok_sh) {
      if (a.kind[s] == SK_SUB) subcycle_body<KIND, T, true>(a.sub, inst, sub_smem);
      else if (a.kind[s] == SK_RESTRICT) small_restrict<KIND, T>(a, s, inst, tile);
      else small_sweep<KIND, T>(a, s, inst, tile);
    }
    // publish: every thread's writes, then the instance's count
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(a.done + inst, 1);
  }
}

template <int KIND, class T>
int go_small(const SmallArgs<T> &a, size_t smem, cudaStream_t s) {
  const void *fn = (const void *)k_small<KIND, T>;
  int st = set_max_dynamic_smem(fn, (int)kSubcycleMaxSmem, "cudaFuncSetAttribute(k_small)");
  if (st) return st;
  int per_sm = 0;
  HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSubThreads, smem));
  if (per_sm < 1) per_sm = 1;
  const int total = a.base[a.nsteps];
  const int blocks = std::min(total, per_sm * sm_count());
  k_small<KIND, T><<<blocks, kSubThreads, smem, s>>>(a);
  HFM_CHECK_LAUNCH("k_small");
  return HFM_OK;
}

template <class T>
int launch_small(int kind, SmallArgs<T> a, int B, cudaStream_t s) {
  const size_t smem = layout_sub<T>(kind, a.sub);
  if (!smem) return fail(HFM_ERR_BAD_ARG, "small-level kernel: coarse levels exceed shared memory");
  (void)B;
  switch (kind) {
    case HFM_OP_SIGMA7: return go_small<HFM_OP_SIGMA7, T>(a, smem, s);
    case HFM_OP_CONST7: return go_small<HFM_OP_CONST7, T>(a, smem, s);
    case HFM_OP_K27: return go_small<HFM_OP_K27, T>(a, smem, s);
    default: return fail(HFM_ERR_UNSUPPORTED, "small-level kernel: operator kind");
  }
}

template int launch_small<float>(int, SmallArgs<float>, int, cudaStream_t);
template int launch_small<__nv_bfloat16>(int, SmallArgs<__nv_bfloat16>, int, cudaStream_t);
template int launch_small<__half>(int, SmallArgs<__half>, int, cudaStream_t);

template <class T>
int launch_subcycle(int kind, SubArgs<T> a, int B, cudaStream_t s) {
  const size_t smem = layout_sub<T>(kind, a);
  if (!smem) return fail(HFM_ERR_BAD_ARG, "subcycle: levels exceed shared memory");
  switch (kind) {
    case HFM_OP_SIGMA7: return go_subcycle<HFM_OP_SIGMA7, T>(a, B, smem, s);
    case HFM_OP_CONST7: return go_subcycle<HFM_OP_CONST7, T>(a, B, smem, s);
    case HFM_OP_K27: return go_subcycle<HFM_OP_K27, T>(a, B, smem, s);
    default: return fail(HFM_ERR_UNSUPPORTED, "subcycle: operator kind");
  }
}

template int launch_subcycle<float>(int, SubArgs<float>, int, cudaStream_t);
template int launch_subcycle<__nv_bfloat16>(int, SubArgs<__nv_bfloat16>, int, cudaStream_t);
template int launch_subcycle<__half>(int, SubArgs<__half>, int, cudaStream_t);

}  // namespace hfm
