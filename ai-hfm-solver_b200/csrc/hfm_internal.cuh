// Internal declarations shared by the libhfm translation units.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <string>

#include "../../include/hfm.h"

namespace hfm {

// ------------------------------------------------------------------ error reporting
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

#define HFM_CUDA(call)                                                    \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) return ::hfm::cuda_status(e_, #call);          \
  } while (0)

// Counts every kernel the library enqueues: direct launches here, graph launches by the
// number of kernel nodes of the graph (launches made while capturing are not counted).
void note_launch();
void note_graph_launch(int64_t kernel_nodes);
void set_capturing(bool on);

#define HFM_CHECK_LAUNCH(what)                                            \
  do {                                                                    \
    cudaError_t e_ = cudaGetLastError();                                  \
    if (e_ != cudaSuccess) return ::hfm::cuda_status(e_, what);           \
    ::hfm::note_launch();                                                 \
  } while (0)

int sm_count();  // SMs of the current device (cached per device)
// Device address (current device) of the two TMA wait-failure counters: [0] plane waits that
// expired, [1] drain waits that expired.  Kernels that must not report success after a
// failed wait read them.
int wait_fail_counters(const int **out);
int current_wait_budget();  // polls of a bounded device wait (hfm_set_wait_budget)
// Raise a kernel's dynamic shared-memory limit on the current device, once per device and
// kernel (a process that drives several GPUs needs it on each).
int set_max_dynamic_smem(const void *kernel, int bytes, const char *what);

// ------------------------------------------------------------------ storage types
template <class T> struct St;
template <> struct St<float> {
  static __device__ __forceinline__ float ld(const float *p) { return __ldg(p); }
  static __device__ __forceinline__ float to(float v) { return v; }
  static __device__ __forceinline__ float from(float v) { return v; }
};
template <> struct St<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) {
    return __bfloat162float(__ldg(p));
  }
  static __device__ __forceinline__ __nv_bfloat16 from(float v) { return __float2bfloat16(v); }
  static __device__ __forceinline__ float to(__nv_bfloat16 v) { return __bfloat162float(v); }
};
template <> struct St<__half> {
  static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
  // saturating: a transient value beyond the fp16 range is stored as +-65504, not inf
  static __device__ __forceinline__ __half from(float v) {
    return __float2half(fminf(fmaxf(v, -65504.f), 65504.f));
  }
  static __device__ __forceinline__ float to(__half v) { return __half2float(v); }
};

// ------------------------------------------------------------------ operator on device
// Resolved operator for one level: `coef` point at instance 0, instance i is at
// coef + i * coef_stride.  `k` already includes `scale` (coefficients for CONST7/K27),
// and `scale` is kept for the array forms (SIGMA7 / DIR7) whose coefficients are in memory.
// Internal launch flag (never set by callers): residual kernels accumulate sum(res * phi)
// instead of sum(res^2) in their partials, i.e. p . (A p) for CG when b is absent.
constexpr unsigned HFM_INT_DOT_PHI = 1u << 30;
// Internal launch flag: smoothing kernels write block partial sums of out * rhs (z . r for a
// CG preconditioner whose right-hand side is r) when given a partials buffer.
constexpr unsigned HFM_INT_DOT_RHS = 1u << 29;

struct DevOp {
  float k[27];
  float c[3];  // cz, cy, cx
  float scale;
  const void *coef[7];
  int64_t coef_stride;
};

DevOp make_devop(const hfm_operator &op, int64_t coef_stride);

// phi'(cell) = base(cell) + corr_sign * corr(cell or its parent), optionally zero on x = X-1.
template <class T> struct PhiSrc {
  const T *base;
  const T *corr;
  int64_t base_stride, corr_stride;
  float corr_sign;
  int corr_coarse;  // corr lives on the coarse grid (Zc, Yc, Xc) = fine / 2
  int Yc, Xc;
  int zero_xend;
  __device__ __forceinline__ float operator()(int64_t inst, int z, int y, int x, int Y,
                                              int X) const {
    if (zero_xend && x == X - 1) return 0.f;
    float v = 0.f;
    if (base) v = St<T>::ld(base + inst * base_stride + ((int64_t)z * Y + y) * X + x);
    if (corr) {
      int64_t ci = corr_coarse ? (((int64_t)(z >> 1) * Yc + (y >> 1)) * Xc + (x >> 1))
                               : (((int64_t)z * Y + y) * X + x);
      v += corr_sign * St<T>::ld(corr + inst * corr_stride + ci);
    }
    return v;
  }
};

// FACE7 arrays: elements per instance of Fx [Z][Y][X + 8], Fy [Z][Y + 1][X], Fz [Z + 1][Y][X].
__host__ __device__ __forceinline__ int64_t face7_nx(int Z, int Y, int X) { return (int64_t)Z * Y * (X + 8); }
__host__ __device__ __forceinline__ int64_t face7_ny(int Z, int Y, int X) { return (int64_t)Z * (Y + 1) * X; }
__host__ __device__ __forceinline__ int64_t face7_nz(int Z, int Y, int X) { return (int64_t)(Z + 1) * Y * X; }

// Evaluate (A phi')(z,y,x) and the Jacobi diagonal for operator KIND.
template <int KIND, class T, class F>
__device__ __forceinline__ float op_apply_at(const DevOp &op, const F &phi, int64_t inst,
                                             int z, int y, int x, int Z, int Y, int X,
                                             float *diag) {
  auto P = [&](int zz, int yy, int xx) -> float {
    if (zz < 0 || zz >= Z || yy < 0 || yy >= Y || xx < 0 || xx >= X) return 0.f;
    return phi(inst, zz, yy, xx, Y, X);
  };
  if (KIND == HFM_OP_K27) {
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float w = op.k[9 * a + 3 * b + c];
          if (w != 0.f) acc += w * P(z + a - 1, y + b - 1, x + c - 1);
        }
    *diag = op.k[13];
    return acc;
  } else if (KIND == HFM_OP_CONST7) {
    const float kz = op.k[0], ky = op.k[1], kx = op.k[2];
    const float d = 2.f * (kz + ky + kx);
    float pc = P(z, y, x);
    *diag = d;
    return d * pc - kz * (P(z - 1, y, x) + P(z + 1, y, x)) - ky * (P(z, y - 1, x) + P(z, y + 1, x)) -
           kx * (P(z, y, x - 1) + P(z, y, x + 1));
  } else if (KIND == HFM_OP_SIGMA7) {
    const T *sx = (const T *)op.coef[0] + inst * op.coef_stride;
    const T *sy = (const T *)op.coef[1] + inst * op.coef_stride;
    const T *sz = (const T *)op.coef[2] + inst * op.coef_stride;
    const int64_t i = ((int64_t)z * Y + y) * X + x;
    const float s = op.scale;
    const float cz = op.c[0] * s, cy = op.c[1] * s, cx = op.c[2] * s;
    float pc = P(z, y, x);
    float vx = St<T>::ld(sx + i), vy = St<T>::ld(sy + i), vz = St<T>::ld(sz + i);
    float axm = cx * (x > 0 ? 0.5f * (vx + St<T>::ld(sx + i - 1)) : vx);
    float axp = cx * (x < X - 1 ? 0.5f * (vx + St<T>::ld(sx + i + 1)) : vx);
    float aym = cy * (y > 0 ? 0.5f * (vy + St<T>::ld(sy + i - X)) : vy);
    float ayp = cy * (y < Y - 1 ? 0.5f * (vy + St<T>::ld(sy + i + X)) : vy);
    const int64_t P2 = (int64_t)X * Y;
    float azm = cz * (z > 0 ? 0.5f * (vz + St<T>::ld(sz + i - P2)) : vz);
    float azp = cz * (z < Z - 1 ? 0.5f * (vz + St<T>::ld(sz + i + P2)) : vz);
    *diag = axm + axp + aym + ayp + azm + azp;
    return axm * (pc - P(z, y, x - 1)) + axp * (pc - P(z, y, x + 1)) +
           aym * (pc - P(z, y - 1, x)) + ayp * (pc - P(z, y + 1, x)) +
           azm * (pc - P(z - 1, y, x)) + azp * (pc - P(z + 1, y, x));
  } else if (KIND == HFM_OP_FACE7) {
    const T *fx = (const T *)op.coef[0] + inst * face7_nx(Z, Y, X) + ((int64_t)z * Y + y) * (X + 8) + x;
    const T *fy = (const T *)op.coef[1] + inst * face7_ny(Z, Y, X) + ((int64_t)z * (Y + 1) + y) * X + x;
    const T *fz = (const T *)op.coef[2] + inst * face7_nz(Z, Y, X) + ((int64_t)z * Y + y) * X + x;
    const float s = op.scale;
    const float axm = s * St<T>::ld(fx), axp = s * St<T>::ld(fx + 1);
    const float aym = s * St<T>::ld(fy), ayp = s * St<T>::ld(fy + X);
    const float azm = s * St<T>::ld(fz), azp = s * St<T>::ld(fz + (int64_t)Y * X);
    float pc = P(z, y, x);
    *diag = ((axm + axp) + (aym + ayp)) + (azm + azp);
    return axm * (pc - P(z, y, x - 1)) + axp * (pc - P(z, y, x + 1)) +
           aym * (pc - P(z, y - 1, x)) + ayp * (pc - P(z, y + 1, x)) +
           azm * (pc - P(z - 1, y, x)) + azp * (pc - P(z + 1, y, x));
  } else {  // HFM_OP_DIR7
    const int64_t i = ((int64_t)z * Y + y) * X + x + inst * op.coef_stride;
    const float s = op.scale;
    float pc = P(z, y, x);
    auto A = [&](int d) { return s * St<T>::ld((const T *)op.coef[d] + i); };
    *diag = A(6);
    return A(0) * (pc - P(z, y, x - 1)) + A(1) * (pc - P(z, y, x + 1)) +
           A(2) * (pc - P(z, y - 1, x)) + A(3) * (pc - P(z, y + 1, x)) +
           A(4) * (pc - P(z - 1, y, x)) + A(5) * (pc - P(z + 1, y, x));
  }
}

// ------------------------------------------------------------------ generic launchers
// (ops_generic.cu).  All take instance strides in elements and an optional per-instance
// `active` mask (nullptr = all instances) and optional per-block float64 partial sums of the
// squared output (`partials`, laid out [inst][block]); `nblk_out` returns blocks per instance.
struct Grid3 {
  int Z, Y, X;
  int64_t n() const { return (int64_t)Z * Y * X; }
};

template <class T>
int launch_smooth(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                  int64_t rhs_stride, T *out, int64_t out_stride, int B, Grid3 g, float omega,
                  unsigned flags, const int *active, cudaStream_t s, double *partials = nullptr,
                  int *nblk_out = nullptr);
template <class T>
int launch_residual(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *b,
                    int64_t b_stride, T *r, int64_t r_stride, int B, Grid3 g, unsigned flags,
                    const int *active, double *partials, int *nblk_out, cudaStream_t s);
template <class T>
int launch_apply(int kind, const DevOp &op, const PhiSrc<T> &phi, T *out, int64_t out_stride,
                 int B, Grid3 g, const int *active, cudaStream_t s);
// Fused residual + restriction on an even grid g (fine).  r_fine may be null.
template <class T>
int launch_residual_restrict(int kind, const DevOp &op, const PhiSrc<T> &phi, const T *b,
                             int64_t b_stride, T *r_fine, int64_t rf_stride, T *r_coarse,
                             int64_t rc_stride, int B, Grid3 g, unsigned flags,
                             const int *active, double *partials, int *nblk_out,
                             cudaStream_t s);
template <class T>
int launch_restrict(const T *fine, int64_t f_stride, T *coarse, int64_t c_stride, int B,
                    Grid3 g, const int *active, cudaStream_t s);
template <class T>
int launch_prolong(const T *coarse, int64_t c_stride, T *fine, int64_t f_stride, int B,
                   Grid3 gc, const int *active, cudaStream_t s);
// Three same-shape arrays (the conductivities) restricted by one launch where the vector
// kernel applies.
template <class T>
int launch_restrict3(const T *const fine[3], int64_t f_stride, T *const coarse[3], int64_t c_stride,
                     int B, Grid3 g, cudaStream_t s);
// Jacobi sweeps on a small grid held in shared memory, one block per instance.
template <class T>
int launch_coarse_jacobi(int kind, const DevOp &op, const T *rhs, int64_t rhs_stride,
                         const T *phi0, T *out, int64_t stride, int B, Grid3 g, float omega,
                         int sweeps, const int *active, cudaStream_t s);
int coarse_smem_limit();  // max cells for launch_coarse_jacobi

// Plane-marching kernels (ops_fast.cu) for X % 4 == 0; mode 0 smooth, 1 residual,
// 2 residual + restriction.  The generic launchers call them when fast_eligible().
enum { FAST_SMOOTH = 0, FAST_RESID = 1, FAST_RESTRICT = 2 };
bool fast_eligible(int kind, Grid3 g, bool restrict_mode);
template <class T>
int fast_launch(int kind, int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                T *out, T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g,
                float omega, unsigned flags, const int *active, double *partials,
                int *nblk_out, cudaStream_t s);
// TMA-pipelined kernels (ops_tma.cu) for X >= 64: same modes as fast_launch.
bool tma_eligible(int kind, Grid3 g, int mode, const void *corr, int corr_coarse, int es);
// Vector access alignment: every pointer the plane-marching kernels load or store in vectors
// is aligned to `bytes` (16 for the TMA kernels, whose tensor maps also need it; 4 elements
// for the register-queue kernels) and so are the per-instance strides.  Callers whose
// pointers violate this take the generic one-cell-per-thread kernels.
template <class T>
bool vec_aligned(int kind, const DevOp &op, const PhiSrc<T> &phi, const void *rhs,
                 const void *out, const void *coarse, int64_t stride, int64_t bytes) {
  auto al = [bytes](const void *p) { return ((uintptr_t)p % (uintptr_t)bytes) == 0; };
  const int64_t es = (int64_t)sizeof(T);
  if (!al(phi.base) || !al(phi.corr) || !al(rhs) || !al(out) || !al(coarse)) return false;
  if ((stride * es) % bytes) return false;
  if (phi.corr && (phi.corr_stride * es) % bytes) return false;
  if (kind == HFM_OP_SIGMA7) {
    for (int k = 0; k < 3; ++k)
      if (!al(op.coef[k])) return false;
    if ((op.coef_stride * es) % bytes) return false;
  }
  if (kind == HFM_OP_FACE7) {  // instance strides follow from the extents (rows of X + 8 / X)
    for (int k = 0; k < 3; ++k)
      if (!al(op.coef[k])) return false;
  }
  return true;
}
template <class T>
int tma_launch(int kind, int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs, T *out,
               T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g, float omega,
               unsigned flags, const int *active, double *partials, int *nblk_out,
               cudaStream_t s);
// The coarse end of a V-cycle in one kernel (subcycle.cu): levels l0 .. coarsest of a SIGMA7,
// CONST7 or K27 hierarchy, one block per instance, all fields in shared memory.
constexpr int kMaxSubLevels = 8;
constexpr size_t kSubcycleMaxSmem = 200 * 1024;
template <class T> struct SubLevel {
  int Z, Y, X, n;
  float cz, cy, cx;          // SIGMA7: face multipliers of this level (c_d times its scale)
  float k[27];               // CONST7 (k[0..2] = kz, ky, kx) / K27 weights of this level
  const T *sx, *sy, *sz;     // the level's conductivities, instance stride n
  int o_phi, o_tmp, o_rhs;   // float offsets of the level's fields in shared memory
  int o_face;                // float offset of its face arrays and diagonal (SIGMA7)
};
template <class T> struct SubArgs {
  SubLevel<T> lv[kMaxSubLevels];
  int nlev;
  const T *rhs;  // right-hand side of level l0, instance stride lv[0].n
  T *out;        // its approximate solution
  const int *active;
  float omega, coarse_omega;
  int nu_pre, nu_post, coarse_sweeps;
};
size_t subcycle_smem_bytes(const Grid3 *g, int nlev, bool sigma);
template <class T> int launch_subcycle(int kind, SubArgs<T> a, int B, cudaStream_t s);

// The small end of a V-cycle as one persistent kernel (subcycle.cu): a level l1 that the
// plane-marching TMA kernels do not take, with the fused coarse cycle directly below it.
// Work items (step, instance, z tile) in step order; an item starts once every item of its
// instance's earlier steps is done (per-instance counters, bounded waits).
constexpr int kSmallMaxSteps = 16;
enum { SK_PRE2 = 0, SK_SMOOTH = 1, SK_RESTRICT = 2, SK_SUB = 3 };
template <class T> struct SmallArgs {
  SubArgs<T> sub;            // levels below l1: rhs = the restricted residual, out = the correction
  DevOp op;                  // level l1's operator (coefficients of type T, instance stride n)
  int Z, Y, X;               // level l1
  int64_t n;
  const T *f;                // right-hand side of level l1
  const T *invd;             // level l1's 1 / diagonal (SK_PRE2)
  T *buf[2];                 // level l1's iterate buffers
  int nsteps;
  int kind[kSmallMaxSteps];  // SK_*
  int src[kSmallMaxSteps];   // iterate read (-1: zero)
  int dst[kSmallMaxSteps];   // iterate written
  int corr[kSmallMaxSteps];  // SK_SMOOTH: subtract the prolonged coarse correction
  int dot[kSmallMaxSteps];   // SK_SMOOTH: partial sums of out * f into `partials`
  float om[kSmallMaxSteps];
  int base[kSmallMaxSteps + 1];  // first item of each step
  int need[kSmallMaxSteps];      // items of an instance done before the step may start
  int tiles, zc;             // z tiles of level l1 (zc planes each, even)
  const int *active;
  double *partials;          // [instance][tile]
  int *ticket;               // next work item (zeroed before the launch)
  int *done;                 // items done per instance (zeroed before the launch)
  int wait_budget;
  int *wait_fail;            // the device's wait-failure counters
};
// Blocks the persistent kernel is launched with, for SUB shared memory `smem`.
template <class T> int launch_small(int kind, SmallArgs<T> a, int B, cudaStream_t s);

// The first two Jacobi sweeps from a zero iterate in one pass (SIGMA7, TMA-eligible grids):
// out = J(phi1) with phi1 = omega f * invd, invd = 1 / diag of the level.
// Two Jacobi sweeps of a FACE7 level in one pass (16-bit storage; tma_face2.cuh).
enum { PAIR_SS = 0, PAIR_PR = 1 };
bool face2_eligible(int pair, bool corr, Grid3 g);
template <class T>
int tma_launch_face2(int pair, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                     const T *invd, T *out, T *coarse, int64_t stride, int64_t coarse_stride,
                     int B, Grid3 g, float omega, unsigned flags, const int *active,
                     double *partials, int *nblk_out, cudaStream_t s);
template <class T>
int tma_launch_pre2(int kind, const DevOp &op, const T *f, const T *invd, T *out, int64_t stride,
                    int B, Grid3 g, float omega, const int *active, cudaStream_t s);
// The FACE7 plane-marching kernel takes neither the x-end rule, the top copy nor the p . A p
// sums; launches that need them run the generic kernels.
template <class T>
bool face_tma_ok(int kind, const PhiSrc<T> &phi, unsigned flags) {
  return kind != HFM_OP_FACE7 ||
         (!phi.zero_xend && !(flags & (HFM_FLAG_ZERO_XEND | HFM_FLAG_TOP_COPY | HFM_INT_DOT_PHI)));
}

// 1 / diagonal of a FACE7 level from its faces (faces.cu), the diagonal the face kernels use.
template <class T>
int launch_invdiag_faces(const T *fx, const T *fy, const T *fz, float scale, T *out,
                         int64_t out_stride, int B, Grid3 g, cudaStream_t s);
// FACE7 arrays of the SIGMA7 operator (faces.cu) from conductivities of type TS (instance
// stride s_stride), stored as T; `div` (per-slot divisors, may be null) divides the
// conductivities of instance slot0 + b first.
template <class TS, class T>
int launch_sigma_faces(const TS *sx, const TS *sy, const TS *sz, int64_t s_stride, float cz,
                       float cy, float cx, const double *div, int slot0, T *fx, T *fy, T *fz,
                       int B, Grid3 g, cudaStream_t s);

// Upper bound of blocks per instance of any residual launch on grid g (partials sizing).
int64_t max_partial_blocks(Grid3 g, int B);

// Reductions (reduce.cu)
template <class T>
int launch_sumsq_partials(const T *x, int64_t n, int64_t stride, int B, double *partials,
                          int *nblk_out, const int *active, cudaStream_t s);
int launch_finalize_sum(const double *partials, int nblk, int B, double *out_sum,
                        cudaStream_t s);
int reduce_blocks_for(int64_t n);

template <class T>
int launch_convert(const void *src, int src_dtype, T *dst, int64_t n, cudaStream_t s);
template <class T>
int launch_convert_out(const T *src, float *dst, int64_t n, cudaStream_t s);

}  // namespace hfm
