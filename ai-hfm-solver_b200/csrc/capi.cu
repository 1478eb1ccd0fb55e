// C ABI: library information, error plumbing and the stateless operators.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "hfm_internal.cuh"

namespace hfm {

static thread_local std::string g_last_error;
static thread_local bool g_capturing = false;
static std::atomic<int64_t> g_launches{0};

void note_launch() {
  if (!g_capturing) g_launches.fetch_add(1, std::memory_order_relaxed);
}
void note_graph_launch(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void set_capturing(bool on) { g_capturing = on; }

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int status, const std::string &msg) {
  set_error(msg);
  return status;
}

int cuda_status(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return HFM_ERR_CUDA;
}

int sm_count() {
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
  if (!cache[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cache[dev] = v;
  }
  return cache[dev];
}

int set_max_dynamic_smem(const void *kernel, int bytes, const char *what) {
  static std::mutex mu;
  static std::vector<std::pair<int, const void *>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, what);
  std::lock_guard<std::mutex> lk(mu);
  for (const auto &d : done)
    if (d.first == dev && d.second == kernel) return HFM_OK;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return cuda_status(e, what);
  done.emplace_back(dev, kernel);
  return HFM_OK;
}

DevOp make_devop(const hfm_operator &op, int64_t coef_stride) {
  DevOp d;
  memset(&d, 0, sizeof(d));
  const float s = op.scale == 0.f ? 1.f : op.scale;
  d.scale = s;
  for (int i = 0; i < 3; ++i) d.c[i] = op.c[i];
  if (op.kind == HFM_OP_K27) {
    for (int i = 0; i < 27; ++i) d.k[i] = op.k[i] * s;
  } else if (op.kind == HFM_OP_CONST7) {
    for (int i = 0; i < 3; ++i) d.k[i] = op.k[i] * s;
  }
  for (int i = 0; i < 7; ++i) d.coef[i] = op.coef[i];
  d.coef_stride = coef_stride;
  return d;
}

}  // namespace hfm

using namespace hfm;

namespace {

int check_grid(int B, int Z, int Y, int X) {
  if (B <= 0 || Z <= 0 || Y <= 0 || X <= 0)
    return fail(HFM_ERR_BAD_ARG, "extents and batch must be positive");
  if ((int64_t)Z * Y * X > (int64_t)1 << 34) return fail(HFM_ERR_BAD_ARG, "grid too large");
  if (B > 65535) return fail(HFM_ERR_BAD_ARG, "batch too large (max 65535)");
  return HFM_OK;
}

int check_op(const hfm_operator *op) {
  if (!op) return fail(HFM_ERR_BAD_ARG, "operator is NULL");
  if (op->coef_dtype != HFM_F32)
    return fail(HFM_ERR_BAD_ARG, "stateless calls take float32 coefficient arrays");
  switch (op->kind) {
    case HFM_OP_CONST7:
    case HFM_OP_K27:
      return HFM_OK;
    case HFM_OP_SIGMA7:
      for (int i = 0; i < 3; ++i)
        if (!op->coef[i]) return fail(HFM_ERR_BAD_ARG, "SIGMA7 needs sx, sy, sz");
      return HFM_OK;
    case HFM_OP_DIR7:
      for (int i = 0; i < 7; ++i)
        if (!op->coef[i]) return fail(HFM_ERR_BAD_ARG, "DIR7 needs seven coefficient arrays");
      return HFM_OK;
    case HFM_OP_FACE7:
      for (int i = 0; i < 3; ++i)
        if (!op->coef[i]) return fail(HFM_ERR_BAD_ARG, "FACE7 needs Fx, Fy, Fz");
      return HFM_OK;
    default:
      return fail(HFM_ERR_BAD_ARG, "unknown operator kind");
  }
}

// Operator of a typed (storage-dtype) call: the coefficient arrays are stored as dtype.
int check_op_typed(const hfm_operator *op, int dtype, const char *who) {
  if (!op) return fail(HFM_ERR_BAD_ARG, std::string(who) + ": operator is NULL");
  if (dtype != HFM_F32 && dtype != HFM_BF16 && dtype != HFM_F16)
    return fail(HFM_ERR_BAD_ARG, std::string(who) + ": dtype must be F32, BF16 or F16");
  int na = 0;
  switch (op->kind) {
    case HFM_OP_SIGMA7: case HFM_OP_FACE7: na = 3; break;
    case HFM_OP_DIR7: na = 7; break;
    case HFM_OP_CONST7: case HFM_OP_K27: na = 0; break;
    default: return fail(HFM_ERR_BAD_ARG, "unknown operator kind");
  }
  if (na && op->coef_dtype != dtype)
    return fail(HFM_ERR_BAD_ARG, std::string(who) + ": coef_dtype must equal dtype");
  for (int i = 0; i < na; ++i)
    if (!op->coef[i]) return fail(HFM_ERR_BAD_ARG, std::string(who) + ": missing coefficient array");
  return HFM_OK;
}

template <class T> PhiSrc<T> typed_src(const void *phi, int64_t n, unsigned flags) {
  PhiSrc<T> p;
  memset(&p, 0, sizeof(p));
  p.base = (flags & HFM_FLAG_ZERO_GUESS) ? nullptr : (const T *)phi;
  p.base_stride = n;
  p.zero_xend = (flags & HFM_FLAG_ZERO_XEND) ? 1 : 0;
  return p;
}

#define HFM_BY_DTYPE(dtype, BODY)                                  \
  switch (dtype) {                                                 \
    case HFM_F32: { using T = float; BODY; }                       \
    case HFM_BF16: { using T = __nv_bfloat16; BODY; }              \
    default: { using T = __half; BODY; }                           \
  }

PhiSrc<float> plain_src(const float *phi, int64_t stride, unsigned flags) {
  PhiSrc<float> p;
  memset(&p, 0, sizeof(p));
  p.base = (flags & HFM_FLAG_ZERO_GUESS) ? nullptr : phi;
  p.base_stride = stride;
  p.zero_xend = (flags & HFM_FLAG_ZERO_XEND) ? 1 : 0;
  return p;
}

hfm_operator k27_op(const float *w27) {
  hfm_operator op;
  memset(&op, 0, sizeof(op));
  op.kind = HFM_OP_K27;
  op.coef_dtype = HFM_F32;
  op.scale = 1.f;
  for (int i = 0; i < 27; ++i) op.k[i] = w27[i];
  return op;
}

hfm_operator const7_op(float kz, float ky, float kx) {
  hfm_operator op;
  memset(&op, 0, sizeof(op));
  op.kind = HFM_OP_CONST7;
  op.coef_dtype = HFM_F32;
  op.scale = 1.f;
  op.k[0] = kz;
  op.k[1] = ky;
  op.k[2] = kx;
  return op;
}

hfm_operator sigma7_op(const float *sx, const float *sy, const float *sz, float cz, float cy,
                       float cx) {
  hfm_operator op;
  memset(&op, 0, sizeof(op));
  op.kind = HFM_OP_SIGMA7;
  op.coef_dtype = HFM_F32;
  op.scale = 1.f;
  op.coef[0] = sx;
  op.coef[1] = sy;
  op.coef[2] = sz;
  op.c[0] = cz;
  op.c[1] = cy;
  op.c[2] = cx;
  return op;
}

}  // namespace

extern "C" {

int hfm_abi_version(void) { return HFM_ABI_VERSION; }

const char *hfm_status_string(int status) {
  switch (status) {
    case HFM_OK: return "HFM_OK";
    case HFM_ERR_BAD_ARG: return "HFM_ERR_BAD_ARG";
    case HFM_ERR_OOM: return "HFM_ERR_OOM";
    case HFM_ERR_NOT_CONVERGED: return "HFM_ERR_NOT_CONVERGED";
    case HFM_ERR_NAN: return "HFM_ERR_NAN";
    case HFM_ERR_TIMEOUT: return "HFM_ERR_TIMEOUT";
    case HFM_ERR_CUDA: return "HFM_ERR_CUDA";
    case HFM_ERR_UNSUPPORTED: return "HFM_ERR_UNSUPPORTED";
    case HFM_ERR_CANCELLED: return "HFM_ERR_CANCELLED";
    default: return "HFM_ERR_UNKNOWN";
  }
}

const char *hfm_last_error(void) { return g_last_error.c_str(); }

int64_t hfm_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int hfm_device_sm_count(int *out) {
  if (!out) return fail(HFM_ERR_BAD_ARG, "NULL");
  *out = sm_count();
  return HFM_OK;
}

int hfm_op_apply(const hfm_operator *op, const float *phi, float *out, int B, int Z, int Y,
                 int X, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X)) || (st = check_op(op))) return st;
  if (!phi || !out) return fail(HFM_ERR_BAD_ARG, "hfm_op_apply: NULL field");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  return launch_apply<float>(op->kind, d, plain_src(phi, n, 0), out, n, B, Grid3{Z, Y, X},
                             nullptr, (cudaStream_t)stream);
}

int hfm_op_residual(const hfm_operator *op, const float *phi, const float *b, float *r, int B,
                    int Z, int Y, int X, unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X)) || (st = check_op(op))) return st;
  if (!phi || !b || !r) return fail(HFM_ERR_BAD_ARG, "hfm_op_residual: NULL field");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  return launch_residual<float>(op->kind, d, plain_src(phi, n, flags & HFM_FLAG_ZERO_GUESS), b,
                                n, r, n, B, Grid3{Z, Y, X}, flags, nullptr, nullptr, nullptr,
                                (cudaStream_t)stream);
}

int hfm_op_jacobi(const hfm_operator *op, const float *phi, const float *rhs, float *out,
                  float *tmp, int B, int Z, int Y, int X, float omega, int sweeps,
                  unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X)) || (st = check_op(op))) return st;
  if (!rhs || !out || (!phi && !(flags & HFM_FLAG_ZERO_GUESS)))
    return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi: NULL field");
  if (sweeps < 1) return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi: sweeps must be >= 1");
  if (sweeps > 1 && !tmp) return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi: sweeps > 1 needs tmp");
  if (phi == out || (tmp && phi == tmp)) return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi: phi aliases out/tmp");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  const float *src = phi;
  for (int s = 0; s < sweeps; ++s) {
    float *dst = ((sweeps - s) % 2 == 1) ? out : tmp;
    unsigned f = (s == 0) ? flags : (flags & ~HFM_FLAG_ZERO_GUESS);
    st = launch_smooth<float>(op->kind, d, plain_src(src, n, f), rhs, n, dst, n, B,
                              Grid3{Z, Y, X}, omega, f, nullptr, (cudaStream_t)stream);
    if (st) return st;
    src = dst;
  }
  return HFM_OK;
}

int hfm_op_jacobi_typed(const hfm_operator *op, int dtype, const void *phi, const void *rhs,
                        void *out, int B, int Z, int Y, int X, float omega, unsigned flags,
                        hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!op || !rhs || !out || (!phi && !(flags & HFM_FLAG_ZERO_GUESS)))
    return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi_typed: NULL argument");
  if ((st = check_op_typed(op, dtype, "hfm_op_jacobi_typed"))) return st;
  if (phi == out) return fail(HFM_ERR_BAD_ARG, "hfm_op_jacobi_typed: phi aliases out");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  HFM_BY_DTYPE(dtype, return launch_smooth<T>(op->kind, d, typed_src<T>(phi, n, flags),
                                              (const T *)rhs, n, (T *)out, n, B, Grid3{Z, Y, X},
                                              omega, flags, nullptr, (cudaStream_t)stream))
}

int hfm_op_residual_typed(const hfm_operator *op, int dtype, const void *phi, const void *b,
                          void *r, int B, int Z, int Y, int X, unsigned flags,
                          hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!phi || !b || !r) return fail(HFM_ERR_BAD_ARG, "hfm_op_residual_typed: NULL field");
  if ((st = check_op_typed(op, dtype, "hfm_op_residual_typed"))) return st;
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  HFM_BY_DTYPE(dtype, return launch_residual<T>(op->kind, d, typed_src<T>(phi, n, flags), (const T *)b,
                                                n, (T *)r, n, B, Grid3{Z, Y, X}, flags, nullptr,
                                                nullptr, nullptr, (cudaStream_t)stream))
}

int hfm_residual_restrict_typed(const hfm_operator *op, int dtype, const void *phi,
                                const void *b, void *r_fine, void *r_coarse, int B, int Z,
                                int Y, int X, unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!phi || !b || !r_coarse) return fail(HFM_ERR_BAD_ARG, "hfm_residual_restrict_typed: NULL field");
  if ((st = check_op_typed(op, dtype, "hfm_residual_restrict_typed"))) return st;
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  HFM_BY_DTYPE(dtype, return launch_residual_restrict<T>(
                          op->kind, d, typed_src<T>(phi, n, flags & HFM_FLAG_ZERO_GUESS),
                          (const T *)b, n, (T *)r_fine, n, (T *)r_coarse, n / 8, B,
                          Grid3{Z, Y, X}, flags, nullptr, nullptr, nullptr, (cudaStream_t)stream))
}

int hfm_prolong_correct_smooth_typed(const hfm_operator *op, int dtype, const void *phi,
                                     const void *w_coarse, const void *rhs, void *out, int B,
                                     int Z, int Y, int X, float omega, unsigned flags,
                                     hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!w_coarse || !rhs || !out) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth_typed: NULL field");
  if ((Z | Y | X) & 1) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth_typed: fine extents must be even");
  if (phi == out) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth_typed: phi aliases out");
  if ((st = check_op_typed(op, dtype, "hfm_prolong_correct_smooth_typed"))) return st;
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  HFM_BY_DTYPE(dtype, {
    PhiSrc<T> p = typed_src<T>(phi, n, flags);
    p.corr = (const T *)w_coarse;
    p.corr_stride = n / 8;
    p.corr_coarse = 1;
    p.corr_sign = phi ? -1.f : 1.f;
    p.Yc = Y / 2;
    p.Xc = X / 2;
    return launch_smooth<T>(op->kind, d, p, (const T *)rhs, n, (T *)out, n, B, Grid3{Z, Y, X},
                            omega, flags, nullptr, (cudaStream_t)stream);
  })
}

int hfm_face7_smooth2_typed(const hfm_operator *op, int dtype, const void *phi,
                            const void *w_coarse, const void *rhs, void *out, int B, int Z,
                            int Y, int X, float omega, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!phi || !rhs || !out) return fail(HFM_ERR_BAD_ARG, "hfm_face7_smooth2_typed: NULL field");
  if (phi == out) return fail(HFM_ERR_BAD_ARG, "hfm_face7_smooth2_typed: phi aliases out");
  if ((st = check_op_typed(op, dtype, "hfm_face7_smooth2_typed"))) return st;
  if (op->kind != HFM_OP_FACE7 || dtype == HFM_F32)
    return fail(HFM_ERR_UNSUPPORTED, "hfm_face7_smooth2_typed: FACE7 in 16-bit storage only");
  if (!face2_eligible(PAIR_SS, w_coarse != nullptr, Grid3{Z, Y, X}))
    return fail(HFM_ERR_UNSUPPORTED, "hfm_face7_smooth2_typed: X >= 48 and a multiple of 8 "
                                     "(16 with w_coarse), Y >= 16, Z >= 2, even with w_coarse");
  for (const void *q : {phi, w_coarse, rhs, (const void *)out, op->coef[0], op->coef[1], op->coef[2]})
    if ((uintptr_t)q & 15) return fail(HFM_ERR_BAD_ARG, "hfm_face7_smooth2_typed: fields must be 16-byte aligned");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  HFM_BY_DTYPE(dtype, {
    PhiSrc<T> p;
    memset(&p, 0, sizeof(p));
    p.base = (const T *)phi;
    p.base_stride = n;
    if (w_coarse) {
      p.corr = (const T *)w_coarse;
      p.corr_stride = n / 8;
      p.corr_coarse = 1;
      p.corr_sign = -1.f;
      p.Yc = Y / 2;
      p.Xc = X / 2;
    }
    return tma_launch_face2<T>(PAIR_SS, d, p, (const T *)rhs, nullptr, (T *)out, nullptr, n, 0, B,
                               Grid3{Z, Y, X}, omega, 0u, nullptr, nullptr, nullptr,
                               (cudaStream_t)stream);
  })
}

int hfm_residual_restrict(const hfm_operator *op, const float *phi, const float *b,
                          float *r_fine, float *r_coarse, int B, int Z, int Y, int X,
                          unsigned flags, hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X)) || (st = check_op(op))) return st;
  if (!phi || !b || !r_coarse) return fail(HFM_ERR_BAD_ARG, "hfm_residual_restrict: NULL field");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  return launch_residual_restrict<float>(op->kind, d, plain_src(phi, n, flags & HFM_FLAG_ZERO_GUESS), b, n, r_fine, n,
                                         r_coarse, n / 8, B, Grid3{Z, Y, X}, flags, nullptr,
                                         nullptr, nullptr, (cudaStream_t)stream);
}

int hfm_prolong_correct_smooth(const hfm_operator *op, const float *phi,
                               const float *w_coarse, const float *rhs, float *out, int B,
                               int Z, int Y, int X, float omega, unsigned flags,
                               hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X)) || (st = check_op(op))) return st;
  if (!w_coarse || !rhs || !out) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth: NULL field");
  if ((Z | Y | X) & 1) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth: fine extents must be even");
  if (phi == out) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_correct_smooth: phi aliases out");
  const int64_t n = (int64_t)Z * Y * X;
  DevOp d = make_devop(*op, n);
  PhiSrc<float> p = plain_src(phi, n, flags);
  p.corr = w_coarse;
  p.corr_stride = n / 8;
  p.corr_coarse = 1;
  p.corr_sign = phi ? -1.f : 1.f;  // phi - P w, or P w alone (sawtooth coarse levels)
  p.Yc = Y / 2;
  p.Xc = X / 2;
  return launch_smooth<float>(op->kind, d, p, rhs, n, out, n, B, Grid3{Z, Y, X}, omega, flags,
                              nullptr, (cudaStream_t)stream);
}

int hfm_conv3d_k3(const float *x, float *y, int B, int Z, int Y, int X, const float *w27,
                  hfm_stream_t stream) {
  if (!w27) return fail(HFM_ERR_BAD_ARG, "hfm_conv3d_k3: NULL weights");
  hfm_operator op = k27_op(w27);
  return hfm_op_apply(&op, x, y, B, Z, Y, X, stream);
}

int hfm_restrict_avg(const float *fine, float *coarse, int B, int Z, int Y, int X,
                     hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Z, Y, X))) return st;
  if (!fine || !coarse) return fail(HFM_ERR_BAD_ARG, "hfm_restrict_avg: NULL field");
  if (Z < 2 || Y < 2 || X < 2) return fail(HFM_ERR_BAD_ARG, "hfm_restrict_avg: extent < 2");
  const int64_t n = (int64_t)Z * Y * X, nc = (int64_t)(Z / 2) * (Y / 2) * (X / 2);
  return launch_restrict<float>(fine, n, coarse, nc, B, Grid3{Z, Y, X}, nullptr,
                                (cudaStream_t)stream);
}

int hfm_prolong_nearest(const float *coarse, float *fine, int B, int Zc, int Yc, int Xc,
                        hfm_stream_t stream) {
  int st;
  if ((st = check_grid(B, Zc, Yc, Xc))) return st;
  if (!fine || !coarse) return fail(HFM_ERR_BAD_ARG, "hfm_prolong_nearest: NULL field");
  const int64_t nc = (int64_t)Zc * Yc * Xc;
  return launch_prolong<float>(coarse, nc, fine, nc * 8, B, Grid3{Zc, Yc, Xc}, nullptr,
                               (cudaStream_t)stream);
}

int hfm_stencil7_const_apply(const float *phi, float *out, int B, int Z, int Y, int X,
                             float kz, float ky, float kx, hfm_stream_t stream) {
  hfm_operator op = const7_op(kz, ky, kx);
  return hfm_op_apply(&op, phi, out, B, Z, Y, X, stream);
}
int hfm_stencil7_const_residual(const float *phi, const float *b, float *r, int B, int Z,
                                int Y, int X, float kz, float ky, float kx, unsigned flags,
                                hfm_stream_t stream) {
  hfm_operator op = const7_op(kz, ky, kx);
  return hfm_op_residual(&op, phi, b, r, B, Z, Y, X, flags, stream);
}
int hfm_stencil7_const_jacobi(const float *phi, const float *rhs, float *out, float *tmp,
                              int B, int Z, int Y, int X, float kz, float ky, float kx,
                              float omega, int sweeps, unsigned flags, hfm_stream_t stream) {
  hfm_operator op = const7_op(kz, ky, kx);
  return hfm_op_jacobi(&op, phi, rhs, out, tmp, B, Z, Y, X, omega, sweeps, flags, stream);
}
int hfm_stencil7_var_apply(const float *phi, float *out, const float *sx, const float *sy,
                           const float *sz, int B, int Z, int Y, int X, float cz, float cy,
                           float cx, hfm_stream_t stream) {
  hfm_operator op = sigma7_op(sx, sy, sz, cz, cy, cx);
  return hfm_op_apply(&op, phi, out, B, Z, Y, X, stream);
}
int hfm_stencil7_var_residual(const float *phi, const float *b, float *r, const float *sx,
                              const float *sy, const float *sz, int B, int Z, int Y, int X,
                              float cz, float cy, float cx, unsigned flags,
                              hfm_stream_t stream) {
  hfm_operator op = sigma7_op(sx, sy, sz, cz, cy, cx);
  return hfm_op_residual(&op, phi, b, r, B, Z, Y, X, flags, stream);
}
int hfm_stencil7_var_jacobi(const float *phi, const float *rhs, float *out, float *tmp,
                            const float *sx, const float *sy, const float *sz, int B, int Z,
                            int Y, int X, float cz, float cy, float cx, float omega,
                            int sweeps, unsigned flags, hfm_stream_t stream) {
  hfm_operator op = sigma7_op(sx, sy, sz, cz, cy, cx);
  return hfm_op_jacobi(&op, phi, rhs, out, tmp, B, Z, Y, X, omega, sweeps, flags, stream);
}
int hfm_stencil27_apply(const float *phi, float *out, int B, int Z, int Y, int X,
                        const float *w27, hfm_stream_t stream) {
  return hfm_conv3d_k3(phi, out, B, Z, Y, X, w27, stream);
}
int hfm_stencil27_residual(const float *phi, const float *b, float *r, int B, int Z, int Y,
                           int X, const float *w27, unsigned flags, hfm_stream_t stream) {
  if (!w27) return fail(HFM_ERR_BAD_ARG, "NULL weights");
  hfm_operator op = k27_op(w27);
  return hfm_op_residual(&op, phi, b, r, B, Z, Y, X, flags, stream);
}
int hfm_stencil27_jacobi(const float *phi, const float *rhs, float *out, float *tmp, int B,
                         int Z, int Y, int X, const float *w27, float omega, int sweeps,
                         unsigned flags, hfm_stream_t stream) {
  if (!w27) return fail(HFM_ERR_BAD_ARG, "NULL weights");
  hfm_operator op = k27_op(w27);
  return hfm_op_jacobi(&op, phi, rhs, out, tmp, B, Z, Y, X, omega, sweeps, flags, stream);
}

}  // extern "C"
