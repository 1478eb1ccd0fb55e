// Face coefficients of the per-cell conductivity operator in the FACE7 layout.
//
// The SIGMA7 operator's face between cells i and j on axis d is c_d (s_i + s_j) / 2, a wall
// face c_d s_i (Anisotropic Resistivity Tomography/README:14-26, ghost sigma = interior
// sigma).  FACE7 stores every face once, walls included - Fx [Z][Y][X + 8] (element i of a
// row: the face between cells i-1 and i, i = 0 .. X; the rest zero), Fy [Z][Y + 1][X],
// Fz [Z + 1][Y][X] - so a kernel reads the two faces of a cell on each axis and the diagonal
// is their sum.  Each face is formed in float32 from the conductivities as the SIGMA7
// kernels form it (c_d (0.5 (s_i + s_j))) and rounded once to the storage type.
#include "hfm_internal.cuh"

namespace hfm {

namespace {

template <class TS> __device__ __forceinline__ float ldf(const TS *p) { return St<TS>::to(*p); }
template <> __device__ __forceinline__ float ldf<double>(const double *p) { return (float)*p; }

// One thread per face element of the three arrays of instance blockIdx.y (concatenated:
// Fx, then Fy, then Fz).  `div` (per-slot divisors, may be null) divides the conductivities
// of instance slot0 + b before the face is formed (the fp16 cycles' normalisation).
template <class TS, class T>
__global__ void k_sigma_faces(const TS *__restrict__ sx, const TS *__restrict__ sy,
                              const TS *__restrict__ sz, int64_t s_stride, float cz, float cy,
                              float cx, const double *__restrict__ div, int slot0,
                              T *__restrict__ fx, T *__restrict__ fy, T *__restrict__ fz, int Z,
                              int Y, int X) {
  const int64_t b = blockIdx.y;
  const int64_t nx = face7_nx(Z, Y, X), ny = face7_ny(Z, Y, X), nz = face7_nz(Z, Y, X);
  const float inv = div ? (float)(1.0 / div[slot0 + b]) : 1.f;
  const TS *bx = sx + b * s_stride, *by = sy + b * s_stride, *bz = sz + b * s_stride;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nx + ny + nz;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (k < nx) {
      const int i = (int)(k % (X + 8));
      const int64_t row = k / (X + 8);  // z * Y + y
      float v = 0.f;
      if (i <= X) {
        const TS *r = bx + row * X;
        const float a = i > 0 ? ldf(r + i - 1) * inv : 0.f, c = i < X ? ldf(r + i) * inv : 0.f;
        v = i == 0 ? cx * c : (i == X ? cx * a : cx * (0.5f * (a + c)));
      }
      fx[b * nx + k] = St<T>::from(v);
    } else if (k < nx + ny) {
      const int64_t q = k - nx;
      const int x = (int)(q % X);
      const int64_t t = q / X;
      const int j = (int)(t % (Y + 1)), z = (int)(t / (Y + 1));
      const TS *col = by + (int64_t)z * Y * X + x;
      const float a = j > 0 ? ldf(col + (int64_t)(j - 1) * X) * inv : 0.f;
      const float c = j < Y ? ldf(col + (int64_t)j * X) * inv : 0.f;
      const float v = j == 0 ? cy * c : (j == Y ? cy * a : cy * (0.5f * (a + c)));
      fy[b * ny + q] = St<T>::from(v);
    } else {
      const int64_t q = k - nx - ny;
      const int64_t P = (int64_t)Y * X;
      const int64_t yx = q % P;
      const int kz = (int)(q / P);
      const float a = kz > 0 ? ldf(bz + (int64_t)(kz - 1) * P + yx) * inv : 0.f;
      const float c = kz < Z ? ldf(bz + (int64_t)kz * P + yx) * inv : 0.f;
      const float v = kz == 0 ? cz * c : (kz == Z ? cz * a : cz * (0.5f * (a + c)));
      fz[b * nz + q] = St<T>::from(v);
    }
  }
}

// 1 / diagonal of a FACE7 level: the cell's six faces summed in the order the face kernels
// sum them (x left, x right, y below, y above, z below, z above, from zero), times the
// operator's scale when it is not 1, so the fused first two sweeps divide by exactly the
// diagonal the other sweeps use.
template <class T>
__global__ void k_invdiag_faces(const T *__restrict__ fx, const T *__restrict__ fy,
                                const T *__restrict__ fz, float scale, int Z, int Y, int X,
                                T *__restrict__ out, int64_t out_stride) {
  const int64_t b = blockIdx.y;
  const int n = Z * Y * X, P = Y * X;
  fx += b * face7_nx(Z, Y, X);
  fy += b * face7_ny(Z, Y, X);
  fz += b * face7_nz(Z, Y, X);
  out += b * out_stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = i % X, t = i / X, y = t % Y, z = t / Y;
    const int64_t ix = ((int64_t)z * Y + y) * (X + 8) + x, iy = ((int64_t)z * (Y + 1) + y) * X + x;
    float d = __fadd_rn(St<T>::to(fx[ix]), 0.f);
    d = __fadd_rn(St<T>::to(fx[ix + 1]), d);
    d = __fadd_rn(St<T>::to(fy[iy]), d);
    d = __fadd_rn(St<T>::to(fy[iy + X]), d);
    d = __fadd_rn(St<T>::to(fz[i]), d);
    d = __fadd_rn(St<T>::to(fz[(int64_t)i + P]), d);
    if (scale != 1.f) d = __fmul_rn(d, scale);
    out[i] = St<T>::from(1.f / d);
  }
}

}  // namespace

template <class T>
int launch_invdiag_faces(const T *fx, const T *fy, const T *fz, float scale, T *out,
                         int64_t out_stride, int B, Grid3 g, cudaStream_t s) {
  int64_t nb = (g.n() + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 8;
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  k_invdiag_faces<T><<<dim3((unsigned)nb, B), 256, 0, s>>>(fx, fy, fz, scale, g.Z, g.Y, g.X, out,
                                                          out_stride);
  HFM_CHECK_LAUNCH("k_invdiag_faces");
  return HFM_OK;
}
template int launch_invdiag_faces<__nv_bfloat16>(const __nv_bfloat16 *, const __nv_bfloat16 *,
                                                 const __nv_bfloat16 *, float, __nv_bfloat16 *,
                                                 int64_t, int, Grid3, cudaStream_t);
template int launch_invdiag_faces<__half>(const __half *, const __half *, const __half *, float,
                                          __half *, int64_t, int, Grid3, cudaStream_t);

template <class TS, class T>
int launch_sigma_faces(const TS *sx, const TS *sy, const TS *sz, int64_t s_stride, float cz,
                       float cy, float cx, const double *div, int slot0, T *fx, T *fy, T *fz,
                       int B, Grid3 g, cudaStream_t s) {
  const int64_t tot = face7_nx(g.Z, g.Y, g.X) + face7_ny(g.Z, g.Y, g.X) + face7_nz(g.Z, g.Y, g.X);
  int64_t nb = (tot + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 8;
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  k_sigma_faces<TS, T><<<dim3((unsigned)nb, B), 256, 0, s>>>(sx, sy, sz, s_stride, cz, cy, cx, div,
                                                             slot0, fx, fy, fz, g.Z, g.Y, g.X);
  HFM_CHECK_LAUNCH("k_sigma_faces");
  return HFM_OK;
}

#define HFM_FACES_INST(TS, T)                                                                  \
  template int launch_sigma_faces<TS, T>(const TS *, const TS *, const TS *, int64_t, float, \
                                         float, float, const double *, int, T *, T *, T *,   \
                                         int, Grid3, cudaStream_t);
HFM_FACES_INST(float, float)
HFM_FACES_INST(float, __nv_bfloat16)
HFM_FACES_INST(float, __half)
HFM_FACES_INST(double, __nv_bfloat16)
HFM_FACES_INST(double, __half)
HFM_FACES_INST(double, float)
HFM_FACES_INST(__nv_bfloat16, __nv_bfloat16)
HFM_FACES_INST(__half, __half)
#undef HFM_FACES_INST

}  // namespace hfm

using namespace hfm;

extern "C" int hfm_face7_elems(int Z, int Y, int X, int64_t *nfx, int64_t *nfy, int64_t *nfz) {
  if (Z <= 0 || Y <= 0 || X <= 0 || !nfx || !nfy || !nfz)
    return fail(HFM_ERR_BAD_ARG, "hfm_face7_elems: bad argument");
  *nfx = face7_nx(Z, Y, X);
  *nfy = face7_ny(Z, Y, X);
  *nfz = face7_nz(Z, Y, X);
  return HFM_OK;
}

extern "C" int hfm_sigma7_faces(int dtype, const float *sx, const float *sy, const float *sz,
                                float cz, float cy, float cx, void *fx, void *fy, void *fz,
                                int B, int Z, int Y, int X, hfm_stream_t stream) {
  if (!sx || !sy || !sz || !fx || !fy || !fz) return fail(HFM_ERR_BAD_ARG, "hfm_sigma7_faces: NULL argument");
  if (B <= 0 || B > 65535 || Z <= 0 || Y <= 0 || X <= 0)
    return fail(HFM_ERR_BAD_ARG, "hfm_sigma7_faces: bad extents or batch");
  const Grid3 g{Z, Y, X};
  const int64_t n = g.n();
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HFM_F32:
      return launch_sigma_faces<float, float>(sx, sy, sz, n, cz, cy, cx, nullptr, 0, (float *)fx,
                                              (float *)fy, (float *)fz, B, g, s);
    case HFM_BF16:
      return launch_sigma_faces<float, __nv_bfloat16>(sx, sy, sz, n, cz, cy, cx, nullptr, 0,
                                                      (__nv_bfloat16 *)fx, (__nv_bfloat16 *)fy,
                                                      (__nv_bfloat16 *)fz, B, g, s);
    case HFM_F16:
      return launch_sigma_faces<float, __half>(sx, sy, sz, n, cz, cy, cx, nullptr, 0, (__half *)fx,
                                               (__half *)fy, (__half *)fz, B, g, s);
    default:
      return fail(HFM_ERR_BAD_ARG, "hfm_sigma7_faces: dtype must be F32, BF16 or F16");
  }
}
