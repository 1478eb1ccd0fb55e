// Operators of the NS time stepper: fused two-stage momentum
// update, pressure-gradient correction, divergence right-hand side with the source boundary
// rule, sigma-mask immersed body, and the velocity / pressure boundary rules.
//
// Every 3x3x3 kernel (diffusion w1, smoothed central differences w2-w4, divergence w6-w8) is
// passed by value as 27 weights (dz, dy, dx) and applied as a cross-correlation with zero
// padding, exactly like the reference's frozen Conv3D layers (naiver_stokes_3D.py:166-236).
#include <cstring>

#include "hfm_internal.cuh"

namespace hfm {
namespace {

struct K4 {
  float k[4][27];  // diffusion, x, y, z kernels
};
struct K3 {
  float k[3][27];
};

__device__ __forceinline__ float at(const float *f, int z, int y, int x, int Z, int Y, int X) {
  if (z < 0 || z >= Z || y < 0 || y >= Y || x < 0 || x >= X) return 0.f;
  return __ldg(f + ((int64_t)z * Y + y) * X + x);
}

// out_f = base_f + coef * (Dif(a_f) - a_u Dx(a_f) - a_v Dy(a_f) - a_w Dz(a_f)), f in {u, v, w}
// (naiver_stokes_3D.py:580-622: stage 1 with a = base = u^n, coef 1/2; stage 2 with a = b,
// base = u^n, coef 1).  With ex / ey / ez (and a zero diffusion kernel) the diffusion term is
// the given field instead: the Petrov-Galerkin form of INHALE_demo.ipynb cell 24.
__global__ void __launch_bounds__(256)
    k_momentum(const float *__restrict__ au, const float *__restrict__ av,
               const float *__restrict__ aw, const float *__restrict__ bu,
               const float *__restrict__ bv, const float *__restrict__ bw, float *__restrict__ ou,
               float *__restrict__ ov, float *__restrict__ ow, int Z, int Y, int X, K4 K,
               float coef, const float *__restrict__ ex, const float *__restrict__ ey,
               const float *__restrict__ ez) {
  const int64_t n = (int64_t)Z * Y * X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    const float uc = __ldg(au + i), vc = __ldg(av + i), wc = __ldg(aw + i);
    const float *fs[3] = {au, av, aw};
    const float *bs[3] = {bu, bv, bw};
    float *os[3] = {ou, ov, ow};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int j = 9 * a + 3 * b + c;
            const float v = at(fs[f], z + a - 1, y + b - 1, x + c - 1, Z, Y, X);
#pragma unroll
            for (int q = 0; q < 4; ++q) d[q] += K.k[q][j] * v;
          }
      const float *es[3] = {ex, ey, ez};
      const float d0 = es[f] ? __ldg(es[f] + i) : d[0];
      const float acc = ((d0 - uc * d[1]) - vc * d[2]) - wc * d[3];
      os[f][i] = coef * acc + __ldg(bs[f] + i);
    }
  }
}

// Petrov-Galerkin dissipation (INHALE_demo.ipynb cell 20), on the velocities damped by the
// immersed body, u_d = u / (1 + dt sigma).  Pass 1, per component f:
//   k_f = min(2 |(|u_d| + |v_d| + |w_d|) / 3 * Dif(f_d)| /
//             (eps + (|Dx f_d| + |Dy f_d| + |Dz f_d|) / 3), 0.5) / (1 + dt sigma)
__device__ __forceinline__ float damped(const float *f, const float *sg, float dt, int z, int y,
                                        int x, int Z, int Y, int X) {
  if (z < 0 || z >= Z || y < 0 || y >= Y || x < 0 || x >= X) return 0.f;
  const int64_t i = ((int64_t)z * Y + y) * X + x;
  return __ldg(f + i) / (1.f + dt * __ldg(sg + i));
}

__global__ void __launch_bounds__(256)
    k_pg_coef(const float *__restrict__ u, const float *__restrict__ v, const float *__restrict__ w,
              const float *__restrict__ sg, float *__restrict__ ku, float *__restrict__ kv,
              float *__restrict__ kw, int Z, int Y, int X, K4 K, float dt, float eps) {
  const int64_t n = (int64_t)Z * Y * X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    const float den = 1.f + dt * __ldg(sg + i);
    const float speed = (fabsf(__ldg(u + i) / den) + fabsf(__ldg(v + i) / den)) + fabsf(__ldg(w + i) / den);
    const float *fs[3] = {u, v, w};
    float *ks[3] = {ku, kv, kw};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int j = 9 * a + 3 * b + c;
            const float val = damped(fs[f], sg, dt, z + a - 1, y + b - 1, x + c - 1, Z, Y, X);
#pragma unroll
            for (int q = 0; q < 4; ++q) d[q] += K.k[q][j] * val;
          }
      const float num = 2.f * fabsf(speed / 3.f * d[0]);
      const float k = num / (eps + ((fabsf(d[1]) + fabsf(d[2])) + fabsf(d[3])) / 3.f);
      ks[f][i] = fminf(k, 0.5f) / den;
    }
  }
}

// Pass 2: out_f = 1.5 (k_f Dif(f_d) + Dif(f_d k_f) - f_d Dif(k_f)).
__global__ void __launch_bounds__(256)
    k_pg_flux(const float *__restrict__ u, const float *__restrict__ v, const float *__restrict__ w,
              const float *__restrict__ sg, const float *__restrict__ ku,
              const float *__restrict__ kv, const float *__restrict__ kw, float *__restrict__ ox,
              float *__restrict__ oy, float *__restrict__ oz, int Z, int Y, int X, K4 K,
              float dt) {
  const int64_t n = (int64_t)Z * Y * X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    const float *fs[3] = {u, v, w};
    const float *ks[3] = {ku, kv, kw};
    float *os[3] = {ox, oy, oz};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float df = 0.f, dfk = 0.f, dk = 0.f;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float wgt = K.k[0][9 * a + 3 * b + c];
            const int zz = z + a - 1, yy = y + b - 1, xx = x + c - 1;
            const float fv = damped(fs[f], sg, dt, zz, yy, xx, Z, Y, X);
            const float kv_ = at(ks[f], zz, yy, xx, Z, Y, X);
            df += wgt * fv;
            dfk += wgt * (fv * kv_);
            dk += wgt * kv_;
          }
      const float fc = __ldg(fs[f] + i) / (1.f + dt * __ldg(sg + i));
      os[f][i] = 1.5f * ((__ldg(ks[f] + i) * df + dfk) - fc * dk);
    }
  }
}

// u -= conv(p, Kx), v -= conv(p, Ky), w -= conv(p, Kz)  (naiver_stokes_3D.py:631-633)
__global__ void __launch_bounds__(256)
    k_pgrad(const float *__restrict__ p, float *__restrict__ u, float *__restrict__ v,
            float *__restrict__ w, int Z, int Y, int X, K3 K) {
  const int64_t n = (int64_t)Z * Y * X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    float d[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 27; ++j) {
      const float pv = at(p, z + j / 9 - 1, y + (j / 3) % 3 - 1, x + j % 3 - 1, Z, Y, X);
#pragma unroll
      for (int q = 0; q < 3; ++q) d[q] += K.k[q][j] * pv;
    }
    u[i] -= d[0];
    v[i] -= d[1];
    w[i] -= d[2];
  }
}

// b = -(Su(u) + Sv(v) + Sw(w)); with bc_source the plane x = 0 takes the value of x = 1
// (boundary_condition_source, naiver_stokes_3D.py:467-473), computed in place.
__global__ void __launch_bounds__(256)
    k_divergence(const float *__restrict__ u, const float *__restrict__ v,
                 const float *__restrict__ w, float *__restrict__ b, int Z, int Y, int X, K3 K,
                 int bc_source) {
  const int64_t n = (int64_t)Z * Y * X;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    if (bc_source && x == 0 && X > 1) x = 1;
    float s = 0.f;
    const float *fs[3] = {u, v, w};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float d = 0.f;
#pragma unroll
      for (int j = 0; j < 27; ++j)
        d += K.k[q][j] * at(fs[q], z + j / 9 - 1, y + (j / 3) % 3 - 1, x + j % 3 - 1, Z, Y, X);
      s += d;
    }
    b[i] = -s;
  }
}

__global__ void k_ibm(float *__restrict__ u, float *__restrict__ v, float *__restrict__ w,
                      const float *__restrict__ sigma, int64_t n, float dt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float d = 1.f + dt * __ldg(sigma + i);
    u[i] = u[i] / d;
    v[i] = v[i] / d;
    w[i] = w[i] / d;
  }
}

// Boundary shell enumeration: planes z = 0, Z-1 (2XY cells), then y = 0, Y-1 for interior z
// (2(Z-2)X), then x = 0, X-1 for interior z, y (2(Z-2)(Y-2)).
__device__ __forceinline__ void shell_cell(int64_t k, int Z, int Y, int X, int &z, int &y, int &x) {
  const int64_t A = 2LL * Y * X, Bn = 2LL * (Z - 2) * X;
  if (k < A) {
    z = k < (int64_t)Y * X ? 0 : Z - 1;
    const int64_t r = k % ((int64_t)Y * X);
    y = (int)(r / X);
    x = (int)(r % X);
  } else if (k < A + Bn) {
    const int64_t r = k - A;
    const int64_t half = (int64_t)(Z - 2) * X;
    y = r < half ? 0 : Y - 1;
    const int64_t q = r % half;
    z = 1 + (int)(q / X);
    x = (int)(q % X);
  } else {
    const int64_t r = k - A - Bn;
    const int64_t half = (int64_t)(Z - 2) * (Y - 2);
    x = r < half ? 0 : X - 1;
    const int64_t q = r % half;
    z = 1 + (int)(q / (Y - 2));
    y = 1 + (int)(q % (Y - 2));
  }
}

// Final boundary values of boundary_condition_velocity / _pressure (later assignments win:
// z planes over y planes over x planes; copies read the input arrays), gathered into scratch
// before any is written.
__global__ void k_bc_gather(const float *__restrict__ u, const float *__restrict__ v,
                            const float *__restrict__ w, float *__restrict__ scratch, int64_t S,
                            int Z, int Y, int X, float ub, int pressure) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < S;
       k += (int64_t)gridDim.x * blockDim.x) {
    int z, y, x;
    shell_cell(k, Z, Y, X, z, y, x);
    auto I = [&](int zz, int yy, int xx) { return ((int64_t)zz * Y + yy) * X + xx; };
    if (pressure) {
      float p;
      if (z == Z - 1) p = u[I(Z - 2, y, x)];
      else if (z == 0) p = u[I(1, y, x)];
      else if (y == Y - 1) p = u[I(z, Y - 2, x)];
      else if (y == 0) p = u[I(z, 1, x)];
      else if (x == 0) p = u[I(z, y, 1)];
      else p = 0.f;  // x = X-1 (outflow)
      scratch[k] = p;
    } else {
      float fu, fv;
      if (z == Z - 1) {
        fu = u[I(Z - 2, y, x)];
        fv = v[I(Z - 2, y, x)];
      } else if (z == 0) {
        fu = fv = 0.f;
      } else if (y == Y - 1) {
        fu = u[I(z, Y - 2, x)];
        fv = 0.f;
      } else if (y == 0) {
        fu = u[I(z, 1, x)];
        fv = 0.f;
      } else {  // x = 0 (inflow) or x = X-1
        fu = ub;
        fv = 0.f;
      }
      scratch[k] = fu;
      scratch[S + k] = fv;
      scratch[2 * S + k] = 0.f;  // w = 0 on every boundary plane
    }
  }
}

__global__ void k_bc_scatter(float *__restrict__ u, float *__restrict__ v, float *__restrict__ w,
                             const float *__restrict__ scratch, int64_t S, int Z, int Y, int X,
                             int pressure) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < S;
       k += (int64_t)gridDim.x * blockDim.x) {
    int z, y, x;
    shell_cell(k, Z, Y, X, z, y, x);
    const int64_t i = ((int64_t)z * Y + y) * X + x;
    u[i] = scratch[k];
    if (!pressure) {
      v[i] = scratch[S + k];
      w[i] = scratch[2 * S + k];
    }
  }
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 8;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

int64_t shell_size(int Z, int Y, int X) {
  return 2LL * Y * X + 2LL * (Z - 2) * X + 2LL * (Z - 2) * (Y - 2);
}

int check_ns(int Z, int Y, int X) {
  if (Z < 3 || Y < 3 || X < 3) return fail(HFM_ERR_BAD_ARG, "NS operators need extents >= 3");
  return HFM_OK;
}

}  // namespace
}  // namespace hfm

using namespace hfm;

extern "C" {

size_t hfm_ns_bc_scratch_bytes(int Z, int Y, int X) {
  if (Z < 3 || Y < 3 || X < 3) return 0;
  return (size_t)shell_size(Z, Y, X) * 3 * sizeof(float);
}

int hfm_ns_bc_velocity(float *u, float *v, float *w, int Z, int Y, int X, float ub,
                       void *scratch, hfm_stream_t stream) {
  int st;
  if ((st = check_ns(Z, Y, X))) return st;
  if (!u || !v || !w || !scratch) return fail(HFM_ERR_BAD_ARG, "hfm_ns_bc_velocity: NULL");
  const int64_t S = shell_size(Z, Y, X);
  cudaStream_t s = (cudaStream_t)stream;
  k_bc_gather<<<grid_for(S), 256, 0, s>>>(u, v, w, (float *)scratch, S, Z, Y, X, ub, 0);
  HFM_CHECK_LAUNCH("k_bc_gather");
  k_bc_scatter<<<grid_for(S), 256, 0, s>>>(u, v, w, (const float *)scratch, S, Z, Y, X, 0);
  HFM_CHECK_LAUNCH("k_bc_scatter");
  return HFM_OK;
}

int hfm_ns_bc_pressure(float *p, int Z, int Y, int X, void *scratch, hfm_stream_t stream) {
  int st;
  if ((st = check_ns(Z, Y, X))) return st;
  if (!p || !scratch) return fail(HFM_ERR_BAD_ARG, "hfm_ns_bc_pressure: NULL");
  const int64_t S = shell_size(Z, Y, X);
  cudaStream_t s = (cudaStream_t)stream;
  k_bc_gather<<<grid_for(S), 256, 0, s>>>(p, p, p, (float *)scratch, S, Z, Y, X, 0.f, 1);
  HFM_CHECK_LAUNCH("k_bc_gather");
  k_bc_scatter<<<grid_for(S), 256, 0, s>>>(p, p, p, (const float *)scratch, S, Z, Y, X, 1);
  HFM_CHECK_LAUNCH("k_bc_scatter");
  return HFM_OK;
}

int hfm_ns_momentum(const float *adv_u, const float *adv_v, const float *adv_w,
                    const float *base_u, const float *base_v, const float *base_w, float *out_u,
                    float *out_v, float *out_w, int Z, int Y, int X, const float *w_dif,
                    const float *w_dx, const float *w_dy, const float *w_dz, float coef,
                    hfm_stream_t stream) {
  int st;
  if ((st = check_ns(Z, Y, X))) return st;
  if (!adv_u || !adv_v || !adv_w || !base_u || !base_v || !base_w || !out_u || !out_v || !out_w ||
      !w_dif || !w_dx || !w_dy || !w_dz)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_momentum: NULL");
  if (out_u == adv_u || out_v == adv_v || out_w == adv_w || out_u == adv_v || out_u == adv_w ||
      out_v == adv_u || out_v == adv_w || out_w == adv_u || out_w == adv_v)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_momentum: outputs must not alias the advected fields");
  K4 K;
  memcpy(K.k[0], w_dif, 27 * 4);
  memcpy(K.k[1], w_dx, 27 * 4);
  memcpy(K.k[2], w_dy, 27 * 4);
  memcpy(K.k[3], w_dz, 27 * 4);
  const int64_t n = (int64_t)Z * Y * X;
  k_momentum<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(adv_u, adv_v, adv_w, base_u, base_v,
                                                             base_w, out_u, out_v, out_w, Z, Y, X,
                                                             K, coef, nullptr, nullptr, nullptr);
  HFM_CHECK_LAUNCH("k_momentum");
  return HFM_OK;
}

int hfm_ns_momentum_pg(const float *adv_u, const float *adv_v, const float *adv_w,
                       const float *base_u, const float *base_v, const float *base_w,
                       float *out_u, float *out_v, float *out_w, const float *k_x,
                       const float *k_y, const float *k_z, int Z, int Y, int X, const float *w_dx,
                       const float *w_dy, const float *w_dz, float coef, hfm_stream_t stream) {
  int st;
  if ((st = check_ns(Z, Y, X))) return st;
  if (!adv_u || !adv_v || !adv_w || !base_u || !base_v || !base_w || !out_u || !out_v || !out_w ||
      !k_x || !k_y || !k_z || !w_dx || !w_dy || !w_dz)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_momentum_pg: NULL");
  if (out_u == adv_u || out_v == adv_v || out_w == adv_w || out_u == adv_v || out_u == adv_w ||
      out_v == adv_u || out_v == adv_w || out_w == adv_u || out_w == adv_v)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_momentum_pg: outputs must not alias the advected fields");
  K4 K;
  memset(K.k[0], 0, 27 * 4);
  memcpy(K.k[1], w_dx, 27 * 4);
  memcpy(K.k[2], w_dy, 27 * 4);
  memcpy(K.k[3], w_dz, 27 * 4);
  const int64_t n = (int64_t)Z * Y * X;
  k_momentum<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(adv_u, adv_v, adv_w, base_u, base_v,
                                                             base_w, out_u, out_v, out_w, Z, Y, X,
                                                             K, coef, k_x, k_y, k_z);
  HFM_CHECK_LAUNCH("k_momentum");
  return HFM_OK;
}

size_t hfm_ns_pg_scratch_bytes(int Z, int Y, int X) {
  if (Z <= 0 || Y <= 0 || X <= 0) return 0;
  return (size_t)3 * Z * Y * X * sizeof(float);
}

int hfm_ns_pg_dissipation(const float *u, const float *v, const float *w, const float *sigma,
                          float *k_x, float *k_y, float *k_z, int Z, int Y, int X,
                          const float *w_dif, const float *w_dx, const float *w_dy,
                          const float *w_dz, float dt, float eps_k, void *scratch,
                          hfm_stream_t stream) {
  int st;
  if ((st = check_ns(Z, Y, X))) return st;
  if (!u || !v || !w || !sigma || !k_x || !k_y || !k_z || !w_dif || !w_dx || !w_dy || !w_dz || !scratch)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_pg_dissipation: NULL");
  K4 K;
  memcpy(K.k[0], w_dif, 27 * 4);
  memcpy(K.k[1], w_dx, 27 * 4);
  memcpy(K.k[2], w_dy, 27 * 4);
  memcpy(K.k[3], w_dz, 27 * 4);
  const int64_t n = (int64_t)Z * Y * X;
  float *ku = (float *)scratch, *kv = ku + n, *kw = kv + n;
  k_pg_coef<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(u, v, w, sigma, ku, kv, kw, Z, Y, X, K,
                                                            dt, eps_k);
  HFM_CHECK_LAUNCH("k_pg_coef");
  k_pg_flux<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(u, v, w, sigma, ku, kv, kw, k_x, k_y, k_z,
                                                            Z, Y, X, K, dt);
  HFM_CHECK_LAUNCH("k_pg_flux");
  return HFM_OK;
}

int hfm_ns_pressure_gradient(const float *p, float *u, float *v, float *w, int Z, int Y, int X,
                             const float *w_px, const float *w_py, const float *w_pz,
                             hfm_stream_t stream) {
  if (!p || !u || !v || !w || !w_px || !w_py || !w_pz || Z < 1 || Y < 1 || X < 1)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_pressure_gradient: bad argument");
  K3 K;
  memcpy(K.k[0], w_px, 27 * 4);
  memcpy(K.k[1], w_py, 27 * 4);
  memcpy(K.k[2], w_pz, 27 * 4);
  const int64_t n = (int64_t)Z * Y * X;
  k_pgrad<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, u, v, w, Z, Y, X, K);
  HFM_CHECK_LAUNCH("k_pgrad");
  return HFM_OK;
}

int hfm_ns_divergence(const float *u, const float *v, const float *w, float *b, int Z, int Y,
                      int X, const float *w_su, const float *w_sv, const float *w_sw,
                      int bc_source, hfm_stream_t stream) {
  if (!u || !v || !w || !b || !w_su || !w_sv || !w_sw || Z < 1 || Y < 1 || X < 1)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_divergence: bad argument");
  K3 K;
  memcpy(K.k[0], w_su, 27 * 4);
  memcpy(K.k[1], w_sv, 27 * 4);
  memcpy(K.k[2], w_sw, 27 * 4);
  const int64_t n = (int64_t)Z * Y * X;
  k_divergence<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(u, v, w, b, Z, Y, X, K, bc_source);
  HFM_CHECK_LAUNCH("k_divergence");
  return HFM_OK;
}

int hfm_ns_immersed_body(float *u, float *v, float *w, const float *sigma, int Z, int Y, int X,
                         float dt, hfm_stream_t stream) {
  if (!u || !v || !w || !sigma || Z < 1 || Y < 1 || X < 1)
    return fail(HFM_ERR_BAD_ARG, "hfm_ns_immersed_body: bad argument");
  const int64_t n = (int64_t)Z * Y * X;
  k_ibm<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(u, v, w, sigma, n, dt);
  HFM_CHECK_LAUNCH("k_ibm");
  return HFM_OK;
}

}  // extern "C"
