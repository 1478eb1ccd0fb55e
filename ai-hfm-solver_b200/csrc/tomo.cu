// Misfit gradient with respect to per-cell log-conductivities (resistivity tomography).
//
// For the operator (A u)_c = sum over the six faces a_f (u_c - u_nb), with interior face
// coefficients a = c_d (s_i + s_j) / 2 and wall faces a = c_d s_c (ghost potential zero),
// the bilinear form is  lam^T A u = sum_interior a_f (lam_i - lam_j)(u_i - u_j)
//                                 + sum_wall a_f lam_c u_c.
// With forward fields u_s (A u_s = q_s) and adjoint fields lam_s (A lam_s = P^T (P u_s - d_s),
// A is symmetric), the misfit J = 1/2 sum_s |P u_s - d_s|^2 has
//   dJ / d log s_d(c) = - s_d(c) sum_s dA/ds_d(c) [lam_s, u_s],
// and dA/ds_d(c) collects 1/2 c_d (lam_c - lam_nb)(u_c - u_nb) over the (at most two)
// interior faces of c on axis d, and c_d lam_c u_c for each wall face of c on that axis.
#include "hfm_internal.cuh"

namespace hfm {
namespace {

__global__ void k_grad_logsigma(const float *__restrict__ sx, const float *__restrict__ sy,
                                const float *__restrict__ sz, const double *__restrict__ u,
                                const double *__restrict__ lam, int S, int Z, int Y, int X,
                                float cz, float cy, float cx, double *__restrict__ gx,
                                double *__restrict__ gy, double *__restrict__ gz,
                                int accumulate) {
  const int64_t n = (int64_t)Z * Y * X;
  const int64_t PL = (int64_t)X * Y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const int64_t t = i / X;
    const int y = (int)(t % Y), z = (int)(t / Y);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int s = 0; s < S; ++s) {
      const double *us = u + (int64_t)s * n, *ls = lam + (int64_t)s * n;
      const double uc = us[i], lc = ls[i];
      // x faces
      if (x > 0) ax += 0.5 * (lc - ls[i - 1]) * (uc - us[i - 1]); else ax += lc * uc;
      if (x < X - 1) ax += 0.5 * (lc - ls[i + 1]) * (uc - us[i + 1]); else ax += lc * uc;
      if (y > 0) ay += 0.5 * (lc - ls[i - X]) * (uc - us[i - X]); else ay += lc * uc;
      if (y < Y - 1) ay += 0.5 * (lc - ls[i + X]) * (uc - us[i + X]); else ay += lc * uc;
      if (z > 0) az += 0.5 * (lc - ls[i - PL]) * (uc - us[i - PL]); else az += lc * uc;
      if (z < Z - 1) az += 0.5 * (lc - ls[i + PL]) * (uc - us[i + PL]); else az += lc * uc;
    }
    const double vx = -(double)sx[i] * cx * ax;
    const double vy = -(double)sy[i] * cy * ay;
    const double vz = -(double)sz[i] * cz * az;
    if (accumulate) {
      gx[i] += vx;
      gy[i] += vy;
      gz[i] += vz;
    } else {
      gx[i] = vx;
      gy[i] = vy;
      gz[i] = vz;
    }
  }
}

}  // namespace
}  // namespace hfm

using namespace hfm;

extern "C" int hfm_sigma7_grad_logsigma(const float *sx, const float *sy, const float *sz,
                                        const double *u, const double *lam, int S, int Z,
                                        int Y, int X, float cz, float cy, float cx, double *gx,
                                        double *gy, double *gz, int accumulate,
                                        hfm_stream_t stream) {
  if (!sx || !sy || !sz || !u || !lam || !gx || !gy || !gz || S <= 0 || Z <= 0 || Y <= 0 || X <= 0)
    return fail(HFM_ERR_BAD_ARG, "hfm_sigma7_grad_logsigma: bad argument");
  const int64_t n = (int64_t)Z * Y * X;
  int64_t nb = (n + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 8;
  if (nb > cap) nb = cap;
  k_grad_logsigma<<<(int)nb, 256, 0, (cudaStream_t)stream>>>(sx, sy, sz, u, lam, S, Z, Y, X, cz,
                                                              cy, cx, gx, gy, gz, accumulate);
  HFM_CHECK_LAUNCH("k_grad_logsigma");
  return HFM_OK;
}
