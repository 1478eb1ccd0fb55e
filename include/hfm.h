/*
 * hfm.h - C ABI of libhfm, the B200 (sm_100a) stencil + geometric-multigrid library that
 * replaces the frozen-weight TensorFlow layers and the Python multigrid loops of
 * bc1chen/AI-HFM-Solver ("AI4CFD").
 *
 * Conventions shared by every entry point
 *   - Fields are float32 (unless stated) in C order [B][Z][Y][X], X fastest: the reference
 *     tensor (1, Z, Y, X, 1) with the batch of B independent instances stacked in front.
 *     All pointers are device pointers unless the name says "host".
 *   - A 3x3x3 kernel w27 is indexed (dz, dy, dx) row-major, w27[9*a + 3*b + c] applying to
 *     phi[z+a-1][y+b-1][x+c-1] (cross-correlation, like TF Conv3D).  Samples outside the
 *     grid are zero (TF 'SAME' zero padding = homogeneous Dirichlet ghost cells).
 *   - Residual sign follows the reference: r = A phi - b, and corrections are subtracted.
 *   - Every call returns an hfm_status; hfm_last_error() gives a message for the calling
 *     thread.  Calls enqueue work on `stream` (a cudaStream_t) and return without
 *     synchronising, unless documented otherwise.  No stateless call allocates memory.
 */
#ifndef HFM_H_
#define HFM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HFM_ABI_VERSION 1

typedef void *hfm_stream_t; /* cudaStream_t */

typedef enum {
  HFM_OK = 0,
  HFM_ERR_BAD_ARG = 1,       /* malformed shape, null pointer, unsupported combination */
  HFM_ERR_OOM = 2,           /* device allocation failed (handles only) */
  HFM_ERR_NOT_CONVERGED = 3, /* max_cycles reached above tolerance (the reference's guard) */
  HFM_ERR_NAN = 4,           /* NaN/Inf found in a residual norm */
  HFM_ERR_TIMEOUT = 5,       /* a bounded device-side wait expired */
  HFM_ERR_CUDA = 6,          /* CUDA runtime error (message in hfm_last_error) */
  HFM_ERR_UNSUPPORTED = 7,
  HFM_ERR_CANCELLED = 8      /* a served request cancelled before it finished */
} hfm_status;

typedef enum { HFM_F32 = 0, HFM_BF16 = 1, HFM_F16 = 2, HFM_F64 = 3 } hfm_dtype;

/* Operator kinds: the reference's constant-coefficient 7-point, per-cell conductivity and
 * directional forms, and any frozen 3x3x3 kernel. */
typedef enum {
  HFM_OP_CONST7 = 0, /* anisotropic 7-point, constant coefficients kz, ky, kx (7point.ipynb w2) */
  HFM_OP_SIGMA7 = 1, /* 7-point from per-cell conductivities sx, sy, sz (face means) */
  HFM_OP_DIR7 = 2,   /* six per-cell directional coefficient arrays + diagonal (BGS form) */
  HFM_OP_K27 = 3,    /* arbitrary frozen 3x3x3 kernel (27-point pressure / diffusion) */
  HFM_OP_FACE7 = 4   /* 7-point from stored face coefficients, walls included (below) */
} hfm_op_kind;

/* Flags for residual / smoothing calls. */
#define HFM_FLAG_ZERO_XEND 1u  /* NS pressure form: residual / corrected phi zero on plane x = X-1 */
#define HFM_FLAG_TOP_COPY 2u   /* after smoothing copy plane z = 1 onto z = 0 (boundary_condition_top) */
#define HFM_FLAG_ZERO_GUESS 4u /* the input phi is identically zero (not read) */
#define HFM_FLAG_PERIODIC 8u   /* 2D operators: wrap around instead of zero padding */
#define HFM_FLAG_SAME_LEVEL_CORR 16u /* hfm_jacobi2d: `coarse` is on the same grid (no upsampling) */
#define HFM_FLAG_TWO_SWEEPS 32u /* hfm_jacobi2d: two sweeps (the first from base + sign P(coarse),
                                   the second plain) in one pass, the bits of two calls */

/* Operator descriptor (plain data, copied by value into each launch).
 *   CONST7: k[0..2] = (kz, ky, kx) = (Dz/dz^2, Dy/dy^2, Dx/dx^2); diagonal 2(kz+ky+kx).
 *   SIGMA7: coef[0..2] = sx, sy, sz ([B][Z][Y][X] each); c[0..2] = (cz, cy, cx) = 1/h^2.
 *           Face coefficient between cells i, j on axis d: c_d (s_i + s_j)/2; a wall face
 *           uses c_d s_i.  (Anisotropic Resistivity Tomography/README:14-26)
 *   DIR7:   coef[0..6] = A_xm, A_xp, A_ym, A_yp, A_zm, A_zp, A_tot (BGS_multigrid_v1 cell 38),
 *           (A phi)_c = sum_d A_d (phi_c - phi_nb(d)), diagonal A_tot.
 *   K27:    k[0..26] = w27; Jacobi diagonal = k[13].
 *   FACE7:  coef[0..2] = Fx, Fy, Fz, the coefficients of every cell face, walls included:
 *           Fx per instance [Z][Y][X + 8]: element i = 0 .. X of a row is the face between
 *             cells i-1 and i (i = 0 and i = X are the walls; elements past X are unused);
 *           Fy per instance [Z][Y + 1][X]: row j = 0 .. Y is the face between rows j-1, j;
 *           Fz per instance [Z + 1][Y][X]: plane k = 0 .. Z likewise.
 *           (A phi)_c = sum over the six faces F of c of F (phi_c - phi_nb), phi_nb = 0
 *           outside the grid; the Jacobi diagonal is the sum of the six faces.  The
 *           SIGMA7 operator in this form is hfm_sigma7_faces' output; in 16-bit storage it
 *           rounds each face once (SIGMA7 in 16-bit storage rounds the conductivities).
 *           Instance strides follow from the extents.  No counterpart in the reference,
 *           whose per-direction arrays (BGS_multigrid_v1.ipynb cell 38) are per cell.
 *   scale multiplies the operator (1 = reference; coarse levels of a handle use
 *   coarse_scale^level).  coef_dtype is the storage type of coef arrays (HFM_F32 for the
 *   stateless calls). */
typedef struct {
  int kind;
  int coef_dtype;
  float k[27];
  float c[3];
  float scale;
  const void *coef[7];
} hfm_operator;

/* ---------------------------------------------------------------- library information */
int hfm_abi_version(void);
const char *hfm_status_string(int status);
const char *hfm_last_error(void);
int hfm_device_sm_count(int *sm_count); /* current device's SM count */
/* Kernels this library has enqueued since load (a CUDA-graph launch counts its kernel nodes). */
int64_t hfm_kernel_launch_count(void);
/* Bounded device-side waits that expired on the current device (TMA pipeline stages); a
 * non-zero count means results of the affected launches are invalid.  reset != 0 clears it.
 * While this count or the drain count below is non-zero, every multigrid handle's
 * convergence check on this device marks its active slots HFM_ERR_TIMEOUT and switches
 * them off (no slot reports success after a failed wait); clear both to resume. */
int hfm_device_timeouts(int *count, int reset);
/* Drain waits that expired: after a plane wait expires, the block waits (bounded) for the
 * copies it already issued; if that wait expires as well, the block exits with copies
 * possibly still in flight and this count is raised.  A non-zero value means the context is
 * suspect: stop issuing work on the device and report it.  reset != 0 clears it.  No
 * counterpart in the reference. */
int hfm_device_drain_timeouts(int *count, int reset);
/* Poll budget of those waits for launches made after the call (default and maximum 2^20).
 * Budget 0 makes every such wait expire at once - the failure path, for tests: each block
 * stops, lets the copies it issued land, counts the timeout and returns; results of those
 * launches are invalid.  No counterpart in the reference. */
int hfm_set_wait_budget(int polls);

/* ------------------------------------------------ stateless operators (drop-in layers) */
/* Conv3D(1, kernel_size=3, strides=1, padding='SAME') with frozen weights and zero bias:
 * replaces every `keras.models.Sequential([... Conv3D(k=3, 'SAME')])` callable, e.g.
 * CNN3D_A_<n> (Anisotropic_3d_Multigrid_7point.ipynb cell 7, lines 124-183),
 * CNN3D_central_2nd_{dif,xadv,yadv,zadv}, CNN3D_{Su,Sv,Sw,pu,pv,pw} (naiver_stokes_3D.py:166-236). */
int hfm_conv3d_k3(const float *x, float *y, int B, int Z, int Y, int X, const float *w27_host,
                  hfm_stream_t stream);

/* Conv3D(1, kernel_size=2, strides=2, padding='VALID') with weights 0.125 = CNN3D_res_<n>
 * (Anisotropic_3d_Multigrid_7point.ipynb cell 9, lines 194-240).  Output extent floor(n/2). */
int hfm_restrict_avg(const float *fine, float *coarse, int B, int Z, int Y, int X,
                     hfm_stream_t stream);

/* UpSampling3D(size=(2,2,2)) = CNN3D_prol_<n> (Anisotropic_3d_Multigrid_7point.ipynb cell 11,
 * lines 251-289).  (Zc, Yc, Xc) are the coarse extents; the fine output is twice each. */
int hfm_prolong_nearest(const float *coarse, float *fine, int B, int Zc, int Yc, int Xc,
                        hfm_stream_t stream);

/* out = A phi (operator descriptor form): CNN3D_A_<n>(phi) / A_operator_<n>(phi)
 * (BGS_multigrid_v1.ipynb cell 40). */
int hfm_op_apply(const hfm_operator *op, const float *phi, float *out, int B, int Z, int Y,
                 int X, hfm_stream_t stream);

/* r = A phi - b (Anisotropic_3d_Multigrid_7point.ipynb:409; naiver_stokes_3D.py:649-651 with
 * HFM_FLAG_ZERO_XEND). */
int hfm_op_residual(const hfm_operator *op, const float *phi, const float *b, float *r, int B,
                    int Z, int Y, int X, unsigned flags, hfm_stream_t stream);

/* `sweeps` weighted-Jacobi sweeps phi <- phi + omega (rhs - A phi) / diag
 * (reference form w - A(w)/d + r/d with omega = 1, 7point.ipynb:424-449).  The result is in
 * `out`; for sweeps > 1 the sweeps ping-pong between `out` and `tmp` (caller memory, same
 * size; may be NULL when sweeps == 1).  phi may alias neither out nor tmp. */
int hfm_op_jacobi(const hfm_operator *op, const float *phi, const float *rhs, float *out,
                  float *tmp, int B, int Z, int Y, int X, float omega, int sweeps,
                  unsigned flags, hfm_stream_t stream);

/* One weighted-Jacobi sweep with fields and conductivities stored as `dtype` (HFM_F32,
 * HFM_BF16 or HFM_F16; arithmetic in float32): the smoother of the reduced-precision inner
 * cycles, exposed for direct use and measurement.  op->coef_dtype must equal dtype. */
int hfm_op_jacobi_typed(const hfm_operator *op, int dtype, const void *phi, const void *rhs,
                        void *out, int B, int Z, int Y, int X, float omega, unsigned flags,
                        hfm_stream_t stream);

/* The residual and the two fused transfer operators with fields and coefficients stored as
 * `dtype` (as hfm_op_jacobi_typed): r = A phi - b; r_coarse = R (A phi - b) (r_fine may be
 * NULL); out = J(phi - P w_coarse).  The other kernels of the reduced-precision inner cycles,
 * exposed for direct use, testing and measurement.  op->coef_dtype must equal dtype. */
int hfm_op_residual_typed(const hfm_operator *op, int dtype, const void *phi, const void *b,
                          void *r, int B, int Z, int Y, int X, unsigned flags,
                          hfm_stream_t stream);
int hfm_residual_restrict_typed(const hfm_operator *op, int dtype, const void *phi,
                                const void *b, void *r_fine, void *r_coarse, int B, int Z,
                                int Y, int X, unsigned flags, hfm_stream_t stream);
int hfm_prolong_correct_smooth_typed(const hfm_operator *op, int dtype, const void *phi,
                                     const void *w_coarse, const void *rhs, void *out, int B,
                                     int Z, int Y, int X, float omega, unsigned flags,
                                     hfm_stream_t stream);

/* Two weighted-Jacobi sweeps of a FACE7 operator in one pass over the grid (temporal
 * blocking; the two iterations of the reference's sweep loop,
 * Anisotropic_3d_Multigrid_7point.ipynb:424-444): out = J(J(phi - P w_coarse)), or
 * out = J(J(phi)) when w_coarse is NULL.  16-bit storage (dtype BF16 / F16 = coef_dtype),
 * bitwise equal to two hfm_op_jacobi_typed calls (the first with the correction, as
 * hfm_prolong_correct_smooth_typed).  Grids: X >= 48 and a multiple of 8, Y >= 16, Z >= 2;
 * with w_coarse also X a multiple of 16 and Y, Z even; others return HFM_ERR_UNSUPPORTED.
 * Fields 16-byte aligned; phi must not alias out. */
int hfm_face7_smooth2_typed(const hfm_operator *op, int dtype, const void *phi,
                            const void *w_coarse, const void *rhs, void *out, int B, int Z,
                            int Y, int X, float omega, hfm_stream_t stream);

/* Face coefficients of the SIGMA7 operator (face means c_d (s_i + s_j) / 2, wall faces
 * c_d s_i; Anisotropic Resistivity Tomography/README:14-26) in the FACE7 layout, stored in
 * `dtype` (F32, BF16 or F16; each face computed in float32 from the float32 sx, sy, sz and
 * rounded once).  fx, fy, fz hold B instances of hfm_face7_elems' sizes; elements of Fx
 * past X are written as zero. */
int hfm_sigma7_faces(int dtype, const float *sx, const float *sy, const float *sz, float cz,
                     float cy, float cx, void *fx, void *fy, void *fz, int B, int Z, int Y,
                     int X, hfm_stream_t stream);
/* Elements per instance of the FACE7 arrays Fx, Fy, Fz for extents (Z, Y, X). */
int hfm_face7_elems(int Z, int Y, int X, int64_t *nfx, int64_t *nfy, int64_t *nfz);

/* Fused residual + restriction: r_coarse = R (A phi - b) on the even grid (Z, Y, X), and
 * r_fine = A phi - b when r_fine is not NULL (7point.ipynb:409-419). */
int hfm_residual_restrict(const hfm_operator *op, const float *phi, const float *b,
                          float *r_fine, float *r_coarse, int B, int Z, int Y, int X,
                          unsigned flags, hfm_stream_t stream);

/* Fused prolongation + correction + one smoothing sweep:
 * out = J(phi - P w_coarse) against rhs (7point.ipynb:443-449; phi may be NULL = zero, which
 * gives the sawtooth "w_n = prol(w); Jacobi" step). (Z, Y, X) are the fine extents. */
int hfm_prolong_correct_smooth(const hfm_operator *op, const float *phi,
                               const float *w_coarse, const float *rhs, float *out, int B,
                               int Z, int Y, int X, float omega, unsigned flags,
                               hfm_stream_t stream);

/* Named wrappers: constant-coefficient 7-point, per-cell sigma 7-point
 * and 27-point forms of apply / residual / jacobi. */
int hfm_stencil7_const_apply(const float *phi, float *out, int B, int Z, int Y, int X,
                             float kz, float ky, float kx, hfm_stream_t stream);
int hfm_stencil7_const_residual(const float *phi, const float *b, float *r, int B, int Z,
                                int Y, int X, float kz, float ky, float kx, unsigned flags,
                                hfm_stream_t stream);
int hfm_stencil7_const_jacobi(const float *phi, const float *rhs, float *out, float *tmp,
                              int B, int Z, int Y, int X, float kz, float ky, float kx,
                              float omega, int sweeps, unsigned flags, hfm_stream_t stream);
int hfm_stencil7_var_apply(const float *phi, float *out, const float *sx, const float *sy,
                           const float *sz, int B, int Z, int Y, int X, float cz, float cy,
                           float cx, hfm_stream_t stream);
int hfm_stencil7_var_residual(const float *phi, const float *b, float *r, const float *sx,
                              const float *sy, const float *sz, int B, int Z, int Y, int X,
                              float cz, float cy, float cx, unsigned flags,
                              hfm_stream_t stream);
int hfm_stencil7_var_jacobi(const float *phi, const float *rhs, float *out, float *tmp,
                            const float *sx, const float *sy, const float *sz, int B, int Z,
                            int Y, int X, float cz, float cy, float cx, float omega,
                            int sweeps, unsigned flags, hfm_stream_t stream);
int hfm_stencil27_apply(const float *phi, float *out, int B, int Z, int Y, int X,
                        const float *w27_host, hfm_stream_t stream);
int hfm_stencil27_residual(const float *phi, const float *b, float *r, int B, int Z, int Y,
                           int X, const float *w27_host, unsigned flags, hfm_stream_t stream);
int hfm_stencil27_jacobi(const float *phi, const float *rhs, float *out, float *tmp, int B,
                         int Z, int Y, int X, const float *w27_host, float omega, int sweeps,
                         unsigned flags, hfm_stream_t stream);

/* ------------------------------------------------------------------------ reductions */
/* Per-instance reductions over n elements of each of B instances (HFM3 diagnostics
 * np.max(w), np.max(r): Urban Modelling/AI_HFM_v3.ipynb:2622-2627).  Results land in device
 * memory (B values).  `scratch` is caller device memory of hfm_reduce_scratch_bytes(n, B)
 * bytes; the summation order is fixed, so results do not depend on other work in flight.
 * B is at most 65535 (one grid row per instance); larger B returns HFM_ERR_BAD_ARG and
 * hfm_reduce_scratch_bytes returns 0 for it. */
size_t hfm_reduce_scratch_bytes(int64_t n, int B);
int hfm_norm2_f64(const float *x, int64_t n, int B, double *out, void *scratch,
                  hfm_stream_t stream); /* sqrt(sum x^2), accumulated in float64 */
int hfm_max_abs(const float *x, int64_t n, int B, float *out, void *scratch,
                hfm_stream_t stream);
/* Per-instance sum of x * y in float64 (fixed order, scratch as above); instance i starts at
 * x + i * stride (stride >= n when B > 1).  The dot products of the Z-slab conjugate-gradient
 * solver, whose slabs are instances with the halo planes outside the n interior cells.  No
 * counterpart in the reference: its cycles run a fixed count (multi_itr,
 * Anisotropic_3d_Multigrid_7point.ipynb:402-405) and its parallel runs compare norms only
 * afterwards on the host (parallel_multigrid_advection_diffusion_3D.ipynb cell 72). */
int hfm_dot_f64(const float *x, const float *y, int64_t n, int B, int64_t stride, double *out,
                void *scratch, hfm_stream_t stream);

/* hfm_norm2_f64 for callers that cannot allocate device memory: no counterpart in the
 * reference.  Some callers have no way to obtain scratch - a C or Fortran host code that
 * owns no device allocator, or a time-stepping loop under a fixed device-memory budget where
 * a cudaMalloc (which may synchronise the whole device) is not allowed.  This variant keeps
 * its block partial sums in a static device array of HFM_NORM2_NOALLOC_SCRATCH_BYTES inside
 * the library, so it allocates nothing; the caller still passes x and out (device, B
 * doubles).  Limit: hfm_reduce_scratch_bytes(n, B) must not exceed that size (512 KiB, e.g.
 * up to 221 instances of any size, more for small n); larger requests return
 * HFM_ERR_BAD_ARG.  Every GPU that loads the library holds the array until the process
 * exits.  The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it; make that first call before any stream capture.
 * All calls share the one array: calls whose kernels overlap on the GPU (different streams
 * without ordering) race and may return wrong sums; order them on one stream.  Results are
 * bitwise equal to hfm_norm2_f64's. */
#define HFM_NORM2_NOALLOC_SCRATCH_BYTES (512u * 1024u)
int hfm_norm2_f64_noalloc(const float *x, int64_t n, int B, double *out, hfm_stream_t stream);

/* ---------------------------------------------------------- Z-slab conjugate gradients */
/* Vector updates of a conjugate-gradient solve whose grid is cut into B slabs along Z (one
 * slab per instance, instance i at base + i * stride, n interior cells each).  They replace
 * nothing in the reference, whose parallel solver (Anisotropic Resistivity Tomography/
 * scripts/parallel_naiver_stokes_3D.py:745-823) runs stationary cycles with a host halo update
 * (halo_exchange.py:635-719, structured_halo_update_3D) after every stencil call.  The
 * coefficient is num[0] / den[0] read on the device (float64 sums already reduced over every
 * slab of the solve), so no host round trip sits between the dot product and the update.
 *   hfm_cg_update_xr:  a = num / den;  x += a p;  r -= a q
 *   hfm_cg_update_p:   b = num / den (0 when den is NULL or 0);  p = z + b p */
int hfm_cg_update_xr(float *x, float *r, const float *p, const float *q, const double *num,
                     const double *den, int64_t n, int B, int64_t stride, hfm_stream_t stream);
int hfm_cg_update_p(float *p, const float *z, const double *num, const double *den, int64_t n,
                    int B, int64_t stride, hfm_stream_t stream);

/* ---------------------------------------------------------------- NS time-stepper operators */
/* Operators of scripts/naiver_stokes_3D.py (and Urban Modelling/AI_HFM_v3.ipynb cell 19) on
 * single (Z, Y, X) float32 fields; x is the flow direction (inflow x = 0, outflow X-1),
 * extents >= 3.  Kernel arguments are 27 host weights (dz, dy, dx), e.g. w1 (diffusion),
 * w2-w4 (smoothed central differences, naiver_stokes_3D.py:36-94), w6-w8 (divergence). */
/* out_f = base_f + coef (Dif(a_f) - a_u Dx(a_f) - a_v Dy(a_f) - a_w Dz(a_f)) for f = u, v, w:
 * stage 1 of the momentum update with a = base = u^n, coef 0.5; stage 2 with a = b, base = u^n,
 * coef 1 (naiver_stokes_3D.py:580-622).  Outputs must not alias the advected fields. */
int hfm_ns_momentum(const float *adv_u, const float *adv_v, const float *adv_w,
                    const float *base_u, const float *base_v, const float *base_w, float *out_u,
                    float *out_v, float *out_w, int Z, int Y, int X, const float *w_dif,
                    const float *w_dx, const float *w_dy, const float *w_dz, float coef,
                    hfm_stream_t stream);
/* The momentum stage of Urban Modelling/INHALE_demo.ipynb cell 24, where the Petrov-Galerkin
 * dissipation k_f replaces the diffusion stencil: out_f = base_f + coef (k_f - a_u Dx(a_f) -
 * a_v Dy(a_f) - a_w Dz(a_f)). */
int hfm_ns_momentum_pg(const float *adv_u, const float *adv_v, const float *adv_w,
                       const float *base_u, const float *base_v, const float *base_w,
                       float *out_u, float *out_v, float *out_w, const float *k_x,
                       const float *k_y, const float *k_z, int Z, int Y, int X, const float *w_dx,
                       const float *w_dy, const float *w_dz, float coef, hfm_stream_t stream);
/* Petrov_Galerkin_dissipation of INHALE_demo.ipynb cell 20 on the velocities damped by the
 * immersed body (u / (1 + dt sigma)): per component k_f = min(2 |(|u|+|v|+|w|)/3 Dif(f)| /
 * (eps_k + (|Dx f| + |Dy f| + |Dz f|)/3), 0.5) / (1 + dt sigma), then
 * out_f = 1.5 (k_f Dif(f) + Dif(f k_f) - f Dif(k_f)).  scratch: hfm_ns_pg_scratch_bytes. */
size_t hfm_ns_pg_scratch_bytes(int Z, int Y, int X);
int hfm_ns_pg_dissipation(const float *u, const float *v, const float *w, const float *sigma,
                          float *k_x, float *k_y, float *k_z, int Z, int Y, int X,
                          const float *w_dif, const float *w_dx, const float *w_dy,
                          const float *w_dz, float dt, float eps_k, void *scratch,
                          hfm_stream_t stream);
/* u -= conv(p, w_px), v -= conv(p, w_py), w -= conv(p, w_pz) (CNN3D_pu/pv/pw, :631-633). */
int hfm_ns_pressure_gradient(const float *p, float *u, float *v, float *w, int Z, int Y, int X,
                             const float *w_px, const float *w_py, const float *w_pz,
                             hfm_stream_t stream);
/* b = -(Su(u) + Sv(v) + Sw(w)) (:641); bc_source != 0 applies boundary_condition_source
 * (plane x = 0 takes plane x = 1, :467-473). */
int hfm_ns_divergence(const float *u, const float *v, const float *w, float *b, int Z, int Y,
                      int X, const float *w_su, const float *w_sv, const float *w_sw,
                      int bc_source, hfm_stream_t stream);
/* bluff_body: u, v, w /= (1 + dt sigma) (:478-483). */
int hfm_ns_immersed_body(float *u, float *v, float *w, const float *sigma, int Z, int Y, int X,
                         float dt, hfm_stream_t stream);
/* boundary_condition_velocity / _pressure (:420-462) in place, with the reference's
 * assignment order and copies read from the input; scratch: caller device memory of
 * hfm_ns_bc_scratch_bytes(Z, Y, X) bytes. */
size_t hfm_ns_bc_scratch_bytes(int Z, int Y, int X);
int hfm_ns_bc_velocity(float *u, float *v, float *w, int Z, int Y, int X, float ub,
                       void *scratch, hfm_stream_t stream);
int hfm_ns_bc_pressure(float *p, int Z, int Y, int X, void *scratch, hfm_stream_t stream);

/* --------------------------------------------------------------- resistivity tomography */
/* Gradient of the misfit J = 1/2 sum_s |P u_s - d_s|^2 with respect to per-cell log sx, sy,
 * sz for the SIGMA7 operator (face means, wall faces c_d s_c), given the forward fields u_s
 * and adjoint fields lam_s (A lam_s = P^T (P u_s - d_s)), S fields each of [Z][Y][X] float64:
 *   g_d(c) = - s_d(c) sum_s dA/ds_d(c)[lam_s, u_s].
 * accumulate != 0 adds into g (source groups), else overwrites.  No counterpart layer in the
 * reference, whose resistivity notebooks stop at the forward solve; the operator follows
 * Anisotropic Resistivity Tomography/README:14-26. */
int hfm_sigma7_grad_logsigma(const float *sx, const float *sy, const float *sz, const double *u,
                             const double *lam, int S, int Z, int Y, int X, float cz, float cy,
                             float cx, double *gx, double *gy, double *gz, int accumulate,
                             hfm_stream_t stream);

/* ---------------------------------------------------------------- 2D operators
 * The reference's two-dimensional multigrid (Unstructured Mesh/Multigrid_2D.ipynb) on
 * (B, Y, X) fields, x fastest, float32 or bf16 storage (dtype HFM_F32 / HFM_BF16) with
 * float32 arithmetic.  w9 is a host array of 9 weights, w9[3a + b] multiplying
 * phi[y + a - 1][x + b - 1] (cross-correlation, the Conv2D kernel w2[0][a][b][0] of cell 3).
 * Padding is zero (Conv2D 'SAME') unless flags has HFM_FLAG_PERIODIC. */
/* y = conv(x, w9): CNN3D_A_<n> Conv2D(1, 3, 'SAME') layers, Multigrid_2D.ipynb#c7. */
int hfm_conv2d_k3(const float *x, float *y, int B, int Y, int X, const float *w9_host,
                  unsigned flags, hfm_stream_t stream);
/* 2x2 VALID average, weight 0.25 (odd extents floored): CNN3D_res_<n>, Multigrid_2D.ipynb#c9. */
int hfm_restrict_avg2d(int dtype, const void *fine, void *coarse, int B, int Y, int X,
                       hfm_stream_t stream);
/* UpSampling2D(2): CNN3D_prol_<n>, Multigrid_2D.ipynb#c11. */
int hfm_prolong_nearest2d(int dtype, const void *coarse, void *fine, int B, int Yc, int Xc,
                          hfm_stream_t stream);
/* One Jacobi sweep out = phi + omega (rhs - A phi) / w9[4] with phi = base + coarse_sign *
 * P(coarse) (either may be NULL = 0; P = nearest upsampling, even extents, or the identity
 * with HFM_FLAG_SAME_LEVEL_CORR), rhs NULL = 0:
 * the per-level update `w - A(w)/d + r/d` of Multigrid_2D.ipynb#c18 (omega = 1), fused with
 * the prolongation that precedes it. */
int hfm_jacobi2d(int dtype, const float *w9_host, const void *base, const void *coarse,
                 float coarse_sign, const void *rhs, void *out, int B, int Y, int X, float omega,
                 unsigned flags, hfm_stream_t stream);
/* The down leg of a level with two pre-sweeps in one launch: phi = two Jacobi sweeps from
 * zero on rhs, coarse_rhs = 2 x 2 average of (A phi - rhs) on the (Y/2, X/2) grid; the bits
 * of hfm_jacobi2d with HFM_FLAG_TWO_SWEEPS followed by hfm_residual_restrict2d.  Even
 * extents; rhs, phi and coarse_rhs distinct. */
int hfm_pre2_restrict2d(int dtype, const float *w9_host, const void *rhs, void *phi,
                        void *coarse_rhs, int B, int Y, int X, float omega, unsigned flags,
                        hfm_stream_t stream);
/* r = A phi - rhs (rhs NULL = 0): Multigrid_2D.ipynb#c18 `CNN3D_A_128(values) - b`. */
int hfm_residual2d(int dtype, const float *w9_host, const void *phi, const void *rhs, void *r,
                   int B, int Y, int X, unsigned flags, hfm_stream_t stream);
/* r_coarse = R(A phi - rhs) in one pass (phi NULL = 0, even extents). */
int hfm_residual_restrict2d(int dtype, const float *w9_host, const void *phi, const void *rhs,
                            void *r_coarse, int B, int Y, int X, unsigned flags,
                            hfm_stream_t stream);
/* Outer defect of a mixed-precision solve: r (out_dtype) = A phi - rhs from float32 phi and
 * rhs, with per-block float64 partial sums of r^2 in partials[b * nblk + k] when partials is
 * not NULL; nblk (returned in *nblk_out) is at most 8 x the SM count (hfm_device_sm_count).
 * No reference counterpart (the reference runs float32 only). */
int hfm_outer_residual2d(const float *w9_host, const float *phi, const float *rhs, int out_dtype,
                         void *r, int B, int Y, int X, unsigned flags, double *partials,
                         int *nblk_out, hfm_stream_t stream);
/* p += sign * w over n values (float32 p, w in dtype): the correction `values - w_128`. */
int hfm_update2d(float *p, int dtype, const void *w, float sign, int64_t n, hfm_stream_t stream);
/* `sweeps` Jacobi sweeps from zero on a grid of at most 4096 cells, one block per instance in
 * shared memory (the coarsest level of a cycle). */
int hfm_coarse_jacobi2d(int dtype, const float *w9_host, const void *rhs, void *out, int B, int Y,
                        int X, float omega, int sweeps, unsigned flags, hfm_stream_t stream);
/* The V-cycle of the coarse levels in one launch, one 1024-thread block per instance with
 * every field in shared memory (float32 between sweeps): from rhs on a first level of at most
 * 4096 cells (Y x X, each coarser level Y/2 x X/2, extents even above the coarsest), nlev <= 8
 * levels with weights w9_levels[9 l .. 9 l + 8], nu_pre >= 1 weighted-Jacobi sweeps from
 * zero, residual and 2 x 2 averaging restriction, coarse_sweeps sweeps from zero on the
 * coarsest level, nearest-prolongation correction phi - P w and nu_post sweeps.  The steps of
 * the per-level entry points above (hfm_jacobi2d, hfm_residual_restrict2d,
 * hfm_coarse_jacobi2d) in the same order and arithmetic: float32 storage gives their bits;
 * bf16 storage rounds only rhs on load and the result on store.  Levels needing more than
 * 200 KB of shared memory (two padded iterates and the rhs per level) return
 * HFM_ERR_UNSUPPORTED. */
int hfm_subcycle2d(int dtype, const float *w9_levels, const void *rhs, void *out, int B, int Y, int X,
                   int nlev, float omega, int nu_pre, int nu_post, int coarse_sweeps, unsigned flags,
                   hfm_stream_t stream);
/* Subtract each instance's mean from p (B instances of n values): the constant null space of
 * a periodic pressure operator. */
int hfm_mean_subtract2d(float *p, int B, int64_t n, hfm_stream_t stream);

/* ---------------------------------------------------------------- 2D Kolmogorov flow
 * Doubly periodic incompressible flow on a Y x X grid of spacing h forced by
 * famp sin(fk y h) in x.  The reference has no Kolmogorov-flow code (its "2D Kolmogorov
 * Flow" folder holds empty placeholders); the stage follows the two-stage momentum update of
 * Anisotropic Resistivity Tomography/scripts/naiver_stokes_3D.py:580-622 in two dimensions with
 * central differences and a 5-point Laplacian, and the projection its pressure-gradient step
 * (:631-633). */
/* out = base + c dt (nu L phi - phi_u d/dx phi - phi_v d/dy phi + F), both components. */
int hfm_kolmogorov_stage(const float *phi_u, const float *phi_v, const float *base_u,
                         const float *base_v, float *out_u, float *out_v, int Y, int X, float c,
                         float dt, float nu, float h, float famp, float fk, hfm_stream_t stream);
/* f = -(du/dx + dv/dy) / dt (right-hand side of -L p = f). */
int hfm_kolmogorov_divergence(const float *u, const float *v, float *f, int Y, int X, float h,
                              float dt, hfm_stream_t stream);
/* u -= dt dp/dx, v -= dt dp/dy. */
int hfm_kolmogorov_project(float *u, float *v, const float *p, int Y, int X, float h, float dt,
                           hfm_stream_t stream);


/* ------------------------------------------------------------------ multigrid handle */
typedef enum { HFM_CYCLE_SAWTOOTH = 0, HFM_CYCLE_V = 1, HFM_CYCLE_F = 2 } hfm_cycle;
/* NONE: stationary cycles; CG: the cycle preconditions conjugate gradients; IR: float64
 * iterative refinement (outer residual, norm and update in float64) around CG. */
typedef enum { HFM_ACCEL_NONE = 0, HFM_ACCEL_CG = 1, HFM_ACCEL_IR = 2 } hfm_accel;

typedef struct {
  int op_kind;            /* hfm_op_kind: CONST7, SIGMA7, K27; DIR7 with float32 storage
                             and accel NONE or CG (BGS_multigrid_v1.ipynb cells 38-42) */
  int cycle;              /* hfm_cycle */
  int accel;              /* hfm_accel: NONE = stationary cycles, CG = cycle preconditions CG */
  int n_levels;           /* 0 = automatic (halve while extents even and min > min_coarse_edge) */
  int min_coarse_edge;    /* default 4 */
  int nu_pre, nu_post;    /* V/F smoothing sweeps (default 2, 2) */
  int coarse_sweeps;      /* Jacobi sweeps on the coarsest level (V/F; sawtooth uses 1
                             unless HFM_OPT_SAWTOOTH_COARSE_SWEEPS) */
  float omega;            /* smoother weight (default 2/3; sawtooth reference 1) */
  float coarse_omega;
  float coarse_scale;     /* level l operator scaled by coarse_scale^l (1 = reference) */
  int sawtooth_fine_smooth; /* 1: Jacobi on w at the fine level (7point), 0: NS form */
  unsigned flags;         /* HFM_FLAG_TOP_COPY / HFM_FLAG_ZERO_XEND applied as the reference does */
  int storage;            /* hfm_dtype of inner fields and coefficients: F32, BF16, F16 */
  double tol;             /* relative residual ||b - A phi|| / ||b|| (default 1e-6) */
  int max_cycles;         /* NOT_CONVERGED after this many cycles / CG iterations */
  int cycles_per_launch;  /* cycles captured in one CUDA graph between host checks (default 4) */
  double inner_tol;       /* IR: an inner CG solve stops at max(inner_tol ||r0||, 0.3 tol ||b||) */
  int inner_max_cycles;   /* IR: iteration cap of one inner solve (default 200) */
  int options;             /* HFM_OPT_* bits (default 0) */
} hfm_mg_config;

/* options: run every level of the V-cycle as separate kernel launches, including the deep
 * levels that otherwise run as one fused kernel (one block per instance, fields in shared
 * memory, for SIGMA7 levels of at most 4096 cells) */
#define HFM_OPT_NO_FUSED_COARSE 1
/* options: run the first two pre-smoothing sweeps from zero as two passes instead of one
 * (by default the pointwise first sweep phi1 = omega f / diag is formed inside the second) */
#define HFM_OPT_NO_FUSED_PRE 2
/* options: the sawtooth cycle sweeps its coarsest level coarse_sweeps times from zero instead
 * of once (the serial run of notebooks/parallel_multigrid_advection_diffusion_3D.ipynb cell 15
 * sweeps its 2^3 level twice; Anisotropic_3d_Multigrid_7point.ipynb:424-432 once) */
#define HFM_OPT_SAWTOOTH_COARSE_SWEEPS 4
/* options: 16-bit SIGMA7 handles keep the per-cell conductivities on every level (by default
 * the levels the plane-marching kernels take - X >= 48, Y >= 16 - and the levels of more
 * than 4096 cells the register-queue kernels take (X a multiple of 4) also hold the FACE7
 * face arrays of their operator, formed from float32 conductivities on the fine level, and
 * run the face kernels there: each face rounded once to the storage type instead of forming
 * faces from rounded conductivities) */
#define HFM_OPT_NO_FACES 8
/* options: run the small end of a V-cycle - the level above the fused coarse cycle when the
 * plane-marching TMA kernels do not take it (X < 48), and the fused coarse cycle - as one
 * persistent kernel that walks an (instance, step, tile) work list of that level's sweeps,
 * its residual + restriction, the coarse cycle of every instance and the correction, with
 * per-instance dependency counters (handles of at least 8 slots, zero-guess V-cycles such
 * as a CG preconditioner's).  Off by default: the kernel holds every SM for a small amount
 * of work, and handles that share the GPU (the buckets of a server) lose more than the
 * launches it saves; by default the small end runs as separate launches. */
#define HFM_OPT_PERSISTENT 16
/* options: two Jacobi sweeps per pass over the FACE7 levels (temporal blocking): the
 * correction and first post-sweep with the last post-sweep when nu_post = 2, and the fused
 * first two pre-sweeps from zero with the residual and its restriction when nu_pre = 2; the
 * first sweep is recomputed on a one-cell ring around each tile and kept in shared memory.
 * Results are identical to one sweep per pass.  Off by default: the pass halves the bytes
 * but executes more instructions than two one-sweep passes, and the one-sweep face kernel
 * is already close to the copy bandwidth, so it measured slower. */
#define HFM_OPT_TEMPORAL 32

typedef struct {
  int active;       /* 1 while the slot is still iterating */
  int status;       /* hfm_status of the finished solve */
  int cycles;       /* cycles (or CG iterations) done */
  int outer;        /* float64 refinement steps done (IR) */
  double norm_b;    /* ||b||_2 */
  double rel_resid; /* last ||b - A phi|| / ||b|| */
} hfm_slot_stats;

typedef struct hfm_mg hfm_mg;

void hfm_mg_config_default(hfm_mg_config *cfg);
/* Device bytes a handle of this configuration holds (admission control). */
size_t hfm_mg_footprint_bytes(const hfm_mg_config *cfg, int Z, int Y, int X, int slots);
int hfm_mg_create(const hfm_mg_config *cfg, int Z, int Y, int X, int slots, hfm_mg **out);
int hfm_mg_destroy(hfm_mg *mg);
int hfm_mg_num_levels(const hfm_mg *mg);
int hfm_mg_level_shape(const hfm_mg *mg, int level, int *Z, int *Y, int *X);

/* Install the fine operator for one slot (slot = -1: every slot) and build the coefficient
 * hierarchy by the reference restriction (BGS_multigrid_v1.ipynb cell 38, lines 16-33).
 * SIGMA7 coefficient arrays hold one instance each ([Z][Y][X]); they are copied. */
int hfm_mg_set_operator(hfm_mg *mg, int slot, const hfm_operator *op, hfm_stream_t stream);
/* Copy rhs (and phi0, NULL = zero) into a slot, compute ||b|| and mark it active. */
int hfm_mg_load(hfm_mg *mg, int slot, const float *rhs, const float *phi0, hfm_stream_t stream);
/* Advance every active slot by `cycles` cycles (CUDA graph; slots that converge, fail or
 * hit max_cycles stop on the device and do no more work). */
int hfm_mg_run(hfm_mg *mg, int cycles, hfm_stream_t stream);
/* Copy per-slot statistics to host memory (synchronises `stream`). */
int hfm_mg_query(hfm_mg *mg, hfm_slot_stats *stats_host, hfm_stream_t stream);
/* Enqueue a copy of every slot's statistics into stats_host (pinned host memory, `slots`
 * entries) on `stream` without synchronising; read it after the stream reaches this point
 * (e.g. a CUDA event recorded after the call). */
int hfm_mg_query_async(hfm_mg *mg, hfm_slot_stats *stats_host, hfm_stream_t stream);
/* Copy a slot's current solution into phi_out (device, [Z][Y][X] float32). */
int hfm_mg_fetch(hfm_mg *mg, int slot, float *phi_out, hfm_stream_t stream);
/* Stop a slot (request cancelled); its memory can be reloaded at once. */
int hfm_mg_cancel(hfm_mg *mg, int slot, hfm_stream_t stream);
/* Convenience: load all slots from rhs/phi ([slots][Z][Y][X]), run to completion, fetch the
 * solutions into phi, fill stats_host (may be NULL).  Synchronises `stream`. */
int hfm_mg_solve(hfm_mg *mg, const float *rhs, float *phi, hfm_slot_stats *stats_host,
                 hfm_stream_t stream);
/* float64 right-hand side / initial guess (NULL = zero) and solution of a slot (accel = IR). */
int hfm_mg_load_f64(hfm_mg *mg, int slot, const double *rhs, const double *phi0,
                    hfm_stream_t stream);
int hfm_mg_fetch_f64(hfm_mg *mg, int slot, double *phi_out, hfm_stream_t stream);
/* Read an internal level buffer of a slot (0 = phi / w, 1 = rhs / r) for per-level checks. */
int hfm_mg_read_level(hfm_mg *mg, int slot, int level, int which, float *out,
                      hfm_stream_t stream);

/* ------------------------------------------------------------------ serving */
/* Continuous batching of anisotropic forward solves -div(sigma grad phi) = f (SIGMA7, cubic
 * grids of several edges) for hosts that are not Python: one resident multigrid handle
 * ("bucket") per edge with a number of slots, sized so the buckets fit an HBM budget
 * (admission by footprint: the largest buckets halve their slots until the sum fits).
 * hfm_serve_poll never blocks: it retires the finished slots of every bucket whose last
 * launch has completed (copying each solution to the request's output), admits queued
 * requests into free slots and relaunches the bucket (cycles_per_tick iterations as one
 * CUDA graph, each bucket on a stream of its own), so a request that arrives while others
 * run joins its bucket's next launch.  Each slot's arithmetic depends only on its own data,
 * so a result is the same alone and in the mix.  No counterpart in the reference (which
 * solves one problem per script run); the Python server (serving.py) runs the same loop.
 * A server is not thread-safe; use it from one host thread. */
typedef struct hfm_server hfm_server;
#define HFM_SERVE_MAX_EDGES 16
typedef struct {
  int n_edges;               /* cubic edges served, one bucket each */
  int edges[HFM_SERVE_MAX_EDGES];
  int slots;                 /* slots per bucket before admission by footprint (default 64) */
  double budget_bytes;       /* HBM budget of all buckets (default 120e9) */
  int cycles_per_tick;       /* iterations per bucket launch (default 4) */
  hfm_mg_config solver;      /* bucket solver; op_kind must be SIGMA7 and accel IR (default:
                                V(2,2) PCG in float64 refinement, bf16 storage, tol 1e-6,
                                inner_tol 1e-3, max_cycles 600) */
} hfm_serve_config;

typedef struct {
  int64_t ticket;            /* from hfm_serve_submit */
  int status;                /* HFM_OK, HFM_ERR_NOT_CONVERGED, HFM_ERR_NAN, HFM_ERR_TIMEOUT,
                                HFM_ERR_CANCELLED */
  int cycles;                /* CG iterations done */
  int outer;                 /* float64 refinement steps done */
  double rel_resid;          /* float64 relative residual ||b - A x|| / ||b|| */
} hfm_serve_result;

void hfm_serve_config_default(hfm_serve_config *cfg);
/* Create the buckets on the current device (edges 32, 48, 64, 96, 128 by default). */
int hfm_serve_create(const hfm_serve_config *cfg, hfm_server **out);
/* Slots the bucket of `edge` holds after admission by footprint. */
int hfm_serve_bucket_slots(const hfm_server *srv, int edge, int *slots);
/* Queue a request of edge n: conductivities sx, sy, sz and right-hand side f (device
 * float32, n^3 each, [z][y][x]) and the output x (device float64, n^3).  The caller owns
 * all five arrays: its writes to the inputs must be complete before the call (the buckets
 * read them on their own streams), and it keeps them valid and unchanged until the request
 * is reported by hfm_serve_poll; x is complete when reported.  Returns a ticket (increasing
 * from 0). */
int hfm_serve_submit(hfm_server *srv, int n, const float *sx, const float *sy, const float *sz,
                     const float *f, double *x, int64_t *ticket);
/* Advance every bucket without blocking; report up to `cap` finished requests in done[]
 * (their x is complete in device memory) and their number in *n_done. */
int hfm_serve_poll(hfm_server *srv, hfm_serve_result *done, int cap, int *n_done);
/* Cancel a queued or running request: it is reported by a later poll with
 * HFM_ERR_CANCELLED (x not written).  HFM_ERR_BAD_ARG for an unknown or finished ticket. */
int hfm_serve_cancel(hfm_server *srv, int64_t ticket);
/* Requests queued (waiting for a slot) and running (in a slot or copying out). */
int hfm_serve_pending(const hfm_server *srv, int *queued, int *running);
/* Wait for the device work of every bucket, then free the buckets (pending requests are
 * dropped unreported). */
int hfm_serve_destroy(hfm_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* HFM_H_ */
