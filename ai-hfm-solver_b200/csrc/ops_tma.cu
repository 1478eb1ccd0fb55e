// TMA-pipelined plane-marching stencil kernels for the large levels (X >= 64).
//
// A block owns a TY x TX tile of the (y, x) plane (8 x 64 for float32, 16 x 64 for 16-bit
// storage) and marches through a chunk of z
// planes.  For every plane one thread issues `cp.async.bulk.tensor.4d` loads of the plane's
// tiles into a shared-memory stage - phi with a one-row / HX-column halo, the three
// conductivities (sx with x halo, sy with y halo, sz), the right-hand side and, for the fused
// correction, the coarse correction tile - and one mbarrier per stage counts the bytes in.
// NS = 5 stages: planes z-1, z, z+1 are read while z+2, z+3 are in flight.  Tiles that reach
// past the grid (walls, the planes before 0 and after Z-1) are zero-filled by the TMA unit,
// which is exactly the SAME zero padding of the reference's Conv3D layers; the kernels then
// apply the wall rule for conductivities (ghost sigma = interior sigma) from the global
// coordinates.  Every TMA x coordinate is a multiple of 16 bytes (x0 - HX with x0 a multiple
// of 64 and HX = 16 / sizeof(T)); no store uses TMA.
//
// All waits are bounded: an mbarrier wait that does not complete within kMaxSpin polls sets
// the library's device timeout counter, drains the stages this block has in flight (again
// bounded) and returns.
#include <cuda.h>

#include <mutex>

#include "hfm_internal.cuh"

namespace hfm {

static __device__ int g_tma_timeouts;

namespace {

constexpr int TX = 64, NS = 5;
constexpr int kMaxSpin = 1 << 20;

enum { M_SMOOTH = FAST_SMOOTH, M_RESID = FAST_RESID, M_RESTRICT = FAST_RESTRICT };

// Stage layout for storage T; SIG: the stage carries the three conductivity tiles, CC: the
// coarse correction tile (stages of the other kernels are smaller, so more blocks fit).
template <class T, bool SIG = true, bool CC = true> struct Geo {
  // 8 rows x 64 columns per block for float32, 16 rows for 16-bit storage (same bytes per
  // stage); 16 threads per row, 4 consecutive x per thread
  static constexpr int TY = sizeof(T) == 4 ? 8 : 16;
  static constexpr int THREADS = 16 * TY;
  static constexpr int HX = 16 / (int)sizeof(T);
  static constexpr int PW = TX + 2 * HX;           // phi / sx tile width
  static constexpr int CW = TX / 2 + 2 * HX;       // coarse tile width
  static constexpr int PHI = (TY + 2) * PW;  // with the one-row y halo
  static constexpr int SXN = TY * PW;
  static constexpr int SYN = (TY + 2) * TX;
  static constexpr int SZN = TY * TX;
  static constexpr int FN = TY * TX;
  static constexpr int CCN = (TY / 2 + 2) * CW;
  static constexpr int al(int elems) { return ((elems * (int)sizeof(T) + 127) / 128) * 128; }
  // byte offsets inside a stage
  static constexpr int O_PHI = 0;
  static constexpr int O_SX = O_PHI + al(PHI);
  static constexpr int O_SY = O_SX + (SIG ? al(SXN) : 0);
  static constexpr int O_SZ = O_SY + (SIG ? al(SYN) : 0);
  static constexpr int O_F = O_SZ + (SIG ? al(SZN) : 0);
  static constexpr int O_CC = O_F + al(FN);
  static constexpr int STAGE = O_CC + (CC ? al(CCN) : 0);
};

template <class T> struct TmaArgs {
  CUtensorMap m_phi, m_sx, m_sy, m_sz, m_f, m_cc;
  DevOp op;
  T *out;
  T *coarse;
  double *partials;
  const int *active;
  int64_t stride, coarse_stride;
  int Z, Y, X, zc, tiles_x;
  float omega, corr_sign;
  int has_phi, has_f, has_sigma, zero_xend, zero_xend_out, top_copy;
  unsigned stage_bytes;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < kMaxSpin; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n"
        " selp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                         int b, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(b), "r"(bar)
      : "memory");
}

template <class T> __device__ __forceinline__ float sld(const T *p) { return St<T>::to(*p); }

// Four consecutive values from shared memory (16-byte float32 / 8-byte 16-bit load; every
// call site is aligned to four elements).
template <class T> struct V4;
template <> struct V4<float> {
  static __device__ __forceinline__ void get(const float *p, float (&v)[4]) {
    float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
};
template <> struct V4<__nv_bfloat16> {
  static __device__ __forceinline__ void get(const __nv_bfloat16 *p, float (&v)[4]) {
    uint2 u = *reinterpret_cast<const uint2 *>(p);
    float2 a = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&u.x));
    float2 b = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&u.y));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
};
template <> struct V4<__half> {
  static __device__ __forceinline__ void get(const __half *p, float (&v)[4]) {
    uint2 u = *reinterpret_cast<const uint2 *>(p);
    float2 a = __half22float2(*reinterpret_cast<__half2 *>(&u.x));
    float2 b = __half22float2(*reinterpret_cast<__half2 *>(&u.y));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
};

template <class T> __device__ __forceinline__ void gst4(T *p, const float (&v)[4]);
template <> __device__ __forceinline__ void gst4<float>(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <> __device__ __forceinline__ void gst4<__nv_bfloat16>(__nv_bfloat16 *p, const float (&v)[4]) {
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
  uint2 u;
  u.x = *reinterpret_cast<unsigned *>(&a);
  u.y = *reinterpret_cast<unsigned *>(&b);
  *reinterpret_cast<uint2 *>(p) = u;
}
template <> __device__ __forceinline__ void gst4<__half>(__half *p, const float (&v)[4]) {
  const float c0 = fminf(fmaxf(v[0], -65504.f), 65504.f), c1 = fminf(fmaxf(v[1], -65504.f), 65504.f);
  const float c2 = fminf(fmaxf(v[2], -65504.f), 65504.f), c3 = fminf(fmaxf(v[3], -65504.f), 65504.f);
  __half2 a = __floats2half2_rn(c0, c1), b = __floats2half2_rn(c2, c3);
  uint2 u;
  u.x = *reinterpret_cast<unsigned *>(&a);
  u.y = *reinterpret_cast<unsigned *>(&b);
  *reinterpret_cast<uint2 *>(p) = u;
}

// Issue the loads of plane p (may lie outside [0, Z): the TMA unit zero-fills) into `stage`.
template <class T, int CORR, bool SIG>
__device__ __forceinline__ void issue_plane(const TmaArgs<T> &a, char *stage, uint32_t bar, int p,
                                            int x0, int y0, int b) {
  using G = Geo<T, SIG, CORR != 0>;
  constexpr int TY = G::TY;
  (void)TY;
  mbar_expect(bar, a.stage_bytes);
  if (a.has_phi) tma_load(smem_u32(stage + G::O_PHI), &a.m_phi, x0 - G::HX, y0 - 1, p, b, bar);
  if (SIG) {
    tma_load(smem_u32(stage + G::O_SX), &a.m_sx, x0 - G::HX, y0, p, b, bar);
    tma_load(smem_u32(stage + G::O_SY), &a.m_sy, x0, y0 - 1, p, b, bar);
    tma_load(smem_u32(stage + G::O_SZ), &a.m_sz, x0, y0, p, b, bar);
  }
  if (a.has_f) tma_load(smem_u32(stage + G::O_F), &a.m_f, x0, y0, p, b, bar);
  if (CORR) tma_load(smem_u32(stage + G::O_CC), &a.m_cc, (x0 >> 1) - G::HX, (y0 >> 1) - 1, p >> 1, b, bar);
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

template <int KIND, class T, int MODE, int CORR>
__global__ void __launch_bounds__(Geo<T>::THREADS, sizeof(T) == 4 ? 3 : 2)
    k_tma(const __grid_constant__ TmaArgs<T> a) {
  constexpr bool SIG = KIND == HFM_OP_SIGMA7;
  using G = Geo<T, SIG, CORR != 0>;
  constexpr int TY = G::TY;
  extern __shared__ __align__(128) char smem[];
  __shared__ __align__(8) uint64_t bars[NS];
  const int64_t inst = blockIdx.z;
  if (a.active && !a.active[inst]) return;
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int tx = blockIdx.x % a.tiles_x, ty = blockIdx.x / a.tiles_x;
  const int x0 = tx * TX, y0 = ty * TY;
  const int z0 = blockIdx.y * a.zc, z1 = min(Z, z0 + a.zc);
  const int tid = threadIdx.x;
  const int r = tid >> 4, c = tid & 15;
  const int gx = x0 + 4 * c, gy = y0 + r;
  const bool valid = gx < X && gy < Y;
  const int b = (int)inst;

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(smem_u32(&bars[s]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  // planes z0-1 .. z1 are needed; plane p uses stage (p - z0 + 1) % NS
  const int p_first = z0 - 1, p_last = z1;
  int p_next = p_first;
  if (tid == 0) {
    for (; p_next <= p_last && p_next < p_first + NS; ++p_next) {
      const int q = p_next - p_first;
      issue_plane<T, CORR, SIG>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
    }
  }
  int p_waited = p_first - 1;  // last plane whose loads completed
  auto wait_plane = [&](int p) -> bool {
    const int q = p - p_first;
    const bool w = mbar_wait(smem_u32(&bars[q % NS]), (uint32_t)((q / NS) & 1));
    if (w) p_waited = p;
    return w;
  };
  auto stage_of = [&](int p) -> char * { return smem + ((p - p_first) % NS) * G::STAGE; };
  bool ok = wait_plane(z0 - 1);
  ok = wait_plane(z0) && ok;
  // a timeout is acted on by the whole block at once, so no thread is left at a barrier
  if (__syncthreads_or(!ok)) ok = false;

  const float s = a.op.scale;
  const float cz = a.op.c[0] * s, cy = a.op.c[1] * s, cx = a.op.c[2] * s;
  const float kz = a.op.k[0], ky = a.op.k[1], kx = a.op.k[2];
  const float dconst = 2.f * (kz + ky + kx);

  // phi' at tile coordinates (ry, rx) of plane stage st (global y0-1+ry, x0-HX+rx)
  auto phiv = [&](const char *st, int ry, int rx) -> float {
    const T *ph = reinterpret_cast<const T *>(st + G::O_PHI);
    float v = a.has_phi ? sld<T>(ph + ry * G::PW + rx) : 0.f;
    if (CORR) {
      const int yy = y0 - 1 + ry, xx = x0 - G::HX + rx;
      const int cyy = (yy >> 1) - ((y0 >> 1) - 1), cxx = (xx >> 1) - ((x0 >> 1) - G::HX);
      const T *cc = reinterpret_cast<const T *>(st + G::O_CC);
      v += a.corr_sign * sld<T>(cc + cyy * G::CW + cxx);
    }
    if (a.zero_xend && x0 - G::HX + rx == X - 1) v = 0.f;
    return v;
  };
  auto phi4 = [&](const char *st, int ry, float (&v)[4]) {
    const int rx = G::HX + 4 * c;
    if (!a.has_phi && !CORR) {
      v[0] = v[1] = v[2] = v[3] = 0.f;
    } else if (!CORR && !a.zero_xend) {
      V4<T>::get(reinterpret_cast<const T *>(st + G::O_PHI) + ry * G::PW + rx, v);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = phiv(st, ry, rx + e);
    }
  };

  // z-face coefficient below plane z0 (SIGMA7)
  float azlo[4] = {0.f, 0.f, 0.f, 0.f};
  if (KIND == HFM_OP_SIGMA7 && ok) {
    float szc[4], szm[4];
    V4<T>::get(reinterpret_cast<const T *>(stage_of(z0) + G::O_SZ) + r * TX + 4 * c, szc);
    V4<T>::get(reinterpret_cast<const T *>(stage_of(z0 - 1) + G::O_SZ) + r * TX + 4 * c, szm);
#pragma unroll
    for (int e = 0; e < 4; ++e) azlo[e] = z0 > 0 ? cz * 0.5f * (szc[e] + szm[e]) : cz * szc[e];
  }
  double acc = 0.0;
  float cpart[2] = {0.f, 0.f};

  for (int z = z0; z < z1 && ok; ++z) {
    const bool w = wait_plane(z + 1);
    if (__syncthreads_or(!w)) {
      ok = false;
      break;
    }
    const char *sm_ = stage_of(z - 1);
    const char *sc = stage_of(z);
    const char *sp = stage_of(z + 1);
    float res[4];
    float Ax[4], dg[4];
    float pc[4];
    phi4(sc, r + 1, pc);
    if (KIND == HFM_OP_K27) {
      const float *K = a.op.k;
#pragma unroll
      for (int e = 0; e < 4; ++e) Ax[e] = 0.f;
      const char *pl3[3] = {sm_, sc, sp};
#pragma unroll
      for (int aa = 0; aa < 3; ++aa) {
#pragma unroll
        for (int bb = 0; bb < 3; ++bb) {
          float row[6];
          row[0] = phiv(pl3[aa], r + bb, G::HX + 4 * c - 1);
          float m4[4];
          phi4(pl3[aa], r + bb, m4);
          row[1] = m4[0]; row[2] = m4[1]; row[3] = m4[2]; row[4] = m4[3];
          row[5] = phiv(pl3[aa], r + bb, G::HX + 4 * c + 4);
          const float k0 = K[9 * aa + 3 * bb], k1 = K[9 * aa + 3 * bb + 1], k2 = K[9 * aa + 3 * bb + 2];
#pragma unroll
          for (int e = 0; e < 4; ++e) Ax[e] += k0 * row[e] + k1 * row[e + 1] + k2 * row[e + 2];
        }
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) dg[e] = K[13];
    } else {
      float pym[4], pyp[4], pzm[4], pzp[4];
      phi4(sc, r, pym);
      phi4(sc, r + 2, pyp);
      phi4(sm_, r + 1, pzm);
      phi4(sp, r + 1, pzp);
      const float pl = phiv(sc, r + 1, G::HX + 4 * c - 1);
      const float pr = phiv(sc, r + 1, G::HX + 4 * c + 4);
      if (KIND == HFM_OP_CONST7) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float xm = e == 0 ? pl : pc[e - 1];
          const float xp = e == 3 ? pr : pc[e + 1];
          Ax[e] = dconst * pc[e] - kz * (pzm[e] + pzp[e]) - ky * (pym[e] + pyp[e]) - kx * (xm + xp);
          dg[e] = dconst;
        }
      } else {
        const T *SX = reinterpret_cast<const T *>(sc + G::O_SX) + r * G::PW + G::HX + 4 * c;
        const T *SY = reinterpret_cast<const T *>(sc + G::O_SY) + (r + 1) * TX + 4 * c;
        float sxc[4], syc[4], sym[4], syp[4], szc[4], szp[4];
        V4<T>::get(SX, sxc);
        V4<T>::get(SY, syc);
        V4<T>::get(SY - TX, sym);
        V4<T>::get(SY + TX, syp);
        V4<T>::get(reinterpret_cast<const T *>(sc + G::O_SZ) + r * TX + 4 * c, szc);
        V4<T>::get(reinterpret_cast<const T *>(sp + G::O_SZ) + r * TX + 4 * c, szp);
        const float sxl = gx > 0 ? sld<T>(SX - 1) : sxc[0];
        const float sxr = gx + 4 < X ? sld<T>(SX + 4) : sxc[3];
        const bool ylo = gy > 0, yhi = gy + 1 < Y, zhi = z + 1 < Z;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float sxm = e == 0 ? sxl : sxc[e - 1];
          const float sxp = e == 3 ? sxr : sxc[e + 1];
          const float axm = cx * 0.5f * (sxc[e] + sxm);
          const float axp = cx * 0.5f * (sxc[e] + sxp);
          const float aym = cy * 0.5f * (syc[e] + (ylo ? sym[e] : syc[e]));
          const float ayp = cy * 0.5f * (syc[e] + (yhi ? syp[e] : syc[e]));
          const float azhi = cz * 0.5f * (szc[e] + (zhi ? szp[e] : szc[e]));
          const float xm = e == 0 ? pl : pc[e - 1];
          const float xp = e == 3 ? pr : pc[e + 1];
          const float p = pc[e];
          Ax[e] = axm * (p - xm) + axp * (p - xp) + aym * (p - pym[e]) + ayp * (p - pyp[e]) +
                  azlo[e] * (p - pzm[e]) + azhi * (p - pzp[e]);
          dg[e] = axm + axp + aym + ayp + azlo[e] + azhi;
          azlo[e] = azhi;
        }
      }
    }
    float f[4] = {0.f, 0.f, 0.f, 0.f};
    if (a.has_f) V4<T>::get(reinterpret_cast<const T *>(sc + G::O_F) + r * TX + 4 * c, f);
    if (MODE == M_SMOOTH) {
#pragma unroll
      for (int e = 0; e < 4; ++e) res[e] = pc[e] + a.omega * __fdividef(f[e] - Ax[e], dg[e]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) res[e] = Ax[e] - f[e];
      if (a.zero_xend_out && gx + 4 == X) res[3] = 0.f;
      if (valid) {
#pragma unroll
        for (int e = 0; e < 4; ++e) acc += (double)res[e] * res[e];
      }
    }
    const int64_t off = inst * a.stride + ((int64_t)z * Y + gy) * X + gx;
    if (valid && a.out) {
      if (MODE == M_SMOOTH && a.top_copy && z == 1) gst4<T>(a.out + inst * a.stride + (int64_t)gy * X + gx, res);
      if (!(MODE == M_SMOOTH && a.top_copy && z == 0 && Z > 1)) gst4<T>(a.out + off, res);
    }
    if (MODE == M_RESTRICT) {
      // x pairs in the vector, y pairs with the lane 16 above (row r + 1), z pairs over planes
      float p0 = res[0] + res[1], p1 = res[2] + res[3];
      p0 += __shfl_down_sync(0xffffffffu, p0, 16);
      p1 += __shfl_down_sync(0xffffffffu, p1, 16);
      cpart[0] += 0.125f * p0;
      cpart[1] += 0.125f * p1;
      if (z & 1) {
        if (valid && !(r & 1)) {
          T *cp = a.coarse + inst * a.coarse_stride +
                  ((int64_t)(z >> 1) * (Y >> 1) + (gy >> 1)) * (X >> 1) + (gx >> 1);
          cp[0] = St<T>::from(cpart[0]);
          cp[1] = St<T>::from(cpart[1]);
        }
        cpart[0] = cpart[1] = 0.f;
      }
    }
    __syncthreads();  // every thread is done with plane z-1's stage
    if (tid == 0 && p_next <= p_last) {
      const int q = p_next - p_first;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_plane<T, CORR, SIG>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
      ++p_next;
    }
  }
  if (!ok) {
    if (tid == 0) atomicAdd(&g_tma_timeouts, 1);
    // drain: wait (bounded) for the planes whose loads are still in flight, so that no
    // copy lands in shared memory after this block has exited; thread 0 issued them all
    if (tid == 0)
      for (int p = p_waited + 1; p < p_next; ++p) wait_plane(p);
    return;
  }
  if (MODE != M_SMOOTH && a.partials) {
    double t = block_sum(acc);
    if (tid == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

template <class T> CUtensorMapDataType tmap_dtype();
template <> CUtensorMapDataType tmap_dtype<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> CUtensorMapDataType tmap_dtype<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }
template <> CUtensorMapDataType tmap_dtype<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }

template <class T>
int make_map(CUtensorMap *m, const void *ptr, int X, int Y, int Z, int B, int64_t inst_stride,
             int bw, int bh) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(HFM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t es = sizeof(T);
  cuuint64_t dims[4] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z, (cuuint64_t)B};
  cuuint64_t strides[3] = {(cuuint64_t)X * es, (cuuint64_t)X * Y * es, (cuuint64_t)inst_stride * es};
  cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(m, tmap_dtype<T>(), 4, const_cast<void *>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(HFM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return HFM_OK;
}

template <int KIND, class T, int MODE, int CORR>
int go(const TmaArgs<T> &a, dim3 grid, cudaStream_t s) {
  using G = Geo<T, KIND == HFM_OP_SIGMA7, CORR != 0>;
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  const int smem = NS * G::STAGE;
  std::call_once(once, [&] {
    attr_err = cudaFuncSetAttribute(k_tma<KIND, T, MODE, CORR>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
  if (attr_err != cudaSuccess) return cuda_status(attr_err, "cudaFuncSetAttribute(k_tma)");
  k_tma<KIND, T, MODE, CORR><<<grid, G::THREADS, smem, s>>>(a);
  HFM_CHECK_LAUNCH("k_tma");
  return HFM_OK;
}

}  // namespace

bool tma_eligible(int kind, Grid3 g, int mode, const void *corr, int corr_coarse, int es) {
  if (kind != HFM_OP_CONST7 && kind != HFM_OP_SIGMA7 && kind != HFM_OP_K27) return false;
  if (g.X < TX || g.Y < (es == 4 ? 8 : 16)) return false;
  if ((g.X * es) % 16) return false;  // tensor-map strides are multiples of 16 bytes
  if (corr && !corr_coarse) return false;
  if (corr && ((g.X / 2) * es) % 16) return false;
  if (corr && ((g.Y | g.Z) & 1)) return false;
  if (mode == M_RESTRICT && (kind == HFM_OP_K27 || (g.Y & 1) || (g.Z & 1))) return false;
  if (mode != M_SMOOTH && corr) return false;
  return true;
}

template <class T>
int tma_launch(int kind, int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs, T *out,
               T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g, float omega,
               unsigned flags, const int *active, double *partials, int *nblk_out,
               cudaStream_t s) {
  using G = Geo<T>;  // tile extents (identical for every stage layout)
  constexpr int TY = G::TY;
  TmaArgs<T> a;
  memset(&a, 0, sizeof(a));
  int st;
  // phi == null (zero guess) still needs a map: point it at the output, whose loads are
  // never used because the kernel is only called with a base; see below.
  // a zero initial guess (phi.base == NULL) loads no phi tile and reads phi = 0
  a.has_phi = phi.base != nullptr;
  if (a.has_phi &&
      (st = make_map<T>(&a.m_phi, phi.base, g.X, g.Y, g.Z, B, phi.base_stride, G::PW, TY + 2)))
    return st;
  a.has_sigma = kind == HFM_OP_SIGMA7;
  if (a.has_sigma) {
    if ((st = make_map<T>(&a.m_sx, op.coef[0], g.X, g.Y, g.Z, B, op.coef_stride, G::PW, TY))) return st;
    if ((st = make_map<T>(&a.m_sy, op.coef[1], g.X, g.Y, g.Z, B, op.coef_stride, TX, TY + 2))) return st;
    if ((st = make_map<T>(&a.m_sz, op.coef[2], g.X, g.Y, g.Z, B, op.coef_stride, TX, TY))) return st;
  }
  a.has_f = rhs != nullptr;
  if (a.has_f && (st = make_map<T>(&a.m_f, rhs, g.X, g.Y, g.Z, B, stride, TX, TY))) return st;
  const int corr = phi.corr ? 1 : 0;
  if (corr && (st = make_map<T>(&a.m_cc, phi.corr, g.X / 2, g.Y / 2, g.Z / 2, B, phi.corr_stride,
                                G::CW, TY / 2 + 2)))
    return st;
  unsigned bytes = a.has_phi ? (unsigned)(G::PHI * sizeof(T)) : 0u;
  if (a.has_sigma) bytes += (unsigned)((G::SXN + G::SYN + G::SZN) * sizeof(T));
  if (a.has_f) bytes += (unsigned)(G::FN * sizeof(T));
  if (corr) bytes += (unsigned)(G::CCN * sizeof(T));
  a.stage_bytes = bytes;
  a.op = op;
  a.out = out;
  a.coarse = coarse;
  a.partials = partials;
  a.active = active;
  a.stride = stride;
  a.coarse_stride = coarse_stride;
  a.Z = g.Z;
  a.Y = g.Y;
  a.X = g.X;
  a.omega = omega;
  a.corr_sign = phi.corr_sign;
  a.zero_xend = phi.zero_xend ? 1 : 0;
  a.zero_xend_out = (mode != M_SMOOTH && (flags & HFM_FLAG_ZERO_XEND)) ? 1 : 0;
  a.top_copy = (mode == M_SMOOTH && (flags & HFM_FLAG_TOP_COPY)) ? 1 : 0;
  a.tiles_x = (g.X + TX - 1) / TX;
  const int tiles = a.tiles_x * ((g.Y + TY - 1) / TY);
  // z chunks: about 3 resident blocks per SM and four waves; chunks of at least 2 planes
  const int64_t slots = (int64_t)sm_count() * 3 * 4;
  int64_t chunks = (slots + (int64_t)tiles * B - 1) / ((int64_t)tiles * B);
  int zc = (int)((g.Z + chunks - 1) / chunks);
  if (zc < 2) zc = 2;
  if (zc & 1) ++zc;
  if (zc > g.Z) zc = g.Z;
  a.zc = zc;
  dim3 grid(tiles, (g.Z + zc - 1) / zc, B);
  if (nblk_out) *nblk_out = grid.x * grid.y;
#define HFM_TMA_GO(KIND, MODE, CORR) return go<KIND, T, MODE, CORR>(a, grid, s)
#define HFM_TMA_MODES(KIND)                                              \
  if (mode == M_SMOOTH) {                                                \
    if (corr) HFM_TMA_GO(KIND, M_SMOOTH, 1);                             \
    HFM_TMA_GO(KIND, M_SMOOTH, 0);                                       \
  } else if (mode == M_RESID) {                                          \
    HFM_TMA_GO(KIND, M_RESID, 0);                                        \
  }
  if (kind == HFM_OP_SIGMA7) {
    HFM_TMA_MODES(HFM_OP_SIGMA7)
    HFM_TMA_GO(HFM_OP_SIGMA7, M_RESTRICT, 0);
  } else if (kind == HFM_OP_CONST7) {
    HFM_TMA_MODES(HFM_OP_CONST7)
    HFM_TMA_GO(HFM_OP_CONST7, M_RESTRICT, 0);
  } else {
    HFM_TMA_MODES(HFM_OP_K27)
  }
#undef HFM_TMA_MODES
#undef HFM_TMA_GO
  return fail(HFM_ERR_UNSUPPORTED, "tma path: unsupported combination");
}

#define HFM_TMA_INST(T)                                                                       \
  template int tma_launch<T>(int, int, const DevOp &, const PhiSrc<T> &, const T *, T *, T *, \
                             int64_t, int64_t, int, Grid3, float, unsigned, const int *,      \
                             double *, int *, cudaStream_t);
HFM_TMA_INST(float)
HFM_TMA_INST(__nv_bfloat16)
HFM_TMA_INST(__half)

}  // namespace hfm

extern "C" int hfm_device_timeouts(int *count, int reset) {
  if (!count) return hfm::fail(HFM_ERR_BAD_ARG, "NULL");
  HFM_CUDA(cudaMemcpyFromSymbol(count, hfm::g_tma_timeouts, sizeof(int)));
  if (reset) {
    int zero = 0;
    HFM_CUDA(cudaMemcpyToSymbol(hfm::g_tma_timeouts, &zero, sizeof(int)));
  }
  return HFM_OK;
}
