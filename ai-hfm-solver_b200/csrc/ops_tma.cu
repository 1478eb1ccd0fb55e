// TMA-pipelined plane-marching stencil kernels for the large levels (X >= 48).
//
// A block owns a TY x TX tile of the (y, x) plane (8 x 64 for float32, 16 x 64 for 16-bit
// storage) and marches through a chunk of z
// planes.  For every plane one thread issues `cp.async.bulk.tensor.4d` loads of the plane's
// tiles into a shared-memory stage - phi with a one-row / HX-column halo, the three
// conductivities (sx with x halo, sy with y halo, sz), the right-hand side and, for the fused
// correction, the coarse correction tile - and one mbarrier per stage counts the bytes in.
// NS = 5 stages for float32 (planes z-1, z, z+1 are read while z+2, z+3 are in flight) and 4
// for 16-bit storage, whose kernels are issue-bound rather than bandwidth-bound: the smaller
// ring lets four blocks share an SM instead of three.  Tiles that reach
// past the grid (walls, the planes before 0 and after Z-1) are zero-filled by the TMA unit,
// which is exactly the SAME zero padding of the reference's Conv3D layers; the kernels then
// apply the wall rule for conductivities (ghost sigma = interior sigma) from the global
// coordinates.  Every TMA x coordinate is a multiple of 16 bytes (x0 - HX with x0 a multiple
// of 64 and HX = 16 / sizeof(T)); no store uses TMA.
//
// All waits are bounded: a plane wait that does not complete within the wait budget (2^20
// polls unless hfm_set_wait_budget lowers it) counts one timeout in the library's device
// counters; the block then drains the copies it has issued (waits of up to 2^20 polls each)
// and returns.  When every drain wait completes, no copy lands in shared memory after the
// block has exited; a drain wait that itself expires is counted separately (the block exits
// with copies possibly still in flight, and the context is suspect).  The multigrid handle's
// check kernels read both counters and mark their slots HFM_ERR_TIMEOUT while either is
// non-zero.
#include <cuda.h>

#include <atomic>
#include <mutex>
#include <type_traits>
#include <vector>

#include "hfm_internal.cuh"

namespace hfm {

// [0]: plane waits that expired, [1]: drain waits that expired (see the file comment)
static __device__ int g_tma_wait_fail[2];
static std::atomic<int> g_wait_budget{1 << 20};

namespace {

constexpr int TX = 64;
constexpr int kMaxSpin = 1 << 20;

// M_PRE2: the first two Jacobi sweeps from a zero iterate in one pass.  The first sweep is
// pointwise, phi1 = omega f / diag, so the kernel loads f and 1/diag with the phi halos and
// forms phi1 on the fly where the second sweep reads phi.
enum { M_SMOOTH = FAST_SMOOTH, M_RESID = FAST_RESID, M_RESTRICT = FAST_RESTRICT, M_PRE2 = 3 };

// Stage layout for storage T; SIG: the stage carries the three conductivity tiles, CC: the
// coarse correction tile (stages of the other kernels are smaller, so more blocks fit).
template <class T, bool SIG = true, bool CC = true, bool DS = false> struct Geo {
  // 8 rows x 64 columns per block for float32, 16 rows for 16-bit storage (same bytes per
  // stage); a thread owns 16 bytes of x: 4 float32 / 8 16-bit values, so 16 / 8 threads per
  // row and 128 threads per block either way
  static constexpr int TY = sizeof(T) == 4 ? 8 : 16;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int TPR = TX / VEC;
  static constexpr int THREADS = TPR * TY;
  // 4 stages and 4 resident blocks per SM for both: float32 with 5 stages fitted 3 blocks
  // (12 warps per SM), and ncu showed the sweep latency-bound there (issue slots 42 % busy,
  // shared-memory and dependency stalls), not bandwidth-bound
  static constexpr int NS = 4;    // pipeline stages
  static constexpr int MINB = 4;  // resident blocks per SM
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
  static constexpr int O_DS = O_CC + (CC ? al(CCN) : 0);  // 1 / diag with the phi halos (M_PRE2)
  static constexpr int STAGE = O_DS + (DS ? al(PHI) : 0);
};

template <class T> struct TmaArgs {
  CUtensorMap m_phi, m_sx, m_sy, m_sz, m_f, m_cc, m_ds;
  DevOp op;
  T *out;
  T *coarse;
  double *partials;
  const int *active;
  int64_t stride, coarse_stride;
  int Z, Y, X, zc, tiles_x;
  float omega, corr_sign;
  int has_phi, has_f, has_sigma, zero_xend, zero_xend_out, top_copy, dot_phi, dot_rhs;
  unsigned stage_bytes;
  int wait_budget;  // polls of a plane wait before the block gives up (hfm_set_wait_budget)
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

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int budget) {
  for (int i = 0; i < budget; ++i) {
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

// Two 16-bit values packed in 32 bits <-> float2.
template <class T> __device__ __forceinline__ float2 cvt2(unsigned u);
template <> __device__ __forceinline__ float2 cvt2<__nv_bfloat16>(unsigned u) {
  return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&u));
}
template <> __device__ __forceinline__ float2 cvt2<__half>(unsigned u) {
  return __half22float2(*reinterpret_cast<__half2 *>(&u));
}
template <class T> __device__ __forceinline__ unsigned pack2(float x, float y);
template <> __device__ __forceinline__ unsigned pack2<__nv_bfloat16>(float x, float y) {
  __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
  return *reinterpret_cast<unsigned *>(&h);
}
template <> __device__ __forceinline__ unsigned pack2<__half>(float x, float y) {
  // saturating, as St<__half>::from
  __half2 h = __floats2half2_rn(fminf(fmaxf(x, -65504.f), 65504.f), fminf(fmaxf(y, -65504.f), 65504.f));
  return *reinterpret_cast<unsigned *>(&h);
}

// N consecutive values from shared memory as float (one 16-, 8- or 4-byte load; every call
// site is aligned to N elements).
template <class T, int N> __device__ __forceinline__ void vld(const T *p, float (&v)[N]) {
  if constexpr (sizeof(T) == 4) {
    if constexpr (N == 4) {
      const float4 a = *reinterpret_cast<const float4 *>(p);
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
      static_assert(N == 2, "float32 vectors are 2 or 4 wide");
      const float2 a = *reinterpret_cast<const float2 *>(p);
      v[0] = a.x; v[1] = a.y;
    }
  } else if constexpr (N == 8) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const float2 a = cvt2<T>(u.x), b = cvt2<T>(u.y), c = cvt2<T>(u.z), d = cvt2<T>(u.w);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y; v[6] = d.x; v[7] = d.y;
  } else {
    static_assert(N == 4, "16-bit vectors are 4 or 8 wide");
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    const float2 a = cvt2<T>(u.x), b = cvt2<T>(u.y);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}

// N consecutive values to global memory (16-byte store; 16-byte aligned, see tma_eligible).
template <class T, int N> __device__ __forceinline__ void vst(T *p, const float (&v)[N]) {
  if constexpr (sizeof(T) == 4) {
    static_assert(N == 4, "float32 stores are 4 wide");
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    static_assert(N == 8, "16-bit stores are 8 wide");
    uint4 u;
    u.x = pack2<T>(v[0], v[1]);
    u.y = pack2<T>(v[2], v[3]);
    u.z = pack2<T>(v[4], v[5]);
    u.w = pack2<T>(v[6], v[7]);
    *reinterpret_cast<uint4 *>(p) = u;
  }
}

// Issue the loads of plane p (may lie outside [0, Z): the TMA unit zero-fills) into `stage`.
template <class T, int CORR, bool SIG, bool DS = false>
__device__ __forceinline__ void issue_plane(const TmaArgs<T> &a, char *stage, uint32_t bar, int p,
                                            int x0, int y0, int b) {
  using G = Geo<T, SIG, CORR != 0, DS>;
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
  if (DS) tma_load(smem_u32(stage + G::O_DS), &a.m_ds, x0 - G::HX, y0 - 1, p, b, bar);
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
__global__ void __launch_bounds__(Geo<T>::THREADS, Geo<T>::MINB) k_tma(const __grid_constant__ TmaArgs<T> a) {
  constexpr bool SIG = KIND == HFM_OP_SIGMA7;
  constexpr bool PRE2 = MODE == M_PRE2;
  using G = Geo<T, SIG, CORR != 0, PRE2>;
  constexpr int TY = G::TY, V = G::VEC, NS = G::NS;
  extern __shared__ __align__(128) char smem[];
  __shared__ __align__(8) uint64_t bars[NS];
  const int64_t inst = blockIdx.z;
  if (a.active && !a.active[inst]) return;
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int tx = blockIdx.x % a.tiles_x, ty = blockIdx.x / a.tiles_x;
  const int x0 = tx * TX, y0 = ty * TY;
  const int z0 = blockIdx.y * a.zc, z1 = min(Z, z0 + a.zc);
  const int tid = threadIdx.x;
  const int r = tid / G::TPR, c = tid % G::TPR;
  const int gx = x0 + V * c, gy = y0 + r;
  // X is a multiple of V (16-byte rows), so a thread's vector is wholly inside or outside
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
      issue_plane<T, CORR, SIG, PRE2>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
    }
  }
  int p_waited = p_first - 1;  // last plane whose loads completed
  auto wait_plane = [&](int p, int budget) -> bool {
    const int q = p - p_first;
    const bool w = mbar_wait(smem_u32(&bars[q % NS]), (uint32_t)((q / NS) & 1), budget);
    if (w) p_waited = p;
    return w;
  };
  auto stage_of = [&](int p) -> char * { return smem + ((p - p_first) % NS) * G::STAGE; };
  bool ok = wait_plane(z0 - 1, a.wait_budget);
  ok = wait_plane(z0, a.wait_budget) && ok;
  // a timeout is acted on by the whole block at once, so no thread is left at a barrier
  if (__syncthreads_or(!ok)) ok = false;

  const float s = a.op.scale;
  const float cz = a.op.c[0] * s, cy = a.op.c[1] * s, cx = a.op.c[2] * s;
  const float hz = cz * 0.5f, hy = cy * 0.5f, hx = cx * 0.5f;
  const float kz = a.op.k[0], ky = a.op.k[1], kx = a.op.k[2];
  const float dconst = 2.f * (kz + ky + kx);

  // phi' at tile coordinates (ry, rx) of plane stage st (global y0-1+ry, x0-HX+rx)
  auto phiv = [&](const char *st, int ry, int rx) -> float {
    const T *ph = reinterpret_cast<const T *>(st + G::O_PHI);
    if (PRE2)  // phi1 = omega f / diag
      return a.omega * sld<T>(ph + ry * G::PW + rx) *
             sld<T>(reinterpret_cast<const T *>(st + G::O_DS) + ry * G::PW + rx);
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
  // the thread's V values of phi' on tile row ry
  auto phiV = [&](const char *st, int ry, float (&v)[V]) {
    const int rx = G::HX + V * c;
    if (PRE2) {
      float d[V];
      vld<T, V>(reinterpret_cast<const T *>(st + G::O_PHI) + ry * G::PW + rx, v);
      vld<T, V>(reinterpret_cast<const T *>(st + G::O_DS) + ry * G::PW + rx, d);
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] = a.omega * v[e] * d[e];
      return;
    }
    if (a.has_phi) {
      vld<T, V>(reinterpret_cast<const T *>(st + G::O_PHI) + ry * G::PW + rx, v);
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] = 0.f;
    }
    if (CORR) {
      // coarse cells of x pairs: tile column (gx >> 1) - ((x0 >> 1) - HX) = V/2 c + HX
      const int cyy = ((y0 - 1 + ry) >> 1) - ((y0 >> 1) - 1);
      float cv[V / 2];
      vld<T, V / 2>(reinterpret_cast<const T *>(st + G::O_CC) + cyy * G::CW + (V / 2) * c + G::HX, cv);
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] += a.corr_sign * cv[e >> 1];
    }
    if (a.zero_xend && gx + V == X) v[V - 1] = 0.f;
  };

  // z-face coefficient below plane z0 (SIGMA7)
  float azlo[V];
#pragma unroll
  for (int e = 0; e < V; ++e) azlo[e] = 0.f;
  if (KIND == HFM_OP_SIGMA7 && ok) {
    float szc[V], szm[V];
    vld<T, V>(reinterpret_cast<const T *>(stage_of(z0) + G::O_SZ) + r * TX + V * c, szc);
    vld<T, V>(reinterpret_cast<const T *>(stage_of(z0 - 1) + G::O_SZ) + r * TX + V * c, szm);
#pragma unroll
    for (int e = 0; e < V; ++e) azlo[e] = z0 > 0 ? hz * (szc[e] + szm[e]) : cz * szc[e];
  }
  double acc = 0.0;
  float cpart[V / 2];
#pragma unroll
  for (int e = 0; e < V / 2; ++e) cpart[e] = 0.f;

  bool mine = true;  // this thread's latest plane wait completed
  for (int z = z0; z < z1 && ok; ++z) {
    // One barrier per plane.  It certifies that every thread is done with plane z-2, whose
    // stage thread 0 then refills before anyone waits for plane z+1 (so two planes stay in
    // flight), and it publishes the outcome of the previous waits: a thread whose wait ran
    // out computed one plane from an incomplete stage, and the whole block stops here.
    if (__syncthreads_or(!mine)) {
      ok = false;
      break;
    }
    if (tid == 0 && z > z0 && p_next <= p_last) {
      const int q = p_next - p_first;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_plane<T, CORR, SIG, PRE2>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
      ++p_next;
    }
    mine = wait_plane(z + 1, a.wait_budget);
    const char *sm_ = stage_of(z - 1);
    const char *sc = stage_of(z);
    const char *sp = stage_of(z + 1);
    float res[V];
    float Ax[V], dg[V];
    float pc[V];
    phiV(sc, r + 1, pc);
    if (KIND == HFM_OP_K27) {
      const float *K = a.op.k;
#pragma unroll
      for (int e = 0; e < V; ++e) Ax[e] = 0.f;
      const char *pl3[3] = {sm_, sc, sp};
#pragma unroll
      for (int aa = 0; aa < 3; ++aa) {
#pragma unroll
        for (int bb = 0; bb < 3; ++bb) {
          float row[V + 2], mid[V];
          row[0] = phiv(pl3[aa], r + bb, G::HX + V * c - 1);
          phiV(pl3[aa], r + bb, mid);
#pragma unroll
          for (int e = 0; e < V; ++e) row[e + 1] = mid[e];
          row[V + 1] = phiv(pl3[aa], r + bb, G::HX + V * c + V);
          const float k0 = K[9 * aa + 3 * bb], k1 = K[9 * aa + 3 * bb + 1], k2 = K[9 * aa + 3 * bb + 2];
#pragma unroll
          for (int e = 0; e < V; ++e) Ax[e] += k0 * row[e] + k1 * row[e + 1] + k2 * row[e + 2];
        }
      }
#pragma unroll
      for (int e = 0; e < V; ++e) dg[e] = K[13];
    } else {
      float pym[V], pyp[V], pzm[V], pzp[V];
      phiV(sc, r, pym);
      phiV(sc, r + 2, pyp);
      phiV(sm_, r + 1, pzm);
      phiV(sp, r + 1, pzp);
      const float pl = phiv(sc, r + 1, G::HX + V * c - 1);
      const float pr = phiv(sc, r + 1, G::HX + V * c + V);
      if (KIND == HFM_OP_CONST7) {
#pragma unroll
        for (int e = 0; e < V; ++e) {
          const float xm = e == 0 ? pl : pc[e - 1];
          const float xp = e == V - 1 ? pr : pc[e + 1];
          Ax[e] = dconst * pc[e] - kz * (pzm[e] + pzp[e]) - ky * (pym[e] + pyp[e]) - kx * (xm + xp);
          dg[e] = dconst;
        }
      } else {
        const T *SX = reinterpret_cast<const T *>(sc + G::O_SX) + r * G::PW + G::HX + V * c;
        const T *SY = reinterpret_cast<const T *>(sc + G::O_SY) + (r + 1) * TX + V * c;
        const T *SZ = reinterpret_cast<const T *>(sc + G::O_SZ) + r * TX + V * c;
        // at a wall the ghost conductivity is the cell's own: read the cell's row instead,
        // (s + s) / 2 = s exactly
        const bool ylo = gy > 0, yhi = gy + 1 < Y, zhi = z + 1 < Z;
        float sxc[V], syc[V], sym[V], syp[V], szc[V], szp[V];
        vld<T, V>(SX, sxc);
        vld<T, V>(SY, syc);
        vld<T, V>(ylo ? SY - TX : SY, sym);
        vld<T, V>(yhi ? SY + TX : SY, syp);
        vld<T, V>(SZ, szc);
        vld<T, V>(zhi ? reinterpret_cast<const T *>(sp + G::O_SZ) + r * TX + V * c : SZ, szp);
        // the V + 1 x faces of the thread's cells (wall faces: c_x sigma of the cell)
        float ax[V + 1];
        ax[0] = gx > 0 ? hx * (sxc[0] + sld<T>(SX - 1)) : cx * sxc[0];
        ax[V] = gx + V < X ? hx * (sxc[V - 1] + sld<T>(SX + V)) : cx * sxc[V - 1];
#pragma unroll
        for (int e = 1; e < V; ++e) ax[e] = hx * (sxc[e] + sxc[e - 1]);
        // cells in pairs on the packed float32 pipe (fma / add / mul .f32x2); p - q is
        // formed as fma(q, -1, p), which is exact up to the one rounding of the subtraction
        const float2 m1 = make_float2(-1.f, -1.f), hy2 = make_float2(hy, hy), hz2 = make_float2(hz, hz);
#pragma unroll
        for (int e = 0; e < V; e += 2) {
          const float2 p = make_float2(pc[e], pc[e + 1]);
          const float2 aym = __fmul2_rn(hy2, __fadd2_rn(make_float2(syc[e], syc[e + 1]), make_float2(sym[e], sym[e + 1])));
          const float2 ayp = __fmul2_rn(hy2, __fadd2_rn(make_float2(syc[e], syc[e + 1]), make_float2(syp[e], syp[e + 1])));
          const float2 azh = __fmul2_rn(hz2, __fadd2_rn(make_float2(szc[e], szc[e + 1]), make_float2(szp[e], szp[e + 1])));
          const float2 azl = make_float2(azlo[e], azlo[e + 1]);
          const float2 axm = make_float2(ax[e], ax[e + 1]), axp = make_float2(ax[e + 1], ax[e + 2]);
          const float2 xm = make_float2(e == 0 ? pl : pc[e - 1], pc[e]);
          const float2 xp = make_float2(pc[e + 1], e + 2 == V ? pr : pc[e + 2]);
          float2 A = __fmul2_rn(axm, __ffma2_rn(xm, m1, p));
          A = __ffma2_rn(axp, __ffma2_rn(xp, m1, p), A);
          A = __ffma2_rn(aym, __ffma2_rn(make_float2(pym[e], pym[e + 1]), m1, p), A);
          A = __ffma2_rn(ayp, __ffma2_rn(make_float2(pyp[e], pyp[e + 1]), m1, p), A);
          A = __ffma2_rn(azl, __ffma2_rn(make_float2(pzm[e], pzm[e + 1]), m1, p), A);
          A = __ffma2_rn(azh, __ffma2_rn(make_float2(pzp[e], pzp[e + 1]), m1, p), A);
          const float2 d = __fadd2_rn(__fadd2_rn(__fadd2_rn(axm, axp), __fadd2_rn(aym, ayp)),
                                      __fadd2_rn(azl, azh));
          Ax[e] = A.x; Ax[e + 1] = A.y;
          dg[e] = d.x; dg[e + 1] = d.y;
          azlo[e] = azh.x; azlo[e + 1] = azh.y;
        }
      }
    }
    float f[V];
    if (PRE2) {  // f is the phi tile's centre row
      vld<T, V>(reinterpret_cast<const T *>(sc + G::O_PHI) + (r + 1) * G::PW + G::HX + V * c, f);
    } else if (a.has_f) {
      vld<T, V>(reinterpret_cast<const T *>(sc + G::O_F) + r * TX + V * c, f);
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) f[e] = 0.f;
    }
    if (MODE == M_SMOOTH || PRE2) {
      const float2 om = make_float2(a.omega, a.omega), m1 = make_float2(-1.f, -1.f);
#pragma unroll
      for (int e = 0; e < V; e += 2) {
        const float2 num = __ffma2_rn(make_float2(Ax[e], Ax[e + 1]), m1, make_float2(f[e], f[e + 1]));
        const float2 rd = make_float2(__fdividef(1.f, dg[e]), __fdividef(1.f, dg[e + 1]));
        const float2 v = __ffma2_rn(om, __fmul2_rn(num, rd), make_float2(pc[e], pc[e + 1]));
        res[e] = v.x;
        res[e + 1] = v.y;
      }
      if (a.dot_rhs && valid) {
#pragma unroll
        for (int e = 0; e < V; ++e) acc += (double)res[e] * f[e];
      }
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) res[e] = Ax[e] - f[e];
      if (a.zero_xend_out && gx + V == X) res[V - 1] = 0.f;
      if (valid) {
#pragma unroll
        for (int e = 0; e < V; ++e) acc += (double)res[e] * (a.dot_phi ? pc[e] : res[e]);
      }
    }
    const int64_t off = inst * a.stride + ((int64_t)z * Y + gy) * X + gx;
    if (valid && a.out) {
      if (MODE == M_SMOOTH && a.top_copy && z == 1) vst<T, V>(a.out + inst * a.stride + (int64_t)gy * X + gx, res);
      if (!(MODE == M_SMOOTH && a.top_copy && z == 0 && Z > 1)) vst<T, V>(a.out + off, res);
    }
    if (MODE == M_RESTRICT) {
      // x pairs in the vector, y pairs with the lane TPR above (row r + 1), z pairs over planes
#pragma unroll
      for (int k = 0; k < V / 2; ++k) {
        float pk = res[2 * k] + res[2 * k + 1];
        pk += __shfl_down_sync(0xffffffffu, pk, G::TPR);
        cpart[k] += 0.125f * pk;
      }
      if (z & 1) {
        if (valid && !(r & 1)) {
          T *cp = a.coarse + inst * a.coarse_stride +
                  ((int64_t)(z >> 1) * (Y >> 1) + (gy >> 1)) * (X >> 1) + (gx >> 1);
#pragma unroll
          for (int k = 0; k < V / 2; ++k) cp[k] = St<T>::from(cpart[k]);
        }
#pragma unroll
        for (int k = 0; k < V / 2; ++k) cpart[k] = 0.f;
      }
    }
  }
  if (ok && __syncthreads_or(!mine)) ok = false;  // the last plane's wait
  if (!ok) {
    if (tid == 0) atomicAdd(&g_tma_wait_fail[0], 1);
    // drain: wait (bounded) for the planes whose loads are still in flight, so that no
    // copy lands in shared memory after this block has exited; thread 0 issued them all
    if (tid == 0) {
      bool drained = true;
      for (int p = p_waited + 1; p < p_next; ++p) drained = wait_plane(p, kMaxSpin) && drained;
      if (!drained) atomicAdd(&g_tma_wait_fail[1], 1);
    }
    return;
  }
  if ((MODE != M_SMOOTH || a.dot_rhs) && a.partials) {
    double t = block_sum(acc);
    if (tid == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

#include "tma_face.cuh"
#include "tma_face2.cuh"

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
  using G = Geo<T, KIND == HFM_OP_SIGMA7, CORR != 0, MODE == M_PRE2>;
  const int smem = G::NS * G::STAGE;
  int st = set_max_dynamic_smem((const void *)k_tma<KIND, T, MODE, CORR>, smem,
                                "cudaFuncSetAttribute(k_tma)");
  if (st) return st;
  k_tma<KIND, T, MODE, CORR><<<grid, G::THREADS, smem, s>>>(a);
  HFM_CHECK_LAUNCH("k_tma");
  return HFM_OK;
}

template <class T, int MODE, int CORR>
int go_face(const TmaArgs<T> &a, dim3 grid, cudaStream_t s) {
  using G = GeoF<CORR != 0, MODE == M_PRE2>;
  const int smem = G::NS * G::STAGE;
  int st = set_max_dynamic_smem((const void *)k_tma_face<T, MODE, CORR>, smem,
                                "cudaFuncSetAttribute(k_tma_face)");
  if (st) return st;
  k_tma_face<T, MODE, CORR><<<grid, G::THREADS, smem, s>>>(a);
  HFM_CHECK_LAUNCH("k_tma_face");
  return HFM_OK;
}

// Grid (plane tiles, z chunks, instances).  The z chunk length (even, at least 2) minimises
// (rounds of resident blocks) x (planes a block marches + 2 for its two halo planes and the
// pipeline fill): a last round that is only partly filled costs a whole round, and every
// chunk re-reads its halo planes.  (A fixed four waves left the 64^3 levels of 64 instances
// at 3.03 waves - a fourth round for 3 % of the blocks.)
template <class T>
dim3 tma_grid(TmaArgs<T> &a, Grid3 g, int B) {
  constexpr int TY = Geo<T>::TY;
  a.tiles_x = (g.X + TX - 1) / TX;
  const int tiles = a.tiles_x * ((g.Y + TY - 1) / TY);
  const int64_t per = (int64_t)tiles * B;
  const int64_t cap = (int64_t)sm_count() * Geo<T>::MINB;
  int zc = g.Z;
  int64_t best = -1;
  for (int c = 2; c < g.Z + 2; c += 2) {
    const int zcc = c > g.Z ? g.Z : c;
    const int64_t chunks = (g.Z + zcc - 1) / zcc;
    const int64_t cost = ((per * chunks + cap - 1) / cap) * (zcc + 2);
    if (best < 0 || cost <= best) {
      best = cost;
      zc = zcc;
    }
    if (zcc == g.Z) break;
  }
  a.zc = zc;
  return dim3(tiles, (g.Z + zc - 1) / zc, B);
}

}  // namespace

bool tma_eligible(int kind, Grid3 g, int mode, const void *corr, int corr_coarse, int es) {
  if (kind != HFM_OP_CONST7 && kind != HFM_OP_SIGMA7 && kind != HFM_OP_K27 &&
      kind != HFM_OP_FACE7)
    return false;
  if (kind == HFM_OP_FACE7 && es != 2) return false;  // the face kernel is 16-bit only
  // grids narrower than a tile (48 <= X < 64) use the same boxes: the columns past X are
  // zero-filled, not read.  Below X = 48 the register-queue kernels are as fast or faster
  // (measured: 32^3 and 24^3 levels of 64 instances).
  if (g.X < 48 || g.Y < (es == 4 ? 8 : 16)) return false;
  if ((g.X * es) % 16) return false;  // tensor-map strides are multiples of 16 bytes
  if (corr && !corr_coarse) return false;
  if (corr && ((g.X / 2) * es) % 16) return false;
  if (corr && ((g.Y | g.Z) & 1)) return false;
  if (mode == M_RESTRICT && (kind == HFM_OP_K27 || (g.Y & 1) || (g.Z & 1))) return false;
  if (mode != M_SMOOTH && corr) return false;
  return true;
}

// The FACE7 kernel (16-bit storage): tensor maps of phi (or f for the fused first two
// sweeps, with invd), the face arrays Fx [Z][Y][X + 8], Fy [Z][Y + 1][X], Fz [Z + 1][Y][X],
// the right-hand side and the coarse correction.  Callers exclude the x-end rule, the top
// copy and the p . A p sums (face_tma_ok).
template <class T>
int tma_launch_face(int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                    const T *invd, T *out, T *coarse, int64_t stride, int64_t coarse_stride,
                    int B, Grid3 g, float omega, unsigned flags, const int *active,
                    double *partials, int *nblk_out, cudaStream_t s) {
  using G = GeoF<false, false>;
  constexpr int TY = G::TY;
  TmaArgs<T> a;
  memset(&a, 0, sizeof(a));
  int st;
  const bool pre2 = mode == M_PRE2;
  const T *base = pre2 ? rhs : phi.base;
  a.has_phi = base != nullptr;
  if (a.has_phi && (st = make_map<T>(&a.m_phi, base, g.X, g.Y, g.Z, B, pre2 ? stride : phi.base_stride,
                                     G::PW, TY + 2)))
    return st;
  if ((st = make_map<T>(&a.m_sx, op.coef[0], g.X + 8, g.Y, g.Z, B, face7_nx(g.Z, g.Y, g.X), G::FXW, TY)))
    return st;
  if ((st = make_map<T>(&a.m_sy, op.coef[1], g.X, g.Y + 1, g.Z, B, face7_ny(g.Z, g.Y, g.X), TX, TY + 1)))
    return st;
  if ((st = make_map<T>(&a.m_sz, op.coef[2], g.X, g.Y, g.Z + 1, B, face7_nz(g.Z, g.Y, g.X), TX, TY)))
    return st;
  a.has_f = !pre2 && rhs != nullptr;
  if (a.has_f && (st = make_map<T>(&a.m_f, rhs, g.X, g.Y, g.Z, B, stride, TX, TY))) return st;
  const int corr = (!pre2 && phi.corr) ? 1 : 0;
  if (corr && (st = make_map<T>(&a.m_cc, phi.corr, g.X / 2, g.Y / 2, g.Z / 2, B, phi.corr_stride,
                                G::CW, TY / 2 + 2)))
    return st;
  if (pre2 && (st = make_map<T>(&a.m_ds, invd, g.X, g.Y, g.Z, B, stride, G::PW, TY + 2))) return st;
  unsigned bytes = (unsigned)((G::FXN + G::FYN + G::FZN) * sizeof(T));
  if (a.has_phi) bytes += (unsigned)(G::PHI * sizeof(T));
  if (a.has_f) bytes += (unsigned)(G::FN * sizeof(T));
  if (corr) bytes += (unsigned)(G::CCN * sizeof(T));
  if (pre2) bytes += (unsigned)(G::PHI * sizeof(T));
  a.stage_bytes = bytes;
  a.wait_budget = g_wait_budget.load();
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
  a.dot_rhs = ((mode == M_SMOOTH || pre2) && (flags & HFM_INT_DOT_RHS) && partials) ? 1 : 0;
  dim3 grid = tma_grid(a, g, B);
  if (nblk_out) *nblk_out = grid.x * grid.y;
  if (pre2) return go_face<T, M_PRE2, 0>(a, grid, s);
  if (mode == M_SMOOTH) {
    if (corr) return go_face<T, M_SMOOTH, 1>(a, grid, s);
    return go_face<T, M_SMOOTH, 0>(a, grid, s);
  }
  if (mode == M_RESID) return go_face<T, M_RESID, 0>(a, grid, s);
  return go_face<T, M_RESTRICT, 0>(a, grid, s);
}

template <class T, int PAIR, int CORR, int W>
int go_face2(const TmaArgs<T> &a, dim3 grid, cudaStream_t s) {
  using G = GeoF2<CORR != 0, PAIR == PAIR_PR, W>;
  int st = set_max_dynamic_smem((const void *)k_tma_face2<T, PAIR, CORR, W>, G::SMEM,
                                "cudaFuncSetAttribute(k_tma_face2)");
  if (st) return st;
  k_tma_face2<T, PAIR, CORR, W><<<grid, G::THREADS, G::SMEM, s>>>(a);
  HFM_CHECK_LAUNCH("k_tma_face2");
  return HFM_OK;
}

// Grid of the two-sweep kernel: every z chunk recomputes the first sweep on its two
// neighbouring planes, so chunks are fewer and longer than tma_grid's - about two waves of
// three resident blocks per SM, at least 4 planes each.
static dim3 face2_grid(int &tiles_x, int &zc, Grid3 g, int B, int W) {
  const int TY = 1024 / W;
  tiles_x = (g.X + W - 1) / W;
  const int tiles = tiles_x * ((g.Y + TY - 1) / TY);
  const int64_t slots = (int64_t)sm_count() * 3 * 2;
  const int64_t chunks = (slots + (int64_t)tiles * B - 1) / ((int64_t)tiles * B);
  zc = (int)((g.Z + chunks - 1) / chunks);
  if (zc < 4) zc = 4;
  if (zc & 1) ++zc;
  if (zc > g.Z) zc = g.Z;
  return dim3(tiles, (g.Z + zc - 1) / zc, B);
}

bool face2_eligible(int pair, bool corr, Grid3 g) {
  if (g.X < 48 || g.Y < 16 || g.Z < 2 || (g.X % 8)) return false;
  if (pair == PAIR_PR) return !((g.Y | g.Z) & 1);
  if (corr) return (g.X % 16) == 0 && !((g.Y | g.Z) & 1);
  return true;
}

template <class T, int W>
int launch_face2_w(int pair, const DevOp &op, const PhiSrc<T> &phi, const T *rhs, const T *invd,
                   T *out, T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g,
                   float omega, unsigned flags, const int *active, double *partials,
                   int *nblk_out, cudaStream_t s) {
  const bool pr = pair == PAIR_PR;
  const int corr = (!pr && phi.corr) ? 1 : 0;
  using G = GeoF2<false, false, W>;
  constexpr int TY = G::TY, PW = G::PW;
  TmaArgs<T> a;
  memset(&a, 0, sizeof(a));
  int st;
  if ((st = make_map<T>(&a.m_phi, pr ? rhs : phi.base, g.X, g.Y, g.Z, B, pr ? stride : phi.base_stride,
                        PW, TY + 4)))
    return st;
  if ((st = make_map<T>(&a.m_sx, op.coef[0], g.X + 8, g.Y, g.Z, B, face7_nx(g.Z, g.Y, g.X), PW, TY + 2)))
    return st;
  if ((st = make_map<T>(&a.m_sy, op.coef[1], g.X, g.Y + 1, g.Z, B, face7_ny(g.Z, g.Y, g.X), PW, TY + 3)))
    return st;
  if ((st = make_map<T>(&a.m_sz, op.coef[2], g.X, g.Y, g.Z + 1, B, face7_nz(g.Z, g.Y, g.X), PW, TY + 2)))
    return st;
  unsigned bytes = (unsigned)((G::PHI + G::FXN + G::FYN + G::FZN) * sizeof(T));
  if (!pr) {
    if ((st = make_map<T>(&a.m_f, rhs, g.X, g.Y, g.Z, B, stride, PW, TY + 2))) return st;
    bytes += (unsigned)(G::FN * sizeof(T));
  }
  if (corr) {
    if ((st = make_map<T>(&a.m_cc, phi.corr, g.X / 2, g.Y / 2, g.Z / 2, B, phi.corr_stride,
                          G::CW, TY / 2 + 2)))
      return st;
    bytes += (unsigned)(G::CCN * sizeof(T));
  }
  if (pr) {
    if ((st = make_map<T>(&a.m_ds, invd, g.X, g.Y, g.Z, B, stride, PW, TY + 4))) return st;
    bytes += (unsigned)(G::PHI * sizeof(T));
  }
  a.stage_bytes = bytes;
  a.wait_budget = g_wait_budget.load();
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
  a.dot_rhs = (!pr && (flags & HFM_INT_DOT_RHS) && partials) ? 1 : 0;
  dim3 grid = face2_grid(a.tiles_x, a.zc, g, B, W);
  if (nblk_out) *nblk_out = grid.x * grid.y;
  if (pr) return go_face2<T, PAIR_PR, 0, W>(a, grid, s);
  if (corr) return go_face2<T, PAIR_SS, 1, W>(a, grid, s);
  return go_face2<T, PAIR_SS, 0, W>(a, grid, s);
}

// Two sweeps in one pass (tma_face2.cuh).  PAIR_SS: phi (with the coarse correction when
// phi.corr is set) -> sweep -> sweep into out (z . r partials with HFM_INT_DOT_RHS); PAIR_PR:
// the fused first two sweeps from zero of f = rhs (1/diag = invd) into out, and the
// restricted residual of that iterate into coarse (|r|^2 partials when partials is given).
// Tiles are 128 wide for 64 < X <= 128 (one tile per row), 64 wide otherwise.
template <class T>
int tma_launch_face2(int pair, const DevOp &op, const PhiSrc<T> &phi, const T *rhs,
                     const T *invd, T *out, T *coarse, int64_t stride, int64_t coarse_stride,
                     int B, Grid3 g, float omega, unsigned flags, const int *active,
                     double *partials, int *nblk_out, cudaStream_t s) {
  if constexpr (sizeof(T) != 2) {
    return fail(HFM_ERR_UNSUPPORTED, "two-sweep kernel: 16-bit storage only");
  } else {
    if (!op.coef[0] || !op.coef[1] || !op.coef[2])
      return fail(HFM_ERR_BAD_ARG, "two-sweep kernel: FACE7 face arrays missing");
    const bool pr = pair == PAIR_PR;
    const int corr = (!pr && phi.corr) ? 1 : 0;
    if (!face2_eligible(pair, corr != 0, g))
      return fail(HFM_ERR_UNSUPPORTED, "two-sweep kernel: grid not eligible");
    if (pr ? (!rhs || !invd || !coarse) : (!phi.base || !rhs))
      return fail(HFM_ERR_BAD_ARG, "two-sweep kernel: missing operand");
    if (corr && !phi.corr_coarse) return fail(HFM_ERR_UNSUPPORTED, "two-sweep kernel: coarse correction only");
    if (g.X > 64 && g.X <= 128)
      return launch_face2_w<T, 128>(pair, op, phi, rhs, invd, out, coarse, stride, coarse_stride, B,
                                    g, omega, flags, active, partials, nblk_out, s);
    return launch_face2_w<T, 64>(pair, op, phi, rhs, invd, out, coarse, stride, coarse_stride, B, g,
                                 omega, flags, active, partials, nblk_out, s);
  }
}

template <class T>
int tma_launch(int kind, int mode, const DevOp &op, const PhiSrc<T> &phi, const T *rhs, T *out,
               T *coarse, int64_t stride, int64_t coarse_stride, int B, Grid3 g, float omega,
               unsigned flags, const int *active, double *partials, int *nblk_out,
               cudaStream_t s) {
  if (kind == HFM_OP_FACE7) {
    if constexpr (sizeof(T) == 2)
      return tma_launch_face<T>(mode, op, phi, rhs, nullptr, out, coarse, stride, coarse_stride,
                                B, g, omega, flags, active, partials, nblk_out, s);
    return fail(HFM_ERR_UNSUPPORTED, "tma path: FACE7 needs 16-bit storage");
  }
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
  a.wait_budget = g_wait_budget.load();
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
  a.dot_phi = (mode == M_RESID && (flags & HFM_INT_DOT_PHI)) ? 1 : 0;
  a.dot_rhs = (mode == M_SMOOTH && (flags & HFM_INT_DOT_RHS) && partials) ? 1 : 0;
  dim3 grid = tma_grid(a, g, B);
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

template <class T>
int tma_launch_pre2(int kind, const DevOp &op, const T *f, const T *invd, T *out, int64_t stride,
                    int B, Grid3 g, float omega, const int *active, cudaStream_t s) {
  if (kind == HFM_OP_FACE7) {
    if constexpr (sizeof(T) == 2) {
      PhiSrc<T> none;
      memset(&none, 0, sizeof(none));
      return tma_launch_face<T>(M_PRE2, op, none, f, invd, out, nullptr, stride, 0, B, g, omega,
                                0u, active, nullptr, nullptr, s);
    }
    return fail(HFM_ERR_UNSUPPORTED, "tma path: FACE7 needs 16-bit storage");
  }
  using G = Geo<T, true, false, true>;
  constexpr int TY = G::TY;
  TmaArgs<T> a;
  memset(&a, 0, sizeof(a));
  int st;
  if ((st = make_map<T>(&a.m_phi, f, g.X, g.Y, g.Z, B, stride, G::PW, TY + 2))) return st;
  if ((st = make_map<T>(&a.m_ds, invd, g.X, g.Y, g.Z, B, stride, G::PW, TY + 2))) return st;
  if ((st = make_map<T>(&a.m_sx, op.coef[0], g.X, g.Y, g.Z, B, op.coef_stride, G::PW, TY))) return st;
  if ((st = make_map<T>(&a.m_sy, op.coef[1], g.X, g.Y, g.Z, B, op.coef_stride, TX, TY + 2))) return st;
  if ((st = make_map<T>(&a.m_sz, op.coef[2], g.X, g.Y, g.Z, B, op.coef_stride, TX, TY))) return st;
  a.has_phi = 1;
  a.has_sigma = 1;
  a.stage_bytes = (unsigned)((2 * G::PHI + G::SXN + G::SYN + G::SZN) * sizeof(T));
  a.wait_budget = g_wait_budget.load();
  a.op = op;
  a.out = out;
  a.active = active;
  a.stride = stride;
  a.Z = g.Z;
  a.Y = g.Y;
  a.X = g.X;
  a.omega = omega;
  dim3 grid = tma_grid(a, g, B);
  return go<HFM_OP_SIGMA7, T, M_PRE2, 0>(a, grid, s);
}

#define HFM_TMA_INST(T)                                                                       \
  template int tma_launch<T>(int, int, const DevOp &, const PhiSrc<T> &, const T *, T *, T *, \
                             int64_t, int64_t, int, Grid3, float, unsigned, const int *,      \
                             double *, int *, cudaStream_t);
HFM_TMA_INST(float)
HFM_TMA_INST(__nv_bfloat16)
HFM_TMA_INST(__half)
#define HFM_FACE2_INST(T)                                                                     \
  template int tma_launch_face2<T>(int, const DevOp &, const PhiSrc<T> &, const T *, const T *, \
                                   T *, T *, int64_t, int64_t, int, Grid3, float, unsigned,     \
                                   const int *, double *, int *, cudaStream_t);
HFM_FACE2_INST(__nv_bfloat16)
HFM_FACE2_INST(__half)
template int tma_launch_pre2<float>(int, const DevOp &, const float *, const float *, float *,
                                    int64_t, int, Grid3, float, const int *, cudaStream_t);
template int tma_launch_pre2<__nv_bfloat16>(int, const DevOp &, const __nv_bfloat16 *,
                                            const __nv_bfloat16 *, __nv_bfloat16 *, int64_t, int,
                                            Grid3, float, const int *, cudaStream_t);
template int tma_launch_pre2<__half>(int, const DevOp &, const __half *, const __half *, __half *,
                                     int64_t, int, Grid3, float, const int *, cudaStream_t);

}  // namespace hfm

extern "C" int hfm_set_wait_budget(int polls) {
  if (polls < 0 || polls > (1 << 20)) return hfm::fail(HFM_ERR_BAD_ARG, "hfm_set_wait_budget: 0 .. 2^20 polls");
  hfm::g_wait_budget.store(polls);
  return HFM_OK;
}

namespace hfm {

int current_wait_budget() { return g_wait_budget.load(); }

// Device address of g_tma_wait_fail on the current device (looked up once per device with
// that device current: in host code the array's name only stands for the symbol).
int wait_fail_counters(const int **out) {
  static std::mutex mu;
  static std::vector<const int *> ptrs;
  int dev = 0;
  HFM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if ((int)ptrs.size() <= dev) ptrs.resize(dev + 1, nullptr);
  if (!ptrs[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_tma_wait_fail);
    if (e != cudaSuccess || !p) return cuda_status(e, "cudaGetSymbolAddress(wait counters)");
    ptrs[dev] = (const int *)p;
  }
  *out = ptrs[dev];
  return HFM_OK;
}

static int read_wait_counter(int which, int *count, int reset) {
  if (!count) return fail(HFM_ERR_BAD_ARG, "NULL");
  HFM_CUDA(cudaMemcpyFromSymbol(count, g_tma_wait_fail, sizeof(int), which * sizeof(int)));
  if (reset) {
    int zero = 0;
    HFM_CUDA(cudaMemcpyToSymbol(g_tma_wait_fail, &zero, sizeof(int), which * sizeof(int)));
  }
  return HFM_OK;
}

}  // namespace hfm

extern "C" int hfm_device_timeouts(int *count, int reset) {
  return hfm::read_wait_counter(0, count, reset);
}

extern "C" int hfm_device_drain_timeouts(int *count, int reset) {
  return hfm::read_wait_counter(1, count, reset);
}
