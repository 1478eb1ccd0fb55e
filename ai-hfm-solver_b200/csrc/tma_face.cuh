// TMA plane-marching kernel of the FACE7 operator in 16-bit storage (included by ops_tma.cu
// inside its anonymous namespace; it uses that file's mbarrier / TMA helpers and wait
// counters).
//
// The face form stores the coefficient of every cell face once (walls included), so a cell
// needs its two faces per axis - Fx[i], Fx[i+1] of its row, Fy of its row and the next,
// Fz of its plane and the next - and no face is formed from conductivities.  With
// S = sum of F * phi_nb over the six faces and D = the sum of the six faces,
//   (A phi)_c = D phi_c - S,
//   Jacobi:   phi_c + omega (f + S - D phi_c) / D.
// S and D are accumulated by the mixed-precision instructions of sm_100
// (fma.rn.f32.bf16 / add.rn.f32.bf16, and the .f16 forms): both 16-bit operands come
// straight from halves of the packed shared-memory words and the sum is float32, so the
// stencil needs no 16-bit -> float32 conversion of faces or neighbours.
//
// Block: 16 rows x 64 columns of the (y, x) plane, 128 threads, 8 cells (one 16-byte vector)
// per thread; per plane p the stage holds the phi tile with a one-row y halo and an 8-column
// x halo, Fx (row of 72 faces from x0), Fy (17 rows from y0), Fz of plane p + 1 (the face
// above plane p; plane z0's face below comes from the stage of plane z0 - 1), f and, for
// the fused correction, the coarse tile.  Waits and the timeout path are those of k_tma.

template <class T> struct Mx;

#define HFM_MX_OPS(TY)                                                                       \
  template <int HA, int HB>                                                                  \
  static __device__ __forceinline__ float fma(uint32_t a, uint32_t b, float c) {             \
    float d;                                                                                 \
    if constexpr (HA == 0 && HB == 0)                                                        \
      asm("{\n .reg .b16 a0, a1, b0, b1;\n mov.b32 {a0, a1}, %1;\n mov.b32 {b0, b1}, %2;\n"  \
          " fma.rn.f32." TY " %0, a0, b0, %3;\n}\n" : "=f"(d) : "r"(a), "r"(b), "f"(c));     \
    else if constexpr (HA == 0 && HB == 1)                                                   \
      asm("{\n .reg .b16 a0, a1, b0, b1;\n mov.b32 {a0, a1}, %1;\n mov.b32 {b0, b1}, %2;\n"  \
          " fma.rn.f32." TY " %0, a0, b1, %3;\n}\n" : "=f"(d) : "r"(a), "r"(b), "f"(c));     \
    else if constexpr (HA == 1 && HB == 0)                                                   \
      asm("{\n .reg .b16 a0, a1, b0, b1;\n mov.b32 {a0, a1}, %1;\n mov.b32 {b0, b1}, %2;\n"  \
          " fma.rn.f32." TY " %0, a1, b0, %3;\n}\n" : "=f"(d) : "r"(a), "r"(b), "f"(c));     \
    else                                                                                     \
      asm("{\n .reg .b16 a0, a1, b0, b1;\n mov.b32 {a0, a1}, %1;\n mov.b32 {b0, b1}, %2;\n"  \
          " fma.rn.f32." TY " %0, a1, b1, %3;\n}\n" : "=f"(d) : "r"(a), "r"(b), "f"(c));     \
    return d;                                                                                \
  }                                                                                          \
  template <int HA>                                                                          \
  static __device__ __forceinline__ float add(uint32_t a, float c) {                         \
    float d;                                                                                 \
    if constexpr (HA == 0)                                                                   \
      asm("{\n .reg .b16 a0, a1;\n mov.b32 {a0, a1}, %1;\n add.rn.f32." TY " %0, a0, %2;\n}\n" \
          : "=f"(d) : "r"(a), "f"(c));                                                       \
    else                                                                                     \
      asm("{\n .reg .b16 a0, a1;\n mov.b32 {a0, a1}, %1;\n add.rn.f32." TY " %0, a1, %2;\n}\n" \
          : "=f"(d) : "r"(a), "f"(c));                                                       \
    return d;                                                                                \
  }

template <> struct Mx<__nv_bfloat16> { HFM_MX_OPS("bf16") };
template <> struct Mx<__half> { HFM_MX_OPS("f16") };
#undef HFM_MX_OPS

// Stage layout of the face kernel (16-bit storage): byte offsets inside a stage.
template <bool CC, bool DS> struct GeoF {
  static constexpr int ES = 2;
  static constexpr int TY = 16, VEC = 8, TPR = TX / VEC, THREADS = TPR * TY;
  static constexpr int NS = 4, MINB = 4;
  static constexpr int HX = 8;
  static constexpr int PW = TX + 2 * HX;      // phi tile width
  static constexpr int FXW = TX + 8;          // Fx faces x0 .. x0 + TX (+ 7 unused)
  static constexpr int CW = TX / 2 + 2 * HX;  // coarse tile width
  static constexpr int PHI = (TY + 2) * PW;
  static constexpr int FXN = TY * FXW;
  static constexpr int FYN = (TY + 1) * TX;
  static constexpr int FZN = TY * TX;
  static constexpr int FN = TY * TX;
  static constexpr int CCN = (TY / 2 + 2) * CW;
  static constexpr int al(int elems) { return ((elems * ES + 127) / 128) * 128; }
  static constexpr int O_PHI = 0;
  static constexpr int O_FX = O_PHI + al(PHI);
  static constexpr int O_FY = O_FX + al(FXN);
  static constexpr int O_FZ = O_FY + al(FYN);
  static constexpr int O_F = O_FZ + al(FZN);
  static constexpr int O_CC = O_F + al(FN);
  static constexpr int O_DS = O_CC + (CC ? al(CCN) : 0);
  static constexpr int STAGE = O_DS + (DS ? al(PHI) : 0);
};

// 8 consecutive 16-bit values (16-byte aligned) as four packed words / 4 values as two.
__device__ __forceinline__ void ld8w(const void *p, uint32_t (&w)[4]) {
  const uint4 u = *reinterpret_cast<const uint4 *>(p);
  w[0] = u.x; w[1] = u.y; w[2] = u.z; w[3] = u.w;
}
__device__ __forceinline__ void ld4w(const void *p, uint32_t (&w)[2]) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p);
  w[0] = u.x; w[1] = u.y;
}
// One 16-bit value in the low half of a word.
__device__ __forceinline__ uint32_t ld1w(const void *p) {
  return (uint32_t)*reinterpret_cast<const unsigned short *>(p);
}

template <class T, int CORR, bool PRE2>
__device__ __forceinline__ void issue_plane_face(const TmaArgs<T> &a, char *stage, uint32_t bar,
                                                 int p, int x0, int y0, int b) {
  using G = GeoF<CORR != 0, PRE2>;
  mbar_expect(bar, a.stage_bytes);
  if (a.has_phi) tma_load(smem_u32(stage + G::O_PHI), &a.m_phi, x0 - G::HX, y0 - 1, p, b, bar);
  tma_load(smem_u32(stage + G::O_FX), &a.m_sx, x0, y0, p, b, bar);
  tma_load(smem_u32(stage + G::O_FY), &a.m_sy, x0, y0, p, b, bar);
  tma_load(smem_u32(stage + G::O_FZ), &a.m_sz, x0, y0, p + 1, b, bar);
  if (a.has_f) tma_load(smem_u32(stage + G::O_F), &a.m_f, x0, y0, p, b, bar);
  if (CORR) tma_load(smem_u32(stage + G::O_CC), &a.m_cc, (x0 >> 1) - G::HX, (y0 >> 1) - 1, p >> 1, b, bar);
  if (PRE2) tma_load(smem_u32(stage + G::O_DS), &a.m_ds, x0 - G::HX, y0 - 1, p, b, bar);
}

// S and D of cell E of the thread's 8 (half E & 1 of word E >> 1): the six faces times the
// six neighbours, and the six faces.  xl / xr: the neighbours left of cell 0 and right of
// cell 7 (low halves); fx8: the face right of cell 7 (low half).
template <class T, int E>
__device__ __forceinline__ void face_cell(const uint32_t (&c)[4], uint32_t xl, uint32_t xr,
                                          const uint32_t (&ym)[4], const uint32_t (&yp)[4],
                                          const uint32_t (&zm)[4], const uint32_t (&zp)[4],
                                          const uint32_t (&fx)[4], uint32_t fx8,
                                          const uint32_t (&fyl)[4], const uint32_t (&fyh)[4],
                                          const uint32_t (&fzl)[4], const uint32_t (&fzh)[4],
                                          float (&S)[8], float (&D)[8]) {
  constexpr int K = E >> 1, H = E & 1;
  using M = Mx<T>;
  float s, d;
  if constexpr (E == 0)
    s = M::template fma<0, 0>(fx[0], xl, 0.f);
  else
    s = M::template fma<H, (E - 1) & 1>(fx[K], c[(E - 1) >> 1], 0.f);
  d = M::template add<H>(fx[K], 0.f);
  if constexpr (E == 7) {
    s = M::template fma<0, 0>(fx8, xr, s);
    d = M::template add<0>(fx8, d);
  } else {
    s = M::template fma<(E + 1) & 1, (E + 1) & 1>(fx[(E + 1) >> 1], c[(E + 1) >> 1], s);
    d = M::template add<(E + 1) & 1>(fx[(E + 1) >> 1], d);
  }
  s = M::template fma<H, H>(fyl[K], ym[K], s);
  d = M::template add<H>(fyl[K], d);
  s = M::template fma<H, H>(fyh[K], yp[K], s);
  d = M::template add<H>(fyh[K], d);
  s = M::template fma<H, H>(fzl[K], zm[K], s);
  d = M::template add<H>(fzl[K], d);
  s = M::template fma<H, H>(fzh[K], zp[K], s);
  d = M::template add<H>(fzh[K], d);
  S[E] = s;
  D[E] = d;
}

// The same six products for the coarse correction: neighbour values are the coarse cells
// of the neighbours (cell E's own coarse cell is E >> 1 of the 4 in cv; cl / cr: left of
// cell 0, right of cell 7; cym / cyp / czm / czp: the coarse rows of the y / z neighbours).
template <class T, int E>
__device__ __forceinline__ float face_cell_coarse(const uint32_t (&cv)[2], uint32_t cl, uint32_t cr,
                                                  const uint32_t (&cym)[2], const uint32_t (&cyp)[2],
                                                  const uint32_t (&czm)[2], const uint32_t (&czp)[2],
                                                  const uint32_t (&fx)[4], uint32_t fx8,
                                                  const uint32_t (&fyl)[4], const uint32_t (&fyh)[4],
                                                  const uint32_t (&fzl)[4], const uint32_t (&fzh)[4]) {
  constexpr int K = E >> 1, H = E & 1;
  constexpr int CE = E >> 1, CW_ = CE >> 1, CH = CE & 1;  // own coarse cell: word, half
  using M = Mx<T>;
  float s;
  if constexpr (E == 0)
    s = M::template fma<0, 0>(fx[0], cl, 0.f);
  else
    s = M::template fma<H, ((E - 1) >> 1) & 1>(fx[K], cv[((E - 1) >> 1) >> 1], 0.f);
  if constexpr (E == 7)
    s = M::template fma<0, 0>(fx8, cr, s);
  else
    s = M::template fma<(E + 1) & 1, ((E + 1) >> 1) & 1>(fx[(E + 1) >> 1], cv[((E + 1) >> 1) >> 1], s);
  s = M::template fma<H, CH>(fyl[K], cym[CW_], s);
  s = M::template fma<H, CH>(fyh[K], cyp[CW_], s);
  s = M::template fma<H, CH>(fzl[K], czm[CW_], s);
  s = M::template fma<H, CH>(fzh[K], czp[CW_], s);
  return s;
}

// S and D of the thread's 8 cells with float32 neighbour values (the faces converted): the
// fused first two sweeps in fp16 storage, where omega f / diag can exceed the fp16 range (a
// residual spike, normalised to O(sqrt(n)), over a small diagonal) and is kept in float32 as
// the conductivity-form kernel keeps it.
template <class T>
__device__ __forceinline__ void face_cells_f32(const float (&c)[8], float xl, float xr,
                                               const float (&ym)[8], const float (&yp)[8],
                                               const float (&zm)[8], const float (&zp)[8],
                                               const uint32_t (&fx)[4], uint32_t fx8,
                                               const uint32_t (&fyl)[4], const uint32_t (&fyh)[4],
                                               const uint32_t (&fzl)[4], const uint32_t (&fzh)[4],
                                               float (&S)[8], float (&D)[8]) {
  float Fx[9], Fyl[8], Fyh[8], Fzl[8], Fzh[8];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float2 v = cvt2<T>(fx[k]);
    Fx[2 * k] = v.x; Fx[2 * k + 1] = v.y;
    v = cvt2<T>(fyl[k]);
    Fyl[2 * k] = v.x; Fyl[2 * k + 1] = v.y;
    v = cvt2<T>(fyh[k]);
    Fyh[2 * k] = v.x; Fyh[2 * k + 1] = v.y;
    v = cvt2<T>(fzl[k]);
    Fzl[2 * k] = v.x; Fzl[2 * k + 1] = v.y;
    v = cvt2<T>(fzh[k]);
    Fzh[2 * k] = v.x; Fzh[2 * k + 1] = v.y;
  }
  Fx[8] = cvt2<T>(fx8).x;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    float s = Fx[e] * (e == 0 ? xl : c[e - 1]);
    s = fmaf(Fx[e + 1], e == 7 ? xr : c[e + 1], s);
    s = fmaf(Fyl[e], ym[e], s);
    s = fmaf(Fyh[e], yp[e], s);
    s = fmaf(Fzl[e], zm[e], s);
    s = fmaf(Fzh[e], zp[e], s);
    S[e] = s;
    D[e] = ((((Fx[e] + Fx[e + 1]) + Fyl[e]) + Fyh[e]) + Fzl[e]) + Fzh[e];
  }
}

template <class T, int MODE, int CORR>
__global__ void __launch_bounds__(GeoF<false, false>::THREADS, GeoF<false, false>::MINB)
    k_tma_face(const __grid_constant__ TmaArgs<T> a) {
  constexpr bool PRE2 = MODE == M_PRE2;
  using G = GeoF<CORR != 0, PRE2>;
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
  const bool valid = gx < X && gy < Y;  // X is a multiple of V
  const int b = (int)inst;

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(smem_u32(&bars[s]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  const int p_first = z0 - 1, p_last = z1;
  int p_next = p_first;
  if (tid == 0) {
    for (; p_next <= p_last && p_next < p_first + NS; ++p_next) {
      const int q = p_next - p_first;
      issue_plane_face<T, CORR, PRE2>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
    }
  }
  int p_waited = p_first - 1;
  auto wait_plane = [&](int p, int budget) -> bool {
    const int q = p - p_first;
    const bool w = mbar_wait(smem_u32(&bars[q % NS]), (uint32_t)((q / NS) & 1), budget);
    if (w) p_waited = p;
    return w;
  };
  auto stage_of = [&](int p) -> const char * { return smem + ((p - p_first) % NS) * G::STAGE; };
  bool ok = wait_plane(z0 - 1, a.wait_budget);
  ok = wait_plane(z0, a.wait_budget) && ok;
  if (__syncthreads_or(!ok)) ok = false;

  const float om = a.omega, sc_ = a.op.scale;
  const bool scaled = sc_ != 1.f;
  using M = Mx<T>;

  // the thread's 8 values of a phi-tile row (tile row ry) and its left / right neighbours
  auto phi_row = [&](const char *st, int ry, uint32_t (&w)[4]) {
    ld8w(st + G::O_PHI + (ry * G::PW + G::HX + V * c) * 2, w);
  };
  // PRE2: g = f * (1 / diag) of a tile row; bf16 rounds it to the storage type (the first
  // sweep's phi1 = omega g, stored as the separate two-sweep form would store it), fp16 keeps
  // it in float32 (pre_rowf: omega f / diag can exceed the fp16 range); pre_one / pre_onef:
  // the single neighbours left and right of the row's 8 values
  auto pre_row = [&](const char *st, int ry, uint32_t (&w)[4]) {
    uint32_t f[4], d[4];
    ld8w(st + G::O_PHI + (ry * G::PW + G::HX + V * c) * 2, f);
    ld8w(st + G::O_DS + (ry * G::PW + G::HX + V * c) * 2, d);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      w[k] = pack2<T>(M::template fma<0, 0>(f[k], d[k], 0.f), M::template fma<1, 1>(f[k], d[k], 0.f));
  };
  auto pre_rowf = [&](const char *st, int ry, float (&g)[8]) {
    uint32_t f[4], d[4];
    ld8w(st + G::O_PHI + (ry * G::PW + G::HX + V * c) * 2, f);
    ld8w(st + G::O_DS + (ry * G::PW + G::HX + V * c) * 2, d);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 fv = cvt2<T>(f[k]), dv = cvt2<T>(d[k]);
      g[2 * k] = fv.x * dv.x;
      g[2 * k + 1] = fv.y * dv.y;
    }
  };
  auto pre_onef = [&](const char *st, int ry, int col) -> float {
    return cvt2<T>(ld1w(st + G::O_PHI + (ry * G::PW + col) * 2)).x *
           cvt2<T>(ld1w(st + G::O_DS + (ry * G::PW + col) * 2)).x;
  };
  auto pre_one = [&](const char *st, int ry, int col) -> uint32_t {
    const uint32_t f = ld1w(st + G::O_PHI + (ry * G::PW + col) * 2);
    const uint32_t d = ld1w(st + G::O_DS + (ry * G::PW + col) * 2);
    return pack2<T>(M::template fma<0, 0>(f, d, 0.f), 0.f);
  };

  // faces below plane z0 (packed), then carried: the face above plane z is the face below z+1
  uint32_t fzl[4] = {0u, 0u, 0u, 0u};
  if (ok) ld8w(stage_of(z0 - 1) + G::O_FZ + (r * TX + V * c) * 2, fzl);
  double acc = 0.0;
  float cpart[V / 2];
#pragma unroll
  for (int e = 0; e < V / 2; ++e) cpart[e] = 0.f;

  bool mine = true;
  for (int z = z0; z < z1 && ok; ++z) {
    if (__syncthreads_or(!mine)) {
      ok = false;
      break;
    }
    if (tid == 0 && z > z0 && p_next <= p_last) {
      const int q = p_next - p_first;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_plane_face<T, CORR, PRE2>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
      ++p_next;
    }
    mine = wait_plane(z + 1, a.wait_budget);
    const char *sm_ = stage_of(z - 1);
    const char *sc = stage_of(z);
    const char *sp = stage_of(z + 1);

    // neighbours (phi, or g for PRE2), faces, right-hand side
    constexpr bool PRE2F = PRE2 && std::is_same<T, __half>::value;  // fp16: g in float32
    uint32_t pc[4], pym[4], pyp[4], pzm[4], pzp[4], pl, pr;
    float gc[8], gym[8], gyp[8], gzm[8], gzp[8], gl = 0.f, gr = 0.f;
    if (PRE2F) {
      pre_rowf(sc, r + 1, gc);
      pre_rowf(sc, r, gym);
      pre_rowf(sc, r + 2, gyp);
      pre_rowf(sm_, r + 1, gzm);
      pre_rowf(sp, r + 1, gzp);
      gl = pre_onef(sc, r + 1, G::HX + V * c - 1);
      gr = pre_onef(sc, r + 1, G::HX + V * c + V);
#pragma unroll
      for (int k = 0; k < 4; ++k) pc[k] = pym[k] = pyp[k] = pzm[k] = pzp[k] = 0u;
      pl = pr = 0u;
    } else if (PRE2) {
      pre_row(sc, r + 1, pc);
      pre_row(sc, r, pym);
      pre_row(sc, r + 2, pyp);
      pre_row(sm_, r + 1, pzm);
      pre_row(sp, r + 1, pzp);
      pl = pre_one(sc, r + 1, G::HX + V * c - 1);
      pr = pre_one(sc, r + 1, G::HX + V * c + V);
    } else if (a.has_phi) {
      phi_row(sc, r + 1, pc);
      phi_row(sc, r, pym);
      phi_row(sc, r + 2, pyp);
      phi_row(sm_, r + 1, pzm);
      phi_row(sp, r + 1, pzp);
      pl = ld1w(sc + G::O_PHI + ((r + 1) * G::PW + G::HX + V * c - 1) * 2);
      pr = ld1w(sc + G::O_PHI + ((r + 1) * G::PW + G::HX + V * c + V) * 2);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) pc[k] = pym[k] = pyp[k] = pzm[k] = pzp[k] = 0u;
      pl = pr = 0u;
    }
    uint32_t fx[4], fyl[4], fyh[4], fzh[4], fr[4];
    ld8w(sc + G::O_FX + (r * G::FXW + V * c) * 2, fx);
    const uint32_t fx8 = ld1w(sc + G::O_FX + (r * G::FXW + V * c + V) * 2);
    ld8w(sc + G::O_FY + (r * TX + V * c) * 2, fyl);
    ld8w(sc + G::O_FY + ((r + 1) * TX + V * c) * 2, fyh);
    ld8w(sc + G::O_FZ + (r * TX + V * c) * 2, fzh);
    if (PRE2)  // f is the phi tile's centre row
      ld8w(sc + G::O_PHI + ((r + 1) * G::PW + G::HX + V * c) * 2, fr);
    else if (a.has_f)
      ld8w(sc + G::O_F + (r * TX + V * c) * 2, fr);
    else
      fr[0] = fr[1] = fr[2] = fr[3] = 0u;

    float S[8], D[8];
    float pcf[8];  // the centre values in float32
    if (PRE2F) {
      face_cells_f32<T>(gc, gl, gr, gym, gyp, gzm, gzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
#pragma unroll
      for (int e = 0; e < 8; ++e) pcf[e] = gc[e];
    } else {
      face_cell<T, 0>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 1>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 2>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 3>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 4>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 5>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 6>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
      face_cell<T, 7>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzl, fzh, S, D);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 v = cvt2<T>(pc[k]);
        pcf[2 * k] = v.x;
        pcf[2 * k + 1] = v.y;
      }
    }
    if (PRE2) {  // phi1 = omega g: the products above are omega-free
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        S[e] *= om;
        pcf[e] *= om;
      }
    }
    if (CORR) {
      // phi' = phi + sign P w on every point: add sign * (the six faces times the coarse
      // values of the neighbours) to S and sign * (the coarse value) to the centre
      const int cb = G::HX + (V / 2) * c;  // column of the thread's first coarse cell
      const char *cct = sc + G::O_CC;
      const int crow = (r >> 1) + 1, cym_r = ((r - 1) >> 1) + 1, cyp_r = ((r + 1) >> 1) + 1;
      uint32_t cv[2], cym[2], cyp[2], czm[2], czp[2];
      ld4w(cct + (crow * G::CW + cb) * 2, cv);
      ld4w(cct + (cym_r * G::CW + cb) * 2, cym);
      ld4w(cct + (cyp_r * G::CW + cb) * 2, cyp);
      ld4w(sm_ + G::O_CC + (crow * G::CW + cb) * 2, czm);
      ld4w(sp + G::O_CC + (crow * G::CW + cb) * 2, czp);
      const uint32_t cl = ld1w(cct + (crow * G::CW + cb - 1) * 2);
      const uint32_t cr = ld1w(cct + (crow * G::CW + cb + V / 2) * 2);
      const float sg = a.corr_sign;
      float Sc[8];
      Sc[0] = face_cell_coarse<T, 0>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[1] = face_cell_coarse<T, 1>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[2] = face_cell_coarse<T, 2>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[3] = face_cell_coarse<T, 3>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[4] = face_cell_coarse<T, 4>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[5] = face_cell_coarse<T, 5>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[6] = face_cell_coarse<T, 6>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      Sc[7] = face_cell_coarse<T, 7>(cv, cl, cr, cym, cyp, czm, czp, fx, fx8, fyl, fyh, fzl, fzh);
      const float2 w01 = cvt2<T>(cv[0]), w23 = cvt2<T>(cv[1]);
      const float wc[4] = {w01.x, w01.y, w23.x, w23.y};
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        S[e] = fmaf(sg, Sc[e], S[e]);
        pcf[e] = fmaf(sg, wc[e >> 1], pcf[e]);
      }
    }
    if (scaled) {
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        S[e] *= sc_;
        D[e] *= sc_;
      }
    }
    // next plane's face below = this plane's face above
#pragma unroll
    for (int k = 0; k < 4; ++k) fzl[k] = fzh[k];

    float res[8];
    float pacc = 0.f;  // this plane's partial sum (float32 over the thread's 8 cells)
    if (MODE == M_SMOOTH || PRE2) {
      const float2 om2 = make_float2(om, om);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        // u = f + S - D phi_c ; out = phi_c + omega u / D
        const float2 t = make_float2(M::template add<0>(fr[k], S[2 * k]), M::template add<1>(fr[k], S[2 * k + 1]));
        const float2 pcv = make_float2(pcf[2 * k], pcf[2 * k + 1]);
        const float2 u = __ffma2_rn(make_float2(-D[2 * k], -D[2 * k + 1]), pcv, t);
        const float2 rd = make_float2(__fdividef(1.f, D[2 * k]), __fdividef(1.f, D[2 * k + 1]));
        const float2 o = __ffma2_rn(om2, __fmul2_rn(u, rd), pcv);
        res[2 * k] = o.x;
        res[2 * k + 1] = o.y;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        // r = D phi_c - (S + f)
        const float t0 = M::template add<0>(fr[k], S[2 * k]), t1 = M::template add<1>(fr[k], S[2 * k + 1]);
        res[2 * k] = fmaf(D[2 * k], pcf[2 * k], -t0);
        res[2 * k + 1] = fmaf(D[2 * k + 1], pcf[2 * k + 1], -t1);
      }
    }
    uint32_t packed[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) packed[k] = pack2<T>(res[2 * k], res[2 * k + 1]);
    if (valid) {
      if ((MODE == M_SMOOTH || PRE2) && a.dot_rhs) {
        // z . r of a preconditioner whose right-hand side is r: the stored z times r
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          pacc = M::template fma<0, 0>(packed[k], fr[k], pacc);
          pacc = M::template fma<1, 1>(packed[k], fr[k], pacc);
        }
      } else if (MODE == M_RESID || MODE == M_RESTRICT) {
#pragma unroll
        for (int e = 0; e < 8; ++e) pacc = fmaf(res[e], res[e], pacc);
      }
      acc += (double)pacc;
      if (a.out) {
        uint4 u;
        u.x = packed[0]; u.y = packed[1]; u.z = packed[2]; u.w = packed[3];
        *reinterpret_cast<uint4 *>(a.out + inst * a.stride + ((int64_t)z * Y + gy) * X + gx) = u;
      }
    }
    if (MODE == M_RESTRICT) {
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
  if (ok && __syncthreads_or(!mine)) ok = false;
  if (!ok) {
    if (tid == 0) atomicAdd(&g_tma_wait_fail[0], 1);
    if (tid == 0) {
      bool drained = true;
      for (int p = p_waited + 1; p < p_next; ++p) drained = wait_plane(p, kMaxSpin) && drained;
      if (!drained) atomicAdd(&g_tma_wait_fail[1], 1);
    }
    return;
  }
  if ((MODE != M_SMOOTH || a.dot_rhs) && !PRE2 && a.partials) {
    double t = block_sum(acc);
    if (tid == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}
