// Two Jacobi sweeps of the FACE7 operator in one pass (temporal blocking), 16-bit storage.
// Included by ops_tma.cu after tma_face.cuh, inside its anonymous namespace.
//
// A block marches its (16 x 64) tile of planes z0 .. z1-1 in z.  The first sweep ("A") is
// computed one cell wider than the tile on every side - rows -1 .. 16, columns -1 .. 64 and
// planes z0-1 .. z1 - into a three-plane shared-memory ring, rounded to the storage type as
// the separate launches store it; the second sweep ("B") reads its neighbours from that ring
// and writes the tile.  Cells outside the grid get A = 0, which is what the second launch of
// the separate form reads there (the TMA boxes are zero-filled outside).  The results equal
// two separate launches bit for bit: the ring cells use the same operation order as the
// cells of the neighbouring tiles that own them.
//
//   PAIR_SS: A = Jacobi sweep (with the coarse correction phi + sign P w first, CORR), B =
//            Jacobi sweep (with the z . r partial sums of a preconditioner, dot_rhs);
//            out = B.
//   PAIR_PR: A = the fused first two sweeps from a zero iterate (M_PRE2: phi1 = omega f /
//            diag is pointwise, so A needs f and 1/diag two cells out), stored to out on the
//            tile; B = residual D phi - S - f of A, restricted to the coarse grid (with the
//            |r|^2 partial sums).
//
// Stage (plane p): phi (or f for PAIR_PR) rows -2 .. 17 and columns -8 .. 71, Fx / Fz / f
// rows -1 .. 16 and the same columns, Fy face rows -1 .. 17, 1/diag like phi (PAIR_PR), the
// coarse tile (CORR).  160 threads: 144 compute A (18 rows x 8 groups of 8 cells, the
// first and last group of a row also its column -1 / 64 cell), the first 128 compute B.
// Loads, waits and the timeout path are those of k_tma_face.

// W: tile width, 64 (16 rows) or 128 (8 rows); either way 128 threads own the tile's 1024
// cells in the second sweep and 144 or 160 threads the first sweep's rows.  A tile as wide
// as the grid has no ring columns inside the grid (they are zero), so grids with
// 64 < X <= 128 take W = 128 and never run the single-cell path.
template <bool CC, bool DS, int W = 64> struct GeoF2 {
  static constexpr int ES = 2;
  static constexpr int TW = W;
  static constexpr int TY = 1024 / W, VEC = 8, TPR = W / VEC;
  static constexpr int BT = TPR * TY;               // threads of the second sweep
  static constexpr int AT = TPR * (TY + 2);         // threads of the first sweep
  static constexpr int THREADS = 160;               // AT rounded up to whole warps
  static constexpr int NS = 4, MINB = 3;
  static constexpr int HX = 8, PW = W + 2 * HX;
  static constexpr int CW = W / 2 + 2 * HX;
  static constexpr int PHI = (TY + 4) * PW;
  static constexpr int FXN = (TY + 2) * PW;
  static constexpr int FYN = (TY + 3) * PW;
  static constexpr int FZN = (TY + 2) * PW;
  static constexpr int FN = (TY + 2) * PW;
  static constexpr int CCN = (TY / 2 + 2) * CW;
  static constexpr int ABN = (TY + 2) * PW;         // one plane of A, the layout of a phi tile
  static constexpr int al(int elems) { return ((elems * ES + 127) / 128) * 128; }
  static constexpr int O_PHI = 0;
  static constexpr int O_FX = O_PHI + al(PHI);
  static constexpr int O_FY = O_FX + al(FXN);
  static constexpr int O_FZ = O_FY + al(FYN);
  static constexpr int O_F = O_FZ + al(FZN);
  static constexpr int O_CC = O_F + (DS ? 0 : al(FN));
  static constexpr int O_DS = O_CC + (CC ? al(CCN) : 0);
  static constexpr int STAGE = O_DS + (DS ? al(PHI) : 0);
  static constexpr int AB = al(ABN);
  static constexpr int SMEM = NS * STAGE + 3 * AB;
};

template <class T, int PAIR, int CORR, int W>
__device__ __forceinline__ void issue_plane_face2(const TmaArgs<T> &a, char *stage, uint32_t bar,
                                                  int p, int x0, int y0, int b) {
  using G = GeoF2<CORR != 0, PAIR == PAIR_PR, W>;
  mbar_expect(bar, a.stage_bytes);
  tma_load(smem_u32(stage + G::O_PHI), &a.m_phi, x0 - G::HX, y0 - 2, p, b, bar);
  tma_load(smem_u32(stage + G::O_FX), &a.m_sx, x0 - G::HX, y0 - 1, p, b, bar);
  tma_load(smem_u32(stage + G::O_FY), &a.m_sy, x0 - G::HX, y0 - 1, p, b, bar);
  tma_load(smem_u32(stage + G::O_FZ), &a.m_sz, x0 - G::HX, y0 - 1, p + 1, b, bar);
  if (PAIR == PAIR_SS) tma_load(smem_u32(stage + G::O_F), &a.m_f, x0 - G::HX, y0 - 1, p, b, bar);
  if (CORR) tma_load(smem_u32(stage + G::O_CC), &a.m_cc, (x0 >> 1) - G::HX, (y0 >> 1) - 1, p >> 1, b, bar);
  if (PAIR == PAIR_PR) tma_load(smem_u32(stage + G::O_DS), &a.m_ds, x0 - G::HX, y0 - 2, p, b, bar);
}

// One 16-bit value of shared memory as float32.
template <class T> __device__ __forceinline__ float sh1(const char *p) {
  return cvt2<T>(ld1w(p)).x;
}

// The Jacobi update of one cell from its S, D (already scaled), centre value and f, in the
// operation order of the packed path (t = f + S; u = t - D c; c + omega u / D).
__device__ __forceinline__ float jacobi1(float S, float D, float pc, float fr, float om) {
  const float t = __fadd_rn(fr, S);
  const float u = __fmaf_rn(-D, pc, t);
  const float rd = __fdividef(1.f, D);
  return __fmaf_rn(om, __fmul_rn(u, rd), pc);
}

template <class T, int PAIR, int CORR, int W>
__global__ void __launch_bounds__(GeoF2<false, false>::THREADS, GeoF2<false, false>::MINB)
    k_tma_face2(const __grid_constant__ TmaArgs<T> a) {
  constexpr bool PR = PAIR == PAIR_PR;
  constexpr bool PRE2F = PR && std::is_same<T, __half>::value;  // fp16: g in float32
  using G = GeoF2<CORR != 0, PR, W>;
  constexpr int TY = G::TY, V = G::VEC, NS = G::NS, PW = G::PW, HX = G::HX, TX = G::TW;
  extern __shared__ __align__(128) char smem[];
  __shared__ __align__(8) uint64_t bars[NS];
  const int64_t inst = blockIdx.z;
  if (a.active && !a.active[inst]) return;
  const int X = a.X, Y = a.Y, Z = a.Z;
  const int tx = blockIdx.x % a.tiles_x, ty = blockIdx.x / a.tiles_x;
  const int x0 = tx * TX, y0 = ty * TY;
  const int z0 = blockIdx.y * a.zc, z1 = min(Z, z0 + a.zc);
  const int tid = threadIdx.x;
  const int c = tid % G::TPR;
  const int ra = tid / G::TPR - 1;  // A row (-1 .. TY) of threads tid < AT
  const int rb = tid / G::TPR;      // B row (0 .. TY-1) of threads tid < BT
  const int b = (int)inst;
  char *ring = smem + NS * G::STAGE;

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(smem_u32(&bars[s]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  // A at plane p needs the stages of p-1, p, p+1; A runs for p = z0-1 .. z1
  const int p_first = z0 - 2, p_last = z1 + 1;
  int p_next = p_first;
  if (tid == 0) {
    for (; p_next <= p_last && p_next < p_first + NS; ++p_next) {
      const int q = p_next - p_first;
      issue_plane_face2<T, PAIR, CORR, W>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
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
  auto ring_of = [&](int p) -> char * { return ring + ((p - z0 + 1) % 3) * G::AB; };
  bool ok = wait_plane(p_first, a.wait_budget);
  ok = wait_plane(p_first + 1, a.wait_budget) && ok;
  if (__syncthreads_or(!ok)) ok = false;

  const float om = a.omega, sc_ = a.op.scale;
  const bool scaled = sc_ != 1.f;
  using M = Mx<T>;

  // byte offsets inside a stage: A row ra / B row rb of the boxes that start one
  // row above the tile (Fx, Fy, Fz, f, ring) and of those that start two rows above (phi, f
  // of PAIR_PR, 1/diag); column x of the tile is HX + x
  auto o1 = [&](int row, int col) { return ((row + 1) * PW + HX + col) * 2; };
  auto o2 = [&](int row, int col) { return ((row + 2) * PW + HX + col) * 2; };

  // PAIR_PR: g = f / diag (rounded to the storage type for bf16, float32 for fp16)
  auto pre_row = [&](const char *st, int row, uint32_t (&w)[4]) {
    uint32_t f[4], d[4];
    ld8w(st + G::O_PHI + o2(row, V * c), f);
    ld8w(st + G::O_DS + o2(row, V * c), d);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      w[k] = pack2<T>(M::template fma<0, 0>(f[k], d[k], 0.f), M::template fma<1, 1>(f[k], d[k], 0.f));
  };
  auto pre_rowf = [&](const char *st, int row, float (&g)[8]) {
    uint32_t f[4], d[4];
    ld8w(st + G::O_PHI + o2(row, V * c), f);
    ld8w(st + G::O_DS + o2(row, V * c), d);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 fv = cvt2<T>(f[k]), dv = cvt2<T>(d[k]);
      g[2 * k] = fv.x * dv.x;
      g[2 * k + 1] = fv.y * dv.y;
    }
  };
  // g of one cell as the packed path sees it (rounded for bf16, float32 for fp16)
  auto pre_one = [&](const char *st, int row, int col) -> float {
    const uint32_t f = ld1w(st + G::O_PHI + o2(row, col));
    const uint32_t d = ld1w(st + G::O_DS + o2(row, col));
    if (PRE2F) return cvt2<T>(f).x * cvt2<T>(d).x;
    return cvt2<T>(pack2<T>(M::template fma<0, 0>(f, d, 0.f), 0.f)).x;
  };

  // ---- A of one 8-cell group (row ra, columns 8c .. 8c+7) at plane p
  auto a_group = [&](const char *sm_, const char *sc, const char *sp, float (&res)[8]) {
    uint32_t pc[4], pym[4], pyp[4], pzm[4], pzp[4], pl, pr;
    float gc[8], gym[8], gyp[8], gzm[8], gzp[8], gl = 0.f, gr = 0.f;
    if (PRE2F) {
      pre_rowf(sc, ra, gc);
      pre_rowf(sc, ra - 1, gym);
      pre_rowf(sc, ra + 1, gyp);
      pre_rowf(sm_, ra, gzm);
      pre_rowf(sp, ra, gzp);
      gl = pre_one(sc, ra, V * c - 1);
      gr = pre_one(sc, ra, V * c + V);
#pragma unroll
      for (int k = 0; k < 4; ++k) pc[k] = pym[k] = pyp[k] = pzm[k] = pzp[k] = 0u;
      pl = pr = 0u;
    } else if (PR) {
      pre_row(sc, ra, pc);
      pre_row(sc, ra - 1, pym);
      pre_row(sc, ra + 1, pyp);
      pre_row(sm_, ra, pzm);
      pre_row(sp, ra, pzp);
      pl = pack2<T>(pre_one(sc, ra, V * c - 1), 0.f);
      pr = pack2<T>(pre_one(sc, ra, V * c + V), 0.f);
    } else {
      ld8w(sc + G::O_PHI + o2(ra, V * c), pc);
      ld8w(sc + G::O_PHI + o2(ra - 1, V * c), pym);
      ld8w(sc + G::O_PHI + o2(ra + 1, V * c), pyp);
      ld8w(sm_ + G::O_PHI + o2(ra, V * c), pzm);
      ld8w(sp + G::O_PHI + o2(ra, V * c), pzp);
      pl = ld1w(sc + G::O_PHI + o2(ra, V * c - 1));
      pr = ld1w(sc + G::O_PHI + o2(ra, V * c + V));
    }
    uint32_t fx[4], fyl[4], fyh[4], fzl[4], fzh[4], fr[4];
    ld8w(sc + G::O_FX + o1(ra, V * c), fx);
    const uint32_t fx8 = ld1w(sc + G::O_FX + o1(ra, V * c + V));
    ld8w(sc + G::O_FY + o1(ra, V * c), fyl);
    ld8w(sc + G::O_FY + o1(ra + 1, V * c), fyh);
    ld8w(sm_ + G::O_FZ + o1(ra, V * c), fzl);
    ld8w(sc + G::O_FZ + o1(ra, V * c), fzh);
    if (PR)
      ld8w(sc + G::O_PHI + o2(ra, V * c), fr);
    else
      ld8w(sc + G::O_F + o1(ra, V * c), fr);
    float S[8], D[8], pcf[8];
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
    if (PR) {
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        S[e] *= om;
        pcf[e] *= om;
      }
    }
    if (CORR) {
      const int cb = HX + (V / 2) * c;
      const int crow = (ra >> 1) + 1, cym_r = ((ra - 1) >> 1) + 1, cyp_r = ((ra + 1) >> 1) + 1;
      uint32_t cv[2], cym[2], cyp[2], czm[2], czp[2];
      ld4w(sc + G::O_CC + (crow * G::CW + cb) * 2, cv);
      ld4w(sc + G::O_CC + (cym_r * G::CW + cb) * 2, cym);
      ld4w(sc + G::O_CC + (cyp_r * G::CW + cb) * 2, cyp);
      ld4w(sm_ + G::O_CC + (crow * G::CW + cb) * 2, czm);
      ld4w(sp + G::O_CC + (crow * G::CW + cb) * 2, czp);
      const uint32_t cl = ld1w(sc + G::O_CC + (crow * G::CW + cb - 1) * 2);
      const uint32_t cr = ld1w(sc + G::O_CC + (crow * G::CW + cb + V / 2) * 2);
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
    const float2 om2 = make_float2(om, om);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 t = make_float2(M::template add<0>(fr[k], S[2 * k]), M::template add<1>(fr[k], S[2 * k + 1]));
      const float2 pcv = make_float2(pcf[2 * k], pcf[2 * k + 1]);
      const float2 u = __ffma2_rn(make_float2(-D[2 * k], -D[2 * k + 1]), pcv, t);
      const float2 rd = make_float2(__fdividef(1.f, D[2 * k]), __fdividef(1.f, D[2 * k + 1]));
      const float2 o = __ffma2_rn(om2, __fmul2_rn(u, rd), pcv);
      res[2 * k] = o.x;
      res[2 * k + 1] = o.y;
    }
  };

  // ---- A of the single cell at column xc (-1 or TX) of row ra: the operations of the
  // packed path for that cell, on float32 values of the same 16-bit operands
  auto a_one = [&](const char *sm_, const char *sc, const char *sp, int xc) -> float {
    float vc, vl, vr, vym, vyp, vzm, vzp;
    if (PR) {
      vc = pre_one(sc, ra, xc);
      vl = pre_one(sc, ra, xc - 1);
      vr = pre_one(sc, ra, xc + 1);
      vym = pre_one(sc, ra - 1, xc);
      vyp = pre_one(sc, ra + 1, xc);
      vzm = pre_one(sm_, ra, xc);
      vzp = pre_one(sp, ra, xc);
    } else {
      vc = sh1<T>(sc + G::O_PHI + o2(ra, xc));
      vl = sh1<T>(sc + G::O_PHI + o2(ra, xc - 1));
      vr = sh1<T>(sc + G::O_PHI + o2(ra, xc + 1));
      vym = sh1<T>(sc + G::O_PHI + o2(ra - 1, xc));
      vyp = sh1<T>(sc + G::O_PHI + o2(ra + 1, xc));
      vzm = sh1<T>(sm_ + G::O_PHI + o2(ra, xc));
      vzp = sh1<T>(sp + G::O_PHI + o2(ra, xc));
    }
    const float fxl = sh1<T>(sc + G::O_FX + o1(ra, xc)), fxr = sh1<T>(sc + G::O_FX + o1(ra, xc + 1));
    const float fyl = sh1<T>(sc + G::O_FY + o1(ra, xc)), fyh = sh1<T>(sc + G::O_FY + o1(ra + 1, xc));
    const float fzl = sh1<T>(sm_ + G::O_FZ + o1(ra, xc)), fzh = sh1<T>(sc + G::O_FZ + o1(ra, xc));
    const float fr = PR ? sh1<T>(sc + G::O_PHI + o2(ra, xc)) : sh1<T>(sc + G::O_F + o1(ra, xc));
    float S, D;
    if (PRE2F) {  // face_cells_f32
      S = __fmul_rn(fxl, vl);
      S = __fmaf_rn(fxr, vr, S);
      S = __fmaf_rn(fyl, vym, S);
      S = __fmaf_rn(fyh, vyp, S);
      S = __fmaf_rn(fzl, vzm, S);
      S = __fmaf_rn(fzh, vzp, S);
      D = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(fxl, fxr), fyl), fyh), fzl), fzh);
    } else {  // face_cell
      S = __fmaf_rn(fxl, vl, 0.f);
      D = __fadd_rn(fxl, 0.f);
      S = __fmaf_rn(fxr, vr, S);
      D = __fadd_rn(fxr, D);
      S = __fmaf_rn(fyl, vym, S);
      D = __fadd_rn(fyl, D);
      S = __fmaf_rn(fyh, vyp, S);
      D = __fadd_rn(fyh, D);
      S = __fmaf_rn(fzl, vzm, S);
      D = __fadd_rn(fzl, D);
      S = __fmaf_rn(fzh, vzp, S);
      D = __fadd_rn(fzh, D);
    }
    float pcf = vc;
    if (PR) {
      S = __fmul_rn(S, om);
      pcf = __fmul_rn(pcf, om);
    }
    if (CORR) {
      const int crow = (ra >> 1) + 1, cym_r = ((ra - 1) >> 1) + 1, cyp_r = ((ra + 1) >> 1) + 1;
      const int cc = HX + (xc >> 1), cl = HX + ((xc - 1) >> 1), cr = HX + ((xc + 1) >> 1);
      const float wv = sh1<T>(sc + G::O_CC + (crow * G::CW + cc) * 2);
      float Sc = __fmaf_rn(fxl, sh1<T>(sc + G::O_CC + (crow * G::CW + cl) * 2), 0.f);
      Sc = __fmaf_rn(fxr, sh1<T>(sc + G::O_CC + (crow * G::CW + cr) * 2), Sc);
      Sc = __fmaf_rn(fyl, sh1<T>(sc + G::O_CC + (cym_r * G::CW + cc) * 2), Sc);
      Sc = __fmaf_rn(fyh, sh1<T>(sc + G::O_CC + (cyp_r * G::CW + cc) * 2), Sc);
      Sc = __fmaf_rn(fzl, sh1<T>(sm_ + G::O_CC + (crow * G::CW + cc) * 2), Sc);
      Sc = __fmaf_rn(fzh, sh1<T>(sp + G::O_CC + (crow * G::CW + cc) * 2), Sc);
      const float sg = a.corr_sign;
      S = __fmaf_rn(sg, Sc, S);
      pcf = __fmaf_rn(sg, wv, pcf);
    }
    if (scaled) {
      S = __fmul_rn(S, sc_);
      D = __fmul_rn(D, sc_);
    }
    return jacobi1(S, D, pcf, fr, om);
  };

  uint32_t fzlB[4] = {0u, 0u, 0u, 0u};  // B: faces below its plane (carried)
  double acc = 0.0;
  float cpart[V / 2];
#pragma unroll
  for (int e = 0; e < V / 2; ++e) cpart[e] = 0.f;

  bool mine = true;
  for (int p = z0 - 1; p <= z1 && ok; ++p) {
    if (__syncthreads_or(!mine)) {
      ok = false;
      break;
    }
    if (tid == 0 && p > z0 - 1 && p_next <= p_last) {
      const int q = p_next - p_first;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_plane_face2<T, PAIR, CORR, W>(a, smem + (q % NS) * G::STAGE, smem_u32(&bars[q % NS]), p_next, x0, y0, b);
      ++p_next;
    }
    mine = wait_plane(p + 1, a.wait_budget);
    const char *sm_ = stage_of(p - 1);
    const char *sc = stage_of(p);
    const char *sp = stage_of(p + 1);

    // ---- A at plane p into the ring (zero outside the grid)
    if (tid < G::AT) {
      char *dst = ring_of(p);
      const int gy = y0 + ra, gx = x0 + V * c;
      const bool row_in = p >= 0 && p < Z && gy >= 0 && gy < Y;
      uint32_t packed[4] = {0u, 0u, 0u, 0u};
      if (row_in && gx < X) {
        float res[8];
        a_group(sm_, sc, sp, res);
#pragma unroll
        for (int k = 0; k < 4; ++k) packed[k] = pack2<T>(res[2 * k], res[2 * k + 1]);
        if (PR && p >= z0 && p < z1 && ra >= 0 && ra < TY) {
          uint4 u;
          u.x = packed[0]; u.y = packed[1]; u.z = packed[2]; u.w = packed[3];
          *reinterpret_cast<uint4 *>(a.out + inst * a.stride + ((int64_t)p * Y + gy) * X + gx) = u;
        }
      }
      {
        uint4 u;
        u.x = packed[0]; u.y = packed[1]; u.z = packed[2]; u.w = packed[3];
        *reinterpret_cast<uint4 *>(dst + o1(ra, V * c)) = u;
      }
      if (c == 0) {
        const float v = (row_in && x0 > 0) ? a_one(sm_, sc, sp, -1) : 0.f;
        *reinterpret_cast<unsigned short *>(dst + o1(ra, -1)) = (unsigned short)(pack2<T>(v, 0.f) & 0xffffu);
      }
      if (c == G::TPR - 1) {
        const float v = (row_in && x0 + TX < X) ? a_one(sm_, sc, sp, TX) : 0.f;
        *reinterpret_cast<unsigned short *>(dst + o1(ra, TX)) = (unsigned short)(pack2<T>(v, 0.f) & 0xffffu);
      }
    }
    __syncthreads();

    // ---- B at plane z = p - 1 from the ring
    const int z = p - 1;
    if (tid < G::BT) {
      const char *sb = stage_of(z);
      uint32_t fzh[4];
      ld8w(sb + G::O_FZ + o1(rb, V * c), fzh);
      if (z >= z0) {
        const char *rc = ring_of(z), *rm = ring_of(z - 1), *rp = ring_of(z + 1);
        const int gy = y0 + rb, gx = x0 + V * c;
        const bool valid = gx < X && gy < Y;
        uint32_t pc[4], pym[4], pyp[4], pzm[4], pzp[4];
        ld8w(rc + o1(rb, V * c), pc);
        ld8w(rc + o1(rb - 1, V * c), pym);
        ld8w(rc + o1(rb + 1, V * c), pyp);
        ld8w(rm + o1(rb, V * c), pzm);
        ld8w(rp + o1(rb, V * c), pzp);
        const uint32_t pl = ld1w(rc + o1(rb, V * c - 1)), pr = ld1w(rc + o1(rb, V * c + V));
        uint32_t fx[4], fyl[4], fyh[4], fr[4];
        ld8w(sb + G::O_FX + o1(rb, V * c), fx);
        const uint32_t fx8 = ld1w(sb + G::O_FX + o1(rb, V * c + V));
        ld8w(sb + G::O_FY + o1(rb, V * c), fyl);
        ld8w(sb + G::O_FY + o1(rb + 1, V * c), fyh);
        if (PR)
          ld8w(sb + G::O_PHI + o2(rb, V * c), fr);
        else
          ld8w(sb + G::O_F + o1(rb, V * c), fr);
        float S[8], D[8];
        face_cell<T, 0>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 1>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 2>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 3>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 4>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 5>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 6>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        face_cell<T, 7>(pc, pl, pr, pym, pyp, pzm, pzp, fx, fx8, fyl, fyh, fzlB, fzh, S, D);
        float pcf[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float2 v = cvt2<T>(pc[k]);
          pcf[2 * k] = v.x;
          pcf[2 * k + 1] = v.y;
        }
        if (scaled) {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            S[e] *= sc_;
            D[e] *= sc_;
          }
        }
        float res[8];
        float pacc = 0.f;
        if (!PR) {
          const float2 om2 = make_float2(om, om);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
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
            const float t0 = M::template add<0>(fr[k], S[2 * k]), t1 = M::template add<1>(fr[k], S[2 * k + 1]);
            res[2 * k] = fmaf(D[2 * k], pcf[2 * k], -t0);
            res[2 * k + 1] = fmaf(D[2 * k + 1], pcf[2 * k + 1], -t1);
          }
        }
        uint32_t packed[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) packed[k] = pack2<T>(res[2 * k], res[2 * k + 1]);
        if (valid) {
          if (!PR && a.dot_rhs) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              pacc = M::template fma<0, 0>(packed[k], fr[k], pacc);
              pacc = M::template fma<1, 1>(packed[k], fr[k], pacc);
            }
          } else if (PR) {
#pragma unroll
            for (int e = 0; e < 8; ++e) pacc = fmaf(res[e], res[e], pacc);
          }
          acc += (double)pacc;
          if (!PR) {
            uint4 u;
            u.x = packed[0]; u.y = packed[1]; u.z = packed[2]; u.w = packed[3];
            *reinterpret_cast<uint4 *>(a.out + inst * a.stride + ((int64_t)z * Y + gy) * X + gx) = u;
          }
        }
        if (PR) {
#pragma unroll
          for (int k = 0; k < V / 2; ++k) {
            float pk = res[2 * k] + res[2 * k + 1];
            pk += __shfl_down_sync(0xffffffffu, pk, G::TPR);
            cpart[k] += 0.125f * pk;
          }
          if (z & 1) {
            if (valid && !(rb & 1)) {
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
#pragma unroll
      for (int k = 0; k < 4; ++k) fzlB[k] = fzh[k];
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
  if ((PR || a.dot_rhs) && a.partials) {
    double t = block_sum(acc);
    if (tid == 0) a.partials[inst * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}
