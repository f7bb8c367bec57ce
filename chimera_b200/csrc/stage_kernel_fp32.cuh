// stage_kernel_fp32.cuh -- the FP32-bulk stage kernel.
//
// Same stage operator and tile structure as stage_kernel (stage_kernel.cuh),
// with the freedom the FP32 form has (it is checked against the FP64 oracle in
// L1, not bit for bit) spent on fewer instructions per cell:
//   * phase 1.5 computes each cell's limited x and y slopes once into shared
//     memory (the FP64 kernel recomputes them for each face that touches the
//     cell, twice per direction), and the MOOD bounds either there too (SB)
//     or in phase 2, once per low cell for its x and y faces;
//   * FP32 min / max / abs are the single hardware instructions;
//   * the translation unit is compiled with fast FP32 division and square
//     root (-use_fast_math), about 1 ulp instead of correctly rounded;
//   * (TMA variants) the inputs of the CTA's next tile are loaded by TMA box
//     copies into the dead slope arrays while the current tile does
//     constrained transport and the cell update, so phase 1 reads shared
//     memory instead of waiting on HBM.  Tiles whose box would leave the
//     array (domain edges, where the index maps wrap or clamp) use the plain
//     loads.
// Kept in FP64: the pressure recovery p = (gamma-1)(E - rho v^2/2 - B^2/2)
// (get_primitive_mixed), the CFL dt reduction and the tOut clip, and the
// conserved-total sums.  The per-cell CFL speed is computed in FP32.
//
// Storage type S: float for the FP32-bulk form.  With S = double (the
// FP32-arithmetic form on FP64 storage) the state stays FP64 in HBM and only
// the reconstruction, limiter, MOOD and Riemann arithmetic (phases 1.5 and 2,
// and the corner Ez of phase 3a) run in FP32: the primitives are recovered in
// FP64 (get_primitive, then rounded to FP32), and the face-B update, the cell
// update, the outflow correction, the floors, the RK blends (the reference's
// forms) and the stage-3 epilogue (CFL speed, div B, |B|, totals) are the FP64
// kernel's arithmetic on the FP32 fluxes.
#pragma once
#include "stage_kernel.cuh"
#include "tma.cuh"

namespace chimera {

// Shared-memory plan.  SB: MOOD bounds stored per cell (12 arrays) or formed
// in phase 2 from the primitives.  The new face-B arrays of phase 3a
// reuse the slope arrays, which are dead once the face fluxes exist.
// TMA staging: the six input fields over the box [i0-4, i0-4+BW) x [j0-3,
// j0-3+BH) -- the primitives' 2-cell halo plus b_x(i-1), b_y(j-1) -- with the
// box origin's x a multiple of 4 floats (16 bytes), each field's box padded to
// 128 bytes, placed in the slope arrays after the face-B arrays.
template <int TX, int TY, bool SB> struct TileGeom32 : TileGeom<TX, TY> {
  using B = TileGeom<TX, TY>;
  static constexpr int SX = TX + 2, SY = TY + 2, NS = SX * SY;   // cells [i0-1, i0+TX] x [j0-1, j0+TY]
  static constexpr int NSA = SB ? 24 : 12;                       // per-cell arrays: slopes (+ bounds)
  static_assert(B::NBX + B::NBY <= 12 * NS, "face-B arrays must fit in the slope arrays");
  static constexpr int BW = ((TX + 6 + 3) / 4) * 4, BH = TY + 5;  // TMA box (floats)
  static constexpr int BOXF = ((BW * BH + 31) / 32) * 32;        // one field's box, 128-byte multiple
  static constexpr int STG0 = ((B::NBX + B::NBY + 31) / 32) * 32; // staging offset in the slope arrays
  static constexpr bool TMA_FITS = STG0 + 32 + 6 * BOXF <= 12 * NS;   // (+32: 128-byte alignment slack)
  static constexpr size_t smem_bytes() {
    return sizeof(float) * (size_t(6) * B::NP + size_t(NSA) * NS + size_t(5) * B::NFX + size_t(5) * B::NFY);
  }
};

// SSP-RK3 blends (src/main.f90:202-207, 261-266) written as U0 + c (U - U0):
// in FP32 the reference's form (1/3) U0 + (2/3) U has float(1/3) + float(2/3)
// = 1 + 3e-8, a systematic 3e-8 gain of every conserved total per step; this
// form conserves exactly what the stage update conserves.
template <int STAGE>
__device__ __forceinline__ float rk_blend(float u0, float u) {
  return (STAGE == 2) ? u0 + 0.25f * (u - u0) : u0 + (2.0f / 3.0f) * (u - u0);
}

// A new face B of stage STAGE: b + dt * db (the curl of the FP32 corner Ez),
// then the RK blend.  FP32 storage: FP32 arithmetic and the blend above; FP64
// storage: FP64 arithmetic and the reference's blend forms
// (src/main.f90:202-207, 261-266).
template <int STAGE>
__device__ __forceinline__ float blend_b(float b, float b0, float db, float dt, double) {
  float val = b + dt * db;
  if (STAGE >= 2) val = rk_blend<STAGE>(b0, val);
  return val;
}
template <int STAGE>
__device__ __forceinline__ double blend_b(double b, double b0, float db, float, double dt) {
  double val = b + dt * double(db);
  if (STAGE == 2) val = 0.75 * b0 + 0.25 * val;
  if (STAGE == 3) val = (1.0 / 3.0) * b0 + (2.0 / 3.0) * val;
  return val;
}

// The MC limiter (apply_slope_limiter, src/mhd_derivatives.f90:86-96) on a
// cell's x and y slopes at once: the adds and multiplies as sm_100's paired
// FP32 instructions (two lanes each, round to nearest like the scalar ones),
// the tests, absolute values and minima per lane -- the same bits as two
// scalar limit_slope<float, LIMITER_MC> calls.
__device__ __forceinline__ float2 limit_slope_mc2(float2 dfL, float2 dfR) {
  const float2 prod = __fmul2_rn(dfL, dfR);
  const float2 den = __fadd2_rn(dfL, dfR);
  const float2 aL = __fmul2_rn(make_float2(2.0f, 2.0f), make_float2(fabsf(dfL.x), fabsf(dfL.y)));
  const float2 aR = __fmul2_rn(make_float2(2.0f, 2.0f), make_float2(fabsf(dfR.x), fabsf(dfR.y)));
  const float2 aD = __fmul2_rn(make_float2(0.5f, 0.5f), make_float2(fabsf(den.x), fabsf(den.y)));
  const float2 m = make_float2(fminf(fminf(aL.x, aR.x), aD.x), fminf(fminf(aL.y, aR.y), aD.y));
  float2 r = __fmul2_rn(make_float2(copysignf(1.0f, dfL.x), copysignf(1.0f, dfL.y)), m);
  if (prod.x <= 0.0f || fabsf(den.x) < 1e-12f) r.x = 0.0f;
  if (prod.y <= 0.0f || fabsf(den.y) < 1e-12f) r.y = 0.0f;
  return r;
}

// rusanov_flux (src/mhd_flux.f90:197-288) in FP32, the same expressions as
// rusanov<float>, with the left and right states' identical work (magnetic,
// thermal and kinetic terms, total energy, fast speed) and the five flux
// corrections as lanes of sm_100's paired FP32 instructions.
__device__ __forceinline__ Flux5<float> rusanov_x2(float gamma, float rho_L, float rho_R, float vx_L, float vx_R,
                                                   float vy_L, float vy_R, float P_L, float P_R, float Bx_L,
                                                   float Bx_R, float By_L, float By_R) {
  const float2 half = make_float2(0.5f, 0.5f);
  const float2 rho = make_float2(rho_L, rho_R), vx = make_float2(vx_L, vx_R), vy = make_float2(vy_L, vy_R);
  const float2 Bx = make_float2(Bx_L, Bx_R), By = make_float2(By_L, By_R);
  const float2 halfB2 = __fmul2_rn(half, __ffma2_rn(Bx, Bx, __fmul2_rn(By, By)));
  float2 p_th = __fadd2_rn(make_float2(P_L, P_R), make_float2(-halfB2.x, -halfB2.y));
  p_th.x = fmaxf(p_th.x, 1.0e-12f);
  p_th.y = fmaxf(p_th.y, 1.0e-12f);
  const float gm1 = gamma - 1.0f;
  const float igm1 = 1.0f / gm1;
  const float2 ke = __fmul2_rn(__fmul2_rn(half, rho), __ffma2_rn(vx, vx, __fmul2_rn(vy, vy)));
  const float2 en = __fadd2_rn(__ffma2_rn(p_th, make_float2(igm1, igm1), ke), halfB2);
  const float2 mx = __fmul2_rn(rho, vx), my = __fmul2_rn(rho, vy);
  const float rho_avg = 0.5f * (rho_L + rho_R);
  const float inv_rho_avg = 1.0f / rho_avg;
  const float momx_avg = 0.5f * (mx.x + mx.y);
  const float momy_avg = 0.5f * (my.x + my.y);
  const float en_avg = 0.5f * (en.x + en.y);
  const float Bx_avg = 0.5f * (Bx_L + Bx_R);
  const float By_avg = 0.5f * (By_L + By_R);
  const float hB = 0.5f * (Bx_avg * Bx_avg + By_avg * By_avg);
  const float P_avg = gm1 * ((en_avg - 0.5f * (momx_avg * momx_avg + momy_avg * momy_avg) * inv_rho_avg) - hB) + hB;
  Flux5<float> F;
  F.mass = momx_avg;
  F.momn = (momx_avg * momx_avg * inv_rho_avg + P_avg) - Bx_avg * Bx_avg;
  F.momt = momx_avg * momy_avg * inv_rho_avg - Bx_avg * By_avg;
  F.energy = (en_avg + P_avg) * momx_avg * inv_rho_avg -
             Bx_avg * (Bx_avg * momx_avg + By_avg * momy_avg) * inv_rho_avg;
  F.bt = (By_avg * momx_avg - Bx_avg * momy_avg) * inv_rho_avg;
  // c^2 = (gamma p_th + B^2) / rho > 0 (the thermal pressure is floored)
  const float2 c2 = __fmul2_rn(__ffma2_rn(make_float2(gamma, gamma), p_th, __fmul2_rn(make_float2(2.0f, 2.0f), halfB2)),
                               make_float2(1.0f / rho_L, 1.0f / rho_R));
  const float2 h = __fmul2_rn(half, __fadd2_rn(c2, make_float2(fabsf(c2.x), fabsf(c2.y))));
  const float2 Cs = __fadd2_rn(make_float2(sqrtf(h.x), sqrtf(h.y)), make_float2(fabsf(vx_L), fabsf(vx_R)));
  const float C = 0.5f * fmaxf(Cs.x, Cs.y);
  const float2 nC = make_float2(-C, -C);
  const float2 f01 = __ffma2_rn(nC, __fadd2_rn(make_float2(rho_R, mx.y), make_float2(-rho_L, -mx.x)),
                                make_float2(F.mass, F.momn));
  const float2 f23 = __ffma2_rn(nC, __fadd2_rn(make_float2(my.y, en.y), make_float2(-my.x, -en.x)),
                                make_float2(F.momt, F.energy));
  F.mass = f01.x; F.momn = f01.y; F.momt = f23.x; F.energy = f23.y;
  F.bt = F.bt - C * (By_R - By_L);
  return F;
}

// Whether work item w's input box lies inside its member's arrays (and the
// member has tensor maps): then it is loaded by TMA.
template <int TX, int TY, int BW, int BH>
__device__ __forceinline__ bool tma_tile(const StageArgs& a, int w) {
  const int m = (a.n_members == 1) ? 0 : a.tile_member[w];
  const Member& g = a.members[m];
  if (!g.tmap) return false;
  const int lt = w - g.tile_begin;
  const int i0 = (lt % g.tiles_x) * TX, j0 = (lt / g.tiles_x) * TY;
  return i0 >= 4 && i0 - 4 + BW <= g.nx && j0 >= 3 && j0 - 3 + BH <= g.ny;
}

// Thread 0: issue the six box loads of work item w's stage input.
template <int STAGE, int TX, int TY, int BW, int BH, int BOXF>
__device__ __forceinline__ void tma_issue(const StageArgs& a, int w, float* stg, uint64_t* bar) {
  const int m = (a.n_members == 1) ? 0 : a.tile_member[w];
  const Member& g = a.members[m];
  const int lt = w - g.tile_begin;
  const int i0 = (lt % g.tiles_x) * TX, j0 = (lt / g.tiles_x) * TY;
  const int sbuf = a.ctl[m].parity;
  const int in_buf = (STAGE == 1) ? sbuf : (STAGE == 2 ? 1 - sbuf : 2);
  const char* maps = reinterpret_cast<const char*>(g.tmap) + size_t(in_buf) * 6 * TMAP_BYTES;
  mbar_arrive_expect_tx(bar, unsigned(6 * BW * BH * sizeof(float)));
#pragma unroll
  for (int q = 0; q < 6; ++q) tma_load_2d(stg + q * BOXF, maps + q * TMAP_BYTES, i0 - 4, j0 - 3, bar);
}

template <int SOLVER, int STAGE, int TX, int TY, int NT, int MINB, bool SB, bool TMA, typename S = float,
          bool MIXBC = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel_f32(StageArgs a) {
  using G = TileGeom32<TX, TY, SB>;
  static_assert(!TMA || G::TMA_FITS, "TMA staging must fit in the slope arrays");
  constexpr bool MIX = sizeof(S) == 8;   // FP64 storage, FP32 flux arithmetic
  static_assert(!(TMA && MIX), "the TMA staging holds FP32 boxes");
  static_assert(!MIX || 2 * (G::NBX + G::NBY) <= 12 * G::NS, "FP64 face-B arrays must fit in the slope arrays");
  using R = float;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw);       // [6][NP]   primitives, tile + 2 halo
  R* sS = sP + 6 * G::NP;                       // [12][NS]  slopes: field q, dir d at (2q+d)
  R* sLo = sS + 12 * G::NS;                     // [6][NS]   MOOD lower bounds (SB)
  R* sHi = sLo + 6 * G::NS;                     // [6][NS]   MOOD upper bounds (SB)
  R* sFx = sS + G::NSA * G::NS;                 // [5][NFX]
  R* sFy = sFx + 5 * G::NFX;                    // [5][NFY]
  S* sBx = reinterpret_cast<S*>(sS);            // new face B (phase 3a on): reuses the slopes
  S* sBy = sBx + G::NBX;
  __shared__ double red[6 * (NT / 32)];
  __shared__ int s_last;
  __shared__ unsigned s_own;   // stage 3: bit r set if tile row r is one of the grid's own rows
  static_assert(TY < 32, "the own-row mask holds one bit per tile row");
  __shared__ __align__(8) uint64_t s_bar;    // TMA completion
  // TMA pipeline state, kept in shared memory rather than in a register that
  // would stay live through the register-bound flux phase: bit 0 = this tile's
  // inputs come by TMA, bit 1 = the barrier parity to wait for.  Thread 0
  // rewrites it only between barriers that every thread's reads precede.
  __shared__ unsigned s_tma;

  const int tid = threadIdx.x;
  const bool slope_on = a.slope_limiting != 0;
  const bool mood_on = a.mood != 0;
  const bool van_leer = a.limiter == LIMITER_VAN_LEER;
  // TMA staging area in the slope arrays, 128-byte aligned (recomputed where used)
  auto staging = [&]() {
    return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(sS + G::STG0) + 127) & ~uintptr_t(127));
  };
  constexpr unsigned TMA_POLLS = 1u << 26;   // bound of every wait for a TMA completion
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(&s_bar, 1);
      const int w0 = a.work_begin + int(blockIdx.x);
      const bool st = w0 < a.total_tiles && tma_tile<TX, TY, G::BW, G::BH>(a, w0);
      s_tma = st ? 1u : 0u;
      if (st) tma_issue<STAGE, TX, TY, G::BW, G::BH, G::BOXF>(a, w0, staging(), &s_bar);
    }
    __syncthreads();
  }

  for (int w = a.work_begin + blockIdx.x; w < a.total_tiles; w += gridDim.x) {
    const int m = (a.n_members == 1) ? 0 : a.tile_member[w];
    const Member& g = a.members[m];
    Control* ctl = a.ctl + m;
    if (ctl->active == 0) {
      if (TMA && (s_tma & 1u)) {   // a copy was issued for this tile: consume it to keep the phases paired
        const bool ok = mbar_wait(&s_bar, (s_tma >> 1) & 1u, TMA_POLLS);
        if (__syncthreads_or(!ok)) {   // a copy that never lands sets the status word and ends the kernel
          if (tid == 0) {
            atomicOr(&ctl->status, STATUS_TIMEOUT);
            mbar_wait(&s_bar, (s_tma >> 1) & 1u, TMA_POLLS);   // a last bounded wait for the copy in flight
          }
          return;
        }
        if (tid == 0) s_tma = (s_tma ^ 2u) & ~1u;
        __syncthreads();
      }
      continue;
    }
    const int nx = g.nx, ny = g.ny;
    const int px = g.periodic_x, py = g.periodic_y;                   // low sides
    // high sides: they differ from the low sides only in a mixed pair (MIXBC
    // instantiations), where a cell wrapped across the pair sees its neighbour
    // across the non-periodic side as itself, as the cell it copies does
    const int pxh = MIXBC ? g.periodic_xhi : px, pyh = MIXBC ? g.periodic_yhi : py;
    const int lt = w - g.tile_begin;
    const int i0 = (lt % g.tiles_x) * TX;
    const int j0 = (lt / g.tiles_x) * TY;
    if (STAGE == 3 && tid == 0) {
      // the tile rows whose cells enter the epilogue's reductions: all but a
      // y-slab's ghost rows (read in phase 3b, after phase 1's barrier; the
      // previous tile's reads ended before its closing barrier)
      const int lo = min(max(g.skip_lo - j0, 0), TY), hi = min(max(ny - g.skip_hi - j0, 0), TY);
      s_own = ((1u << hi) - 1u) & ~((1u << lo) - 1u);
    }
    const R gamma = R(g.gamma);
    const R vol = R(g.vol);
    const double dt64 = ctl->dt;
    const R dt = R(dt64);
    const int sbuf = ctl->parity, obuf = 1 - sbuf;
    const int in_buf = (STAGE == 1) ? sbuf : (STAGE == 2 ? obuf : 2);
    const int out_buf = (STAGE == 2) ? 2 : obuf;
    // FP64 storage: set after phase 2 instead (see there)
    const S* __restrict__ in[6];
    const S* __restrict__ u0[6];
    S* __restrict__ out[6];
    if constexpr (!MIX) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        in[q] = reinterpret_cast<const S*>(g.buf[in_buf][q]);
        u0[q] = reinterpret_cast<const S*>(g.buf[sbuf][q]);
        out[q] = reinterpret_cast<S*>(g.buf[out_buf][q]);
      }
    }
    {
      const int wn = w + gridDim.x;   // the next tile's inputs are prefetched to L2 unless TMA loads them
      prefetch_next_tile<S, TX, TY, NT, STAGE>(
          a, wn, !(TMA && wn < a.total_tiles && tma_tile<TX, TY, G::BW, G::BH>(a, wn)));
    }

    // ---- phase 1: primitives (FP64 pressure recovery) -------------------------
    bool tma_bad = false;
    if (TMA && (s_tma & 1u)) {
      // from the TMA box: element (x, y) of the box is cell (i0-4+x, j0-3+y); the
      // box lies inside the arrays, so both face-B averages apply
      const float* stg = staging();
      tma_bad = !mbar_wait(&s_bar, (s_tma >> 1) & 1u, TMA_POLLS);
      for (int p = tid; p < G::NP && !tma_bad; p += NT) {
        const int qx = p % G::PX, qy = p / G::PX;
        const int b = (qy + 1) * G::BW + (qx + 2);
        const R Bx = R(0.5) * (stg[4 * G::BOXF + b] + stg[4 * G::BOXF + b - 1]);
        const R By = R(0.5) * (stg[5 * G::BOXF + b] + stg[5 * G::BOXF + b - G::BW]);
        const Prim<R> pr = get_primitive_mixed(stg[b], stg[G::BOXF + b], stg[2 * G::BOXF + b],
                                               stg[3 * G::BOXF + b], Bx, By, g.gamma, g.inv_vol,
                                               float(g.inv_vol));
        sP[0 * G::NP + p] = pr.rho;
        sP[1 * G::NP + p] = pr.vx;
        sP[2 * G::NP + p] = pr.vy;
        sP[3 * G::NP + p] = pr.P;
        sP[4 * G::NP + p] = pr.Bx;
        sP[5 * G::NP + p] = pr.By;
      }
    } else if constexpr (MIX) {
      // FP64 storage: one element at a time, as the FP64 kernel (eight FP64
      // loads per element in flight at once would spill); FP64 recovery
      // (src/mhd_change_states.f90:61-113), rounded to FP32
      const S* __restrict__ src[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) src[q] = reinterpret_cast<const S*>(g.buf[in_buf][q]);
      for (int p = tid; p < G::NP; p += NT) {
        const int qx = p % G::PX, qy = p / G::PX;
        const int si = map_index(i0 - 2 + qx, nx, px, pxh);
        const int sj = map_index(j0 - 2 + qy, ny, py, pyh);
        const size_t idx = size_t(sj) * nx + si;
        const double bxc = src[4][idx], byc = src[5][idx];
        double Bx, By;
        if (si > 0) Bx = 0.5 * (bxc + src[4][idx - 1]);
        else Bx = px ? 0.5 * (bxc + src[4][idx + (nx - 1)]) : bxc;
        if (sj > 0) By = 0.5 * (byc + src[5][idx - nx]);
        else By = py ? 0.5 * (byc + src[5][idx + size_t(ny - 1) * nx]) : byc;
        const Prim<double> pd = get_primitive<double>(src[0][idx], src[1][idx], src[2][idx], src[3][idx], Bx, By,
                                                      g.gamma, g.vol, g.rcp_vol);
        sP[0 * G::NP + p] = float(pd.rho);
        sP[1 * G::NP + p] = float(pd.vx);
        sP[2 * G::NP + p] = float(pd.vy);
        sP[3 * G::NP + p] = float(pd.P);
        sP[4 * G::NP + p] = float(pd.Bx);
        sP[5 * G::NP + p] = float(pd.By);
      }
    } else {
      // all of this thread's loads are issued before any arithmetic (memory-level parallelism)
      constexpr int KP = (G::NP + NT - 1) / NT;
      S ld[KP][8];
#pragma unroll
      for (int k = 0; k < KP; ++k) {
        const int p = tid + k * NT;
        if (p < G::NP) {
          const int qx = p % G::PX, qy = p / G::PX;
          const int si = map_index(i0 - 2 + qx, nx, px, pxh);
          const int sj = map_index(j0 - 2 + qy, ny, py, pyh);
          const size_t idx = size_t(sj) * nx + si;
          const size_t ixm = (si > 0) ? idx - 1 : (px ? idx + (nx - 1) : idx);
          const size_t iym = (sj > 0) ? idx - nx : (py ? idx + size_t(ny - 1) * nx : idx);
          ld[k][0] = in[0][idx]; ld[k][1] = in[1][idx]; ld[k][2] = in[2][idx]; ld[k][3] = in[3][idx];
          ld[k][4] = in[4][idx]; ld[k][5] = in[4][ixm]; ld[k][6] = in[5][idx]; ld[k][7] = in[5][iym];
        }
      }
#pragma unroll
      for (int k = 0; k < KP; ++k) {
        const int p = tid + k * NT;
        if (p < G::NP) {
          const int qx = p % G::PX, qy = p / G::PX;
          const int si = map_index(i0 - 2 + qx, nx, px, pxh);
          const int sj = map_index(j0 - 2 + qy, ny, py, pyh);
          const S Bx = (si > 0 || px) ? S(0.5) * (ld[k][4] + ld[k][5]) : ld[k][4];
          const S By = (sj > 0 || py) ? S(0.5) * (ld[k][6] + ld[k][7]) : ld[k][6];
          const Prim<R> pr = get_primitive_mixed(ld[k][0], ld[k][1], ld[k][2], ld[k][3], Bx, By, g.gamma,
                                                 g.inv_vol, float(g.inv_vol));
          sP[0 * G::NP + p] = pr.rho;
          sP[1 * G::NP + p] = pr.vx;
          sP[2 * G::NP + p] = pr.vy;
          sP[3 * G::NP + p] = pr.P;
          sP[4 * G::NP + p] = pr.Bx;
          sP[5 * G::NP + p] = pr.By;
        }
      }
    }
    if constexpr (TMA) {
      if (__syncthreads_or(tma_bad)) {   // a copy that never lands sets the status word and ends the kernel
        if (tid == 0) {
          atomicOr(&ctl->status, STATUS_TIMEOUT);
          mbar_wait(&s_bar, (s_tma >> 1) & 1u, TMA_POLLS);   // a last bounded wait for the copy in flight
        }
        return;
      }
    } else {
      __syncthreads();
    }


    // ---- phase 1.5: per-cell slopes and MOOD bounds -----------------------------
    // apply_slope_limiter (src/mhd_derivatives.f90:50-127) or compute_gradients
    // (:15-47); bounds of the 5-point stencil with the rho/P floor (:190-211).
    const R inv_dx = R(g.inv_dx), inv_dy = R(g.inv_dy);
    const R inv_2dx = R(g.inv_2dx), inv_2dy = R(g.inv_2dy);
    for (int c = tid; c < G::NS; c += NT) {
      const int cx = c % G::SX, cy = c / G::SX;
      const int pc = (cy + 1) * G::PX + (cx + 1);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const R* s = sP + q * G::NP;
        R f0 = s[pc], xm = s[pc - 1], xp = s[pc + 1], ym = s[pc - G::PX], yp = s[pc + G::PX];
        if constexpr (MIXBC) {
          const int gx = i0 + cx - 1, gy = j0 + cy - 1;   // this cell, wrapped across a mixed pair?
          if (px && !pxh && gx == -1) xp = f0;
          if (!px && pxh && gx == nx) xm = f0;
          if (py && !pyh && gy == -1) yp = f0;
          if (!py && pyh && gy == ny) ym = f0;
        }
        R sx, sy;
        if (slope_on) {
          if (van_leer) {
            sx = limit_slope<R, LIMITER_VAN_LEER>((f0 - xm) * inv_dx, (xp - f0) * inv_dx);
            sy = limit_slope<R, LIMITER_VAN_LEER>((f0 - ym) * inv_dy, (yp - f0) * inv_dy);
          } else {   // x and y lanes together (paired FP32 instructions)
            const float2 inv = make_float2(inv_dx, inv_dy);
            const float2 dfL = __fmul2_rn(__fadd2_rn(make_float2(f0, f0), make_float2(-xm, -ym)), inv);
            const float2 dfR = __fmul2_rn(__fadd2_rn(make_float2(xp, yp), make_float2(-f0, -f0)), inv);
            const float2 sl = limit_slope_mc2(dfL, dfR);
            sx = sl.x;
            sy = sl.y;
          }
        } else {
          sx = (xp - xm) * inv_2dx;
          sy = (yp - ym) * inv_2dy;
        }
        sS[(2 * q + 0) * G::NS + c] = sx;
        sS[(2 * q + 1) * G::NS + c] = sy;
        if (SB && mood_on) {
          R lo = fminf(fminf(fminf(fminf(f0, xp), xm), yp), ym);
          const R hi = fmaxf(fmaxf(fmaxf(fmaxf(f0, xp), xm), yp), ym);
          if (q == 0 || q == 3) lo = fmaxf(R(0.1e-8), lo);
          sLo[q * G::NS + c] = lo;
          sHi[q * G::NS + c] = hi;
        }
      }
    }
    __syncthreads();

    // ---- phase 2: face fluxes ------------------------------------------------------
    // One work item per low cell of the slope grid: its x face (i+1/2, j) and
    // its y face (i, j+1/2), where the tile needs them, share the cell's MOOD
    // bounds (the 5-point stencil of src/mhd_derivatives.f90:190-211), which
    // are formed once (SB: loaded once).
    unsigned mood_resets = 0;
    for (int c = tid; c < G::NS; c += NT) {
      const int cx = c % G::SX, cy = c / G::SX;
      const int pa = (cy + 1) * G::PX + (cx + 1);             // the low cell in the primitive grid
      R lo[6], hi[6];
      if (mood_on) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          if (SB) {
            lo[q] = sLo[q * G::NS + c];
            hi[q] = sHi[q * G::NS + c];
          } else {
            const R* s = sP + q * G::NP;
            const R f0 = s[pa];
            R xp = s[pa + 1], xm = s[pa - 1], yp = s[pa + G::PX], ym = s[pa - G::PX];
            if constexpr (MIXBC) {
              const int gx = i0 + cx - 1, gy = j0 + cy - 1;
              if (px && !pxh && gx == -1) xp = f0;
              if (!px && pxh && gx == nx) xm = f0;
              if (py && !pyh && gy == -1) yp = f0;
              if (!py && pyh && gy == ny) ym = f0;
            }
            R l = fminf(fminf(fminf(fminf(f0, xp), xm), yp), ym);
            hi[q] = fmaxf(fmaxf(fmaxf(fmaxf(f0, xp), xm), yp), ym);
            if (q == 0 || q == 3) l = fmaxf(R(0.1e-8), l);
            lo[q] = l;
          }
        }
      }
#pragma unroll 1
      for (int d = 0; d < 2; ++d) {
        const bool ydir = d == 1;
        if (ydir ? (cy >= G::SY - 1) : (cx >= G::SX - 1)) continue;   // face outside the tile's set
        const int ff = ydir ? cy * G::FYW + cx : cy * G::FXW + cx;
        const int sb = c + (ydir ? G::SX : 1);                // high cell in the slope grid
        const int pb = pa + (ydir ? G::PX : 1);
        const R hh = R(ydir ? g.hy : g.hx);
        R L[6], Rv[6];
        bool reset = false;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const R f0 = sP[q * G::NP + pa], fp = sP[q * G::NP + pb];
          // left and right states as the two lanes of one paired FP32 multiply-add
          const float2 v = __ffma2_rn(make_float2(hh, -hh),
                                      make_float2(sS[(2 * q + d) * G::NS + c], sS[(2 * q + d) * G::NS + sb]),
                                      make_float2(f0, fp));
          R vL = v.x;
          R vR = v.y;
          if constexpr (MIXBC) {
            // the face below x = 0 (y = 0) with that side periodic and the far
            // side outflow is the far side's outflow face: its high cell is the
            // low cell's own ghost (value f0, zero slope)
            const int gl = ydir ? j0 + cy - 1 : i0 + cx - 1;
            if (gl == -1 && (ydir ? (py && !pyh) : (px && !pxh))) vR = f0;
          }
          if (mood_on) {   // bounds of the LOW cell, reset to its value (src/mhd_derivatives.f90:213-216)
            if (vL < lo[q] || vL > hi[q]) { vL = f0; reset = true; }
            if (vR < lo[q] || vR > hi[q]) { vR = f0; reset = true; }
          }
          if (q == 0 || q == 3) {
            vL = fmaxf(vL, R(1.0e-8));
            vR = fmaxf(vR, R(1.0e-8));
          }
          L[q] = vL; Rv[q] = vR;
        }
        if (L[3] - R(0.5) * (L[4] * L[4] + L[5] * L[5]) < K<R>::P_floor) {
#pragma unroll
          for (int q = 0; q < 6; ++q) L[q] = sP[q * G::NP + pa];
        }
        if (Rv[3] - R(0.5) * (Rv[4] * Rv[4] + Rv[5] * Rv[5]) < K<R>::P_floor) {
#pragma unroll
          for (int q = 0; q < 6; ++q) Rv[q] = sP[q * G::NP + pa];
        }
        mood_resets += reset ? 1u : 0u;
        const R unL = ydir ? L[2] : L[1], unR = ydir ? Rv[2] : Rv[1];
        const R utL = ydir ? L[1] : L[2], utR = ydir ? Rv[1] : Rv[2];
        const R bnL = ydir ? L[5] : L[4], bnR = ydir ? Rv[5] : Rv[4];
        const R btL = ydir ? L[4] : L[5], btR = ydir ? Rv[4] : Rv[5];
        Flux5<R> F;
        if constexpr (SOLVER == RIEMANN_RUSANOV)
          F = rusanov_x2(gamma, L[0], Rv[0], unL, unR, utL, utR, L[3], Rv[3], bnL, bnR, btL, btR);
        else
          F = riemann<R, SOLVER>(gamma, L[0], Rv[0], unL, unR, utL, utR, L[3], Rv[3], bnL, bnR, btL, btR);
        R* dst = ydir ? sFy : sFx;
        const int NF = ydir ? G::NFY : G::NFX;
        dst[0 * NF + ff] = F.mass;
        dst[1 * NF + ff] = ydir ? F.momt : F.momn;
        dst[2 * NF + ff] = ydir ? F.momn : F.momt;
        dst[3 * NF + ff] = F.energy;
        dst[4 * NF + ff] = F.bt;
      }
    }
    if (a.counters && !a.dry) {
      unsigned s = __reduce_add_sync(0xffffffffu, mood_resets);
      if ((tid & 31) == 0 && s) atomicAdd(&ctl->mood_resets, (unsigned long long)s);
    }
    __syncthreads();
    // the slopes are dead: the next tile's inputs stream in during phases 3a / 3b
    if constexpr (TMA) {
      if (tid == 0) {
        const unsigned st = s_tma;     // this tile's state (every thread read it before phase 1's barrier)
        const unsigned parity = ((st >> 1) ^ st) & 1u;   // flips if this tile consumed a completion
        const int wn = w + gridDim.x;
        const bool next = wn < a.total_tiles && tma_tile<TX, TY, G::BW, G::BH>(a, wn);
        s_tma = (next ? 1u : 0u) | (parity << 1);
        if (next) {
          fence_proxy_async_smem();
          tma_issue<STAGE, TX, TY, G::BW, G::BH, G::BOXF>(a, wn, staging(), &s_bar);
        }
      }
    }

    if constexpr (MIX) {
      // the buffer pointers, read here rather than kept in registers through
      // phases 1.5 and 2 (as the FP64 kernel does)
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        in[q] = static_cast<const S*>(load_ptr(&g.buf[in_buf][q]));
        u0[q] = static_cast<const S*>(load_ptr(&g.buf[sbuf][q]));
        out[q] = static_cast<S*>(load_ptr(&g.buf[out_buf][q]));
      }
    }

    // ---- phase 3a: constrained transport -> new face B ----------------------------
    const R* FByX = sFx + 4 * G::NFX;
    const R* FBxY = sFy + 4 * G::NFY;
    // corner Ez (src/mhd_flux.f90:79-136) at two corners, as the lanes of paired FP32 adds and a
    // multiply: 0.25 (((-FByX(i,j) - FByX(i,j+1)) + FBxY(i,j)) + FBxY(i+1,j)), zero-gradient at
    // non-periodic top / right
    auto Ez2 = [&](int ci0, int cj0, int ci1, int cj1) -> float2 {
      const int xi0 = (cj0 - j0 + 1) * G::FXW + (ci0 - i0 + 1), xi1 = (cj1 - j0 + 1) * G::FXW + (ci1 - i0 + 1);
      const int yi0 = (cj0 - j0 + 1) * G::FYW + (ci0 - i0 + 1), yi1 = (cj1 - j0 + 1) * G::FYW + (ci1 - i0 + 1);
      const R fa0 = FByX[xi0], fa1 = FByX[xi1];
      // (also for the corner row below y = 0 that wraps to a non-periodic top: mixed pair)
      const bool u0own = (cj0 == ny - 1 && !pyh) || (MIXBC && cj0 == -1 && py && !pyh);
      const bool u1own = (cj1 == ny - 1 && !pyh) || (MIXBC && cj1 == -1 && py && !pyh);
      const R up0 = u0own ? fa0 : FByX[xi0 + G::FXW];
      const R up1 = u1own ? fa1 : FByX[xi1 + G::FXW];
      const R fb0 = FBxY[yi0], fb1 = FBxY[yi1];
      const bool r0own = (ci0 == nx - 1 && !pxh) || (MIXBC && ci0 == -1 && px && !pxh);
      const bool r1own = (ci1 == nx - 1 && !pxh) || (MIXBC && ci1 == -1 && px && !pxh);
      const R rt0 = r0own ? fb0 : FBxY[yi0 + 1];
      const R rt1 = r1own ? fb1 : FBxY[yi1 + 1];
      float2 t = __fadd2_rn(make_float2(-fa0, -fa1), make_float2(-up0, -up1));
      t = __fadd2_rn(t, make_float2(fb0, fb1));
      t = __fadd2_rn(t, make_float2(rt0, rt1));
      return __fmul2_rn(make_float2(0.25f, 0.25f), t);
    };
    const int bx_lo = (STAGE == 3 && (i0 > 0 || px)) ? -1 : 0;
    const int by_lo = (STAGE == 3 && (j0 > 0 || py)) ? -1 : 0;
    for (int e = tid; e < G::NBX + G::NBY; e += NT) {
      const bool isy = e >= G::NBX;
      const int ee = isy ? e - G::NBX : e;
      int li, lj;
      if (!isy) { li = ee % G::BXW - 1; lj = ee / G::BXW; }
      else { li = ee % G::BYW; lj = ee / G::BYW - 1; }
      const int i = i0 + li, j = j0 + lj;
      if ((!isy && li < bx_lo) || (isy && lj < by_lo)) continue;
      if (i >= nx || j >= ny) continue;
      const int gi = (i < 0) ? i + nx : i;
      const int gj = (j < 0) ? j + ny : j;
      const size_t idx = size_t(gj) * nx + gi;
      S val;
      if (!isy) {
        const bool inner = j > 0 || py;
        const float2 e = Ez2(i, j, i, inner ? j - 1 : 1);
        const R dbx = inner ? ((-e.x) - (-e.y)) * inv_dy : ((-e.y) - (-e.x)) * inv_dy;   // outflow ylo: copy row 2
        val = blend_b<STAGE>(in[4][idx], u0[4][idx], dbx, dt, dt64);
        if (STAGE == 3) sBx[lj * G::BXW + (li + 1)] = val;   // the epilogue reads neighbours' new B
        else out[4][idx] = val;                                // stages 1, 2: straight to the output
      } else {
        const bool inner = i > 0 || px;
        const float2 e = Ez2(i, j, inner ? i - 1 : 1, j);
        const R dby = inner ? -(((-e.x) - (-e.y)) * inv_dx) : -(((-e.y) - (-e.x)) * inv_dx);   // outflow xlo: copy column 2
        val = blend_b<STAGE>(in[5][idx], u0[5][idx], dby, dt, dt64);
        if (STAGE == 3) sBy[(lj + 1) * G::BYW + li] = val;
        else out[5][idx] = val;
      }
    }
    if (STAGE == 3) __syncthreads();   // stages 1, 2 read no phase-3a result in phase 3b

    // ---- phase 3b: cell update --------------------------------------------------------
    double e_speed = 0.0, e_dmax = 0.0, e_dsum = 0.0, e_bmax = 0.0, e_mass = 0.0, e_en = 0.0;
    unsigned floor_hits = 0;
    const R ax = dt * R(g.dy);
    const R ay = dt * R(g.dx);
    for (int c = tid; c < TX * TY; c += NT) {
      const int li = c % TX, lj = c / TX;
      const int i = i0 + li, j = j0 + lj;
      if (i >= nx || j >= ny) continue;
      const size_t idx = size_t(j) * nx + i;
      const int fxr = (lj + 1) * G::FXW + (li + 1);
      const int fyt = (lj + 1) * G::FYW + (li + 1);
      if constexpr (MIX) {
        // FP64 storage: the FP64 kernel's update on the FP32 fluxes --
        // update_conserved (src/mhd_flux.f90:20-76), x pass then y pass,
        // apply_conserved_floors with the stage's cell B, the outflow boundary
        // correction (src/main.f90:118-148), the RK blend + floors
        // (src/main.f90:202-208, 261-267)
        const double ax64 = dt64 * g.dy, ay64 = dt64 * g.dx;
        double U[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double F = in[q][idx];
          const R* fx = sFx + q * G::NFX;
          const R* fy = sFy + q * G::NFY;
          if (i > 0 || px) F = (F - ax64 * double(fx[fxr])) + ax64 * double(fx[fxr - 1]);
          else F = F - ax64 * double(fx[fxr]);
          if (j > 0 || py) F = (F - ay64 * double(fy[fyt])) + ay64 * double(fy[fyt - G::FYW]);
          else F = F - ay64 * double(fy[fyt]);
          U[q] = F;
        }
        const int pc = (lj + 2) * G::PX + (li + 2);
        const double cr = sP[0 * G::NP + pc], cu = sP[1 * G::NP + pc], cv = sP[2 * G::NP + pc];
        const double cP = sP[3 * G::NP + pc], cBx = sP[4 * G::NP + pc], cBy = sP[5 * G::NP + pc];
        floor_hits += conserved_floors<double>(U[0], U[1], U[2], U[3], cBx, cBy, g.gamma, g.vol) ? 1u : 0u;
        if (!px && i == 0) {
          const double hb = 0.5 * (cBx * cBx + cBy * cBy);
          const double en = ((cP - hb) / (g.gamma - 1.0) + 0.5 * cr * (cu * cu + cv * cv)) + hb;
          U[0] = U[0] + ax64 * cr * cu;
          U[1] = U[1] + ax64 * ((cr * (cu * cu) + cP) - cBx * cBx);
          U[2] = U[2] + ax64 * (cr * cu * cv - cBx * cBy);
          U[3] = U[3] + ax64 * ((en + cP) * cu - cBx * (cBx * cu + cBy * cv));
        }
        if (!py && j == 0) {
          const double hb = 0.5 * (cBx * cBx + cBy * cBy);
          const double en = ((cP - hb) / (g.gamma - 1.0) + 0.5 * cr * (cu * cu + cv * cv)) + hb;
          U[0] = U[0] + ay64 * cr * cv;
          U[2] = U[2] + ay64 * ((cr * (cv * cv) + cP) - cBy * cBy);
          U[1] = U[1] + ay64 * (cr * cv * cu - cBy * cBx);
          U[3] = U[3] + ay64 * ((en + cP) * cv - cBy * (cBy * cv + cBx * cu));
        }
        if (STAGE == 2) {
#pragma unroll
          for (int q = 0; q < 4; ++q) U[q] = 0.75 * u0[q][idx] + 0.25 * U[q];
        }
        if (STAGE == 3) {
#pragma unroll
          for (int q = 0; q < 4; ++q) U[q] = (1.0 / 3.0) * u0[q][idx] + (2.0 / 3.0) * U[q];
        }
        if (STAGE >= 2)
          floor_hits += conserved_floors<double>(U[0], U[1], U[2], U[3], cBx, cBy, g.gamma, g.vol) ? 1u : 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q][idx] = U[q];
        if (STAGE == 3) {
          const double bxn = sBx[lj * G::BXW + (li + 1)];
          const double byn = sBy[(lj + 1) * G::BYW + li];
          out[4][idx] = bxn;
          out[5][idx] = byn;
          if ((s_own >> lj) & 1u) {   // the FP64 epilogue (the CFL kernel's arithmetic)
            const double bxm = sBx[lj * G::BXW + li];
            const double bym = sBy[lj * G::BYW + li];
            const bool hx = (i > 0) || px, hy = (j > 0) || py;
            const double Bx = hx ? 0.5 * (bxn + bxm) : bxn;
            const double By = hy ? 0.5 * (byn + bym) : byn;
            const Prim<double> pr = get_primitive<double>(U[0], U[1], U[2], U[3], Bx, By, g.gamma, g.vol, g.rcp_vol);
            e_speed = run_max(e_speed, cfl_speed(pr.rho, pr.vx, pr.vy, pr.P, Bx, By, g.gamma));
            const double dv = fabs(divb_cell(bxn, bxm, byn, bym, hx, hy, g.inv_dx, g.inv_dy, g.square != 0));
            e_dmax = run_max(e_dmax, dv);
            e_dsum += dv;
            e_bmax = run_max(e_bmax, Bx * Bx + By * By);   // |B|^2 (root taken at the finish)
            e_mass += U[0];
            e_en += U[3];
          }
        }
        continue;
      } else {
      // update_conserved (src/mhd_flux.f90:20-76), x pass then y pass, fields
      // (0, 1) and (2, 3) as lanes of paired FP32 fused multiply-adds
      R U[4];
      {
        float2 F[2] = {make_float2(in[0][idx], in[1][idx]), make_float2(in[2][idx], in[3][idx])};
        const float2 nax = make_float2(-ax, -ax), pax = make_float2(ax, ax);
        const float2 nay = make_float2(-ay, -ay), pay = make_float2(ay, ay);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const R* fx0 = sFx + (2 * h) * G::NFX;
          const R* fx1 = fx0 + G::NFX;
          const R* fy0 = sFy + (2 * h) * G::NFY;
          const R* fy1 = fy0 + G::NFY;
          F[h] = __ffma2_rn(nax, make_float2(fx0[fxr], fx1[fxr]), F[h]);
          if (i > 0 || px) F[h] = __ffma2_rn(pax, make_float2(fx0[fxr - 1], fx1[fxr - 1]), F[h]);
          F[h] = __ffma2_rn(nay, make_float2(fy0[fyt], fy1[fyt]), F[h]);
          if (j > 0 || py) F[h] = __ffma2_rn(pay, make_float2(fy0[fyt - G::FYW], fy1[fyt - G::FYW]), F[h]);
        }
        U[0] = F[0].x; U[1] = F[0].y; U[2] = F[1].x; U[3] = F[1].y;
      }
      const int pc = (lj + 2) * G::PX + (li + 2);
      const R cr = sP[0 * G::NP + pc], cu = sP[1 * G::NP + pc], cv = sP[2 * G::NP + pc];
      const R cP = sP[3 * G::NP + pc], cBx = sP[4 * G::NP + pc], cBy = sP[5 * G::NP + pc];
      floor_hits += conserved_floors<R>(U[0], U[1], U[2], U[3], cBx, cBy, gamma, vol) ? 1u : 0u;
      if (!px && i == 0) {
        const R hb = R(0.5) * (cBx * cBx + cBy * cBy);
        const R en = ((cP - hb) / (gamma - R(1)) + R(0.5) * cr * (cu * cu + cv * cv)) + hb;
        U[0] = U[0] + ax * cr * cu;
        U[1] = U[1] + ax * ((cr * (cu * cu) + cP) - cBx * cBx);
        U[2] = U[2] + ax * (cr * cu * cv - cBx * cBy);
        U[3] = U[3] + ax * ((en + cP) * cu - cBx * (cBx * cu + cBy * cv));
      }
      if (!py && j == 0) {
        const R hb = R(0.5) * (cBx * cBx + cBy * cBy);
        const R en = ((cP - hb) / (gamma - R(1)) + R(0.5) * cr * (cu * cu + cv * cv)) + hb;
        U[0] = U[0] + ay * cr * cv;
        U[2] = U[2] + ay * ((cr * (cv * cv) + cP) - cBy * cBy);
        U[1] = U[1] + ay * (cr * cv * cu - cBy * cBx);
        U[3] = U[3] + ay * ((en + cP) * cv - cBy * (cBy * cv + cBx * cu));
      }
      if (STAGE >= 2) {   // rk_blend, fields in pairs: u0 + c (u - u0)
        const float c = (STAGE == 2) ? 0.25f : (2.0f / 3.0f);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float2 a0 = make_float2(u0[2 * h][idx], u0[2 * h + 1][idx]);
          const float2 d = __fadd2_rn(make_float2(U[2 * h], U[2 * h + 1]), make_float2(-a0.x, -a0.y));
          const float2 r = __ffma2_rn(make_float2(c, c), d, a0);
          U[2 * h] = r.x;
          U[2 * h + 1] = r.y;
        }
      }
      if (STAGE >= 2) floor_hits += conserved_floors<R>(U[0], U[1], U[2], U[3], cBx, cBy, gamma, vol) ? 1u : 0u;
#pragma unroll
      for (int q = 0; q < 4; ++q) out[q][idx] = U[q];
      const R bxn = (STAGE == 3) ? sBx[lj * G::BXW + (li + 1)] : R(0);
      const R byn = (STAGE == 3) ? sBy[(lj + 1) * G::BYW + li] : R(0);
      if (STAGE == 3) {   // (stages 1, 2 stored the new face B in phase 3a)
        out[4][idx] = bxn;
        out[5][idx] = byn;
      }

      if (STAGE == 3 && ((s_own >> lj) & 1u)) {   // a y-slab's ghost rows are left out
        const R bxm = sBx[lj * G::BXW + li];
        const R bym = sBy[lj * G::BYW + li];
        const bool hx = (i > 0) || px, hy = (j > 0) || py;
        const R Bx = hx ? R(0.5) * (bxn + bxm) : bxn;
        const R By = hy ? R(0.5) * (byn + bym) : byn;
        double spc, bm;
        speed_f32(U[0], U[1], U[2], U[3], Bx, By, g, spc, bm);
        e_speed = run_max(e_speed, spc);
        const double dv = fabs(divb_cell(double(bxn), double(bxm), double(byn), double(bym), hx, hy,
                                         g.inv_dx, g.inv_dy, g.square != 0));
        e_dmax = run_max(e_dmax, dv);
        e_dsum += dv;
        e_bmax = run_max(e_bmax, bm);
        e_mass += double(U[0]);
        e_en += double(U[3]);
      }
          }
}
    if (a.counters && !a.dry) {
      unsigned s = __reduce_add_sync(0xffffffffu, floor_hits);
      if ((tid & 31) == 0 && s) atomicAdd(&ctl->floor_hits, (unsigned long long)s);
    }

    if (STAGE == 3 && !a.dry) {
      double r[6] = {e_speed, e_dmax, e_dsum, e_bmax, e_mass, e_en};
      block_reduce_partials<NT>(r, red);
      if (tid == 0) {
        double* p = a.partials + size_t(w) * NPART;
        p[0] = r[0]; p[1] = r[1]; p[2] = r[2]; p[3] = r[3]; p[4] = r[4]; p[5] = r[5];
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->tiles_done, 1u);
        s_last = (prev == unsigned(g.tiles_x * g.tiles_y - 1)) ? 1 : 0;
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        member_finish<NT>(g, ctl, a.partials, g.tiles_x * g.tiles_y, true, red);
      }
    }
    __syncthreads();
  }
}

}  // namespace chimera
