// stage_kernel.cuh -- the fused SSP-RK3 stage kernel and the CFL kernel.
//
// One CTA handles one TX x TY tile of output cells of one grid member (a
// persistent grid-stride loop over a work list of (member, tile)):
//
//   phase 1  primitives (rho, vx, vy, P_total, Bx, By) on the tile plus a
//            2-cell halo, computed straight from the conserved state in HBM
//            (coalesced loads; boundary conditions are index maps, so no ghost
//            arrays are materialised) -> shared memory
//   phase 2  every x- and y-face flux the tile needs: limited slopes, MUSCL
//            face states, MOOD bounds check, face floors, thermal-pressure
//            check, Riemann solver -> shared memory (each face once)
//   phase 3a constrained transport: corner Ez from the face fluxes, curl,
//            face-B update (+ RK blend) -> shared memory
//   phase 3b cell update: flux divergence (x pass then y pass), conserved
//            floors, outflow boundary correction, RK blend, floors -> HBM
//   stage 3  epilogue: primitives of the new state, CFL speed, div B, |B|,
//            totals -> per-tile partials; the last tile of a member reduces
//            them in a fixed order and advances t, outputCount and dt.
//
// Each step of a phase cites the reference routine it restates.
#pragma once
#include "mhd_device.cuh"
#include "chimera_types.h"
#include "tma.cuh"

namespace chimera {

// Work-list / member descriptors (device side), see chimera_types.h.

// The translation unit that instantiates a kernel template, a template
// argument of the stage and CFL kernels.  Units are compiled with different
// floating-point flags (the FP64 units without multiply-add contraction, the
// FP32 unit with fast math), and one template instantiation -- one kernel
// symbol -- compiled in two units would give two device bodies under one name,
// of which a launch runs whichever module the runtime resolved the name to.
// Each unit passes its own value, so every instantiation is defined once.
enum { UNIT_FP64 = 0, UNIT_FP32 = 1, UNIT_NOALLOC = 2 };

// A pointer read from global memory where it is used (inline PTX, so that the
// compiler neither hoists the read nor merges it with an earlier one): keeps
// the value out of registers through a phase that needs them all.  Only for
// data no kernel writes (the member descriptors).
__device__ __forceinline__ void* load_ptr(void* const* p) {
  unsigned long long v;
  asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return reinterpret_cast<void*>(v);
}

// Source cell of a (possibly out-of-domain) tile position: periodic wrap or
// the nearest cell, by the rule of the side it lies beyond (plo below 0, phi
// at n and above; src/mhd_bc.f90:36-121 takes each side on its own).
// Positions of a ragged last tile can lie more than one period beyond a small
// grid, so the wrap is a true modulo.
__device__ __forceinline__ int map_index(int g, int n, int plo, int phi) {
  if (g >= 0 && g < n) return g;
  if (g < 0 ? plo : phi) {
    // g mod n by whole periods: one step for every grid of at least a tile's
    // width, a few for tiny ones -- no integer division on the common path
    while (g < 0) g += n;
    while (g >= n) g -= n;
    return g;
  }
  return g < 0 ? 0 : n - 1;
}

template <typename R> struct StageTileSmem;

template <int TX, int TY> struct TileGeom {
  static constexpr int PX = TX + 4, PY = TY + 4, NP = PX * PY;
  static constexpr int FXW = TX + 1, FXH = TY + 2, NFX = FXW * FXH;   // x faces i in [i0-1,i0+TX), j in [j0-1,j0+TY+1)
  static constexpr int FYW = TX + 2, FYH = TY + 1, NFY = FYW * FYH;   // y faces i in [i0-1,i0+TX+1), j in [j0-1,j0+TY)
  static constexpr int BXW = TX + 1, NBX = BXW * TY;                  // new b_x: i in [i0-1,i0+TX), j in tile
  static constexpr int BYW = TX, NBY = BYW * (TY + 1);                // new b_y: i in tile, j in [j0-1,j0+TY)
  // KEEP_IN (FP64 kernel): four more per-cell arrays, the tile's own cells of
  // the stage input, for phase 3b
  template <typename R, bool KEEP_IN = false> static constexpr size_t smem_bytes() {
    return sizeof(R) * (size_t(6) * NP + size_t(5) * NFX + size_t(5) * NFY + NBX + NBY +
                        (KEEP_IN ? size_t(4) * TX * TY : 0));
  }
};

// TMA box of the FP64 stage input (variants with TMA): the six fields over
// cells [i0-4, i0-4+BW) x [j0-3, j0-3+BH) -- the primitives' 2-cell halo plus
// the face-B neighbours b_x(i-1), b_y(j-1) -- with the origin's x even (a
// multiple of 16 bytes: TX is even), each field's box padded to 128 bytes.
// The boxes land in the face-flux arrays, which phase 1 does not use.
template <int TX, int TY> struct TmaBox64 {
  static_assert(TX % 2 == 0, "the box origin i0 - 4 must be a multiple of 2 doubles");
  static constexpr int BW = ((TX + 6 + 1) / 2) * 2;
  static constexpr int BH = TY + 5;
  static constexpr int BOXF = ((BW * BH + 15) / 16) * 16;
  static constexpr bool FITS = 6 * BOXF + 16 <=
                               5 * TileGeom<TX, TY>::NFX + 5 * TileGeom<TX, TY>::NFY;   // (+16: alignment slack)
};

// L2 prefetch of the input rows the CTA's NEXT tile (work item w_next) will
// read: the conserved fields over [i0-3, i0+TX+2) x [j0-3, j0+TY+2) of the
// stage input and, for stages 2 and 3, U^n over the tile (+1 halo face).
// Issued at the start of the current tile so the next tile's phase-1 loads
// hit L2 instead of HBM.  Pure hints: no result, no synchronisation.  With
// inputs = false only the U^n rows are prefetched (the inputs come by TMA).
template <typename R, int TX, int TY, int NT, int STAGE>
__device__ __forceinline__ void prefetch_next_tile(const StageArgs& a, int w_next, bool inputs = true) {
  if (w_next >= a.total_tiles) return;
  const int m = (a.n_members == 1) ? 0 : a.tile_member[w_next];
  const Member& g = a.members[m];
  const Control* ctl = a.ctl + m;
  const int nx = g.nx, ny = g.ny;
  const int lt = w_next - g.tile_begin;
  const int i0 = (lt % g.tiles_x) * TX, j0 = (lt / g.tiles_x) * TY;
  const int sbuf = ctl->parity, obuf = 1 - sbuf;
  const int in_buf = (STAGE == 1) ? sbuf : (STAGE == 2 ? obuf : 2);
  constexpr int LPR = ((TX + 5) * int(sizeof(R)) + 127) / 128 + 1;   // 128-B lines per row
  // line l of the segment [a0, a1]; line 0 starts at a0 itself so no address precedes the row
  auto touch = [](const char* a0, const char* a1, int l) {
    const char* pl = (l == 0) ? a0
                              : reinterpret_cast<const char*>((reinterpret_cast<uintptr_t>(a0) & ~uintptr_t(127)) +
                                                              size_t(l) * 128);
    if (pl <= a1) asm volatile("prefetch.global.L2 [%0];" ::"l"(pl));
  };
  if (inputs) {   // the stage input over [i0-3, i0+TX+2) x [j0-3, j0+TY+2)
    constexpr int ROWS = TY + 5;
    const int c0 = max(i0 - 3, 0), c1 = min(i0 + TX + 2, nx) - 1;
    for (int it = threadIdx.x; it < 6 * ROWS * LPR; it += NT) {
      const int q = it / (ROWS * LPR), rem = it % (ROWS * LPR);
      const int r = rem / LPR, l = rem % LPR;
      const char* row = reinterpret_cast<const char*>(g.buf[in_buf][q]) +
                        size_t(map_index(j0 - 3 + r, ny, g.periodic_y, g.periodic_yhi)) * nx * sizeof(R);
      touch(row + size_t(c0) * sizeof(R), row + size_t(c1) * sizeof(R), l);
    }
  }
  if (STAGE >= 2) {   // U^n over the tile (+1 halo face)
    constexpr int ROWS0 = TY + 1;
    const int c0 = max(i0 - 1, 0), c1 = min(i0 + TX, nx) - 1;
    for (int it = threadIdx.x; it < 6 * ROWS0 * LPR; it += NT) {
      const int q = it / (ROWS0 * LPR), rem = it % (ROWS0 * LPR);
      const int r = rem / LPR, l = rem % LPR;
      const char* row = reinterpret_cast<const char*>(g.buf[sbuf][q]) +
                        size_t(map_index(j0 - 1 + r, ny, g.periodic_y, g.periodic_yhi)) * nx * sizeof(R);
      touch(row + size_t(c0) * sizeof(R), row + size_t(c1) * sizeof(R), l);
    }
  }
}

// The six per-tile partials (max CFL speed, max |div B|, sum |div B|, max
// |B|, mass, energy) reduced over the block in one pass, deterministically for
// a fixed block size: a shuffle tree within each warp, then the warps in
// order, with one barrier.  red holds [6][NT / 32]; the results are valid on
// thread 0.
template <int NT>
__device__ __forceinline__ void block_reduce_partials(double (&v)[6], double* red) {
  constexpr int NW = NT / 32;
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = fmax(v[0], __shfl_down_sync(0xffffffffu, v[0], o));
    v[1] = fmax(v[1], __shfl_down_sync(0xffffffffu, v[1], o));
    v[2] += __shfl_down_sync(0xffffffffu, v[2], o);
    v[3] = fmax(v[3], __shfl_down_sync(0xffffffffu, v[3], o));
    v[4] += __shfl_down_sync(0xffffffffu, v[4], o);
    v[5] += __shfl_down_sync(0xffffffffu, v[5], o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k * NW + w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v[0] = red[0 * NW]; v[1] = red[1 * NW]; v[3] = red[3 * NW];
    v[2] = 0.0; v[4] = 0.0; v[5] = 0.0;
    for (int k = 0; k < NW; ++k) {
      if (k > 0) {
        v[0] = fmax(v[0], red[0 * NW + k]);
        v[1] = fmax(v[1], red[1 * NW + k]);
        v[3] = fmax(v[3], red[3 * NW + k]);
      }
      v[2] += red[2 * NW + k];
      v[4] += red[4 * NW + k];
      v[5] += red[5 * NW + k];
    }
  }
}

// Per-cell CFL speed cf + |v| (src/main.f90:72-79), FP64.
__device__ __forceinline__ double cfl_speed(double rho, double vx, double vy, double P, double Bx,
                                            double By, double gamma) {
  double inv_rho = 1.0 / rho;
  double c0_sq = gamma * (P - 0.5 * (Bx * Bx + By * By)) * inv_rho;
  double ca_sq = (Bx * Bx + By * By) * inv_rho;
  double cf = sqrt(c0_sq + ca_sq);
  if (rho < 1.0e-3) cf = fmin(cf, 50.0);
  return cf + sqrt(vx * vx + vy * vy);
}

// divB of one cell from face values (src/mhd_field_ops.f90:60-117).
// FP32-bulk form: a cell's CFL speed c_f + |v| (FP64 pressure recovery, FP32
// wave speeds) and |B|^2.  The stage-3 epilogue and the CFL kernel both use it,
// so that a dt is the same whichever of the two computed it.
__device__ __forceinline__ void speed_f32(float M, float Mx, float My, float E, float Bx, float By,
                                          const Member& g, double& speed, double& bmag2) {
  const Prim<float> pr = get_primitive_mixed(M, Mx, My, E, Bx, By, g.gamma, g.inv_vol, float(g.inv_vol));
  const float gamma = float(g.gamma);
  const float inv_rho = 1.0f / pr.rho;
  const float B2 = Bx * Bx + By * By;
  float cf = sqrtf(gamma * (pr.P - 0.5f * B2) * inv_rho + B2 * inv_rho);
  if (pr.rho < 1.0e-3f) cf = fminf(cf, 50.0f);
  speed = double(cf + sqrtf(pr.vx * pr.vx + pr.vy * pr.vy));
  bmag2 = double(B2);
}

__device__ __forceinline__ double divb_cell(double bx, double bxm, double by, double bym, bool has_x,
                                            bool has_y, double inv_dx, double inv_dy, bool square) {
  if (square) {
    if (has_x && has_y) return (((bx - bxm) + by) - bym) * inv_dx;
    if (has_x) return (bx - bxm) * inv_dx;
    if (has_y) return (by - bym) * inv_dx;
    return 0.0;
  }
  if (has_x && has_y) return (bx - bxm) * inv_dx + (by - bym) * inv_dy;
  if (has_x) return (bx - bxm) * inv_dx;
  if (has_y) return (by - bym) * inv_dy;
  return 0.0;
}

// Finish of one member's step, run by the CTA that completed its last tile:
// fixed-order reduction of the tile partials, then the time-loop bookkeeping
// of src/main.f90:72-83 and :273-292.
template <int NT>
__device__ void member_finish(const Member& g, Control* ctl, const double* part, int ntiles,
                              bool advance_time, double* red) {
  double sp = 0.0, dmx = 0.0, dsum = 0.0, bmx = 0.0, ms = 0.0, es = 0.0;
  for (int k = threadIdx.x; k < ntiles; k += NT) {
    const double* p = part + size_t(g.tile_begin + k) * NPART;
    sp = fmax(sp, __ldcg(p + 0));
    dmx = fmax(dmx, __ldcg(p + 1));
    dsum += __ldcg(p + 2);
    bmx = fmax(bmx, __ldcg(p + 3));
    ms += __ldcg(p + 4);
    es += __ldcg(p + 5);
  }
  double r[6] = {sp, dmx, dsum, bmx, ms, es};
  block_reduce_partials<NT>(r, red);
  sp = r[0]; dmx = r[1]; dsum = r[2]; bmx = r[3]; ms = r[4]; es = r[5];
  // the partials carry max |B|^2: a correctly rounded square root is monotonic,
  // so the root of the maximum is the maximum of the roots, bit for bit
  bmx = sqrt(bmx);
  if (threadIdx.x == 0) {
    double t = ctl->t;
    int oc = ctl->output_count;
    bool output_reached = false;
    if (advance_time) {
      t = t + ctl->dt;                                           // src/main.f90:273
      if (t >= double(oc) * g.t_out || t >= g.t_end) {           // src/main.f90:279,291
        oc += 1;
        output_reached = true;
      }
      ctl->steps += 1;
      ctl->parity = 1 - ctl->parity;                             // U^{n+1} now in the other buffer
    }
    // src/main.f90:79: courant * minval(len / speed) == courant * (len / maxval(speed))
    // because correctly rounded division is monotone in the divisor.
    double dt = g.courant * (g.len / sp);
    if (t + dt > double(oc) * g.t_out) dt = double(oc) * g.t_out - t;   // :82
    dt = fmax(dt, double(1e-12f));                                       // :83 (single-precision literal)
    ctl->t = t;
    ctl->output_count = oc;
    ctl->dt = dt;
    ctl->active = (t < g.t_end) ? 1 : 0;
    // a run that stops at every output time pauses after the step that
    // reached one -- where the reference writes its snapshot (src/main.f90:279-292)
    if (output_reached && (ctl->flags & CTL_PAUSE_AT_OUTPUT)) {
      ctl->active = 0;
      ctl->flags |= CTL_PAUSED;
    }
    ctl->cfl_speed = sp;
    ctl->divb_max = dmx;
    ctl->divb_sum = dsum;
    ctl->bmax = bmx;
    ctl->mass = ms;
    ctl->energy = es;
    ctl->tiles_done = 0u;
    if (!(sp > 0.0) || !isfinite(ms) || !isfinite(es)) atomicOr(&ctl->status, STATUS_NONFINITE);
  }
}

// ----------------------------------------------------------------------------
// The fused stage kernel.
// Buffers rotate through a device-resident parity bit: S = buf[parity] holds
// U^n, O = buf[1 - parity] and buf[2] are scratch.
//   STAGE 1: in = S (U^n), out = O (U1)
//   STAGE 2: in = O, u0 = S, out = buf[2] (U2)
//   STAGE 3: in = buf[2], u0 = S, out = O (U^{n+1}); the member finish flips
//            the parity.  (Writing U^{n+1} over U^n in place would race: the
//            epilogue's halo faces read U^n at the neighbour tile's cells.)
//
// KEEP_IN: phase 1, which loads the stage input of the tile and its halo
// anyway, keeps the four conserved fields of the tile's own cells in shared
// memory, and phase 3b reads them there instead of from L2 (16 KB more for a
// 32 x 16 tile; fewer live registers through the update, and fewer spills).
// MIXBC: a periodic side may face a non-periodic one (a mixed pair).  A halo
// cell that wraps across such a pair must see its neighbours as the cell it
// copies does (its neighbour across the non-periodic side is itself), and the
// face and corner values computed in the halo must be the ones the owning
// tile computes; the checks cost instructions on every face, so grids without
// a mixed pair run the MIXBC = false instantiations.
// ----------------------------------------------------------------------------
template <typename R, int SOLVER, int STAGE, int TX, int TY, int NT, int MINB, bool KEEP_IN = false,
          bool TMA = false, int UNIT = UNIT_FP64, bool MIXBC = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(StageArgs a) {
  using G = TileGeom<TX, TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw);
  R* sFx = sP + 6 * G::NP;
  R* sFy = sFx + 5 * G::NFX;
  R* sBx = sFy + 5 * G::NFY;
  R* sBy = sBx + G::NBX;
  R* sU = sBy + G::NBY;            // KEEP_IN: [4][TX * TY] the stage input of the tile's own cells
  __shared__ double red[6 * (NT / 32)];
  __shared__ int s_last;
  __shared__ unsigned s_own;   // stage 3: bit r set if tile row r is one of the grid's own rows
  static_assert(TY < 32, "the own-row mask holds one bit per tile row");
  using BX = TmaBox64<TX, TY>;
  static_assert(!TMA || (sizeof(R) == 8 && BX::FITS), "FP64 boxes in the face-flux arrays");
  __shared__ __align__(8) uint64_t s_bar;   // TMA completion
  __shared__ unsigned s_phase;              // parity of the mbarrier phase the next box completes

  const int tid = threadIdx.x;
  const bool slope_on = a.slope_limiting != 0;
  const bool mood_on = a.mood != 0;
  const bool van_leer = a.limiter == LIMITER_VAN_LEER;
  constexpr unsigned TMA_POLLS = 1u << 26;   // bound of every wait for a TMA completion
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(&s_bar, 1);
      s_phase = 0u;
    }
    __syncthreads();
  }

  for (int w = a.work_begin + blockIdx.x; w < a.total_tiles; w += gridDim.x) {
    const int m = (a.n_members == 1) ? 0 : a.tile_member[w];
    const Member& g = a.members[m];
    Control* ctl = a.ctl + m;
    if (ctl->active == 0) continue;  // uniform across the CTA
    const int nx = g.nx, ny = g.ny;
    const int px = g.periodic_x, py = g.periodic_y;                   // low sides
    const int pxh = MIXBC ? g.periodic_xhi : px, pyh = MIXBC ? g.periodic_yhi : py;   // high sides
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
    const double rcp_vol = g.rcp_vol, rcp_gm1 = g.rcp_gm1;
    const R dt = R(ctl->dt);
    const int sbuf = ctl->parity, obuf = 1 - sbuf;
    const int in_buf = (STAGE == 1) ? sbuf : (STAGE == 2 ? obuf : 2);
    const int out_buf = (STAGE == 2) ? 2 : obuf;

    // ---- phase 1: primitives on the tile + 2-cell halo ---------------------
    // average_face_to_cell_B (src/mhd_field_ops.f90:120-156) + get_primitive
    // (src/mhd_change_states.f90:61-113).  Out-of-domain positions take the
    // primitive of the cell that fill_ghost_cells would copy there
    // (src/mhd_bc.f90:36-121): wrap if periodic, else the nearest cell.
    // TMA variants: a tile whose box lies inside the arrays (no index map
    // applies: every position is a cell of the grid) reads its inputs from six
    // box copies; the others take the plain loads below.
    bool from_box = false;
    if constexpr (TMA) {
      from_box = g.tmap != nullptr && i0 >= 4 && i0 - 4 + BX::BW <= nx && j0 >= 3 && j0 - 3 + BX::BH <= ny;
      if (from_box) {   // uniform across the CTA
        const R* stg = reinterpret_cast<const R*>((reinterpret_cast<uintptr_t>(sFx) + 127) & ~uintptr_t(127));
        if (tid == 0) {
          // the previous tile's generic reads of these arrays (ordered before the
          // loop's closing barrier) precede the async-proxy writes
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&s_bar, unsigned(6 * BX::BW * BX::BH * sizeof(R)));
          const char* maps = reinterpret_cast<const char*>(g.tmap) + size_t(in_buf) * 6 * TMAP_BYTES;
#pragma unroll
          for (int q = 0; q < 6; ++q)
            tma_load_2d(const_cast<R*>(stg) + q * BX::BOXF, maps + q * TMAP_BYTES, i0 - 4, j0 - 3, &s_bar);
        }
        const bool ok = mbar_wait(&s_bar, s_phase, TMA_POLLS);
        for (int p = tid; p < G::NP && ok; p += NT) {
          const int qx = p % G::PX, qy = p / G::PX;
          const int b = (qy + 1) * BX::BW + (qx + 2);   // box element of cell (i0-2+qx, j0-2+qy)
          const R Bx = R(0.5) * (stg[4 * BX::BOXF + b] + stg[4 * BX::BOXF + b - 1]);
          const R By = R(0.5) * (stg[5 * BX::BOXF + b] + stg[5 * BX::BOXF + b - BX::BW]);
          const R c0 = stg[b], c1 = stg[BX::BOXF + b], c2 = stg[2 * BX::BOXF + b], c3 = stg[3 * BX::BOXF + b];
          if constexpr (KEEP_IN) {
            const int ox = qx - 2, oy = qy - 2;
            if (ox >= 0 && ox < TX && oy >= 0 && oy < TY) {
              const int c = oy * TX + ox;
              sU[0 * (TX * TY) + c] = c0;
              sU[1 * (TX * TY) + c] = c1;
              sU[2 * (TX * TY) + c] = c2;
              sU[3 * (TX * TY) + c] = c3;
            }
          }
          Prim<R> pr = get_primitive<R>(c0, c1, c2, c3, Bx, By, gamma, vol, rcp_vol);
          sP[0 * G::NP + p] = pr.rho;
          sP[1 * G::NP + p] = pr.vx;
          sP[2 * G::NP + p] = pr.vy;
          sP[3 * G::NP + p] = pr.P;
          sP[4 * G::NP + p] = pr.Bx;
          sP[5 * G::NP + p] = pr.By;
        }
        if (__syncthreads_or(!ok)) {   // a copy that never landed: status word, end the kernel
          if (tid == 0) {
            atomicOr(&ctl->status, STATUS_TIMEOUT);
            // one more bounded wait for the copies in flight, with the CTA (and
            // its shared memory) still resident, before it exits
            mbar_wait(&s_bar, s_phase, TMA_POLLS);
          }
          return;
        }
        if (tid == 0) s_phase ^= 1u;   // every thread has read it (before the barrier above)
      }
    }
    if (!from_box) {
      const R* __restrict__ in[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) in[q] = reinterpret_cast<const R*>(g.buf[in_buf][q]);
      for (int p = tid; p < G::NP; p += NT) {
        const int qx = p % G::PX, qy = p / G::PX;
        const int si = map_index(i0 - 2 + qx, nx, px, pxh);
        const int sj = map_index(j0 - 2 + qy, ny, py, pyh);
        const size_t idx = size_t(sj) * nx + si;
        const R bxc = in[4][idx];
        const R byc = in[5][idx];
        R Bx, By;
        if (si > 0) Bx = R(0.5) * (bxc + in[4][idx - 1]);
        else Bx = px ? R(0.5) * (bxc + in[4][idx + (nx - 1)]) : bxc;
        if (sj > 0) By = R(0.5) * (byc + in[5][idx - nx]);
        else By = py ? R(0.5) * (byc + in[5][idx + size_t(ny - 1) * nx]) : byc;
        const R c0 = in[0][idx], c1 = in[1][idx], c2 = in[2][idx], c3 = in[3][idx];
        if constexpr (KEEP_IN) {   // the tile's own cells: kept for phase 3b
          const int ox = qx - 2, oy = qy - 2;
          if (ox >= 0 && ox < TX && oy >= 0 && oy < TY) {
            const int c = oy * TX + ox;
            sU[0 * (TX * TY) + c] = c0;
            sU[1 * (TX * TY) + c] = c1;
            sU[2 * (TX * TY) + c] = c2;
            sU[3 * (TX * TY) + c] = c3;
          }
        }
        Prim<R> pr = get_primitive<R>(c0, c1, c2, c3, Bx, By, gamma, vol, rcp_vol);
        sP[0 * G::NP + p] = pr.rho;
        sP[1 * G::NP + p] = pr.vx;
        sP[2 * G::NP + p] = pr.vy;
        sP[3 * G::NP + p] = pr.P;
        sP[4 * G::NP + p] = pr.Bx;
        sP[5 * G::NP + p] = pr.By;
      }
    }
    if (!from_box) __syncthreads();   // (the box path ended with its own barrier)

    // ---- phase 2: face fluxes ------------------------------------------------
    unsigned mood_resets = 0;
    for (int f = tid; f < G::NFX + G::NFY; f += NT) {
      const bool ydir = f >= G::NFX;
      const int ff = ydir ? f - G::NFX : f;
      // constant divisors in each branch (a runtime divisor costs a full integer division)
      const int li = ydir ? ff % G::FYW : ff % G::FXW;
      const int lj = ydir ? ff / G::FYW : ff / G::FXW;
      const int pa = (lj + 1) * G::PX + (li + 1);    // cell on the low side of the face
      const int on = ydir ? G::PX : 1;               // offset along the face normal
      const R inv_h = R(ydir ? g.inv_dy : g.inv_dx);
      const R inv_2h = R(ydir ? g.inv_2dy : g.inv_2dx);
      const R hh = R(ydir ? g.hy : g.hx);             // 0.5 * spacing
      R L[6], Rv[6];
      bool reset = false;
      // mixed pairs: the low cell's neighbours that are its own ghost (a cell
      // wrapped across a pair, next to the non-periodic side), and a high cell
      // wrapped from the far side whose low neighbour is its own ghost
      bool own_xp = false, own_xm = false, own_yp = false, own_ym = false, own_bm = false;
      if constexpr (MIXBC) {
        const int gax = i0 + li - 1, gay = j0 + lj - 1;   // the low cell
        own_xp = px && !pxh && gax == -1;
        own_xm = !px && pxh && gax == nx;
        own_yp = py && !pyh && gay == -1;
        own_ym = !py && pyh && gay == ny;
        own_bm = ydir ? (!py && pyh && gay + 1 == ny) : (!px && pxh && gax + 1 == nx);
      }
      const bool own_np = ydir ? own_yp : own_xp;   // the high cell is the low cell's own ghost
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const R* s = sP + q * G::NP;
        const R fm = s[pa - on], f0 = s[pa];
        R fp = s[pa + on], fpp = s[pa + 2 * on];
        if (MIXBC && own_np) { fp = f0; fpp = f0; }
        const R fb0 = (MIXBC && own_bm) ? fp : f0;    // the high cell's low neighbour
        // apply_slope_limiter (src/mhd_derivatives.f90:50-127) or compute_gradients (:15-47)
        R sa, sb;
        if (slope_on) {
          if (van_leer) {
            sa = limit_slope<R, LIMITER_VAN_LEER>((f0 - fm) * inv_h, (fp - f0) * inv_h);
            sb = limit_slope<R, LIMITER_VAN_LEER>((fp - fb0) * inv_h, (fpp - fp) * inv_h);
          } else {
            sa = limit_slope<R, LIMITER_MC>((f0 - fm) * inv_h, (fp - f0) * inv_h);
            sb = limit_slope<R, LIMITER_MC>((fp - fb0) * inv_h, (fpp - fp) * inv_h);
          }
        } else {
          sa = (fp - fm) * inv_2h;
          sb = (fpp - fb0) * inv_2h;
        }
        // reconstruction (src/mhd_derivatives.f90:160-182): left state from the low
        // cell, right state = the high cell extrapolated back (temp_x(i+1)).
        R vL = f0 + hh * sa;
        R vR = fp - hh * sb;
        const bool rp = (q == 0 || q == 3);
        if (mood_on) {
          // MOOD bounds of the LOW cell (:190-216), applied to both states and
          // resetting both to the low cell's value (the reference's XR/YR rule).
          // (the bounds only feed comparisons: hardware min / max)
          R nxp = s[pa + 1], nxm = s[pa - 1], nyp = s[pa + G::PX], nym = s[pa - G::PX];
          if (MIXBC && own_xp) nxp = f0;
          if (MIXBC && own_xm) nxm = f0;
          if (MIXBC && own_yp) nyp = f0;
          if (MIXBC && own_ym) nym = f0;
          R lo = hmin(hmin(hmin(hmin(f0, nxp), nxm), nyp), nym);
          const R hi = hmax(hmax(hmax(hmax(f0, nxp), nxm), nyp), nym);
          if (rp) lo = hmax(R(0.1e-8), lo);
          if (vL < lo || vL > hi) { vL = f0; reset = true; }
          if (vR < lo || vR > hi) { vR = f0; reset = true; }
        }
        if (rp) {                      // face floors (:223-227)
          vL = hmax(vL, R(1.0e-8));
          vR = hmax(vR, R(1.0e-8));
        }
        L[q] = vL; Rv[q] = vR;
      }
      // thermal_pressure_check (src/mhd_derivatives.f90:232-293): reset all six
      // fields of a face slot to the low cell's values.
      if (L[3] - R(0.5) * (L[4] * L[4] + L[5] * L[5]) < K<R>::P_floor) {
#pragma unroll
        for (int q = 0; q < 6; ++q) L[q] = sP[q * G::NP + pa];
      }
      if (Rv[3] - R(0.5) * (Rv[4] * Rv[4] + Rv[5] * Rv[5]) < K<R>::P_floor) {
#pragma unroll
        for (int q = 0; q < 6; ++q) Rv[q] = sP[q * G::NP + pa];
      }
      mood_resets += reset ? 1u : 0u;
      // compute_fluxes, rotated for y faces (src/main.f90:394-401)
      const R unL = ydir ? L[2] : L[1], unR = ydir ? Rv[2] : Rv[1];
      const R utL = ydir ? L[1] : L[2], utR = ydir ? Rv[1] : Rv[2];
      const R bnL = ydir ? L[5] : L[4], bnR = ydir ? Rv[5] : Rv[4];
      const R btL = ydir ? L[4] : L[5], btR = ydir ? Rv[4] : Rv[5];
      Flux5<R> F = riemann<R, SOLVER>(gamma, L[0], Rv[0], unL, unR, utL, utR, L[3], Rv[3], bnL, bnR, btL, btR,
                                      rcp_gm1);
      R* dst = ydir ? sFy : sFx;
      const int NF = ydir ? G::NFY : G::NFX;
      dst[0 * NF + ff] = F.mass;
      dst[1 * NF + ff] = ydir ? F.momt : F.momn;   // x momentum flux
      dst[2 * NF + ff] = ydir ? F.momn : F.momt;   // y momentum flux
      dst[3 * NF + ff] = F.energy;
      dst[4 * NF + ff] = F.bt;                     // By flux (x faces) / Bx flux (y faces)
    }
    if (a.counters && !a.dry) {
      unsigned s = __reduce_add_sync(0xffffffffu, mood_resets);
      if ((tid & 31) == 0 && s) atomicAdd(&ctl->mood_resets, (unsigned long long)s);
    }
    __syncthreads();

    // the buffer pointers, read here rather than kept in registers through
    // phase 2 (the kernel's register peak)
    const R* __restrict__ in[6];
    const R* __restrict__ u0[6];
    R* __restrict__ out[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      in[q] = static_cast<const R*>(load_ptr(&g.buf[in_buf][q]));
      u0[q] = static_cast<const R*>(load_ptr(&g.buf[sbuf][q]));
      out[q] = static_cast<R*>(load_ptr(&g.buf[out_buf][q]));
    }

    // ---- phase 3a: constrained transport -> new face B ------------------------
    // constrained_transport (src/mhd_flux.f90:79-136) + compute_curl_2d(-Ez)
    // (src/mhd_field_ops.f90:15-57), then the RK blend of b_x, b_y.
    const R* FByX = sFx + 4 * G::NFX;
    const R* FBxY = sFy + 4 * G::NFY;
    auto Ez = [&](int ci, int cj) -> R {
      const int xi = (cj - j0 + 1) * G::FXW + (ci - i0 + 1);
      const R fa = FByX[xi];
      // zero gradient past a non-periodic high side -- also for the corner row
      // below y = 0 that wraps to it (mixed pair)
      const bool up_own = (cj == ny - 1 && !pyh) || (MIXBC && cj == -1 && py && !pyh);
      const R up = up_own ? fa : FByX[xi + G::FXW];
      const int yi = (cj - j0 + 1) * G::FYW + (ci - i0 + 1);
      const R fb = FBxY[yi];
      const bool right_own = (ci == nx - 1 && !pxh) || (MIXBC && ci == -1 && px && !pxh);
      const R right = right_own ? fb : FBxY[yi + 1];
      return R(0.25) * (((-fa - up) + fb) + right);
    };
    const R inv_dx = R(g.inv_dx), inv_dy = R(g.inv_dy);
    const int bx_lo = (STAGE == 3 && (i0 > 0 || px)) ? -1 : 0;   // halo face column for the epilogue
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
      R val;
      if (!isy) {
        const R e0 = Ez(i, j);
        R dbx;
        if (j > 0 || py) dbx = ((-e0) - (-Ez(i, j - 1))) * inv_dy;
        else dbx = ((-Ez(i, 1)) - (-e0)) * inv_dy;           // outflow ylo: copy row 2
        val = in[4][idx] + dt * dbx;
        if (STAGE == 2) val = R(0.75) * u0[4][idx] + R(0.25) * val;
        if (STAGE == 3) val = R(1.0 / 3.0) * u0[4][idx] + R(2.0 / 3.0) * val;
        if (STAGE == 3) sBx[lj * G::BXW + (li + 1)] = val;   // the epilogue reads neighbours' new B
        else out[4][idx] = val;                                // stages 1, 2: straight to the output
      } else {
        const R e0 = Ez(i, j);
        R dby;
        if (i > 0 || px) dby = -(((-e0) - (-Ez(i - 1, j))) * inv_dx);
        else dby = -(((-Ez(1, j)) - (-e0)) * inv_dx);        // outflow xlo: copy column 2
        val = in[5][idx] + dt * dby;
        if (STAGE == 2) val = R(0.75) * u0[5][idx] + R(0.25) * val;
        if (STAGE == 3) val = R(1.0 / 3.0) * u0[5][idx] + R(2.0 / 3.0) * val;
        if (STAGE == 3) sBy[(lj + 1) * G::BYW + li] = val;
        else out[5][idx] = val;
      }
    }
    if (STAGE == 3) __syncthreads();   // stages 1, 2 read no phase-3a result in phase 3b

    // ---- phase 3b: cell update -------------------------------------------------
    double e_speed = 0.0, e_dmax = 0.0, e_dsum = 0.0, e_bmax = 0.0, e_mass = 0.0, e_en = 0.0;
    unsigned floor_hits = 0;
    const R ax = dt * R(g.dy);   // x-face weight (dt*dx in the square reference)
    const R ay = dt * R(g.dx);
    for (int c = tid; c < TX * TY; c += NT) {
      const int li = c % TX, lj = c / TX;
      const int i = i0 + li, j = j0 + lj;
      if (i >= nx || j >= ny) continue;
      const size_t idx = size_t(j) * nx + i;
      const int fxr = (lj + 1) * G::FXW + (li + 1);  // x face i+1/2
      const int fyt = (lj + 1) * G::FYW + (li + 1);  // y face j+1/2
      R U[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        // update_conserved (src/mhd_flux.f90:20-76): x pass, then y pass
        R F = KEEP_IN ? sU[q * (TX * TY) + c] : in[q][idx];
        const R* fx = sFx + q * G::NFX;
        const R* fy = sFy + q * G::NFY;
        if (i > 0 || px) F = (F - ax * fx[fxr]) + ax * fx[fxr - 1];
        else F = F - ax * fx[fxr];
        if (j > 0 || py) F = (F - ay * fy[fyt]) + ay * fy[fyt - G::FYW];
        else F = F - ay * fy[fyt];
        U[q] = F;
      }
      const int pc = (lj + 2) * G::PX + (li + 2);
      const R cr = sP[0 * G::NP + pc], cu = sP[1 * G::NP + pc], cv = sP[2 * G::NP + pc];
      const R cP = sP[3 * G::NP + pc], cBx = sP[4 * G::NP + pc], cBy = sP[5 * G::NP + pc];
      // apply_conserved_floors with the stage's (pre-CT) cell B (src/main.f90:113)
      floor_hits += conserved_floors<R>(U[0], U[1], U[2], U[3], cBx, cBy, gamma, vol) ? 1u : 0u;
      // outflow boundary flux correction (src/main.f90:118-148)
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
      // RK blend + floors with the same stale cell B (src/main.f90:202-208, 261-267)
      if (STAGE == 2) {
#pragma unroll
        for (int q = 0; q < 4; ++q) U[q] = R(0.75) * u0[q][idx] + R(0.25) * U[q];
      }
      if (STAGE == 3) {
#pragma unroll
        for (int q = 0; q < 4; ++q) U[q] = R(1.0 / 3.0) * u0[q][idx] + R(2.0 / 3.0) * U[q];
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

      // epilogue: primitives of U^{n+1} (next step's CFL, src/main.f90:69-79),
      // div B (src/main.f90:276), |B| and totals -- over the grid's own rows (a
      // y-slab's ghost rows are left out)
      if (STAGE == 3 && ((s_own >> lj) & 1u)) {
        const R bxm = sBx[lj * G::BXW + li];
        const R bym = sBy[lj * G::BYW + li];
        const bool hx = (i > 0) || px, hy = (j > 0) || py;
        const double Bx = hx ? 0.5 * (double(bxn) + double(bxm)) : double(bxn);
        const double By = hy ? 0.5 * (double(byn) + double(bym)) : double(byn);
        Prim<double> pr = get_primitive<double>(double(U[0]), double(U[1]), double(U[2]), double(U[3]),
                                                Bx, By, g.gamma, g.vol, g.rcp_vol);
        e_speed = run_max(e_speed, cfl_speed(pr.rho, pr.vx, pr.vy, pr.P, Bx, By, g.gamma));
        const double d = fabs(divb_cell(double(bxn), double(bxm), double(byn), double(bym), hx, hy,
                                        g.inv_dx, g.inv_dy, g.square != 0));
        e_dmax = run_max(e_dmax, d);
        e_dsum += d;
        e_bmax = run_max(e_bmax, Bx * Bx + By * By);   // |B|^2 (root taken once, at the finish)
        e_mass += double(U[0]);
        e_en += double(U[3]);
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
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// ----------------------------------------------------------------------------
// CFL kernel: dt of the current state (src/main.f90:69-83) without advancing
// time; used before the first step after the state is set.
// UNIT: the translation unit that instantiates it (see UNIT_FP64).
// ----------------------------------------------------------------------------
template <typename R, int TX, int TY, int NT, int UNIT>
__global__ void __launch_bounds__(NT) cfl_kernel(StageArgs a) {
  __shared__ double red[6 * (NT / 32)];
  __shared__ int s_last;
  for (int w = a.work_begin + blockIdx.x; w < a.total_tiles; w += gridDim.x) {
    const int m = (a.n_members == 1) ? 0 : a.tile_member[w];
    const Member& g = a.members[m];
    Control* ctl = a.ctl + m;
    const int nx = g.nx, ny = g.ny;
    const int lt = w - g.tile_begin;
    const int i0 = (lt % g.tiles_x) * TX;
    const int j0 = (lt / g.tiles_x) * TY;
    const R* in[6];
    for (int q = 0; q < 6; ++q) in[q] = reinterpret_cast<const R*>(g.buf[ctl->parity][q]);
    double sp = 0.0, dmx = 0.0, dsum = 0.0, bmx = 0.0, ms = 0.0, es = 0.0;
    for (int c = threadIdx.x; c < TX * TY; c += NT) {
      const int i = i0 + c % TX, j = j0 + c / TX;
      if (i >= nx || j >= ny - g.skip_hi || j < g.skip_lo) continue;
      const size_t k = size_t(j) * nx + i;
      const bool hx = (i > 0) || g.periodic_x, hy = (j > 0) || g.periodic_y;
      const R bxr = in[4][k], byr = in[5][k];
      const R bxmr = hx ? in[4][(i > 0) ? k - 1 : k + (nx - 1)] : bxr;
      const R bymr = hy ? in[5][(j > 0) ? k - nx : k + size_t(ny - 1) * nx] : byr;
      const double bxc = double(bxr), byc = double(byr), bxm = double(bxmr), bym = double(bymr);
      if constexpr (sizeof(R) == 4) {   // the FP32-bulk epilogue's arithmetic
        const R Bx = hx ? R(0.5) * (bxr + bxmr) : bxr;
        const R By = hy ? R(0.5) * (byr + bymr) : byr;
        double spc, bm;
        speed_f32(in[0][k], in[1][k], in[2][k], in[3][k], Bx, By, g, spc, bm);
        sp = run_max(sp, spc);
        bmx = run_max(bmx, bm);
      } else {
        const double Bx = hx ? 0.5 * (bxc + bxm) : bxc;
        const double By = hy ? 0.5 * (byc + bym) : byc;
        Prim<double> pr = get_primitive<double>(double(in[0][k]), double(in[1][k]), double(in[2][k]),
                                                double(in[3][k]), Bx, By, g.gamma, g.vol, g.rcp_vol);
        sp = run_max(sp, cfl_speed(pr.rho, pr.vx, pr.vy, pr.P, Bx, By, g.gamma));
        bmx = run_max(bmx, Bx * Bx + By * By);
      }
      const double d = fabs(divb_cell(bxc, bxm, byc, bym, hx, hy, g.inv_dx, g.inv_dy, g.square != 0));
      dmx = run_max(dmx, d);
      dsum += d;
      ms += double(in[0][k]);
      es += double(in[3][k]);
    }
    double r[6] = {sp, dmx, dsum, bmx, ms, es};
    block_reduce_partials<NT>(r, red);
    if (threadIdx.x == 0) {
      double* p = a.partials + size_t(w) * NPART;
      p[0] = r[0]; p[1] = r[1]; p[2] = r[2]; p[3] = r[3]; p[4] = r[4]; p[5] = r[5];
      __threadfence();
      const unsigned prev = atomicAdd(&ctl->tiles_done, 1u);
      s_last = (prev == unsigned(g.tiles_x * g.tiles_y - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      member_finish<NT>(g, ctl, a.partials, g.tiles_x * g.tiles_y, false, red);
    }
    __syncthreads();
  }
}

}  // namespace chimera
