// adjoint.cu -- hand-written discrete adjoint of one SSP-RK3 step (FP64).
//
// For a state U_n and the adjoint lambda_{n+1} = dL/dU_{n+1}, computes
// lambda_n = (dU_{n+1}/dU_n)^T lambda_{n+1} with the time step held at its
// forward value (the CFL dt is not differentiated: "frozen dt").
//
// Structure.  The step is re-run forward by simple per-cell / per-face "tape"
// kernels that reproduce the fused stage kernel bit for bit (same device
// functions, same operation order, --fmad=false) and record what the reverse
// sweep needs: stage primitives, face fluxes, the pre-floor and pre-blend
// conserved values, and per-face decision flags (MOOD resets, face floors,
// thermal-pressure resets).  The reverse sweep then transposes, stage 3 to 1:
//   floors + RK blend      (src/mhd_change_states.f90:116-166, src/main.f90:202-267)
//   flux divergence        (src/mhd_flux.f90:20-76)
//   constrained transport  (src/mhd_flux.f90:79-136): lambda_Ez at the corners
//   Riemann solver         (src/mhd_flux.f90:197-779)
//   thermal check, face floors, MOOD  (src/mhd_derivatives.f90:130-293): the
//                          decisions are taken from the forward (a reset face
//                          passes its adjoint to the cell it was reset to)
//   slope limiter          (src/mhd_derivatives.f90:50-127); where a one-sided
//                          difference is exactly zero (uniform neighbourhood) the
//                          limiter is not differentiable: (1/2, 1/2) if both are
//                          zero, else 1 w.r.t. the zero one (k_rev_slopes)
//   primitive recovery     (src/mhd_change_states.f90:61-113)
//   face->cell B average   (src/mhd_field_ops.f90:120-156)
// as gather kernels (no atomics; deterministic).  Local Jacobians of the
// pointwise functions come from evaluating the same templated device code
// with forward-mode dual numbers (dual.cuh): at a kink (limiter branch, min /
// max, floor) the derivative is that of the branch the forward took.
//
// Boundary conditions: periodic or outflow (zero-gradient ghost cells), each
// side on its own -- a periodic side may face an outflow one, whose faces and
// ghosts then follow the rules of the side they lie beyond.  At an outflow side the forward
// takes the nearest cell for every ghost position (src/mhd_bc.f90:36-121), the
// outflow face->cell B (src/mhd_field_ops.f90:120-156), curl copy
// (src/mhd_flux.f90:79-136), update without the incoming face
// (src/mhd_flux.f90:20-76) and boundary flux correction (src/main.f90:118-148);
// the reverse gathers transpose each of them.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <new>

#include "../../include/chimera_gpu.h"
#include "abi_check.h"
#include "dual.cuh"
#include "mhd_device.cuh"

using namespace chimera;

namespace {

struct AdjGeom {
  int nx, ny;
  double dx, dy, inv_dx, inv_dy, inv_2dx, inv_2dy, hx, hy, gamma, vol;
  int riemann, limiter, slope, mood;
  int px, py;     // the low side (x = 0 / y = 0) is periodic (else outflow)
  int pxh, pyh;   // the high side is periodic (differs from the low side in a mixed pair)
};

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
// the cell a ghost position i (one or two cells beyond the grid) takes its
// value from, by the rule of the side it lies beyond (plo below 0, phi at n
// and above): periodic wrap, or the nearest cell (outflow)
__device__ __forceinline__ int src(int i, int n, int plo, int phi) {
  if (i >= 0 && i < n) return i;
  return (i < 0 ? plo : phi) ? wrap(i, n) : (i < 0 ? 0 : n - 1);
}

// ---------------------------------------------------------------------------
// forward tape kernels
// ---------------------------------------------------------------------------
struct StageTape {
  double* P[6];      // stage primitives rho, vx, vy, P_total, Bx, By
  double* Fx[5];     // x-face fluxes (face i+1/2): mass, momx, momy, energy, By
  double* Fy[5];     // y-face fluxes (face j+1/2): mass, momx, momy, energy, Bx
  uint32_t* flx;     // x-face decision flags
  uint32_t* fly;     // y-face decision flags
  double* Upre[4];   // conserved after the flux update, before the first floors
  double* Ublend[4]; // conserved after the RK blend, before the second floors
};

__global__ void k_tape_prims(AdjGeom g, const double* const* __restrict__ U, StageTape t) {
  const int n = g.nx * g.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    // average_face_to_cell_B: at an outflow low side the face value itself
    const double Bx = (i > 0 || g.px) ? 0.5 * (U[4][c] + U[4][j * g.nx + wrap(i - 1, g.nx)]) : U[4][c];
    const double By = (j > 0 || g.py) ? 0.5 * (U[5][c] + U[5][wrap(j - 1, g.ny) * g.nx + i]) : U[5][c];
    Prim<double> p = get_primitive<double>(U[0][c], U[1][c], U[2][c], U[3][c], Bx, By, g.gamma, g.vol);
    t.P[0][c] = p.rho; t.P[1][c] = p.vx; t.P[2][c] = p.vy;
    t.P[3][c] = p.P; t.P[4][c] = p.Bx; t.P[5][c] = p.By;
  }
}

// Face states of one face (low cell a, high cell b along direction d), with the
// decision flags; the same operations as phase 2 of stage_kernel.
template <typename R>
__device__ __forceinline__ void face_states(const AdjGeom& g, const StageTape& t, int a, int b, int am, int bp,
                                            int ax_p, int ax_m, int ay_p, int ay_m, bool ydir, bool b_own, R* L,
                                            R* Rv, uint32_t* flags) {
  const double inv_h = ydir ? g.inv_dy : g.inv_dx;
  const double inv_2h = ydir ? g.inv_2dy : g.inv_2dx;
  const double hh = ydir ? g.hy : g.hx;
  uint32_t fl = 0;
  for (int q = 0; q < 6; ++q) {
    const double* s = t.P[q];
    const double fm = s[am], f0 = s[a], fp = s[b], fpp = s[bp];
    const double fb0 = b_own ? fp : f0;   // the high cell's low neighbour in its slope
    double sa, sb;
    if (g.slope) {
      if (g.limiter == LIMITER_VAN_LEER) {
        sa = limit_slope<double, LIMITER_VAN_LEER>((f0 - fm) * inv_h, (fp - f0) * inv_h);
        sb = limit_slope<double, LIMITER_VAN_LEER>((fp - fb0) * inv_h, (fpp - fp) * inv_h);
      } else {
        sa = limit_slope<double, LIMITER_MC>((f0 - fm) * inv_h, (fp - f0) * inv_h);
        sb = limit_slope<double, LIMITER_MC>((fp - fb0) * inv_h, (fpp - fp) * inv_h);
      }
    } else {
      sa = (fp - fm) * inv_2h;
      sb = (fpp - fb0) * inv_2h;
    }
    double vL = f0 + hh * sa;
    double vR = fp - hh * sb;
    const bool rp = (q == 0 || q == 3);
    if (g.mood) {
      double lo = dmin(dmin(dmin(dmin(f0, s[ax_p]), s[ax_m]), s[ay_p]), s[ay_m]);
      const double hi = dmax(dmax(dmax(dmax(f0, s[ax_p]), s[ax_m]), s[ay_p]), s[ay_m]);
      if (rp) lo = dmax(0.1e-8, lo);
      if (vL < lo || vL > hi) { vL = f0; fl |= 1u << (4 * q + 0); }
      if (vR < lo || vR > hi) { vR = f0; fl |= 1u << (4 * q + 1); }
    }
    if (rp) {
      if (!(vL > 1.0e-8)) fl |= 1u << (4 * q + 2);
      if (!(vR > 1.0e-8)) fl |= 1u << (4 * q + 3);
      vL = dmax(vL, 1.0e-8);
      vR = dmax(vR, 1.0e-8);
    }
    L[q] = R(vL);
    Rv[q] = R(vR);
  }
  if (L[3] - R(0.5) * (L[4] * L[4] + L[5] * L[5]) < K<R>::P_floor) {
    for (int q = 0; q < 6; ++q) L[q] = R(t.P[q][a]);
    fl |= 1u << 24;
  }
  if (Rv[3] - R(0.5) * (Rv[4] * Rv[4] + Rv[5] * Rv[5]) < K<R>::P_floor) {
    for (int q = 0; q < 6; ++q) Rv[q] = R(t.P[q][a]);
    fl |= 1u << 25;
  }
  *flags = fl;
}

// neighbour indices for the face with low cell (i, j) in direction ydir
struct FaceIdx {
  int a, b, am, bp, axp, axm, ayp, aym;
  int to;       // the cell above the face, whose update takes the face's flux if b_in
  bool b_in;    // the flux enters that cell (not past an outflow high side, nor into an
                // outflow low side's first cell through a wrap)
  bool b_own;   // mixed pair, outflow low / periodic high side: the high cell is cell 0
                // through the wrap, and its slope's low neighbour is its own ghost
};
__device__ __forceinline__ FaceIdx face_idx(const AdjGeom& g, int i, int j, bool ydir) {
  FaceIdx f;
  const int nx = g.nx, ny = g.ny;
  f.a = j * nx + i;
  if (!ydir) {
    f.b = j * nx + src(i + 1, nx, g.px, g.pxh);
    f.am = j * nx + src(i - 1, nx, g.px, g.pxh);
    f.bp = j * nx + src(i + 2, nx, g.px, g.pxh);
    f.to = j * nx + wrap(i + 1, nx);
    f.b_in = i + 1 < nx || g.px;
    f.b_own = !g.px && g.pxh && i == nx - 1;
  } else {
    f.b = src(j + 1, ny, g.py, g.pyh) * nx + i;
    f.am = src(j - 1, ny, g.py, g.pyh) * nx + i;
    f.bp = src(j + 2, ny, g.py, g.pyh) * nx + i;
    f.to = wrap(j + 1, ny) * nx + i;
    f.b_in = j + 1 < ny || g.py;
    f.b_own = !g.py && g.pyh && j == ny - 1;
  }
  f.axp = j * nx + src(i + 1, nx, g.px, g.pxh);
  f.axm = j * nx + src(i - 1, nx, g.px, g.pxh);
  f.ayp = src(j + 1, ny, g.py, g.pyh) * nx + i;
  f.aym = src(j - 1, ny, g.py, g.pyh) * nx + i;
  return f;
}

template <int SOLVER>
__global__ void k_tape_faces(AdjGeom g, StageTape t) {
  const int n = g.nx * g.ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n; k += gridDim.x * blockDim.x) {
    const bool ydir = k >= n;
    const int c = ydir ? k - n : k;
    const int i = c % g.nx, j = c / g.nx;
    const FaceIdx f = face_idx(g, i, j, ydir);
    double L[6], Rv[6];
    uint32_t fl;
    face_states<double>(g, t, f.a, f.b, f.am, f.bp, f.axp, f.axm, f.ayp, f.aym, ydir, f.b_own, L, Rv, &fl);
    const double unL = ydir ? L[2] : L[1], unR = ydir ? Rv[2] : Rv[1];
    const double utL = ydir ? L[1] : L[2], utR = ydir ? Rv[1] : Rv[2];
    const double bnL = ydir ? L[5] : L[4], bnR = ydir ? Rv[5] : Rv[4];
    const double btL = ydir ? L[4] : L[5], btR = ydir ? Rv[4] : Rv[5];
    Flux5<double> F = riemann<double, SOLVER>(g.gamma, L[0], Rv[0], unL, unR, utL, utR, L[3], Rv[3], bnL, bnR, btL, btR);
    double* const* dst = ydir ? t.Fy : t.Fx;
    dst[0][c] = F.mass;
    dst[1][c] = ydir ? F.momt : F.momn;
    dst[2][c] = ydir ? F.momn : F.momt;
    dst[3][c] = F.energy;
    dst[4][c] = F.bt;
    (ydir ? t.fly : t.flx)[c] = fl;
  }
}

__device__ __forceinline__ double Ez_at(const AdjGeom& g, const StageTape& t, int i, int j) {
  const int nx = g.nx, ny = g.ny;
  i = wrap(i, nx);
  j = wrap(j, ny);
  const double fa = t.Fx[4][j * nx + i];
  const double up = (j == ny - 1 && !g.pyh) ? fa : t.Fx[4][wrap(j + 1, ny) * nx + i];   // outflow: zero gradient
  const double fb = t.Fy[4][j * nx + i];
  const double right = (i == nx - 1 && !g.pxh) ? fb : t.Fy[4][j * nx + wrap(i + 1, nx)];
  return 0.25 * (((-fa - up) + fb) + right);
}

// Outflow boundary flux correction (src/main.f90:118-148): a cell on an
// outflow low side gets dt*dx times the physical flux of its own stage
// primitives, in x (sx) and / or in y (sy).  Same operations as the fused
// stage kernel's; R = double in the tape, dual numbers in the reverse sweep.
template <typename R>
__device__ __forceinline__ void outflow_correction(bool sx, bool sy, R ax, R ay, R gamma, R cr, R cu, R cv, R cP,
                                                   R cBx, R cBy, R* U) {
  if (sx) {
    const R hb = R(0.5) * (cBx * cBx + cBy * cBy);
    const R en = ((cP - hb) / (gamma - R(1)) + R(0.5) * cr * (cu * cu + cv * cv)) + hb;
    U[0] = U[0] + ax * cr * cu;
    U[1] = U[1] + ax * ((cr * (cu * cu) + cP) - cBx * cBx);
    U[2] = U[2] + ax * (cr * cu * cv - cBx * cBy);
    U[3] = U[3] + ax * ((en + cP) * cu - cBx * (cBx * cu + cBy * cv));
  }
  if (sy) {
    const R hb = R(0.5) * (cBx * cBx + cBy * cBy);
    const R en = ((cP - hb) / (gamma - R(1)) + R(0.5) * cr * (cu * cu + cv * cv)) + hb;
    U[0] = U[0] + ay * cr * cv;
    U[2] = U[2] + ay * ((cr * (cv * cv) + cP) - cBy * cBy);
    U[1] = U[1] + ay * (cr * cv * cu - cBy * cBx);
    U[3] = U[3] + ay * ((en + cP) * cv - cBy * (cBy * cv + cBx * cu));
  }
}

__global__ void k_tape_update(AdjGeom g, int stage, double dt, const double* const* __restrict__ Uin,
                              const double* const* __restrict__ U0, StageTape t, double* const* __restrict__ out) {
  const int n = g.nx * g.ny;
  const double ax = dt * g.dy, ay = dt * g.dx;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    const int cxm = j * g.nx + wrap(i - 1, g.nx), cym = wrap(j - 1, g.ny) * g.nx + i;
    double U[4];
    for (int q = 0; q < 4; ++q) {
      double F = Uin[q][c];
      // at an outflow low side the incoming face flux is left out
      if (i > 0 || g.px) F = (F - ax * t.Fx[q][c]) + ax * t.Fx[q][cxm];
      else F = F - ax * t.Fx[q][c];
      if (j > 0 || g.py) F = (F - ay * t.Fy[q][c]) + ay * t.Fy[q][cym];
      else F = F - ay * t.Fy[q][c];
      U[q] = F;
      t.Upre[q][c] = F;
    }
    const double Bx = t.P[4][c], By = t.P[5][c];
    conserved_floors<double>(U[0], U[1], U[2], U[3], Bx, By, g.gamma, g.vol);
    outflow_correction<double>(!g.px && i == 0, !g.py && j == 0, ax, ay, g.gamma, t.P[0][c], t.P[1][c], t.P[2][c],
                               t.P[3][c], Bx, By, U);
    const double e0 = Ez_at(g, t, i, j);
    // curl of -Ez; at an outflow low side the second row / column's difference
    const double dbx = (j > 0 || g.py) ? ((-e0) - (-Ez_at(g, t, i, j - 1))) * g.inv_dy
                                       : ((-Ez_at(g, t, i, 1)) - (-e0)) * g.inv_dy;
    const double dby = (i > 0 || g.px) ? -(((-e0) - (-Ez_at(g, t, i - 1, j))) * g.inv_dx)
                                       : -(((-Ez_at(g, t, 1, j)) - (-e0)) * g.inv_dx);
    double bx = Uin[4][c] + dt * dbx;
    double by = Uin[5][c] + dt * dby;
    if (stage == 2) {
      for (int q = 0; q < 4; ++q) U[q] = 0.75 * U0[q][c] + 0.25 * U[q];
      bx = 0.75 * U0[4][c] + 0.25 * bx;
      by = 0.75 * U0[5][c] + 0.25 * by;
    } else if (stage == 3) {
      for (int q = 0; q < 4; ++q) U[q] = (1.0 / 3.0) * U0[q][c] + (2.0 / 3.0) * U[q];
      bx = (1.0 / 3.0) * U0[4][c] + (2.0 / 3.0) * bx;
      by = (1.0 / 3.0) * U0[5][c] + (2.0 / 3.0) * by;
    }
    if (stage >= 2) {
      for (int q = 0; q < 4; ++q) t.Ublend[q][c] = U[q];
      conserved_floors<double>(U[0], U[1], U[2], U[3], Bx, By, g.gamma, g.vol);
    }
    for (int q = 0; q < 4; ++q) out[q][c] = U[q];
    out[4][c] = bx;
    out[5][c] = by;
  }
}

// ---------------------------------------------------------------------------
// reverse kernels
// ---------------------------------------------------------------------------
struct RevBuf {
  double* lUp[4];    // adjoint of the post-update (pre-floor) conserved values
  double* lBc[2];    // adjoint of the stage cell B through the floors
  double* lbp[2];    // adjoint of the post-CT face B
  double* lEz;       // adjoint of the corner Ez
  double* fX[24];    // x faces: per field q: lambda_fa, lambda_sa, lambda_fb, lambda_sb
  double* fY[24];
  double* w[24];     // per cell, field q, dir d: wL, wR at index (q*2+d)*2 + {0,1}
  double* lPc[6];    // direct face adjoints to each cell's primitives
  double* lB2[2];    // adjoint of cell Bx, By (for the face->cell average)
  double* lPcor[6];  // adjoint of a cell's primitives through the outflow flux correction
};

// floors Jacobian-transpose product at inputs (M, Mx, My, E) with cell B
__device__ __forceinline__ void floors_vjp(const AdjGeom& g, const double* Uin4, double Bx, double By,
                                           const double* lam4, double* out4, double* lB) {
  using D = Dual<6>;
  D M = seed<6>(Uin4[0], 0), Mx = seed<6>(Uin4[1], 1), My = seed<6>(Uin4[2], 2), E = seed<6>(Uin4[3], 3);
  D bx = seed<6>(Bx, 4), by = seed<6>(By, 5);
  conserved_floors<D>(M, Mx, My, E, bx, by, D(g.gamma), D(g.vol));
  const D* o[4] = {&M, &Mx, &My, &E};
  for (int k = 0; k < 6; ++k) {
    double s = 0.0;
    for (int q = 0; q < 4; ++q) s += lam4[q] * o[q]->d[k];
    if (k < 4) out4[k] = s;
    else lB[k - 4] += s;
  }
}

__global__ void k_rev_cells1(AdjGeom g, int stage, double stage_dt, const StageTape t,
                             const double* const* __restrict__ lout, RevBuf r, double* const* __restrict__ lU0acc) {
  const int n = g.nx * g.ny;
  const double c0 = (stage == 2) ? 0.75 : (1.0 / 3.0);
  const double c1 = (stage == 2) ? 0.25 : (2.0 / 3.0);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const double Bx = t.P[4][c], By = t.P[5][c];
    double lB[2] = {0.0, 0.0};
    double lpp[4];
    double lbp0, lbp1;
    if (stage >= 2) {
      double ub[4] = {t.Ublend[0][c], t.Ublend[1][c], t.Ublend[2][c], t.Ublend[3][c]};
      double lo[4] = {lout[0][c], lout[1][c], lout[2][c], lout[3][c]};
      double lbl[4];
      floors_vjp(g, ub, Bx, By, lo, lbl, lB);
      for (int q = 0; q < 4; ++q) {
        lU0acc[q][c] += c0 * lbl[q];
        lpp[q] = c1 * lbl[q];
      }
      lU0acc[4][c] += c0 * lout[4][c];
      lU0acc[5][c] += c0 * lout[5][c];
      lbp0 = c1 * lout[4][c];
      lbp1 = c1 * lout[5][c];
    } else {
      for (int q = 0; q < 4; ++q) lpp[q] = lout[q][c];
      lbp0 = lout[4][c];
      lbp1 = lout[5][c];
    }
    // outflow flux correction (added after the first floors): lpp is the
    // adjoint of the correction too; through it to the cell's stage primitives
    const int i = c % g.nx, j = c / g.nx;
    const bool sx = !g.px && i == 0, sy = !g.py && j == 0;
    double lcor[6] = {0, 0, 0, 0, 0, 0};
    if (sx || sy) {
      using D = Dual<6>;
      const double ax = stage_dt * g.dy, ay = stage_dt * g.dx;
      D pv[6];
      for (int k = 0; k < 6; ++k) pv[k] = seed<6>(t.P[k][c], k);
      D U[4] = {D(0.0), D(0.0), D(0.0), D(0.0)};
      outflow_correction<D>(sx, sy, D(ax), D(ay), D(g.gamma), pv[0], pv[1], pv[2], pv[3], pv[4], pv[5], U);
      for (int k = 0; k < 6; ++k) {
        double sacc = 0.0;
        for (int q = 0; q < 4; ++q) sacc += lpp[q] * U[q].d[k];
        lcor[k] = sacc;
      }
    }
    for (int k = 0; k < 6; ++k) r.lPcor[k][c] = lcor[k];
    double up[4] = {t.Upre[0][c], t.Upre[1][c], t.Upre[2][c], t.Upre[3][c]};
    double lu[4];
    floors_vjp(g, up, Bx, By, lpp, lu, lB);
    for (int q = 0; q < 4; ++q) r.lUp[q][c] = lu[q];
    r.lBc[0][c] = lB[0];
    r.lBc[1][c] = lB[1];
    r.lbp[0][c] = lbp0;
    r.lbp[1][c] = lbp1;
  }
}

// lambda_Ez at corner (i+1/2, j+1/2): b_x(i,j) gets -dt/dy Ez(i,j), b_x(i,j+1)
// gets +dt/dy Ez(i,j); b_y(i,j) gets +dt/dx Ez(i,j), b_y(i+1,j) gets -dt/dx.
// At an outflow low side b_x(i,0) takes row 1's difference, dt/dy (Ez(i,0) -
// Ez(i,1)), and b_y(0,j) column 1's, dt/dx (Ez(1,j) - Ez(0,j)); past an
// outflow high side there is no b_x(i,ny) / b_y(nx,j).
__global__ void k_rev_corners(AdjGeom g, double dt, RevBuf r) {
  const int n = g.nx * g.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    const int cyp = wrap(j + 1, g.ny) * g.nx + i;
    const int cxp = j * g.nx + wrap(i + 1, g.nx);
    double sx = 0.0, sy = 0.0;
    if (j + 1 < g.ny || g.py) sx += r.lbp[0][cyp];
    if (j > 0 || g.py) sx -= r.lbp[0][c];
    if (!g.py && j == 0) sx += r.lbp[0][i];
    if (!g.py && j == 1) sx -= r.lbp[0][i];
    if (i > 0 || g.px) sy += r.lbp[1][c];
    if (i + 1 < g.nx || g.px) sy -= r.lbp[1][cxp];
    if (!g.px && i == 0) sy -= r.lbp[1][j * g.nx];
    if (!g.px && i == 1) sy += r.lbp[1][j * g.nx];
    r.lEz[c] = dt * g.inv_dy * sx + dt * g.inv_dx * sy;
  }
}

template <int SOLVER>
__global__ void k_rev_faces(AdjGeom g, double dt, StageTape t, RevBuf r) {
  const int n = g.nx * g.ny;
  const double ax = dt * g.dy, ay = dt * g.dx;
  using D = Dual<12>;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n; k += gridDim.x * blockDim.x) {
    const bool ydir = k >= n;
    const int c = ydir ? k - n : k;
    const int i = c % g.nx, j = c / g.nx;
    const FaceIdx f = face_idx(g, i, j, ydir);
    // adjoint of this face's 5 fluxes (conserved ordering)
    double lF[5];
    const double wgt = ydir ? ay : ax;
    // the flux leaves cell a and enters cell b (none past an outflow high side)
    for (int q = 0; q < 4; ++q) lF[q] = wgt * ((f.b_in ? r.lUp[q][f.to] : 0.0) - r.lUp[q][c]);
    // Ez(i,j) = 1/4 (-Fx(i,j) - Fx(i,j+1) + Fy(i,j) + Fy(i+1,j)); at an outflow
    // high side Fx(i,ny) / Fy(nx,j) is the face itself (zero gradient)
    const double e0 = r.lEz[c];
    if (!ydir) {
      double s4 = (j > 0 || g.pyh) ? e0 + r.lEz[wrap(j - 1, g.ny) * g.nx + i] : e0;
      if (j == g.ny - 1 && !g.pyh) s4 += e0;
      lF[4] = -0.25 * s4;
    } else {
      double s4 = (i > 0 || g.pxh) ? e0 + r.lEz[j * g.nx + wrap(i - 1, g.nx)] : e0;
      if (i == g.nx - 1 && !g.pxh) s4 += e0;
      lF[4] = 0.25 * s4;
    }
    // recompute the face states (values + flags), then the flux Jacobian
    double L[6], Rv[6];
    uint32_t fl;
    face_states<double>(g, t, f.a, f.b, f.am, f.bp, f.axp, f.axm, f.ayp, f.aym, ydir, f.b_own, L, Rv, &fl);
    // solver inputs in (normal, tangential) order, seeded 0..11
    const int perm[6] = {0, ydir ? 2 : 1, ydir ? 1 : 2, 3, ydir ? 5 : 4, ydir ? 4 : 5};  // input slot -> field
    D in[12];
    for (int s = 0; s < 6; ++s) {
      in[2 * s] = seed<12>(L[perm[s]], 2 * s);
      in[2 * s + 1] = seed<12>(Rv[perm[s]], 2 * s + 1);
    }
    Flux5<D> F = riemann<D, SOLVER>(D(g.gamma), in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8],
                                    in[9], in[10], in[11]);
    // map conserved-ordered lF onto the solver outputs (mass, momn, momt, energy, bt)
    const double lo_mass = lF[0], lo_mn = ydir ? lF[2] : lF[1], lo_mt = ydir ? lF[1] : lF[2];
    const double lo_e = lF[3], lo_bt = lF[4];
    double lL[6] = {0, 0, 0, 0, 0, 0}, lR[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < 6; ++s) {
      for (int side = 0; side < 2; ++side) {
        const int kk = 2 * s + side;
        const double v = lo_mass * F.mass.d[kk] + lo_mn * F.momn.d[kk] + lo_mt * F.momt.d[kk] +
                         lo_e * F.energy.d[kk] + lo_bt * F.bt.d[kk];
        if (side == 0) lL[perm[s]] += v;
        else lR[perm[s]] += v;
      }
    }
    // through the thermal check, face floors and MOOD to cell values and slopes
    const double hh = ydir ? g.hy : g.hx;
    double* const* dst = ydir ? r.fY : r.fX;
    const bool thL = fl & (1u << 24), thR = fl & (1u << 25);
    for (int q = 0; q < 6; ++q) {
      double l_fa = 0.0, l_sa = 0.0, l_fb = 0.0, l_sb = 0.0;
      if (thL) {
        l_fa += lL[q];
      } else if (!(fl & (1u << (4 * q + 2)))) {
        if (fl & (1u << (4 * q + 0))) l_fa += lL[q];
        else { l_fa += lL[q]; l_sa += hh * lL[q]; }
      }
      if (thR) {
        l_fa += lR[q];
      } else if (!(fl & (1u << (4 * q + 3)))) {
        if (fl & (1u << (4 * q + 1))) l_fa += lR[q];
        else { l_fb += lR[q]; l_sb -= hh * lR[q]; }
      }
      dst[4 * q + 0][c] = l_fa;
      dst[4 * q + 1][c] = l_sa;
      dst[4 * q + 2][c] = l_fb;
      dst[4 * q + 3][c] = l_sb;
    }
  }
}

// per cell: gather the slope adjoints from the faces, apply the limiter's
// local derivative, and gather the direct value adjoints
__global__ void k_rev_slopes(AdjGeom g, StageTape t, RevBuf r) {
  const int n = g.nx * g.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    // the slope stencil of this cell (each side's ghost rule)
    const int cxm = j * g.nx + src(i - 1, g.nx, g.px, g.pxh), cym = src(j - 1, g.ny, g.py, g.pyh) * g.nx + i;
    const int cxp = j * g.nx + src(i + 1, g.nx, g.px, g.pxh), cyp = src(j + 1, g.ny, g.py, g.pyh) * g.nx + i;
    // the face below this cell, whose high cell it is: none at x = 0 / y = 0
    // unless the high side wraps to it; past an outflow high side the ghost's
    // value is this cell's (its slope, from two equal differences, depends on
    // no cell)
    const int fxm = j * g.nx + wrap(i - 1, g.nx), fym = wrap(j - 1, g.ny) * g.nx + i;
    const bool hx = i > 0 || g.pxh, hy = j > 0 || g.pyh;
    const bool ex = !g.pxh && i == g.nx - 1, ey = !g.pyh && j == g.ny - 1;
    for (int q = 0; q < 6; ++q) {
      // this cell is the low cell of faces (c, x) and (c, y), the high cell of (cxm, x) and (cym, y)
      double lv = r.fX[4 * q + 0][c] + r.fY[4 * q + 0][c] + (hx ? r.fX[4 * q + 2][fxm] : 0.0) +
                  (hy ? r.fY[4 * q + 2][fym] : 0.0);
      if (ex) lv += r.fX[4 * q + 2][c];
      if (ey) lv += r.fY[4 * q + 2][c];
      r.lPc[q][c] = lv;
      for (int d = 0; d < 2; ++d) {
        const double ls = (d == 0) ? (r.fX[4 * q + 1][c] + (hx ? r.fX[4 * q + 3][fxm] : 0.0))
                                   : (r.fY[4 * q + 1][c] + (hy ? r.fY[4 * q + 3][fym] : 0.0));
        const double fm = t.P[q][d == 0 ? cxm : cym], f0 = t.P[q][c], fp = t.P[q][d == 0 ? cxp : cyp];
        const double inv_h = d == 0 ? g.inv_dx : g.inv_dy;
        double wl, wr;
        if (g.slope) {
          using D2 = Dual<2>;
          D2 dl = seed<2>((f0 - fm) * inv_h, 0), dr = seed<2>((fp - f0) * inv_h, 1);
          D2 s = (g.limiter == LIMITER_VAN_LEER) ? limit_slope<D2, LIMITER_VAN_LEER>(dl, dr)
                                                 : limit_slope<D2, LIMITER_MC>(dl, dr);
          double dsl = s.d[0], dsr = s.d[1];
          // Kink convention where a one-sided difference is exactly zero (a
          // uniform neighbourhood): both zero -> the centred slope's (1/2, 1/2),
          // the limit along dfL = dfR for MC and Van Leer; one zero -> the mean
          // of the one-sided derivatives, 1 w.r.t. the zero argument (the
          // limiters grow as 2|df| on the active side), 0 w.r.t. the other.
          if (dl.v == 0.0 && dr.v == 0.0) { dsl = 0.5; dsr = 0.5; }
          else if (dl.v == 0.0) { dsl = 1.0; dsr = 0.0; }
          else if (dr.v == 0.0) { dsl = 0.0; dsr = 1.0; }
          wl = ls * dsl * inv_h;
          wr = ls * dsr * inv_h;
        } else {
          const double inv_2h = d == 0 ? g.inv_2dx : g.inv_2dy;
          wl = ls * inv_2h;
          wr = ls * inv_2h;
        }
        r.w[(q * 2 + d) * 2 + 0][c] = wl;
        r.w[(q * 2 + d) * 2 + 1][c] = wr;
      }
    }
  }
}

// per cell: primitive adjoints -> conserved adjoints (+ cell B adjoints)
__global__ void k_rev_prims(AdjGeom g, StageTape t, RevBuf r, const double* const* __restrict__ Uin,
                            double* const* __restrict__ lin) {
  const int n = g.nx * g.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    const int cxm = j * g.nx + wrap(i - 1, g.nx), cym = wrap(j - 1, g.ny) * g.nx + i;
    const int cxp = j * g.nx + wrap(i + 1, g.nx), cyp = wrap(j + 1, g.ny) * g.nx + i;
    double lP[6];
    for (int q = 0; q < 6; ++q) {
      double v = r.lPc[q][c];
      // slopes: s(p) uses f(p-1), f(p), f(p+1).  At an outflow side the ghost
      // beyond is this cell: at the low side s(0)'s f(-1) and f(0) terms
      // cancel to -w1, at the high side s(nx-1)'s f(nx-1) and f(nx) terms to w0
      for (int d = 0; d < 2; ++d) {
        const double* w0 = r.w[(q * 2 + d) * 2 + 0];
        const double* w1 = r.w[(q * 2 + d) * 2 + 1];
        const bool per = d == 0 ? g.px : g.py, perh = d == 0 ? g.pxh : g.pyh;
        const int k = d == 0 ? i : j, nk = d == 0 ? g.nx : g.ny;
        const int cm = d == 0 ? cxm : cym, cp = d == 0 ? cxp : cyp;
        if (per != perh) {
          // a mixed pair: this cell's own slope, with its own ghost below / above
          // where that side is outflow, then the slopes of the cells whose low /
          // high neighbour it is (across a periodic side, through the wrap)
          const int wm = d == 0 ? j * g.nx + wrap(i - 1, g.nx) : wrap(j - 1, g.ny) * g.nx + i;
          const int wp = d == 0 ? j * g.nx + wrap(i + 1, g.nx) : wrap(j + 1, g.ny) * g.nx + i;
          double own = w0[c] - w1[c];
          if (k == 0 && !per) own -= w0[c];
          if (k == nk - 1 && !perh) own += w1[c];
          v += own;
          if (k + 1 < nk || per) v -= w0[wp];
          if (k > 0 || perh) v += w1[wm];
        } else if (per || (k > 0 && k < nk - 1)) {
          v += w0[c] - w1[c] - w0[cp] + w1[cm];
        } else if (k == 0) {
          v += (-w1[c]) - w0[cp];
        } else {
          v += w0[c] + w1[cm];
        }
      }
      lP[q] = v;
    }
    lP[4] += r.lBc[0][c];
    lP[5] += r.lBc[1][c];
    for (int q = 0; q < 6; ++q) lP[q] += r.lPcor[q][c];
    using D = Dual<6>;
    const double Bx = t.P[4][c], By = t.P[5][c];
    D M = seed<6>(Uin[0][c], 0), Mx = seed<6>(Uin[1][c], 1), My = seed<6>(Uin[2][c], 2);
    D E = seed<6>(Uin[3][c], 3), bx = seed<6>(Bx, 4), by = seed<6>(By, 5);
    Prim<D> p = get_primitive<D>(M, Mx, My, E, bx, by, D(g.gamma), D(g.vol));
    const D* o[4] = {&p.rho, &p.vx, &p.vy, &p.P};
    double lv[6];
    for (int k = 0; k < 6; ++k) {
      double s = 0.0;
      for (int q = 0; q < 4; ++q) s += lP[q] * o[q]->d[k];
      lv[k] = s;
    }
    for (int q = 0; q < 4; ++q) lin[q][c] = r.lUp[q][c] + lv[q];   // identity path of the update
    r.lB2[0][c] = lP[4] + lv[4];
    r.lB2[1][c] = lP[5] + lv[5];
  }
}

// per cell: face B adjoint = CT identity + the two cell averages it enters
__global__ void k_rev_faceB(AdjGeom g, RevBuf r, double* const* __restrict__ lin) {
  const int n = g.nx * g.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % g.nx, j = c / g.nx;
    const int cxp = j * g.nx + wrap(i + 1, g.nx), cyp = wrap(j + 1, g.ny) * g.nx + i;
    // b_x(i) enters Bx(i) (alone at an outflow low side) and Bx(i+1) (none past the high side)
    lin[4][c] = r.lbp[0][c] + ((i > 0 || g.px) ? 0.5 : 1.0) * r.lB2[0][c] +
                ((i + 1 < g.nx || g.px) ? 0.5 * r.lB2[0][cxp] : 0.0);
    lin[5][c] = r.lbp[1][c] + ((j > 0 || g.py) ? 0.5 : 1.0) * r.lB2[1][c] +
                ((j + 1 < g.ny || g.py) ? 0.5 * r.lB2[1][cyp] : 0.0);
  }
}

__global__ void k_axpy6(double* const* __restrict__ y, const double* const* __restrict__ x, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    for (int q = 0; q < 6; ++q) y[q][c] += x[q][c];
}

__global__ void k_zero6(double* const* __restrict__ y, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    for (int q = 0; q < 6; ++q) y[q][c] = 0.0;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct chimera_adjoint {
  AdjGeom g;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int n = 0;
  int grid = 0;
  double* pool = nullptr;
  StageTape tape[3];
  RevBuf rev;
  double* U1[6];
  double* U2[6];
  double* lA[6];     // stage adjoint buffers
  double* lB[6];
  double* lU0[6];    // accumulated U^n adjoint from the blends
  double** dptrs = nullptr;   // device copies of pointer arrays
};

namespace {
// device pointer-array slots
enum { P_UN = 0, P_U1 = 6, P_U2 = 12, P_LA = 18, P_LB = 24, P_LU0 = 30, P_LNEXT = 36, P_LOUT = 42, P_UNEXT = 48,
       P_COUNT = 54 };
}

static int adj_fail() {
  cudaGetLastError();
  return CHIMERA_ERR_CUDA;
}

extern "C" int chimera_adjoint_create(const chimera_cfg* cfg, void* stream, chimera_adjoint** out) {
  if (!cfg || !out) return CHIMERA_ERR_BAD_ARG;
  *out = nullptr;
  if (cfg->nx < 4 || cfg->ny < 4 || !(cfg->dx > 0) || !(cfg->dy > 0) || !(cfg->gamma > 1.0)) return CHIMERA_ERR_BAD_ARG;
  if (cfg->riemann < 1 || cfg->riemann > 3 || cfg->limiter < 1 || cfg->limiter > 2) return CHIMERA_ERR_BAD_ARG;
  for (int b : {cfg->bc_xlo, cfg->bc_xhi, cfg->bc_ylo, cfg->bc_yhi})
    if (b < CHIMERA_BC_PERIODIC || b > CHIMERA_BC_INFLOW) return CHIMERA_ERR_BAD_ARG;
  // every non-periodic kind acts as outflow (src/mhd_bc.f90:36-121), each
  // side on its own (a periodic side may face an outflow one)
  if (cfg->precision != CHIMERA_FP64) return CHIMERA_ERR_UNSUPPORTED;
  if ((long long)cfg->nx * cfg->ny >= (1LL << 31)) return CHIMERA_ERR_TOO_LARGE;   // int cell indices
  chimera_adjoint* a = new (std::nothrow) chimera_adjoint();
  if (!a) return CHIMERA_ERR_NOMEM;
  AdjGeom& g = a->g;
  g.nx = cfg->nx; g.ny = cfg->ny;
  g.dx = cfg->dx; g.dy = cfg->dy;
  g.inv_dx = 1.0 / cfg->dx; g.inv_dy = 1.0 / cfg->dy;
  g.inv_2dx = 1.0 / (2.0 * cfg->dx); g.inv_2dy = 1.0 / (2.0 * cfg->dy);
  g.hx = 0.5 * cfg->dx; g.hy = 0.5 * cfg->dy;
  g.gamma = cfg->gamma;
  g.vol = cfg->dx * cfg->dy;
  g.riemann = cfg->riemann; g.limiter = cfg->limiter;
  g.slope = cfg->use_slope_limiting ? 1 : 0;
  g.mood = cfg->mood ? 1 : 0;
  g.px = cfg->bc_xlo == CHIMERA_BC_PERIODIC;
  g.py = cfg->bc_ylo == CHIMERA_BC_PERIODIC;
  g.pxh = cfg->bc_xhi == CHIMERA_BC_PERIODIC;
  g.pyh = cfg->bc_yhi == CHIMERA_BC_PERIODIC;
  a->n = cfg->nx * cfg->ny;
  if (stream) a->stream = (cudaStream_t)stream;
  else {
    if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess) { delete a; return adj_fail(); }
    a->own_stream = true;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  a->grid = sms * 8;
  // doubles per cell: tapes 3 x (6 P + 10 F + 4 Upre + 4 Ublend) + 2 flag words (as 1 double)
  // + reverse (4 + 2 + 2 + 1 + 48 + 24 + 6 + 2 + 6) + U1, U2, lA, lB, lU0 (30)
  const size_t per_cell = 3 * (24 + 1) + (4 + 2 + 2 + 1 + 48 + 24 + 6 + 2 + 6) + 30;
  const size_t n = size_t(a->n);
  if (cudaMalloc(&a->pool, per_cell * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&a->dptrs, P_COUNT * sizeof(double*)) != cudaSuccess) {
    cudaGetLastError();
    chimera_adjoint_destroy(a);
    return CHIMERA_ERR_NOMEM;
  }
  double* p = a->pool;
  auto take = [&]() { double* r = p; p += n; return r; };
  for (int k = 0; k < 3; ++k) {
    StageTape& t = a->tape[k];
    for (int q = 0; q < 6; ++q) t.P[q] = take();
    for (int q = 0; q < 5; ++q) t.Fx[q] = take();
    for (int q = 0; q < 5; ++q) t.Fy[q] = take();
    for (int q = 0; q < 4; ++q) t.Upre[q] = take();
    for (int q = 0; q < 4; ++q) t.Ublend[q] = take();
    uint32_t* fw = reinterpret_cast<uint32_t*>(take());   // 2 x n flag words in n doubles
    t.flx = fw;
    t.fly = fw + n;
  }
  RevBuf& r = a->rev;
  for (int q = 0; q < 4; ++q) r.lUp[q] = take();
  for (int q = 0; q < 2; ++q) r.lBc[q] = take();
  for (int q = 0; q < 2; ++q) r.lbp[q] = take();
  r.lEz = take();
  for (int q = 0; q < 24; ++q) r.fX[q] = take();
  for (int q = 0; q < 24; ++q) r.fY[q] = take();
  for (int q = 0; q < 24; ++q) r.w[q] = take();
  for (int q = 0; q < 6; ++q) r.lPc[q] = take();
  for (int q = 0; q < 2; ++q) r.lB2[q] = take();
  for (int q = 0; q < 6; ++q) r.lPcor[q] = take();
  for (int q = 0; q < 6; ++q) a->U1[q] = take();
  for (int q = 0; q < 6; ++q) a->U2[q] = take();
  for (int q = 0; q < 6; ++q) a->lA[q] = take();
  for (int q = 0; q < 6; ++q) a->lB[q] = take();
  for (int q = 0; q < 6; ++q) a->lU0[q] = take();
  *out = a;
  return CHIMERA_OK;
}

extern "C" void chimera_adjoint_destroy(chimera_adjoint* a) {
  if (!a) return;
  if (a->stream) cudaStreamSynchronize(a->stream);
  cudaFree(a->pool);
  cudaFree(a->dptrs);
  if (a->own_stream && a->stream) cudaStreamDestroy(a->stream);
  cudaGetLastError();
  delete a;
}

// Upload the pointer arrays a launch needs (one H2D copy per call).
static int upload_ptrs(chimera_adjoint* a, const double* const* Un, const double* const* lnext, double* const* lout,
                       double* const* Unext) {
  double* h[P_COUNT];
  memset(h, 0, sizeof(h));
  for (int q = 0; q < 6; ++q) {
    h[P_UN + q] = const_cast<double*>(Un ? Un[q] : nullptr);
    h[P_U1 + q] = a->U1[q];
    h[P_U2 + q] = a->U2[q];
    h[P_LA + q] = a->lA[q];
    h[P_LB + q] = a->lB[q];
    h[P_LU0 + q] = a->lU0[q];
    h[P_LNEXT + q] = const_cast<double*>(lnext ? lnext[q] : nullptr);
    h[P_LOUT + q] = lout ? lout[q] : nullptr;
    h[P_UNEXT + q] = Unext ? Unext[q] : nullptr;
  }
  if (cudaMemcpyAsync(a->dptrs, h, sizeof(h), cudaMemcpyHostToDevice, a->stream) != cudaSuccess) return adj_fail();
  return CHIMERA_OK;
}

template <int SOLVER>
static void tape_stage(chimera_adjoint* a, int stage, double dt, double** in, double** u0, double** out) {
  const int grid = a->grid;
  StageTape& t = a->tape[stage - 1];
  k_tape_prims<<<grid, 256, 0, a->stream>>>(a->g, in, t);
  k_tape_faces<SOLVER><<<grid, 128, 0, a->stream>>>(a->g, t);
  k_tape_update<<<grid, 256, 0, a->stream>>>(a->g, stage, dt, in, u0, t, out);
}

template <int SOLVER>
static void rev_stage(chimera_adjoint* a, int stage, double dt, double** in, double** lout, double** lin,
                      double** lU0) {
  const int grid = a->grid;
  StageTape& t = a->tape[stage - 1];
  k_rev_cells1<<<grid, 256, 0, a->stream>>>(a->g, stage, dt, t, lout, a->rev, lU0);
  k_rev_corners<<<grid, 256, 0, a->stream>>>(a->g, dt, a->rev);
  k_rev_faces<SOLVER><<<grid, 64, 0, a->stream>>>(a->g, dt, t, a->rev);
  k_rev_slopes<<<grid, 128, 0, a->stream>>>(a->g, t, a->rev);
  k_rev_prims<<<grid, 128, 0, a->stream>>>(a->g, t, a->rev, in, lin);
  k_rev_faceB<<<grid, 256, 0, a->stream>>>(a->g, a->rev, lin);
}

template <int SOLVER>
static void forward_step(chimera_adjoint* a, double dt, double** d) {
  tape_stage<SOLVER>(a, 1, dt, d + P_UN, d + P_UN, d + P_U1);
  tape_stage<SOLVER>(a, 2, dt, d + P_U1, d + P_UN, d + P_U2);
  tape_stage<SOLVER>(a, 3, dt, d + P_U2, d + P_UN, d + P_UNEXT);
}

template <int SOLVER>
static void adjoint_step(chimera_adjoint* a, double dt, double** d) {
  forward_step<SOLVER>(a, dt, d);
  k_zero6<<<a->grid, 256, 0, a->stream>>>(d + P_LU0, a->n);
  rev_stage<SOLVER>(a, 3, dt, d + P_U2, d + P_LNEXT, d + P_LA, d + P_LU0);   // lambda_U2 -> lA
  rev_stage<SOLVER>(a, 2, dt, d + P_U1, d + P_LA, d + P_LB, d + P_LU0);      // lambda_U1 -> lB
  rev_stage<SOLVER>(a, 1, dt, d + P_UN, d + P_LB, d + P_LOUT, d + P_LU0);    // direct lambda_Un
  k_axpy6<<<a->grid, 256, 0, a->stream>>>(d + P_LOUT, d + P_LU0, a->n);
}

extern "C" int chimera_adjoint_step(chimera_adjoint* a, const double* const* U_n, double dt,
                                    const double* const* lambda_next, double* const* lambda_n) {
  if (!a || !U_n || !lambda_next || !lambda_n || !(dt > 0.0)) return CHIMERA_ERR_BAD_ARG;
  for (int q = 0; q < 6; ++q)
    if (!doubles_ok({U_n[q], lambda_next[q], lambda_n[q]})) return CHIMERA_ERR_BAD_ARG;
  // U_{n+1} of the tape forward is not needed: write it into the stage-1 adjoint buffer
  int rc = upload_ptrs(a, U_n, lambda_next, lambda_n, a->lA);
  if (rc) return rc;
  switch (a->g.riemann) {
    case CHIMERA_RIEMANN_RUSANOV: adjoint_step<RIEMANN_RUSANOV>(a, dt, a->dptrs); break;
    case CHIMERA_RIEMANN_HLLE: adjoint_step<RIEMANN_HLLE>(a, dt, a->dptrs); break;
    default: adjoint_step<RIEMANN_HLLD>(a, dt, a->dptrs); break;
  }
  if (cudaGetLastError() != cudaSuccess) return CHIMERA_ERR_CUDA;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return adj_fail();
  return CHIMERA_OK;
}

extern "C" int chimera_adjoint_forward_step(chimera_adjoint* a, const double* const* U_n, double dt,
                                            double* const* U_next) {
  if (!a || !U_n || !U_next || !(dt > 0.0)) return CHIMERA_ERR_BAD_ARG;
  for (int q = 0; q < 6; ++q)
    if (!doubles_ok({U_n[q], U_next[q]})) return CHIMERA_ERR_BAD_ARG;
  int rc = upload_ptrs(a, U_n, nullptr, nullptr, U_next);
  if (rc) return rc;
  switch (a->g.riemann) {
    case CHIMERA_RIEMANN_RUSANOV: forward_step<RIEMANN_RUSANOV>(a, dt, a->dptrs); break;
    case CHIMERA_RIEMANN_HLLE: forward_step<RIEMANN_HLLE>(a, dt, a->dptrs); break;
    default: forward_step<RIEMANN_HLLD>(a, dt, a->dptrs); break;
  }
  if (cudaGetLastError() != cudaSuccess) return CHIMERA_ERR_CUDA;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return adj_fail();
  return CHIMERA_OK;
}
