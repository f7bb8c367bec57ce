// unit_ops.cu -- the reference's module routines, one GPU kernel each.
//
// Same names, argument meaning and boundary handling as the Fortran routines
// they cite (including a side that is periodic while its opposite side is
// not), on dense device arrays (nx, ny) with x fastest; the arithmetic is the
// device code of mhd_device.cuh that the fused stage kernel uses, compiled
// with --fmad=false.  They exist so that each routine can be checked on its
// own -- the reference's Fortran known-answer tests run on them -- and for
// callers that port the time loop routine by routine.
#include <cuda_runtime.h>

#include "../../include/chimera_gpu.h"
#include "abi_check.h"
#include "mhd_device.cuh"

using namespace chimera;

namespace {

struct OpGeom {
  int nx, ny;
  int xlo, xhi, ylo, yhi;       // periodic flags per side
  double dx, dy, gamma, vol;
  int riemann, limiter;
};

int make_geom(const chimera_cfg* c, OpGeom* g) {
  if (!c || c->nx < 2 || c->ny < 2 || !(c->dx > 0) || !(c->dy > 0)) return CHIMERA_ERR_BAD_ARG;
  for (int side : {c->bc_xlo, c->bc_xhi, c->bc_ylo, c->bc_yhi})
    if (side < CHIMERA_BC_PERIODIC || side > CHIMERA_BC_INFLOW) return CHIMERA_ERR_BAD_ARG;
  // the kernels index the (nx + 2) x (ny + 2) padded arrays with int
  if ((long long)(c->nx + 2) * (c->ny + 2) > 0x7fffffffLL) return CHIMERA_ERR_TOO_LARGE;
  g->nx = c->nx; g->ny = c->ny;
  g->xlo = c->bc_xlo == CHIMERA_BC_PERIODIC; g->xhi = c->bc_xhi == CHIMERA_BC_PERIODIC;
  g->ylo = c->bc_ylo == CHIMERA_BC_PERIODIC; g->yhi = c->bc_yhi == CHIMERA_BC_PERIODIC;
  g->dx = c->dx; g->dy = c->dy; g->gamma = c->gamma; g->vol = c->dx * c->dy;
  g->riemann = c->riemann; g->limiter = c->limiter;
  if (c->riemann < 1 || c->riemann > 3 || c->limiter < 1 || c->limiter > 2) return CHIMERA_ERR_BAD_ARG;
  return CHIMERA_OK;
}

#define GRID_LOOP(n) for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < (n); c += gridDim.x * blockDim.x)

int finish(cudaStream_t s) {
  (void)s;
  return cudaGetLastError() == cudaSuccess ? CHIMERA_OK : CHIMERA_ERR_CUDA;
}

constexpr int NB = 256;
int nblocks(long long n) { return int((n + NB - 1) / NB > 4096 ? 4096 : (n + NB - 1) / NB); }

// src/mhd_field_ops.f90:120-156
__global__ void k_avg_B(OpGeom g, const double* bx, const double* by, double* Bx, double* By) {
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    if (i > 0) Bx[c] = 0.5 * (bx[c] + bx[c - 1]);
    else Bx[c] = g.xlo ? 0.5 * (bx[c] + bx[c + g.nx - 1]) : bx[c];
    if (j > 0) By[c] = 0.5 * (by[c] + by[c - g.nx]);
    else By[c] = g.ylo ? 0.5 * (by[c] + by[c + (g.ny - 1) * g.nx]) : by[c];
  }
}

// src/mhd_change_states.f90:61-113
__global__ void k_get_primitive(OpGeom g, const double* M, const double* Mx, const double* My, const double* E,
                                const double* Bx, const double* By, double* rho, double* vx, double* vy,
                                double* P) {
  GRID_LOOP(g.nx * g.ny) {
    Prim<double> p = get_primitive<double>(M[c], Mx[c], My[c], E[c], Bx[c], By[c], g.gamma, g.vol);
    rho[c] = p.rho; vx[c] = p.vx; vy[c] = p.vy; P[c] = p.P;
  }
}

// src/mhd_change_states.f90:16-58
__global__ void k_get_conserved(OpGeom g, const double* rho, const double* vx, const double* vy, const double* P,
                                const double* Bx, const double* By, double* M, double* Mx, double* My,
                                double* E) {
  GRID_LOOP(g.nx * g.ny) {
    get_conserved<double>(rho[c], vx[c], vy[c], P[c], Bx[c], By[c], g.gamma, g.vol, M[c], Mx[c], My[c], E[c]);
  }
}

// src/mhd_change_states.f90:116-166
__global__ void k_floors(OpGeom g, double* M, double* Mx, double* My, double* E, const double* Bx,
                         const double* By) {
  GRID_LOOP(g.nx * g.ny) {
    double m = M[c], mx = Mx[c], my = My[c], e = E[c];
    conserved_floors<double>(m, mx, my, e, Bx[c], By[c], g.gamma, g.vol);
    M[c] = m; Mx[c] = mx; My[c] = my; E[c] = e;
  }
}

// src/mhd_bc.f90:36-170 (pad (nx+2) x (ny+2), physical (i,j) -> (i+1, j+1))
__device__ double corner_val(const OpGeom& g, const double* f, int ix, int iy, int px, int py) {
  const int ixw = g.nx - 1 - ix, iyw = g.ny - 1 - iy;   // 0-based opposite corner
  if (px && py) return f[iyw * g.nx + ixw];
  if (px) return f[iy * g.nx + ixw];
  if (py) return f[iyw * g.nx + ix];
  return f[iy * g.nx + ix];
}
__global__ void k_fill_ghost(OpGeom g, const double* f, double* pad) {
  const int W = g.nx + 2, H = g.ny + 2;
  GRID_LOOP(W * H) {
    const int pi = c % W, pj = c / W;
    const int i = pi - 1, j = pj - 1;
    const bool gx = (i < 0 || i >= g.nx), gy = (j < 0 || j >= g.ny);
    double v;
    if (gx && gy) {
      if (i < 0 && j < 0) v = corner_val(g, f, 0, 0, g.xlo, g.ylo);
      else if (i >= g.nx && j < 0) v = corner_val(g, f, g.nx - 1, 0, g.xhi, g.ylo);
      else if (i < 0) v = corner_val(g, f, 0, g.ny - 1, g.xlo, g.yhi);
      else v = corner_val(g, f, g.nx - 1, g.ny - 1, g.xhi, g.yhi);
    } else if (gx) {
      if (i < 0) v = g.xlo ? f[j * g.nx + g.nx - 1] : f[j * g.nx];
      else v = g.xhi ? f[j * g.nx] : f[j * g.nx + g.nx - 1];
    } else if (gy) {
      if (j < 0) v = g.ylo ? f[(g.ny - 1) * g.nx + i] : f[i];
      else v = g.yhi ? f[i] : f[(g.ny - 1) * g.nx + i];
    } else {
      v = f[j * g.nx + i];
    }
    pad[c] = v;
  }
}

// src/mhd_derivatives.f90:15-47 and :50-127
__global__ void k_slopes(OpGeom g, const double* pad, double* fdx, double* fdy, int limited) {
  const int W = g.nx + 2;
  const double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  const double inv_2dx = 1.0 / (2.0 * g.dx), inv_2dy = 1.0 / (2.0 * g.dy);
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    const double f0 = pad[(j + 1) * W + i + 1];
    const double xm = pad[(j + 1) * W + i], xp = pad[(j + 1) * W + i + 2];
    const double ym = pad[j * W + i + 1], yp = pad[(j + 2) * W + i + 1];
    if (!limited) {
      fdx[c] = (xp - xm) * inv_2dx;
      fdy[c] = (yp - ym) * inv_2dy;
    } else if (g.limiter == LIMITER_VAN_LEER) {
      fdx[c] = limit_slope<double, LIMITER_VAN_LEER>((f0 - xm) * inv_dx, (xp - f0) * inv_dx);
      fdy[c] = limit_slope<double, LIMITER_VAN_LEER>((f0 - ym) * inv_dy, (yp - f0) * inv_dy);
    } else {
      fdx[c] = limit_slope<double, LIMITER_MC>((f0 - xm) * inv_dx, (xp - f0) * inv_dx);
      fdy[c] = limit_slope<double, LIMITER_MC>((f0 - ym) * inv_dy, (yp - f0) * inv_dy);
    }
  }
}

// src/mhd_derivatives.f90:130-229
__global__ void k_reconstruction(OpGeom g, const double* f, const double* fdx, const double* fdy, double* XL,
                                 double* XR, double* YL, double* YR, int rho_or_p, int mood) {
  const double hx = 0.5 * g.dx, hy = 0.5 * g.dy;
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    const double f0 = f[c];
    double xl = f0 + hx * fdx[c];
    double yl = f0 + hy * fdy[c];
    double xr, yr;
    if (i < g.nx - 1) xr = f[c + 1] - hx * fdx[c + 1];
    else xr = g.xhi ? f[j * g.nx] - hx * fdx[j * g.nx] : f0;
    if (j < g.ny - 1) yr = f[c + g.nx] - hy * fdy[c + g.nx];
    else yr = g.yhi ? f[i] - hy * fdy[i] : f0;
    if (mood) {
      const int ip1 = g.xhi ? (i + 1) % g.nx : min(i + 1, g.nx - 1);
      const int im1 = g.xlo ? (i - 1 + g.nx) % g.nx : max(i - 1, 0);
      const int jp1 = g.yhi ? (j + 1) % g.ny : min(j + 1, g.ny - 1);
      const int jm1 = g.ylo ? (j - 1 + g.ny) % g.ny : max(j - 1, 0);
      const double a = f[j * g.nx + ip1], b = f[j * g.nx + im1], cc = f[jp1 * g.nx + i], d = f[jm1 * g.nx + i];
      double lo = dmin(dmin(dmin(dmin(f0, a), b), cc), d);
      const double hi = dmax(dmax(dmax(dmax(f0, a), b), cc), d);
      if (rho_or_p) lo = dmax(0.1e-8, lo);
      if (xl < lo || xl > hi) xl = f0;
      if (xr < lo || xr > hi) xr = f0;
      if (yl < lo || yl > hi) yl = f0;
      if (yr < lo || yr > hi) yr = f0;
    }
    if (rho_or_p) {
      xl = dmax(xl, 1.0e-8); xr = dmax(xr, 1.0e-8);
      yl = dmax(yl, 1.0e-8); yr = dmax(yr, 1.0e-8);
    }
    XL[c] = xl; XR[c] = xr; YL[c] = yl; YR[c] = yr;
  }
}

// src/mhd_derivatives.f90:232-293; faces[s*6 + q]: slot s (XL, XR, YL, YR), field q
// (P, Bx, By, rho, vx, vy as in the reference's argument order); cell[6] likewise.
struct FacePtrs { double* f[24]; const double* cell[6]; };
__global__ void k_thermal(OpGeom g, FacePtrs p) {
  GRID_LOOP(g.nx * g.ny) {
    for (int s = 0; s < 4; ++s) {
      double* const* f = p.f + 6 * s;
      const double pth = f[0][c] - 0.5 * (f[1][c] * f[1][c] + f[2][c] * f[2][c]);
      if (pth < 1.0e-12)
        for (int q = 0; q < 6; ++q) f[q][c] = p.cell[q][c];
    }
  }
}

// src/mhd_flux.f90:139-191; in[12] = rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R
struct FluxPtrs { const double* in[12]; double* out[5]; };
template <int SOLVER>
__global__ void k_fluxes(OpGeom g, FluxPtrs p) {
  GRID_LOOP(g.nx * g.ny) {
    Flux5<double> F = riemann<double, SOLVER>(g.gamma, p.in[0][c], p.in[1][c], p.in[2][c], p.in[3][c],
                                              p.in[4][c], p.in[5][c], p.in[6][c], p.in[7][c], p.in[8][c],
                                              p.in[9][c], p.in[10][c], p.in[11][c]);
    p.out[0][c] = F.mass; p.out[1][c] = F.momn; p.out[2][c] = F.momt;
    p.out[3][c] = F.energy; p.out[4][c] = F.bt;
  }
}

// src/mhd_flux.f90:20-76 (x pass, then y pass)
__global__ void k_update_x(OpGeom g, double* F, const double* fX, double w) {
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    if (i > 0) F[c] = (F[c] - w * fX[c]) + w * fX[c - 1];
    else F[c] = g.xlo ? (F[c] - w * fX[c]) + w * fX[j * g.nx + g.nx - 1] : F[c] - w * fX[c];
  }
}
__global__ void k_update_y(OpGeom g, double* F, const double* fY, double w) {
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    if (j > 0) F[c] = (F[c] - w * fY[c]) + w * fY[c - g.nx];
    else F[c] = g.ylo ? (F[c] - w * fY[c]) + w * fY[(g.ny - 1) * g.nx + i] : F[c] - w * fY[c];
  }
}

// src/mhd_flux.f90:79-136 step 1: -Ez at the corners
__global__ void k_neg_ez(OpGeom g, const double* fByX, const double* fBxY, double* negEz) {
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    const double up = (j < g.ny - 1) ? fByX[c + g.nx] : (g.yhi ? fByX[i] : fByX[c]);
    const double right = (i < g.nx - 1) ? fBxY[c + 1] : (g.xhi ? fBxY[j * g.nx] : fBxY[c]);
    const double e = 0.25 * (((-fByX[c] - up) + fBxY[c]) + right);
    negEz[c] = -e;
  }
}

// src/mhd_field_ops.f90:15-57 as an update: b += scale * curl(Az) (scale 1 with b = 0 gives the curl)
__global__ void k_curl_add(OpGeom g, const double* Az, double* bx, double* by, double scale, int add) {
  const double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    double dbx, dby;
    if (j > 0) dbx = (Az[c] - Az[c - g.nx]) * inv_dy;
    else if (g.ylo) dbx = (Az[c] - Az[(g.ny - 1) * g.nx + i]) * inv_dy;
    else dbx = (Az[c + g.nx] - Az[c]) * inv_dy;                       // copy of row 2
    if (i > 0) dby = -((Az[c] - Az[c - 1]) * inv_dx);
    else if (g.xlo) dby = -((Az[c] - Az[j * g.nx + g.nx - 1]) * inv_dx);
    else dby = -((Az[c + 1] - Az[c]) * inv_dx);                       // copy of column 2
    if (add) { bx[c] = bx[c] + scale * dbx; by[c] = by[c] + scale * dby; }
    else { bx[c] = dbx; by[c] = dby; }
  }
}

// src/mhd_field_ops.f90:60-117
__global__ void k_divb(OpGeom g, const double* bx, const double* by, double* divB) {
  const double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  const bool square = g.dx == g.dy;
  GRID_LOOP(g.nx * g.ny) {
    const int i = c % g.nx, j = c / g.nx;
    const bool hx = (i > 0) || g.xlo, hy = (j > 0) || g.ylo;
    const double bxm = hx ? bx[(i > 0) ? c - 1 : c + g.nx - 1] : 0.0;
    const double bym = hy ? by[(j > 0) ? c - g.nx : c + (g.ny - 1) * g.nx] : 0.0;
    double r;
    if (square) {
      if (hx && hy) r = (((bx[c] - bxm) + by[c]) - bym) * inv_dx;
      else if (hx) r = (bx[c] - bxm) * inv_dx;
      else if (hy) r = (by[c] - bym) * inv_dx;
      else r = 0.0;
    } else {
      if (hx && hy) r = (bx[c] - bxm) * inv_dx + (by[c] - bym) * inv_dy;
      else if (hx) r = (bx[c] - bxm) * inv_dx;
      else if (hy) r = (by[c] - bym) * inv_dy;
      else r = 0.0;
    }
    divB[c] = r;
  }
}

}  // namespace

#define OP_BEGIN(cfg)                  \
  OpGeom g;                            \
  int rc_ = make_geom((cfg), &g);      \
  if (rc_) return rc_;                 \
  cudaStream_t s = (cudaStream_t)stream; \
  const long long n = (long long)g.nx * g.ny; \
  (void)n;

extern "C" {

int chimera_op_average_face_to_cell_B(const chimera_cfg* cfg, const double* b_x, const double* b_y, double* Bx,
                                      double* By, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({b_x, b_y, Bx, By})) return CHIMERA_ERR_BAD_ARG;
  k_avg_B<<<nblocks(n), NB, 0, s>>>(g, b_x, b_y, Bx, By);
  return finish(s);
}

int chimera_op_get_primitive(const chimera_cfg* cfg, const double* Mass, const double* Momx, const double* Momy,
                             const double* Energy, const double* Bx, const double* By, double* rho, double* vx,
                             double* vy, double* P, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({Mass, Momx, Momy, Energy, Bx, By, rho, vx, vy, P})) return CHIMERA_ERR_BAD_ARG;
  k_get_primitive<<<nblocks(n), NB, 0, s>>>(g, Mass, Momx, Momy, Energy, Bx, By, rho, vx, vy, P);
  return finish(s);
}

int chimera_op_get_conserved(const chimera_cfg* cfg, const double* rho, const double* vx, const double* vy,
                             const double* P, const double* Bx, const double* By, double* Mass, double* Momx,
                             double* Momy, double* Energy, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({rho, vx, vy, P, Bx, By, Mass, Momx, Momy, Energy})) return CHIMERA_ERR_BAD_ARG;
  k_get_conserved<<<nblocks(n), NB, 0, s>>>(g, rho, vx, vy, P, Bx, By, Mass, Momx, Momy, Energy);
  return finish(s);
}

int chimera_op_apply_conserved_floors(const chimera_cfg* cfg, double* Mass, double* Momx, double* Momy,
                                      double* Energy, const double* Bx, const double* By, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({Mass, Momx, Momy, Energy, Bx, By})) return CHIMERA_ERR_BAD_ARG;
  k_floors<<<nblocks(n), NB, 0, s>>>(g, Mass, Momx, Momy, Energy, Bx, By);
  return finish(s);
}

int chimera_op_fill_ghost_cells(const chimera_cfg* cfg, const double* f, double* f_pad, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({f, f_pad})) return CHIMERA_ERR_BAD_ARG;
  k_fill_ghost<<<nblocks((long long)(g.nx + 2) * (g.ny + 2)), NB, 0, s>>>(g, f, f_pad);
  return finish(s);
}

int chimera_op_compute_gradients(const chimera_cfg* cfg, const double* f_pad, double* f_dx, double* f_dy,
                                 void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({f_pad, f_dx, f_dy})) return CHIMERA_ERR_BAD_ARG;
  k_slopes<<<nblocks(n), NB, 0, s>>>(g, f_pad, f_dx, f_dy, 0);
  return finish(s);
}

int chimera_op_apply_slope_limiter(const chimera_cfg* cfg, const double* f_pad, double* f_dx, double* f_dy,
                                   void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({f_pad, f_dx, f_dy})) return CHIMERA_ERR_BAD_ARG;
  k_slopes<<<nblocks(n), NB, 0, s>>>(g, f_pad, f_dx, f_dy, 1);
  return finish(s);
}

int chimera_op_reconstruction(const chimera_cfg* cfg, const double* f, const double* f_dx, const double* f_dy,
                              double* f_XL, double* f_XR, double* f_YL, double* f_YR, int rho_or_p,
                              void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({f, f_dx, f_dy, f_XL, f_XR, f_YL, f_YR})) return CHIMERA_ERR_BAD_ARG;
  k_reconstruction<<<nblocks(n), NB, 0, s>>>(g, f, f_dx, f_dy, f_XL, f_XR, f_YL, f_YR, rho_or_p ? 1 : 0,
                                             cfg->mood ? 1 : 0);
  return finish(s);
}

int chimera_op_thermal_pressure_check(const chimera_cfg* cfg, double* const* faces24, const double* const* cell6,
                                      void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({faces24, cell6})) return CHIMERA_ERR_BAD_ARG;
  FacePtrs p;
  for (int k = 0; k < 24; ++k) { if (!double_ok(faces24[k])) return CHIMERA_ERR_BAD_ARG; p.f[k] = faces24[k]; }
  for (int k = 0; k < 6; ++k) { if (!double_ok(cell6[k])) return CHIMERA_ERR_BAD_ARG; p.cell[k] = cell6[k]; }
  k_thermal<<<nblocks(n), NB, 0, s>>>(g, p);
  return finish(s);
}

int chimera_op_compute_fluxes(const chimera_cfg* cfg, const double* const* in12, double* const* out5,
                              void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({in12, out5})) return CHIMERA_ERR_BAD_ARG;
  FluxPtrs p;
  for (int k = 0; k < 12; ++k) { if (!double_ok(in12[k])) return CHIMERA_ERR_BAD_ARG; p.in[k] = in12[k]; }
  for (int k = 0; k < 5; ++k) { if (!double_ok(out5[k])) return CHIMERA_ERR_BAD_ARG; p.out[k] = out5[k]; }
  if (g.riemann == CHIMERA_RIEMANN_RUSANOV) k_fluxes<RIEMANN_RUSANOV><<<nblocks(n), NB, 0, s>>>(g, p);
  else if (g.riemann == CHIMERA_RIEMANN_HLLE) k_fluxes<RIEMANN_HLLE><<<nblocks(n), NB, 0, s>>>(g, p);
  else k_fluxes<RIEMANN_HLLD><<<nblocks(n), NB, 0, s>>>(g, p);
  return finish(s);
}

int chimera_op_update_conserved(const chimera_cfg* cfg, double* F, const double* flux_X, const double* flux_Y,
                                double dt, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({F, flux_X, flux_Y})) return CHIMERA_ERR_BAD_ARG;
  k_update_x<<<nblocks(n), NB, 0, s>>>(g, F, flux_X, dt * g.dy);
  k_update_y<<<nblocks(n), NB, 0, s>>>(g, F, flux_Y, dt * g.dx);
  return finish(s);
}

// scratch: one caller-provided (nx, ny) array for -Ez
int chimera_op_constrained_transport(const chimera_cfg* cfg, double* b_x, double* b_y, const double* flux_By_X,
                                     const double* flux_Bx_Y, double dt, double* scratch, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({b_x, b_y, flux_By_X, flux_Bx_Y, scratch})) return CHIMERA_ERR_BAD_ARG;
  k_neg_ez<<<nblocks(n), NB, 0, s>>>(g, flux_By_X, flux_Bx_Y, scratch);
  k_curl_add<<<nblocks(n), NB, 0, s>>>(g, scratch, b_x, b_y, dt, 1);
  return finish(s);
}

int chimera_op_compute_curl_2d(const chimera_cfg* cfg, const double* Az, double* b_x, double* b_y, void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({Az, b_x, b_y})) return CHIMERA_ERR_BAD_ARG;
  k_curl_add<<<nblocks(n), NB, 0, s>>>(g, Az, b_x, b_y, 1.0, 0);
  return finish(s);
}

int chimera_op_compute_divB(const chimera_cfg* cfg, const double* b_x, const double* b_y, double* divB,
                            void* stream) {
  OP_BEGIN(cfg);
  if (!doubles_ok({b_x, b_y, divB})) return CHIMERA_ERR_BAD_ARG;
  k_divb<<<nblocks(n), NB, 0, s>>>(g, b_x, b_y, divB);
  return finish(s);
}

}  // extern "C"
