// noalloc.cu -- one RK3 step that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host code whose device memory is
// entirely owned by its own allocator or arena, a time loop that must not pay
// cudaMalloc's implicit device synchronisation (it stalls work queued on other
// streams), or a program that forbids allocation after initialisation.  For
// them chimera_rk3_step_noalloc advances a caller-owned FP64 state by one
// SSP-RK3 step using only the scratch below: the two RK stage buffers, the
// per-tile reduction partials and the time-loop descriptors live in one
// file-scope __device__ array of fixed size, which every GPU that loads this
// library holds until the process exits.
//
// The kernels are the same stage and CFL kernel templates as the handle-based
// path, instantiated here in the 16 x 16 tile shape (48 KB of shared memory, no
// opt-in attribute needed), so the result is bit for bit the handle path's.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "../../include/chimera_gpu.h"
#include "abi_check.h"
#include "stage_kernel.cuh"

using namespace chimera;

namespace {

constexpr int NA_TX = 16, NA_TY = 16, NA_NT = 128, NA_MINB = 4;
constexpr size_t NA_MAX_CELLS = CHIMERA_NOALLOC_MAX_CELLS;
// ceil(nx/16)*ceil(ny/16) <= (nx/4)*(ny/4) for nx, ny >= 4
constexpr size_t NA_MAX_TILES = NA_MAX_CELLS / 16;
constexpr size_t NA_FIELD_BYTES = NA_MAX_CELLS * sizeof(double);
constexpr size_t NA_OFF_STAGE = 0;                                         // 12 fields: U1 / U^{n+1}, U2
constexpr size_t NA_OFF_PART = NA_OFF_STAGE + 12 * NA_FIELD_BYTES;          // [tiles][NPART]
constexpr size_t NA_OFF_MEMBER = NA_OFF_PART + NA_MAX_TILES * NPART * sizeof(double);
constexpr size_t NA_OFF_CONTROL = NA_OFF_MEMBER + ((sizeof(Member) + 255) / 256) * 256;
constexpr size_t NA_BYTES = NA_OFF_CONTROL + ((sizeof(Control) + 255) / 256) * 256;

// The scratch.  In host code this name is only a host-side stand-in for the
// symbol, not a device address: the address passed to kernels comes from
// cudaGetSymbolAddress, taken once per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[NA_MAX_DEVICES] = {nullptr};
// One call at a time per device within this process: a call holds its
// device's lock from the first launch to the final stream synchronisation, so
// host threads cannot interleave their use of the one scratch array.
std::mutex g_call_mutex[NA_MAX_DEVICES];

// Per-call set-up of the descriptors inside the scratch.  Control must start
// at zero (tiles_done counts finished tiles); everything else in the scratch is
// fully overwritten by the step before it is read.
__global__ void k_noalloc_init(Member* m, Control* c, Member desc, double t, int output_count) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *m = desc;
    memset(c, 0, sizeof(Control));
    c->t = t;
    c->output_count = output_count;
    c->active = 1;
    c->parity = 0;
  }
}

int scratch_for_current_device(unsigned char** out, int* device) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
    cudaGetLastError();
    return CHIMERA_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // with this device current
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return CHIMERA_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  *device = dev;
  return CHIMERA_OK;
}

}  // namespace

extern "C" int chimera_rk3_step_noalloc(const chimera_cfg* cfg, double* Mass, double* Momx,
                                        double* Momy, double* Energy, double* b_x, double* b_y,
                                        double* t, int* output_count, double* dt_next, void* stream) {
  if (!cfg || !doubles_ok({Mass, Momx, Momy, Energy, b_x, b_y}) || !t || !output_count)
    return CHIMERA_ERR_BAD_ARG;
  if (cfg->nx < 4 || cfg->ny < 4 || !(cfg->dx > 0.0) || !(cfg->dy > 0.0) || !(cfg->gamma > 1.0) ||
      !(cfg->courant > 0.0) || !(cfg->t_out > 0.0) || !(cfg->t_end > 0.0) || *output_count < 1)
    return CHIMERA_ERR_BAD_ARG;
  if (cfg->precision != CHIMERA_FP64) return CHIMERA_ERR_UNSUPPORTED;
  for (int b : {cfg->bc_xlo, cfg->bc_xhi, cfg->bc_ylo, cfg->bc_yhi})
    if (b < CHIMERA_BC_PERIODIC || b > CHIMERA_BC_INFLOW) return CHIMERA_ERR_BAD_ARG;
  if ((cfg->bc_xlo == CHIMERA_BC_PERIODIC) != (cfg->bc_xhi == CHIMERA_BC_PERIODIC) ||
      (cfg->bc_ylo == CHIMERA_BC_PERIODIC) != (cfg->bc_yhi == CHIMERA_BC_PERIODIC))
    return CHIMERA_ERR_UNSUPPORTED;
  if (cfg->riemann < 1 || cfg->riemann > 3 || cfg->limiter < 1 || cfg->limiter > 2) return CHIMERA_ERR_BAD_ARG;
  const size_t cells = size_t(cfg->nx) * size_t(cfg->ny);
  if (cells > NA_MAX_CELLS) return CHIMERA_ERR_TOO_LARGE;
  // The run is over (src/main.f90:65, do while (t < tEnd)): no step is taken
  // and nothing is launched; the state, t and output_count stay as they are.
  if (!(*t < cfg->t_end)) return CHIMERA_OK;

  unsigned char* base = nullptr;
  int dev = -1;
  int rc = scratch_for_current_device(&base, &dev);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (s) {   // the scratch is the current device's: the stream must be on it too
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) {
      cudaGetLastError();
      return CHIMERA_ERR_BAD_ARG;
    }
    if (sdev != dev) return CHIMERA_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> call_lock(g_call_mutex[dev]);
  // Every return after the first launch drains the stream first, while the
  // lock is held: no kernel of this call may still use the scratch (or the
  // caller's arrays) once another call can take it.
  auto fail = [s]() {
    cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaGetLastError();
    return CHIMERA_ERR_CUDA;
  };

  Member g;
  memset(&g, 0, sizeof(g));
  g.nx = cfg->nx; g.ny = cfg->ny;
  g.tiles_x = (cfg->nx + NA_TX - 1) / NA_TX;
  g.tiles_y = (cfg->ny + NA_TY - 1) / NA_TY;
  g.tile_begin = 0;
  g.periodic_x = cfg->bc_xlo == CHIMERA_BC_PERIODIC;
  g.periodic_y = cfg->bc_ylo == CHIMERA_BC_PERIODIC;
  g.periodic_xhi = g.periodic_x;   // (pairs alike: checked above)
  g.periodic_yhi = g.periodic_y;
  g.square = (cfg->dx == cfg->dy) ? 1 : 0;
  g.dx = cfg->dx; g.dy = cfg->dy;
  g.inv_dx = 1.0 / cfg->dx; g.inv_dy = 1.0 / cfg->dy;
  g.inv_2dx = 1.0 / (2.0 * cfg->dx); g.inv_2dy = 1.0 / (2.0 * cfg->dy);
  g.hx = 0.5 * cfg->dx; g.hy = 0.5 * cfg->dy;
  g.gamma = cfg->gamma;
  g.vol = cfg->dx * cfg->dy;
  g.len = (cfg->dx < cfg->dy) ? cfg->dx : cfg->dy;
  g.inv_vol = 1.0 / g.vol;
  g.rcp_vol = shared_reciprocal(g.vol);
  g.rcp_gm1 = shared_reciprocal(cfg->gamma - 1.0);
  g.courant = cfg->courant;
  g.t_out = cfg->t_out;
  g.t_end = cfg->t_end;
  double* user[6] = {Mass, Momx, Momy, Energy, b_x, b_y};
  for (int q = 0; q < 6; ++q) {
    g.buf[0][q] = user[q];
    g.buf[1][q] = base + NA_OFF_STAGE + size_t(q) * NA_FIELD_BYTES;
    g.buf[2][q] = base + NA_OFF_STAGE + size_t(6 + q) * NA_FIELD_BYTES;
  }
  Member* d_member = reinterpret_cast<Member*>(base + NA_OFF_MEMBER);
  Control* d_ctl = reinterpret_cast<Control*>(base + NA_OFF_CONTROL);

  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.members = d_member;
  a.ctl = d_ctl;
  a.partials = reinterpret_cast<double*>(base + NA_OFF_PART);
  a.tile_member = nullptr;
  a.n_members = 1;
  a.total_tiles = g.tiles_x * g.tiles_y;
  a.limiter = cfg->limiter;
  a.slope_limiting = cfg->use_slope_limiting ? 1 : 0;
  a.mood = cfg->mood ? 1 : 0;
  a.counters = 0;
  a.dry = 0;

  if (size_t(a.total_tiles) > NA_MAX_TILES) return CHIMERA_ERR_TOO_LARGE;
  k_noalloc_init<<<1, 32, 0, s>>>(d_member, d_ctl, g, *t, *output_count);
  const int grid = a.total_tiles;
  const size_t smem = TileGeom<NA_TX, NA_TY>::smem_bytes<double>();
  cfl_kernel<double, NA_TX, NA_TY, NA_NT, UNIT_NOALLOC><<<grid, NA_NT, 0, s>>>(a);
  switch (cfg->riemann) {
    case CHIMERA_RIEMANN_RUSANOV:
      stage_kernel<double, 1, 1, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 1, 2, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 1, 3, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      break;
    case CHIMERA_RIEMANN_HLLE:
      stage_kernel<double, 2, 1, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 2, 2, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 2, 3, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      break;
    default:
      stage_kernel<double, 3, 1, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 3, 2, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      stage_kernel<double, 3, 3, NA_TX, NA_TY, NA_NT, NA_MINB, false, false, UNIT_NOALLOC><<<grid, NA_NT, smem, s>>>(a);
      break;
  }
  if (cudaGetLastError() != cudaSuccess) return fail();
  // After stage 3 the new state sits in stage buffer 1; copy it back into the
  // caller's arrays (dense (nx, ny), x fastest).  The step is always taken
  // here (t < t_end was checked above, so the CFL kernel leaves it active).
  for (int q = 0; q < 6; ++q) {
    if (cudaMemcpyAsync(user[q], g.buf[1][q], cells * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return fail();
  }
  Control c;
  if (cudaMemcpyAsync(&c, d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return fail();
  if (dt_next) *dt_next = c.dt;
  *t = c.t;
  *output_count = c.output_count;
  return c.status ? CHIMERA_ERR_NONFINITE : CHIMERA_OK;
}
