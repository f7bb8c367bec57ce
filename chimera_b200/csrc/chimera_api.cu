// chimera_api.cu -- host runtime behind include/chimera_gpu.h.
//
// A handle is a batch of grid members (a single grid is a batch of one).  It
// owns, per member, three sets of six state buffers in HBM (the state and two
// RK stage scratch sets), the device-resident time-loop state (Control), the
// per-tile reduction partials and the (member, tile) work list; the stage
// kernels are launched persistently over that work list, one launch per RK
// stage, optionally replayed from a captured CUDA graph.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/chimera_gpu.h"
#include "chimera_types.h"
#include "kernel_table.h"

using namespace chimera;

constexpr size_t TMAP_BYTES_HOST = sizeof(CUtensorMap);
static_assert(sizeof(CUtensorMap) == 128, "tensor maps are 128 bytes");

namespace {

// ---- FP32-bulk conversion kernels (host <-> storage precision) ---------------
__global__ void k_f64_to_f32(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
    dst[k] = float(src[k]);
}
__global__ void k_f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, size_t n) {
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
    dst[k] = double(src[k]);
}

bool valid_bc(int b) { return b >= CHIMERA_BC_PERIODIC && b <= CHIMERA_BC_INFLOW; }

// NVTX range over the host-side span of an API call or a kernel launch: named
// spans in a profiler's timeline (header-only NVTX; without a tool attached
// each push / pop is a no-op).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
const char* const kLaunchName[4] = {"chimera cfl", "chimera stage 1", "chimera stage 2", "chimera stage 3"};

// cuTensorMapEncodeTiled from the driver, through the runtime (the library
// links only cudart); null if the driver does not provide it.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    cudaGetLastError();
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of one (ny, nx) field of FP32 (elem 4) or FP64 (elem 8) values
// with a bw x bh box; false if the field's shape does not allow one (row pitch
// not a multiple of 16 bytes, or smaller than the box).
bool encode_field_map(void* map, void* base, int nx, int ny, int bw, int bh, int elem) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || (size_t(nx) * elem) % 16 != 0 || (size_t(bw) * elem) % 16 != 0 || nx < bw || ny < bh ||
      (reinterpret_cast<uintptr_t>(base) & 15) != 0)
    return false;
  const cuuint64_t dims[2] = {cuuint64_t(nx), cuuint64_t(ny)};
  const cuuint64_t strides[1] = {cuuint64_t(nx) * cuuint64_t(elem)};
  const cuuint32_t box[2] = {cuuint32_t(bw), cuuint32_t(bh)};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = (elem == 8) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(static_cast<CUtensorMap*>(map), dt, 2, base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

struct chimera_handle {
  int n = 0;
  std::vector<chimera_cfg> cfg;
  std::vector<Member> hm;            // host copies of the member descriptors
  int riemann = 1, limiter = 2, slope = 1, mood = 1, precision = CHIMERA_FP64;
  int counters = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  int num_sms = 148;
  KernelSet ks{};                    // the active variant's kernels
  std::vector<KernelSet> variants;
  int cur_variant = 0;
  int max_tiles = 0;                 // over all variants (partials / work-list capacity)
  int dry = 0;
  int grid_stage[3] = {0, 0, 0};
  int grid_cfl = 0;
  int total_tiles = 0;
  Member* d_members = nullptr;
  Control* d_ctl = nullptr;
  double* d_part = nullptr;
  int* d_tile_member = nullptr;
  void* pool = nullptr;              // all state buffers
  char* d_tmaps = nullptr;           // [TMA variant slot][member][buffer 3][field 6] tensor maps
  std::vector<int> tmap_slot;        // per variant: its slot in d_tmaps, -1 without TMA
  std::vector<unsigned char> tmap_ok;   // [slot][member]: the member's maps exist
  // chimera_step_host: U^{n+1} goes back in chunks of tile rows on
  // copy_stream while the later chunks compute; stages 2 and 3 run on
  // band_stream[0] / [1] so that the chunks' partial waves of CTAs overlap.
  // s1_done / s2_done / band_done: chunk k of stage 1 / 2 / 3 written.
  static constexpr int kChunks = 10;
  cudaStream_t copy_stream = nullptr;
  cudaStream_t band_stream[2] = {};
  cudaEvent_t s1_done[kChunks] = {};
  cudaEvent_t s2_done[kChunks] = {};
  cudaEvent_t band_done[kChunks] = {};
  cudaEvent_t band_join = nullptr;
  double* d_stage64 = nullptr;       // FP64 staging for FP32-bulk set/get
  size_t max_cells = 0;
  std::vector<bool> dt_valid;        // per member: Control::dt matches the state
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int graph_steps_request = 0;
  // CUDA-event timing of each launch on the handle's stream (eager path only)
  int profiling = 0;
  struct Timed { int kind; cudaEvent_t a, b; };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> spare;
  double prof_ms[4] = {0, 0, 0, 0};   // cfl, stage 1, stage 2, stage 3
  long long prof_n[4] = {0, 0, 0, 0};
};

static int cuda_fail(cudaError_t e) {
  (void)e;
  cudaGetLastError();  // clear sticky-free errors
  return CHIMERA_ERR_CUDA;
}
#define CK(call)                                   \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return cuda_fail(_e);   \
  } while (0)

static bool mixed_pair(const chimera_cfg& c) {
  return (c.bc_xlo == CHIMERA_BC_PERIODIC) != (c.bc_xhi == CHIMERA_BC_PERIODIC) ||
         (c.bc_ylo == CHIMERA_BC_PERIODIC) != (c.bc_yhi == CHIMERA_BC_PERIODIC);
}

static int validate_cfg(const chimera_cfg* c) {
  if (!c) return CHIMERA_ERR_BAD_ARG;
  if (c->nx < 4 || c->ny < 4) return CHIMERA_ERR_BAD_ARG;                 // N >= 4 (src/mhd_init.f90:208)
  if ((long long)c->nx * c->ny > (1LL << 31)) return CHIMERA_ERR_TOO_LARGE;
  if (!(c->dx > 0.0) || !(c->dy > 0.0) || !(c->gamma > 1.0)) return CHIMERA_ERR_BAD_ARG;
  if (!(c->courant > 0.0) || !(c->t_out > 0.0)) return CHIMERA_ERR_BAD_ARG;
  if (!valid_bc(c->bc_xlo) || !valid_bc(c->bc_xhi) || !valid_bc(c->bc_ylo) || !valid_bc(c->bc_yhi))
    return CHIMERA_ERR_BAD_ARG;
  if (c->riemann < 1 || c->riemann > 3) return CHIMERA_ERR_BAD_ARG;
  if (c->limiter < 1 || c->limiter > 2) return CHIMERA_ERR_BAD_ARG;
  if (c->precision != CHIMERA_FP64 && c->precision != CHIMERA_FP32_BULK && c->precision != CHIMERA_FP32_MIXED)
    return CHIMERA_ERR_BAD_ARG;
  return CHIMERA_OK;
}

static cudaEvent_t take_event(chimera_handle* h) {
  if (!h->spare.empty()) {
    cudaEvent_t e = h->spare.back();
    h->spare.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  return e;
}

static void harvest_profile(chimera_handle* h) {
  for (auto& t : h->timed) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      h->prof_ms[t.kind] += ms;
      h->prof_n[t.kind] += 1;
    }
    cudaGetLastError();
    h->spare.push_back(t.a);
    h->spare.push_back(t.b);
  }
  h->timed.clear();
}

static int launch_raw(chimera_handle* h, const KernelEntry& k, int grid, int w_begin, int w_end,
                      cudaStream_t stream = nullptr);

// kind: 0 = CFL kernel, 1..3 = stage kernels
static int launch(chimera_handle* h, const KernelEntry& k, int grid, int kind) {
  NvtxRange range(kLaunchName[kind]);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(h->stream, &cs);
  if (!h->profiling || cs != cudaStreamCaptureStatusNone) return launch_raw(h, k, grid, 0, -1);
  if (h->timed.size() > 4096) harvest_profile(h);
  cudaEvent_t a = take_event(h), b = take_event(h);
  if (!a || !b) return launch_raw(h, k, grid, 0, -1);
  cudaEventRecord(a, h->stream);
  int rc = launch_raw(h, k, grid, 0, -1);
  cudaEventRecord(b, h->stream);
  h->timed.push_back({kind, a, b});
  return rc;
}

// stream: the handle's stream unless given
static int launch_raw(chimera_handle* h, const KernelEntry& k, int grid, int w_begin, int w_end,
                      cudaStream_t stream) {
  StageArgs a;
  a.members = h->d_members;
  a.ctl = h->d_ctl;
  a.partials = h->d_part;
  a.tile_member = h->d_tile_member;
  a.n_members = h->n;
  a.total_tiles = (w_end < 0) ? h->total_tiles : w_end;
  a.work_begin = w_begin;
  a.limiter = h->limiter;
  a.slope_limiting = h->slope;
  a.mood = h->mood;
  a.counters = h->counters;
  a.dry = h->dry;
  void* args[] = {&a};
  CK(cudaLaunchKernel(k.fn, dim3(grid), dim3(k.nt), args, k.smem, stream ? stream : h->stream));
  return CHIMERA_OK;
}

static int grid_for(chimera_handle* h, const KernelEntry& k) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.nt, k.smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  cudaGetLastError();
  return std::max(1, std::min(h->total_tiles, per_sm * h->num_sms));
}

static int ensure_dt(chimera_handle* h) {
  bool all = true;
  for (int m = 0; m < h->n; ++m) all = all && h->dt_valid[m];
  if (all) return CHIMERA_OK;
  int rc = launch(h, h->ks.cfl, h->grid_cfl, 0);
  if (rc) return rc;
  for (int m = 0; m < h->n; ++m) h->dt_valid[m] = true;
  return CHIMERA_OK;
}

// Ghost rows of a y-slab (one grid split across ranks): copy `rows` whole rows
// of every field of the current state (the buffer the device-side parity names)
// to or from packed [field 6][rows][nx] buffers.  Pack: lo <- rows [rows, 2 rows),
// hi <- rows [ny - 2 rows, ny - rows) (the interior rows a neighbour needs);
// unpack: rows [0, rows) <- lo, rows [ny - rows, ny) <- hi.  A null side is skipped.
template <typename T>
__global__ void halo_rows_kernel(const Member* members, const Control* ctl, int rows, T* lo, T* hi,
                                 int unpack) {
  const Member& g = members[0];
  const int side = blockIdx.z;
  T* pk = side ? hi : lo;
  if (!pk) return;
  const int q = blockIdx.y;
  const int nx = g.nx, ny = g.ny;
  const int r0 = unpack ? (side ? ny - rows : 0) : (side ? ny - 2 * rows : rows);
  T* st = reinterpret_cast<T*>(g.buf[ctl->parity][q]) + size_t(r0) * nx;
  const size_t n = size_t(rows) * nx;
  pk += size_t(q) * n;
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
    if (unpack) st[k] = pk[k];
    else pk[k] = st[k];
  }
}

static int halo_rows(chimera_handle* h, int rows, void* lo, void* hi, int unpack) {
  if (!h || rows < 1 || (!lo && !hi)) return CHIMERA_ERR_BAD_ARG;
  if (h->n != 1) return CHIMERA_ERR_UNSUPPORTED;
  const chimera_cfg& c = h->cfg[0];
  if (2 * rows > c.ny) return CHIMERA_ERR_BAD_ARG;
  const int eb = h->ks.elem_bytes;
  if ((uintptr_t(lo) % eb) || (uintptr_t(hi) % eb)) return CHIMERA_ERR_BAD_ARG;
  const size_t n = size_t(rows) * c.nx;
  const dim3 grid(unsigned(std::min<size_t>((n + 255) / 256, 1024)), 6, 2);
  if (eb == 8)
    halo_rows_kernel<unsigned long long><<<grid, 256, 0, h->stream>>>(
        h->d_members, h->d_ctl, rows, static_cast<unsigned long long*>(lo), static_cast<unsigned long long*>(hi),
        unpack);
  else
    halo_rows_kernel<unsigned><<<grid, 256, 0, h->stream>>>(h->d_members, h->d_ctl, rows,
                                                             static_cast<unsigned*>(lo),
                                                             static_cast<unsigned*>(hi), unpack);
  CK(cudaGetLastError());
  // the dt stays valid when only rows that its reduction leaves out changed
  const Member& g = h->hm[0];
  if (unpack && ((lo && rows > g.skip_lo) || (hi && rows > g.skip_hi))) h->dt_valid[0] = false;
  return CHIMERA_OK;
}

static int one_step(chimera_handle* h) {
  for (int s = 0; s < 3; ++s) {
    int rc = launch(h, h->ks.stage[h->riemann - 1][s], h->grid_stage[s], s + 1);
    if (rc) return rc;
  }
  return CHIMERA_OK;
}

static void drop_graph(chimera_handle* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_steps = 0;
}

static int run_steps(chimera_handle* h, int nsteps) {
  int rc = ensure_dt(h);
  if (rc) return rc;
  if (h->graph_steps_request > 0 && nsteps == h->graph_steps_request) {
    if (!h->graph || h->graph_steps != nsteps) {
      drop_graph(h);
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int crc = CHIMERA_OK;
      for (int s = 0; s < nsteps && crc == CHIMERA_OK; ++s) crc = one_step(h);
      cudaError_t e = cudaStreamEndCapture(h->stream, &g);
      if (crc) { if (g) cudaGraphDestroy(g); return crc; }
      if (e != cudaSuccess) return cuda_fail(e);
      e = cudaGraphInstantiate(&h->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { h->graph = nullptr; return cuda_fail(e); }
      h->graph_steps = nsteps;
    }
    CK(cudaGraphLaunch(h->graph, h->stream));
    return CHIMERA_OK;
  }
  for (int s = 0; s < nsteps; ++s) {
    rc = one_step(h);
    if (rc) return rc;
  }
  return CHIMERA_OK;
}

static size_t cells_of(const chimera_cfg& c) { return size_t(c.nx) * size_t(c.ny); }

static int tiles_for(const chimera_handle* h, int tx, int ty) {
  int t = 0;
  for (int m = 0; m < h->n; ++m) t += ((h->cfg[m].nx + tx - 1) / tx) * ((h->cfg[m].ny + ty - 1) / ty);
  return t;
}

// Switch the tile decomposition to variant v: member tiling, work list and
// persistent grid sizes (descriptors are re-uploaded; state is untouched).
static int layout(chimera_handle* h, int v) {
  h->ks = h->variants[v];
  h->cur_variant = v;
  const int tx = h->ks.stage[0][0].tx, ty = h->ks.stage[0][0].ty;
  int tiles = 0;
  for (int m = 0; m < h->n; ++m) {
    Member& g = h->hm[m];
    g.tiles_x = (g.nx + tx - 1) / tx;
    g.tiles_y = (g.ny + ty - 1) / ty;
    g.tile_begin = tiles;
    tiles += g.tiles_x * g.tiles_y;
  }
  h->total_tiles = tiles;
  // TMA variants: the variant's tensor maps (encoded once at creation and never
  // modified) for the members whose shape allows them; the others, and every
  // edge tile, use plain loads
  const int slot = h->tmap_slot.empty() ? -1 : h->tmap_slot[v];
  for (int m = 0; m < h->n; ++m)
    h->hm[m].tmap = (slot >= 0 && h->tmap_ok[size_t(slot) * h->n + m])
                        ? h->d_tmaps + (size_t(slot) * h->n + m) * 18 * TMAP_BYTES_HOST
                        : nullptr;
  std::vector<int> tm(tiles);
  for (int m = 0; m < h->n; ++m)
    for (int k = 0; k < h->hm[m].tiles_x * h->hm[m].tiles_y; ++k) tm[h->hm[m].tile_begin + k] = m;
  CK(cudaMemcpyAsync(h->d_members, h->hm.data(), sizeof(Member) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_tile_member, tm.data(), sizeof(int) * tiles, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int st = 0; st < 3; ++st) h->grid_stage[st] = grid_for(h, h->ks.stage[h->riemann - 1][st]);
  h->grid_cfl = grid_for(h, h->ks.cfl);
  drop_graph(h);
  return CHIMERA_OK;
}

// Autotuner results per problem shape, shared by the handles of a process.
using TuneKey = std::tuple<int, int, int, int, int, long long, int>;
static std::map<TuneKey, int>& tune_cache() {
  static std::map<TuneKey, int> c;
  return c;
}
static std::mutex& tune_mutex() {
  static std::mutex m;
  return m;
}
static TuneKey tune_key(const chimera_handle* h) {
  long long cells = 0;
  for (int m = 0; m < h->n; ++m) cells += (long long)cells_of(h->cfg[m]);
  return TuneKey(h->precision, h->riemann, h->limiter, h->mood, h->slope, cells, h->n);
}

extern "C" {

int chimera_version(void) { return 10000; }

const char* chimera_strerror(int code) {
  switch (code) {
    case CHIMERA_OK: return "ok";
    case CHIMERA_ERR_BAD_ARG: return "invalid argument";
    case CHIMERA_ERR_CUDA: return "CUDA runtime error";
    case CHIMERA_ERR_NONFINITE: return "non-finite state reported by the device";
    case CHIMERA_ERR_TIMEOUT: return "bounded device wait timed out";
    case CHIMERA_ERR_UNSUPPORTED: return "configuration not supported on this path";
    case CHIMERA_ERR_NO_DEVICE: return "no usable CUDA device";
    case CHIMERA_ERR_NOMEM: return "device allocation failed";
    case CHIMERA_ERR_TOO_LARGE: return "size exceeds capacity";
    default: return "unknown error";
  }
}

int chimera_batch_create(int n_members, const chimera_cfg* cfgs, void* stream, chimera_handle** out) {
  if (!out || !cfgs || n_members < 1) return CHIMERA_ERR_BAD_ARG;
  *out = nullptr;
  for (int m = 0; m < n_members; ++m) {
    int rc = validate_cfg(&cfgs[m]);
    if (rc) return rc;
    const chimera_cfg& a = cfgs[0];
    const chimera_cfg& b = cfgs[m];
    if (a.riemann != b.riemann || a.limiter != b.limiter || a.use_slope_limiting != b.use_slope_limiting ||
        a.mood != b.mood || a.precision != b.precision)
      return CHIMERA_ERR_BAD_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { cudaGetLastError(); return CHIMERA_ERR_NO_DEVICE; }
  chimera_handle* h = new (std::nothrow) chimera_handle();
  if (!h) return CHIMERA_ERR_NOMEM;
  h->n = n_members;
  h->cfg.assign(cfgs, cfgs + n_members);
  h->riemann = cfgs[0].riemann;
  h->limiter = cfgs[0].limiter;
  h->slope = cfgs[0].use_slope_limiting ? 1 : 0;
  h->mood = cfgs[0].mood ? 1 : 0;
  h->precision = cfgs[0].precision;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  // a periodic side facing a non-periodic one (a mixed pair; the reference
  // takes each side on its own, src/mhd_bc.f90:45-100) in any member: the one
  // tile of the form compiled for it
  bool mixed = false;
  for (int m = 0; m < n_members; ++m) mixed = mixed || mixed_pair(cfgs[m]);
  const int nv = mixed                                 ? 1
                 : (h->precision == CHIMERA_FP64)       ? fp64_variant_count()
                 : (h->precision == CHIMERA_FP32_BULK) ? fp32_variant_count()
                                                       : fp32m_variant_count();
  h->variants.resize(nv);
  for (int v = 0; v < nv; ++v) {
    if (mixed && h->precision == CHIMERA_FP64) fp64_mixed_pair_kernels(&h->variants[v]);
    else if (mixed && h->precision == CHIMERA_FP32_BULK) fp32_mixed_pair_kernels(&h->variants[v]);
    else if (mixed) fp32m_mixed_pair_kernels(&h->variants[v]);
    else if (h->precision == CHIMERA_FP64) fp64_kernels(v, &h->variants[v]);
    else if (h->precision == CHIMERA_FP32_BULK) fp32_kernels(v, &h->variants[v]);
    else fp32m_kernels(v, &h->variants[v]);
    for (int r = 0; r < 3; ++r)
      for (int st = 0; st < 3; ++st)
        cudaFuncSetAttribute(h->variants[v].stage[r][st].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(h->variants[v].stage[r][st].smem));
  }
  cudaGetLastError();
  h->ks = h->variants[0];
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return CHIMERA_ERR_CUDA;
    }
    h->own_stream = true;
  }
  // members (tiling is set by layout())
  const int eb = h->ks.elem_bytes;
  h->hm.resize(n_members);
  size_t pool_bytes = 0;
  int tiles = 0;
  for (int v = 0; v < nv; ++v)
    tiles = std::max(tiles, tiles_for(h, h->variants[v].stage[0][0].tx, h->variants[v].stage[0][0].ty));
  h->max_tiles = tiles;
  for (int m = 0; m < n_members; ++m) {
    const chimera_cfg& c = cfgs[m];
    Member& g = h->hm[m];
    memset(&g, 0, sizeof(g));
    g.nx = c.nx; g.ny = c.ny;
    g.periodic_x = c.bc_xlo == CHIMERA_BC_PERIODIC;
    g.periodic_y = c.bc_ylo == CHIMERA_BC_PERIODIC;
    g.periodic_xhi = c.bc_xhi == CHIMERA_BC_PERIODIC;
    g.periodic_yhi = c.bc_yhi == CHIMERA_BC_PERIODIC;
    g.square = (c.dx == c.dy) ? 1 : 0;
    g.dx = c.dx; g.dy = c.dy;
    g.inv_dx = 1.0 / c.dx; g.inv_dy = 1.0 / c.dy;
    g.inv_2dx = 1.0 / (2.0 * c.dx); g.inv_2dy = 1.0 / (2.0 * c.dy);
    g.hx = 0.5 * c.dx; g.hy = 0.5 * c.dy;
    g.gamma = c.gamma;
    g.vol = c.dx * c.dy;
    g.len = (c.dx < c.dy) ? c.dx : c.dy;
    g.inv_vol = 1.0 / g.vol;
    g.rcp_vol = shared_reciprocal(g.vol);
    g.rcp_gm1 = shared_reciprocal(c.gamma - 1.0);
    g.courant = c.courant;
    g.t_out = c.t_out;
    g.t_end = c.t_end;
    const size_t n = cells_of(c);
    h->max_cells = std::max(h->max_cells, n);
    pool_bytes += 18 * ((n * eb + 255) / 256) * 256;
  }
  h->dt_valid.assign(n_members, false);
  if (cudaMalloc(&h->pool, pool_bytes) != cudaSuccess) { cudaGetLastError(); chimera_destroy(h); return CHIMERA_ERR_NOMEM; }
  cudaMemsetAsync(h->pool, 0, pool_bytes, h->stream);
  char* p = (char*)h->pool;
  for (int m = 0; m < n_members; ++m) {
    const size_t fb = ((cells_of(cfgs[m]) * eb + 255) / 256) * 256;
    for (int b = 0; b < 3; ++b)
      for (int q = 0; q < 6; ++q) { h->hm[m].buf[b][q] = p; p += fb; }
  }
  std::vector<Control> ctl(n_members);
  for (int m = 0; m < n_members; ++m) {
    memset(&ctl[m], 0, sizeof(Control));
    ctl[m].t = 0.0;
    ctl[m].output_count = 1;
    ctl[m].active = 1;
  }
  if (cudaMalloc(&h->d_members, sizeof(Member) * n_members) != cudaSuccess ||
      cudaMalloc(&h->d_ctl, sizeof(Control) * n_members) != cudaSuccess ||
      cudaMalloc(&h->d_part, sizeof(double) * NPART * size_t(h->max_tiles)) != cudaSuccess ||
      cudaMalloc(&h->d_tile_member, sizeof(int) * size_t(h->max_tiles)) != cudaSuccess) {
    cudaGetLastError();
    chimera_destroy(h);
    return CHIMERA_ERR_NOMEM;
  }
  // tensor maps of every TMA variant, written once here and never modified
  h->tmap_slot.assign(nv, -1);
  int slots = 0;
  for (int v = 0; v < nv; ++v)
    if (h->variants[v].stage[0][0].box_w > 0) h->tmap_slot[v] = slots++;
  if (slots > 0) {
    const size_t per_slot = size_t(n_members) * 18 * TMAP_BYTES_HOST;
    std::vector<unsigned char> maps(per_slot * slots, 0);
    h->tmap_ok.assign(size_t(slots) * n_members, 0);
    for (int v = 0; v < nv; ++v) {
      const int sl = h->tmap_slot[v];
      if (sl < 0) continue;
      const int bw = h->variants[v].stage[0][0].box_w, bh = h->variants[v].stage[0][0].box_h;
      for (int m = 0; m < n_members; ++m) {
        const Member& g = h->hm[m];
        bool ok = true;
        for (int b = 0; b < 3 && ok; ++b)
          for (int q = 0; q < 6 && ok; ++q)
            ok = encode_field_map(&maps[sl * per_slot + (size_t(m) * 18 + b * 6 + q) * TMAP_BYTES_HOST],
                                  g.buf[b][q], g.nx, g.ny, bw, bh, h->variants[v].elem_bytes);
        h->tmap_ok[size_t(sl) * n_members + m] = ok ? 1 : 0;
      }
    }
    if (cudaMalloc(&h->d_tmaps, maps.size()) != cudaSuccess ||
        cudaMemcpyAsync(h->d_tmaps, maps.data(), maps.size(), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      cudaGetLastError();
      chimera_destroy(h);
      return CHIMERA_ERR_NOMEM;
    }
  }
  if (h->precision == CHIMERA_FP32_BULK) {
    if (cudaMalloc(&h->d_stage64, sizeof(double) * h->max_cells) != cudaSuccess) {
      cudaGetLastError();
      chimera_destroy(h);
      return CHIMERA_ERR_NOMEM;
    }
  }
  cudaMemcpyAsync(h->d_ctl, ctl.data(), sizeof(Control) * n_members, cudaMemcpyHostToDevice, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) { cudaGetLastError(); chimera_destroy(h); return CHIMERA_ERR_CUDA; }
  int v0 = 0;
  {
    std::lock_guard<std::mutex> lk(tune_mutex());
    auto it = tune_cache().find(tune_key(h));
    if (it != tune_cache().end()) v0 = it->second;
  }
  if (layout(h, v0) != CHIMERA_OK) { chimera_destroy(h); return CHIMERA_ERR_CUDA; }
  *out = h;
  return CHIMERA_OK;
}

int chimera_create(const chimera_cfg* cfg, void* stream, chimera_handle** out) {
  if (!cfg) return CHIMERA_ERR_BAD_ARG;
  return chimera_batch_create(1, cfg, stream, out);
}

void chimera_destroy(chimera_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  harvest_profile(h);
  for (auto e : h->spare) cudaEventDestroy(e);
  cudaFree(h->pool);
  cudaFree(h->d_members);
  cudaFree(h->d_ctl);
  cudaFree(h->d_part);
  cudaFree(h->d_tile_member);
  cudaFree(h->d_stage64);
  cudaFree(h->d_tmaps);
  for (auto e : h->band_done)
    if (e) cudaEventDestroy(e);
  for (auto e : h->s1_done)
    if (e) cudaEventDestroy(e);
  for (auto e : h->s2_done)
    if (e) cudaEventDestroy(e);
  if (h->band_join) cudaEventDestroy(h->band_join);
  for (auto st : h->band_stream)
    if (st) cudaStreamDestroy(st);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  cudaGetLastError();
  delete h;
}

void* chimera_stream(chimera_handle* h) { return h ? (void*)h->stream : nullptr; }
int chimera_batch_size(chimera_handle* h) { return h ? h->n : CHIMERA_ERR_BAD_ARG; }

static int read_ctl(chimera_handle* h, int m, Control* c) {
  CK(cudaMemcpyAsync(c, h->d_ctl + m, sizeof(Control), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return CHIMERA_OK;
}

// Copy one field between a caller array (ld pitch, host or device) and a
// dense device buffer of the handle's storage precision.
static int copy_field_in(chimera_handle* h, int m, void* dst, const double* src, int ld, int where) {
  const chimera_cfg& c = h->cfg[m];
  const size_t w = size_t(c.nx) * sizeof(double);
  const cudaMemcpyKind kind = (where == CHIMERA_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (h->ks.elem_bytes == 8) {   // FP64 storage
    CK(cudaMemcpy2DAsync(dst, w, src, size_t(ld) * sizeof(double), w, c.ny, kind, h->stream));
  } else {
    CK(cudaMemcpy2DAsync(h->d_stage64, w, src, size_t(ld) * sizeof(double), w, c.ny, kind, h->stream));
    const size_t n = cells_of(c);
    k_f64_to_f32<<<h->num_sms * 4, 256, 0, h->stream>>>(h->d_stage64, (float*)dst, n);
    CK(cudaGetLastError());
  }
  return CHIMERA_OK;
}

static int copy_field_out(chimera_handle* h, int m, double* dst, const void* src, int ld, int where) {
  const chimera_cfg& c = h->cfg[m];
  const size_t w = size_t(c.nx) * sizeof(double);
  const cudaMemcpyKind kind = (where == CHIMERA_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (h->ks.elem_bytes == 8) {   // FP64 storage
    CK(cudaMemcpy2DAsync(dst, size_t(ld) * sizeof(double), src, w, w, c.ny, kind, h->stream));
  } else {
    const size_t n = cells_of(c);
    k_f32_to_f64<<<h->num_sms * 4, 256, 0, h->stream>>>((const float*)src, h->d_stage64, n);
    CK(cudaGetLastError());
    CK(cudaMemcpy2DAsync(dst, size_t(ld) * sizeof(double), h->d_stage64, w, w, c.ny, kind, h->stream));
  }
  return CHIMERA_OK;
}

static int check_io(chimera_handle* h, int m, const void* const* ptrs, int ld, int where) {
  if (!h || m < 0 || m >= h->n) return CHIMERA_ERR_BAD_ARG;
  if (where != CHIMERA_HOST && where != CHIMERA_DEVICE) return CHIMERA_ERR_BAD_ARG;
  if (ld < h->cfg[m].nx) return CHIMERA_ERR_BAD_ARG;
  for (int q = 0; q < 6; ++q)
    if (!ptrs[q]) return CHIMERA_ERR_BAD_ARG;
  return CHIMERA_OK;
}

int chimera_batch_set_state(chimera_handle* h, int m, const double* Mass, const double* Momx,
                            const double* Momy, const double* Energy, const double* b_x,
                            const double* b_y, int ld, int where) {
  const void* ptrs[6] = {Mass, Momx, Momy, Energy, b_x, b_y};
  int rc = check_io(h, m, ptrs, ld, where);
  if (rc) return rc;
  Control c;
  rc = read_ctl(h, m, &c);
  if (rc) return rc;
  for (int q = 0; q < 6 && !rc; ++q)
    rc = copy_field_in(h, m, h->hm[m].buf[c.parity][q], (const double*)ptrs[q], ld, where);
  h->dt_valid[m] = false;
  // Host arrays have been read completely when the call returns: copies from
  // page-locked memory would otherwise still be in flight.
  if (where == CHIMERA_HOST) {
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e);
  }
  return rc;
}

int chimera_set_state(chimera_handle* h, const double* Mass, const double* Momx, const double* Momy,
                      const double* Energy, const double* b_x, const double* b_y, int ld, int where) {
  return chimera_batch_set_state(h, 0, Mass, Momx, Momy, Energy, b_x, b_y, ld, where);
}

static int get_buffer(chimera_handle* h, int m, int which, double* const* ptrs, int ld, int where) {
  const void* p6[6] = {ptrs[0], ptrs[1], ptrs[2], ptrs[3], ptrs[4], ptrs[5]};
  int rc = check_io(h, m, p6, ld, where);
  if (rc) return rc;
  Control c;
  rc = read_ctl(h, m, &c);
  if (rc) return rc;
  const int b = (which == 0) ? c.parity : (which == 1 ? 1 - c.parity : 2);
  for (int q = 0; q < 6 && !rc; ++q) rc = copy_field_out(h, m, ptrs[q], h->hm[m].buf[b][q], ld, where);
  const cudaError_t e = cudaStreamSynchronize(h->stream);   // on the error path too: no copy outlives the call
  if (rc) { cudaGetLastError(); return rc; }
  if (e != cudaSuccess) return cuda_fail(e);
  return c.status ? CHIMERA_ERR_NONFINITE : CHIMERA_OK;
}

int chimera_batch_get_state(chimera_handle* h, int m, double* Mass, double* Momx, double* Momy,
                            double* Energy, double* b_x, double* b_y, int ld, int where) {
  double* p[6] = {Mass, Momx, Momy, Energy, b_x, b_y};
  return get_buffer(h, m, 0, p, ld, where);
}

int chimera_get_state(chimera_handle* h, double* Mass, double* Momx, double* Momy, double* Energy,
                      double* b_x, double* b_y, int ld, int where) {
  return chimera_batch_get_state(h, 0, Mass, Momx, Momy, Energy, b_x, b_y, ld, where);
}

int chimera_get_stage_buffer(chimera_handle* h, int b, double* Mass, double* Momx, double* Momy,
                             double* Energy, double* b_x, double* b_y, int ld, int where) {
  if (b < 0 || b > 2) return CHIMERA_ERR_BAD_ARG;
  double* p[6] = {Mass, Momx, Momy, Energy, b_x, b_y};
  return get_buffer(h, 0, b, p, ld, where);
}

// One RK3 step of a single-grid FP64 handle on host arrays: the state comes
// in from `in`, advances one step and goes out to `out` (which may alias
// `in`).  Stage 3 runs in bands of tile rows and each band's rows go back to
// the host on a second stream as soon as the band is written, so the
// device-to-host copy overlaps the rest of stage 3.  Other handles take the
// set_state / step / get_state sequence.
int chimera_step_host(chimera_handle* h, const double* const* in, double* const* out, int ld) {
  NvtxRange range("chimera_step_host");
  if (!h || !in || !out) return CHIMERA_ERR_BAD_ARG;
  const void* pi[6] = {in[0], in[1], in[2], in[3], in[4], in[5]};
  const void* po[6] = {out[0], out[1], out[2], out[3], out[4], out[5]};
  int rc = check_io(h, 0, pi, ld, CHIMERA_HOST);
  if (!rc) rc = check_io(h, 0, po, ld, CHIMERA_HOST);
  if (rc) return rc;
  if (h->n != 1 || h->precision != CHIMERA_FP64 || h->graph_steps_request > 0) {
    rc = chimera_set_state(h, in[0], in[1], in[2], in[3], in[4], in[5], ld, CHIMERA_HOST);
    if (!rc) rc = chimera_step(h, 1);
    if (!rc) rc = chimera_get_state(h, out[0], out[1], out[2], out[3], out[4], out[5], ld, CHIMERA_HOST);
    return rc;
  }
  Control c;
  rc = read_ctl(h, 0, &c);
  if (rc) return rc;
  const chimera_cfg& cf = h->cfg[0];
  const Member& g = h->hm[0];
  h->dt_valid[0] = false;
  // Everything issued here is asynchronous, on the handle's stream, the two
  // wavefront streams and the copy stream; the exit below drains all four, so
  // that no copy from in[] or into out[] outlives the call, on the error paths
  // too.
  auto issue = [&]() -> int {
    for (int q = 0; q < 6; ++q) {
      const int e = copy_field_in(h, 0, g.buf[c.parity][q], in[q], ld, CHIMERA_HOST);
      if (e) return e;
    }
    if (!c.active) {   // t >= t_end: no step is taken, the state goes back unchanged
      for (int q = 0; q < 6; ++q) {
        const int e = copy_field_out(h, 0, out[q], g.buf[c.parity][q], ld, CHIMERA_HOST);
        if (e) return e;
      }
      return CHIMERA_OK;
    }
    int e = ensure_dt(h);
    if (e) return e;
    if (!h->copy_stream) {
      CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
      for (auto& st : h->band_stream) CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      for (auto* evs : {h->s1_done, h->s2_done, h->band_done})
        for (int k = 0; k < chimera_handle::kChunks; ++k) CK(cudaEventCreateWithFlags(&evs[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h->band_join, cudaEventDisableTiming));
    }
    // Chunks of tile rows (work items are row-major within the grid) that
    // double in size -- 1, 2, 4, ... tile rows, the last one taking a remainder
    // smaller than itself -- so that the first rows go back early and later
    // chunks need few copies.  A tile reads rows
    // [j0 - 3, j0 + TY + 2) of its stage's input: tile row r of a stage needs
    // tile rows r - 1 .. r + 1 of the stage before it.
    const int ty = h->ks.stage[0][0].ty;
    const int rows = g.tiles_y;
    int end[chimera_handle::kChunks], nc = 0;   // chunk k: tile rows [end[k - 1], end[k])
    for (int r = 1;; r = 2 * r + 1) {
      const int prev = nc ? end[nc - 1] : 0;
      const bool last = rows - r < r - prev || nc == chimera_handle::kChunks - 1;
      end[nc++] = last ? rows : r;
      if (last) break;
    }
    const int out_buf = 1 - c.parity;   // stage 3 writes U^{n+1} there; the finish flips the parity
    const size_t w = size_t(cf.nx) * sizeof(double);
    const KernelEntry* ks = h->ks.stage[h->riemann - 1];
    // stage s over tile rows [r0, r1) on stream st (nothing for an empty range)
    auto rows_launch = [&](int s, int r0, int r1, cudaStream_t st) -> int {
      r0 = std::max(r0, 0);
      r1 = std::min(r1, rows);
      if (r1 <= r0) return CHIMERA_OK;
      const int w0 = r0 * g.tiles_x, w1 = r1 * g.tiles_x;
      return launch_raw(h, ks[s], std::max(1, std::min(h->grid_stage[s], w1 - w0)), w0, w1, st);
    };
    // stage 3 over chunk k, then its rows of the six fields back to the host
    auto finish_chunk = [&](int k, cudaStream_t st) -> int {
      const int r0 = k ? end[k - 1] : 0;
      const int e3 = rows_launch(2, r0, end[k], st);
      if (e3) return e3;
      CK(cudaEventRecord(h->band_done[k], st));
      CK(cudaStreamWaitEvent(h->copy_stream, h->band_done[k], 0));
      const int y0 = r0 * ty, y1 = std::min(end[k] * ty, cf.ny);
      for (int q = 0; q < 6; ++q)
        CK(cudaMemcpy2DAsync(out[q] + size_t(y0) * ld, size_t(ld) * sizeof(double),
                             static_cast<const char*>(g.buf[out_buf][q]) + size_t(y0) * w, w, w, y1 - y0,
                             cudaMemcpyDeviceToHost, h->copy_stream));
      return CHIMERA_OK;
    };
    if (!g.periodic_y && !g.periodic_yhi) {
      // a wavefront: stage 1 runs two tile rows ahead of stage 3 on the
      // handle's stream, stage 2 one row ahead on band_stream[0], stage 3 on
      // band_stream[1].  Stage 3 writes U^{n+1} over U1's rows of chunk k only
      // after stage 2 has finished the tile row above the chunk, the last
      // reader of those rows; later stage-2 rows read none of them.
      cudaStream_t s2 = h->band_stream[0], s3 = h->band_stream[1];
      int d1 = 0, d2 = 0;   // stage 1 / 2 issued for tile rows [0, d1) / [0, d2)
      for (int k = 0; k < nc; ++k) {
        const int t1 = std::min(end[k] + 2, rows), t2 = std::min(end[k] + 1, rows);
        if ((e = rows_launch(0, d1, t1, h->stream))) return e;
        d1 = std::max(d1, t1);
        CK(cudaEventRecord(h->s1_done[k], h->stream));
        CK(cudaStreamWaitEvent(s2, h->s1_done[k], 0));
        if ((e = rows_launch(1, d2, t2, s2))) return e;
        d2 = std::max(d2, t2);
        CK(cudaEventRecord(h->s2_done[k], s2));
        CK(cudaStreamWaitEvent(s3, h->s2_done[k], 0));
        if ((e = finish_chunk(k, s3))) return e;
      }
      // later work on the handle's stream comes after the wavefront
      CK(cudaEventRecord(h->band_join, s3));
      CK(cudaStreamWaitEvent(h->stream, h->band_join, 0));
    } else {   // y wraps: tile row 0 (or the last) reads the other end, so stages 1 and 2 take the whole grid
      for (int s = 0; s < 2; ++s)
        if ((e = launch(h, ks[s], h->grid_stage[s], s + 1))) return e;
      for (int k = 0; k < nc; ++k)
        if ((e = finish_chunk(k, h->stream))) return e;
    }
    return CHIMERA_OK;
  };
  rc = issue();
  for (auto st : h->band_stream)
    if (st) cudaStreamSynchronize(st);
  const cudaError_t e_copy = h->copy_stream ? cudaStreamSynchronize(h->copy_stream) : cudaSuccess;
  const cudaError_t e_main = cudaStreamSynchronize(h->stream);
  if (rc) { cudaGetLastError(); return rc; }
  if (e_copy != cudaSuccess) return cuda_fail(e_copy);
  if (e_main != cudaSuccess) return cuda_fail(e_main);
  if (!c.active) return CHIMERA_OK;
  h->dt_valid[0] = true;   // the stage-3 finish computed the next dt
  rc = read_ctl(h, 0, &c);
  if (rc) return rc;
  return c.status ? CHIMERA_ERR_NONFINITE : CHIMERA_OK;
}

int chimera_batch_set_time(chimera_handle* h, int m, double t, int output_count) {
  if (!h || m < 0 || m >= h->n || output_count < 1) return CHIMERA_ERR_BAD_ARG;
  Control c;
  int rc = read_ctl(h, m, &c);
  if (rc) return rc;
  c.t = t;
  c.output_count = output_count;
  c.active = (t < h->cfg[m].t_end) ? 1 : 0;
  CK(cudaMemcpyAsync(h->d_ctl + m, &c, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->dt_valid[m] = false;
  return CHIMERA_OK;
}

int chimera_set_time(chimera_handle* h, double t, int output_count) {
  return chimera_batch_set_time(h, 0, t, output_count);
}

int chimera_step(chimera_handle* h, int nsteps) {
  NvtxRange range("chimera_step");
  if (!h || nsteps < 0) return CHIMERA_ERR_BAD_ARG;
  if (nsteps == 0) return CHIMERA_OK;
  return run_steps(h, nsteps);
}

int chimera_set_graph_steps(chimera_handle* h, int nsteps) {
  if (!h || nsteps < 0) return CHIMERA_ERR_BAD_ARG;
  h->graph_steps_request = nsteps;
  if (nsteps == 0) drop_graph(h);
  return CHIMERA_OK;
}

int chimera_advance(chimera_handle* h, int max_steps, int* steps_taken) {
  NvtxRange range("chimera_advance");
  if (!h || max_steps < 0) return CHIMERA_ERR_BAD_ARG;
  std::vector<Control> c(h->n);
  std::vector<unsigned long long> s0(h->n);
  CK(cudaMemcpyAsync(c.data(), h->d_ctl, sizeof(Control) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  bool any_active = false;
  for (int m = 0; m < h->n; ++m) {
    s0[m] = c[m].steps;
    any_active = any_active || c[m].active;
  }
  int done = 0;
  const int chunk = 16;
  while (any_active && done < max_steps) {
    const int k = std::min(chunk, max_steps - done);
    int rc = run_steps(h, k);
    if (rc) return rc;
    done += k;
    CK(cudaMemcpyAsync(c.data(), h->d_ctl, sizeof(Control) * h->n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    bool any = false;
    for (int m = 0; m < h->n; ++m) any = any || c[m].active;
    if (!any) break;
  }
  if (steps_taken) {
    unsigned long long mx = 0;
    for (int m = 0; m < h->n; ++m) mx = std::max(mx, c[m].steps - s0[m]);
    *steps_taken = int(mx);
  }
  for (int m = 0; m < h->n; ++m)
    if (c[m].status) return CHIMERA_ERR_NONFINITE;
  return CHIMERA_OK;
}

// Set (pause = true) or clear the pause-at-output flag of every member; a
// member that paused is resumed (active again while t < t_end).
static int set_pause(chimera_handle* h, bool pause) {
  std::vector<Control> c(h->n);
  CK(cudaMemcpyAsync(c.data(), h->d_ctl, sizeof(Control) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int m = 0; m < h->n; ++m) {
    if (c[m].flags & CTL_PAUSED) c[m].active = (c[m].t < h->cfg[m].t_end) ? 1 : 0;
    c[m].flags = pause ? CTL_PAUSE_AT_OUTPUT : 0;
  }
  CK(cudaMemcpyAsync(h->d_ctl, c.data(), sizeof(Control) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return CHIMERA_OK;
}

int chimera_advance_output(chimera_handle* h, int max_steps, int* steps_taken) {
  NvtxRange range("chimera_advance_output");
  if (!h || max_steps < 0) return CHIMERA_ERR_BAD_ARG;
  int rc = set_pause(h, true);
  if (rc) return rc;
  rc = chimera_advance(h, max_steps, steps_taken);
  const int rc2 = set_pause(h, false);   // on the error path too: no member stays paused
  return rc ? rc : rc2;
}

int chimera_stage(chimera_handle* h, int k, double dt) {
  if (!h || k < 1 || k > 3) return CHIMERA_ERR_BAD_ARG;
  for (int m = 0; m < h->n; ++m) {
    Control c;
    int rc = read_ctl(h, m, &c);
    if (rc) return rc;
    c.dt = dt;
    c.active = 1;
    CK(cudaMemcpyAsync(h->d_ctl + m, &c, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->dt_valid[m] = false;
  }
  return launch(h, h->ks.stage[h->riemann - 1][k - 1], h->grid_stage[k - 1], k);
}

int chimera_batch_diag(chimera_handle* h, int m, chimera_diag_out* out) {
  if (!h || !out || m < 0 || m >= h->n) return CHIMERA_ERR_BAD_ARG;
  int rc = ensure_dt(h);
  if (rc) return rc;
  Control c;
  rc = read_ctl(h, m, &c);
  if (rc) return rc;
  const chimera_cfg& cf = h->cfg[m];
  out->t = c.t;
  out->dt = c.dt;
  out->output_count = c.output_count;
  out->active = c.active;
  out->steps = c.steps;
  out->divb_max = c.divb_max;
  out->divb_mean = c.divb_sum / double(cells_of(cf));
  out->bmax = c.bmax;
  out->divb_rel = (c.bmax > 0.0) ? c.divb_max * std::min(cf.dx, cf.dy) / c.bmax : 0.0;
  out->mass = c.mass;
  out->energy = c.energy;
  out->cfl_speed = c.cfl_speed;
  out->mood_resets = c.mood_resets;
  out->floor_hits = c.floor_hits;
  out->status = c.status;
  return CHIMERA_OK;
}

int chimera_diag(chimera_handle* h, chimera_diag_out* out) { return chimera_batch_diag(h, 0, out); }

int chimera_set_profiling(chimera_handle* h, int on) {
  if (!h) return CHIMERA_ERR_BAD_ARG;
  h->profiling = on ? 1 : 0;
  return CHIMERA_OK;
}

int chimera_get_profile(chimera_handle* h, double* ms, long long* launches, int reset) {
  if (!h || !ms || !launches) return CHIMERA_ERR_BAD_ARG;
  CK(cudaStreamSynchronize(h->stream));
  harvest_profile(h);
  for (int k = 0; k < 4; ++k) {
    ms[k] = h->prof_ms[k];
    launches[k] = h->prof_n[k];
    if (reset) { h->prof_ms[k] = 0.0; h->prof_n[k] = 0; }
  }
  return CHIMERA_OK;
}

int chimera_variant_count(chimera_handle* h) { return h ? int(h->variants.size()) : CHIMERA_ERR_BAD_ARG; }

int chimera_get_variant(chimera_handle* h, int* variant, int* tile_x, int* tile_y, int* threads) {
  if (!h) return CHIMERA_ERR_BAD_ARG;
  if (variant) *variant = h->cur_variant;
  if (tile_x) *tile_x = h->ks.stage[0][0].tx;
  if (tile_y) *tile_y = h->ks.stage[0][0].ty;
  if (threads) *threads = h->ks.stage[0][0].nt;
  return CHIMERA_OK;
}

int chimera_set_variant(chimera_handle* h, int v) {
  if (!h || v < 0 || v >= int(h->variants.size())) return CHIMERA_ERR_BAD_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return layout(h, v);
}

int chimera_autotune(chimera_handle* h, int reps, int* chosen, double* best_ms) {
  NvtxRange range("chimera_autotune");
  if (!h || reps < 1) return CHIMERA_ERR_BAD_ARG;
  int rc = ensure_dt(h);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int saved_prof = h->profiling;
  h->profiling = 0;
  int best = h->cur_variant;
  float best_t = 1e30f;
  for (int v = 0; v < int(h->variants.size()) && rc == CHIMERA_OK; ++v) {
    rc = layout(h, v);
    if (rc) break;
    h->dry = 1;
    rc = one_step(h);                       // warm-up
    if (rc == CHIMERA_OK) {
      cudaEventRecord(e0, h->stream);
      for (int r = 0; r < reps && rc == CHIMERA_OK; ++r) rc = one_step(h);
      cudaEventRecord(e1, h->stream);
    }
    h->dry = 0;
    float ms = 0.f;
    if (rc == CHIMERA_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
      if (ms < best_t) { best_t = ms; best = v; }
    } else if (rc == CHIMERA_OK) {
      rc = CHIMERA_ERR_CUDA;
    }
  }
  h->dry = 0;
  h->profiling = saved_prof;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  int lrc = layout(h, best);
  if (rc) return rc;
  if (lrc) return lrc;
  {
    std::lock_guard<std::mutex> lk(tune_mutex());
    tune_cache()[tune_key(h)] = best;
  }
  if (chosen) *chosen = best;
  if (best_ms) *best_ms = double(best_t) / reps;
  return CHIMERA_OK;
}

int chimera_set_counters(chimera_handle* h, int on) {
  if (!h) return CHIMERA_ERR_BAD_ARG;
  h->counters = on ? 1 : 0;
  drop_graph(h);
  return CHIMERA_OK;
}

int chimera_halo_pack(chimera_handle* h, int rows, void* lo, void* hi) {
  return halo_rows(h, rows, lo, hi, 0);
}

int chimera_halo_unpack(chimera_handle* h, int rows, const void* lo, const void* hi) {
  return halo_rows(h, rows, const_cast<void*>(lo), const_cast<void*>(hi), 1);
}

int chimera_slab_ghost_rows(chimera_handle* h, int ghost_lo, int ghost_hi) {
  if (!h || ghost_lo < 0 || ghost_hi < 0) return CHIMERA_ERR_BAD_ARG;
  if (h->n != 1) return CHIMERA_ERR_UNSUPPORTED;
  if (ghost_lo + ghost_hi >= h->cfg[0].ny) return CHIMERA_ERR_BAD_ARG;
  h->hm[0].skip_lo = ghost_lo;
  h->hm[0].skip_hi = ghost_hi;
  CK(cudaMemcpyAsync(h->d_members, h->hm.data(), sizeof(Member) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->dt_valid[0] = false;
  return CHIMERA_OK;
}

int chimera_refresh_dt(chimera_handle* h, double* d_dt) {
  if (!h) return CHIMERA_ERR_BAD_ARG;
  for (int m = 0; m < h->n; ++m) h->dt_valid[m] = false;
  int rc = ensure_dt(h);
  if (rc) return rc;
  if (d_dt)   // member m's Control::dt -> d_dt[m]
    CK(cudaMemcpy2DAsync(d_dt, sizeof(double), &h->d_ctl[0].dt, sizeof(Control), sizeof(double), h->n,
                         cudaMemcpyDeviceToDevice, h->stream));
  return CHIMERA_OK;
}

int chimera_get_dt_device(chimera_handle* h, double* d_dt) {
  if (!h || !d_dt) return CHIMERA_ERR_BAD_ARG;
  int rc = ensure_dt(h);
  if (rc) return rc;
  CK(cudaMemcpy2DAsync(d_dt, sizeof(double), &h->d_ctl[0].dt, sizeof(Control), sizeof(double), h->n,
                       cudaMemcpyDeviceToDevice, h->stream));
  return CHIMERA_OK;
}

int chimera_set_dt_device(chimera_handle* h, const double* d_dt) {
  if (!h || !d_dt) return CHIMERA_ERR_BAD_ARG;
  CK(cudaMemcpy2DAsync(&h->d_ctl[0].dt, sizeof(Control), d_dt, sizeof(double), sizeof(double), h->n,
                       cudaMemcpyDeviceToDevice, h->stream));
  for (int m = 0; m < h->n; ++m) h->dt_valid[m] = true;
  return CHIMERA_OK;
}

}  // extern "C"
