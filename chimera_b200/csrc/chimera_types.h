// chimera_types.h -- device-resident descriptors shared by the host runtime
// (chimera_api.cu) and the kernels.  Plain structs, no CUDA types.
#pragma once
#include <stdint.h>

namespace chimera {

constexpr int NPART = 6;  // per-tile partials: cfl speed max, |divB| max, |divB| sum, |B|^2 max, mass, energy

// Control::flags
enum : int {
  CTL_PAUSE_AT_OUTPUT = 1,   // stop (active = 0) after the step that reaches an output time
  CTL_PAUSED = 2,            // stopped there; the host resumes the member
};

enum : unsigned {
  STATUS_NONFINITE = 1u,   // a non-finite or non-positive quantity reached a reduction
  STATUS_TIMEOUT = 2u,     // a bounded wait gave up
  STATUS_BOUNDS = 4u,      // an index check failed (debug builds)
};

// One grid of the batch.  buf[b][q]: buffer b, field q; buffers 0 and 1
// alternate as the state U^n and the stage-1 scratch U1 (Control::parity
// says which holds the state), buffer 2 is the stage-2 scratch U2; field q (Mass, Momx, Momy, Energy, b_x, b_y), dense (ny, nx) with
// x fastest, element type given by the handle's precision.
struct Member {
  int nx, ny;
  int tiles_x, tiles_y;
  int tile_begin;          // first global work-list index of this member
  int periodic_x, periodic_y;      // the low side (x = 0, y = 0) wraps
  int periodic_xhi, periodic_yhi;  // the high side wraps (differs from the low side only in a mixed pair)
  int square;              // dx == dy: the reference's single-spacing expressions apply
  double dx, dy;
  double inv_dx, inv_dy;   // 1/dx, 1/dy as the reference computes them
  double inv_2dx, inv_2dy; // 1/(2 dx), 1/(2 dy)
  double hx, hy;           // 0.5*dx, 0.5*dy
  double gamma, vol, len;  // vol = dx*dy, len = min(dx, dy)
  double inv_vol;          // 1/vol (FP32-bulk pressure recovery)
  double rcp_vol, rcp_gm1; // RN(1/vol), RN(1/(gamma - 1)) for the reciprocal divisions (div_by),
                           // or 0 for a divisor outside 2^-120 <= b < 2^121 (shared_reciprocal)
  double courant, t_out, t_end;
  int skip_lo, skip_hi;     // rows at the bottom / top that the CFL kernel's dt and diagnostics
                           // leave out (the ghost rows of a y-slab; 0 otherwise)
  void* buf[3][6];
  const void* tmap;        // TMA variants: this member's tensor maps [buffer 3][field 6] (CUtensorMap,
                           // 128 bytes each, boxes of the variant's tile) in device memory, or null
};

// RN(1/b) for a divisor b fixed for the launch, or 0 (IEEE division throughout)
// where b lies outside 2^-120 <= |b| < 2^121, the range the reciprocal
// division (div_by in mhd_device.cuh) is exact for.
inline double shared_reciprocal(double b) {
  const double m = b < 0 ? -b : b;
  return (m >= 0x1p-120 && m < 0x1p121) ? 1.0 / b : 0.0;
}

// Time-loop state of one member, resident on the device so that whole runs
// can be captured in a CUDA graph.
struct Control {
  double t, dt;
  int output_count, active;
  int parity, flags;       // buf[parity] holds the current state; flags: CTL_*
  unsigned tiles_done, status;
  unsigned long long steps, mood_resets, floor_hits;
  double cfl_speed, divb_max, divb_sum, bmax, mass, energy;
};

struct StageArgs {
  const Member* members;
  Control* ctl;
  double* partials;        // [total_tiles][NPART]
  const int* tile_member;  // work index -> member (n_members > 1)
  int n_members;
  int total_tiles;          // one past the last work item of this launch
  int work_begin;           // first work item of this launch (0 unless a launch covers a band of rows)
  int limiter, slope_limiting, mood;
  int counters;            // count MOOD resets / floor hits
  int dry;                 // timing run: write scratch only, leave Control untouched
};

}  // namespace chimera
