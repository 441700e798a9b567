// Internal declarations shared by the CUDA translation units of libfluid_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fluid_b200.h"

// ------------------------------------------------------------------ layout --
// Cell-sorted particle data lives in the context (HBM), one slot per particle
// in hash-cell order, so every neighbour loop reads contiguous slot ranges:
//   xs[s]  float4 (x, y, z, packed flags)        -- position stream
//   vs[s]  float4 (vx, vy, vz, mass)              -- velocity stream
//   mv[s]  float   rest_density * volume          -- density weight
// Packed flags (bits of the .w word): PF_ACTIVE = ParticleFlags.ACTIVE,
// PF_DYNAMIC = active && particle_mask == 0.
namespace fs {

constexpr int PF_ACTIVE = 1;
constexpr int PF_DYNAMIC = 2;
constexpr int kBlock = 256;

struct DfsphDev {     // device-resident per-step DFSPH control block
  int32_t done;       // residual test passed: later kernels of this half exit
  int32_t iters;      // iterations entered in this half
  uint32_t ticket;    // last-block-done counter of the residual reduction
  int32_t worlds_done;  // batched contexts: worlds whose residual test passed (all: done = 1)
  double residual;    // last residual of this half
};

struct DfsphWorld {   // batched contexts: one world's decisions in one half of the substep
  int32_t done;       // this world's residual test passed: its particles leave the iterations
  int32_t iters;      // iterations this world entered
  double residual;    // its last residual (mean over its dynamic particles)
};

// Passes for the per-pass CUDA-event timer (fs_timer_*) and launch counter.
enum Pass {
  P_GRID = 0, P_GATHER, P_WCSPH_DENSITY, P_WCSPH_FORCE, P_DFSPH_DENSITY_FACTOR, P_DFSPH_ACCEL, P_DFSPH_RATE,
  P_DFSPH_CORRECT, P_DFSPH_INTEGRATE, P_DFSPH_FINAL, P_PBF_PREDICT, P_PBF_DENSITY, P_PBF_ACCEL, P_PBF_LAMBDA,
  P_PBF_DELTA, P_PBF_VELOCITY, P_PBF_XSPH, P_ADJ_INTEGRATE, P_ADJ_FORCE, P_ADJ_DENSITY, P_OTHER, P_APIC_SEPARATION, P_COUNT
};

struct PassTimer {
  bool on = false;
  int cap = 0, used = 0, dropped = 0;
  cudaEvent_t* ev = nullptr;  // 2 * cap events
  int* pass_of = nullptr;     // pass of each recorded pair
};

// One world (scene) of a batched context: its own box of cells (no hashing,
// no aliasing between worlds) and its own walls.
struct WorldDev {
  int32_t clo[3];  // cell coordinate of the box's first cell per axis
  int32_t dims[3]; // cells per axis
  int32_t base;    // key of its first cell
  float walls[3];  // bound_width, bound_height, bound_length of its tank
};

struct GridDev {
  const WorldDev* worlds = nullptr;  // batched context: per-world boxes (nullptr: the reference hash grid)
  int32_t nworlds = 0;
  const int32_t* off;   // [ncell + 1] exclusive prefix of cell occupancy (hash-key order)
  const int32_t* perm;  // [n] sorted slot -> original particle index (warp's point_ids)
  const int32_t* skey;  // [n] cell key of each sorted slot (warp's point_cells)
  int32_t dim_x, dim_y, dim_z, rounding;
  int32_t mask_x, mask_y, mask_z;  // dim - 1 when the dim is a power of two, else -1
  float inv;            // 1 / cell width, float32 as warp
  unsigned long long* tile_stats;  // list counters (fs_list_stats), null while counting is off
};

}  // namespace fs

struct fs_context {
  int32_t device = 0;
  int64_t capacity = 0;
  fs_grid_config grid{};
  int64_t ncell = 0;
  int64_t built_n = -1;      // n of the last grid build, -1 = none
  float built_inv = 0.f;
  cudaStream_t last_stream = nullptr;

  // grid build
  int32_t* key = nullptr;        // [cap] cell key of original particle i
  int32_t* slot = nullptr;       // [cap] arrival slot inside the cell
  int32_t* cell_count = nullptr; // [ncell + 1]; the last bucket holds non-finite positions
  int32_t* cell_off = nullptr;   // [ncell + 2]
  int32_t* tmp_ids = nullptr;    // [cap] unordered-in-cell ids
  int32_t* big_cells = nullptr;  // [max_big_cells(cap)] cells too crowded to rank in place
  int32_t* big_n = nullptr;      // [1] how many
  int32_t* perm = nullptr;       // [cap] sorted slot -> original index
  int32_t* skey = nullptr;       // [cap] cell key of each sorted slot
  int32_t* scan_part = nullptr;  // [scan blocks + 1]

  // cell-sorted streams
  float4* xs = nullptr;   // positions + packed flags
  float4* xs2 = nullptr;  // second position buffer (PBF Jacobi double buffer)
  float4* vs = nullptr;   // velocities + mass
  float4* vs2 = nullptr;  // second velocity buffer (DFSPH v*, PBF x_in)
  float* mv = nullptr;    // rest_density * volume
  float2* sc2 = nullptr;  // per-slot scalar pair (rho, p) / (rho, factor)
  float* sc1 = nullptr;   // per-slot scalar (kappa / lambda)
  float* sc1b = nullptr;  // per-slot scalar (second)
  float2* krm = nullptr;  // per-slot (kappa / rho, mass) for the DFSPH correction, (lambda, mass) for PBF's delta
  float* xo_tmp = nullptr;  // [cap*3] original-order scratch positions (PBF x_pred)
  float* vo_tmp = nullptr;  // [cap*3] original-order scratch velocities (PBF v_pred)

  // reductions / status
  double* red_part = nullptr;   // [reduction blocks]
  int64_t* red_cnt = nullptr;   // [reduction blocks]
  fs::DfsphDev* dfsph = nullptr; // [2] control blocks (density half, divergence half)
  fs::DfsphWorld* dfsph_worlds = nullptr;  // batched contexts: [2][nworlds] per-world decisions
  uint32_t* status = nullptr;
  uint32_t* pbf_disp = nullptr;  // PBF: largest displacement (float bits) since the lists' recording
  unsigned long long* tile_stats = nullptr;  // list counters (fs_list_stats)
  bool stats_on = false;                     // count them (fs_list_stats_enable)

  // neighbour lists (fs_nbr.cuh)
  int32_t* nb_idx = nullptr;     // [kNbMax][cap]
  int32_t* nb_cnt = nullptr;     // [cap]
  void* nb_ctl = nullptr;        // ListCtl

  // batched (multi-world) contexts
  fs::WorldDev* worlds = nullptr;  // [nworlds] device table
  int32_t nworlds = 0;
  float world_cell = 0.f;          // cell width of the world boxes (the solvers' h)

  // frame metrics scratch (fs_metrics.cu)
  void* metrics = nullptr;

  // the frame clock of the clocked substep in progress (null otherwise)
  const fs_frame_clock* clock = nullptr;

  // launch tuning of the neighbour kernels (fs_context_set_tuning)
  int32_t nb_block = 128;      // threads per block: 64, 128 or 256
  int32_t nb_ppt = 1;          // particles per thread: 1, 2 or 4
  float cell_ratio = 1.f;      // WCSPH grid cell width / h: 1 or 1/2
  float list_skin = 0.02f;     // PBF first-density list skin / h (0: the first lambda pass scans)

  // instrumentation
  fs::PassTimer timer;
  int64_t launches = 0;  // kernels launched through this context (host count)
};

namespace fs {

// --------------------------------------------------------------- host util --
int set_error(int code, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);
int launch_check(const char* what);

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

inline int blocks_for(int64_t n, int b = kBlock) { return (int)((n + b - 1) / b); }

// Blocks of a neighbour-kernel launch under the context's tuning.
inline int nb_blocks(const fs_context* c, int64_t n) {
  const int64_t per = (int64_t)c->nb_block * c->nb_ppt;
  const int64_t b = (n + per - 1) / per;
  return (int)(b > 0 ? b : 1);
}

// Brackets the launches of one pass: counts them and, when the timer is on,
// records a CUDA event pair around them on the launching stream.
struct PassScope {
  fs_context* c;
  cudaStream_t st;
  int slot = -1;
  PassScope(fs_context* ctx, int pass, cudaStream_t stream, int nkernels = 1) : c(ctx), st(stream) {
    c->launches += nkernels;
    PassTimer& t = c->timer;
    if (!t.on) return;
    if (t.used >= t.cap) {
      ++t.dropped;
      return;
    }
    slot = t.used++;
    t.pass_of[slot] = pass;
    cudaEventRecord(t.ev[2 * slot], st);
  }
  ~PassScope() {
    if (slot >= 0) cudaEventRecord(c->timer.ev[2 * slot + 1], st);
  }
};

// grid build (fs_grid.cu)
// world: particle_world of the model (required by batched contexts, unused otherwise)
// clock (optional): a device-side frame clock; its kernels do nothing while
// clock->active == 0 (the frame is complete).
int grid_build(fs_context* c, const float* x, int64_t n, float radius, cudaStream_t st, const int32_t* world,
               const fs_frame_clock* clock = nullptr);

// Whether a kernel of a clocked substep has work (no clock: always).
__device__ __forceinline__ bool clock_idle(const fs_frame_clock* clock) { return clock && !clock->active; }
GridDev grid_view(const fs_context* c);

// DFSPH residual helper shared with the separate-pass entry (fs_dfsph.cu)
int reduction_blocks(int64_t n);

// bytes of the frame-metrics scratch of a context (fs_metrics.cu)
size_t metrics_scratch_bytes(int64_t capacity);

// Grid-stride loop over cell-sorted slots: thread k of a grid of G threads
// takes slots k, k + G, ...  Launched with ceil(n / (block * p)) blocks,
// every thread handles p particles (fs_tuning.particles_per_thread).
template <class F>
__device__ __forceinline__ void for_slots(int64_t n, F&& f) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) f(s);
}

// ----------------------------------------------------------- device math --
#define FS_DEV __device__ __forceinline__

constexpr float kPi = 3.14159265358979323846f;

// The .w word of a position: PF bits (a denormal, adds nothing measurable to
// an r^2) for an active particle, +inf for an inactive one, so that an
// r^2 + w test rejects inactive candidates without reading any flag.
// Bits 2..21 carry the world index in batched contexts (still a denormal).
FS_DEV int pf_of(float4 p) { return __float_as_int(p.w) & (PF_ACTIVE | PF_DYNAMIC); }
FS_DEV float pack_pf(int pf, int world = 0) {
  return __int_as_float((pf & PF_ACTIVE) ? (pf | ((world & 0xFFFFF) << 2)) : 0x7f800000);
}
FS_DEV int world_of(float4 p) { return (__float_as_int(p.w) >> 2) & 0xFFFFF; }

// Distance computed with individually rounded operations (no FMA), so that
// decisions such as `r < h` are bit-identical to a strict FP32 evaluation.
FS_DEV float dist2_rn(float dx, float dy, float dz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

struct CubicK {   // constants of the cubic spline of support h
  float h, k;     // k = 8 / (pi h^3)
  FS_DEV explicit CubicK(float h_) : h(h_), k(8.0f / (kPi * (h_ * h_ * h_))) {}
  // W(r), solver_wcsph.py:21-34
  FS_DEV float w(float r) const {
    const float q = r / h;
    float res = 0.f;
    if (q <= 1.f) {
      if (q <= 0.5f) {
        const float q2 = q * q;
        const float q3 = q2 * q;
        res = k * (6.f * q3 - 6.f * q2 + 1.f);
      } else {
        const float t = 1.f - q;
        res = 2.f * k * (t * t * t);
      }
    }
    return res;
  }
  // scalar s with grad W(d) = s * d for |d| = r, solver_wcsph.py:37-51
  FS_DEV float dw_scale(float r) const {
    const float q = r / h;
    float s = 0.f;
    if (r > 1.0e-5f && q <= 1.f) {
      const float inv = 1.f / (r * h);
      if (q <= 0.5f) {
        s = 6.f * k * q * (3.f * q - 2.f) * inv;
      } else {
        const float t = 1.f - q;
        s = -6.f * k * t * t * inv;
      }
    }
    return s;
  }
};

struct PbfK {     // poly6 / spiky constants, solver_pbf.py:24-45
  float h, h2, kw, kg;
  FS_DEV explicit PbfK(float h_) : h(h_), h2(h_ * h_) {
    const float c = h_ * h_ * h_;
    kw = 315.0f / (64.0f * kPi * (c * c * c));
    kg = -45.0f / (kPi * (c * c));
  }
  FS_DEV float w(float r) const {
    float res = 0.f;
    if (h > 0.f && r < h) {
      const float rhs = h2 - r * r;
      res = kw * (rhs * rhs * rhs);
    }
    return res;
  }
  FS_DEV float dw_scale(float r) const {  // spiky gradient = s * d
    float s = 0.f;
    if (h > 0.f && r > 1.0e-6f && r < h) s = kg * ((h - r) * (h - r) / r);
    return s;
  }
};

// ------------------------------------------------------ neighbour queries --
FS_DEV int to_cell(float v, int rounding) {
  if (!(v == v)) return 0;
  if (rounding == 1) v = floorf(v);
  if (v > 536870912.0f) return 536870912;
  if (v < -536870912.0f) return -536870912;
  return __float2int_rz(v);
}

FS_DEV int wrap_axis(int v, int dim) {
  v += (1 << 20);
  v = v < 0 ? 0 : v;
  return v % dim;
}

// same, with a power-of-two mask when there is one (mask >= 0)
FS_DEV int wrap_axis(int v, int dim, int mask) {
  v += (1 << 20);
  v = v < 0 ? 0 : v;
  return mask >= 0 ? (v & mask) : v % dim;
}

FS_DEV int phys_cell(const GridDev& g, int x, int y, int z) {
  return (wrap_axis(z, g.dim_z, g.mask_z) * g.dim_y + wrap_axis(y, g.dim_y, g.mask_y)) * g.dim_x +
         wrap_axis(x, g.dim_x, g.mask_x);
}

// Visits the candidates of warp's hash_grid_query(grid, p, r) in the same
// order: cells z-outer, y-middle, x-inner, each cell's slots in sorted order.
// f(t) receives the cell-sorted SLOT t (original index = perm[t]).  A run of
// consecutive x cells is one contiguous slot range because cell offsets are a
// prefix sum in hash-key order; a run that wraps modulo dim_x splits in two.
FS_DEV int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Batched contexts.  A world's cell along one axis is the reference's cell
// coordinate (warp's truncating int(v / cell), as the hash grid bins it)
// relative to the box's first cell, clamped into the box.  The map is
// monotone in v, so a query box [p - r, p + r] mapped the same way covers
// every particle of the world within r of p, including particles outside the
// box (they sit in its edge cells).  Inside the box the cells, their order
// and the order inside each cell are those of the hash grid of the world
// alone (no aliasing while a world spans fewer cells than the hash dims), so
// a batched step reproduces the step of each world by itself.  No hashing:
// cells of different worlds never alias, and a query never leaves its world.
FS_DEV int world_axis_cell(float v, float inv, int clo, int d) {
  return clampi(to_cell(__fmul_rn(v, inv), 0) - clo, 0, d - 1);
}

FS_DEV int world_index(int w, int nworlds) { return clampi(w, 0, nworlds - 1); }

FS_DEV int world_cell_key(const WorldDev& W, float inv, float px, float py, float pz) {
  const int cx = world_axis_cell(px, inv, W.clo[0], W.dims[0]);
  const int cy = world_axis_cell(py, inv, W.clo[1], W.dims[1]);
  const int cz = world_axis_cell(pz, inv, W.clo[2], W.dims[2]);
  return W.base + (cz * W.dims[1] + cy) * W.dims[0] + cx;
}

// The cells a query at p with radius r visits: [x0, x1] x [y0, y1] x [z0, z1]
// in the world's box coordinates (batched contexts) or in unwrapped hash-grid
// cell coordinates (wrapped modulo the dims when visited).
struct QueryBox {
  int x0, x1, y0, y1, z0, z1;
};

FS_DEV QueryBox query_box_world(const GridDev& g, const WorldDev& W, float px, float py, float pz, float r) {
  auto cell = [&](float v, int k) { return world_axis_cell(v, g.inv, W.clo[k], W.dims[k]); };
  return QueryBox{cell(__fsub_rn(px, r), 0), cell(__fadd_rn(px, r), 0), cell(__fsub_rn(py, r), 1),
                  cell(__fadd_rn(py, r), 1), cell(__fsub_rn(pz, r), 2), cell(__fadd_rn(pz, r), 2)};
}

FS_DEV QueryBox query_box_hash(const GridDev& g, float px, float py, float pz, float r) {
  QueryBox b;
  b.x0 = to_cell(__fmul_rn(__fsub_rn(px, r), g.inv), g.rounding);
  b.y0 = to_cell(__fmul_rn(__fsub_rn(py, r), g.inv), g.rounding);
  b.z0 = to_cell(__fmul_rn(__fsub_rn(pz, r), g.inv), g.rounding);
  b.x1 = min(to_cell(__fmul_rn(__fadd_rn(px, r), g.inv), g.rounding), b.x0 + g.dim_x - 1);
  b.y1 = min(to_cell(__fmul_rn(__fadd_rn(py, r), g.inv), g.rounding), b.y0 + g.dim_y - 1);
  b.z1 = min(to_cell(__fmul_rn(__fadd_rn(pz, r), g.inv), g.rounding), b.z0 + g.dim_z - 1);
  return b;
}

// Whether queries at p and q (same world w) visit the same cells.
FS_DEV bool same_query_cells(const GridDev& g, int w, float4 p, float4 q, float r) {
  QueryBox a, b;
  if (g.worlds) {
    const WorldDev& W = g.worlds[world_index(w, g.nworlds)];
    a = query_box_world(g, W, p.x, p.y, p.z, r);
    b = query_box_world(g, W, q.x, q.y, q.z, r);
  } else {
    a = query_box_hash(g, p.x, p.y, p.z, r);
    b = query_box_hash(g, q.x, q.y, q.z, r);
  }
  return a.x0 == b.x0 && a.x1 == b.x1 && a.y0 == b.y0 && a.y1 == b.y1 && a.z0 == b.z0 && a.z1 == b.z1;
}

// The query cells of world w in the order z-outer, y, x-inner; each row of
// x cells is one contiguous slot range, passed to rf(first, end).
template <class RF>
FS_DEV void for_each_range_world(const GridDev& g, int w, float px, float py, float pz, float r, RF&& rf) {
  const WorldDev& W = g.worlds[world_index(w, g.nworlds)];
  const QueryBox b = query_box_world(g, W, px, py, pz, r);
  // the offsets of the next row load before the current row is scanned,
  // as in for_each_range_hash
  if (b.z0 > b.z1 || b.y0 > b.y1) return;
  auto row_of = [&](int z, int y) { return W.base + (z * W.dims[1] + y) * W.dims[0]; };
  int z = b.z0, y = b.y0, row = row_of(z, y);
  int a = __ldg(g.off + row + b.x0), e = __ldg(g.off + row + b.x1 + 1);
  while (true) {
    int zn = z, yn = y + 1;
    if (yn > b.y1) {
      yn = b.y0;
      ++zn;
    }
    const bool more = zn <= b.z1;
    int an = 0, en = 0;
    if (more) {
      row = row_of(zn, yn);
      an = __ldg(g.off + row + b.x0);
      en = __ldg(g.off + row + b.x1 + 1);
    }
    rf(a, e);
    if (!more) break;
    z = zn;
    y = yn;
    a = an;
    e = en;
  }
}

// Visits the candidates of warp's hash_grid_query(grid, p, r) in the same
// order as contiguous slot ranges rf(first, end): cells z-outer, y-middle,
// x-inner, each cell's slots in sorted order.  A run of consecutive x cells
// is one range because cell offsets are a prefix sum in hash-key order; a
// run that wraps modulo dim_x splits in two.
template <class RF>
FS_DEV void for_each_range_hash(const GridDev& g, float px, float py, float pz, float r, RF&& rf) {
  const QueryBox b = query_box_hash(g, px, py, pz, r);
  const int x0 = b.x0, x1 = b.x1, y0 = b.y0, y1 = b.y1, z0 = b.z0, z1 = b.z1;
  const int nx = x1 - x0 + 1;
  const int xa = x0 + (1 << 20);
  if (xa >= 0 && z0 <= z1 && y0 <= y1) {
    // the offsets of the next row are loaded before the current row is
    // scanned, so their latency overlaps the scan (PBF substep -0.6 %)
    const int cx0 = g.mask_x >= 0 ? (xa & g.mask_x) : xa % g.dim_x;
    const int len1 = min(nx, g.dim_x - cx0);
    auto row_of = [&](int z, int y) {
      return (wrap_axis(z, g.dim_z, g.mask_z) * g.dim_y + wrap_axis(y, g.dim_y, g.mask_y)) * g.dim_x;
    };
    int z = z0, y = y0, row = row_of(z, y);
    int a = __ldg(g.off + row + cx0), e = __ldg(g.off + row + cx0 + len1);
    while (true) {
      int zn = z, yn = y + 1;
      if (yn > y1) {
        yn = y0;
        ++zn;
      }
      const bool more = zn <= z1;
      int rown = 0, an = 0, en = 0;
      if (more) {
        rown = row_of(zn, yn);
        an = __ldg(g.off + rown + cx0);
        en = __ldg(g.off + rown + cx0 + len1);
      }
      rf(a, e);
      if (nx > len1) rf(__ldg(g.off + row), __ldg(g.off + row + (nx - len1)));
      if (!more) break;
      z = zn;
      y = yn;
      row = rown;
      a = an;
      e = en;
    }
    return;
  }
  // far outside the shifted range (cells clamp): visit one by one
  for (int z = z0; z <= z1; ++z) {
    const int cz = wrap_axis(z, g.dim_z, g.mask_z);
    for (int y = y0; y <= y1; ++y) {
      const int row = (cz * g.dim_y + wrap_axis(y, g.dim_y, g.mask_y)) * g.dim_x;
      for (int x = x0; x <= x1; ++x) {
        const int c = row + wrap_axis(x, g.dim_x, g.mask_x);
        rf(__ldg(g.off + c), __ldg(g.off + c + 1));
      }
    }
  }
}

// The candidate ranges of a query at (px, py, pz) of world w (w is ignored
// by the reference hash grid).
template <class RF>
FS_DEV void for_each_range(const GridDev& g, int w, float px, float py, float pz, float r, RF&& rf) {
  if (g.worlds)
    for_each_range_world(g, w, px, py, pz, r, rf);
  else
    for_each_range_hash(g, px, py, pz, r, rf);
}

// The same candidates one slot at a time: f(t), t = cell-sorted SLOT
// (original index = perm[t]).
template <class F>
FS_DEV void for_each_candidate(const GridDev& g, int w, float px, float py, float pz, float r, F&& f) {
  for_each_range(g, w, px, py, pz, r, [&](int a, int e) {
    for (int t = a; t < e; ++t) f(t);
  });
}

template <class F>
FS_DEV void for_each_candidate(const GridDev& g, float px, float py, float pz, float r, F&& f) {
  for_each_range_hash(g, px, py, pz, r, [&](int a, int e) {
    for (int t = a; t < e; ++t) f(t);
  });
}

// Box walls of the reference's apply_bounds variants.
//   mode 0: WCSPH  (solver_wcsph.py:264-305) clamp to [-W,W]x[-H,H]x[0,2L], damp outward v
//   mode 1: DFSPH  (solver_dfsph.py:407-442) same walls, damping unconditional
//   mode 2: PBF    (solver_pbf.py:467-517)  walls inset by radius + eps, damp outward v
struct Walls {
  float xmin, xmax, ymin, ymax, zmin, zmax, damping, radius, eps;
  int mode;
};

__host__ __device__ inline Walls make_walls(float w, float hgt, float l, float damping, int mode, float radius, float eps) {
  Walls b;
  b.radius = radius;
  b.eps = eps;
  b.mode = mode;
  b.damping = damping;
  if (mode == 2) {
    b.xmin = -w + radius + eps;
    b.xmax = w - radius - eps;
    b.ymin = -hgt + radius + eps;
    b.ymax = hgt - radius - eps;
    b.zmin = radius + eps;
    b.zmax = l * 2.0f - radius - eps;
  } else {
    b.xmin = -w;
    b.xmax = w;
    b.ymin = -hgt;
    b.ymax = hgt;
    b.zmin = 0.f;
    b.zmax = l * 2.0f;
  }
  return b;
}

// The walls of world w in a batched context (its tank), else the step's walls.
FS_DEV Walls walls_of(const Walls& b, const GridDev& g, int w) {
  if (!g.worlds) return b;
  const WorldDev& W = g.worlds[world_index(w, g.nworlds)];
  return make_walls(W.walls[0], W.walls[1], W.walls[2], b.damping, b.mode, b.radius, b.eps);
}

FS_DEV void apply_walls(const Walls& b, float3& p, float3& v) {
  const bool cond = b.mode != 1;
  if (p.x < b.xmin) { p.x = b.xmin; if (!cond || v.x < 0.f) v.x = v.x * b.damping; }
  if (p.x > b.xmax) { p.x = b.xmax; if (!cond || v.x > 0.f) v.x = v.x * b.damping; }
  if (p.y < b.ymin) { p.y = b.ymin; if (!cond || v.y < 0.f) v.y = v.y * b.damping; }
  if (p.y > b.ymax) { p.y = b.ymax; if (!cond || v.y > 0.f) v.y = v.y * b.damping; }
  if (p.z < b.zmin) { p.z = b.zmin; if (!cond || v.z < 0.f) v.z = v.z * b.damping; }
  if (p.z > b.zmax) { p.z = b.zmax; if (!cond || v.z > 0.f) v.z = v.z * b.damping; }
}

// apply_position_bounds, solver_pbf.py:367-399 (walls of mode 2, no velocity)
FS_DEV void clamp_position(const Walls& b, float3& p) {
  if (p.x < b.xmin) p.x = b.xmin;
  if (p.x > b.xmax) p.x = b.xmax;
  if (p.y < b.ymin) p.y = b.ymin;
  if (p.y > b.ymax) p.y = b.ymax;
  if (p.z < b.zmin) p.z = b.zmin;
  if (p.z > b.zmax) p.z = b.zmax;
}

FS_DEV float3 ld3(const float* p, int64_t i) { return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
FS_DEV void st3(float* p, int64_t i, float3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
FS_DEV float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }

FS_DEV int particle_pf(const int32_t* flags, const int32_t* mask, int64_t i) {
  const bool act = (flags[i] & 1) != 0;
  const bool dyn = act && (mask ? mask[i] == 0 : true);
  return (act ? PF_ACTIVE : 0) | (dyn ? PF_DYNAMIC : 0);
}

// Slot s (particle i = perm[s]) of the cell-order copies that the neighbour
// loops read: xs = (x, flags + world), vs = (v, mass) when vs, and mv =
// rest_density * volume with volume = mass / max(rest_density, 1e-6)
// (compute_particle_volume, solver_wcsph.py:110-116) when mv.  A world index
// past the model's worlds raises FS_STATUS_BOUNDS.
FS_DEV void gather_common_slot(int64_t s, int32_t i, const fs_model& m, const float* __restrict__ x,
                               const float* __restrict__ v, float4* __restrict__ xs, float4* __restrict__ vs,
                               float* __restrict__ mv, uint32_t* status, int nworlds) {
  const float3 p = ld3(x, i);
  const int pf = particle_pf(m.particle_flags, m.particle_mask, i);
  // batched contexts carry the world in the flags word (queries stay in it)
  const int w = (nworlds > 0 && m.particle_world) ? world_index(m.particle_world[i], nworlds) : 0;
  xs[s] = make_float4(p.x, p.y, p.z, pack_pf(pf, w));
  const float mass = m.particle_mass[i];
  if (vs) {
    const float3 u = ld3(v, i);
    vs[s] = make_float4(u.x, u.y, u.z, mass);
  }
  if (mv) {
    const float rd = m.rest_density[i];
    mv[s] = rd * (mass / fmaxf(rd, 1.0e-6f));
  }
  if (m.particle_world) {
    const int wi = m.particle_world[i];
    if (wi >= m.n_worlds) atomicOr(status, FS_STATUS_BOUNDS);
  }
}

// walls_of for a kernel in original particle order (world from particle_world)
FS_DEV Walls walls_of_particle(const Walls& b, const GridDev& g, const fs_model& m, int64_t i) {
  if (!g.worlds) return b;
  return walls_of(b, g, m.particle_world ? m.particle_world[i] : 0);
}

FS_DEV float3 gravity_of(const fs_model& m, int64_t i) {
  // reference: gravity[max(world, 0)]; an index past the last world (which
  // the reference would read out of bounds) is clamped here and reported as
  // FS_STATUS_BOUNDS by the gather.
  int w = m.particle_world ? m.particle_world[i] : 0;
  w = w < 0 ? 0 : w;
  w = w >= m.n_worlds ? m.n_worlds - 1 : w;
  return ld3(m.gravity, w);
}

}  // namespace fs
