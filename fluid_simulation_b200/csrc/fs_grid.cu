// Hash-grid build: the B200 replacement of warp's wp.HashGrid.build
// (called at solver_wcsph.py:456, solver_dfsph.py:624/783, solver_pbf.py:737/858).
//
// Result (identical to a stable radix sort of (cell key, particle id)):
//   perm[s]      original index of the particle in sorted slot s
//   off[c]       first slot of cell c; off[c+1] one past its last slot
// Algorithm (O(N) + O(cells) HBM traffic, deterministic):
//   1. keys:    cell key per particle, arrival slot by atomicAdd on the cell count
//   2. scan:    exclusive prefix of the counts (tile sums, then a down-sweep
//               in which each tile adds up the sums before it)
//   3. scatter: tmp[off[key] + arrival] = i        (order inside a cell arbitrary)
//   4. rank:    slot = off[key] + #{j in cell : j < i}; perm[slot] = i, for
//               cells of up to kSmallCell particles
//   5. crowded cells: one block sorts each cell's ids (fs_sort.cuh)
// Steps 4-5 restore ascending original index inside each cell, which is the
// order warp's stable radix sort produces, so results do not depend on the
// order in which atomics were served; the work is O(N) at any occupancy.
// Non-finite positions are not binned into a cell: they take the extra key
// ncell (after every cell, visited by no query) and raise
// FS_STATUS_NONFINITE, so a blown-up state costs no more than a finite one.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "fs_nbr.cuh"
#include "fs_sort.cuh"

namespace fs {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096 cells per block

// A thread's kScanItems consecutive counts: two 16-byte loads when all lie
// below m (base is a multiple of 8, the arrays come from cudaMalloc).
__device__ __forceinline__ void load_items(const int32_t* __restrict__ in, int64_t base, int64_t m,
                                           int32_t (&v)[kScanItems]) {
  static_assert(kScanItems == 8, "two int4 per thread");
  if (base + kScanItems <= m) {
    const int4 a = __ldg(reinterpret_cast<const int4*>(in + base));
    const int4 b = __ldg(reinterpret_cast<const int4*>(in + base) + 1);
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = base + k < m ? in[base + k] : 0;
  }
}

__global__ void k_cell_keys(int64_t n, const float* __restrict__ x, float inv, int dim_x, int dim_y, int dim_z,
                            int rounding, int32_t discard, int32_t* __restrict__ key, int32_t* __restrict__ slot,
                            int32_t* __restrict__ count, int32_t* big_n, uint32_t* status,
                            const fs_frame_clock* clock) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || clock_idle(clock)) return;
  if (i == 0) *big_n = 0;  // crowded cells of this build, counted by k_rank
  const float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  int k = discard;
  if (!(isfinite(px) && isfinite(py) && isfinite(pz))) {
    atomicOr(status, FS_STATUS_NONFINITE);
  } else {
    GridDev g;
    g.dim_x = dim_x;
    g.dim_y = dim_y;
    g.dim_z = dim_z;
    g.mask_x = g.mask_y = g.mask_z = -1;
    k = phys_cell(g, to_cell(__fmul_rn(px, inv), rounding), to_cell(__fmul_rn(py, inv), rounding),
                  to_cell(__fmul_rn(pz, inv), rounding));
  }
  key[i] = k;
  slot[i] = atomicAdd(count + k, 1);
}

// Batched contexts: key = (world, cell) as the world's base + its local cell.
__global__ void k_cell_keys_worlds(int64_t n, const float* __restrict__ x, const int32_t* __restrict__ world,
                                   const WorldDev* __restrict__ worlds, int nworlds, float inv, int32_t discard,
                                   int32_t* __restrict__ key, int32_t* __restrict__ slot,
                                   int32_t* __restrict__ count, int32_t* big_n, uint32_t* status,
                                   const fs_frame_clock* clock) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || clock_idle(clock)) return;
  if (i == 0) *big_n = 0;
  const float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  const int w = world[i];
  if (w < 0 || w >= nworlds) atomicOr(status, FS_STATUS_BOUNDS);
  int k = discard;
  if (!(isfinite(px) && isfinite(py) && isfinite(pz)))
    atomicOr(status, FS_STATUS_NONFINITE);
  else
    k = world_cell_key(worlds[world_index(w, nworlds)], inv, px, py, pz);
  key[i] = k;
  slot[i] = atomicAdd(count + k, 1);
}

// phase 1: per-tile sums
__global__ void k_scan_reduce(const int32_t* __restrict__ in, int64_t m, int32_t* __restrict__ part,
                              const fs_frame_clock* clock) {
  if (clock_idle(clock)) return;
  __shared__ int32_t warp_sums[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  load_items(in, base, m, v);
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int32_t v = threadIdx.x < kScanThreads / 32 ? warp_sums[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
  }
}

// block-wide exclusive scan of one value per thread (blockDim multiple of 32, <= 1024)
__device__ int32_t block_exclusive_scan(int32_t v, int32_t* total) {
  __shared__ int32_t ws[32];
  __shared__ int32_t block_total;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int32_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int32_t w = lane < nw ? ws[lane] : 0;
    int32_t wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nw) ws[lane] = wi - w;  // exclusive prefix of warp sums
    if (lane == nw - 1) block_total = wi;
  }
  __syncthreads();
  const int32_t res = inc - v + ws[wid];
  if (total) *total = block_total;
  __syncthreads();
  return res;
}

// phase 2: scan inside tiles, offset by the sum of the preceding tiles
// counts (each block adds up part[0 .. blockIdx.x) itself: at most a few
// thousand integers, exact in any order); out has m + 1 entries
__global__ void k_scan_down(const int32_t* __restrict__ in, int64_t m, const int32_t* __restrict__ part,
                            int32_t* __restrict__ out, const fs_frame_clock* clock) {
  if (clock_idle(clock)) return;
  int32_t before = 0;
  for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) before += __ldcg(part + k);
  int32_t prefix = 0;
  block_exclusive_scan(before, &prefix);
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  load_items(in, base, m, v);
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  int32_t tile = 0;
  int32_t run = block_exclusive_scan(s, &tile) + prefix;
  int32_t o[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    o[k] = run;
    run += v[k];
  }
  if (base + kScanItems <= m) {  // two 16-byte stores
    reinterpret_cast<int4*>(out + base)[0] = make_int4(o[0], o[1], o[2], o[3]);
    reinterpret_cast<int4*>(out + base)[1] = make_int4(o[4], o[5], o[6], o[7]);
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (base + k < m) out[base + k] = o[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[m] = prefix + tile;
}

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ key, const int32_t* __restrict__ slot,
                          const int32_t* __restrict__ off, int32_t* __restrict__ tmp, const fs_frame_clock* clock) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || clock_idle(clock)) return;
  tmp[off[key[i]] + slot[i]] = (int32_t)i;
}

__global__ void k_rank(int64_t n, const int32_t* __restrict__ key, const int32_t* __restrict__ off,
                       const int32_t* __restrict__ tmp, int32_t* __restrict__ perm, int32_t* __restrict__ skey,
                       int32_t* big_cells, int32_t* big_n, const fs_frame_clock* clock) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || clock_idle(clock)) return;
  const int32_t i = tmp[s];
  const int32_t c = key[i];
  const int32_t a = off[c], b = off[c + 1];
  if (b - a > kSmallCell) {  // crowded: sorted by k_big_sort
    if (s == a) big_cells[atomicAdd(big_n, 1)] = c;
    return;
  }
  int32_t rank = 0;
  for (int32_t t = a; t < b; ++t) rank += tmp[t] < i ? 1 : 0;
  perm[a + rank] = i;
  skey[a + rank] = c;
}

// The crowded cells listed by k_rank, one block each (grid-stride over the
// list): ids sorted ascending, then perm / skey written.
__global__ void __launch_bounds__(kSortThreads) k_big_sort(int64_t n, const int32_t* __restrict__ off,
                                                           int32_t* tmp, int32_t* perm, int32_t* skey,
                                                           const int32_t* __restrict__ big_cells,
                                                           const int32_t* __restrict__ big_n,
                                                           const fs_frame_clock* clock) {
  extern __shared__ int32_t sort_smem[];
  if (clock_idle(clock)) return;
  const int nbig = *big_n;
  const int bits = id_bits(n);
  for (int b = blockIdx.x; b < nbig; b += gridDim.x) {
    const int32_t c = big_cells[b];
    const int32_t a = off[c], len = off[c + 1] - a;
    int32_t* sorted = block_sort_ids(tmp + a, perm + a, len, bits, sort_smem);
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
      perm[a + k] = sorted[k];  // same element when sorted == perm + a
      skey[a + k] = c;
    }
    __syncthreads();
  }
}

__global__ void k_tables(int64_t n, int64_t ncell, const int32_t* __restrict__ perm, const int32_t* __restrict__ key,
                         const int32_t* __restrict__ off, int32_t* point_ids, int32_t* point_cells,
                         int32_t* cell_starts, int32_t* cell_ends) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    const int32_t i = perm[t];
    if (point_ids) point_ids[t] = i;
    if (point_cells) point_cells[t] = key[i];  // == skey[t]
  }
  if (t < ncell) {
    if (cell_starts) cell_starts[t] = off[t];
    if (cell_ends) cell_ends[t] = off[t + 1];
  }
}

template <bool FILL>
__global__ void k_candidates(GridDev g, const float* __restrict__ q, const int32_t* __restrict__ qworld, int64_t nq,
                             float r, int64_t* counts, const int64_t* __restrict__ offsets, int32_t* cand) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  int64_t k = 0;
  const int64_t base = FILL ? offsets[i] : 0;
  const int w = qworld ? qworld[i] : 0;
  for_each_candidate(g, w, q[3 * i], q[3 * i + 1], q[3 * i + 2], r, [&](int t) {
    if (FILL) cand[base + k] = g.perm[t];
    ++k;
  });
  counts[i] = k;
}

}  // namespace

int scan_blocks(int64_t m) { return (int)((m + kScanTile - 1) / kScanTile); }

constexpr int kBigSortBlocks = 148;  // one per SM

NbrList nbr_list(const fs_context* c) {
  NbrList L;
  L.idx = c->nb_idx;
  L.cnt = c->nb_cnt;
  L.stride = c->capacity > 0 ? c->capacity : 1;
  L.ctl = (ListCtl*)c->nb_ctl;
  return L;
}

GridDev grid_view(const fs_context* c) {
  GridDev g;
  g.off = c->cell_off;
  g.perm = c->perm;
  g.skey = c->skey;
  g.dim_x = c->grid.dim_x;
  g.dim_y = c->grid.dim_y;
  g.dim_z = c->grid.dim_z;
  g.rounding = c->grid.rounding;
  auto pow2mask = [](int d) { return (d & (d - 1)) == 0 ? d - 1 : -1; };
  g.mask_x = pow2mask(g.dim_x);
  g.mask_y = pow2mask(g.dim_y);
  g.mask_z = pow2mask(g.dim_z);
  g.inv = c->built_inv;
  g.tile_stats = c->stats_on ? c->tile_stats : nullptr;
  g.worlds = c->worlds;
  g.nworlds = c->nworlds;
  return g;
}

int grid_build(fs_context* c, const float* x, int64_t n, float radius, cudaStream_t st, const int32_t* world,
               const fs_frame_clock* clock) {
  if (n < 0 || (n > 0 && !x) || !(radius > 0.f)) return set_error(FS_ERR_INVALID, "grid_build: bad arguments");
  if (c->worlds && n > 0 && !world)
    return set_error(FS_ERR_INVALID, "grid_build: a batched context needs particle_world");
  if (n > c->capacity) return set_error(FS_ERR_CAPACITY, "grid_build: n=%lld > capacity=%lld", (long long)n,
                                        (long long)c->capacity);
  const float inv = 1.0f / radius;
  PassScope ps_(c, P_GRID, st, n > 0 ? 6 : 2);
  // ncell + 1 buckets: the cells, then the non-finite positions
  const int64_t nbucket = c->ncell + 1;
  const int32_t discard = (int32_t)c->ncell;
  int rc = check_cuda(cudaMemsetAsync(c->cell_count, 0, sizeof(int32_t) * nbucket, st), "memset cell counts");
  if (rc) return rc;
  // a new grid invalidates recorded neighbour lists
  rc = check_cuda(cudaMemsetAsync(c->nb_ctl, 0, sizeof(ListCtl), st), "memset list control");
  if (rc) return rc;
  if (n > 0 && c->worlds)
    k_cell_keys_worlds<<<blocks_for(n), kBlock, 0, st>>>(n, x, world, c->worlds, c->nworlds, inv, discard, c->key,
                                                         c->slot, c->cell_count, c->big_n, c->status, clock);
  else if (n > 0)
    k_cell_keys<<<blocks_for(n), kBlock, 0, st>>>(n, x, inv, c->grid.dim_x, c->grid.dim_y, c->grid.dim_z,
                                                   c->grid.rounding, discard, c->key, c->slot, c->cell_count, c->big_n,
                                                   c->status, clock);
  const int nb = scan_blocks(nbucket);
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(c->cell_count, nbucket, c->scan_part, clock);
  k_scan_down<<<nb, kScanThreads, 0, st>>>(c->cell_count, nbucket, c->scan_part, c->cell_off, clock);
  if (n > 0) {
    k_scatter<<<blocks_for(n), kBlock, 0, st>>>(n, c->key, c->slot, c->cell_off, c->tmp_ids, clock);
    k_rank<<<blocks_for(n), kBlock, 0, st>>>(n, c->key, c->cell_off, c->tmp_ids, c->perm, c->skey, c->big_cells,
                                             c->big_n, clock);
    // a few blocks, each taking crowded cells from the list (none: they return at once)
    k_big_sort<<<kBigSortBlocks, kSortThreads, kSortSmemBytes, st>>>(n, c->cell_off, c->tmp_ids, c->perm, c->skey,
                                                                      c->big_cells, c->big_n, clock);
  }
  rc = launch_check("grid_build");
  if (rc) return rc;
  c->built_n = n;
  c->built_inv = inv;
  c->last_stream = st;
  return FS_OK;
}

}  // namespace fs

using namespace fs;

// ------------------------------------------------------------ error state --
namespace fs {
static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FS_OK;
  return set_error(FS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int launch_check(const char* what) { return check_cuda(cudaGetLastError(), what); }
}  // namespace fs

namespace fs {
// tallies the current lists: [0] usable, [1] overflowed (their particles rescan)
__global__ void k_list_tally(int64_t n, const int32_t* __restrict__ cnt, unsigned long long* out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = s < n && cnt[s] <= kNbMax, over = s < n && cnt[s] > kNbMax;
  const unsigned a = __ballot_sync(0xffffffffu, ok), b = __ballot_sync(0xffffffffu, over);
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(out, (unsigned long long)__popc(a));
    if (b) atomicAdd(out + 1, (unsigned long long)__popc(b));
  }
}
}  // namespace fs

extern "C" {

const char* fs_last_error_string(void) { return fs::g_err; }
const char* fs_version(void) { return "fluid_b200 0.1 (sm_100a)"; }

static int context_alloc(fs_context* c, int64_t capacity, int64_t ncell);

int fs_context_create(fs_context** out, int64_t capacity, const fs_grid_config* grid, int32_t device) {
  if (!out || capacity < 0 || !grid || grid->dim_x <= 0 || grid->dim_y <= 0 || grid->dim_z <= 0 ||
      (grid->rounding != 0 && grid->rounding != 1))
    return set_error(FS_ERR_INVALID, "fs_context_create: bad arguments");
  const int64_t ncell = (int64_t)grid->dim_x * grid->dim_y * grid->dim_z;
  if (ncell >= (int64_t)kScanTile * 4096 || capacity > (int64_t)0x7fffffff)
    return set_error(FS_ERR_INVALID, "fs_context_create: grid of %lld cells or capacity too large",
                     (long long)ncell);
  DeviceGuard dg(device);
  fs_context* c = new fs_context();
  c->device = device;
  c->grid = *grid;
  int rc = context_alloc(c, capacity, ncell);
  if (rc) return rc;
  *out = c;
  return FS_OK;
}

int fs_context_create_worlds(fs_context** out, int64_t capacity, const fs_world_box* worlds, int32_t nworlds,
                             int32_t device) {
  if (!out || capacity < 0 || !worlds || nworlds < 1 || nworlds > (1 << 20) || capacity > (int64_t)0x7fffffff)
    return set_error(FS_ERR_INVALID, "fs_context_create_worlds: bad arguments");
  WorldDev* host = new WorldDev[nworlds];
  int64_t ncell = 0;
  for (int w = 0; w < nworlds; ++w) {
    const fs_world_box& b = worlds[w];
    if (b.dims[0] <= 0 || b.dims[1] <= 0 || b.dims[2] <= 0 || !(b.bound_width >= 0.f) || !(b.bound_height >= 0.f) ||
        !(b.bound_length >= 0.f)) {
      delete[] host;
      return set_error(FS_ERR_INVALID, "fs_context_create_worlds: world %d has an empty box or bad walls", w);
    }
    const int64_t cells = (int64_t)b.dims[0] * b.dims[1] * b.dims[2];
    WorldDev& d = host[w];
    for (int k = 0; k < 3; ++k) {
      d.clo[k] = b.cell_lo[k];
      d.dims[k] = b.dims[k];
    }
    d.walls[0] = b.bound_width;
    d.walls[1] = b.bound_height;
    d.walls[2] = b.bound_length;
    d.base = (int32_t)(ncell < 0x7fffffff ? ncell : 0x7fffffff);
    ncell += cells;
    if (ncell >= (int64_t)kScanTile * 4096) {
      delete[] host;
      return set_error(FS_ERR_INVALID, "fs_context_create_worlds: more than %lld cells in all",
                       (long long)kScanTile * 4096);
    }
  }
  DeviceGuard dg(device);
  fs_context* c = new fs_context();
  c->device = device;
  c->grid = fs_grid_config{0, 0, 0, 1};
  int rc = context_alloc(c, capacity, ncell);  // frees c on failure
  if (rc) {
    delete[] host;
    return rc;
  }
  rc = check_cuda(cudaMalloc((void**)&c->worlds, sizeof(WorldDev) * nworlds), "fs_context_create_worlds");
  if (!rc)
    rc = check_cuda(cudaMemcpy(c->worlds, host, sizeof(WorldDev) * nworlds, cudaMemcpyHostToDevice),
                    "fs_context_create_worlds: copy");
  if (!rc)
    rc = check_cuda(cudaMalloc((void**)&c->dfsph_worlds, sizeof(DfsphWorld) * 2 * nworlds),
                    "fs_context_create_worlds: decisions");
  if (!rc)
    rc = check_cuda(cudaMemset(c->dfsph_worlds, 0, sizeof(DfsphWorld) * 2 * nworlds),
                    "fs_context_create_worlds: memset");
  delete[] host;
  if (rc) {
    fs_context_destroy(c);
    return rc;
  }
  c->nworlds = nworlds;
  *out = c;
  return FS_OK;
}

int fs_context_set_tuning(fs_context* c, const fs_tuning* t) {
  if (!c || !t) return set_error(FS_ERR_INVALID, "fs_context_set_tuning: null argument");
  if (t->block_size != 64 && t->block_size != 128 && t->block_size != 256)
    return set_error(FS_ERR_INVALID, "fs_context_set_tuning: block_size must be 64, 128 or 256 (got %d)",
                     (int)t->block_size);
  if (t->particles_per_thread != 1 && t->particles_per_thread != 2 && t->particles_per_thread != 4)
    return set_error(FS_ERR_INVALID, "fs_context_set_tuning: particles_per_thread must be 1, 2 or 4 (got %d)",
                     (int)t->particles_per_thread);
  if (t->cell_ratio != 1.0f && t->cell_ratio != 0.5f)
    return set_error(FS_ERR_INVALID, "fs_context_set_tuning: cell_ratio must be 1 or 0.5");
  if (c->worlds && t->cell_ratio != 1.0f)
    return set_error(FS_ERR_INVALID, "fs_context_set_tuning: batched contexts bin in cells of width h");
  if (!(t->list_skin >= 0.f && t->list_skin <= 0.25f))
    return set_error(FS_ERR_INVALID, "fs_context_set_tuning: list_skin must lie in [0, 0.25]");
  c->nb_block = t->block_size;
  c->nb_ppt = t->particles_per_thread;
  c->cell_ratio = t->cell_ratio;
  c->list_skin = t->list_skin;
  return FS_OK;
}

int fs_context_get_tuning(const fs_context* c, fs_tuning* t) {
  if (!c || !t) return set_error(FS_ERR_INVALID, "fs_context_get_tuning: null argument");
  t->block_size = c->nb_block;
  t->particles_per_thread = c->nb_ppt;
  t->cell_ratio = c->cell_ratio;
  t->list_skin = c->list_skin;
  return FS_OK;
}

int32_t fs_context_worlds(const fs_context* c) { return c ? c->nworlds : -1; }
int64_t fs_context_cells(const fs_context* c) { return c ? c->ncell : -1; }

// Device scratch of a context; frees the context on failure.
static int context_alloc(fs_context* c, int64_t capacity, int64_t ncell) {
  c->capacity = capacity;
  c->ncell = ncell;
  const int64_t cap = capacity > 0 ? capacity : 1;
  const int nb = scan_blocks(ncell + 1);
  const int rb = reduction_blocks(cap);
  struct A {
    void** p;
    size_t bytes;
  } allocs[] = {
      {(void**)&c->key, sizeof(int32_t) * cap},         {(void**)&c->slot, sizeof(int32_t) * cap},
      {(void**)&c->cell_count, sizeof(int32_t) * (ncell + 1)}, {(void**)&c->cell_off, sizeof(int32_t) * (ncell + 2)},
      {(void**)&c->big_cells, sizeof(int32_t) * max_big_cells(cap)}, {(void**)&c->big_n, sizeof(int32_t)},
      {(void**)&c->tmp_ids, sizeof(int32_t) * cap},     {(void**)&c->perm, sizeof(int32_t) * cap},
      {(void**)&c->skey, sizeof(int32_t) * cap},
      {(void**)&c->scan_part, sizeof(int32_t) * (nb + 1)},
      {(void**)&c->xs, sizeof(float4) * cap},           {(void**)&c->xs2, sizeof(float4) * cap},
      {(void**)&c->vs, sizeof(float4) * cap},           {(void**)&c->vs2, sizeof(float4) * cap},
      {(void**)&c->mv, sizeof(float) * cap},            {(void**)&c->sc2, sizeof(float2) * cap},
      {(void**)&c->sc1, sizeof(float) * cap},           {(void**)&c->sc1b, sizeof(float) * cap},
      {(void**)&c->krm, sizeof(float2) * cap},
      {(void**)&c->xo_tmp, sizeof(float) * 3 * cap},    {(void**)&c->vo_tmp, sizeof(float) * 3 * cap},
      {(void**)&c->red_part, sizeof(double) * rb},      {(void**)&c->red_cnt, sizeof(int64_t) * rb},
      {(void**)&c->dfsph, sizeof(DfsphDev) * 2},         {(void**)&c->status, sizeof(uint32_t)},
      {(void**)&c->pbf_disp, sizeof(uint32_t)},
      {(void**)&c->tile_stats, sizeof(unsigned long long) * 8},
      {(void**)&c->nb_idx, sizeof(int32_t) * kNbMax * cap},  {(void**)&c->nb_cnt, sizeof(int32_t) * cap},
      {(void**)&c->nb_ctl, sizeof(ListCtl)},
      {(void**)&c->metrics, metrics_scratch_bytes(cap)},
  };
  for (auto& a : allocs) {
    cudaError_t e = cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) {
      int rc = check_cuda(e, "fs_context_create: cudaMalloc");
      fs_context_destroy(c);
      return rc;
    }
  }
  int rc = check_cuda(cudaMemset(c->status, 0, sizeof(uint32_t)), "fs_context_create: memset");
  if (!rc) rc = check_cuda(cudaMemset(c->dfsph, 0, sizeof(DfsphDev) * 2), "fs_context_create: memset");
  if (!rc) rc = check_cuda(cudaMemset(c->tile_stats, 0, sizeof(unsigned long long) * 8), "fs_context_create: memset");
  if (!rc) rc = check_cuda(cudaMemset(c->nb_ctl, 0, sizeof(ListCtl)), "fs_context_create: memset");
  if (rc) {
    fs_context_destroy(c);
    return rc;
  }
  return FS_OK;
}

static void timer_free(PassTimer& t);

int fs_context_destroy(fs_context* c) {
  if (!c) return FS_OK;
  DeviceGuard dg(c->device);
  timer_free(c->timer);
  void* ps[] = {c->key, c->slot, c->cell_count, c->cell_off, c->big_cells, c->big_n, c->tmp_ids, c->perm, c->skey, c->scan_part, c->xs, c->xs2,
                c->vs, c->vs2, c->mv, c->sc2, c->sc1, c->sc1b, c->krm, c->xo_tmp, c->vo_tmp, c->red_part, c->red_cnt,
                c->dfsph, c->status, c->tile_stats, c->nb_idx, c->nb_cnt, c->nb_ctl, c->worlds, c->metrics,
                c->dfsph_worlds, c->pbf_disp};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete c;
  return FS_OK;
}

int64_t fs_context_capacity(const fs_context* c) { return c ? c->capacity : -1; }

int fs_grid_build(fs_context* c, const float* x, int64_t n, float radius, fs_stream_t stream) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_grid_build: null context");
  if (c->worlds) return set_error(FS_ERR_INVALID, "fs_grid_build: batched context, use fs_grid_build_worlds");
  DeviceGuard dg(c->device);
  return grid_build(c, x, n, radius, (cudaStream_t)stream, nullptr);
}

int fs_grid_build_worlds(fs_context* c, const float* x, const int32_t* world, int64_t n, float radius,
                         fs_stream_t stream) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_grid_build_worlds: null context");
  if (!c->worlds) return set_error(FS_ERR_INVALID, "fs_grid_build_worlds: not a batched context");
  DeviceGuard dg(c->device);
  return grid_build(c, x, n, radius, (cudaStream_t)stream, world);
}

int fs_grid_tables(fs_context* c, int32_t* point_ids, int32_t* point_cells, int32_t* cell_starts,
                   int32_t* cell_ends, fs_stream_t stream) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_grid_tables: null context");
  if (c->built_n < 0) return set_error(FS_ERR_NOGRID, "fs_grid_tables: no grid built");
  DeviceGuard dg(c->device);
  const int64_t m = c->built_n > c->ncell ? c->built_n : c->ncell;
  {
    PassScope ps_(c, P_OTHER, (cudaStream_t)stream);
    k_tables<<<blocks_for(m), kBlock, 0, (cudaStream_t)stream>>>(c->built_n, c->ncell, c->perm, c->key, c->cell_off,
                                                               point_ids, point_cells, cell_starts, cell_ends);
  }
  return launch_check("fs_grid_tables");
}

static int grid_candidates(fs_context* c, const float* q, const int32_t* qworld, int64_t nq, float r,
                           int64_t* counts, const int64_t* offsets, int32_t* cand, fs_stream_t stream);

int fs_grid_candidates(fs_context* c, const float* q, int64_t nq, float r, int64_t* counts, const int64_t* offsets,
                       int32_t* cand, fs_stream_t stream) {
  if (c && c->worlds) return set_error(FS_ERR_INVALID, "fs_grid_candidates: batched context, use *_worlds");
  return grid_candidates(c, q, nullptr, nq, r, counts, offsets, cand, stream);
}

int fs_grid_candidates_worlds(fs_context* c, const float* q, const int32_t* qworld, int64_t nq, float r,
                              int64_t* counts, const int64_t* offsets, int32_t* cand, fs_stream_t stream) {
  if (c && !c->worlds) return set_error(FS_ERR_INVALID, "fs_grid_candidates_worlds: not a batched context");
  if (nq > 0 && !qworld) return set_error(FS_ERR_INVALID, "fs_grid_candidates_worlds: null qworld");
  return grid_candidates(c, q, qworld, nq, r, counts, offsets, cand, stream);
}

static int grid_candidates(fs_context* c, const float* q, const int32_t* qworld, int64_t nq, float r,
                           int64_t* counts, const int64_t* offsets, int32_t* cand, fs_stream_t stream) {
  if (!c || nq < 0 || (nq > 0 && (!q || !counts)) || (cand && !offsets))
    return set_error(FS_ERR_INVALID, "fs_grid_candidates: bad arguments");
  if (c->built_n < 0) return set_error(FS_ERR_NOGRID, "fs_grid_candidates: no grid built");
  if (nq == 0) return FS_OK;
  DeviceGuard dg(c->device);
  GridDev g = grid_view(c);
  cudaStream_t st = (cudaStream_t)stream;
  if (cand) {
    PassScope ps_(c, P_OTHER, st);
    k_candidates<true><<<blocks_for(nq), kBlock, 0, st>>>(g, q, qworld, nq, r, counts, offsets, cand);
  }
  else
    {
      PassScope ps_(c, P_OTHER, st);
      k_candidates<false><<<blocks_for(nq), kBlock, 0, st>>>(g, q, qworld, nq, r, counts, nullptr, nullptr);
    }
  return launch_check("fs_grid_candidates");
}

static const char* kPassNames[P_COUNT] = {
    "grid_build", "gather", "wcsph_density", "wcsph_force", "dfsph_density_factor", "dfsph_accel", "dfsph_rate",
    "dfsph_correct", "dfsph_integrate", "dfsph_final", "pbf_predict", "pbf_density", "pbf_accel", "pbf_lambda",
    "pbf_delta", "pbf_velocity", "pbf_xsph", "wcsph_adjoint_integrate", "wcsph_adjoint_force",
    "wcsph_adjoint_density", "other", "apic_separation"};

int32_t fs_pass_count(void) { return P_COUNT; }

const char* fs_pass_name(int32_t pass) { return (pass >= 0 && pass < P_COUNT) ? kPassNames[pass] : ""; }

int64_t fs_launch_count(const fs_context* c) { return c ? c->launches : -1; }

static void timer_free(PassTimer& t) {
  if (t.ev) {
    for (int k = 0; k < 2 * t.cap; ++k) cudaEventDestroy(t.ev[k]);
    delete[] t.ev;
    delete[] t.pass_of;
  }
  t = PassTimer{};
}

int fs_timer_enable(fs_context* c, int32_t capacity) {
  if (!c || capacity < 0) return set_error(FS_ERR_INVALID, "fs_timer_enable: bad arguments");
  DeviceGuard dg(c->device);
  PassTimer& t = c->timer;
  if (capacity == 0) {
    timer_free(t);
    return FS_OK;
  }
  if (t.cap != capacity) {
    timer_free(t);
    t.ev = new cudaEvent_t[2 * (size_t)capacity];
    t.pass_of = new int[capacity];
    for (int k = 0; k < 2 * capacity; ++k) {
      int rc = check_cuda(cudaEventCreate(&t.ev[k]), "fs_timer_enable: cudaEventCreate");
      if (rc) {
        t.cap = k / 2;
        timer_free(t);
        return rc;
      }
    }
    t.cap = capacity;
  }
  t.used = 0;
  t.dropped = 0;
  t.on = true;
  return FS_OK;
}

int fs_timer_read(fs_context* c, float* ms_per_pass, int32_t* launches_per_pass, int32_t npass, int32_t* dropped) {
  if (!c || !ms_per_pass || !launches_per_pass || npass < P_COUNT)
    return set_error(FS_ERR_INVALID, "fs_timer_read: bad arguments");
  DeviceGuard dg(c->device);
  PassTimer& t = c->timer;
  for (int p = 0; p < npass; ++p) {
    ms_per_pass[p] = 0.f;
    launches_per_pass[p] = 0;
  }
  for (int k = 0; k < t.used; ++k) {
    int rc = check_cuda(cudaEventSynchronize(t.ev[2 * k + 1]), "fs_timer_read: sync");
    if (rc) return rc;
    float ms = 0.f;
    rc = check_cuda(cudaEventElapsedTime(&ms, t.ev[2 * k], t.ev[2 * k + 1]), "fs_timer_read: elapsed");
    if (rc) return rc;
    ms_per_pass[t.pass_of[k]] += ms;
    launches_per_pass[t.pass_of[k]] += 1;
  }
  if (dropped) *dropped = t.dropped;
  t.on = false;
  t.used = 0;
  return FS_OK;
}

int fs_status_read(fs_context* c, uint32_t* status) {
  if (!c || !status) return set_error(FS_ERR_INVALID, "fs_status_read: bad arguments");
  DeviceGuard dg(c->device);
  int rc = check_cuda(cudaMemcpyAsync(status, c->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->last_stream),
                      "fs_status_read");
  if (rc) return rc;
  return check_cuda(cudaStreamSynchronize(c->last_stream), "fs_status_read: sync");
}

int fs_list_stats(fs_context* c, int64_t* counters, int32_t ncounters, int32_t reset) {
  if (!c || !counters || ncounters < 0) return set_error(FS_ERR_INVALID, "fs_list_stats: bad arguments");
  DeviceGuard dg(c->device);
  unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int rc = check_cuda(cudaStreamSynchronize(c->last_stream), "fs_list_stats: sync");
  if (!rc) rc = check_cuda(cudaMemset(c->tile_stats, 0, 2 * sizeof(unsigned long long)), "fs_list_stats: clear");
  const int64_t n = c->built_n > 0 ? c->built_n : 0;
  if (!rc && n > 0) {
    k_list_tally<<<blocks_for(n), kBlock>>>(n, c->nb_cnt, c->tile_stats);
    rc = launch_check("fs_list_stats");
  }
  if (!rc) rc = check_cuda(cudaMemcpy(h, c->tile_stats, sizeof(h), cudaMemcpyDeviceToHost), "fs_list_stats");
  if (rc) return rc;
  for (int k = 0; k < ncounters && k < 8; ++k) counters[k] = (int64_t)h[k];
  if (reset) rc = check_cuda(cudaMemset(c->tile_stats, 0, sizeof(h)), "fs_list_stats: reset");
  return rc;
}

int fs_list_stats_enable(fs_context* c, int32_t on) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_list_stats_enable: null context");
  c->stats_on = on != 0;
  return FS_OK;
}

int fs_status_clear(fs_context* c, fs_stream_t stream) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_status_clear: null context");
  DeviceGuard dg(c->device);
  return check_cuda(cudaMemsetAsync(c->status, 0, sizeof(uint32_t), (cudaStream_t)stream), "fs_status_clear");
}

}  // extern "C"
