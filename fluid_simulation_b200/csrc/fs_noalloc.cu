// WCSPH density + EOS for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at all: code running
// under an allocator that forbids device allocations after start-up, or a
// plugin inside another runtime that owns all device memory.  For them
// fs_wcsph_density_noalloc computes what fs_grid_build + fs_wcsph_density
// compute (compute_density_pressure, solver_wcsph.py:120-158) using only the
// caller's input/output arrays and one fixed scratch area that is part of the
// library image: a file-scope __device__ array sized for kNoAllocMaxParticles
// particles and a 32^3-cell hash table (about 1 MB; every GPU that loads the
// library holds it until the process exits).
//
// The hash dimensions do not change any result: the query still visits every
// cell overlapped by [x - h, x + h], extra (aliased) candidates lie outside
// the support and contribute W = 0, so only the summation order differs from
// the 128^3 grid of the other entry points.  The in-cell order is the same
// stable one as fs_grid_build's (crowded cells sorted by one block,
// fs_sort.cuh), and non-finite positions go to a bucket no query visits.
#include <cuda.h>

#include <mutex>

#include "fs_internal.cuh"
#include "fs_sort.cuh"

namespace fs {
namespace {

constexpr int kNoAllocMaxParticles = 16384;
constexpr int kNoAllocDim = 32;
constexpr int kNoAllocCells = kNoAllocDim * kNoAllocDim * kNoAllocDim;
constexpr int kCacheSlots = 64;  // CUDA contexts whose scratch address is cached

struct NoAllocScratch {
  int32_t key[kNoAllocMaxParticles];   // cell key per original particle
  int32_t slot[kNoAllocMaxParticles];  // arrival slot inside its cell; then the crowded-cell sort's second buffer
  int32_t tmp[kNoAllocMaxParticles];   // ids, unordered inside cells
  int32_t perm[kNoAllocMaxParticles];  // sorted slot -> original id
  int32_t count[kNoAllocCells + 1];    // occupancy (cleared by every call); the last bucket: non-finite positions
  int32_t off[kNoAllocCells + 2];      // exclusive prefix of count
  int32_t big_cells[kNoAllocMaxParticles / (kSmallCell + 1) + 1];  // cells too crowded to rank in place
  int32_t big_n;
  uint32_t status;                     // FS_STATUS_NONFINITE when a position is not finite
  float4 xs[kNoAllocMaxParticles];     // cell-sorted positions + flags word
  float mv[kNoAllocMaxParticles];      // rest_density * volume, cell order
};

// The scratch area.  Host code must not take this symbol's address directly:
// in host code the name is only a stand-in for the device object, so its
// device address is looked up with cudaGetSymbolAddress (scratch_address).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

__global__ void k_na_clear(NoAllocScratch* sc) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= kNoAllocCells; c += gridDim.x * blockDim.x)
    sc->count[c] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->big_n = 0;
    sc->status = 0;
  }
}

__global__ void k_na_keys(NoAllocScratch* sc, int n, const float* __restrict__ x, float inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  int k = kNoAllocCells;  // non-finite: the bucket after the cells, which no query visits
  if (isfinite(px) && isfinite(py) && isfinite(pz)) {
    GridDev g;
    g.dim_x = g.dim_y = g.dim_z = kNoAllocDim;
    g.mask_x = g.mask_y = g.mask_z = kNoAllocDim - 1;
    k = phys_cell(g, to_cell(__fmul_rn(px, inv), 0), to_cell(__fmul_rn(py, inv), 0), to_cell(__fmul_rn(pz, inv), 0));
  } else {
    atomicOr(&sc->status, FS_STATUS_NONFINITE);
  }
  sc->key[i] = k;
  sc->slot[i] = atomicAdd(&sc->count[k], 1);
}

// one block: exclusive prefix over the 32^3 cell counts
__global__ void k_na_scan(NoAllocScratch* sc) {
  constexpr int kPer = kNoAllocCells / 1024;
  __shared__ int32_t warp_tot[32];
  const int base = threadIdx.x * kPer;
  int32_t s = 0;
  for (int k = 0; k < kPer; ++k) s += sc->count[base + k];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int32_t w = warp_tot[lane];
    int32_t wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_tot[lane] = wi - w;
  }
  __syncthreads();
  int32_t run = inc - s + warp_tot[wid];
  for (int k = 0; k < kPer; ++k) {
    sc->off[base + k] = run;
    run += sc->count[base + k];
  }
  if (threadIdx.x == 1023) {
    sc->off[kNoAllocCells] = run;  // the non-finite bucket
    sc->off[kNoAllocCells + 1] = run + sc->count[kNoAllocCells];
  }
}

__global__ void k_na_scatter(NoAllocScratch* sc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sc->tmp[sc->off[sc->key[i]] + sc->slot[i]] = i;
}

// particle i into sorted slot d
__device__ __forceinline__ void na_gather(NoAllocScratch* sc, int d, int32_t i, const fs_model& m,
                                          const float* __restrict__ x) {
  sc->perm[d] = i;
  const int pf = particle_pf(m.particle_flags, m.particle_mask, i);
  sc->xs[d] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], pack_pf(pf));
  const float rd = m.rest_density[i];
  sc->mv[d] = rd * (m.particle_mass[i] / fmaxf(rd, 1.0e-6f));
}

// stable order inside each cell (ascending original id), then the gather;
// cells of more than kSmallCell particles are left to k_na_big_sort
__global__ void k_na_rank_gather(NoAllocScratch* sc, int n, fs_model m, const float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = sc->tmp[s];
  const int32_t c = sc->key[i];
  const int32_t a = sc->off[c], b = sc->off[c + 1];
  if (b - a > kSmallCell) {
    if (s == a) sc->big_cells[atomicAdd(&sc->big_n, 1)] = c;
    return;
  }
  int32_t rank = 0;
  for (int32_t t = a; t < b; ++t) rank += sc->tmp[t] < i ? 1 : 0;
  na_gather(sc, a + rank, i, m, x);
}

// the crowded cells, one block each: ids sorted ascending, then the gather
__global__ void __launch_bounds__(kSortThreads) k_na_big_sort(NoAllocScratch* sc, int n, fs_model m,
                                                              const float* __restrict__ x) {
  extern __shared__ int32_t sort_smem[];
  const int nbig = sc->big_n;
  for (int b = blockIdx.x; b < nbig; b += gridDim.x) {
    const int32_t c = sc->big_cells[b];
    const int32_t a = sc->off[c], len = sc->off[c + 1] - a;
    const int32_t* sorted = block_sort_ids(sc->tmp + a, sc->slot + a, len, id_bits(n), sort_smem);
    for (int k = threadIdx.x; k < len; k += blockDim.x) na_gather(sc, a + k, sorted[k], m, x);
    __syncthreads();
  }
}

__global__ void k_na_density(const NoAllocScratch* sc, int n, float inv, float h, const float* __restrict__ rest,
                             const float* __restrict__ stiffness, const float* __restrict__ exponent, int clamp,
                             float* rho, float* pressure) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  GridDev g;
  g.off = sc->off;
  g.perm = sc->perm;
  g.dim_x = g.dim_y = g.dim_z = kNoAllocDim;
  g.mask_x = g.mask_y = g.mask_z = kNoAllocDim - 1;
  g.rounding = 0;
  g.inv = inv;
  const float4 xi = sc->xs[s];
  const int32_t i = sc->perm[s];
  if (!(pf_of(xi) & PF_ACTIVE)) {
    rho[i] = 0.f;
    pressure[i] = 0.f;
    return;
  }
  const CubicK K(h);
  const float h2m = h * h * 1.000002f;
  float acc = 0.f;
  for_each_candidate(g, xi.x, xi.y, xi.z, h, [&](int t) {
    const float4 xj = sc->xs[t];
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, xj.w)));  // +inf for inactive
    if (r2 <= h2m) acc += sc->mv[t] * K.w(sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz))));
  });
  float p = stiffness[i] * (powf(acc / fmaxf(rest[i], 1.0e-6f), exponent[i]) - 1.0f);
  if (clamp) p = fmaxf(p, 0.f);
  rho[i] = acc;
  pressure[i] = p;
}

// Device address of the scratch area in the CUDA context current on the
// calling thread.  A module's __device__ symbol has its own address in each
// context (a runtime-managed primary context, or a context a host runtime
// created and made current), so the address is looked up once per context
// and cached under that context's id (cuCtxGetId: never reused within a
// process).  Without the driver entry points, or before any context exists
// on the thread, it is looked up on every call (cudaGetSymbolAddress makes
// the device's primary context current when none is).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct ScratchCache {
  std::mutex mutex;
  std::once_flag resolved;
  CtxGetCurrentFn get_current = nullptr;
  CtxGetIdFn get_id = nullptr;
  unsigned long long ctx_id[kCacheSlots] = {};
  NoAllocScratch* ptr[kCacheSlots] = {};
  int used = 0;
};
ScratchCache g_cache;

bool current_context_id(unsigned long long* id) {
  std::call_once(g_cache.resolved, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_cache.get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_cache.get_id = (CtxGetIdFn)f;
  });
  CUcontext ctx = nullptr;
  if (!g_cache.get_current || !g_cache.get_id || g_cache.get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return g_cache.get_id(ctx, id) == CUDA_SUCCESS;
}

int scratch_address(NoAllocScratch** out) {
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  if (have_id) {
    std::lock_guard<std::mutex> lock(g_cache.mutex);
    for (int k = 0; k < g_cache.used; ++k)
      if (g_cache.ctx_id[k] == id) {
        *out = g_cache.ptr[k];
        return FS_OK;
      }
  }
  void* p = nullptr;
  const int rc =
      check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "fs_wcsph_density_noalloc: cudaGetSymbolAddress");
  if (rc) return rc;
  *out = (NoAllocScratch*)p;
  if (have_id) {
    std::lock_guard<std::mutex> lock(g_cache.mutex);
    if (g_cache.used < kCacheSlots) {  // a full cache only means a lookup per call
      g_cache.ctx_id[g_cache.used] = id;
      g_cache.ptr[g_cache.used] = *out;
      ++g_cache.used;
    }
  }
  return FS_OK;
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

int32_t fs_noalloc_max_particles(void) { return kNoAllocMaxParticles; }

int fs_wcsph_density_noalloc(const fs_model* m, const float* x, float h, int32_t clamp_negative, float* rho,
                             float* pressure, fs_stream_t stream) {
  if (!m || m->n < 0 || !(h > 0.f)) return set_error(FS_ERR_INVALID, "fs_wcsph_density_noalloc: bad arguments");
  if (m->n > kNoAllocMaxParticles)
    return set_error(FS_ERR_CAPACITY,
                     "fs_wcsph_density_noalloc: %lld particles exceed the fixed scratch of %d particles; use "
                     "fs_grid_build + fs_wcsph_density",
                     (long long)m->n, kNoAllocMaxParticles);
  if (m->n == 0) return FS_OK;
  if (!x || !rho || !pressure || !m->particle_flags || !m->particle_mass || !m->rest_density || !m->stiffness ||
      !m->exponent)
    return set_error(FS_ERR_INVALID, "fs_wcsph_density_noalloc: missing array");
  NoAllocScratch* sc = nullptr;
  int rc = scratch_address(&sc);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = (int)m->n;
  const float inv = 1.0f / h;
  const int nb = (n + kBlock - 1) / kBlock;
  k_na_clear<<<33, 1024, 0, st>>>(sc);
  k_na_keys<<<nb, kBlock, 0, st>>>(sc, n, x, inv);
  k_na_scan<<<1, 1024, 0, st>>>(sc);
  k_na_scatter<<<nb, kBlock, 0, st>>>(sc, n);
  k_na_rank_gather<<<nb, kBlock, 0, st>>>(sc, n, *m, x);
  k_na_big_sort<<<16, kSortThreads, kSortSmemBytes, st>>>(sc, n, *m, x);
  k_na_density<<<nb, kBlock, 0, st>>>(sc, n, inv, h, m->rest_density, m->stiffness, m->exponent, clamp_negative, rho,
                                      pressure);
  rc = launch_check("fs_wcsph_density_noalloc");
  if (rc) return rc;
  // the status word comes back with the results: the call waits for its stream
  uint32_t status = 0;
  rc = check_cuda(cudaMemcpyAsync(&status, &sc->status, sizeof(status), cudaMemcpyDeviceToHost, st),
                  "fs_wcsph_density_noalloc: status read");
  if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "fs_wcsph_density_noalloc: sync");
  if (rc) return rc;
  if (status & FS_STATUS_NONFINITE)
    return set_error(FS_ERR_NONFINITE, "fs_wcsph_density_noalloc: a particle position is not finite (its density "
                                       "is 0 and it adds nothing to its neighbours')");
  return FS_OK;
}

}  // extern "C"
