// Frame metrics of the dam-break harness (simulation.py:198-225) as device
// reductions: the reference copies positions, velocities, densities and
// pressures to the host every frame and reduces them with numpy; here one
// call reduces them on the device and the host reads back 14 doubles.
//
//   out[0]  1 if any position or velocity is non-finite     out[7]  density mean
//   out[1]  1 if any density is non-finite                   out[8]  density min
//   out[2]  1 if any pressure is non-finite                  out[9]  density max
//   out[3]  speed max (float32 |v| as numpy.linalg.norm)     out[10] k-th smallest density
//   out[4]  height mean (z)                                  out[11] (k+1)-th smallest density
//   out[5]  height min                                       out[12] pressure min
//   out[6]  height max                                       out[13] pressure max
//
// Minima and maxima are exact (ordered-integer atomics on float bits);
// means add per-block partial sums in a fixed order (double precision,
// deterministic).  The two order statistics come from a radix select over
// the order-preserving 32-bit keys of the densities (four passes of 8-bit
// digits), from which the host interpolates the percentile as numpy does.
#include "fs_internal.cuh"

namespace fs {
namespace {

constexpr int kMetricBlock = 256;

// order-preserving map of float bits to unsigned keys (and back)
FS_DEV uint32_t fkey(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
FS_DEV float funkey(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }

struct MetricsAcc {
  uint32_t speed_max;          // key
  uint32_t zmin, zmax;         // keys
  uint32_t rmin, rmax;         // keys
  uint32_t pmin, pmax;         // keys
  int32_t bad_state, bad_rho, bad_p;
  uint32_t sel_prefix[2];      // radix select: digits fixed so far (high bits)
  int64_t sel_rank[2];         // rank still to find inside the prefix
  int32_t hist[2][256];
};

__global__ void k_metrics_init(MetricsAcc* a, int64_t k, int64_t nr) {
  if (threadIdx.x == 0) {
    a->speed_max = fkey(0.f);
    a->zmin = a->rmin = a->pmin = 0xffffffffu;
    a->zmax = a->rmax = a->pmax = 0u;
    a->bad_state = a->bad_rho = a->bad_p = 0;
    a->sel_prefix[0] = a->sel_prefix[1] = 0u;
    a->sel_rank[0] = k;
    a->sel_rank[1] = k + 1 < nr ? k + 1 : k;  // numpy takes the last value twice at the top
  }
  for (int i = threadIdx.x; i < 512; i += blockDim.x) (&a->hist[0][0])[i] = 0;
}

template <class Op>
FS_DEV uint32_t block_reduce_u32(uint32_t v, Op op) {
  __shared__ uint32_t sm[kMetricBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < kMetricBlock / 32 ? sm[threadIdx.x] : sm[0];
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  return v;
}

FS_DEV double block_sum(double v) {
  __shared__ double sm[kMetricBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kMetricBlock / 32; ++w) r += sm[w];
  __syncthreads();
  return r;
}

struct UMax {
  FS_DEV uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};
struct UMin {
  FS_DEV uint32_t operator()(uint32_t a, uint32_t b) const { return a < b ? a : b; }
};

__global__ void __launch_bounds__(kMetricBlock) k_metrics_main(const float* __restrict__ x, const float* __restrict__ v,
                                                               int64_t n, const float* __restrict__ rho,
                                                               const float* __restrict__ pr, int64_t nr,
                                                               MetricsAcc* acc, double* part_z, double* part_r) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t sp = fkey(0.f), zmin = 0xffffffffu, zmax = 0u, rmin = 0xffffffffu, rmax = 0u, pmin = 0xffffffffu,
           pmax = 0u;
  double sz = 0.0, sr = 0.0;
  int bad_s = 0, bad_r = 0, bad_p = 0;
  if (i < n) {
    const float3 p = ld3(x, i), u = ld3(v, i);
    bad_s = !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(u.x) && isfinite(u.y) && isfinite(u.z));
    // numpy.linalg.norm of a float32 row: sqrt((vx^2 + vy^2) + vz^2), each op rounded
    const float s2 = __fadd_rn(__fadd_rn(__fmul_rn(u.x, u.x), __fmul_rn(u.y, u.y)), __fmul_rn(u.z, u.z));
    sp = fkey(__fsqrt_rn(s2));
    zmin = zmax = fkey(p.z);
    sz = (double)p.z;
  }
  if (i < nr) {
    const float r = rho[i];
    bad_r = !isfinite(r);
    rmin = rmax = fkey(r);
    sr = (double)r;
    if (pr) {
      const float q = pr[i];
      bad_p = !isfinite(q);
      pmin = pmax = fkey(q);
    }
  }
  sp = block_reduce_u32(sp, UMax());
  zmin = block_reduce_u32(zmin, UMin());
  zmax = block_reduce_u32(zmax, UMax());
  rmin = block_reduce_u32(rmin, UMin());
  rmax = block_reduce_u32(rmax, UMax());
  pmin = block_reduce_u32(pmin, UMin());
  pmax = block_reduce_u32(pmax, UMax());
  const double bz = block_sum(sz), br = block_sum(sr);
  const int any_s = __syncthreads_or(bad_s), any_r = __syncthreads_or(bad_r), any_p = __syncthreads_or(bad_p);
  if (threadIdx.x == 0) {
    atomicMax(&acc->speed_max, sp);
    atomicMin(&acc->zmin, zmin);
    atomicMax(&acc->zmax, zmax);
    atomicMin(&acc->rmin, rmin);
    atomicMax(&acc->rmax, rmax);
    atomicMin(&acc->pmin, pmin);
    atomicMax(&acc->pmax, pmax);
    if (any_s) atomicOr(&acc->bad_state, 1);
    if (any_r) atomicOr(&acc->bad_rho, 1);
    if (any_p) atomicOr(&acc->bad_p, 1);
    part_z[blockIdx.x] = bz;
    part_r[blockIdx.x] = br;
  }
}

// Histogram of digit `pass` (8 bits, most significant first) of the keys
// that match the prefix fixed so far, for both order statistics.
__global__ void __launch_bounds__(kMetricBlock) k_select_hist(const float* __restrict__ rho, int64_t nr, int pass,
                                                              MetricsAcc* acc) {
  __shared__ int32_t h[2][256];
  for (int t = threadIdx.x; t < 512; t += blockDim.x) (&h[0][0])[t] = 0;
  __syncthreads();
  const int shift = 24 - 8 * pass;
  const uint32_t mask = pass == 0 ? 0u : (0xffffffffu << (32 - 8 * pass));
  const uint32_t pre0 = acc->sel_prefix[0], pre1 = acc->sel_prefix[1];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = fkey(rho[i]);
    const int d = (k >> shift) & 0xff;
    if ((k & mask) == pre0) atomicAdd(&h[0][d], 1);
    if ((k & mask) == pre1) atomicAdd(&h[1][d], 1);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 512; t += blockDim.x) {
    const int c = (&h[0][0])[t];
    if (c) atomicAdd(&(&acc->hist[0][0])[t], c);
  }
}

// Picks the digit whose bin holds the wanted rank, narrows the prefix, and
// clears the histogram for the next pass.
__global__ void k_select_pick(int pass, MetricsAcc* acc) {
  const int shift = 24 - 8 * pass;
  if (threadIdx.x < 2) {
    const int q = threadIdx.x;
    int64_t r = acc->sel_rank[q];
    int d = 0;
    for (; d < 255; ++d) {
      const int c = acc->hist[q][d];
      if (r < c) break;
      r -= c;
    }
    acc->sel_rank[q] = r;
    acc->sel_prefix[q] |= (uint32_t)d << shift;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 512; t += blockDim.x) (&acc->hist[0][0])[t] = 0;
}

__global__ void k_metrics_final(const MetricsAcc* acc, const double* part_z, const double* part_r, int nblk,
                                int64_t n, int64_t nr, int has_p, double* out) {
  if (threadIdx.x != 0) return;
  double sz = 0.0, sr = 0.0;
  for (int b = 0; b < nblk; ++b) {
    sz += part_z[b];
    sr += part_r[b];
  }
  out[0] = acc->bad_state ? 1.0 : 0.0;
  out[1] = acc->bad_rho ? 1.0 : 0.0;
  out[2] = acc->bad_p ? 1.0 : 0.0;
  out[3] = n > 0 ? (double)funkey(acc->speed_max) : 0.0;
  out[4] = n > 0 ? sz / (double)n : 0.0;
  out[5] = n > 0 ? (double)funkey(acc->zmin) : 0.0;
  out[6] = n > 0 ? (double)funkey(acc->zmax) : 0.0;
  out[7] = nr > 0 ? sr / (double)nr : 0.0;
  out[8] = nr > 0 ? (double)funkey(acc->rmin) : 0.0;
  out[9] = nr > 0 ? (double)funkey(acc->rmax) : 0.0;
  out[10] = nr > 0 ? (double)funkey(acc->sel_prefix[0]) : 0.0;
  out[11] = nr > 0 ? (double)funkey(acc->sel_prefix[1]) : 0.0;
  out[12] = nr > 0 && has_p ? (double)funkey(acc->pmin) : 0.0;
  out[13] = nr > 0 && has_p ? (double)funkey(acc->pmax) : 0.0;
}

}  // namespace

size_t metrics_scratch_bytes(int64_t capacity) {
  const int64_t nb = (capacity + kMetricBlock - 1) / kMetricBlock + 1;
  return sizeof(MetricsAcc) + 2 * sizeof(double) * (size_t)nb + 256;
}

}  // namespace fs

using namespace fs;

extern "C" {

int fs_frame_metrics(fs_context* c, const float* x, const float* v, int64_t n, const float* rho,
                     const float* pressure, int64_t nrho, int64_t k, double* out, fs_stream_t stream) {
  if (!c || !out || n < 0 || nrho < 0 || (n > 0 && (!x || !v)) || (nrho > 0 && !rho))
    return set_error(FS_ERR_INVALID, "fs_frame_metrics: bad arguments");
  if (n > c->capacity || nrho > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_frame_metrics: n > capacity");
  if (nrho > 0 && (k < 0 || k >= nrho))
    return set_error(FS_ERR_INVALID, "fs_frame_metrics: rank k=%lld outside [0, %lld)", (long long)k,
                     (long long)nrho);
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  MetricsAcc* acc = (MetricsAcc*)c->metrics;
  const int64_t m = n > nrho ? n : nrho;
  const int nb = (int)((m + kMetricBlock - 1) / kMetricBlock);
  double* part_z = (double*)(acc + 1);
  double* part_r = part_z + (nb > 0 ? nb : 1);
  PassScope ps_(c, P_OTHER, st, 4 + (nrho > 0 ? 8 : 0));
  k_metrics_init<<<1, 256, 0, st>>>(acc, k, nrho);
  if (nb > 0)
    k_metrics_main<<<nb, kMetricBlock, 0, st>>>(x, v, n, rho, pressure, nrho, acc, part_z, part_r);
  if (nrho > 0) {
    const int sb = (int)((nrho + kMetricBlock - 1) / kMetricBlock) < 4 * 148
                       ? (int)((nrho + kMetricBlock - 1) / kMetricBlock)
                       : 4 * 148;
    for (int pass = 0; pass < 4; ++pass) {
      k_select_hist<<<sb, kMetricBlock, 0, st>>>(rho, nrho, pass, acc);
      k_select_pick<<<1, 256, 0, st>>>(pass, acc);
    }
  }
  k_metrics_final<<<1, 32, 0, st>>>(acc, part_z, part_r, nb, n, nrho, pressure ? 1 : 0, out);
  return launch_check("fs_frame_metrics");
}

}  // extern "C"
