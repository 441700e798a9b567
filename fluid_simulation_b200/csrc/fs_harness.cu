// Harness reductions of the dam-break driver (examples/dam_break/simulation.py):
//   particle_norm_maxima (19-36): max |v|^2 and max |a|^2 for the CFL rule,
//     a non-finite vector counts as +inf
//   check_particle_finite (39-53): one flag if any x, v or density is non-finite
// Both reduce per block first and issue one atomic per block.
#include "fs_internal.cuh"

namespace fs {
namespace {

FS_DEV float sq_or_inf(float3 a) {
  const float s = a.x * a.x + a.y * a.y + a.z * a.z;
  const bool ok = isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(s);
  return ok ? s : __int_as_float(0x7f800000);
}

FS_DEV float block_max(float v) {
  __shared__ float sm[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.f;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmaxf(r, sm[w]);
  __syncthreads();
  return r;
}

// out[0] = max |v|^2 over nv, out[1] = max |a|^2 over na (both >= 0, inf if
// any non-finite); out must be zeroed first.  Non-negative floats order like
// their bit patterns, so the cross-block maximum is an integer atomicMax.
__global__ void k_norm_maxima(const float* __restrict__ v, int64_t nv, const float* __restrict__ a, int64_t na,
                              float* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float sv = i < nv ? sq_or_inf(ld3(v, i)) : 0.f;
  const float sa = i < na ? sq_or_inf(ld3(a, i)) : 0.f;
  const float bv = block_max(sv);
  const float ba = block_max(sa);
  if (threadIdx.x == 0) {
    atomicMax((int*)out, __float_as_int(bv));
    atomicMax((int*)out + 1, __float_as_int(ba));
  }
}

__global__ void k_check_finite(const float* __restrict__ x, const float* __restrict__ v, int64_t n,
                               const float* __restrict__ rho, int64_t nrho, int32_t* invalid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (i < n) {
    const float3 p = ld3(x, i), u = ld3(v, i);
    bad = !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(u.x) && isfinite(u.y) && isfinite(u.z));
    if (i < nrho) bad = bad || !isfinite(rho[i]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicMax(invalid, 1);
}

__global__ void k_clock_start(fs_frame_clock* c, double frame_dt) {
  c->remaining = frame_dt;
  c->substeps = 0;
  c->active = frame_dt > 1.0e-12 ? 1 : 0;
  c->dt = 0.f;
}

// The harness's substep rule (simulation.py:167-182 and the loop of
// 185-196) on the device, in double precision as the Python harness
// evaluates it; maxima[] were just reduced from the current state.
__global__ void k_clock_rule(fs_frame_clock* c, fs_cfl_rule r) {
  if (c->fault) {
    c->active = 0;
    return;
  }
  if (!(c->remaining > 1.0e-12)) {
    c->active = 0;
    c->dt = 0.f;
    return;
  }
  const bool use_acc = r.method == 0 && r.use_accel && c->run_substeps > 0;
  const float v2 = c->maxima[0], a2 = use_acc ? c->maxima[1] : 0.f;
  if (!isfinite(v2) || !isfinite(a2)) {
    c->fault |= 1;
    c->active = 0;
    return;
  }
  const double speed = sqrt((double)v2), accel = sqrt((double)a2);
  double limit = r.substep_limit;
  if (r.method == 0) {
    limit = fmin(limit, 0.25 * r.h / (r.sound_speed + speed));
    if (accel > 0.0) limit = fmin(limit, 0.25 * sqrt(r.h / accel));
    if (r.viscosity > 0.0) limit = fmin(limit, 0.025 * r.h * r.h / r.viscosity);
  } else if (speed > 0.0) {
    limit = fmin(limit, 0.4 * r.spacing / speed);
  }
  const double dt = fmin(c->remaining, limit);
  if (dt < 1.0e-10) {
    c->fault |= 2;
    c->active = 0;
    return;
  }
  c->dt = (float)dt;
  c->active = 1;
  c->remaining -= dt;
  c->substeps += 1;
  c->run_substeps += 1;
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

int fs_norm_maxima(const float* v, int64_t nv, const float* a, int64_t na, float* out, fs_stream_t stream) {
  if (!out || nv < 0 || na < 0 || (nv > 0 && !v) || (na > 0 && !a))
    return set_error(FS_ERR_INVALID, "fs_norm_maxima: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = check_cuda(cudaMemsetAsync(out, 0, 2 * sizeof(float), st), "fs_norm_maxima: memset");
  if (rc) return rc;
  const int64_t m = nv > na ? nv : na;
  if (m == 0) return FS_OK;
  k_norm_maxima<<<blocks_for(m), kBlock, 0, st>>>(v, nv, a, na, out);
  return launch_check("fs_norm_maxima");
}

int fs_check_finite(const float* x, const float* v, int64_t n, const float* rho, int64_t nrho, int32_t* invalid,
                    fs_stream_t stream) {
  if (!invalid || n < 0 || nrho < 0 || (n > 0 && (!x || !v)) || (nrho > 0 && !rho))
    return set_error(FS_ERR_INVALID, "fs_check_finite: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = check_cuda(cudaMemsetAsync(invalid, 0, sizeof(int32_t), st), "fs_check_finite: memset");
  if (rc) return rc;
  if (n == 0) return FS_OK;
  k_check_finite<<<blocks_for(n), kBlock, 0, st>>>(x, v, n, rho, nrho, invalid);
  return launch_check("fs_check_finite");
}

int fs_frame_clock_start(fs_frame_clock* clock, double frame_dt, fs_stream_t stream) {
  if (!clock || !(frame_dt >= 0.0)) return set_error(FS_ERR_INVALID, "fs_frame_clock_start: bad arguments");
  k_clock_start<<<1, 1, 0, (cudaStream_t)stream>>>(clock, frame_dt);
  return launch_check("fs_frame_clock_start");
}

int fs_frame_clock_advance(fs_frame_clock* clock, const fs_cfl_rule* rule, const float* v, int64_t nv,
                           const float* accel, int64_t na, fs_stream_t stream) {
  if (!clock || !rule || nv < 0 || na < 0 || (nv > 0 && !v) || (na > 0 && !accel) ||
      (rule->method != 0 && rule->method != 1))
    return set_error(FS_ERR_INVALID, "fs_frame_clock_advance: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = check_cuda(cudaMemsetAsync(clock->maxima, 0, sizeof(clock->maxima), st), "fs_frame_clock_advance: memset");
  if (rc) return rc;
  const int64_t m = nv > na ? nv : na;
  if (m > 0) k_norm_maxima<<<blocks_for(m), kBlock, 0, st>>>(v, nv, accel, na, clock->maxima);
  k_clock_rule<<<1, 1, 0, st>>>(clock, *rule);
  return launch_check("fs_frame_clock_advance");
}

}  // extern "C"
