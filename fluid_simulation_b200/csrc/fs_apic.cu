// APIC particle separation on B200 (replaces the neighbour pass of
// SolverAPIC._apply_particle_separation, solver_apic.py:1003-1064, with its
// kernels accumulate_particle_separation, 193-248, and
// apply_particle_separation_delta, 251-266).
//
// Per iteration: the hash grid of the context (dims chosen by the caller as
// the reference does: the bounds' extent over the query radius, at least 4)
// is built over the current positions with cell width query_radius, the
// positions are gathered into cell order, one thread per cell-sorted slot
// averages the pushes of its active neighbours closer than rest_dist in the
// reference's visiting order, and a per-particle pass adds the push and
// clamps to the bounds inset by wall_margin.  The pair arithmetic uses
// individually rounded operations (no contraction into FMAs), as the
// reference's float32 expression does, so the result equals the reference's
// bit for bit.
#include "fs_internal.cuh"

namespace fs {
namespace {

// positions (original order) into cell order, with the active bit in .w
__global__ void k_sep_gather(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ x,
                             const int32_t* __restrict__ flags, float4* __restrict__ xs) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = perm[s];
  const float3 p = ld3(x, i);
  xs[s] = make_float4(p.x, p.y, p.z, pack_pf((flags[i] & 1) ? PF_ACTIVE : 0));
}

struct SepArgs {
  GridDev g;
  int64_t n;
  const float4* xs;
  float rest, qr, strength, band;
  float lo[3], hi[3];
  float* delta;  // original order [n][3]
};

// accumulate_particle_separation
__global__ void k_sep_accumulate(SepArgs a) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const float4 xi = a.xs[s];
  const int32_t i = a.g.perm[s];
  if (!(pf_of(xi) & PF_ACTIVE)) {
    st3(a.delta, i, make_float3(0.f, 0.f, 0.f));
    return;
  }
  float dx_ = 0.f, dy_ = 0.f, dz_ = 0.f, count = 0.f;
  // d2 above rest^2 (1 + 1e-6) gives a rounded sqrt(d2) >= rest (at least
  // ~3 ulps above it), which the test d < rest rejects: only the remaining
  // candidates pay for the correctly rounded square root
  const float r2lim = __fmul_rn(__fmul_rn(a.rest, a.rest), 1.000001f);
  for_each_range(a.g, 0, xi.x, xi.y, xi.z, a.qr, [&](int b, int e) {
    for (int t = b; t < e; ++t) {
      const float4 xj = __ldg(a.xs + t);
      if (t == (int)s || !(pf_of(xj) & PF_ACTIVE)) continue;
      const float rx = __fsub_rn(xi.x, xj.x), ry = __fsub_rn(xi.y, xj.y), rz = __fsub_rn(xi.z, xj.z);
      const float d2 = dist2_rn(rx, ry, rz);
      if (!(d2 <= r2lim)) continue;
      const float d = __fsqrt_rn(d2);
      if (d > 1.0e-8f && d < a.rest) {
        const float w = __fmul_rn(a.strength, __fsub_rn(a.rest, d));
        dx_ = __fadd_rn(dx_, __fmul_rn(__fdiv_rn(rx, d), w));
        dy_ = __fadd_rn(dy_, __fmul_rn(__fdiv_rn(ry, d), w));
        dz_ = __fadd_rn(dz_, __fmul_rn(__fdiv_rn(rz, d), w));
        count = __fadd_rn(count, 1.0f);
      }
    }
  });
  if (count > 0.f) {
    dx_ = __fdiv_rn(dx_, count);
    dy_ = __fdiv_rn(dy_, count);
    dz_ = __fdiv_rn(dz_, count);
  } else {
    dx_ = dy_ = dz_ = 0.f;
  }
  // components that push into a wall within the band are removed
  if (xi.x <= __fadd_rn(a.lo[0], a.band) && dx_ < 0.f) dx_ = 0.f;
  if (xi.x >= __fsub_rn(a.hi[0], a.band) && dx_ > 0.f) dx_ = 0.f;
  if (xi.y <= __fadd_rn(a.lo[1], a.band) && dy_ < 0.f) dy_ = 0.f;
  if (xi.y >= __fsub_rn(a.hi[1], a.band) && dy_ > 0.f) dy_ = 0.f;
  if (xi.z <= __fadd_rn(a.lo[2], a.band) && dz_ < 0.f) dz_ = 0.f;
  if (xi.z >= __fsub_rn(a.hi[2], a.band) && dz_ > 0.f) dz_ = 0.f;
  st3(a.delta, i, make_float3(dx_, dy_, dz_));
}

FS_DEV float clamp_ref(float v, float lo, float hi) {  // min(max(v, lo), hi) with the reference's comparisons
  const float t = v > lo ? v : lo;
  return t < hi ? t : hi;
}

// apply_particle_separation_delta
__global__ void k_sep_apply(int64_t n, const int32_t* __restrict__ flags, const float* __restrict__ delta, float lox,
                            float loy, float loz, float hix, float hiy, float hiz, float* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(flags[i] & 1)) return;
  const float3 p = ld3(x, i), d = ld3(delta, i);
  st3(x, i, make_float3(clamp_ref(__fadd_rn(p.x, d.x), lox, hix), clamp_ref(__fadd_rn(p.y, d.y), loy, hiy),
                        clamp_ref(__fadd_rn(p.z, d.z), loz, hiz)));
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

int fs_apic_separation(fs_context* c, float* x, const int32_t* flags, int64_t n, const fs_separation_params* p,
                       float* delta, fs_stream_t stream) {
  if (!c || !p) return set_error(FS_ERR_INVALID, "fs_apic_separation: null argument");
  if (n < 0) return set_error(FS_ERR_INVALID, "fs_apic_separation: negative n");
  if (n == 0) return FS_OK;
  if (!x || !flags || !delta) return set_error(FS_ERR_INVALID, "fs_apic_separation: missing array");
  if (c->worlds) return set_error(FS_ERR_INVALID, "fs_apic_separation: needs a hash-grid context");
  if (n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_apic_separation: n > capacity");
  if (!(p->query_radius > 0.f)) return set_error(FS_ERR_INVALID, "fs_apic_separation: query_radius must be > 0");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int iters = p->iterations > 1 ? p->iterations : 1;
  // bounds inset by the wall margin (apply_particle_separation_delta, 263-264)
  const float lox = p->bound_lo[0] + p->wall_margin, loy = p->bound_lo[1] + p->wall_margin,
              loz = p->bound_lo[2] + p->wall_margin;
  const float hix = p->bound_hi[0] - p->wall_margin, hiy = p->bound_hi[1] - p->wall_margin,
              hiz = p->bound_hi[2] - p->wall_margin;
  int rc;
  for (int it = 0; it < iters; ++it) {
    if ((rc = grid_build(c, x, n, p->query_radius, st, nullptr))) return rc;
    {
      PassScope ps_(c, P_GATHER, st);
      k_sep_gather<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, x, flags, c->xs);
    }
    SepArgs a;
    a.g = grid_view(c);
    a.n = n;
    a.xs = c->xs;
    a.rest = p->rest_dist;
    a.qr = p->query_radius;
    a.strength = p->strength;
    a.band = p->wall_band;
    for (int k = 0; k < 3; ++k) {
      a.lo[k] = p->bound_lo[k];
      a.hi[k] = p->bound_hi[k];
    }
    a.delta = delta;
    {
      PassScope ps_(c, P_APIC_SEPARATION, st, 2);
      k_sep_accumulate<<<blocks_for(n), kBlock, 0, st>>>(a);
      k_sep_apply<<<blocks_for(n), kBlock, 0, st>>>(n, flags, delta, lox, loy, loz, hix, hiy, hiz, x);
    }
    if ((rc = launch_check("fs_apic_separation"))) return rc;
  }
  c->last_stream = st;
  return FS_OK;
}

}  // extern "C"
