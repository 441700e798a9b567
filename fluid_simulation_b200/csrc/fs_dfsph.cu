// DFSPH substep on B200 (replaces SolverDFSPH.step, solver_dfsph.py:598-898).
//
// The reference reads the residual back to the host once per solver
// iteration (solver_dfsph.py:733, 849).  Here each iteration is a pair of
// launches whose decision stays on the device:
//   rate    : d_rho_dt (+ rho_star) + the candidate kappa of every particle +
//             a deterministic residual reduction; its last block stores the
//             residual and sets `done` when it > 0 and residual <= eta
//   correct : if !done, commit kappa and apply the velocity correction
// Launches of iterations after the break see `done` and return at once, so
// the whole step is launch-only (graph capturable) and takes exactly the
// reference's decisions.
//
// Batched contexts (independent scenes, one world each) take the decisions
// per world: the rate pass stores each dynamic particle's residual term per
// slot (-1 marks a non-dynamic one), a segmented pass with one block per
// world (its slots are contiguous in cell order) sums them in a fixed order
// and sets that world's `done`; the rate and correction passes skip the
// particles of finished worlds, and every kernel returns at once when all
// worlds are done.  Each scene iterates exactly as it would alone.
#include <algorithm>

#include "fs_nbr.cuh"

namespace fs {

// Partial-sum slots for the residual reductions: one per block of the
// smallest block size that launches them (the 64-thread floor leaves room for
// any block size used here).
int reduction_blocks(int64_t n) { return blocks_for(n > 0 ? n : 1, 64); }

// gather of fs_wcsph.cu reused here
__global__ void k_gather_common(int64_t n, const int32_t* __restrict__ perm, fs_model m, const float* __restrict__ x,
                                const float* __restrict__ v, float4* __restrict__ xs, float4* __restrict__ vs,
                                float* __restrict__ mv, uint32_t* status, int nworlds);

namespace {

// xyz of a cell-order float4 stream into an original-order [n][3] array
__global__ void k_scatter_xyz(int64_t n, const int32_t* __restrict__ perm, const float4* __restrict__ in,
                              float* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) st3(out, perm[s], xyz(in[s]));
}

// (a[i], b[i]) of original order into cell order
__global__ void k_gather_pair(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ a,
                              const float* __restrict__ b, float2* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = perm[s];
  out[s] = make_float2(a[i], b ? b[i] : 0.f);
}

__global__ void k_gather_scalar(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ a,
                                float* __restrict__ out, float* __restrict__ copy_to) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = perm[s];
  const float v = a[i];
  out[s] = v;
  if (copy_to) copy_to[i] = v;
}

// compute_density (107-133) + compute_factor_dfsph (137-174), one candidate loop.
struct DensFactorArgs {
  GridDev g;
  NbrList L;
  int64_t n;
  const float4* xs;
  const float4* vs;  // .w = mass
  const float* mv;
  float h;
  int min_nb;
  float* rho;
  float* factor;
  int32_t* count;
  float2* sc2;       // (rho, factor) cell order
  const fs_frame_clock* clock;  // clocked substep: nothing to do once the frame is complete
};

// Records the neighbour lists of this grid (positions stay fixed for the half
// step, so every later pass of the half reuses them exactly).
// 64-register budget (4 resident 256-thread blocks): the compiler's own
// choice was 48 registers with 52 bytes of spills; 0.306 -> 0.287 ms per
// launch at 401,856 particles
__global__ void __launch_bounds__(kNbBlockMax, 4) k_density_factor(DensFactorArgs a) {
  if (clock_idle(a.clock)) return;
  lists_recorded(a.L);
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_ACTIVE)) {
      a.rho[i] = 0.f;
      a.factor[i] = 0.f;
      a.count[i] = 0;
      a.sc2[s] = make_float2(0.f, 0.f);
      a.L.cnt[s] = 0;
      return;
    }
    const float h2m = a.h * a.h * kSupportMargin;
    // the candidate count (no distance test, solver_dfsph.py:163-164) comes from the scan
    const int cnt = record_list<true>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L);
    const Cubic K(a.h);
    float rho = 0.f, sgx = 0.f, sgy = 0.f, sgz = 0.f, sq = 0.f;
    visit_with<true, true>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L, true,
                           [&](int t) { return make_float2(__ldg(a.mv + t), __ldg(&a.vs[t].w)); },
                           [&](int t, float4 xj, const float2& mm) {  // (rest_density * volume, mass)
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      float r, rinv;
      r_and_inv(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), r, rinv);
      rho = fmaf(mm.x, K.w(r), rho);
      const float gsc = mm.y * K.grad_scale(r, rinv);
      const float gx = gsc * dx, gy = gsc * dy, gz = gsc * dz;
      sgx += gx;
      sgy += gy;
      sgz += gz;
      sq = fmaf(gx, gx, fmaf(gy, gy, fmaf(gz, gz, sq)));
    });
    const float denom = (sgx * sgx + sgy * sgy + sgz * sgz) + sq;
    const float f = (cnt < a.min_nb || denom < 1.0e-6f) ? 0.f : 1.0f / denom;
    a.rho[i] = rho;
    a.factor[i] = f;
    a.count[i] = cnt;
    a.sc2[s] = make_float2(rho, f);
  });
}

// acceleration_non_pressure (178-226) + predict_velocity (230-242).
struct AccelArgs {
  GridDev g;
  NbrList L;
  int use_lists;
  int64_t n;
  const float4* xs;
  const float4* vs;
  const float2* sc2;
  fs_model m;
  float h, particle_radius, dt;
  float* accel;
  float4* vstar;     // cell order (v*, mass)
  const fs_frame_clock* clock;
};

__global__ void FS_NB_BOUNDS k_accel_predict(AccelArgs a) {
  if (clock_idle(a.clock)) return;
  const float dt = a.clock ? a.clock->dt : a.dt;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const float4 vi = a.vs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_DYNAMIC)) {
      st3(a.accel, i, make_float3(0.f, 0.f, 0.f));
      a.vstar[s] = make_float4(0.f, 0.f, 0.f, vi.w);
      return;
    }
    const float mu10 = 10.f * a.m.viscosity[i];
    const float coh = a.m.surface_tension[i] / vi.w;
    const float visc_den_add = 0.01f * (a.h * a.h);
    const Cubic K(a.h);
    float ax = 0.f, ay = 0.f, az = 0.f;
    const bool lists_ok = a.use_lists && lists_usable(a.L);
    visit<false, false>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                        [&](int t, float4 xj) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (r2 == 0.f) return;  // zero vector d: every term vanishes
      const float4 vj = __ldg(a.vs + t);
      const float rho_j = __ldg(&a.sc2[t].x);
      float r, rinv;
      r_and_inv(r2, r, rinv);
      const float wc = coh * vj.w * K.w(fmaxf(r, a.particle_radius));
      const float vdot = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
      const float visc = mu10 * __fdividef(vj.w, fmaxf(rho_j, 1.0e-6f)) * __fdividef(vdot, r2 + visc_den_add);
      const float c = fmaf(visc, K.grad_scale(r, rinv), -wc);
      ax = fmaf(c, dx, ax);
      ay = fmaf(c, dy, ay);
      az = fmaf(c, dz, az);
    });
    const float3 g = gravity_of(a.m, i);
    const float3 acc = make_float3(ax + g.x, ay + g.y, az + g.z);
    st3(a.accel, i, acc);
    a.vstar[s] = make_float4(vi.x + dt * acc.x, vi.y + dt * acc.y, vi.z + dt * acc.z, vi.w);
  });
}

// ---------------------------------------------------- rate + residual ----
// compute_density_change_rate (246-272), then per mode:
//   mode 0 (density):    predict_density_star (276-287) and compute_kappa_density (291-306)
//   mode 1 (divergence): compute_kappa_divergence (357-372)
// and the residual of _density_residual / _divergence_residual (579-596).
struct RateArgs {
  GridDev g;
  int64_t n;
  const float4* xs;
  const float4* vstar;      // (v*, mass)
  const float2* sc2;        // (rho, factor)
  const float* rest_density;
  float h, dt, max_kappa, eta;
  int mode, it;
  float* d_rho_dt;          // API
  float* rho_star;          // API (mode 0)
  float* kappa_new;         // cell order candidate kappa
  float2* kratio_new;       // cell order (kappa / max(rho, 1e-6), mass): what the correction gathers per neighbour
  NbrList L;
  int use_lists;
  DfsphDev* ctrl;           // null: separate-pass use, no residual
  double* red_part;
  int64_t* red_cnt;
  const fs_frame_clock* clock;
  const DfsphWorld* wctl;   // batched decisions ([nworlds]) or null
  const int32_t* pworld;    // particle_world (batched)
  int nworlds;
  float* term;              // batched: per-slot residual term, -1 = not dynamic
};

// A particle of a world whose iterations have ended (batched contexts).
FS_DEV bool world_finished(const DfsphWorld* wctl, const int32_t* pworld, int nworlds, int32_t i) {
  return wctl && wctl[world_index(pworld[i], nworlds)].done;
}

__device__ void residual_finish(DfsphDev* ctrl, const double* part, const int64_t* cntp, int nblk, int it,
                                float eta) {
  // fixed-order sum over block partials: deterministic
  __shared__ double sd[kBlock / 32];
  __shared__ long long sc[kBlock / 32];
  // four partial sums per thread keep four loads in flight; they combine in
  // a fixed order, so the result does not depend on timing
  const int step = (int)blockDim.x;
  double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
  long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
  int b = threadIdx.x;
  for (; b + 3 * step < nblk; b += 4 * step) {
    v0 += __ldcg(part + b);
    v1 += __ldcg(part + b + step);
    v2 += __ldcg(part + b + 2 * step);
    v3 += __ldcg(part + b + 3 * step);
    c0 += __ldcg((const long long*)cntp + b);
    c1 += __ldcg((const long long*)cntp + b + step);
    c2 += __ldcg((const long long*)cntp + b + 2 * step);
    c3 += __ldcg((const long long*)cntp + b + 3 * step);
  }
  for (; b < nblk; b += step) {
    v0 += __ldcg(part + b);
    c0 += __ldcg((const long long*)cntp + b);
  }
  double v = (v0 + v1) + (v2 + v3);
  long long c = (c0 + c1) + (c2 + c3);
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sd[threadIdx.x >> 5] = v;
    sc[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    long long cn = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      tot += sd[w];
      cn += sc[w];
    }
    const double res = cn > 0 ? tot / (double)cn : 0.0;
    ctrl->residual = res;
    ctrl->iters = it + 1;
    if (it > 0 && res <= (double)eta) ctrl->done = 1;
    ctrl->ticket = 0;
  }
}

__device__ void block_reduce_store(double v, long long c, double* part, int64_t* cntp) {
  __shared__ double sd[kBlock / 32];
  __shared__ long long sc[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sd[threadIdx.x >> 5] = v;
    sc[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    long long cn = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      tot += sd[w];
      cn += sc[w];
    }
    part[blockIdx.x] = tot;
    cntp[blockIdx.x] = cn;
  }
}

// last-block-done: returns true in exactly one block, after every block's partial is visible
__device__ bool last_block(uint32_t* ticket) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (am_last) __threadfence();
  return am_last;
}

__global__ void FS_NB_BOUNDS k_rate(RateArgs a) {
  if (a.ctrl && a.ctrl->done) return;  // uniform across the grid: set by an earlier launch
  if (clock_idle(a.clock)) return;     // uniform: the frame is complete
  const float dt = a.clock ? a.clock->dt : a.dt;
  double term = 0.0;  // this thread's residual terms and dynamic particles
  long long dyn = 0;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (world_finished(a.wctl, a.pworld, a.nworlds, i)) return;
    const int pf = pf_of(xi);
    float d = 0.f;
    if (pf & PF_ACTIVE) {
      const float4 vi = a.vstar[s];
      const Cubic K(a.h);
      const bool lists_ok = a.use_lists && lists_usable(a.L);
      visit_with<false>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                        [&](int t) { return __ldg(a.vstar + t); }, [&](int t, float4 xj, const float4& vj) {
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        float r, rinv;
        r_and_inv(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), r, rinv);
        const float vdot = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
        d = fmaf(vj.w * K.grad_scale(r, rinv), vdot, d);
      });
    }
    a.d_rho_dt[i] = d;
    const float2 rf = a.sc2[s];
    const bool is_dyn = (pf & PF_DYNAMIC) != 0;
    float kap = 0.f, tv = -1.f;  // tv: this particle's residual term (>= 0) if dynamic
    if (a.mode == 0) {
      const float rs = (pf & PF_ACTIVE) ? rf.x + dt * d : 0.f;
      a.rho_star[i] = rs;
      if (is_dyn) {
        const float err = fmaxf(rs - a.rest_density[i], 0.f);
        kap = fminf((err / (dt * dt)) * rf.y, a.max_kappa);
        tv = err;
      }
    } else if (is_dyn) {
      const float dc = fmaxf(d, 0.f);
      kap = fminf((1.0f / dt) * dc * rf.x * rf.y, a.max_kappa);
      tv = dc;
    }
    if (a.kappa_new) {
      a.kappa_new[s] = kap;
      a.kratio_new[s] = make_float2(kap / fmaxf(rf.x, 1.0e-6f), a.vstar[s].w);
    }
    if (a.term) a.term[s] = tv;
    if (is_dyn) {
      term += (double)tv;
      dyn += 1;
    }
  });
  if (!a.ctrl || a.wctl) return;  // no residual, or the per-world pass takes it
  block_reduce_store(term, dyn, a.red_part, a.red_cnt);
  if (last_block(&a.ctrl->ticket)) residual_finish(a.ctrl, a.red_part, a.red_cnt, gridDim.x, a.it, a.eta);
}

// Batched contexts: the residual of each world (block w sums the terms of
// world w's slots, contiguous in cell order, in a fixed order) and its break
// test (_density_residual / _divergence_residual, 579-596, per scene).
constexpr int kWorldBlock = 512;  // threads per world of the residual pass

__global__ void __launch_bounds__(kWorldBlock) k_world_residual(GridDev g, const float* __restrict__ term,
                                                                DfsphWorld* wctl, DfsphDev* gctl, int it, float eta,
                                                                const fs_frame_clock* clock) {
  if (gctl->done || clock_idle(clock)) return;
  const int w = blockIdx.x;
  DfsphWorld& W = wctl[w];
  if (W.done) return;  // uniform in the block
  const WorldDev& box = g.worlds[w];
  const int32_t s0 = g.off[box.base];
  const int32_t s1 = g.off[box.base + box.dims[0] * box.dims[1] * box.dims[2]];
  double v = 0.0;
  long long c = 0;
  auto add = [&](float t) {
    if (t >= 0.f) {
      v += (double)t;
      c += 1;
    }
  };
  const int32_t step = (int32_t)blockDim.x;
  int32_t s = s0 + (int32_t)threadIdx.x;
  for (; s + 3 * step < s1; s += 4 * step) {  // four loads in flight, summed in slot order
    const float t0 = __ldcg(term + s), t1 = __ldcg(term + s + step), t2 = __ldcg(term + s + 2 * step),
                t3 = __ldcg(term + s + 3 * step);
    add(t0);
    add(t1);
    add(t2);
    add(t3);
  }
  for (; s < s1; s += step) add(__ldcg(term + s));
  __shared__ double sd[kWorldBlock / 32];
  __shared__ long long sc[kWorldBlock / 32];
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sd[threadIdx.x >> 5] = v;
    sc[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    long long cn = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      tot += sd[k];
      cn += sc[k];
    }
    const double res = cn > 0 ? tot / (double)cn : 0.0;
    W.residual = res;
    W.iters = it + 1;
    if (it > 0 && res <= (double)eta) {
      W.done = 1;
      if (atomicAdd(&gctl->worlds_done, 1) + 1 == (int)gridDim.x) gctl->done = 1;
    }
  }
}

// apply_constant_density_correction (310-337) / apply_divergence_free_correction (376-403)
struct CorrectArgs {
  GridDev g;
  int64_t n;
  const float4* xs;
  float4* vstar;          // in/out (own slot only)
  const float* kappa;     // cell order (committed to the API array)
  const float2* kratio;   // cell order (kappa / max(rho, 1e-6), mass): one gather per neighbour
  float h, dt;
  float* kappa_api;       // commit kappa to the API array (may be null)
  float* vstar_api;       // optional original-order v* output
  NbrList L;
  int use_lists;
  const DfsphDev* ctrl;
  const fs_frame_clock* clock;
  const DfsphWorld* wctl;   // batched decisions ([nworlds]) or null
  const int32_t* pworld;
  int nworlds;
};

// Four resident 256-thread blocks per SM: a 64-register budget (the compiler
// otherwise settles at 48 registers and spills; 3.7 % faster measured).
__global__ void __launch_bounds__(kNbBlockMax, 4) k_correct(CorrectArgs a) {
  if (a.ctrl && a.ctrl->done) return;
  if (clock_idle(a.clock)) return;
  const float dt = a.clock ? a.clock->dt : a.dt;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (world_finished(a.wctl, a.pworld, a.nworlds, i)) return;
    if (a.kappa_api) a.kappa_api[i] = a.kappa[s];
    float4 v = a.vstar[s];
    if (pf_of(xi) & PF_DYNAMIC) {
      const Cubic K(a.h);
      const float ci = a.kratio[s].x;
      float dvx = 0.f, dvy = 0.f, dvz = 0.f;
      const bool lists_ok = a.use_lists && lists_usable(a.L);
      visit_with<false>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                        [&](int t) { return __ldg(a.kratio + t); }, [&](int t, float4 xj, const float2& kj) {
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        float r, rinv;
        r_and_inv(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), r, rinv);
        const float c = kj.y * (ci + kj.x) * K.grad_scale(r, rinv);
        dvx = fmaf(c, dx, dvx);
        dvy = fmaf(c, dy, dvy);
        dvz = fmaf(c, dz, dvz);
      });
      v.x = v.x - dt * dvx;
      v.y = v.y - dt * dvy;
      v.z = v.z - dt * dvz;
      a.vstar[s] = v;
    }
    if (a.vstar_api) st3(a.vstar_api, i, xyz(v));
  });
}

// kappa / max(rho, 1e-6) of gathered kappas (warm start, separate pass)
__global__ void k_kappa_ratio(int64_t n, const float* __restrict__ kappa, const float2* __restrict__ sc2,
                              const float4* __restrict__ vm, float2* __restrict__ kratio) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) kratio[s] = make_float2(kappa[s] / fmaxf(sc2[s].x, 1.0e-6f), vm[s].w);
}

// integrate_positions (341-353); also publishes v* in original order.
__global__ void k_integrate(int64_t n, const int32_t* __restrict__ perm, const float4* __restrict__ xs,
                            const float4* __restrict__ vstar, float dt, float* x_out, float* vstar_api,
                            const fs_frame_clock* clock) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || clock_idle(clock)) return;
  if (clock) dt = clock->dt;
  const float4 xi = xs[s];
  const float4 v = vstar[s];
  const int32_t i = perm[s];
  float3 p = xyz(xi);
  if (pf_of(xi) & PF_DYNAMIC) p = make_float3(xi.x + v.x * dt, xi.y + v.y * dt, xi.z + v.z * dt);
  st3(x_out, i, p);
  st3(vstar_api, i, xyz(v));
}

// copy v* -> particle_qd then apply_bounds (407-442, unconditional damping);
// batched contexts apply each world's own tank.
__global__ void k_final(int64_t n, GridDev g, const float4* __restrict__ xs, const float4* __restrict__ vstar,
                        Walls walls, float* x_out, float* v_out, float* vstar_api, const fs_frame_clock* clock) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || clock_idle(clock)) return;
  const float4 xi = xs[s];
  const float4 v4 = vstar[s];
  const int32_t i = g.perm[s];
  float3 p = xyz(xi), v = xyz(v4);
  st3(vstar_api, i, v);
  if (pf_of(xi) & PF_DYNAMIC) apply_walls(walls_of(walls, g, world_of(xi)), p, v);
  st3(x_out, i, p);
  st3(v_out, i, v);
}

// mean over dynamic particles of max(a - b, 0): separate-pass residual
__global__ void k_residual(int64_t n, const int32_t* __restrict__ flags, const int32_t* __restrict__ mask,
                           const float* __restrict__ av, const float* __restrict__ bv, double* part, int64_t* cntp,
                           DfsphDev* ctrl, double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double term = 0.0;
  long long dyn = 0;
  if (i < n && (particle_pf(flags, mask, i) & PF_DYNAMIC)) {
    term = (double)fmaxf(bv ? av[i] - bv[i] : av[i], 0.f);
    dyn = 1;
  }
  block_reduce_store(term, dyn, part, cntp);
  if (last_block(&ctrl->ticket)) {
    residual_finish(ctrl, part, cntp, gridDim.x, 0, -1.f);
    if (threadIdx.x == 0) *out = ctrl->residual;
  }
}

int run_rate(fs_context* c, const fs_model* m, int mode, int it, float h, float dt, float max_kappa, float eta,
             float* d_rho_dt, float* rho_star, float* kappa_new, float2* kratio_new, DfsphDev* ctrl,
             cudaStream_t st, bool use_lists = true) {
  RateArgs a;
  a.clock = c->clock;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.use_lists = use_lists ? 1 : 0;
  a.n = m->n;
  a.xs = c->xs;
  a.vstar = c->vs2;
  a.sc2 = c->sc2;
  a.rest_density = m->rest_density;
  a.h = h;
  a.dt = dt;
  a.max_kappa = max_kappa;
  a.eta = eta;
  a.mode = mode;
  a.it = it;
  a.d_rho_dt = d_rho_dt;
  a.rho_star = rho_star;
  a.kappa_new = kappa_new;
  a.kratio_new = kratio_new;
  a.ctrl = ctrl;
  a.red_part = c->red_part;
  a.red_cnt = c->red_cnt;
  const bool per_world = ctrl && c->worlds;
  a.wctl = per_world ? c->dfsph_worlds + (ctrl - c->dfsph) * c->nworlds : nullptr;
  a.pworld = m->particle_world;
  a.nworlds = c->nworlds;
  a.term = per_world ? c->sc1b : nullptr;
  if (per_world && !m->particle_world) return set_error(FS_ERR_INVALID, "dfsph rate: a batched context needs particle_world");
  if (ctrl && !per_world && nb_blocks(c, a.n) > reduction_blocks(c->capacity))
    return set_error(FS_ERR_INVALID, "dfsph rate: reduction buffer too small");
  {
    PassScope ps_(c, P_DFSPH_RATE, st, per_world ? 2 : 1);
    k_rate<<<nb_blocks(c, a.n), c->nb_block, 0, st>>>(a);
    if (per_world)
      k_world_residual<<<c->nworlds, kWorldBlock, 0, st>>>(a.g, c->sc1b, c->dfsph_worlds + (ctrl - c->dfsph) * c->nworlds,
                                                           ctrl, it, eta, c->clock);
  }
  return launch_check("dfsph rate");
}

int run_correct(fs_context* c, const fs_model* m, float h, float dt, const float* kappa, const float2* kratio,
                float* kappa_api, float* vstar_api, const DfsphDev* ctrl, cudaStream_t st, bool use_lists = true) {
  CorrectArgs a;
  a.clock = c->clock;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.use_lists = use_lists ? 1 : 0;
  a.n = m->n;
  a.xs = c->xs;
  a.vstar = c->vs2;
  a.kappa = kappa;
  a.kratio = kratio;
  a.h = h;
  a.dt = dt;
  a.kappa_api = kappa_api;
  a.vstar_api = vstar_api;
  a.ctrl = ctrl;
  const bool per_world = ctrl && c->worlds;
  a.wctl = per_world ? c->dfsph_worlds + (ctrl - c->dfsph) * c->nworlds : nullptr;
  a.pworld = m->particle_world;
  a.nworlds = c->nworlds;
  {
    PassScope ps_(c, P_DFSPH_CORRECT, st);
    k_correct<<<nb_blocks(c, a.n), c->nb_block, 0, st>>>(a);
  }
  return launch_check("dfsph correct");
}

int run_density_factor(fs_context* c, const fs_model* m, float h, int min_nb, float* rho, float* factor,
                       int32_t* count, cudaStream_t st) {
  DensFactorArgs a;
  a.clock = c->clock;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.n = m->n;
  a.xs = c->xs;
  a.vs = c->vs2;
  a.mv = c->mv;
  a.h = h;
  a.min_nb = min_nb;
  a.rho = rho;
  a.factor = factor;
  a.count = count;
  a.sc2 = c->sc2;
  {
    PassScope ps_(c, P_DFSPH_DENSITY_FACTOR, st);
    k_density_factor<<<nb_blocks(c, a.n), c->nb_block, 0, st>>>(a);
  }
  return launch_check("dfsph density/factor");
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

}  // extern "C"

namespace fs {
namespace {
// A clocked substep after its frame is complete: state_out = state_in for
// every field both states give.
__global__ void k_idle_copy_dfsph(int64_t n, const fs_frame_clock* clock, fs_state si, fs_state so) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !clock_idle(clock)) return;
  st3(so.particle_q, i, ld3(si.particle_q, i));
  st3(so.particle_qd, i, ld3(si.particle_qd, i));
  if (si.v_star && so.v_star) st3(so.v_star, i, ld3(si.v_star, i));
  const float* in[] = {si.rho, si.factor, si.rho_star, si.d_rho_dt, si.kappa, si.kappa_v};
  float* out[] = {so.rho, so.factor, so.rho_star, so.d_rho_dt, so.kappa, so.kappa_v};
  for (int k = 0; k < 6; ++k)
    if (in[k] && out[k]) out[k][i] = in[k][i];
  if (si.neighbor_count && so.neighbor_count) so.neighbor_count[i] = si.neighbor_count[i];
}

// Sets the context's clock for the span of a clocked substep.
struct ClockScope {
  fs_context* c;
  ClockScope(fs_context* ctx, const fs_frame_clock* clock) : c(ctx) { c->clock = clock; }
  ~ClockScope() { c->clock = nullptr; }
};
}  // namespace

int dfsph_substep(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so, const fs_dfsph_params* p,
                  float* accel, fs_stream_t stream);
}  // namespace fs

extern "C" {

int fs_dfsph_substep(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so, const fs_dfsph_params* p,
                     float* accel, fs_stream_t stream) {
  if (!c) return set_error(FS_ERR_INVALID, "fs_dfsph_substep: null argument");
  ClockScope cs(c, nullptr);
  return dfsph_substep(c, m, si, so, p, accel, stream);
}

int fs_dfsph_substep_clocked(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so,
                             const fs_dfsph_params* p, float* accel, const fs_frame_clock* clock,
                             fs_stream_t stream) {
  if (!c || !clock || !si || !so || !m) return set_error(FS_ERR_INVALID, "fs_dfsph_substep_clocked: null argument");
  int rc;
  {
    ClockScope cs(c, clock);
    rc = dfsph_substep(c, m, si, so, p, accel, stream);
  }
  if (rc || m->n == 0) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  {
    PassScope ps_(c, P_OTHER, st);
    k_idle_copy_dfsph<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, clock, *si, *so);
  }
  return launch_check("fs_dfsph_substep_clocked");
}

}  // extern "C"

namespace fs {

int dfsph_substep(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so, const fs_dfsph_params* p,
                  float* accel, fs_stream_t stream) {
  if (!c || !m || !si || !so || !p) return set_error(FS_ERR_INVALID, "fs_dfsph_substep: null argument");
  if (m->n < 0) return set_error(FS_ERR_INVALID, "fs_dfsph_substep: negative n");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mask || !m->particle_mass || !m->gravity || m->n_worlds < 1 ||
      !m->rest_density || !m->viscosity || !m->surface_tension || !si->particle_q || !si->particle_qd ||
      !so->particle_q || !so->particle_qd || !so->rho || !so->factor || !so->rho_star || !so->d_rho_dt ||
      !so->kappa || !so->kappa_v || !so->neighbor_count || !so->v_star || !accel)
    return set_error(FS_ERR_INVALID, "fs_dfsph_substep: missing array");
  if (p->warm_start && (!si->kappa || !si->kappa_v))
    return set_error(FS_ERR_INVALID, "fs_dfsph_substep: warm_start needs state_in kappa/kappa_v");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_dfsph_substep: n > capacity");
  if (c->worlds && !m->particle_world)
    return set_error(FS_ERR_INVALID, "fs_dfsph_substep: a batched context needs particle_world");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = m->n;
  const float h = p->smoothing_length, dt = p->dt;
  int rc;
  if ((rc = check_cuda(cudaMemsetAsync(c->dfsph, 0, sizeof(DfsphDev) * 2, st), "dfsph reset"))) return rc;
  if (c->worlds &&
      (rc = check_cuda(cudaMemsetAsync(c->dfsph_worlds, 0, sizeof(DfsphWorld) * 2 * c->nworlds, st), "dfsph reset")))
    return rc;
  // ---- first half: positions x_in
  if ((rc = grid_build(c, si->particle_q, n, h, st, m->particle_world, c->clock))) return rc;
  {
    PassScope ps_(c, P_GATHER, st);
    k_gather_common<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, *m, si->particle_q, si->particle_qd, c->xs, c->vs,
                                                    c->mv, c->status, c->nworlds);
  }
  {
    // density/factor reads masses from vs2.w: fill it from vs (v_in, mass) first
    if ((rc = check_cuda(cudaMemcpyAsync(c->vs2, c->vs, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st),
                         "dfsph copy")))
      return rc;
  }
  if ((rc = run_density_factor(c, m, h, p->min_neighbors_for_factor, so->rho, so->factor, so->neighbor_count, st)))
    return rc;
  AccelArgs aa;
  aa.g = grid_view(c);
  aa.L = nbr_list(c);
  aa.use_lists = 1;
  aa.n = n;
  aa.xs = c->xs;
  aa.vs = c->vs;
  aa.sc2 = c->sc2;
  aa.m = *m;
  aa.h = h;
  aa.particle_radius = p->particle_radius;
  aa.dt = dt;
  aa.accel = accel;
  aa.vstar = c->vs2;
  aa.clock = c->clock;
  {
    PassScope ps_(c, P_DFSPH_ACCEL, st);
    k_accel_predict<<<nb_blocks(c, n), c->nb_block, 0, st>>>(aa);
  }
  if ((rc = launch_check("dfsph accel"))) return rc;
  if (p->warm_start) {
    {
      PassScope ps_(c, P_GATHER, st, 2);
      k_gather_scalar<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, si->kappa, c->sc1, nullptr);
      k_kappa_ratio<<<blocks_for(n), kBlock, 0, st>>>(n, c->sc1, c->sc2, c->vs2, c->krm);
    }
    if ((rc = run_correct(c, m, h, dt, c->sc1, c->krm, so->kappa, nullptr, nullptr, st))) return rc;
  }
  for (int it = 0; it < p->max_rho_iterations; ++it) {
    if ((rc = run_rate(c, m, 0, it, h, dt, p->max_kappa, p->eta_density, so->d_rho_dt, so->rho_star, c->sc1,
                       c->krm, c->dfsph + 0, st)))
      return rc;
    if ((rc = run_correct(c, m, h, dt, c->sc1, c->krm, so->kappa, nullptr, c->dfsph + 0, st))) return rc;
  }
  {
    PassScope ps_(c, P_DFSPH_INTEGRATE, st);
    k_integrate<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, c->xs, c->vs2, dt, so->particle_q, so->v_star,
                                                   c->clock);
  }
  if ((rc = launch_check("dfsph integrate"))) return rc;
  // ---- second half: positions x_out
  if ((rc = grid_build(c, so->particle_q, n, h, st, m->particle_world, c->clock))) return rc;
  {
    PassScope ps_(c, P_GATHER, st);
    k_gather_common<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, *m, so->particle_q, so->v_star, c->xs, c->vs2, c->mv,
                                                    c->status, c->nworlds);
  }
  if ((rc = run_density_factor(c, m, h, p->min_neighbors_for_factor, so->rho, so->factor, so->neighbor_count, st)))
    return rc;
  if (p->warm_start) {
    {
      PassScope ps_(c, P_GATHER, st, 2);
      k_gather_scalar<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, si->kappa_v, c->sc1, nullptr);
      k_kappa_ratio<<<blocks_for(n), kBlock, 0, st>>>(n, c->sc1, c->sc2, c->vs2, c->krm);
    }
    if ((rc = run_correct(c, m, h, dt, c->sc1, c->krm, so->kappa_v, nullptr, nullptr, st))) return rc;
  }
  for (int it = 0; it < p->max_vel_iterations; ++it) {
    if ((rc = run_rate(c, m, 1, it, h, dt, p->max_kappa_v, p->eta_divergence, so->d_rho_dt, nullptr, c->sc1,
                       c->krm, c->dfsph + 1, st)))
      return rc;
    if ((rc = run_correct(c, m, h, dt, c->sc1, c->krm, so->kappa_v, nullptr, c->dfsph + 1, st))) return rc;
  }
  const Walls w = make_walls(p->bound_width, p->bound_height, p->bound_length, p->boundary_damping, 1, 0.f, 0.f);
  {
    PassScope ps_(c, P_DFSPH_FINAL, st);
    k_final<<<blocks_for(n), kBlock, 0, st>>>(n, grid_view(c), c->xs, c->vs2, w, so->particle_q, so->particle_qd,
                                              so->v_star, c->clock);
  }
  c->last_stream = st;
  return launch_check("dfsph final");
}

}  // namespace fs

extern "C" {

int fs_dfsph_info_worlds(fs_context* c, fs_dfsph_info* info, int32_t nworlds) {
  if (!c || !info || nworlds < 0) return set_error(FS_ERR_INVALID, "fs_dfsph_info_worlds: bad arguments");
  if (!c->worlds) return set_error(FS_ERR_INVALID, "fs_dfsph_info_worlds: not a batched context");
  if (nworlds > c->nworlds) return set_error(FS_ERR_INVALID, "fs_dfsph_info_worlds: nworlds > the context's worlds");
  if (nworlds == 0) return FS_OK;
  DeviceGuard dg(c->device);
  DfsphWorld* h = new DfsphWorld[2 * (size_t)c->nworlds];
  int rc = check_cuda(cudaMemcpyAsync(h, c->dfsph_worlds, sizeof(DfsphWorld) * 2 * c->nworlds,
                                      cudaMemcpyDeviceToHost, c->last_stream),
                      "fs_dfsph_info_worlds");
  if (!rc) rc = check_cuda(cudaStreamSynchronize(c->last_stream), "fs_dfsph_info_worlds: sync");
  if (!rc)
    for (int w = 0; w < nworlds; ++w) {
      const DfsphWorld& a = h[w];
      const DfsphWorld& b = h[c->nworlds + w];
      info[w].rho_iterations = a.iters;
      info[w].vel_iterations = b.iters;
      info[w].density_residual = a.residual;
      info[w].divergence_residual = b.residual;
    }
  delete[] h;
  return rc;
}

int fs_dfsph_info_read(fs_context* c, fs_dfsph_info* info) {
  if (!c || !info) return set_error(FS_ERR_INVALID, "fs_dfsph_info_read: bad arguments");
  if (c->worlds) {
    fs_dfsph_info* all = new fs_dfsph_info[c->nworlds];
    const int rc = fs_dfsph_info_worlds(c, all, c->nworlds);
    if (!rc) {
      *info = all[0];
      for (int w = 1; w < c->nworlds; ++w) {
        info->rho_iterations = std::max(info->rho_iterations, all[w].rho_iterations);
        info->vel_iterations = std::max(info->vel_iterations, all[w].vel_iterations);
        info->density_residual = std::max(info->density_residual, all[w].density_residual);
        info->divergence_residual = std::max(info->divergence_residual, all[w].divergence_residual);
      }
    }
    delete[] all;
    return rc;
  }
  DeviceGuard dg(c->device);
  DfsphDev h[2];
  int rc = check_cuda(cudaMemcpyAsync(h, c->dfsph, sizeof(h), cudaMemcpyDeviceToHost, c->last_stream),
                      "fs_dfsph_info_read");
  if (!rc) rc = check_cuda(cudaStreamSynchronize(c->last_stream), "fs_dfsph_info_read: sync");
  if (rc) return rc;
  info->rho_iterations = h[0].iters;
  info->vel_iterations = h[1].iters;
  info->density_residual = h[0].residual;
  info->divergence_residual = h[1].residual;
  return FS_OK;
}

int fs_dfsph_density_factor(fs_context* c, const fs_model* m, const float* x, float h, int32_t min_nb, float* rho,
                            float* factor, int32_t* neighbor_count, fs_stream_t stream) {
  if (!c || !m || !x || !rho || !factor || !neighbor_count)
    return set_error(FS_ERR_INVALID, "fs_dfsph_density_factor: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_dfsph_density_factor: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x, x, c->xs, c->vs2, c->mv, c->status, c->nworlds);
  return run_density_factor(c, m, h, min_nb, rho, factor, neighbor_count, st);
}

int fs_dfsph_nonpressure_predict(fs_context* c, const fs_model* m, const float* x, const float* v, const float* rho,
                                 float h, float particle_radius, float dt, float* accel, float* v_star,
                                 fs_stream_t stream) {
  if (!c || !m || !x || !v || !rho || !accel || !v_star)
    return set_error(FS_ERR_INVALID, "fs_dfsph_nonpressure_predict: null argument");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mass || !m->gravity || m->n_worlds < 1 || !m->viscosity ||
      !m->surface_tension)
    return set_error(FS_ERR_INVALID, "fs_dfsph_nonpressure_predict: missing model array");
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_dfsph_nonpressure_predict: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = m->n;
  k_gather_common<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, *m, x, v, c->xs, c->vs, c->mv, c->status,
                                                    c->nworlds);
  k_gather_pair<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, rho, nullptr, c->sc2);
  AccelArgs aa;
  aa.g = grid_view(c);
  aa.L = nbr_list(c);
  aa.use_lists = 0;
  aa.n = n;
  aa.xs = c->xs;
  aa.vs = c->vs;
  aa.sc2 = c->sc2;
  aa.m = *m;
  aa.h = h;
  aa.particle_radius = particle_radius;
  aa.dt = dt;
  aa.accel = accel;
  aa.vstar = c->vs2;
  aa.clock = nullptr;
  k_accel_predict<<<nb_blocks(c, n), c->nb_block, 0, st>>>(aa);
  k_scatter_xyz<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, c->vs2, v_star);
  return launch_check("fs_dfsph_nonpressure_predict");
}

int fs_dfsph_divergence(fs_context* c, const fs_model* m, const float* x, const float* v, float h, float* d_rho_dt,
                        fs_stream_t stream) {
  if (!c || !m || !x || !v || !d_rho_dt) return set_error(FS_ERR_INVALID, "fs_dfsph_divergence: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_dfsph_divergence: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x, v, c->xs, c->vs2, nullptr, c->status, c->nworlds);
  // rho/factor are not needed for the rate itself (mode 1 reads them only for kappa, which is discarded)
  if (cudaMemsetAsync(c->sc2, 0, sizeof(float2) * m->n, st) != cudaSuccess)
    return set_error(FS_ERR_CUDA, "fs_dfsph_divergence: memset");
  return run_rate(c, m, 1, 0, h, 1.f, 0.f, 0.f, d_rho_dt, nullptr, nullptr, nullptr, nullptr, st, false);
}

int fs_dfsph_correct(fs_context* c, const fs_model* m, const float* x, float* v_star, const float* rho,
                     const float* kappa, float h, float dt, fs_stream_t stream) {
  if (!c || !m || !x || !v_star || !rho || !kappa) return set_error(FS_ERR_INVALID, "fs_dfsph_correct: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_dfsph_correct: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x, v_star, c->xs, c->vs2, nullptr,
                                                       c->status, c->nworlds);
  k_gather_pair<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, rho, nullptr, c->sc2);
  k_gather_scalar<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, kappa, c->sc1, nullptr);
  {
    PassScope ps_(c, P_GATHER, st);
    k_kappa_ratio<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->sc1, c->sc2, c->vs2, c->krm);
  }
  return run_correct(c, m, h, dt, c->sc1, c->krm, nullptr, v_star, nullptr, st, false);
}

int fs_dfsph_residual(fs_context* c, const fs_model* m, const float* a, const float* b, double* out,
                      fs_stream_t stream) {
  if (!c || !m || !a || !out || !m->particle_flags) return set_error(FS_ERR_INVALID, "fs_dfsph_residual: bad args");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_dfsph_residual: n > capacity");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = m->n > 0 ? m->n : 1;
  if (blocks_for(n) > reduction_blocks(c->capacity > 0 ? c->capacity : 1))
    return set_error(FS_ERR_INVALID, "fs_dfsph_residual: reduction buffer too small");
  if (cudaMemsetAsync(c->dfsph, 0, sizeof(DfsphDev), st) != cudaSuccess)
    return set_error(FS_ERR_CUDA, "fs_dfsph_residual: memset");
  {
    PassScope ps_(c, P_OTHER, st);
    k_residual<<<blocks_for(n), kBlock, 0, st>>>(m->n, m->particle_flags, m->particle_mask, a, b, c->red_part,
                                               c->red_cnt, c->dfsph, out);
  }
  return launch_check("fs_dfsph_residual");
}

}  // extern "C"
