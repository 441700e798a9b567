// PBF substep on B200 (replaces SolverPBF.step, solver_pbf.py:676-954).
//
//   predict   v_pred = v + dt g; x_pred = x + dt v_pred; position bounds  (original order)
//   grid build(x_pred)          -- the only build unless rebuild_grid_each_iteration
//   gather    x_pred, v_pred, x_in, mass, flags -> cell order          (one pass)
//   density   (poly6)
//   accel     non-pressure (PBF variant) + apply_non_pressure_prediction + bounds -> x_pred'
//   repeat max_iterations:
//     lambda  rho, C, lambda, neighbour count
//     delta   dx (+ s_corr, clamp) and apply into the OTHER x_pred buffer (Jacobi)
//   density   (final) + velocity (x_pred - x_in) / dt                  (fused)
//   xsph      XSPH viscosity, copy to state_out, apply_bounds      (fused)
// As in the reference, the candidate set of every pass after the build is the
// one binned at build time, queried from the particle's current position.
#include "fs_nbr.cuh"

// The PBF neighbour kernels run fastest with a 64-register budget (1024
// resident threads per SM, no spills): measured 3 % faster per substep on
// the 401,856-particle dam break than the compiler's own choice (56
// registers with spills) and than an 85-register budget.
#define FS_NB_BOUNDS_PBF __launch_bounds__(kNbBlockMax, 1024 / kNbBlockMax)

namespace fs {

__global__ void k_gather_common(int64_t n, const int32_t* __restrict__ perm, fs_model m, const float* __restrict__ x,
                                const float* __restrict__ v, float4* __restrict__ xs, float4* __restrict__ vs,
                                float* __restrict__ mv, uint32_t* status, int nworlds);

namespace {

// predict_velocity_with_gravity (193-208) + predict_positions (212-224) +
// apply_position_bounds (367-399); original order.
__global__ void k_predict(int64_t n, fs_model m, GridDev g, const float* __restrict__ x, const float* __restrict__ v,
                          float dt, Walls walls, float* __restrict__ x_pred, float* __restrict__ v_pred) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float3 p = ld3(x, i), u = ld3(v, i);
  if (particle_pf(m.particle_flags, m.particle_mask, i) & PF_DYNAMIC) {
    const float3 gv = gravity_of(m, i);
    u = make_float3(u.x + dt * gv.x, u.y + dt * gv.y, u.z + dt * gv.z);
    p = make_float3(p.x + dt * u.x, p.y + dt * u.y, p.z + dt * u.z);
    clamp_position(walls_of_particle(walls, g, m, i), p);
  }
  st3(x_pred, i, p);
  st3(v_pred, i, u);
}

// The common gather of x_pred / v_pred plus the substep's input positions
// x_in (xin_s, for the velocity update) in one pass over the permutation.
__global__ void k_gather_pbf(int64_t n, const int32_t* __restrict__ perm, fs_model m, const float* __restrict__ x_pred,
                             const float* __restrict__ v_pred, const float* __restrict__ x_in, float4* __restrict__ xs,
                             float4* __restrict__ vs, float* __restrict__ mv, float4* __restrict__ xin_s,
                             uint32_t* status, int nworlds) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = perm[s];
  gather_common_slot(s, i, m, x_pred, v_pred, xs, vs, mv, status, nworlds);
  const float3 p = ld3(x_in, i);
  xin_s[s] = make_float4(p.x, p.y, p.z, 0.f);
}

// compute_density (115-141), poly6, self included.  sc2[s] = (rho,
// mass / max(rho, 1e-6)): the neighbour term of the viscosity and XSPH passes.
// With `record` it records the neighbour lists that the next pass at the
// same positions (accel, or XSPH) reuses.  With vout (the final density of a
// substep) it also writes update_velocity_from_positions (403-416):
// vout[s] = ((x_pred - x_in) / max(dt, 1e-8), m / max(rho, 1e-6)), v_pred
// for non-dynamic particles.
__global__ void FS_NB_BOUNDS_PBF k_density(GridDev g, NbrList L, int record, int64_t n,
                                                      const float4* __restrict__ xs, const float4* __restrict__ vs,
                                                      const float* __restrict__ mv, float h, float skin, float* rho,
                                                      float2* __restrict__ sc2, const float4* __restrict__ xin = nullptr,
                                                      float dt = 0.f, float4* __restrict__ vout = nullptr) {
  if (record) lists_recorded(L);
  for_slots(n, [&](int64_t s) {
    const float4 xi = xs[s];
    const int32_t i = g.perm[s];
    float acc = 0.f;
    const float h2m = h * h * kSupportMargin;
    const Poly6Spiky K(h);
    auto pair = [&](int t, float4 xj) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      acc = fmaf(__ldg(mv + t), K.w_r2(fmaf(dx, dx, fmaf(dy, dy, dz * dz))), acc);
    };
    if (pf_of(xi) & PF_ACTIVE) {
      if (record) {
        // entries out to h (1 + skin): the first lambda pass reuses them (k_lambda)
        const float hr = h * (1.0f + skin);
        record_list<false>(g, xs, (int)s, xi, h, hr * hr * kSupportMargin, L);
        visit_with<true, true>(g, xs, (int)s, xi, h, h2m, L, true, [&](int t) { return __ldg(mv + t); },
                               [&](int t, float4 xj, const float& m) {
          const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
          acc = fmaf(m, K.w_r2(fmaf(dx, dx, fmaf(dy, dy, dz * dz))), acc);
        });
      } else {
        scan_grid<true>(g, xs, (int)s, xi, h, h2m, pair);
      }
    } else if (record) {
      L.cnt[s] = 0;
    }
    rho[i] = acc;
    const float4 vi = vs[s];
    const float wgt = vi.w / fmaxf(acc, 1.0e-6f);
    sc2[s] = make_float2(acc, wgt);
    if (vout) {
      float3 u = xyz(vi);  // non-dynamic: v_pred == v_in
      if (pf_of(xi) & PF_DYNAMIC) {
        const float4 x0 = xin[s];
        const float d = fmaxf(dt, 1.0e-8f);
        u = make_float3((xi.x - x0.x) / d, (xi.y - x0.y) / d, (xi.z - x0.z) / d);
      }
      vout[s] = make_float4(u.x, u.y, u.z, wgt);  // .w: m / max(rho, 1e-6), XSPH's neighbour weight
    }
  });
}

// acceleration_non_pressure (145-189, PBF branches) + apply_non_pressure_prediction
// (228-242) + apply_position_bounds; writes the updated x_pred to xs_out.
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
  Walls walls;
  float* accel;
  float4* xs_out;
  uint32_t* disp_max = nullptr;  // largest |x_out - x| (float bits; null: not tracked)
};

__global__ void FS_NB_BOUNDS_PBF k_accel_apply(AccelArgs a) {
  float dmax = 0.f;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_DYNAMIC)) {
      st3(a.accel, i, make_float3(0.f, 0.f, 0.f));
      a.xs_out[s] = xi;
      return;
    }
    const float4 vi = a.vs[s];
    const float mu = a.m.viscosity[i];
    const float gamma = a.m.surface_tension[i];
    const float coh = gamma / vi.w;
    const float mu10 = 10.f * mu;
    const float visc_den_add = 0.01f * (a.h * a.h);
    const float rp2 = a.particle_radius * a.particle_radius;
    const Poly6Spiky K(a.h);
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (gamma != 0.f || mu != 0.f) {
      const bool lists_ok = a.use_lists && lists_usable(a.L);
      visit_with<false, false, true>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                        [&](int t) { return __ldg(a.vs + t); }, [&](int t, float4 xj, const float4& vj) {
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        float c = 0.f;
        if (gamma != 0.f) c -= coh * vj.w * K.w_r2(fmaxf(r2, rp2));  // W(max(r, r_p))
        if (mu != 0.f) {
          const float vdot = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
          if (vdot != 0.f) {
            float r, rinv;
            r_and_inv(r2, r, rinv);
            c += mu10 * __ldg(&a.sc2[t].y) * __fdividef(vdot, r2 + visc_den_add) * K.grad_scale(r, rinv);
          }
        }
        ax = fmaf(c, dx, ax);
        ay = fmaf(c, dy, ay);
        az = fmaf(c, dz, az);
      });
    }
    st3(a.accel, i, make_float3(ax, ay, az));
    const float dvx = a.dt * ax, dvy = a.dt * ay, dvz = a.dt * az;
    float3 p = make_float3(xi.x + a.dt * dvx, xi.y + a.dt * dvy, xi.z + a.dt * dvz);
    clamp_position(walls_of(a.walls, a.g, world_of(xi)), p);
    a.xs_out[s] = make_float4(p.x, p.y, p.z, xi.w);
    const float ex = p.x - xi.x, ey = p.y - xi.y, ez = p.z - xi.z;
    dmax = fmaxf(dmax, sqrtf(ex * ex + ey * ey + ez * ez));
  });
  if (a.disp_max) {  // non-negative floats order as their bit patterns
    const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(dmax));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(a.disp_max, m);
  }
}

// compute_pbf_lambda (246-302)
struct LambdaArgs {
  GridDev g;
  NbrList L;
  int use_lists;
  int64_t n;
  const float4* xs;
  const float4* vs;   // .w = mass
  const float* rest_density;
  float h, eps;
  int min_nb;
  float2* lam_s;      // cell order (lambda, mass): what the delta pass gathers per neighbour
  float* lam;         // API
  float* rho;         // API
  int32_t* count;     // API
  // Reuse of the density pass's lists (first iteration): positions at their
  // recording (null: always scan), the largest displacement since, and the
  // displacement up to which the recorded skin still holds every neighbour.
  const float4* xs_rec = nullptr;
  const uint32_t* disp_max = nullptr;
  float reuse_limit = 0.f;
};

// A list recorded at positions x out to h (1 + skin) holds, in visiting order,
// every candidate that a scan at positions x' would accept (r^2 <= h^2 at x')
// when (a) every particle moved at most skin h / 2 (|x'_i - x'_j| <= h implies
// |x_i - x_j| <= h + 2 max|x' - x|) and (b) the query at x'_i visits the same
// cells as at x_i; visiting that list with the support test at x' then
// reproduces the scan's pair sequence exactly.  Particles failing (b), and
// every particle when (a) fails, scan the grid.
__global__ void FS_NB_BOUNDS_PBF k_lambda(LambdaArgs a) {
  lists_recorded(a.L);
  const bool reuse_ok = a.xs_rec && __uint_as_float(*a.disp_max) <= a.reuse_limit;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_DYNAMIC)) {
      a.L.cnt[s] = 0;
      a.lam_s[s] = make_float2(0.f, a.vs[s].w);
      if (a.lam) a.lam[i] = 0.f;
      if (a.rho) a.rho[i] = 0.f;
      if (a.count) a.count[i] = 0;
      return;
    }
    const float rho0 = fmaxf(a.rest_density[i], 1.0e-6f);
    const float inv_rho0 = 1.0f / rho0;
    const Poly6Spiky K(a.h);
    float rho = 0.f, sq = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    int cnt = 0;
    const float h2m = a.h * a.h * kSupportMargin;
    // records the lists the delta pass of this iteration (same positions) reuses
    const bool reuse = reuse_ok && a.L.cnt[s] <= kNbMax && same_query_cells(a.g, world_of(xi), a.xs_rec[s], xi, a.h);
    if (a.g.tile_stats && a.xs_rec) {
      const unsigned full = __activemask();
      const unsigned b = __ballot_sync(full, reuse);
      if ((int)(threadIdx.x & 31) == __ffs(full) - 1) atomicAdd(a.g.tile_stats + 2, (unsigned long long)__popc(b));
    }
    if (!reuse) record_list<false>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L);
    visit_with<true, true>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L, true, [&](int t) { return __ldg(&a.vs[t].w); },
                           [&](int t, float4 xj, const float& mj) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (t != (int)s && exact_lt_h(r2, dx, dy, dz, a.h, K.h2)) ++cnt;
      float r, rinv;
      r_and_inv(r2, r, rinv);
      rho = fmaf(mj, K.w_r2(r2), rho);
      const float c = -(mj * inv_rho0) * K.grad_scale(r, rinv);
      const float gjx = c * dx, gjy = c * dy, gjz = c * dz;
      sq = fmaf(gjx, gjx, fmaf(gjy, gjy, fmaf(gjz, gjz, sq)));
      gx -= gjx;
      gy -= gjy;
      gz -= gjz;
    });
    sq = fmaf(gx, gx, fmaf(gy, gy, fmaf(gz, gz, sq)));
    const float ci = fmaxf(rho / rho0 - 1.0f, 0.f);
    const float l = (a.min_nb > 0 && cnt < a.min_nb) ? 0.f : -ci / (sq + a.eps);
    a.lam_s[s] = make_float2(l, a.vs[s].w);
    if (a.lam) a.lam[i] = l;
    if (a.rho) a.rho[i] = rho;
    if (a.count) a.count[i] = cnt;
  });
}

// compute_delta_position + compute_scorr (306-350, 91-101), then
// apply_delta_position (354-363) into xs_out (+ position bounds when asked).
struct DeltaArgs {
  GridDev g;
  NbrList L;
  int use_lists;
  int64_t n;
  const float4* xs;
  const float4* vs;   // .w = mass
  const float2* lam_s;  // (lambda, mass), one gather per neighbour
  const float* rest_density;
  float h, scorr_k, scorr_n, w_dq, max_dp;
  int clamp;
  Walls walls;
  float* delta_p;     // API
  float4* xs_out;     // may be null (separate-pass use)
};

// x^n for a small positive integer n by repeated squaring (2 products for
// the usual n = 4, against a general powf per pair); within 2 ulp of x^n.
FS_DEV float pow_uint(float x, int n) {
  float r = 1.f;
  for (; n; n >>= 1) {
    if (n & 1) r *= x;
    x *= x;
  }
  return r;
}

__global__ void FS_NB_BOUNDS_PBF k_delta(DeltaArgs a) {
  // an integral exponent 1..8 (the class default is 4) takes pow_uint
  const int n_int = (a.scorr_n >= 1.f && a.scorr_n <= 8.f && a.scorr_n == rintf(a.scorr_n)) ? (int)a.scorr_n : 0;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_DYNAMIC)) {
      st3(a.delta_p, i, make_float3(0.f, 0.f, 0.f));
      if (a.xs_out) a.xs_out[s] = xi;
      return;
    }
    const float rho0 = fmaxf(a.rest_density[i], 1.0e-6f);
    const float li = a.lam_s[s].x;
    const Poly6Spiky K(a.h);
    const bool scorr = a.scorr_k != 0.f && !(a.w_dq <= 1.0e-6f);
    const float inv_wdq = scorr ? 1.0f / a.w_dq : 0.f;
    float dx_ = 0.f, dy_ = 0.f, dz_ = 0.f;
    const bool lists_ok = a.use_lists && lists_usable(a.L);
    visit_with<false, false, true>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                      [&](int t) { return __ldg(a.lam_s + t); }, [&](int t, float4 xj, const float2& lj) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      float r, rinv;
      r_and_inv(r2, r, rinv);
      float sc = 0.f;
      if (scorr) {
        const float q = K.w_r2(r2) * inv_wdq;
        sc = -a.scorr_k * (n_int ? pow_uint(q, n_int) : powf(q, a.scorr_n));
      }
      const float c = (li + lj.x + sc) * lj.y * K.grad_scale(r, rinv);
      dx_ = fmaf(c, dx, dx_);
      dy_ = fmaf(c, dy, dy_);
      dz_ = fmaf(c, dz, dz_);
    });
    float3 d = make_float3(dx_ / rho0, dy_ / rho0, dz_ / rho0);
    if (a.max_dp > 0.f) {
      const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
      if (len > a.max_dp) {
        const float sc = a.max_dp / fmaxf(len, 1.0e-12f);
        d = make_float3(d.x * sc, d.y * sc, d.z * sc);
      }
    }
    st3(a.delta_p, i, d);
    if (a.xs_out) {
      float3 p = make_float3(xi.x + d.x, xi.y + d.y, xi.z + d.z);
      if (a.clamp) clamp_position(walls_of(a.walls, a.g, world_of(xi)), p);
      a.xs_out[s] = make_float4(p.x, p.y, p.z, xi.w);
    }
  });
}

// update_velocity_from_positions (403-416), cell order; .w keeps the mass
// apply_xsph_viscosity (435-463) + copy x_pred -> particle_q + apply_bounds (467-517)
struct XsphArgs {
  GridDev g;
  NbrList L;
  int use_lists;
  int64_t n;
  const float4* xs;
  const float4* vel;   // (v, m / max(rho, 1e-6)) cell order
  const float2* sc2;   // rho
  float h, c;
  Walls walls;
  int bounds;          // fused apply_bounds (substep) or not (separate pass)
  float* x_out;
  float* v_out;
  float* x_pred_api;   // optional
};

__global__ void FS_NB_BOUNDS_PBF k_xsph_final(XsphArgs a) {
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const float4 vi = a.vel[s];
    const int32_t i = a.g.perm[s];
    float3 v = xyz(vi);
    float3 p = xyz(xi);
    if (a.x_pred_api) st3(a.x_pred_api, i, p);
    if (pf_of(xi) & PF_DYNAMIC) {
      if (a.c > 0.f) {
        const Poly6Spiky K(a.h);
        float cx = 0.f, cy = 0.f, cz = 0.f;
        const bool lists_ok = a.use_lists && lists_usable(a.L);
        visit_with<false, false, true>(a.g, a.xs, (int)s, xi, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok,
                          [&](int t) { return __ldg(a.vel + t); }, [&](int t, float4 xj, const float4& vj) {
          const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
          // vj = (v, m / max(rho, 1e-6))
          // (m_j / max(rho_j, 1e-6)) W(r), the ratio from the final density pass
          const float w = vj.w * K.w_r2(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
          cx = fmaf(vj.x - vi.x, w, cx);
          cy = fmaf(vj.y - vi.y, w, cy);
          cz = fmaf(vj.z - vi.z, w, cz);
        });
        v = make_float3(fmaf(a.c, cx, vi.x), fmaf(a.c, cy, vi.y), fmaf(a.c, cz, vi.z));
      }
      if (a.bounds) apply_walls(walls_of(a.walls, a.g, world_of(xi)), p, v);
    }
    if (a.x_out) st3(a.x_out, i, p);
    st3(a.v_out, i, v);
  });
}

__global__ void k_scatter_x(int64_t n, const int32_t* __restrict__ perm, const float4* __restrict__ xs,
                            float* __restrict__ x) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  st3(x, perm[s], xyz(xs[s]));
}

__global__ void k_gather_lambda(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ a,
                                float* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) out[s] = a[perm[s]];
}

// (rho, mass / max(rho, 1e-6)) from a cell-order density and the mass in
// vel.w; vel.w then holds the ratio (XSPH's neighbour weight)
__global__ void k_rho_ratio(int64_t n, const float* __restrict__ rho, float4* __restrict__ vel,
                            float2* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float ratio = vel[s].w / fmaxf(rho[s], 1.0e-6f);
  out[s] = make_float2(rho[s], ratio);
  vel[s].w = ratio;
}

// (lambda[i], mass) of original order into cell order (mass from the gathered vs.w)
__global__ void k_gather_lambda_mass(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ lam,
                                     const float4* __restrict__ vs, float2* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) out[s] = make_float2(lam[perm[s]], vs[s].w);
}

int gather_pbf(fs_context* c, const fs_model* m, const float* x_in, cudaStream_t st) {
  const int64_t n = m->n;
  {
    PassScope ps_(c, P_GATHER, st);
    k_gather_pbf<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, *m, c->xo_tmp, c->vo_tmp, x_in, c->xs, c->vs, c->mv,
                                                 c->vs2, c->status, c->nworlds);
  }
  return launch_check("pbf gather");
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

int fs_pbf_substep(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so, const fs_pbf_params* p,
                   float* accel, float* x_pred, fs_stream_t stream) {
  if (!c || !m || !si || !so || !p) return set_error(FS_ERR_INVALID, "fs_pbf_substep: null argument");
  if (m->n < 0) return set_error(FS_ERR_INVALID, "fs_pbf_substep: negative n");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mask || !m->particle_mass || !m->gravity || m->n_worlds < 1 ||
      !m->rest_density || !m->viscosity || !m->surface_tension || !si->particle_q || !si->particle_qd ||
      !so->particle_q || !so->particle_qd || !so->rho || !so->pbf_lambda || !so->neighbor_count || !so->delta_p ||
      !accel)
    return set_error(FS_ERR_INVALID, "fs_pbf_substep: missing array");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_pbf_substep: n > capacity");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = m->n;
  const float h = p->smoothing_length, dt = p->dt;
  const Walls w = make_walls(p->bound_width, p->bound_height, p->bound_length, p->boundary_damping, 2,
                             p->particle_radius, p->boundary_epsilon);
  int rc;
  {
    PassScope ps_(c, P_PBF_PREDICT, st);
    k_predict<<<blocks_for(n), kBlock, 0, st>>>(n, *m, grid_view(c), si->particle_q, si->particle_qd, dt, w, c->xo_tmp,
                                                c->vo_tmp);
  }
  if ((rc = launch_check("pbf predict"))) return rc;
  if ((rc = grid_build(c, c->xo_tmp, n, h, st, m->particle_world))) return rc;
  if ((rc = gather_pbf(c, m, si->particle_q, st))) return rc;
  const GridDev g = grid_view(c);
  // neighbour lists: density -> accel, lambda -> delta, final density -> XSPH
  const NbrList L = nbr_list(c);
  const int use_lists = 1;
  // the first density records its lists out to h (1 + skin) so that the first
  // lambda pass can reuse them instead of scanning the grid (k_lambda).  The
  // non-pressure update between the two moves particles by dt^2 |a|: at most
  // 0.003 h in the 401,856-particle dam break, well inside the default
  // 0.02 h skin (+6 % list entries).
  const float skin = (!p->rebuild_grid_each_iteration && p->max_iterations > 0) ? c->list_skin : 0.f;
  if (skin > 0.f && (rc = check_cuda(cudaMemsetAsync(c->pbf_disp, 0, sizeof(uint32_t), st), "pbf reset")))
    return rc;
  {
    PassScope ps_(c, P_PBF_DENSITY, st);
    k_density<<<nb_blocks(c, n), c->nb_block, 0, st>>>(g, L, 1, n, c->xs, c->vs, c->mv, h, skin, so->rho, c->sc2);
  }
  AccelArgs aa;
  aa.g = g;
  aa.L = L;
  aa.use_lists = use_lists;
  aa.n = n;
  aa.xs = c->xs;
  aa.vs = c->vs;
  aa.sc2 = c->sc2;
  aa.m = *m;
  aa.h = h;
  aa.particle_radius = p->particle_radius;
  aa.dt = dt;
  aa.walls = w;
  aa.accel = accel;
  aa.xs_out = c->xs2;
  aa.disp_max = skin > 0.f ? c->pbf_disp : nullptr;
  {
    PassScope ps_(c, P_PBF_ACCEL, st);
    k_accel_apply<<<nb_blocks(c, n), c->nb_block, 0, st>>>(aa);
  }
  if ((rc = launch_check("pbf accel"))) return rc;
  float4* cur = c->xs2;
  float4* nxt = c->xs;
  for (int it = 0; it < p->max_iterations; ++it) {
    const GridDev gi = grid_view(c);
    LambdaArgs la;
    la.g = gi;
    la.L = L;
    la.use_lists = use_lists;
    la.n = n;
    la.xs = cur;
    la.vs = c->vs;
    la.rest_density = m->rest_density;
    la.h = h;
    la.eps = p->lambda_epsilon;
    la.min_nb = p->min_neighbors_for_lambda;
    la.lam_s = c->krm;
    la.lam = so->pbf_lambda;
    la.rho = so->rho;
    la.count = so->neighbor_count;
    la.xs_rec = (skin > 0.f && it == 0) ? c->xs : nullptr;  // the first density's positions
    la.disp_max = c->pbf_disp;
    la.reuse_limit = 0.5f * h * (skin - 1.0e-4f);
    {
      PassScope ps_(c, P_PBF_LAMBDA, st);
      k_lambda<<<nb_blocks(c, n), c->nb_block, 0, st>>>(la);
    }
    DeltaArgs da;
    da.g = gi;
    da.L = L;
    da.use_lists = use_lists;
    da.n = n;
    da.xs = cur;
    da.vs = c->vs;
    da.lam_s = c->krm;
    da.rest_density = m->rest_density;
    da.h = h;
    da.scorr_k = p->scorr_k;
    da.scorr_n = p->scorr_n;
    da.w_dq = p->scorr_w_delta_q;
    da.max_dp = p->max_delta_position;
    da.clamp = (p->rebuild_grid_each_iteration || it == p->max_iterations - 1) ? 1 : 0;
    da.walls = w;
    da.delta_p = so->delta_p;
    da.xs_out = nxt;
    {
      PassScope ps_(c, P_PBF_DELTA, st);
      k_delta<<<nb_blocks(c, n), c->nb_block, 0, st>>>(da);
    }
    if ((rc = launch_check("pbf iteration"))) return rc;
    float4* t = cur;
    cur = nxt;
    nxt = t;
    if (p->rebuild_grid_each_iteration) {
      // x_pred back to original order, rebuild, regather (v_pred/x_in follow)
      {
        PassScope ps_(c, P_GATHER, st);
        k_scatter_x<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, cur, c->xo_tmp);
      }
      if ((rc = grid_build(c, c->xo_tmp, n, h, st, m->particle_world))) return rc;
      if ((rc = gather_pbf(c, m, si->particle_q, st))) return rc;
      cur = c->xs;
      nxt = c->xs2;
    }
  }
  // final density on the bounded x_pred (bounds were fused into the last apply)
  const GridDev gf = grid_view(c);
  {
    // + update_velocity_from_positions into nxt (the other x_pred buffer)
    PassScope ps_(c, P_PBF_DENSITY, st);
    k_density<<<nb_blocks(c, n), c->nb_block, 0, st>>>(gf, L, 1, n, cur, c->vs, c->mv, h, 0.f, so->rho, c->sc2,
                                                       c->vs2, dt, nxt);
  }
  XsphArgs xa;
  xa.g = gf;
  xa.L = L;
  xa.use_lists = use_lists;
  xa.n = n;
  xa.xs = cur;
  xa.vel = nxt;
  xa.sc2 = c->sc2;
  xa.h = h;
  xa.c = p->xsph_c;
  xa.walls = w;
  xa.bounds = 1;
  xa.x_out = so->particle_q;
  xa.v_out = so->particle_qd;
  xa.x_pred_api = x_pred;
  {
    PassScope ps_(c, P_PBF_XSPH, st);
    k_xsph_final<<<nb_blocks(c, n), c->nb_block, 0, st>>>(xa);
  }
  c->last_stream = st;
  return launch_check("pbf final");
}

int fs_pbf_predict(fs_context* c, const fs_model* m, const float* x, const float* v, const fs_pbf_params* p,
                   float* x_pred, float* v_pred, fs_stream_t stream) {
  if (!c || !m || !x || !v || !p || !x_pred || !v_pred) return set_error(FS_ERR_INVALID, "fs_pbf_predict: null argument");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mask || !m->gravity || m->n_worlds < 1)
    return set_error(FS_ERR_INVALID, "fs_pbf_predict: missing model array");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const Walls w = make_walls(p->bound_width, p->bound_height, p->bound_length, p->boundary_damping, 2,
                             p->particle_radius, p->boundary_epsilon);
  k_predict<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, *m, grid_view(c), x, v, p->dt, w, x_pred, v_pred);
  return launch_check("fs_pbf_predict");
}

int fs_pbf_density(fs_context* c, const fs_model* m, const float* x, float h, float* rho, fs_stream_t stream) {
  if (!c || !m || !x || !rho) return set_error(FS_ERR_INVALID, "fs_pbf_density: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_pbf_density: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x, x, c->xs, c->vs, c->mv,
                                                       c->status, c->nworlds);
  k_density<<<nb_blocks(c, m->n), c->nb_block, 0, st>>>(grid_view(c), nbr_list(c), 0, m->n, c->xs, c->vs, c->mv, h, 0.f,
                                                                rho, c->sc2);
  return launch_check("fs_pbf_density");
}

int fs_pbf_lambda(fs_context* c, const fs_model* m, const float* x_pred, const fs_pbf_params* p, float* pbf_lambda,
                  float* rho, int32_t* neighbor_count, fs_stream_t stream) {
  if (!c || !m || !x_pred || !p || !pbf_lambda) return set_error(FS_ERR_INVALID, "fs_pbf_lambda: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_pbf_lambda: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x_pred, x_pred, c->xs, c->vs, nullptr,
                                                       c->status, c->nworlds);
  LambdaArgs la;
  la.g = grid_view(c);
  la.L = nbr_list(c);
  la.use_lists = 0;
  la.n = m->n;
  la.xs = c->xs;
  la.vs = c->vs;
  la.rest_density = m->rest_density;
  la.h = p->smoothing_length;
  la.eps = p->lambda_epsilon;
  la.min_nb = p->min_neighbors_for_lambda;
  la.lam_s = c->krm;
  la.lam = pbf_lambda;
  la.rho = rho;
  la.count = neighbor_count;
  k_lambda<<<nb_blocks(c, m->n), c->nb_block, 0, st>>>(la);
  return launch_check("fs_pbf_lambda");
}

int fs_pbf_delta(fs_context* c, const fs_model* m, const float* x_pred, const float* pbf_lambda,
                 const fs_pbf_params* p, float* delta_p, fs_stream_t stream) {
  if (!c || !m || !x_pred || !pbf_lambda || !p || !delta_p)
    return set_error(FS_ERR_INVALID, "fs_pbf_delta: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_pbf_delta: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x_pred, x_pred, c->xs, c->vs, nullptr,
                                                       c->status, c->nworlds);
  k_gather_lambda_mass<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, pbf_lambda, c->vs, c->krm);
  DeltaArgs da;
  da.g = grid_view(c);
  da.L = nbr_list(c);
  da.use_lists = 0;
  da.n = m->n;
  da.xs = c->xs;
  da.vs = c->vs;
  da.lam_s = c->krm;
  da.rest_density = m->rest_density;
  da.h = p->smoothing_length;
  da.scorr_k = p->scorr_k;
  da.scorr_n = p->scorr_n;
  da.w_dq = p->scorr_w_delta_q;
  da.max_dp = p->max_delta_position;
  da.clamp = 0;
  da.walls = Walls{};
  da.delta_p = delta_p;
  da.xs_out = nullptr;
  k_delta<<<nb_blocks(c, m->n), c->nb_block, 0, st>>>(da);
  return launch_check("fs_pbf_delta");
}

int fs_pbf_xsph(fs_context* c, const fs_model* m, const float* x_pred, const float* v_in, const float* rho, float h,
                float xsph_c, float* v_out, fs_stream_t stream) {
  if (!c || !m || !x_pred || !v_in || !rho || !v_out) return set_error(FS_ERR_INVALID, "fs_pbf_xsph: null argument");
  if (m->n == 0) return FS_OK;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_pbf_xsph: build the grid first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x_pred, v_in, c->xs, c->vs2, nullptr,
                                                       c->status, c->nworlds);
  k_gather_lambda<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, rho, c->sc1);
  k_rho_ratio<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->sc1, c->vs2, c->sc2);
  XsphArgs xa;
  xa.g = grid_view(c);
  xa.L = nbr_list(c);
  xa.use_lists = 0;
  xa.n = m->n;
  xa.xs = c->xs;
  xa.vel = c->vs2;
  xa.sc2 = c->sc2;
  xa.h = h;
  xa.c = xsph_c;
  xa.walls = Walls{};
  xa.bounds = 0;
  xa.x_out = nullptr;
  xa.v_out = v_out;
  xa.x_pred_api = nullptr;
  k_xsph_final<<<nb_blocks(c, m->n), c->nb_block, 0, st>>>(xa);
  return launch_check("fs_pbf_xsph");
}

}  // extern "C"
