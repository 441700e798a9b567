// WCSPH substep on B200 (replaces SolverWCSPH.step, solver_wcsph.py:431-535).
//
// Pass structure (one thread per cell-sorted slot; neighbour reads are
// contiguous slot ranges of the cell-sorted streams):
//   grid build(x_in)                       -- fs_grid.cu
//   gather    x_in, v_in, mass, flags      -> xs, vs, mv     (cell order)
//   density   rho, p (EOS)                 -> sc2 (cell order) + rho/pressure (original order)
//   force     pressure + viscosity + cohesion + gravity, then
//             integrate_velocity, integrate_positions and apply_bounds fused
//             -> accel, particle_qd, particle_q (original order)
#include "fs_nbr.cuh"

namespace fs {

// -------------------------------------------------------------- gather ----
// Cell-order copies of what neighbour loops read.  mv = rest_density * volume
// with volume = mass / max(rest_density, 1e-6) (compute_particle_volume,
// solver_wcsph.py:110-116).
__global__ void k_gather_common(int64_t n, const int32_t* __restrict__ perm, fs_model m, const float* __restrict__ x,
                                const float* __restrict__ v, float4* __restrict__ xs, float4* __restrict__ vs,
                                float* __restrict__ mv, uint32_t* status, int nworlds) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  gather_common_slot(s, perm[s], m, x, v, xs, vs, mv, status, nworlds);
}

// ------------------------------------------------------------- density ----
// compute_density_pressure, solver_wcsph.py:120-158.  Self included.
// sc2[s] = (p / max(rho^2, 1e-6), 1 / max(rho, 1e-6)): the two per-particle
// ratios of the force pass (cal_acc_with_pressure / _non_pressure).
struct DensityArgs {
  GridDev g;
  NbrList L;
  int64_t n;
  const float4* xs;
  const float* mv;
  const float* rest_density;  // original order
  const float* stiffness;     // original order
  const float* exponent;
  float h;
  int clamp;
  float* rho;                 // original order (API)
  float* pressure;            // original order (API)
  float2* sc2;                // cell order
  const fs_frame_clock* clock;  // clocked substep: nothing to do once the frame is complete
};

__global__ void FS_NB_BOUNDS k_wcsph_density(DensityArgs a) {
  if (clock_idle(a.clock)) return;
  lists_recorded(a.L);
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_ACTIVE)) {
      a.rho[i] = 0.f;
      a.pressure[i] = 0.f;
      a.sc2[s] = make_float2(0.f, 0.f);
      a.L.cnt[s] = 0;
      return;
    }
    const float h2m = a.h * a.h * kSupportMargin;
    record_list<false>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L);
    const Cubic K(a.h);
    float acc = 0.f;
    visit_with<true, true>(a.g, a.xs, (int)s, xi, a.h, h2m, a.L, true, [&](int t) { return __ldg(a.mv + t); },
                           [&](int t, float4 xj, const float& m) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      float r, rinv;
      r_and_inv(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), r, rinv);
      acc = fmaf(m, K.w(r), acc);
    });
    float p = a.stiffness[i] * (powf(acc / fmaxf(a.rest_density[i], 1.0e-6f), a.exponent[i]) - 1.0f);
    if (a.clamp) p = fmaxf(p, 0.f);
    a.rho[i] = acc;
    a.pressure[i] = p;
    a.sc2[s] = make_float2(p / fmaxf(acc * acc, 1.0e-6f), 1.0f / fmaxf(acc, 1.0e-6f));
  });
}

// --------------------------------------------------------------- force ----
// acceleration_wcsph (162-228) + integrate_velocity (232-244) +
// integrate_positions (248-260) + apply_bounds (264-305).
struct ForceArgs {
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
  float* x_out;
  float* v_out;
  const fs_frame_clock* clock;  // clocked substep: dt from the clock, nothing to do once the frame is complete
};

__global__ void FS_NB_BOUNDS k_wcsph_force(ForceArgs a) {
  if (clock_idle(a.clock)) return;
  const float dt = a.clock ? a.clock->dt : a.dt;
  for_slots(a.n, [&](int64_t s) {
    const float4 xi = a.xs[s];
    const float4 vi = a.vs[s];
    const int32_t i = a.g.perm[s];
    if (!(pf_of(xi) & PF_DYNAMIC)) {
      st3(a.accel, i, make_float3(0.f, 0.f, 0.f));
      st3(a.v_out, i, xyz(vi));
      st3(a.x_out, i, xyz(xi));
      return;
    }
    const float dp_i = a.sc2[s].x;
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
      if (r2 == 0.f) return;  // coincident particles: every term carries the zero vector d
      const float4 vj = __ldg(a.vs + t);
      const float2 rj = __ldg(a.sc2 + t);  // (p_j / rho_j^2, 1 / rho_j)
      float r, rinv;
      r_and_inv(r2, r, rinv);
      const float m_j = vj.w;
      // cohesion -gamma/m_i m_j W(max(r, r_p)) d
      const float wc = coh * m_j * K.w(fmaxf(r, a.particle_radius));
      // viscosity 10 mu (m_j / rho_j) (v_ij . d) / (r^2 + 0.01 h^2) grad W
      const float vdot = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
      const float visc = mu10 * m_j * rj.y * __fdividef(vdot, r2 + visc_den_add);
      // pressure -m_j (p_i / rho_i^2 + p_j / rho_j^2) grad W
      const float pres = -m_j * (dp_i + rj.x);
      const float c = fmaf(visc + pres, K.grad_scale(r, rinv), -wc);
      ax = fmaf(c, dx, ax);
      ay = fmaf(c, dy, ay);
      az = fmaf(c, dz, az);
    });
    const float3 g = gravity_of(a.m, i);
    const float3 acc = make_float3(ax + g.x, ay + g.y, az + g.z);
    st3(a.accel, i, acc);
    float3 v = make_float3(vi.x + dt * acc.x, vi.y + dt * acc.y, vi.z + dt * acc.z);
    float3 p = make_float3(xi.x + v.x * dt, xi.y + v.y * dt, xi.z + v.z * dt);
    apply_walls(walls_of(a.walls, a.g, world_of(xi)), p, v);
    st3(a.v_out, i, v);
    st3(a.x_out, i, p);
  });
}

// (rho, p) of original order -> force-pass ratios in cell order
__global__ void k_gather_ratios(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ rho,
                                const float* __restrict__ p, float2* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = perm[s];
  const float r = rho[i];
  out[s] = make_float2(p[i] / fmaxf(r * r, 1.0e-6f), 1.0f / fmaxf(r, 1.0e-6f));
}

// A clocked substep after its frame is complete: state_out = state_in.
__global__ void k_idle_copy(int64_t n, const fs_frame_clock* clock, const float* __restrict__ x_in,
                            const float* __restrict__ v_in, const float* __restrict__ rho_in,
                            const float* __restrict__ p_in, float* x_out, float* v_out, float* rho_out, float* p_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !clock_idle(clock)) return;
  st3(x_out, i, ld3(x_in, i));
  st3(v_out, i, ld3(v_in, i));
  if (rho_in && rho_out) rho_out[i] = rho_in[i];
  if (p_in && p_out) p_out[i] = p_in[i];
}

int wcsph_gather(fs_context* c, const fs_model* m, const float* x, const float* v, cudaStream_t st) {
  const int64_t n = m->n;
  {
    PassScope ps_(c, P_GATHER, st);
    k_gather_common<<<blocks_for(n), kBlock, 0, st>>>(n, c->perm, *m, x, v, c->xs, c->vs, c->mv, c->status, c->nworlds);
  }
  return launch_check("wcsph gather");
}

int launch_density(fs_context* c, const fs_model* m, float h, int clamp, bool eos, float* rho, float* pressure,
                   cudaStream_t st, const fs_frame_clock* clock = nullptr) {
  DensityArgs a;
  a.clock = clock;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.n = m->n;
  a.xs = c->xs;
  a.mv = c->mv;
  a.rest_density = m->rest_density;
  a.stiffness = m->stiffness;
  a.exponent = m->exponent;
  a.h = h;
  a.clamp = clamp;
  a.rho = rho;
  a.pressure = pressure;
  a.sc2 = c->sc2;
  {
    PassScope ps_(c, P_WCSPH_DENSITY, st);
    k_wcsph_density<<<nb_blocks(c, a.n), c->nb_block, 0, st>>>(a);
  }
  return launch_check("wcsph density");
}

int launch_force(fs_context* c, const fs_model* m, const fs_wcsph_params* p, float* accel, float* x_out,
                 float* v_out, cudaStream_t st, bool use_lists, const fs_frame_clock* clock = nullptr) {
  ForceArgs a;
  a.clock = clock;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.use_lists = use_lists ? 1 : 0;
  a.n = m->n;
  a.xs = c->xs;
  a.vs = c->vs;
  a.sc2 = c->sc2;
  a.m = *m;
  a.h = p->smoothing_length;
  a.particle_radius = p->particle_radius;
  a.dt = p->dt;
  a.walls = make_walls(p->bound_width, p->bound_height, p->bound_length, p->boundary_damping, 0, 0.f, 0.f);
  a.accel = accel;
  a.x_out = x_out;
  a.v_out = v_out;
  {
    PassScope ps_(c, P_WCSPH_FORCE, st);
    k_wcsph_force<<<nb_blocks(c, a.n), c->nb_block, 0, st>>>(a);
  }
  return launch_check("wcsph force");
}

int validate_model(const fs_model* m, bool wcsph) {
  if (!m || m->n < 0) return set_error(FS_ERR_INVALID, "model: null or negative n");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mass || !m->gravity || m->n_worlds < 1 || !m->rest_density)
    return set_error(FS_ERR_INVALID, "model: missing particle_flags/particle_mass/gravity/rest_density");
  if (wcsph && (!m->stiffness || !m->exponent))
    return set_error(FS_ERR_INVALID, "model: WCSPH needs stiffness and exponent");
  return FS_OK;
}

}  // namespace fs

using namespace fs;

extern "C" {

int fs_wcsph_substep(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so, const fs_wcsph_params* p,
                     float* accel, fs_stream_t stream) {
  if (!c || !si || !so || !p) return set_error(FS_ERR_INVALID, "fs_wcsph_substep: null argument");
  int rc = validate_model(m, true);
  if (rc) return rc;
  if (m->n == 0) return FS_OK;
  if (!m->particle_mask || !m->viscosity || !m->surface_tension || !si->particle_q || !si->particle_qd ||
      !so->particle_q || !so->particle_qd || !so->rho || !so->pressure || !accel)
    return set_error(FS_ERR_INVALID, "fs_wcsph_substep: missing array");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_wcsph_substep: n > capacity");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const float h = p->smoothing_length;
  if ((rc = grid_build(c, si->particle_q, m->n, h * c->cell_ratio, st, m->particle_world))) return rc;
  if ((rc = wcsph_gather(c, m, si->particle_q, si->particle_qd, st))) return rc;
  if ((rc = launch_density(c, m, h, p->clamp_negative_pressure, true, so->rho, so->pressure, st))) return rc;
  return launch_force(c, m, p, accel, so->particle_q, so->particle_qd, st, true);
}

int fs_wcsph_substep_clocked(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so,
                             const fs_wcsph_params* p, float* accel, const fs_frame_clock* clock, fs_stream_t stream) {
  if (!c || !si || !so || !p || !clock) return set_error(FS_ERR_INVALID, "fs_wcsph_substep_clocked: null argument");
  int rc = validate_model(m, true);
  if (rc) return rc;
  if (m->n == 0) return FS_OK;
  if (!m->particle_mask || !m->viscosity || !m->surface_tension || !si->particle_q || !si->particle_qd ||
      !so->particle_q || !so->particle_qd || !so->rho || !so->pressure || !accel)
    return set_error(FS_ERR_INVALID, "fs_wcsph_substep_clocked: missing array");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_wcsph_substep_clocked: n > capacity");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const float h = p->smoothing_length;
  if ((rc = grid_build(c, si->particle_q, m->n, h * c->cell_ratio, st, m->particle_world, clock))) return rc;
  if ((rc = wcsph_gather(c, m, si->particle_q, si->particle_qd, st))) return rc;
  if ((rc = launch_density(c, m, h, p->clamp_negative_pressure, true, so->rho, so->pressure, st, clock))) return rc;
  if ((rc = launch_force(c, m, p, accel, so->particle_q, so->particle_qd, st, true, clock))) return rc;
  {
    PassScope ps_(c, P_OTHER, st);
    k_idle_copy<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, clock, si->particle_q, si->particle_qd, si->rho,
                                                     si->pressure, so->particle_q, so->particle_qd, so->rho,
                                                     so->pressure);
  }
  c->last_stream = st;
  return launch_check("fs_wcsph_substep_clocked");
}

int fs_wcsph_density(fs_context* c, const fs_model* m, const float* x, float h, int32_t clamp_negative, float* rho,
                     float* pressure, fs_stream_t stream) {
  if (!c || !x || !rho || !pressure) return set_error(FS_ERR_INVALID, "fs_wcsph_density: null argument");
  int rc = validate_model(m, true);
  if (rc || m->n == 0) return rc;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_wcsph_density: build the grid for these points first");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_common<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, *m, x, nullptr, c->xs, nullptr, c->mv,
                                                       c->status, c->nworlds);
  return launch_density(c, m, h, clamp_negative, true, rho, pressure, st);
}

int fs_wcsph_force_integrate(fs_context* c, const fs_model* m, const fs_state* si, fs_state* so,
                             const fs_wcsph_params* p, float* accel, fs_stream_t stream) {
  if (!c || !si || !so || !p || !accel) return set_error(FS_ERR_INVALID, "fs_wcsph_force_integrate: null argument");
  int rc = validate_model(m, true);
  if (rc || m->n == 0) return rc;
  if (c->built_n != m->n) return set_error(FS_ERR_NOGRID, "fs_wcsph_force_integrate: build the grid first");
  if (!so->rho || !so->pressure) return set_error(FS_ERR_INVALID, "fs_wcsph_force_integrate: needs state_out rho/p");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = wcsph_gather(c, m, si->particle_q, si->particle_qd, st))) return rc;
  k_gather_ratios<<<blocks_for(m->n), kBlock, 0, st>>>(m->n, c->perm, so->rho, so->pressure, c->sc2);
  if ((rc = launch_check("wcsph gather rho/p"))) return rc;
  return launch_force(c, m, p, accel, so->particle_q, so->particle_qd, st, false);
}

}  // extern "C"
