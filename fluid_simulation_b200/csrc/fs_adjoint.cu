// Adjoint (reverse-mode derivative) of one WCSPH substep (fs_wcsph.cu;
// reference SolverWCSPH.step, solver_wcsph.py:431-535), with the neighbour
// set of the step held fixed (the grid is a piecewise-constant function of
// the positions: it contributes no derivative).
//
// Forward, per dynamic particle i (j over active neighbours within h):
//   rho_i = sum_j mv_j W(r_ij)                              (self included)
//   p_i   = B_i ((rho_i / rho0_i)^gamma_i - 1)   [max(p, 0) when clamped;
//           its derivative is taken as 1 where p > 0 and 0 elsewhere]
//   P_i   = p_i / max(rho_i^2, 1e-6),  R_i = 1 / max(rho_i, 1e-6)
//   a_i   = g + sum_{j != i} c_ij d_ij,          d_ij = x_i - x_j,
//   c_ij  = (visc_ij + pres_ij) gs(r) - coh_i m_j W(max(r, r_p))
//   visc_ij = 10 nu_i m_j R_j (u_ij . d_ij) / (r^2 + 0.01 h^2),  u_ij = v_i - v_j
//   pres_ij = -m_j (P_i + P_j),                   grad W(d) = gs(r) d
//   u' = v + dt a;  x' = x + dt u';  walls(x', u')
// Given the adjoints of the outputs (xb', vb') the three passes compute:
//   prepare    elementwise: cell-order copies of the step's data, and
//              walls^T and the integrator -> ab_i
//   force      per particle k, both sides of every pair (k, j): its own term
//              of a_k (weights ab_k) and its term in a_j (weights ab_j), so
//              each thread sums into its own slot (a gather, no atomics):
//                xb_k += dc/dd-terms,  vb_k += visc terms,
//                Pb_k, Rb_k, nub_k;  then the EOS chain rule per particle:
//                rhob_k, Bb_k (stiffness), rho0b_k (rest density).
//   density    xb_k += sum_j (rhob_k mv_j + rhob_j mv_k) gs(r) d_kj
// The force pass records the neighbour lists of the step's positions; the
// density pass reuses them.
#include "fs_nbr.cuh"

namespace fs {

namespace {

// Backward of apply_walls (mode 0/1), one axis: forward p, v before the walls;
// in: pb, vb adjoints after the walls; out: adjoints before the walls.
FS_DEV void wall_axis_adjoint(float p0, float v0, float lo, float hi, float damping, bool cond, float& pb, float& vb) {
  const bool c1 = p0 < lo;
  const bool d1 = c1 && (!cond || v0 < 0.f);
  const float p1 = c1 ? lo : p0;
  const float v1 = d1 ? v0 * damping : v0;
  const bool c2 = p1 > hi;
  const bool d2 = c2 && (!cond || v1 > 0.f);
  if (d2) vb *= damping;
  if (c2) pb = 0.f;
  if (d1) vb *= damping;
  if (c1) pb = 0.f;
}

// Adjoint of integrate_velocity / integrate_positions / apply_bounds for one
// dynamic particle: returns ab (= dt * ub) and the direct xb, vb.
FS_DEV void integrate_adjoint(const Walls& w, float3 x, float3 v, float3 a, float dt, float3 xbo, float3 vbo,
                              float3& xb, float3& vb, float3& ab) {
  const float3 u = make_float3(v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z);
  const float3 p = make_float3(x.x + u.x * dt, x.y + u.y * dt, x.z + u.z * dt);
  const bool cond = w.mode != 1;
  float3 pb = xbo, ub = vbo;
  wall_axis_adjoint(p.x, u.x, w.xmin, w.xmax, w.damping, cond, pb.x, ub.x);
  wall_axis_adjoint(p.y, u.y, w.ymin, w.ymax, w.damping, cond, pb.y, ub.y);
  wall_axis_adjoint(p.z, u.z, w.zmin, w.zmax, w.damping, cond, pb.z, ub.z);
  // p = x + u dt;  u = v + dt a
  ub = make_float3(ub.x + dt * pb.x, ub.y + dt * pb.y, ub.z + dt * pb.z);
  xb = pb;
  vb = ub;
  ab = make_float3(dt * ub.x, dt * ub.y, dt * ub.z);
}

struct AdjArgs {
  GridDev g;
  NbrList L;
  int64_t n;
  fs_model m;
  const float4* xs;    // (x, flags)
  const float4* vs;    // (v, mass)
  const float* mv;     // rest_density * volume
  const float2* sc2;   // (P, R)
  const float* nu;     // viscosity, cell order
  const float* coh;    // surface_tension / mass, cell order
  float4* ab;          // (ab, 0), cell order
  float4* xr;          // (xb partial, rhob), cell order
  const float* xin;    // step input positions, original order
  const float* vin;    // step input velocities
  const float* accel;  // forward accel, original order
  const float* rho;    // forward rho, original order
  const float* pressure;
  const float* xbo;    // adjoint of particle_q out, original order
  const float* vbo;    // adjoint of particle_qd out
  float* xbi;          // adjoint of particle_q in
  float* vbi;          // adjoint of particle_qd in
  float* gb_stiffness; // += (may be null)
  float* gb_viscosity;
  float* gb_rest_density;
  float h, particle_radius, dt;
  int clamp;
  Walls walls;
};

// Cell-order copies of what the adjoint passes read (one kernel): positions
// + flags, velocities + mass, mv, (P, R) from the step's rho and pressure,
// viscosity, cohesion / mass, and ab from the walls / integrator adjoint.
__global__ void k_adj_prepare(AdjArgs a, float* __restrict__ nu, float* __restrict__ coh, float4* __restrict__ xs,
                              float4* __restrict__ vs, float* __restrict__ mv, float2* __restrict__ sc2) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int32_t i = a.g.perm[s];
  const fs_model& m = a.m;
  const float3 x = ld3(a.xin, i), v = ld3(a.vin, i);
  const int pf = particle_pf(m.particle_flags, m.particle_mask, i);
  const int w = (a.g.nworlds > 0 && m.particle_world) ? world_index(m.particle_world[i], a.g.nworlds) : 0;
  const float4 x4 = make_float4(x.x, x.y, x.z, pack_pf(pf, w));
  const float mass = m.particle_mass[i];
  xs[s] = x4;
  vs[s] = make_float4(v.x, v.y, v.z, mass);
  const float rd = m.rest_density[i];
  mv[s] = rd * (mass / fmaxf(rd, 1.0e-6f));
  const float r = a.rho[i];
  sc2[s] = make_float2(a.pressure[i] / fmaxf(r * r, 1.0e-6f), 1.0f / fmaxf(r, 1.0e-6f));
  nu[s] = m.viscosity[i];
  coh[s] = m.surface_tension[i] / mass;
  float3 ab = make_float3(0.f, 0.f, 0.f);
  if (pf & PF_DYNAMIC) {
    float3 xb, vb;
    integrate_adjoint(walls_of(a.walls, a.g, w), x, v, ld3(a.accel, i), a.dt, ld3(a.xbo, i), ld3(a.vbo, i), xb, vb,
                      ab);
  }
  a.ab[s] = make_float4(ab.x, ab.y, ab.z, 0.f);
}

// d (c d) / d(d) applied to ab:  rb = c ab + (ab . d) dc/dd, and the
// velocity adjoint ub of the pair, for the term of a_i with neighbour j.
struct PairAdj {
  float3 rb, ub;
  float pb_sum;  // coefficient of (P_i + P_j):  -m_j gs (ab . d)
  float nub;     // d/d nu_i
  float rb_j;    // d/d R_j
};

FS_DEV PairAdj pair_adjoint(const Cubic& K, float h, float particle_radius, float3 d, float r2, float3 u, float3 ab,
                            float nu_i, float coh_i, float m_j, float R_j, float Psum) {
  PairAdj o;
  float r, rinv;
  r_and_inv(r2, r, rinv);
  const float q = r * K.inv_h;
  // gs(r) and its derivative d gs / dr (Cubic.grad_scale)
  float gs = 0.f, dgs = 0.f;
  if (r > 1.0e-5f && q <= 1.f) {
    if (q <= 0.5f) {
      gs = K.g_in * fmaf(3.f, q, -2.f);
      dgs = K.g_in * 3.f * K.inv_h;
    } else {
      const float t = 1.f - q;
      gs = K.g_out * t * t * rinv;
      dgs = K.g_out * (-2.f * t * K.inv_h * rinv - t * t * rinv * rinv);
    }
  }
  const float eps = 0.01f * (h * h);
  const float den = 1.0f / (r2 + eps);
  const float ud = u.x * d.x + u.y * d.y + u.z * d.z;
  const float kv = 10.f * nu_i * m_j * R_j;
  const float visc = kv * ud * den;
  const float A = visc - m_j * Psum;
  // cohesion -coh_i m_j W(s) with s = max(r, r_p)
  const float s = fmaxf(r, particle_radius);
  const float wc = coh_i * m_j * K.w(s);
  float dwc = 0.f;  // d wc / dr
  if (coh_i != 0.f && r > particle_radius && s > 1.0e-5f) dwc = coh_i * m_j * K.grad_scale(s, 1.0f / s) * s;
  const float c = A * gs - wc;
  const float abd = ab.x * d.x + ab.y * d.y + ab.z * d.z;
  // dc/dd = gs dA/dd + (A dgs - dwc) d / r
  //   dA/dd = kv (u den - 2 ud d den^2)
  const float radial = (A * dgs - dwc) * rinv - 2.f * kv * ud * den * den * gs;
  const float tang = kv * den * gs;
  o.rb = make_float3(c * ab.x + abd * (tang * u.x + radial * d.x), c * ab.y + abd * (tang * u.y + radial * d.y),
                     c * ab.z + abd * (tang * u.z + radial * d.z));
  o.ub = make_float3(abd * tang * d.x, abd * tang * d.y, abd * tang * d.z);
  o.pb_sum = -m_j * gs * abd;
  o.nub = abd * gs * 10.f * m_j * R_j * ud * den;
  o.rb_j = abd * gs * 10.f * nu_i * m_j * ud * den;
  return o;
}

__global__ void FS_NB_BOUNDS k_adj_force(AdjArgs a) {
  lists_recorded(a.L);
  for_slots(a.n, [&](int64_t s) {
    const float4 xk = a.xs[s];
    const int32_t i = a.g.perm[s];
    const int pfk = pf_of(xk);
    if (!(pfk & PF_ACTIVE)) {  // untouched by the step: identity
      a.L.cnt[s] = 0;
      a.xr[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      st3(a.xbi, i, ld3(a.xbo, i));
      st3(a.vbi, i, ld3(a.vbo, i));
      return;
    }
    const float4 vk = a.vs[s];
    const float m_k = vk.w;
    const float2 PRk = a.sc2[s];
    const float nu_k = a.nu[s], coh_k = a.coh[s];
    float3 xb = make_float3(0.f, 0.f, 0.f), vb = make_float3(0.f, 0.f, 0.f), abk = make_float3(0.f, 0.f, 0.f);
    if (pfk & PF_DYNAMIC) {
      integrate_adjoint(walls_of(a.walls, a.g, world_of(xk)), xyz(xk), xyz(vk), ld3(a.accel, i), a.dt, ld3(a.xbo, i),
                        ld3(a.vbo, i), xb, vb, abk);
    } else {
      xb = ld3(a.xbo, i);
      vb = ld3(a.vbo, i);
    }
    const Cubic K(a.h);
    const float h2m = a.h * a.h * kSupportMargin;
    float Pb = 0.f, Rb = 0.f, nub = 0.f;
    record_list<false>(a.g, a.xs, (int)s, xk, a.h, h2m, a.L);
    visit<false, true>(a.g, a.xs, (int)s, xk, a.h, h2m, a.L, true, [&](int t, float4 xj) {
      const float3 d = make_float3(xk.x - xj.x, xk.y - xj.y, xk.z - xj.z);
      const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
      if (r2 == 0.f) return;  // the forward skips coincident pairs
      const float4 vj = __ldg(a.vs + t);
      const float2 PRj = __ldg(a.sc2 + t);
      const float3 u = make_float3(vk.x - vj.x, vk.y - vj.y, vk.z - vj.z);
      const float Psum = PRk.x + PRj.x;
      if (pfk & PF_DYNAMIC) {  // term of a_k with neighbour j
        const PairAdj o = pair_adjoint(K, a.h, a.particle_radius, d, r2, u, abk, nu_k, coh_k, vj.w, PRj.y, Psum);
        xb = make_float3(xb.x + o.rb.x, xb.y + o.rb.y, xb.z + o.rb.z);
        vb = make_float3(vb.x + o.ub.x, vb.y + o.ub.y, vb.z + o.ub.z);
        Pb += o.pb_sum;
        nub += o.nub;
      }
      if (pf_of(xj) & PF_DYNAMIC) {  // term of a_j with neighbour k: d_jk = -d, u_jk = -u
        const float4 abj4 = __ldg(a.ab + t);
        const float3 abj = make_float3(abj4.x, abj4.y, abj4.z);
        const float3 dn = make_float3(-d.x, -d.y, -d.z), un = make_float3(-u.x, -u.y, -u.z);
        const PairAdj o = pair_adjoint(K, a.h, a.particle_radius, dn, r2, un, abj, __ldg(a.nu + t), __ldg(a.coh + t),
                                       m_k, PRk.y, Psum);
        xb = make_float3(xb.x - o.rb.x, xb.y - o.rb.y, xb.z - o.rb.z);
        vb = make_float3(vb.x - o.ub.x, vb.y - o.ub.y, vb.z - o.ub.z);
        Pb += o.pb_sum;
        Rb += o.rb_j;
      }
    });
    // P = p / max(rho^2, 1e-6), R = 1 / max(rho, 1e-6), then the EOS
    const float rho = a.rho[i], p = a.pressure[i];
    const float rr = rho * rho;
    const float inv_rr = 1.0f / fmaxf(rr, 1.0e-6f);
    float rhob = 0.f;
    if (rr > 1.0e-6f) rhob -= 2.f * Pb * p * inv_rr / rho;
    if (rho > 1.0e-6f) rhob -= Rb / rr;
    const float pb = Pb * inv_rr;
    const float B = a.m.stiffness[i], gam = a.m.exponent[i], rd = a.m.rest_density[i];
    const float rho0 = fmaxf(rd, 1.0e-6f);
    const float ratio = rho / rho0;
    const float pw = powf(ratio, gam);
    const float p_raw = B * (pw - 1.0f);
    // max(p, 0) has no derivative at p = 0; there the clamped side is taken
    // (d/dp = 0), as for a ReLU: the pressure responds only where p > 0
    if (!(a.clamp && !(p_raw > 0.f)) && pb != 0.f) {
      const float dp_dratio = B * gam * (ratio > 0.f ? pw / ratio : 0.f);
      rhob += pb * dp_dratio / rho0;
      if (a.gb_stiffness) a.gb_stiffness[i] += pb * (pw - 1.0f);
      if (a.gb_rest_density && rd > 1.0e-6f) a.gb_rest_density[i] += -pb * dp_dratio * ratio / rho0;
    }
    if (a.gb_viscosity) a.gb_viscosity[i] += nub;
    a.xr[s] = make_float4(xb.x, xb.y, xb.z, rhob);
    st3(a.vbi, i, vb);
  });
}

__global__ void FS_NB_BOUNDS k_adj_density(AdjArgs a) {
  for_slots(a.n, [&](int64_t s) {
    const float4 xk = a.xs[s];
    if (!(pf_of(xk) & PF_ACTIVE)) return;  // written by the force pass
    const int32_t i = a.g.perm[s];
    const float4 xr = a.xr[s];
    const float mv_k = a.mv[s];
    const Cubic K(a.h);
    float3 xb = make_float3(xr.x, xr.y, xr.z);
    const bool lists_ok = lists_usable(a.L);
    visit<false, false>(a.g, a.xs, (int)s, xk, a.h, a.h * a.h * kSupportMargin, a.L, lists_ok, [&](int t, float4 xj) {
      const float dx = xk.x - xj.x, dy = xk.y - xj.y, dz = xk.z - xj.z;
      float r, rinv;
      r_and_inv(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), r, rinv);
      const float w = (xr.w * __ldg(a.mv + t) + __ldg(&a.xr[t].w) * mv_k) * K.grad_scale(r, rinv);
      xb = make_float3(fmaf(w, dx, xb.x), fmaf(w, dy, xb.y), fmaf(w, dz, xb.z));
    });
    st3(a.xbi, i, xb);
  });
}


}  // namespace
}  // namespace fs

using namespace fs;

extern "C" {

int fs_wcsph_substep_adjoint(fs_context* c, const fs_model* m, const fs_state* si, const float* rho,
                             const float* pressure, const float* accel, const float* adj_x_out, const float* adj_v_out,
                             float* adj_x_in, float* adj_v_in, float* adj_stiffness, float* adj_viscosity,
                             float* adj_rest_density, const fs_wcsph_params* p, fs_stream_t stream) {
  if (!c || !m || !si || !p) return set_error(FS_ERR_INVALID, "fs_wcsph_substep_adjoint: null argument");
  if (m->n < 0) return set_error(FS_ERR_INVALID, "fs_wcsph_substep_adjoint: negative n");
  if (m->n == 0) return FS_OK;
  if (!m->particle_flags || !m->particle_mask || !m->particle_mass || !m->gravity || m->n_worlds < 1 ||
      !m->rest_density || !m->viscosity || !m->surface_tension || !m->stiffness || !m->exponent ||
      !si->particle_q || !si->particle_qd || !rho || !pressure || !accel || !adj_x_out || !adj_v_out || !adj_x_in ||
      !adj_v_in)
    return set_error(FS_ERR_INVALID, "fs_wcsph_substep_adjoint: missing array");
  if (m->n > c->capacity) return set_error(FS_ERR_CAPACITY, "fs_wcsph_substep_adjoint: n > capacity");
  DeviceGuard dg(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = m->n;
  const float h = p->smoothing_length;
  int rc;
  if ((rc = grid_build(c, si->particle_q, n, h * c->cell_ratio, st, m->particle_world))) return rc;
  AdjArgs a;
  a.g = grid_view(c);
  a.L = nbr_list(c);
  a.n = n;
  a.m = *m;
  a.xs = c->xs;
  a.vs = c->vs;
  a.mv = c->mv;
  a.sc2 = c->sc2;
  a.nu = c->sc1;
  a.coh = c->sc1b;
  a.ab = c->xs2;
  a.xr = c->vs2;
  a.xin = si->particle_q;
  a.vin = si->particle_qd;
  a.accel = accel;
  a.rho = rho;
  a.pressure = pressure;
  a.xbo = adj_x_out;
  a.vbo = adj_v_out;
  a.xbi = adj_x_in;
  a.vbi = adj_v_in;
  a.gb_stiffness = adj_stiffness;
  a.gb_viscosity = adj_viscosity;
  a.gb_rest_density = adj_rest_density;
  a.h = h;
  a.particle_radius = p->particle_radius;
  a.dt = p->dt;
  a.clamp = p->clamp_negative_pressure;
  a.walls = make_walls(p->bound_width, p->bound_height, p->bound_length, p->boundary_damping, 0, 0.f, 0.f);
  {
    PassScope ps_(c, P_ADJ_INTEGRATE, st);
    k_adj_prepare<<<blocks_for(n), kBlock, 0, st>>>(a, c->sc1, c->sc1b, c->xs, c->vs, c->mv, c->sc2);
  }
  {
    PassScope ps_(c, P_ADJ_FORCE, st);
    k_adj_force<<<nb_blocks(c, n), c->nb_block, 0, st>>>(a);
  }
  {
    PassScope ps_(c, P_ADJ_DENSITY, st);
    k_adj_density<<<nb_blocks(c, n), c->nb_block, 0, st>>>(a);
  }
  c->last_stream = st;
  return launch_check("fs_wcsph_substep_adjoint");
}

}  // extern "C"
