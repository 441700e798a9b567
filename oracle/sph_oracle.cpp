// CPU oracle for the particle-fluid hot path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, pass by pass, the reference solvers of
// SParksLz/fluid_simulation so that the CUDA library can be checked against it:
//   solver/sph/solver_wcsph.py  (WCSPH, lines 21-305 and step 431-535)
//   solver/sph/solver_dfsph.py  (DFSPH, lines 24-442 and step 574-898)
//   solver/pbf/solver_pbf.py    (PBF,   lines 24-517 and step 671-954)
//   solver/apic/solver_apic.py  (particle separation, lines 193-266 and
//                                _apply_particle_separation 1003-1064)
// and the third-party neighbour search those solvers call, warp-lang 1.17.0
// `wp.HashGrid` (not vendored by the reference; its published algorithm is
// restated in `Grid` below).  Only tests, the smoke check and the CPU-baseline
// leg of the benchmark may load this library; the product never does.
//
// Arithmetic follows the reference's expression trees operation by operation
// (build with -ffp-contract=off so that no FMA is formed), templated on the
// scalar type so the same code gives the FP32 oracle and the FP64 oracle.
// Each per-particle pass is an OpenMP loop over particles: every particle owns
// its outputs, as in the reference kernels, so the result does not depend on
// the thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- vec3 ----
template <class T>
struct V3 {
  T x, y, z;
};
template <class T> inline V3<T> mk(T a, T b, T c) { return V3<T>{a, b, c}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return mk(s * a.x, s * a.y, s * a.z); }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return mk(a.x / s, a.y / s, a.z / s); }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline V3<T> ld(const T* p, int64_t i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
template <class T> inline void st(T* p, int64_t i, V3<T> v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
template <class T> inline T tmax(T a, T b) { return a > b ? a : b; }
template <class T> inline T tmin(T a, T b) { return a < b ? a : b; }
template <class T> inline T cube(T x) { return x * x * x; }
template <class T> inline T square(T x) { return x * x; }

// Warp's float32 pi constant when T = float, the double value otherwise.
template <class T> inline T kPi() { return T(3.14159265358979323846); }

// ParticleFlags.ACTIVE (newton 1.6.0) is bit 0.
constexpr int32_t kActive = 1;
inline bool active(int32_t f) { return (f & kActive) != 0; }
inline bool dynamic(int32_t f, int32_t m) { return active(f) && m == 0; }

// ------------------------------------------------------------- kernels ----
// Cubic spline of solver_wcsph.py:21-34 / solver_dfsph.py:24-38.
template <class T>
inline T cubic_w(T r_norm, T h) {
  T res = T(0);
  T k = T(8) / (kPi<T>() * cube(h));
  T q = r_norm / h;
  if (q <= T(1)) {
    if (q <= T(0.5)) {
      T q2 = square(q);
      T q3 = q2 * q;
      res = k * (T(6) * q3 - T(6) * q2 + T(1));
    } else {
      res = T(2) * k * cube(T(1) - q);
    }
  }
  return res;
}

// Cubic-spline gradient of solver_wcsph.py:37-51 / solver_dfsph.py:41-54.
template <class T>
inline V3<T> cubic_dw(V3<T> r, T h) {
  V3<T> res = mk(T(0), T(0), T(0));
  T r_norm = length(r);
  T k = T(8) / (kPi<T>() * cube(h));
  T q = r_norm / h;
  if (r_norm > T(1.0e-5) && q <= T(1)) {
    V3<T> grad_q = r / (r_norm * h);
    if (q <= T(0.5)) {
      res = (T(6) * k * q * (T(3) * q - T(2))) * grad_q;
    } else {
      T q_term = T(1) - q;
      res = (T(-6) * k * q_term * q_term) * grad_q;
    }
  }
  return res;
}

// Poly6 of solver_pbf.py:24-32 (named get_cubic there).
template <class T>
inline T poly6_w(T r_norm, T h) {
  T res = T(0);
  if (h > T(0) && r_norm < h) {
    T h2 = h * h;
    T rhs = h2 - r_norm * r_norm;
    T k = T(315) / (T(64) * kPi<T>() * cube(cube(h)));
    res = k * cube(rhs);
  }
  return res;
}

// Spiky gradient of solver_pbf.py:36-45 (named get_cubic_derivative there).
template <class T>
inline V3<T> spiky_dw(V3<T> r, T h) {
  V3<T> res = mk(T(0), T(0), T(0));
  T r_norm = length(r);
  if (h > T(0) && r_norm > T(1.0e-6) && r_norm < h) {
    T h6 = cube(h) * cube(h);
    T coeff = T(-45) / (kPi<T>() * h6);
    T term = (h - r_norm) * (h - r_norm) / r_norm;
    res = (coeff * term) * r;
  }
  return res;
}

// ---------------------------------------------------------------- grid ----
// Restatement of warp-lang 1.17.0 wp.HashGrid (native hashgrid.h/.cpp):
//  * build(points, radius): cell_width = radius, cell_width_inv = 1/radius
//    (float32); each point gets the physical cell of its virtual integer cell
//    coords (p * inv converted to int); the pairs (cell, id) are radix sorted
//    (stable, so ids stay ascending inside a cell); cell_starts/ends are the
//    first/one-past-last sorted slot of each occupied cell.
//  * physical cell: coords shifted by 2^20, clamped at 0, taken modulo the
//    grid dims, linearised x-fastest.
//  * query(pos, r): per axis start = int((pos - r) * inv),
//    end = min(int((pos + r) * inv), start + dim - 1); cells are visited
//    z-outer, y-middle, x-inner; each cell's slots in sorted order;
//    candidates are NOT distance filtered.
// Float-to-int conversion: warp converts with a C cast (truncation toward
// zero).  That choice is not pinned by any reference test; `rounding`
// selects truncation (0, the reference geometry) or floor (1).  NaN maps to
// cell 0 and values beyond +-2^29 saturate, in this oracle and on the GPU.
struct GridCfg {
  int32_t dim_x, dim_y, dim_z;
  int32_t rounding;  // 0 = truncate toward zero, 1 = floor
};

inline int32_t to_cell(float v, int32_t rounding) {
  if (!(v == v)) return 0;
  if (rounding == 1) v = std::floor(v);
  if (v > 536870912.0f) return 536870912;
  if (v < -536870912.0f) return -536870912;
  return (int32_t)v;  // truncation toward zero
}
inline int32_t to_cell(double v, int32_t rounding) {
  if (!(v == v)) return 0;
  if (rounding == 1) v = std::floor(v);
  if (v > 536870912.0) return 536870912;
  if (v < -536870912.0) return -536870912;
  return (int32_t)v;
}

inline int32_t phys_cell(const GridCfg& g, int32_t x, int32_t y, int32_t z) {
  const int32_t origin = 1 << 20;
  x += origin;
  y += origin;
  z += origin;
  x = std::max(0, x);
  y = std::max(0, y);
  z = std::max(0, z);
  int32_t cx = x % g.dim_x, cy = y % g.dim_y, cz = z % g.dim_z;
  return cz * (g.dim_x * g.dim_y) + cy * g.dim_x + cx;
}

template <class T>
struct Grid {
  GridCfg cfg{};
  T inv = T(0);
  int64_t n = 0;
  std::vector<int32_t> point_ids, point_cells, cell_starts, cell_ends;

  void build(const T* x, int64_t count, T radius, const GridCfg& c) {
    cfg = c;
    n = count;
    inv = T(1) / radius;
    const int64_t ncell = (int64_t)c.dim_x * c.dim_y * c.dim_z;
    std::vector<int32_t> key(count);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
      V3<T> p = ld(x, i);
      key[i] = phys_cell(c, to_cell(p.x * inv, c.rounding), to_cell(p.y * inv, c.rounding),
                         to_cell(p.z * inv, c.rounding));
    }
    // stable counting sort on the cell key == stable radix sort of (key, id)
    cell_starts.assign(ncell, 0);
    cell_ends.assign(ncell, 0);
    std::vector<int32_t> cnt(ncell, 0);
    for (int64_t i = 0; i < count; ++i) cnt[key[i]]++;
    std::vector<int64_t> off(ncell + 1, 0);
    for (int64_t k = 0; k < ncell; ++k) off[k + 1] = off[k] + cnt[k];
    point_ids.assign(count, 0);
    point_cells.assign(count, 0);
    std::vector<int64_t> fill(off.begin(), off.end() - 1);
    for (int64_t i = 0; i < count; ++i) {
      int64_t s = fill[key[i]]++;
      point_ids[s] = (int32_t)i;
      point_cells[s] = key[i];
    }
    for (int64_t k = 0; k < ncell; ++k)
      if (cnt[k]) {
        cell_starts[k] = (int32_t)off[k];
        cell_ends[k] = (int32_t)off[k + 1];
      }
  }

  // Calls f(j) for every candidate of a query at pos with radius r, in the
  // reference's visiting order.
  template <class F>
  inline void query(V3<T> pos, T r, F&& f) const {
    const int32_t x0 = to_cell((pos.x - r) * inv, cfg.rounding);
    const int32_t y0 = to_cell((pos.y - r) * inv, cfg.rounding);
    const int32_t z0 = to_cell((pos.z - r) * inv, cfg.rounding);
    const int32_t x1 = std::min(to_cell((pos.x + r) * inv, cfg.rounding), x0 + cfg.dim_x - 1);
    const int32_t y1 = std::min(to_cell((pos.y + r) * inv, cfg.rounding), y0 + cfg.dim_y - 1);
    const int32_t z1 = std::min(to_cell((pos.z + r) * inv, cfg.rounding), z0 + cfg.dim_z - 1);
    for (int32_t z = z0; z <= z1; ++z)
      for (int32_t y = y0; y <= y1; ++y)
        for (int32_t xx = x0; xx <= x1; ++xx) {
          const int32_t c = phys_cell(cfg, xx, y, z);
          const int32_t e = cell_ends[c];
          for (int32_t s = cell_starts[c]; s < e; ++s) f(point_ids[s]);
        }
  }
};

}  // namespace

// ------------------------------------------------------------ C structs ----
extern "C" {

typedef struct {
  int64_t n;
  int32_t n_worlds;
  const int32_t* flags;     // Model.particle_flags
  const int32_t* mask;      // Model.sph.particle_mask
  const int32_t* world;     // Model.particle_world
  const void* mass;         // Model.particle_mass
  const void* gravity;      // Model.gravity [n_worlds][3]
  const void* rest_density; // Model.sph.rest_density
  const void* surface_tension;
  const void* viscosity;
  const void* stiffness;    // WCSPH only
  const void* exponent;     // WCSPH only
} OracleModel;

typedef struct {
  void* q;    // particle_q  [n][3]
  void* qd;   // particle_qd [n][3]
  void* rho;
  void* pressure;        // WCSPH
  void* factor;          // DFSPH
  void* rho_star;
  void* d_rho_dt;
  void* kappa;
  void* kappa_v;
  int32_t* neighbor_count;  // DFSPH, PBF
  void* v_star;          // DFSPH [n][3]
  void* pbf_lambda;      // PBF
  void* delta_p;         // PBF [n][3]
} OracleState;

typedef struct {
  double particle_radius;  // config value (<= 0 selects particle_max_radius)
  double particle_max_radius;
  double particle_length;
  double smoothing_length_coff;
  double bound_width, bound_height, bound_length;
  double boundary_damping;
  int32_t clamp_negative_pressure;
  GridCfg grid;
} OracleWcsphCfg;

typedef struct {
  int32_t max_rho_iterations, max_vel_iterations, warm_start, min_neighbors_for_factor;
  double eta_density, eta_divergence, max_kappa, max_kappa_v;
  double particle_radius, particle_max_radius, particle_length, smoothing_length_coff;
  double bound_width, bound_height, bound_length, boundary_damping;
  GridCfg grid;
} OracleDfsphCfg;

typedef struct {
  int32_t max_iterations, min_neighbors_for_lambda, rebuild_grid_each_iteration;
  double lambda_epsilon, scorr_k, scorr_n, scorr_q, max_delta_position, xsph_c;
  double particle_radius, particle_max_radius, particle_length, smoothing_length_coff;
  double bound_width, bound_height, bound_length, boundary_damping, boundary_epsilon;
  GridCfg grid;
} OraclePbfCfg;

typedef struct {
  double rest_dist, query_radius, strength;
  double bound_lo[3], bound_hi[3];
  double wall_band, wall_margin;
  int32_t iterations;
  GridCfg grid;
} OracleSeparationCfg;

typedef struct {
  int32_t rho_iterations;   // density iterations entered (kernels launched for d_rho_dt)
  int32_t vel_iterations;   // divergence iterations entered
  double last_density_residual;
  double last_divergence_residual;
} OracleDfsphInfo;

}  // extern "C"

namespace {

template <class T>
struct Model {
  int64_t n;
  int32_t nw;
  const int32_t *flags, *mask, *world;
  const T *mass, *gravity, *rest_density, *surface_tension, *viscosity, *stiffness, *exponent;
  explicit Model(const OracleModel& m)
      : n(m.n), nw(m.n_worlds), flags(m.flags), mask(m.mask), world(m.world),
        mass((const T*)m.mass), gravity((const T*)m.gravity), rest_density((const T*)m.rest_density),
        surface_tension((const T*)m.surface_tension), viscosity((const T*)m.viscosity),
        stiffness((const T*)m.stiffness), exponent((const T*)m.exponent) {}
  V3<T> g(int64_t i) const {
    int32_t w = world ? world[i] : 0;
    return ld(gravity, (int64_t)std::max(w, 0));
  }
};

// compute_particle_volume, solver_wcsph.py:110-116 (same in DFSPH, PBF)
template <class T>
void particle_volume(const Model<T>& m, std::vector<T>& vol) {
  vol.resize(m.n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) vol[i] = m.mass[i] / tmax(m.rest_density[i], T(1.0e-6));
}

// compute_density_pressure, solver_wcsph.py:120-158 (pressure == nullptr:
// compute_density of solver_dfsph.py:107-133 / solver_pbf.py:115-141, which
// differ from it only in using the poly6 kernel for PBF).
template <class T, bool POLY6>
void density_pass(const Model<T>& m, const Grid<T>& g, const T* x, const std::vector<T>& vol, T h,
                  T* rho, T* pressure, bool clamp) {
#pragma omp parallel for schedule(static)
  for (int64_t tid = 0; tid < m.n; ++tid) {
    const int64_t i = g.point_ids[tid];
    if (!active(m.flags[i])) {
      rho[i] = T(0);
      if (pressure) pressure[i] = T(0);
      continue;
    }
    const V3<T> xi = ld(x, i);
    T acc = T(0);
    g.query(xi, h, [&](int32_t j) {
      if (!active(m.flags[j])) return;
      V3<T> d = xi - ld(x, j);
      T mj = m.rest_density[j] * vol[j];
      acc += mj * (POLY6 ? poly6_w(length(d), h) : cubic_w(length(d), h));
    });
    rho[i] = acc;
    if (pressure) {
      T p = m.stiffness[i] * (std::pow(acc / tmax(m.rest_density[i], T(1.0e-6)), m.exponent[i]) - T(1));
      if (clamp) p = tmax(p, T(0));
      pressure[i] = p;
    }
  }
}

// cal_acc_with_non_pressure, solver_wcsph.py:64-90 (PBF variant 59-87 skips
// the zero-coefficient branches: PBF == true).
template <class T, bool PBF>
inline V3<T> acc_non_pressure(V3<T> a, T rho_nei, V3<T> vel, V3<T> vel_nei, T mass, T mass_nei, T mu, T gamma,
                              V3<T> d, T e_dist, T distance, T h) {
  if (!PBF || gamma != T(0)) {
    T w = PBF ? poly6_w(e_dist, h) : cubic_w(e_dist, h);
    a = a - ((gamma / mass * mass_nei) * d) * w;
  }
  if (!PBF || mu != T(0)) {
    T vcn = dot(vel - vel_nei, d);
    if (!PBF || vcn != T(0)) {
      V3<T> dw = PBF ? spiky_dw(d, h) : cubic_dw(d, h);
      a = a + (T(10) * mu * (mass_nei / tmax(rho_nei, T(1.0e-6))) * vcn / (distance * distance + T(0.01) * (h * h))) * dw;
    }
  }
  return a;
}

// cal_acc_with_pressure, solver_wcsph.py:93-106
template <class T>
inline V3<T> acc_pressure(V3<T> a, V3<T> d, T p, T pn, T rho, T rn, T mn, T h) {
  T dpi = p / tmax(rho * rho, T(1.0e-6));
  T dpn = pn / tmax(rn * rn, T(1.0e-6));
  return a + ((-mn) * (dpi + dpn)) * cubic_dw(d, h);
}

// acceleration_wcsph (solver_wcsph.py:162-228) when PRESSURE; else
// acceleration_non_pressure (solver_dfsph.py:178-226; solver_pbf.py:145-189
// when PBF, which has no gravity term).
template <class T, bool PRESSURE, bool PBF>
void accel_pass(const Model<T>& m, const Grid<T>& g, const T* x, const T* v, const T* rho, const T* pressure,
                T particle_radius, T h, T* accel) {
#pragma omp parallel for schedule(static)
  for (int64_t tid = 0; tid < m.n; ++tid) {
    const int64_t i = g.point_ids[tid];
    if (!dynamic(m.flags[i], m.mask[i])) {
      st(accel, i, mk(T(0), T(0), T(0)));
      continue;
    }
    const V3<T> xi = ld(x, i);
    const V3<T> vi = ld(v, i);
    const T rho_i = rho[i];
    const T p_i = PRESSURE ? pressure[i] : T(0);
    V3<T> acc = mk(T(0), T(0), T(0));
    g.query(xi, h, [&](int32_t j) {
      if (j == i || !active(m.flags[j])) return;
      V3<T> d = xi - ld(x, j);
      T dist = length(d);
      acc = acc_non_pressure<T, PBF>(acc, rho[j], vi, ld(v, j), m.mass[i], m.mass[j], m.viscosity[i],
                                     m.surface_tension[i], d, tmax(dist, particle_radius), dist, h);
      if (PRESSURE) acc = acc_pressure(acc, d, p_i, pressure[j], rho_i, rho[j], m.mass[j], h);
    });
    if (PBF)
      st(accel, i, acc);
    else
      st(accel, i, acc + m.g(i));
  }
}

// apply_bounds: WCSPH (solver_wcsph.py:264-305, conditional damping, mode 0),
// DFSPH (solver_dfsph.py:407-442, unconditional damping, mode 1),
// PBF (solver_pbf.py:467-517, inset walls + conditional damping, mode 2).
template <class T>
void apply_bounds(const Model<T>& m, T* x, T* v, V3<T> size, T damping, int mode, T radius, T eps) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) continue;
    V3<T> p = ld(x, i), u = ld(v, i);
    T xmin = -size.x, xmax = size.x, ymin = -size.y, ymax = size.y, zmin = T(0), zmax = size.z * T(2);
    if (mode == 2) {
      xmin = -size.x + radius + eps;
      xmax = size.x - radius - eps;
      ymin = -size.y + radius + eps;
      ymax = size.y - radius - eps;
      zmin = radius + eps;
      zmax = size.z * T(2) - radius - eps;
    }
    const bool cond = mode != 1;
    if (p.x < xmin) { p.x = xmin; if (!cond || u.x < T(0)) u.x = u.x * damping; }
    if (p.x > xmax) { p.x = xmax; if (!cond || u.x > T(0)) u.x = u.x * damping; }
    if (p.y < ymin) { p.y = ymin; if (!cond || u.y < T(0)) u.y = u.y * damping; }
    if (p.y > ymax) { p.y = ymax; if (!cond || u.y > T(0)) u.y = u.y * damping; }
    if (p.z < zmin) { p.z = zmin; if (!cond || u.z < T(0)) u.z = u.z * damping; }
    if (p.z > zmax) { p.z = zmax; if (!cond || u.z > T(0)) u.z = u.z * damping; }
    st(x, i, p);
    st(v, i, u);
  }
}

template <class T>
T particle_radius_of(double cfg_radius, double max_radius) {
  return T(cfg_radius > 0.0 ? cfg_radius : max_radius);
}

// ------------------------------------------------------------ WCSPH step ----
// SolverWCSPH.step, solver_wcsph.py:431-535.
template <class T>
void wcsph_step(const OracleModel& om, const OracleState& si, OracleState& so, const OracleWcsphCfg& c, T dt,
                T* accel) {
  Model<T> m(om);
  if (m.n == 0) return;
  const T h = T(c.particle_length * c.smoothing_length_coff);
  const T pr = particle_radius_of<T>(c.particle_radius, c.particle_max_radius);
  std::vector<T> vol;
  particle_volume(m, vol);
  Grid<T> g;
  const T* xin = (const T*)si.q;
  const T* vin = (const T*)si.qd;
  g.build(xin, m.n, h, c.grid);
  T* rho = (T*)so.rho;
  T* p = (T*)so.pressure;
  density_pass<T, false>(m, g, xin, vol, h, rho, p, c.clamp_negative_pressure != 0);
  accel_pass<T, true, false>(m, g, xin, vin, rho, p, pr, h, accel);
  T* xo = (T*)so.q;
  T* vo = (T*)so.qd;
  // integrate_velocity (232-244) and integrate_positions (248-260)
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) {
      st(vo, i, ld(vin, i));
      st(xo, i, ld(xin, i));
      continue;
    }
    V3<T> nv = ld(vin, i) + dt * ld(accel, i);
    st(vo, i, nv);
    st(xo, i, ld(xin, i) + nv * dt);
  }
  apply_bounds(m, xo, vo, mk(T(c.bound_width), T(c.bound_height), T(c.bound_length)), T(c.boundary_damping), 0,
               T(0), T(0));
}

// ------------------------------------------------------------ DFSPH step ----
template <class T>
void factor_pass(const Model<T>& m, const Grid<T>& g, const T* x, T h, int min_nb, T* factor, int32_t* count_out) {
  // compute_factor_dfsph, solver_dfsph.py:137-174
#pragma omp parallel for schedule(static)
  for (int64_t tid = 0; tid < m.n; ++tid) {
    const int64_t i = g.point_ids[tid];
    if (!active(m.flags[i])) {
      factor[i] = T(0);
      count_out[i] = 0;
      continue;
    }
    const V3<T> xi = ld(x, i);
    V3<T> sg = mk(T(0), T(0), T(0));
    T sq = T(0);
    int32_t count = 0;
    g.query(xi, h, [&](int32_t j) {
      if (!active(m.flags[j])) return;
      if (j != i) count += 1;
      V3<T> gr = m.mass[j] * cubic_dw(xi - ld(x, j), h);
      sg = sg + gr;
      sq += dot(gr, gr);
    });
    count_out[i] = count;
    T denom = dot(sg, sg) + sq;
    factor[i] = (count < min_nb || denom < T(1.0e-6)) ? T(0) : T(1) / denom;
  }
}

template <class T>
void drho_pass(const Model<T>& m, const Grid<T>& g, const T* x, const T* v, T h, T* d_rho_dt) {
  // compute_density_change_rate, solver_dfsph.py:246-272
#pragma omp parallel for schedule(static)
  for (int64_t tid = 0; tid < m.n; ++tid) {
    const int64_t i = g.point_ids[tid];
    if (!active(m.flags[i])) {
      d_rho_dt[i] = T(0);
      continue;
    }
    const V3<T> xi = ld(x, i), vi = ld(v, i);
    T acc = T(0);
    g.query(xi, h, [&](int32_t j) {
      if (!active(m.flags[j])) return;
      V3<T> gw = cubic_dw(xi - ld(x, j), h);
      acc += m.mass[j] * dot(vi - ld(v, j), gw);
    });
    d_rho_dt[i] = acc;
  }
}

template <class T>
void correction_pass(const Model<T>& m, const Grid<T>& g, const T* x, T* v_star, const T* rho, const T* kappa, T h,
                     T dt) {
  // apply_constant_density_correction (solver_dfsph.py:310-337) and
  // apply_divergence_free_correction (376-403): identical bodies.
#pragma omp parallel for schedule(static)
  for (int64_t tid = 0; tid < m.n; ++tid) {
    const int64_t i = g.point_ids[tid];
    if (!dynamic(m.flags[i], m.mask[i])) continue;
    const V3<T> xi = ld(x, i);
    V3<T> dv = mk(T(0), T(0), T(0));
    g.query(xi, h, [&](int32_t j) {
      if (!active(m.flags[j])) return;
      T coeff = m.mass[j] * (kappa[i] / tmax(rho[i], T(1.0e-6)) + kappa[j] / tmax(rho[j], T(1.0e-6)));
      dv = dv + coeff * cubic_dw(xi - ld(x, j), h);
    });
    st(v_star, i, ld(v_star, i) - dt * dv);
  }
}

// Mean over dynamic particles of max(a - b, 0) (b may be null), the
// residuals of solver_dfsph.py:579-596.  Accumulated in double.
template <class T>
double dyn_mean_pos(const Model<T>& m, const T* a, const T* b) {
  double s = 0.0;
  int64_t cnt = 0;
#pragma omp parallel for reduction(+ : s, cnt) schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) continue;
    T e = b ? tmax(a[i] - b[i], T(0)) : tmax(a[i], T(0));
    s += (double)e;
    cnt += 1;
  }
  return cnt ? s / (double)cnt : 0.0;
}

// SolverDFSPH.step, solver_dfsph.py:598-898.
template <class T>
void dfsph_step(const OracleModel& om, const OracleState& si, OracleState& so, const OracleDfsphCfg& c, T dt,
                T* accel, OracleDfsphInfo* info) {
  Model<T> m(om);
  if (m.n == 0) return;
  const T h = T(c.particle_length * c.smoothing_length_coff);
  const T pr = particle_radius_of<T>(c.particle_radius, c.particle_max_radius);
  std::vector<T> vol;
  particle_volume(m, vol);
  const T* xin = (const T*)si.q;
  const T* vin = (const T*)si.qd;
  T* xo = (T*)so.q;
  T* vo = (T*)so.qd;
  T* rho = (T*)so.rho;
  T* factor = (T*)so.factor;
  T* vstar = (T*)so.v_star;
  T* kappa = (T*)so.kappa;
  T* kappa_v = (T*)so.kappa_v;
  T* drho = (T*)so.d_rho_dt;
  T* rho_star = (T*)so.rho_star;
  Grid<T> g;
  g.build(xin, m.n, h, c.grid);
  density_pass<T, false>(m, g, xin, vol, h, rho, nullptr, false);
  factor_pass(m, g, xin, h, c.min_neighbors_for_factor, factor, so.neighbor_count);
  accel_pass<T, false, false>(m, g, xin, vin, rho, nullptr, pr, h, accel);
  // predict_velocity, 230-242
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i)
    st(vstar, i, dynamic(m.flags[i], m.mask[i]) ? ld(vin, i) + dt * ld(accel, i) : mk(T(0), T(0), T(0)));
  if (c.warm_start) {
    std::memcpy(kappa, si.kappa, sizeof(T) * m.n);
    correction_pass(m, g, xin, vstar, rho, kappa, h, dt);
  }
  int rho_it = 0, vel_it = 0;
  double dres = 0.0, vres = 0.0;
  for (int it = 0; it < c.max_rho_iterations; ++it) {
    rho_it++;
    drho_pass(m, g, xin, vstar, h, drho);
    // predict_density_star, 276-287
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m.n; ++i) rho_star[i] = active(m.flags[i]) ? rho[i] + dt * drho[i] : T(0);
    dres = dyn_mean_pos(m, rho_star, m.rest_density);
    if (it > 0 && dres <= c.eta_density) break;
    // compute_kappa_density, 291-306
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m.n; ++i) {
      if (!dynamic(m.flags[i], m.mask[i])) {
        kappa[i] = T(0);
        continue;
      }
      T err = tmax(rho_star[i] - m.rest_density[i], T(0));
      kappa[i] = tmin((err / (dt * dt)) * factor[i], T(c.max_kappa));
    }
    correction_pass(m, g, xin, vstar, rho, kappa, h, dt);
  }
  // integrate_positions, 341-353
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i)
    st(xo, i, dynamic(m.flags[i], m.mask[i]) ? ld(xin, i) + ld(vstar, i) * dt : ld(xin, i));
  g.build(xo, m.n, h, c.grid);
  density_pass<T, false>(m, g, xo, vol, h, rho, nullptr, false);
  factor_pass(m, g, xo, h, c.min_neighbors_for_factor, factor, so.neighbor_count);
  if (c.warm_start) {
    std::memcpy(kappa_v, si.kappa_v, sizeof(T) * m.n);
    correction_pass(m, g, xo, vstar, rho, kappa_v, h, dt);
  }
  for (int it = 0; it < c.max_vel_iterations; ++it) {
    vel_it++;
    drho_pass(m, g, xo, vstar, h, drho);
    vres = dyn_mean_pos(m, drho, (const T*)nullptr);
    if (it > 0 && vres <= c.eta_divergence) break;
    // compute_kappa_divergence, 357-372
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m.n; ++i) {
      if (!dynamic(m.flags[i], m.mask[i])) {
        kappa_v[i] = T(0);
        continue;
      }
      T dc = tmax(drho[i], T(0));
      kappa_v[i] = tmin((T(1) / dt) * dc * rho[i] * factor[i], T(c.max_kappa_v));
    }
    correction_pass(m, g, xo, vstar, rho, kappa_v, h, dt);
  }
  std::memcpy(vo, vstar, sizeof(T) * 3 * m.n);
  apply_bounds(m, xo, vo, mk(T(c.bound_width), T(c.bound_height), T(c.bound_length)), T(c.boundary_damping), 1,
               T(0), T(0));
  if (info) {
    info->rho_iterations = rho_it;
    info->vel_iterations = vel_it;
    info->last_density_residual = dres;
    info->last_divergence_residual = vres;
  }
}

// -------------------------------------------------------------- PBF step ----
template <class T>
void position_bounds(const Model<T>& m, T* x, V3<T> size, T radius, T eps) {
  // apply_position_bounds, solver_pbf.py:367-399
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) continue;
    V3<T> p = ld(x, i);
    T xmin = -size.x + radius + eps, xmax = size.x - radius - eps;
    T ymin = -size.y + radius + eps, ymax = size.y - radius - eps;
    T zmin = radius + eps, zmax = size.z * T(2) - radius - eps;
    if (p.x < xmin) p.x = xmin;
    if (p.x > xmax) p.x = xmax;
    if (p.y < ymin) p.y = ymin;
    if (p.y > ymax) p.y = ymax;
    if (p.z < zmin) p.z = zmin;
    if (p.z > zmax) p.z = zmax;
    st(x, i, p);
  }
}

template <class T>
T pbf_w_delta_q(double scorr_q, double h) {
  // SolverPBF._w_delta_q, solver_pbf.py:671-674: evaluated on the host in
  // double precision, then passed to the kernel as float.
  double r = scorr_q * h;
  double res = 0.0;
  if (h > 0.0 && r < h) {
    double rhs = h * h - r * r;
    double c = h * h * h;
    double k = 315.0 / (64.0 * 3.14159265358979323846 * (c * c * c));
    res = k * rhs * rhs * rhs;
  }
  return T(res);
}

// SolverPBF.step, solver_pbf.py:676-954.
template <class T>
void pbf_step(const OracleModel& om, const OracleState& si, OracleState& so, const OraclePbfCfg& c, T dt, T* accel,
              T* x_pred_out) {
  Model<T> m(om);
  if (m.n == 0) return;
  const T h = T(c.particle_length * c.smoothing_length_coff);
  const T pr = particle_radius_of<T>(c.particle_radius, c.particle_max_radius);
  const V3<T> size = mk(T(c.bound_width), T(c.bound_height), T(c.bound_length));
  const T eps = T(c.boundary_epsilon);
  std::vector<T> vol;
  particle_volume(m, vol);
  const T* xin = (const T*)si.q;
  const T* vin = (const T*)si.qd;
  T* xo = (T*)so.q;
  T* vo = (T*)so.qd;
  T* rho = (T*)so.rho;
  T* lam = (T*)so.pbf_lambda;
  T* dp = (T*)so.delta_p;
  int32_t* cnt = so.neighbor_count;
  std::vector<T> vpred(3 * m.n), xpred(3 * m.n), vtmp(3 * m.n);
  // predict_velocity_with_gravity (193-208) and predict_positions (212-224)
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) {
      st(vpred.data(), i, ld(vin, i));
      st(xpred.data(), i, ld(xin, i));
      continue;
    }
    V3<T> vp = ld(vin, i) + dt * m.g(i);
    st(vpred.data(), i, vp);
    st(xpred.data(), i, ld(xin, i) + dt * vp);
  }
  position_bounds(m, xpred.data(), size, pr, eps);
  Grid<T> g;
  g.build(xpred.data(), m.n, h, c.grid);
  density_pass<T, true>(m, g, xpred.data(), vol, h, rho, nullptr, false);
  accel_pass<T, false, true>(m, g, xpred.data(), vpred.data(), rho, nullptr, pr, h, accel);
  // apply_non_pressure_prediction, 228-242
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    if (!dynamic(m.flags[i], m.mask[i])) continue;
    V3<T> dv = dt * ld(accel, i);
    st(vpred.data(), i, ld(vpred.data(), i) + dv);
    st(xpred.data(), i, ld(xpred.data(), i) + dt * dv);
  }
  position_bounds(m, xpred.data(), size, pr, eps);
  const T wdq = pbf_w_delta_q<T>(c.scorr_q, (double)h);
  const T lambda_eps = T(c.lambda_epsilon), sk = T(c.scorr_k), sn = T(c.scorr_n), maxd = T(c.max_delta_position);
  for (int it = 0; it < c.max_iterations; ++it) {
    const T* xp = xpred.data();
    // compute_pbf_lambda, 246-302
#pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < m.n; ++tid) {
      const int64_t i = g.point_ids[tid];
      if (!dynamic(m.flags[i], m.mask[i])) {
        lam[i] = T(0);
        rho[i] = T(0);
        cnt[i] = 0;
        continue;
      }
      const T rho0 = tmax(m.rest_density[i], T(1.0e-6));
      const V3<T> xi = ld(xp, i);
      T rho_i = T(0), sq = T(0);
      V3<T> gi = mk(T(0), T(0), T(0));
      int32_t count = 0;
      g.query(xi, h, [&](int32_t j) {
        if (!active(m.flags[j])) return;
        V3<T> xij = xi - ld(xp, j);
        T r = length(xij);
        if (j != i && r < h) count += 1;
        T mj = m.mass[j];
        rho_i += mj * poly6_w(r, h);
        V3<T> gj = (-(mj / rho0)) * spiky_dw(xij, h);
        sq += dot(gj, gj);
        gi = gi - gj;
      });
      sq += dot(gi, gi);
      T ci = tmax(rho_i / rho0 - T(1), T(0));
      rho[i] = rho_i;
      cnt[i] = count;
      lam[i] = (c.min_neighbors_for_lambda > 0 && count < c.min_neighbors_for_lambda) ? T(0)
                                                                                     : -ci / (sq + lambda_eps);
    }
    // compute_delta_position, 306-350
#pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < m.n; ++tid) {
      const int64_t i = g.point_ids[tid];
      if (!dynamic(m.flags[i], m.mask[i])) {
        st(dp, i, mk(T(0), T(0), T(0)));
        continue;
      }
      const V3<T> xi = ld(xp, i);
      const T rho0 = tmax(m.rest_density[i], T(1.0e-6));
      V3<T> d = mk(T(0), T(0), T(0));
      g.query(xi, h, [&](int32_t j) {
        if (j == i || !active(m.flags[j])) return;
        V3<T> xij = xi - ld(xp, j);
        V3<T> gr = spiky_dw(xij, h);
        T sc = T(0);
        if (sk != T(0)) {
          // compute_scorr, 91-101
          if (!(wdq <= T(1.0e-6))) sc = -sk * std::pow(poly6_w(length(xij), h) / wdq, sn);
        }
        d = d + ((lam[i] + lam[j] + sc) * m.mass[j]) * gr;
      });
      d = d / rho0;
      if (maxd > T(0)) {
        T len = length(d);
        if (len > maxd) d = d * (maxd / tmax(len, T(1.0e-12)));
      }
      st(dp, i, d);
    }
    // apply_delta_position, 354-363
    T* xpw = xpred.data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m.n; ++i)
      if (dynamic(m.flags[i], m.mask[i])) st(xpw, i, ld(xpw, i) + ld(dp, i));
    if (c.rebuild_grid_each_iteration) {
      position_bounds(m, xpw, size, pr, eps);
      g.build(xpw, m.n, h, c.grid);
    }
  }
  position_bounds(m, xpred.data(), size, pr, eps);
  density_pass<T, true>(m, g, xpred.data(), vol, h, rho, nullptr, false);
  // update_velocity_from_positions, 403-416
  const T dtc = tmax(dt, T(1.0e-8));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i)
    st(vo, i, dynamic(m.flags[i], m.mask[i]) ? (ld(xpred.data(), i) - ld(xin, i)) / dtc : ld(vin, i));
  if (c.xsph_c > 0.0) {
    // apply_xsph_viscosity, 435-463
    const T xc = T(c.xsph_c);
    const T* xp = xpred.data();
#pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < m.n; ++tid) {
      const int64_t i = g.point_ids[tid];
      if (!dynamic(m.flags[i], m.mask[i])) {
        st(vtmp.data(), i, ld(vo, i));
        continue;
      }
      const V3<T> vi = ld(vo, i), xi = ld(xp, i);
      V3<T> corr = mk(T(0), T(0), T(0));
      g.query(xi, h, [&](int32_t j) {
        if (j == i || !active(m.flags[j])) return;
        T w = poly6_w(length(xi - ld(xp, j)), h);
        corr = corr + ((m.mass[j] / tmax(rho[j], T(1.0e-6))) * (ld(vo, j) - vi)) * w;
      });
      st(vtmp.data(), i, vi + xc * corr);
    }
    std::memcpy(vo, vtmp.data(), sizeof(T) * 3 * m.n);
  }
  std::memcpy(xo, xpred.data(), sizeof(T) * 3 * m.n);
  apply_bounds(m, xo, vo, size, T(c.boundary_damping), 2, pr, eps);
  if (x_pred_out) std::memcpy(x_pred_out, xpred.data(), sizeof(T) * 3 * m.n);
}

// SolverAPIC._apply_particle_separation (solver_apic.py:1003-1064): per
// iteration a hash grid of cell width query_radius over the current
// positions, accumulate_particle_separation (193-248: mean push of the
// active neighbours closer than rest_dist, components into a wall band
// removed) and apply_particle_separation_delta (251-266: add, clamp to the
// bounds inset by wall_margin).  x is updated in place; delta keeps the last
// iteration's pushes.
template <class T>
inline T warp_max(T a, T b) { return a > b ? a : b; }
template <class T>
inline T warp_min(T a, T b) { return a < b ? a : b; }

template <class T>
void apic_separation(T* x, const int32_t* flags, int64_t n, const OracleSeparationCfg& c, T* delta) {
  const T rest = T(c.rest_dist), qr = T(c.query_radius), strength = T(c.strength), band = T(c.wall_band);
  const T margin = T(c.wall_margin);
  const V3<T> lo = mk(T(c.bound_lo[0]), T(c.bound_lo[1]), T(c.bound_lo[2]));
  const V3<T> hi = mk(T(c.bound_hi[0]), T(c.bound_hi[1]), T(c.bound_hi[2]));
  const int iters = c.iterations > 1 ? c.iterations : 1;
  Grid<T> g;
  for (int it = 0; it < iters; ++it) {
    g.build(x, n, qr, c.grid);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      if (!active(flags[i])) {
        st(delta, i, mk(T(0), T(0), T(0)));
        continue;
      }
      const V3<T> xi = ld(x, i);
      V3<T> disp = mk(T(0), T(0), T(0));
      T count = T(0);
      g.query(xi, qr, [&](int32_t j) {
        if (j != i && active(flags[j])) {
          const V3<T> rij = xi - ld(x, j);
          const T d = length(rij);
          if (d > T(1.0e-8) && d < rest) {
            const V3<T> nrm = rij / d;
            disp = disp + nrm * (strength * (rest - d));
            count = count + T(1);
          }
        }
      });
      if (count > T(0))
        disp = disp / count;
      else
        disp = mk(T(0), T(0), T(0));
      if (xi.x <= lo.x + band && disp.x < T(0)) disp.x = T(0);
      if (xi.x >= hi.x - band && disp.x > T(0)) disp.x = T(0);
      if (xi.y <= lo.y + band && disp.y < T(0)) disp.y = T(0);
      if (xi.y >= hi.y - band && disp.y > T(0)) disp.y = T(0);
      if (xi.z <= lo.z + band && disp.z < T(0)) disp.z = T(0);
      if (xi.z >= hi.z - band && disp.z > T(0)) disp.z = T(0);
      st(delta, i, disp);
    }
    const V3<T> blo = lo + mk(margin, margin, margin), bhi = hi - mk(margin, margin, margin);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      if (!active(flags[i])) continue;
      const V3<T> p = ld(x, i) + ld(delta, i);
      st(x, i, mk(warp_min(warp_max(p.x, blo.x), bhi.x), warp_min(warp_max(p.y, blo.y), bhi.y),
                  warp_min(warp_max(p.z, blo.z), bhi.z)));
    }
  }
}

}  // namespace

// ----------------------------------------------------------- C entries ----
extern "C" {

int oracle_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// Grid build: outputs the reference tables (point_ids, point_cells in sorted
// order; cell_starts/ends with 0 for empty cells).
int oracle_grid_build_f32(const float* x, int64_t n, float radius, const GridCfg* cfg, int32_t* point_ids,
                          int32_t* point_cells, int32_t* cell_starts, int32_t* cell_ends) {
  Grid<float> g;
  g.build(x, n, radius, *cfg);
  std::memcpy(point_ids, g.point_ids.data(), sizeof(int32_t) * n);
  std::memcpy(point_cells, g.point_cells.data(), sizeof(int32_t) * n);
  const int64_t nc = (int64_t)cfg->dim_x * cfg->dim_y * cfg->dim_z;
  std::memcpy(cell_starts, g.cell_starts.data(), sizeof(int32_t) * nc);
  std::memcpy(cell_ends, g.cell_ends.data(), sizeof(int32_t) * nc);
  return 0;
}

// Candidate enumeration: for query i (at q[i], radius r) writes the candidates
// in visiting order to cand[offsets[i] .. offsets[i+1]).  With cand == NULL
// only counts[i] is written.
int oracle_grid_candidates_f32(const float* x, int64_t n, float radius, const GridCfg* cfg, const float* q,
                               int64_t nq, float r, int64_t* counts, const int64_t* offsets, int32_t* cand) {
  Grid<float> g;
  g.build(x, n, radius, *cfg);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nq; ++i) {
    int64_t k = 0;
    int64_t base = offsets ? offsets[i] : 0;
    g.query(ld(q, i), r, [&](int32_t j) {
      if (cand) cand[base + k] = j;
      ++k;
    });
    counts[i] = k;
  }
  return 0;
}

int oracle_wcsph_step_f32(const OracleModel* m, const OracleState* si, OracleState* so, const OracleWcsphCfg* c,
                          float dt, float* accel) {
  wcsph_step<float>(*m, *si, *so, *c, dt, accel);
  return 0;
}
int oracle_wcsph_step_f64(const OracleModel* m, const OracleState* si, OracleState* so, const OracleWcsphCfg* c,
                          double dt, double* accel) {
  wcsph_step<double>(*m, *si, *so, *c, dt, accel);
  return 0;
}
int oracle_dfsph_step_f32(const OracleModel* m, const OracleState* si, OracleState* so, const OracleDfsphCfg* c,
                          float dt, float* accel, OracleDfsphInfo* info) {
  dfsph_step<float>(*m, *si, *so, *c, dt, accel, info);
  return 0;
}
int oracle_dfsph_step_f64(const OracleModel* m, const OracleState* si, OracleState* so, const OracleDfsphCfg* c,
                          double dt, double* accel, OracleDfsphInfo* info) {
  dfsph_step<double>(*m, *si, *so, *c, dt, accel, info);
  return 0;
}
int oracle_pbf_step_f32(const OracleModel* m, const OracleState* si, OracleState* so, const OraclePbfCfg* c,
                        float dt, float* accel, float* x_pred) {
  pbf_step<float>(*m, *si, *so, *c, dt, accel, x_pred);
  return 0;
}
int oracle_pbf_step_f64(const OracleModel* m, const OracleState* si, OracleState* so, const OraclePbfCfg* c,
                        double dt, double* accel, double* x_pred) {
  pbf_step<double>(*m, *si, *so, *c, dt, accel, x_pred);
  return 0;
}

int oracle_apic_separation_f32(float* x, const int32_t* flags, int64_t n, const OracleSeparationCfg* c, float* delta) {
  apic_separation<float>(x, flags, n, *c, delta);
  return 0;
}

int oracle_apic_separation_f64(double* x, const int32_t* flags, int64_t n, const OracleSeparationCfg* c,
                               double* delta) {
  apic_separation<double>(x, flags, n, *c, delta);
  return 0;
}

}  // extern "C"
