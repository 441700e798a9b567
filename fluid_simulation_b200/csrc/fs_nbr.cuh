// Neighbour loops of the per-particle passes.
//
// One thread per cell-sorted slot.  Only ~15 % of a particle's 27-cell grid
// candidates (the reference's hash_grid_query set) lie inside the support,
// and every pass of a substep after the first reuses the same grid.  The
// first pass over a grid therefore records each particle's in-support
// candidates (plus a skin when positions will move) as a list in the
// reference's visiting order; later passes iterate those ~35-60 entries
// instead of ~216 candidates, with all lanes of a warp busy on pair terms.
#pragma once

#include "fs_internal.cuh"

namespace fs {

// Neighbour kernels are compiled for blocks of up to kNbBlockMax threads;
// the launch size (64, 128 or 256) and the particles per thread come from
// the context's tuning (fs_context_set_tuning, chosen by the autotuner).
constexpr int kNbBlockMax = 256;
#define FS_NB_BOUNDS __launch_bounds__(kNbBlockMax)

// support test margin: FMA-evaluated r^2 may differ from the individually
// rounded r^2 by about one ulp; anything the reference counts (r <= h) passes
constexpr float kSupportMargin = 1.000002f;

// ---------------------------------------------------- fast kernel math --
// Division-free forms; every pair term stays within a few ulp of the
// reference expression (the passes are checked at 1e-5 relative).
struct Cubic {        // cubic spline, support h (solver_wcsph.py:21-51)
  float inv_h, k, g_in, g_out;  // g_in = 6 k / h^2, g_out = -6 k / h
  FS_DEV explicit Cubic(float h) {
    inv_h = 1.0f / h;
    k = 8.0f / (kPi * (h * h * h));
    g_in = 6.0f * k * inv_h * inv_h;
    g_out = -6.0f * k * inv_h;
  }
  FS_DEV float w_of_q(float q) const {
    if (q > 1.f) return 0.f;
    if (q <= 0.5f) return k * fmaf(6.f * q, q * q, fmaf(-6.f, q * q, 1.f));
    const float t = 1.f - q;
    return 2.f * k * (t * t * t);
  }
  FS_DEV float w(float r) const { return w_of_q(r * inv_h); }
  // grad W(d) = s * d for |d| = r; rinv = 1 / r
  FS_DEV float grad_scale(float r, float rinv) const {
    const float q = r * inv_h;
    if (!(r > 1.0e-5f) || q > 1.f) return 0.f;
    if (q <= 0.5f) return g_in * fmaf(3.f, q, -2.f);
    const float t = 1.f - q;
    return g_out * t * t * rinv;
  }
};

struct Poly6Spiky {   // PBF kernels (solver_pbf.py:24-45)
  float h, h2, kw, kg;
  FS_DEV explicit Poly6Spiky(float h_) : h(h_), h2(h_ * h_) {
    const float c = h_ * h_ * h_;
    kw = 315.0f / (64.0f * kPi * (c * c * c));
    kg = -45.0f / (kPi * (c * c));
  }
  FS_DEV float w_r2(float r2) const {  // poly6 from r^2
    if (!(r2 < h2)) return 0.f;
    const float d = h2 - r2;
    return kw * (d * d * d);
  }
  FS_DEV float grad_scale(float r, float rinv) const {  // spiky
    if (!(r > 1.0e-6f) || !(r < h)) return 0.f;
    const float d = h - r;
    return kg * d * d * rinv;
  }
};

// r and 1/r from r^2 (r2 == 0 gives r = 0, 1/r = 0)
FS_DEV void r_and_inv(float r2, float& r, float& rinv) {
  rinv = r2 > 0.f ? rsqrtf(r2) : 0.f;
  r = r2 * rinv;
}

// `r < h` with r = sqrt(r^2) rounded as in a strict FP32 evaluation, from
// an r^2 the caller already has (any rounding within a few ulp, e.g. FMA
// contracted): only the few pairs within 2e-6 of the support boundary
// recompute r^2 with individually rounded operations and take the exact
// square root.
FS_DEV bool exact_lt_h(float r2_any, float dx, float dy, float dz, float h, float h2) {
  if (r2_any < h2 * 0.999998f) return true;
  if (r2_any > h2 * 1.000002f) return false;
  return sqrtf(dist2_rn(dx, dy, dz)) < h;
}


// ======================================================= neighbour lists ==
// The first pass over a set of positions scans the grid and records, per
// particle, its candidates within the support (in the reference's visiting
// order); the following passes at the same positions iterate those entries.
//   idx[k * stride + s]  k-th entry (cell-sorted slot) of slot s  -- a warp
//                        reads one row k with consecutive addresses
//   cnt[s]               entries of s; kNbMax + 1 marks an overflow (s rescans)
// A list is exact for a later pass at unchanged positions: the grid, the
// positions and hence the candidate set and every distance are the ones
// recorded.  Each new grid build invalidates the lists (ListCtl.valid).
// 192 entries: about 5x the ~35 neighbours of fluid at rest.  DFSPH's
// iteration caps let the dam break compress well past that where the column
// hits the wall (0.2 % of the particles above 96 entries after 300 substeps,
// 1.1 % after 500), and each overflowing particle rescans the grid in every
// pass at those positions, its whole warp with it.
constexpr int kNbMax = 192;
// Entry offsets k * stride (k < kNbMax) fit 32 bits up to this stride (capacity).
constexpr int64_t kListStride32Max = 0xffffffffLL / kNbMax;

struct ListCtl {
  int32_t valid;  // lists recorded for the current grid and positions
  int32_t pad;
};

struct NbrList {
  int32_t* idx;
  int32_t* cnt;
  int64_t stride;
  ListCtl* ctl;
};

// Records the grid candidates of slot s with r^2 + w <= h2m (self included)
// in visiting order; returns the active candidates other than s (the DFSPH
// neighbour count, no distance test) when COUNT.
//
// A row range that fits in the list whatever it holds (n + its length <=
// kNbMax) takes the short loop: no per-candidate capacity test, and the
// entry offset is 32-bit when the list fits (stride <= kListStride32Max).
// Other ranges take the checked loop.  Both record the same entries.
template <bool COUNT>
FS_DEV int record_list(const GridDev& g, const float4* __restrict__ xs, int s, float4 xi, float h, float h2m,
                       const NbrList& L) {
  int n = 0, ncand = 0;
  int32_t* const col = L.idx + s;  // entry k of slot s lives at col[k * stride]
  const int64_t stride = L.stride;
  const bool off32 = stride <= kListStride32Max;  // uniform across the launch
  const uint32_t stride32 = (uint32_t)stride;
  auto r2_of = [&](float4 xj) {
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    return fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, xj.w)));  // +inf for inactive
  };
  auto count = [&](int t, float4 xj) {
    if (COUNT) ncand += (t != s) ? (__float_as_int(xj.w) & PF_ACTIVE) : 0;
  };
  auto checked = [&](int t, float4 xj) {
    count(t, xj);
    if (r2_of(xj) <= h2m) {
      if (n < kNbMax) col[(int64_t)n * stride] = t;
      ++n;
    }
  };
  for_each_range(g, world_of(xi), xi.x, xi.y, xi.z, h, [&](int a, int e) {
    int t = a;
    if (off32 && n + (e - a) <= kNbMax) {
      uint32_t o = (uint32_t)n * stride32;
      auto fast = [&](int tt, float4 xj) {
        count(tt, xj);
        const bool hit = r2_of(xj) <= h2m;
        if (hit) col[o] = tt;
        o += hit ? stride32 : 0u;
        n += hit ? 1 : 0;
      };
      for (; t + 4 <= e; t += 4) {  // four independent loads in flight
        const float4 x0 = __ldg(xs + t), x1 = __ldg(xs + t + 1), x2 = __ldg(xs + t + 2), x3 = __ldg(xs + t + 3);
        fast(t, x0);
        fast(t + 1, x1);
        fast(t + 2, x2);
        fast(t + 3, x3);
      }
      for (; t < e; ++t) fast(t, __ldg(xs + t));
      return;
    }
    for (; t + 4 <= e; t += 4) {
      const float4 x0 = __ldg(xs + t), x1 = __ldg(xs + t + 1), x2 = __ldg(xs + t + 2), x3 = __ldg(xs + t + 3);
      checked(t, x0);
      checked(t + 1, x1);
      checked(t + 2, x2);
      checked(t + 3, x3);
    }
    for (; t < e; ++t) checked(t, __ldg(xs + t));
  });
  L.cnt[s] = n <= kNbMax ? n : kNbMax + 1;
  return ncand;
}

// Grid scan that calls pair(t, xj) directly (no usable list for this particle).
template <bool WITH_SELF, class Pair>
FS_DEV void scan_grid(const GridDev& g, const float4* __restrict__ xs, int s, float4 xi, float h, float h2m,
                      Pair&& pair) {
  for_each_candidate(g, world_of(xi), xi.x, xi.y, xi.z, h, [&](int t) {
    const float4 xj = __ldg(xs + t);
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    if (fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, xj.w))) <= h2m && (WITH_SELF || t != s)) pair(t, xj);
  });
}

// Visits the neighbours of slot s within h2m through its recorded list when
// lists_ok and the list did not overflow, else by rescanning the grid.
// FRESH: the list was written by the calling kernel, so entries are read
// with coherent loads (each thread reads only the entries it wrote).
template <bool WITH_SELF, bool FRESH, class Pair>
FS_DEV void visit(const GridDev& g, const float4* __restrict__ xs, int s, float4 xi, float h, float h2m,
                  const NbrList& L, bool lists_ok, Pair&& pair) {
  const int n = lists_ok ? (FRESH ? L.cnt[s] : __ldg(L.cnt + s)) : kNbMax + 1;
  const bool use = n <= kNbMax;
  if (use) {
    const int32_t* col = L.idx + s;
    auto entry = [&](int k) { return FRESH ? col[(int64_t)k * L.stride] : __ldg(col + (int64_t)k * L.stride); };
    auto one = [&](int t, float4 xj) {
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      if (fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, xj.w))) <= h2m && (WITH_SELF || t != s)) pair(t, xj);
    };
    int k = 0;
    for (; k + 3 < n; k += 4) {  // four independent gathers in flight
      const int t0 = entry(k), t1 = entry(k + 1), t2 = entry(k + 2), t3 = entry(k + 3);
      const float4 x0 = __ldg(xs + t0), x1 = __ldg(xs + t1), x2 = __ldg(xs + t2), x3 = __ldg(xs + t3);
      one(t0, x0);
      one(t1, x1);
      one(t2, x2);
      one(t3, x3);
    }
    for (; k < n; ++k) {
      const int t0 = entry(k);
      one(t0, __ldg(xs + t0));
    }
  } else {
    scan_grid<WITH_SELF>(g, xs, s, xi, h, h2m, pair);
  }
}

// visit() for pair terms that read a second per-neighbour record (velocity,
// kappa ratio, lambda ...): load(t) is issued together with the position
// gather of each group of four list entries, so the two gathers of a
// neighbour overlap instead of the second waiting for the distance test.
// pair(t, xj, payload) is called in the same order and for the same entries
// as visit() calls pair(t, xj).  Only for lists recorded at the current
// positions (every entry within h2m except the particle itself), where the
// early load fetches nothing that visit() would not.  FRESH as in visit().
// EVICT_FIRST: entries are loaded evict-first (ld.global.cs), leaving the
// caches to the neighbours' data.  Measured faster for the PBF passes whose
// lists at most one later pass reads again (delta, non-pressure, XSPH:
// 1.304 -> 1.287 ms per substep at 401,856 particles); the DFSPH iteration
// passes, which read the same lists 34 times a substep, were slower with it.
template <bool WITH_SELF, bool FRESH = false, bool EVICT_FIRST = false, class Load, class Pair>
FS_DEV void visit_with(const GridDev& g, const float4* __restrict__ xs, int s, float4 xi, float h, float h2m,
                       const NbrList& L, bool lists_ok, Load&& load, Pair&& pair) {
  const int n = lists_ok ? (FRESH ? L.cnt[s] : __ldg(L.cnt + s)) : kNbMax + 1;
  const bool use = n <= kNbMax;
  auto one = [&](int t, float4 xj, const auto& p) {
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    if (fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, xj.w))) <= h2m && (WITH_SELF || t != s)) pair(t, xj, p);
  };
  if (use) {
    const int32_t* col = L.idx + s;
    auto entry = [&](int k) {
      return FRESH ? col[(int64_t)k * L.stride]
                   : (EVICT_FIRST ? __ldcs(col + (int64_t)k * L.stride) : __ldg(col + (int64_t)k * L.stride));
    };
    int k = 0;
    for (; k + 3 < n; k += 4) {
      const int t0 = entry(k), t1 = entry(k + 1), t2 = entry(k + 2), t3 = entry(k + 3);
      const float4 x0 = __ldg(xs + t0), x1 = __ldg(xs + t1), x2 = __ldg(xs + t2), x3 = __ldg(xs + t3);
      const auto p0 = load(t0), p1 = load(t1), p2 = load(t2), p3 = load(t3);
      one(t0, x0, p0);
      one(t1, x1, p1);
      one(t2, x2, p2);
      one(t3, x3, p3);
    }
    for (; k < n; ++k) {
      const int t0 = entry(k);
      const float4 x0 = __ldg(xs + t0);
      one(t0, x0, load(t0));
    }
  } else {
    scan_grid<WITH_SELF>(g, xs, s, xi, h, h2m, [&](int t, float4 xj) { pair(t, xj, load(t)); });
  }
}

// Whether lists recorded for the current grid and positions exist.
FS_DEV bool lists_usable(const NbrList& L) { return L.ctl->valid != 0; }

NbrList nbr_list(const fs_context* c);

// Marks freshly recorded lists valid (first thread of the recording kernel);
// a grid build resets the mark.
FS_DEV void lists_recorded(const NbrList& L) {
  if (blockIdx.x == 0 && threadIdx.x == 0) L.ctl->valid = 1;
}

}  // namespace fs
