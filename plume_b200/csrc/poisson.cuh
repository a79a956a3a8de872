// The variable-coefficient 7-point Poisson stencil of the pressure solve (chadmv/plume
// src/plume/sim/pressure.py:39-92, multigrid.py:36-43), written once for every place that evaluates it:
// global memory, shared-memory tiles and the single-block coarse solve. `load(i, j, k)` returns the
// pressure of an in-grid neighbour; the order of float operations is the reference's.
#pragma once

#include "common.cuh"

namespace plume {

// The share of a cell's width along `axis` inside the domain: 1 except a coarse level's overhang.
__device__ __forceinline__ float cell_fill(const PlumeGridInfo& info, int axis, int index) {
  return index == info.dims[axis] - 1 ? info.fill_hi[axis] : 1.0f;
}

__device__ __forceinline__ float cell_volume(const PlumeGridInfo& info, int i, int j, int k) {
  return cell_fill(info, 0, i) * cell_fill(info, 1, j) * cell_fill(info, 2, k);
}

// neighbor_sum (pressure.py:52-77): (sum of coupling * neighbour pressure, sum of couplings). Open-face ghosts
// hold pressure 0 at ghost_gap; closed faces couple nothing.
template <class Load>
__device__ __forceinline__ void neighbor_sum(const PlumeGridInfo& info, int i, int j, int k, Load load, float& sq,
                                             float& sc) {
  const int c[3] = {i, j, k};
  sq = 0.0f;
  sc = 0.0f;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    float area = 1.0f;
#pragma unroll
    for (int other = 0; other < 3; ++other)
      if (other != axis) area = area * cell_fill(info, other, c[other]);
    const float own = cell_fill(info, axis, c[axis]);
    float tq[2], tc[2];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int step = side == 0 ? -1 : 1;
      const int n = c[axis] + step;
      if (n >= 0 && n < info.dims[axis]) {
        float coupling = area / (0.5f * (own + cell_fill(info, axis, n)));
        const float neighbour = axis == 0 ? load(n, j, k) : (axis == 1 ? load(i, n, k) : load(i, j, n));
        tq[side] = coupling * neighbour;
        tc[side] = coupling;
      } else if ((step < 0 && info.open_lo[axis] == 1) || (step > 0 && info.open_hi[axis] == 1)) {
        tq[side] = 0.0f;
        tc[side] = area / (0.5f * own + info.ghost_gap);
      } else {
        tq[side] = 0.0f;
        tc[side] = 0.0f;
      }
    }
    sq = (sq + tq[0]) + tq[1];
    sc = (sc + tc[0]) + tc[1];
  }
}

// One red-black update (red_black_sweep_kernel, pressure.py:80-92). Returns false, leaving `out` alone, for
// a cell with no coupling at all.
template <class Load>
__device__ __forceinline__ bool relaxed(const PlumeGridInfo& info, int i, int j, int k, float q, float rhs,
                                        float relaxation, Load load, float& out) {
  float sq, sc;
  neighbor_sum(info, i, j, k, load, sq, sc);
  if (sc == 0.0f) return false;
  float source = cell_volume(info, i, j, k) * info.cell_m * info.cell_m * rhs;
  float target = (sq - source) / sc;
  out = q + relaxation * (target - q);
  return true;
}

// residual_kernel (multigrid.py:36-43): rhs - A q.
template <class Load>
__device__ __forceinline__ float residual_at(const PlumeGridInfo& info, int i, int j, int k, float q, float rhs,
                                             Load load) {
  float sq, sc;
  neighbor_sum(info, i, j, k, load, sq, sc);
  float scale = cell_volume(info, i, j, k) * info.cell_m * info.cell_m;
  return rhs - divide(sq - sc * q, divisor(scale));
}

// ---- the uniform-coefficient case ---------------------------------------------------------------------------
// When every fill is 1 (the simulation grid, and every coarse level of an axis that halves evenly), each
// interior coupling is area / (0.5 * (own + neighbour)) = 1 / (0.5 * 2) = 1 exactly, so coupling * q == q, and
// an open face's ghost couples with 1 / (0.5 + ghost_gap). The functions below skip the per-neighbour
// divisions but produce the same floats as the general ones.
__device__ __forceinline__ bool is_uniform(const PlumeGridInfo& info) {
  return info.fill_hi[0] == 1.0f && info.fill_hi[1] == 1.0f && info.fill_hi[2] == 1.0f;
}

__device__ __forceinline__ float ghost_coupling(const PlumeGridInfo& info) { return 1.0f / (0.5f + info.ghost_gap); }

template <class Load>
__device__ __forceinline__ void neighbor_sum_uniform(const PlumeGridInfo& info, float ghost, int i, int j, int k,
                                                     Load load, float& sq, float& sc) {
  const int c[3] = {i, j, k};
  sq = 0.0f;
  sc = 0.0f;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    float tq0 = 0.0f, tc0 = 0.0f, tq1 = 0.0f, tc1 = 0.0f;
    if (c[axis] > 0) {
      tq0 = axis == 0 ? load(i - 1, j, k) : (axis == 1 ? load(i, j - 1, k) : load(i, j, k - 1));
      tc0 = 1.0f;
    } else if (info.open_lo[axis] == 1) {
      tc0 = ghost;
    }
    if (c[axis] < info.dims[axis] - 1) {
      tq1 = axis == 0 ? load(i + 1, j, k) : (axis == 1 ? load(i, j + 1, k) : load(i, j, k + 1));
      tc1 = 1.0f;
    } else if (info.open_hi[axis] == 1) {
      tc1 = ghost;
    }
    sq = (sq + tq0) + tq1;
    sc = (sc + tc0) + tc1;
  }
}

// x / 6, correctly rounded, by the reciprocal with one remainder correction (Brisebarre, Muller and Raina,
// "Accelerating correctly rounded floating-point division when the divisor is known in advance", IEEE Trans.
// Computers 53(8), 2004): q0 = x * RN(1/6), r = fma(-q0, 6, x) (exact), q = fma(r, RN(1/6), q0). For d = 6 this
// returns IEEE x / 6 whenever x and the quotient are normal floats (every float x checked against the division;
// the failures are all subnormal); below |x| = 2^-120, and for zeros, infinities and NaN, it divides.
__device__ __forceinline__ bool div6_in_range(float x) { return fabsf(x) >= 0x1p-120f && fabsf(x) <= 0x1p+127f; }
__device__ __forceinline__ float div6_core(float x) {
  constexpr float z = 0x1.555556p-3f;  // RN(1/6)
  const float q0 = x * z;
  return __fmaf_rn(__fmaf_rn(-q0, 6.0f, x), z, q0);
}
__device__ __forceinline__ float div6(float x) { return div6_in_range(x) ? div6_core(x) : x / 6.0f; }

template <class Load>
__device__ __forceinline__ bool relaxed_uniform(const PlumeGridInfo& info, float ghost, int i, int j, int k, float q,
                                                float rhs, float relaxation, Load load, float& out) {
  float sq, sc;
  const bool interior =
      i > 0 && j > 0 && k > 0 && i < info.dims[0] - 1 && j < info.dims[1] - 1 && k < info.dims[2] - 1;
  if (interior) {
    // an interior cell: six unit couplings; the same sums as neighbor_sum_uniform (0 + x == x in value)
    sq = ((((load(i - 1, j, k) + load(i + 1, j, k)) + load(i, j - 1, k)) + load(i, j + 1, k)) + load(i, j, k - 1)) +
         load(i, j, k + 1);
    sc = 6.0f;
  } else {
    neighbor_sum_uniform(info, ghost, i, j, k, load, sq, sc);
  }
  if (sc == 0.0f) return false;
  float source = info.cell_m * info.cell_m * rhs;  // cell volume 1: (1 * cell_m) * cell_m == cell_m * cell_m
  float target = interior ? div6(sq - source) : (sq - source) / sc;
  out = q + relaxation * (target - q);
  return true;
}

template <class Load>
__device__ __forceinline__ float residual_uniform(const PlumeGridInfo& info, float ghost, int i, int j, int k, float q,
                                                  float rhs, Load load) {
  float sq, sc;
  neighbor_sum_uniform(info, ghost, i, j, k, load, sq, sc);
  return rhs - divide(sq - sc * q, divisor(info.cell_m * info.cell_m));
}

// residual_uniform for a cell whose four x and y neighbours all exist, at any k, from the neighbours passed in:
// neighbor_sum_uniform's sums in its order (a missing z neighbour adds 0 and its face's coupling), so every value
// is residual_uniform's.
__device__ __forceinline__ float residual_xy_interior(const PlumeGridInfo& info, float ghost, int k, float q, float rhs,
                                                      float x0, float x1, float y0, float y1, float zm, float zp) {
  const bool lo = k > 0, hi = k < info.dims[2] - 1;
  const float sq = (((((0.0f + x0) + x1) + y0) + y1) + (lo ? zm : 0.0f)) + (hi ? zp : 0.0f);
  const float c0 = lo ? 1.0f : (info.open_lo[2] == 1 ? ghost : 0.0f);
  const float c1 = hi ? 1.0f : (info.open_hi[2] == 1 ? ghost : 0.0f);
  const float sc = (4.0f + c0) + c1;  // (((0 + 1) + 1) + 1) + 1 == 4 over x and y, then the two z faces
  return rhs - divide(sq - sc * q, divisor(info.cell_m * info.cell_m));
}

// Either path, chosen per level.
template <class Load>
__device__ __forceinline__ bool relax_cell(bool uniform, const PlumeGridInfo& info, float ghost, int i, int j, int k,
                                           float q, float rhs, float relaxation, Load load, float& out) {
  return uniform ? relaxed_uniform(info, ghost, i, j, k, q, rhs, relaxation, load, out)
                 : relaxed(info, i, j, k, q, rhs, relaxation, load, out);
}

template <class Load>
__device__ __forceinline__ float residual_cell(bool uniform, const PlumeGridInfo& info, float ghost, int i, int j,
                                               int k, float q, float rhs, Load load) {
  return uniform ? residual_uniform(info, ghost, i, j, k, q, rhs, load) : residual_at(info, i, j, k, q, rhs, load);
}

// Trilinear sample with plain loads (shared memory, or global data written earlier in the same kernel).
__device__ __forceinline__ float sample_plain(const float* f, const Dims& d, F3 g) {
  float x = clampf_(g[0], 0.0f, (float)(d.n0 - 1));
  float y = clampf_(g[1], 0.0f, (float)(d.n1 - 1));
  float z = clampf_(g[2], 0.0f, (float)(d.n2 - 1));
  int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  int i1 = imin_(i0 + 1, d.n0 - 1), j1 = imin_(j0 + 1, d.n1 - 1), k1 = imin_(k0 + 1, d.n2 - 1);
  float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
  float c00 = lerpf_(f[at(d, i0, j0, k0)], f[at(d, i1, j0, k0)], tx);
  float c10 = lerpf_(f[at(d, i0, j1, k0)], f[at(d, i1, j1, k0)], tx);
  float c01 = lerpf_(f[at(d, i0, j0, k1)], f[at(d, i1, j0, k1)], tx);
  float c11 = lerpf_(f[at(d, i0, j1, k1)], f[at(d, i1, j1, k1)], tx);
  return lerpf_(lerpf_(c00, c10, ty), lerpf_(c01, c11, ty), tz);
}

// ---- the same stencil in double (no reference counterpart) -------------------------------------------------
// The defect-correction solve evaluates the residual, and sweeps the coarsest level, in double: the couplings
// and sums of neighbor_sum / relaxed / residual_at with the level's float geometry widened to double.
template <class Load>
__device__ __forceinline__ void neighbor_sum_f64(const PlumeGridInfo& info, int i, int j, int k, Load load, double& sq,
                                                 double& sc) {
  const int c[3] = {i, j, k};
  sq = 0.0;
  sc = 0.0;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    double area = 1.0;
#pragma unroll
    for (int other = 0; other < 3; ++other)
      if (other != axis) area = area * (double)cell_fill(info, other, c[other]);
    const double own = cell_fill(info, axis, c[axis]);
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int step = side == 0 ? -1 : 1;
      const int n = c[axis] + step;
      if (n >= 0 && n < info.dims[axis]) {
        const double coupling = area / (0.5 * (own + (double)cell_fill(info, axis, n)));
        const double neighbour = axis == 0 ? load(n, j, k) : (axis == 1 ? load(i, n, k) : load(i, j, n));
        sq = sq + coupling * neighbour;
        sc = sc + coupling;
      } else if ((step < 0 && info.open_lo[axis] == 1) || (step > 0 && info.open_hi[axis] == 1)) {
        sc = sc + area / (0.5 * own + (double)info.ghost_gap);
      }
    }
  }
}

__device__ __forceinline__ double cell_scale_f64(const PlumeGridInfo& info, int i, int j, int k) {
  const double cell_m = info.cell_m;
  return (double)cell_fill(info, 0, i) * (double)cell_fill(info, 1, j) * (double)cell_fill(info, 2, k) * cell_m * cell_m;
}

// rhs - A q in double.
template <class Load>
__device__ __forceinline__ double residual_f64(const PlumeGridInfo& info, int i, int j, int k, double q, double rhs,
                                               Load load) {
  double sq, sc;
  neighbor_sum_f64(info, i, j, k, load, sq, sc);
  return rhs - (sq - sc * q) / cell_scale_f64(info, i, j, k);
}

// One red-black update in double; false for a cell with no coupling.
template <class Load>
__device__ __forceinline__ bool relaxed_f64(const PlumeGridInfo& info, int i, int j, int k, double q, double rhs,
                                            double relaxation, Load load, double& out) {
  double sq, sc;
  neighbor_sum_f64(info, i, j, k, load, sq, sc);
  if (sc == 0.0) return false;
  const double target = (sq - cell_scale_f64(info, i, j, k) * rhs) / sc;
  out = q + relaxation * (target - q);
  return true;
}

// Where a fine cell centre sits in its coarse level's index space (multigrid.py:66-67).
__device__ __forceinline__ F3 prolong_point(int i, int j, int k) {
  return sub3(mul3(f3((float)i, (float)j, (float)k), 0.5f), f3(0.25f, 0.25f, 0.25f));
}

// Host side of the pressure solve (multigrid.cu).
int red_black_sweeps(const PlumeGridInfo& info, float* q, float* scratch, const float* rhs, int sweeps,
                     float relaxation, cudaStream_t st);
// coarse_f64: sweep the coarsest level in double (the defect-correction solve's correction cycles)
// split_scratch: plume_split_scratch_floats(levels[0].info) floats; with it the top level may run in
// colour-split storage (same values)
int multigrid_cycles(const PlumeLevel* levels, int count, int cycles, int sweeps, cudaStream_t st, int coarse_f64 = 0,
                     float* split_scratch = nullptr);

}  // namespace plume
