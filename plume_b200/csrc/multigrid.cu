// The pressure solve on the device (chadmv/plume src/plume/sim/pressure.py:124-141, multigrid.py:24-147):
// red-black Gauss-Seidel sweeps and multigrid V-cycles, with the reference's update order and arithmetic.
//
// Launch structure of one V-cycle:
//   - each full sweep (red then black) is one launch of k_rb_sweep: a tile of 8x8x32 cells and a 2-cell halo
//     in shared memory; red is updated on the tile and a 1-cell shell, then black on the tile, so every value
//     equals the one the two separate colour passes produce;
//   - the residual, its restriction to the coarse level and the zeroing of the coarse pressure are one
//     launch (k_residual_restrict);
//   - prolongation is folded into the first post-smoothing sweep (the tile loads q + prolong(coarse));
//   - every level from the first of at most 2048 cells down to the coarsest solve runs in one launch: one
//     1024-thread block with all its arrays in shared memory (k_block_solve), or, selectable, one 8-CTA
//     thread-block cluster with the larger levels split in x-slabs over distributed shared memory
//     (k_cluster_solve).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "poisson.cuh"

namespace plume {

constexpr int TILE_I = 8, TILE_J = 8, TILE_K = 32, HALO = 2;
constexpr int QI = TILE_I + 2 * HALO, QJ = TILE_J + 2 * HALO, QK = TILE_K + 2 * HALO;  // pressure region
constexpr int RI = TILE_I + 2, RJ = TILE_J + 2, RK = TILE_K + 2;                      // rhs region
constexpr int SWEEP_THREADS = 256;
constexpr int COARSEST_SWEEPS = 20;  // multigrid.py:24-33
constexpr int COARSEST_SWEEPS_PER_CELL = 4;
constexpr int BOTTOM_THREADS = 1024;
constexpr int BOTTOM_MAX_LEVELS = 8;
constexpr int BOTTOM_WARP_PAIRS = 128;  // levels with at most this many cell pairs per colour run on one warp
// Per-level strategy (set by plume_tune_solver): levels of at least g_tiled_min_cells cells sweep in tiles,
// smaller ones one colour per launch; the first level of at most g_bottom_max_cells cells and everything
// below it runs in one block.
static long g_tiled_min_cells = 1L << 40;  // measured: per-colour sweeps win while the levels fit in L2
// Measured on B200 (128x192x128 and 256x384x256 hierarchies, 4 V-cycles): the one-block solve beats the 8-CTA
// cluster solve, whose passes are bound by barrier latency, and starting it at the first level of at most
// 2048 cells (rather than 8192) saves 9% of the solve: a 16x24x16 level sweeps faster as per-colour launches
// across the GPU than inside one block on one SM.
static long g_bottom_max_cells = 2048;
// The top level runs in colour-split storage (given caller scratch) when it has at least this many cells
// (plume_tune_split): levels whose q and rhs do not fit in L2. Measured on B200 at 256x384x256, 4 V-cycles: the
// solve takes 3.14 ms split against 3.52 ms natural (colour pass 45.5 against 59.9 us, prolongation 91 against
// 109 us, residual and restriction about 110 against 107 us, plus 0.15 ms of layout conversions per solve); at
// 128x192x128, whose levels fit in L2, split is slower (0.97 against 0.78 ms).
static long g_split_min_cells = 1L << 23;
static int g_bottom_kind = 0;  // 0: the one-block solve, 1: the cluster solve
constexpr size_t BOTTOM_MAX_SMEM = 200 * 1024;

// The solve's kernels are launched with programmatic dependent launch: each may be scheduled while the
// previous one drains and waits here, before touching memory, until that one has finished and its writes are
// visible (a no-op when launched without it). Measured on B200: 4% off the 4-cycle solve at 128x192x128
// (0.868 -> 0.833 ms). Triggering the successor early (griddepcontrol.launch_dependents) measured slower: the
// waiting blocks take SM slots from the running kernel.
__device__ __forceinline__ void wait_for_previous_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }


// One full red-black sweep of a tile; with PROLONG the tile first adds the coarse correction
// (prolong_add_kernel, multigrid.py:63-68) to every pressure it loads.
// The sweep reads `q_in` and writes `q_out` (different arrays): a tile's halo belongs to its neighbours, which
// may already have written their cells in the same launch.
template <bool PROLONG, bool UNIFORM>
__global__ void __launch_bounds__(SWEEP_THREADS)
    k_rb_sweep(PlumeGridInfo info, const float* __restrict__ q_in, float* __restrict__ q_out,
               const float* __restrict__ rhs, float relaxation, const float* __restrict__ coarse_q, Dims coarse) {
  wait_for_previous_grid();
  __shared__ float sq[QI * QJ * QK];
  __shared__ float sr[RI * RJ * RK];
  const int n0 = info.dims[0], n1 = info.dims[1], n2 = info.dims[2];
  const int i0 = blockIdx.z * TILE_I, j0 = blockIdx.y * TILE_J, k0 = blockIdx.x * TILE_K;
  const int t = threadIdx.x;
  for (int idx = t; idx < QI * QJ * QK; idx += SWEEP_THREADS) {
    const int a = idx / (QJ * QK), rem = idx - a * (QJ * QK), b = rem / QK, c = rem - b * QK;
    const int gi = i0 - HALO + a, gj = j0 - HALO + b, gk = k0 - HALO + c;
    float value = 0.0f;
    if (gi >= 0 && gi < n0 && gj >= 0 && gj < n1 && gk >= 0 && gk < n2) {
      value = __ldg(q_in + (gi * n1 + gj) * n2 + gk);
      if (PROLONG) value = value + sample_index_space(coarse_q, coarse, prolong_point(gi, gj, gk));
    }
    sq[idx] = value;
  }
  for (int idx = t; idx < RI * RJ * RK; idx += SWEEP_THREADS) {
    const int a = idx / (RJ * RK), rem = idx - a * (RJ * RK), b = rem / RK, c = rem - b * RK;
    const int gi = i0 - 1 + a, gj = j0 - 1 + b, gk = k0 - 1 + c;
    sr[idx] = (gi >= 0 && gi < n0 && gj >= 0 && gj < n1 && gk >= 0 && gk < n2) ? __ldg(rhs + (gi * n1 + gj) * n2 + gk)
                                                                              : 0.0f;
  }
  __syncthreads();
  auto qi = [&](int gi, int gj, int gk) { return ((gi - i0 + HALO) * QJ + (gj - j0 + HALO)) * QK + (gk - k0 + HALO); };
  auto load = [&](int gi, int gj, int gk) { return sq[qi(gi, gj, gk)]; };
  const float ghost = ghost_coupling(info);
  // red (colour 0: i + j + k even) on the tile and its 1-cell shell; one red cell per pair along k
  constexpr int RPK = RK / 2;
  for (int p = t; p < RI * RJ * RPK; p += SWEEP_THREADS) {
    const int a = p / (RJ * RPK), rem = p - a * (RJ * RPK), b = rem / RPK, kp = rem - b * RPK;
    const int gi = i0 - 1 + a, gj = j0 - 1 + b, kbase = k0 - 1 + 2 * kp;
    const int gk = kbase + ((gi + gj + kbase) & 1);
    if (gi < 0 || gi >= n0 || gj < 0 || gj >= n1 || gk < 0 || gk >= n2) continue;
    const int at_q = qi(gi, gj, gk);
    const float r = sr[((gi - i0 + 1) * RJ + (gj - j0 + 1)) * RK + (gk - k0 + 1)];
    float out;
    if (relax_cell(UNIFORM, info, ghost, gi, gj, gk, sq[at_q], r, relaxation, load, out)) sq[at_q] = out;
  }
  __syncthreads();
  // black (colour 1) on the tile
  constexpr int TPK = TILE_K / 2;
  for (int p = t; p < TILE_I * TILE_J * TPK; p += SWEEP_THREADS) {
    const int a = p / (TILE_J * TPK), rem = p - a * (TILE_J * TPK), b = rem / TPK, kp = rem - b * TPK;
    const int gi = i0 + a, gj = j0 + b, kbase = k0 + 2 * kp;
    const int gk = kbase + (((gi + gj + kbase) & 1) ^ 1);
    if (gi >= n0 || gj >= n1 || gk >= n2) continue;
    const int at_q = qi(gi, gj, gk);
    const float r = sr[((gi - i0 + 1) * RJ + (gj - j0 + 1)) * RK + (gk - k0 + 1)];
    float out;
    if (relax_cell(UNIFORM, info, ghost, gi, gj, gk, sq[at_q], r, relaxation, load, out)) sq[at_q] = out;
  }
  __syncthreads();
  for (int idx = t; idx < TILE_I * TILE_J * TILE_K; idx += SWEEP_THREADS) {
    const int a = idx / (TILE_J * TILE_K), rem = idx - a * (TILE_J * TILE_K), b = rem / TILE_K, c = rem - b * TILE_K;
    const int gi = i0 + a, gj = j0 + b, gk = k0 + c;
    if (gi < n0 && gj < n1 && gk < n2) q_out[(gi * n1 + gj) * n2 + gk] = sq[qi(gi, gj, gk)];
  }
}

// One colour of a sweep in place (red_black_sweep_kernel, pressure.py:80-92): for levels too small to fill
// the GPU with tiles. A colour reads only the other colour, so the in-place update is race-free.
template <bool UNIFORM>
__global__ void k_rb_colour(PlumeGridInfo info, float* q, const float* __restrict__ rhs, int color, float relaxation,
                            const float* __restrict__ coarse_q, Dims coarse) {
  wait_for_previous_grid();
  const int ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((i + j + color) & 1);
  if (j >= ny || k >= nz) return;
  const Dims d = dims_of(info);
  auto load = [&](int a, int b, int c) { return q[at(d, a, b, c)]; };
  const int idx = at(d, i, j, k);
  float out;
  if (relax_cell(UNIFORM, info, ghost_coupling(info), i, j, k, q[idx], __ldg(rhs + idx), relaxation, load, out))
    q[idx] = out;
}

// The same colour pass with each thread updating one cell in each of two neighbouring planes (i, i + 1): two
// independent updates whose loads are in flight together. The two cells are the same colour and not face
// neighbours, and every update is the one above, so the result is the same. Measured on B200: the 4-cycle
// solve at 256x384x256 went from 3.727 to 3.570 ms with every level swept this way, but at 128x192x128 from
// 0.780 to 0.828 ms: it pays only on levels that do not fit in L2 (RB_PAIR_MIN_CELLS).
template <bool UNIFORM>
__global__ void k_rb_colour_pair(PlumeGridInfo info, float* q, const float* __restrict__ rhs, int color,
                                 float relaxation) {
  wait_for_previous_grid();
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i = 2 * blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kp = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int k0 = kp + ((i + j + color) & 1), k1 = kp + ((i + 1 + j + color) & 1);
  if (j >= ny) return;
  const bool has0 = k0 < nz, has1 = i + 1 < nx && k1 < nz;
  const Dims d = dims_of(info);
  auto load = [&](int a, int b, int c) { return q[at(d, a, b, c)]; };
  const float ghost = ghost_coupling(info);
  const int idx0 = at(d, i, j, k0), idx1 = at(d, i + 1, j, k1);
  float out0 = 0.0f, out1 = 0.0f;
  bool w0 = false, w1 = false;
  if (has0) w0 = relax_cell(UNIFORM, info, ghost, i, j, k0, q[idx0], __ldg(rhs + idx0), relaxation, load, out0);
  if (has1) w1 = relax_cell(UNIFORM, info, ghost, i + 1, j, k1, q[idx1], __ldg(rhs + idx1), relaxation, load, out1);
  if (w0) q[idx0] = out0;
  if (w1) q[idx1] = out1;
}

// prolong_add_kernel (multigrid.py:63-68), used when a level has no post-smoothing sweep to fold it into.
__global__ void k_prolong_add(Dims coarse, Dims fine, const float* __restrict__ cq, float* __restrict__ q) {
  wait_for_previous_grid();
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= fine.n1 || k >= fine.n2) return;
  const int idx = at(fine, i, j, k);
  q[idx] = q[idx] + sample_index_space(cq, coarse, prolong_point(i, j, k));
}

// residual_kernel + restrict_kernel (multigrid.py:36-60) + coarse.q.zero_() (:143): each coarse cell averages
// the residuals of its (up to 8) children, summed in the reference's child order.
__global__ void k_residual_restrict(PlumeGridInfo fine, const float* __restrict__ q, const float* __restrict__ rhs,
                                    Dims coarse, float* __restrict__ coarse_rhs, float* __restrict__ coarse_q) {
  wait_for_previous_grid();
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= coarse.n1 || k >= coarse.n2) return;
  const Dims fd = dims_of(fine);
  auto load = [&](int a, int b, int c) { return __ldg(q + at(fd, a, b, c)); };
  const bool uniform = is_uniform(fine);
  const float ghost = ghost_coupling(fine);
  float total = 0.0f, count = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const int fi = 2 * i + di, fj = 2 * j + dj, fk = 2 * k + dk;
        if (fi < fd.n0 && fj < fd.n1 && fk < fd.n2) {
          const int idx = at(fd, fi, fj, fk);
          if (uniform && fi > 0 && fi < fd.n0 - 1 && fj > 0 && fj < fd.n1 - 1) {
            const int plane = fd.n1 * fd.n2;
            const float zm = fk > 0 ? __ldg(q + idx - 1) : 0.0f, zp = fk < fd.n2 - 1 ? __ldg(q + idx + 1) : 0.0f;
            total = total + residual_xy_interior(fine, ghost, fk, __ldg(q + idx), __ldg(rhs + idx), __ldg(q + idx - plane),
                                                 __ldg(q + idx + plane), __ldg(q + idx - fd.n2), __ldg(q + idx + fd.n2),
                                                 zm, zp);
          } else {
            total = total + residual_cell(uniform, fine, ghost, fi, fj, fk, __ldg(q + idx), __ldg(rhs + idx), load);
          }
          count = count + 1.0f;
        }
      }
  const int out = at(coarse, i, j, k);
  coarse_rhs[out] = divide(total, divisor(count));  // count is 1, 2, 4 or 8
  coarse_q[out] = 0.0f;
}

// ---- the top level in colour-split storage -----------------------------------------------------------------
// A level larger than L2 is swept from two arrays per quantity, one per colour: cell (i, j, k) of colour
// c = (i + j + k) & 1 sits at ((c * nx + i) * ny + j) * H + (k >> 1), H = (nz + 1) / 2 rounded up to a multiple
// of four. A colour pass then reads and writes whole sectors of the cells it needs (its own q and rhs, the other
// colour's q) instead of sectors shared by both colours. A cell's six face neighbours all sit in the other
// colour's array: its x and y neighbours at the same half index m, one plane (ny * H) or one row (H) away; its
// z neighbours at m - 1 + p and m + p, p = k & 1. The split kernels load whole rows of four half indices and
// hand the natural-layout stencil functions (relax_cell, residual_cell) those values through a loader, so every
// value is the same as in the natural layout.
// natural -> split (to_split) or split -> natural: thread (i, j, m) moves the cells k = 2m and 2m + 1
template <bool TO_SPLIT>
__global__ void k_split_layout(Dims d, int H, const float* __restrict__ in, float* __restrict__ out) {
  wait_for_previous_grid();
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.n1 || m >= H) return;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int k = 2 * m + ((i + j + c) & 1);
    const long s = ((long)(c * d.n0 + i) * d.n1 + j) * H + m;
    if (k < d.n2) {
      const long n = ((long)i * d.n1 + j) * d.n2 + k;
      if (TO_SPLIT) out[s] = in[n];
      else out[n] = in[s];
    } else if (TO_SPLIT) {
      out[s] = 0.0f;  // the padding slot of an odd row
    }
  }
}

// The same colour pass with four cells of a row per thread and 16-byte loads: the thread's own q and rhs, the
// other colour's rows one plane and one row away (x and y neighbours, at the same half indices), and the other
// colour's own row (z neighbours) plus the one value beyond the four that the row's parity needs. Rows are
// padded to a multiple of four. Every cell's update is relax_cell's, its neighbours taken from those values.
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// The cells of a row with all four x and y neighbours (the row is neither on a face of the level in x or y):
// relaxed_uniform's floats with straight-line arithmetic. A z neighbour beyond the level reads 0 (the value
// beyond the row, and the split rows' padding slots, hold 0), which is what neighbor_sum_uniform adds there; the
// two cells at the row's ends divide by its couplings, every other cell by six (div6's reciprocal form, with
// IEEE division where x is outside its range).
template <int P>
__device__ __forceinline__ void split_row_interior(const PlumeGridInfo& info, int H, float* __restrict__ qs,
                                                   const float* __restrict__ rs, long own, long oth, long plane,
                                                   int m0, float relaxation) {
  const int nz = info.dims[2];
  const float4 q4 = ld4(qs + own), r4 = ldg4(rs + own);
  const float4 x0 = ldg4(qs + oth - plane), x1 = ldg4(qs + oth + plane);
  const float4 y0 = ldg4(qs + oth - H), y1 = ldg4(qs + oth + H);
  const float4 zc = ldg4(qs + oth);
  const int mz = P == 0 ? m0 - 1 : m0 + 4;  // the other colour's value beyond the four that this parity needs
  const float zx = (P == 0 ? mz >= 0 : mz < H) ? __ldg(qs + oth - m0 + mz) : 0.0f;
  const float zs[6] = {P == 0 ? zx : 0.0f, zc.x, zc.y, zc.z, zc.w, P == 0 ? 0.0f : zx};  // m0 - 1 .. m0 + 4
  const float qv[4] = {q4.x, q4.y, q4.z, q4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
  const float xa[4] = {x0.x, x0.y, x0.z, x0.w}, xb[4] = {x1.x, x1.y, x1.z, x1.w};
  const float ya[4] = {y0.x, y0.y, y0.z, y0.w}, yb[4] = {y1.x, y1.y, y1.z, y1.w};
  const float h2 = info.cell_m * info.cell_m;
  float out[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const int k = 2 * (m0 + n) + P;
    out[n] = qv[n];
    if (k >= nz) continue;
    const float sq = ((((xa[n] + xb[n]) + ya[n]) + yb[n]) + zs[n + P]) + zs[n + 1 + P];
    const float x = sq - h2 * rv[n];  // (cell_m * cell_m) * rhs, as relaxed_uniform forms the source
    float target = div6_core(x);
    if (k == 0 || k == nz - 1 || !div6_in_range(x)) {
      const float c0 = k > 0 ? 1.0f : (info.open_lo[2] == 1 ? ghost_coupling(info) : 0.0f);
      const float c1 = k < nz - 1 ? 1.0f : (info.open_hi[2] == 1 ? ghost_coupling(info) : 0.0f);
      target = x / ((4.0f + c0) + c1);  // neighbor_sum_uniform's couplings: 4 over x and y, then the z faces
    }
    out[n] = qv[n] + relaxation * (target - qv[n]);
  }
  *reinterpret_cast<float4*>(qs + own) = make_float4(out[0], out[1], out[2], out[3]);
}

__global__ void k_rb_split4(PlumeGridInfo info, int H, float* __restrict__ qs, const float* __restrict__ rs, int color,
                            float relaxation) {
  wait_for_previous_grid();
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int m0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= ny || m0 >= H) return;
  const int p = (i + j + color) & 1;  // cell k = 2 m + p
  const long plane = (long)ny * H;
  const long own = ((long)(color * nx + i) * ny + j) * H + m0;
  const long oth = ((long)((1 - color) * nx + i) * ny + j) * H + m0;
  // the other colour is not written by this pass
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {  // the same for a whole row: one branch per warp
    if (p == 0) split_row_interior<0>(info, H, qs, rs, own, oth, plane, m0, relaxation);
    else split_row_interior<1>(info, H, qs, rs, own, oth, plane, m0, relaxation);
    return;
  }
  const float4 q4 = ld4(qs + own), r4 = ldg4(rs + own);
  const float4 x0 = ldg4(qs + (i > 0 ? oth - plane : oth)), x1 = ldg4(qs + (i < nx - 1 ? oth + plane : oth));
  const float4 y0 = ldg4(qs + (j > 0 ? oth - H : oth)), y1 = ldg4(qs + (j < ny - 1 ? oth + H : oth));
  const float4 zc = ldg4(qs + oth);
  const int mz = p == 0 ? m0 - 1 : m0 + 4;
  const float zx = mz >= 0 && mz < H ? __ldg(qs + oth - m0 + mz) : 0.0f;
  const float qv[4] = {q4.x, q4.y, q4.z, q4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
  const float xa[4] = {x0.x, x0.y, x0.z, x0.w}, xb[4] = {x1.x, x1.y, x1.z, x1.w};
  const float ya[4] = {y0.x, y0.y, y0.z, y0.w}, yb[4] = {y1.x, y1.y, y1.z, y1.w};
  const float zs[6] = {zx, zc.x, zc.y, zc.z, zc.w, zx};  // the other colour's row at m0 - 1 .. m0 + 4
  const float ghost = ghost_coupling(info);
  float out[4] = {qv[0], qv[1], qv[2], qv[3]};
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const int k = 2 * (m0 + n) + p;
    if (k >= nz) continue;
    const float zm = p ? zs[n + 1] : zs[n], zp = p ? zs[n + 2] : zs[n + 1];  // at m - 1 + p and m + p
    auto load = [&](int a, int b, int c) {
      return a < i ? xa[n] : (a > i ? xb[n] : (b < j ? ya[n] : (b > j ? yb[n] : (c < k ? zm : zp))));
    };
    float value;
    if (relax_cell(true, info, ghost, i, j, k, qv[n], rv[n], relaxation, load, value)) out[n] = value;
  }
  *reinterpret_cast<float4*>(qs + own) = make_float4(out[0], out[1], out[2], out[3]);
}

// The natural-layout colour pass (k_rb_colour) with four consecutive cells of a row per thread, two of them of
// the colour: 16-byte loads of the row, of its four neighbouring rows and of rhs, and the one value beyond the
// four that the row's parity needs. The other colour's two values are stored back unchanged: this pass never
// writes them, so any thread reading them sees the same floats. Every update is relax_cell's. Rows of a
// multiple of four cells, 16-byte-aligned arrays.
// k_rb_colour4's two cells of a row with all four x and y neighbours on a uniform level, with split_row_interior's
// straight-line arithmetic (the value beyond the row's ends reads 0).
template <int P>
__device__ __forceinline__ void colour4_row_interior(const PlumeGridInfo& info, float* __restrict__ q,
                                                     const float* __restrict__ rhs, long row, long plane, int k0,
                                                     float relaxation) {
  const int nz = info.dims[2];
  const float4 c4 = ld4(q + row), r4 = ldg4(rhs + row);
  const float4 x0 = ld4(q + row - plane), x1 = ld4(q + row + plane);
  const float4 y0 = ld4(q + row - nz), y1 = ld4(q + row + nz);
  const int ze = P == 0 ? k0 - 1 : k0 + 4;
  const float zx = (P == 0 ? ze >= 0 : ze < nz) ? q[row - k0 + ze] : 0.0f;
  const float cv[4] = {c4.x, c4.y, c4.z, c4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
  const float xa[4] = {x0.x, x0.y, x0.z, x0.w}, xb[4] = {x1.x, x1.y, x1.z, x1.w};
  const float ya[4] = {y0.x, y0.y, y0.z, y0.w}, yb[4] = {y1.x, y1.y, y1.z, y1.w};
  const float h2 = info.cell_m * info.cell_m;
  float out[4] = {cv[0], cv[1], cv[2], cv[3]};
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    const int a = P + 2 * n, k = k0 + a;
    const float zm = a == 0 ? zx : cv[a > 0 ? a - 1 : 0], zp = a == 3 ? zx : cv[a < 3 ? a + 1 : 3];
    const float sq = ((((xa[a] + xb[a]) + ya[a]) + yb[a]) + zm) + zp;
    const float x = sq - h2 * rv[a];
    float target = div6_core(x);
    if (k == 0 || k == nz - 1 || !div6_in_range(x)) {
      const float c0 = k > 0 ? 1.0f : (info.open_lo[2] == 1 ? ghost_coupling(info) : 0.0f);
      const float c1 = k < nz - 1 ? 1.0f : (info.open_hi[2] == 1 ? ghost_coupling(info) : 0.0f);
      target = x / ((4.0f + c0) + c1);
    }
    out[a] = cv[a] + relaxation * (target - cv[a]);
  }
  *reinterpret_cast<float4*>(q + row) = make_float4(out[0], out[1], out[2], out[3]);
}

template <bool UNIFORM>
__global__ void k_rb_colour4(PlumeGridInfo info, float* __restrict__ q, const float* __restrict__ rhs, int color,
                             float relaxation) {
  wait_for_previous_grid();
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= ny || k0 >= nz) return;
  const int p = (i + j + color) & 1;  // this colour's cells: k0 + p and k0 + p + 2
  const long plane = (long)ny * nz, row = ((long)i * ny + j) * nz + k0;
  if (UNIFORM && i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {  // the same for a whole row
    if (p == 0) colour4_row_interior<0>(info, q, rhs, row, plane, k0, relaxation);
    else colour4_row_interior<1>(info, q, rhs, row, plane, k0, relaxation);
    return;
  }
  const float4 c4 = ld4(q + row), r4 = ldg4(rhs + row);
  const float4 x0 = ld4(q + (i > 0 ? row - plane : row)), x1 = ld4(q + (i < nx - 1 ? row + plane : row));
  const float4 y0 = ld4(q + (j > 0 ? row - nz : row)), y1 = ld4(q + (j < ny - 1 ? row + nz : row));
  const int ze = p == 0 ? k0 - 1 : k0 + 4;
  const float zx = ze >= 0 && ze < nz ? q[row - k0 + ze] : 0.0f;
  const float cv[4] = {c4.x, c4.y, c4.z, c4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
  const float xa[4] = {x0.x, x0.y, x0.z, x0.w}, xb[4] = {x1.x, x1.y, x1.z, x1.w};
  const float ya[4] = {y0.x, y0.y, y0.z, y0.w}, yb[4] = {y1.x, y1.y, y1.z, y1.w};
  const float ghost = ghost_coupling(info);
  float out[4] = {cv[0], cv[1], cv[2], cv[3]};
#pragma unroll
  for (int n = 0; n < 2; ++n) {
#pragma unroll
    for (int pp = 0; pp < 2; ++pp) {  // a = p + 2 n with p known per thread: both cases unrolled
      if (pp != p) continue;
      const int a = pp + 2 * n, k = k0 + a;
      const float zm = a == 0 ? zx : cv[a > 0 ? a - 1 : 0], zp = a == 3 ? zx : cv[a < 3 ? a + 1 : 3];
      auto load = [&](int aa, int b, int c) {
        return aa < i ? xa[a] : (aa > i ? xb[a] : (b < j ? ya[a] : (b > j ? yb[a] : (c < k ? zm : zp))));
      };
      float value;
      if (relax_cell(UNIFORM, info, ghost, i, j, k, cv[a], rv[a], relaxation, load, value)) out[a] = value;
    }
  }
  *reinterpret_cast<float4*>(q + row) = make_float4(out[0], out[1], out[2], out[3]);
}

// k_residual_restrict with the fine level in split storage, V (2 or 4) coarse cells kc0 .. kc0 + V - 1 per
// thread. The children of coarse cell kc sit at half index m = kc in both colours' rows (fk = 2 kc and
// 2 kc + 1 are one of each colour), so for each child (di, dj, dk) of the V cells the thread loads, as 8- or
// 16-byte rows at m = kc0 .., the child's own row and rhs, the other colour's row (its z neighbours) and the
// other colour's four neighbouring rows, plus the value beyond the V that an end's z neighbour needs. Every
// child's residual is residual_cell's on those values, and each coarse cell adds its children in the
// reference's order (di, dj, dk).
template <int V>
struct Row {
  float v[V];
};
template <int V>
__device__ __forceinline__ Row<V> ldg_row(const float* p) {
  Row<V> r;
  if constexpr (V == 4) {
    const float4 a = ldg4(p);
    r.v[0] = a.x, r.v[1] = a.y, r.v[2] = a.z, r.v[3] = a.w;
  } else {
    const float2 a = __ldg(reinterpret_cast<const float2*>(p));
    r.v[0] = a.x, r.v[1] = a.y;
  }
  return r;
}

#ifndef PLUME_RESTRICT_MINB
#define PLUME_RESTRICT_MINB 3
#endif
#ifndef PLUME_RESTRICT_CELLS
#define PLUME_RESTRICT_CELLS 4
#endif
template <int V, bool UNIFORM>
__global__ void __launch_bounds__(256, PLUME_RESTRICT_MINB)
    k_residual_restrict_split(PlumeGridInfo fine, int H, const float* __restrict__ qs, const float* __restrict__ rs,
                              Dims coarse, float* __restrict__ coarse_rhs, float* __restrict__ coarse_q) {
  wait_for_previous_grid();
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kc0 = V * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= coarse.n1 || kc0 >= coarse.n2) return;
  const Dims fd = dims_of(fine);
  constexpr bool uniform = UNIFORM;  // the level's couplings are all 1 (is_uniform), chosen on the host
  const float ghost = ghost_coupling(fine);
  const long colour_floats = (long)fd.n0 * fd.n1 * H;
  auto row = [&](int c, int a, int b) {  // (a, b)'s row of colour c at m = kc0, a and b clamped into the level
    a = imin_(imax_(a, 0), fd.n0 - 1);
    b = imin_(imax_(b, 0), fd.n1 - 1);
    return c * colour_floats + ((long)a * fd.n1 + b) * H + kc0;
  };
  float total[V], count[V];
#pragma unroll
  for (int n = 0; n < V; ++n) total[n] = count[n] = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int fi = 2 * i + di, fj = 2 * j + dj;
      if (fi >= fd.n0 || fj >= fd.n1) continue;
      const bool xy_interior = uniform && fi > 0 && fi < fd.n0 - 1 && fj > 0 && fj < fd.n1 - 1;
      const int c0 = (fi + fj) & 1;  // the colour of child dk = 0; child dk = 1 has the other
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const int cc = dk == 0 ? c0 : 1 - c0, oc = 1 - cc;
        const Row<V> own = ldg_row<V>(qs + row(cc, fi, fj)), rhs = ldg_row<V>(rs + row(cc, fi, fj));
        const Row<V> other = ldg_row<V>(qs + row(oc, fi, fj));
        const Row<V> xm = ldg_row<V>(qs + row(oc, fi - 1, fj)), xp = ldg_row<V>(qs + row(oc, fi + 1, fj));
        const Row<V> ym = ldg_row<V>(qs + row(oc, fi, fj - 1)), yp = ldg_row<V>(qs + row(oc, fi, fj + 1));
        // z neighbours in the other colour's row: child dk = 0 (fk = 2 kc) at m = kc - 1 and kc, child dk = 1
        // (fk = 2 kc + 1) at m = kc and kc + 1; the first needs m = kc0 - 1, the second m = kc0 + V
        const float beyond = dk == 0 ? (kc0 >= 1 ? __ldg(qs + row(oc, fi, fj) - 1) : 0.0f)
                                     : (kc0 + V < H ? __ldg(qs + row(oc, fi, fj) + V) : 0.0f);
#pragma unroll
        for (int n = 0; n < V; ++n) {
          const int fk = 2 * (kc0 + n) + dk;
          if (fk >= fd.n2) continue;
          const float zm = dk == 0 ? (n == 0 ? beyond : other.v[n > 0 ? n - 1 : 0]) : other.v[n];
          const float zp = dk == 0 ? other.v[n] : (n == V - 1 ? beyond : other.v[n < V - 1 ? n + 1 : V - 1]);
          if (xy_interior) {
            total[n] = total[n] + residual_xy_interior(fine, ghost, fk, own.v[n], rhs.v[n], xm.v[n], xp.v[n], ym.v[n],
                                                       yp.v[n], zm, zp);
            count[n] = count[n] + 1.0f;
            continue;
          }
          auto load = [&](int a, int b, int c) {
            return a < fi ? xm.v[n]
                          : (a > fi ? xp.v[n] : (b < fj ? ym.v[n] : (b > fj ? yp.v[n] : (c < fk ? zm : zp))));
          };
          total[n] = total[n] + residual_cell(uniform, fine, ghost, fi, fj, fk, own.v[n], rhs.v[n], load);
          count[n] = count[n] + 1.0f;
        }
      }
    }
#pragma unroll
  for (int n = 0; n < V; ++n) {
    if (kc0 + n >= coarse.n2) break;
    const int out = at(coarse, i, j, kc0 + n);
    coarse_rhs[out] = divide(total[n], divisor(count[n]));  // count is 1, 2, 4 or 8
    coarse_q[out] = 0.0f;
  }
}

// k_prolong_add with the fine level in split storage, four cells of a row per thread: thread (c, i, j, m0)
// adds to its cells m0 .. m0 + 3 of colour c. The four share the coarse sample's x and y axes; along z they
// read six consecutive coarse columns (m0 - 1 + p .. m0 + 4 + p, clamped), each blended in x then y once
// (sample_index_space's first lerps, which run per column in that order), and each cell blends its two
// columns in z: the same float operations as sample_index_space at prolong_point, with fewer loads and less
// index arithmetic.
__global__ void k_prolong_add_split4(Dims coarse, Dims fine, int H, const float* __restrict__ cq,
                                     float* __restrict__ qs) {
  wait_for_previous_grid();
  const int c = blockIdx.z / fine.n0, i = blockIdx.z - c * fine.n0;
  const int j = blockIdx.y * blockDim.y + threadIdx.y, m0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= fine.n1 || m0 >= H) return;
  const int p = (i + j + c) & 1;  // cell k = 2 m + p
  const F3 g = prolong_point(i, j, 2 * m0 + p);
  const Axis1 x = axis_of(g[0], coarse.n0, coarse.n1 * coarse.n2), y = axis_of(g[1], coarse.n1, coarse.n2);
  const float* base = cq + (x.i0 * coarse.n1 + y.i0) * coarse.n2;
  const int zbase = m0 - 1 + p;
  float e[6];
#pragma unroll
  for (int o = 0; o < 6; ++o) {
    const float* col = base + imin_(imax_(zbase + o, 0), coarse.n2 - 1);
    e[o] = lerp_w(lerp_w(__ldg(col), __ldg(col + x.step), x), lerp_w(__ldg(col + y.step), __ldg(col + x.step + y.step), x),
                  y);
  }
  const long own = ((long)(c * fine.n0 + i) * fine.n1 + j) * H + m0;
  const float4 q4 = ld4(qs + own);
  float out[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const int k = 2 * (m0 + n) + p;
    if (k >= fine.n2) continue;
    const F3 gk = prolong_point(i, j, k);
    const Axis1 z = axis_of(gk[2], coarse.n2, 1);
    const int off = z.i0 - zbase;  // n, or n + 1 where the lower clamp holds the first cell at column 0
    float value;
    if (off == n || off == n + 1) {
      const float lo = off == n ? e[n] : e[n + 1];
      const float hi = z.step == 0 ? lo : (off == n ? e[n + 1] : e[n + 2]);
      value = lerp_w(lo, hi, z);
    } else {
      value = sample_index_space(cq, coarse, gk);
    }
    out[n] = out[n] + value;
  }
  *reinterpret_cast<float4*>(qs + own) = make_float4(out[0], out[1], out[2], out[3]);
}

// k_prolong_add_split4 for both colours of four half indices m0 .. m0 + 3 of a row per thread (eight fine cells
// k = 2 m0 .. 2 m0 + 7), on a coarse level whose rows hold a multiple of four cells. The eight share the coarse
// sample's x and y axes, and along z they read the seven coarse columns m0 - 1 .. m0 + 5 (clamped), fetched
// from each of the four (x, y) rows as one 16-byte load, one 8-byte load and one 4-byte load. Each column is
// blended in x then y once, and each cell blends its two columns in z: sample_index_space's operations at
// prolong_point, as in k_prolong_add_split4.
__device__ __forceinline__ float pick7(const float* e, int o) {
  return o == 0 ? e[0] : o == 1 ? e[1] : o == 2 ? e[2] : o == 3 ? e[3] : o == 4 ? e[4] : o == 5 ? e[5] : e[6];
}

// The z blend of k_prolong_add_split8 for the four cells k = 2 (m0 + n) + P of a row. Cell m of parity P sits at
// coarse z = m - 0.25 (P = 0: columns m - 1 and m, weight 0.75 on m) or m + 0.25 (P = 1: columns m and m + 1,
// weight 0.25 on m + 1); axis_of forms exactly those indices and weights (t = 0.75 or 0.25, 1 - t = 0.25 or
// 0.75, all exact) except where a clamp holds: cell m = 0 of parity 0 and cell m = n2 - 1 of parity 1, which
// take the general blend.
template <int P>
__device__ __forceinline__ void prolong_row(const float* e, float* out, int i, int j, int m0, const Dims& coarse,
                                            const Dims& fine, const float* __restrict__ cq) {
  constexpr float t = P == 0 ? 0.75f : 0.25f, u = P == 0 ? 0.25f : 0.75f;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const int m = m0 + n, k = 2 * m + P;
    if (k >= fine.n2) continue;
    float value = e[n + P] * u + e[n + P + 1] * t;  // lerp_w(column m - 1 + P, column m + P, z)
    if ((P == 0 && m == 0) || (P == 1 && m == coarse.n2 - 1)) {
      const F3 gk = prolong_point(i, j, k);
      const Axis1 z = axis_of(gk[2], coarse.n2, 1);
      const int off = z.i0 - (m0 - 1);  // the clamped cell's column in e
      if (off >= 0 && off <= 5) {
        const float lo = pick7(e, off);
        value = lerp_w(lo, z.step == 0 ? lo : pick7(e, off + 1), z);
      } else {
        value = sample_index_space(cq, coarse, gk);
      }
    }
    out[n] = out[n] + value;
  }
}

__global__ void k_prolong_add_split8(Dims coarse, Dims fine, int H, const float* __restrict__ cq,
                                     float* __restrict__ qs) {
  wait_for_previous_grid();
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, m0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= fine.n1 || m0 >= H) return;
  const F3 g = prolong_point(i, j, 0);
  const Axis1 x = axis_of(g[0], coarse.n0, coarse.n1 * coarse.n2), y = axis_of(g[1], coarse.n1, coarse.n2);
  const float* base = cq + (x.i0 * coarse.n1 + y.i0) * coarse.n2;
  const float* rows[4] = {base, base + x.step, base + y.step, base + x.step + y.step};
  float c[4][7];  // row r's columns m0 - 1 .. m0 + 5, clamped into the row
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float4 mid = ldg4(rows[r] + m0);
    const float lo = m0 > 0 ? __ldg(rows[r] + m0 - 1) : mid.x;
    float2 hi;
    if (m0 + 4 < coarse.n2) hi = __ldg(reinterpret_cast<const float2*>(rows[r] + m0 + 4));
    else hi = make_float2(mid.w, mid.w);
    c[r][0] = lo, c[r][1] = mid.x, c[r][2] = mid.y, c[r][3] = mid.z, c[r][4] = mid.w, c[r][5] = hi.x, c[r][6] = hi.y;
  }
  float e[7];
#pragma unroll
  for (int o = 0; o < 7; ++o) e[o] = lerp_w(lerp_w(c[0][o], c[1][o], x), lerp_w(c[2][o], c[3][o], x), y);
#pragma unroll
  for (int col = 0; col < 2; ++col) {
    const int p = (i + j + col) & 1;  // cell k = 2 m + p
    const long own = ((long)(col * fine.n0 + i) * fine.n1 + j) * H + m0;
    const float4 q4 = ld4(qs + own);
    float out[4] = {q4.x, q4.y, q4.z, q4.w};
    if (p == 0) prolong_row<0>(e, out, i, j, m0, coarse, fine, cq);
    else prolong_row<1>(e, out, i, j, m0, coarse, fine, cq);
    *reinterpret_cast<float4*>(qs + own) = make_float4(out[0], out[1], out[2], out[3]);
  }
}

// ---- the cluster coarse solve --------------------------------------------------------------------------------
// Every level from `first` down runs in one launch of one thread-block cluster (CLUSTER CTAs, one per SM).
// A level above SINGLE_MAX_CELLS cells is split into slabs of whole x-planes, one slab per CTA, held in that
// CTA's shared memory; a CTA reads its neighbours' boundary planes through distributed shared memory and
// the cluster barrier separates the passes. Smaller levels live in CTA 0 alone and run with block or warp
// barriers while the other CTAs wait at the next cluster barrier. Every cell gets exactly the reference's
// update; only where the values are stored differs.

constexpr int CLUSTER = 8;
constexpr long SINGLE_MAX_CELLS = 1024;

struct LevelView {
  PlumeGridInfo info;
  float* q;        // global arrays (loaded for the first level, written back for all)
  float* rhs;
  int planes;      // x-planes per CTA (the whole level when single)
  int single;      // 1: the level lives in CTA 0
  int offset;      // shared-memory float offset of the level's q block; its rhs block follows
};

struct ClusterArgs {
  int count;
  int sweeps;
  LevelView lv[BOTTOM_MAX_LEVELS];
};

namespace cg = cooperative_groups;

struct ClusterCtx {
  cg::cluster_group cluster;
  float* smem;
  int rank;
};

// The CTA holding plane i (no division: slabs are `planes` planes long, CLUSTER of them).
__device__ __forceinline__ int owner_of(const LevelView& L, int i) {
  if (L.single) return 0;
  int owner = 0;
#pragma unroll
  for (int r = 1; r < CLUSTER; ++r) owner += i >= r * L.planes;
  return owner;
}

__device__ __forceinline__ int local_index(const LevelView& L, int owner, int i, int j, int k, bool rhs) {
  const int n1 = L.info.dims[1], n2 = L.info.dims[2];
  const int li = L.single ? i : i - owner * L.planes;
  return L.offset + (rhs ? L.planes * n1 * n2 : 0) + (li * n1 + j) * n2 + k;
}

// q (or rhs) of a cell, read from whichever CTA holds its plane: a shared-memory load when it is this CTA.
__device__ __forceinline__ float cell_load(const ClusterCtx& c, const LevelView& L, int i, int j, int k, bool rhs) {
  const int owner = owner_of(L, i);
  const int idx = local_index(L, owner, i, j, k, rhs);
  if (owner == c.rank) return c.smem[idx];
  return *c.cluster.map_shared_rank(c.smem + idx, owner);
}

__device__ __forceinline__ void cell_store(const ClusterCtx& c, const LevelView& L, int i, int j, int k, bool rhs,
                                           float value) {
  const int owner = owner_of(L, i);
  const int idx = local_index(L, owner, i, j, k, rhs);
  if (owner == c.rank) c.smem[idx] = value;
  else *c.cluster.map_shared_rank(c.smem + idx, owner) = value;
}

// The x-planes [lo, hi) a CTA works on in a pass over level L: its own slab, or everything in CTA 0.
__device__ __forceinline__ void my_planes(const ClusterCtx& c, const LevelView& L, int& lo, int& hi) {
  const int n0 = L.info.dims[0];
  if (L.single) {
    lo = 0;
    hi = c.rank == 0 ? n0 : 0;
    return;
  }
  lo = imin_(c.rank * L.planes, n0);
  hi = imin_(lo + L.planes, n0);
}

// One pass of cells of one colour over the planes [lo, hi), `threads` threads from thread 0.
template <class Update>
__device__ __forceinline__ void for_colour(const LevelView& L, int lo, int hi, int color, int threads, Update update) {
  const int n1 = L.info.dims[1], n2 = L.info.dims[2];
  const int pairs_k = (n2 + 1) / 2;
  const int per_plane = n1 * pairs_k;
  const int pairs = (hi - lo) * per_plane;
  for (int p = threadIdx.x; p < pairs; p += threads) {
    const int a = p / per_plane, rem = p - a * per_plane, j = rem / pairs_k, kp = rem - j * pairs_k;
    const int i = lo + a;
    const int k = 2 * kp + ((i + j + color) & 1);
    if (k < n2) update(i, j, k);
  }
}

// `sweeps` red-black sweeps of level L. Neighbours in the same x-plane are always this CTA's; the x-1 and
// x+1 planes come from the neighbouring CTAs' shared memory at the slab edges. A single level small enough
// for one warp syncs at warp level.
__device__ void cluster_smooth(const ClusterCtx& c, const LevelView& L, int sweeps, float relaxation) {
  const PlumeGridInfo& info = L.info;
  const bool uniform = is_uniform(info);
  const float ghost = ghost_coupling(info);
  const int n0 = info.dims[0], n1 = info.dims[1], n2 = info.dims[2];
  const int plane = n1 * n2;
  int lo, hi;
  my_planes(c, L, lo, hi);
  float* q = c.smem + L.offset;               // this CTA's planes [lo, hi), then their rhs
  const float* rhs = q + L.planes * plane;
  const float* q_prev = (!L.single && lo > 0 && lo < hi) ? c.cluster.map_shared_rank(q + (L.planes - 1) * plane, c.rank - 1)
                                                         : nullptr;
  const float* q_next = (!L.single && hi < n0 && lo < hi) ? c.cluster.map_shared_rank(q, c.rank + 1) : nullptr;
  auto update = [&](int i, int j, int k) {
    const int idx = (i - lo) * plane + j * n2 + k;
    auto load = [&](int a, int b, int cc) {
      if (a == i) return q[idx + (b - j) * n2 + (cc - k)];
      if (a == i - 1) return i - 1 >= lo ? q[idx - plane] : q_prev[j * n2 + k];
      return i + 1 < hi ? q[idx + plane] : q_next[j * n2 + k];
    };
    float out;
    if (relax_cell(uniform, info, ghost, i, j, k, q[idx], rhs[idx], relaxation, load, out)) q[idx] = out;
  };
  const int pairs_k = (n2 + 1) / 2;
  const int per_plane = n1 * pairs_k;
  const int t = threadIdx.x;
  auto colour_pass = [&](int color, int threads) {
    if (per_plane <= threads && (hi - lo) * per_plane > threads) {  // each thread owns a column of every plane
      if (t < per_plane) {
        const int j = t / pairs_k, kp = t - j * pairs_k;
        for (int i = lo; i < hi; ++i) {
          const int k = 2 * kp + ((i + j + color) & 1);
          if (k < n2) update(i, j, k);
        }
      }
    } else {
      for_colour(L, lo, hi, color, threads, update);
    }
  };
  if (L.single) {
    const int pairs = n0 * per_plane;
    const bool one_warp = pairs <= BOTTOM_WARP_PAIRS;
    if (c.rank == 0 && (!one_warp || t < 32)) {
      for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
          if (one_warp) {
            for_colour(L, lo, hi, color, 32, update);
            __syncwarp();
          } else {
            colour_pass(color, BOTTOM_THREADS);
            __syncthreads();
          }
        }
    }
    if (c.rank == 0) __syncthreads();  // the rest of CTA 0 waits for the warp that did the work
    return;
  }
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      colour_pass(color, BOTTOM_THREADS);
      c.cluster.sync();
    }
}

// residual + restriction + zero coarse pressure (multigrid.py:36-60, :143) from F into C. Coarse planes are
// shared out over the CTAs by slab; each writes into whichever CTA holds the coarse plane.
__device__ void cluster_restrict(const ClusterCtx& c, const LevelView& F, const LevelView& C, bool single_only) {
  const PlumeGridInfo& info = F.info;
  const Dims fd = dims_of(info), cd = dims_of(C.info);
  const bool uniform = is_uniform(info);
  const float ghost = ghost_coupling(info);
  auto load = [&](int a, int b, int k) { return cell_load(c, F, a, b, k, false); };
  int lo, hi;
  if (single_only) {
    lo = 0;
    hi = c.rank == 0 ? cd.n0 : 0;
  } else {
    const int per = (cd.n0 + CLUSTER - 1) / CLUSTER;
    lo = imin_(c.rank * per, cd.n0);
    hi = imin_(lo + per, cd.n0);
  }
  const int cells = (hi - lo) * cd.n1 * cd.n2;
  for (int idx = threadIdx.x; idx < cells; idx += BOTTOM_THREADS) {
    const int a = idx / (cd.n1 * cd.n2), rem = idx - a * (cd.n1 * cd.n2), j = rem / cd.n2, k = rem - j * cd.n2;
    const int i = lo + a;
    float total = 0.0f, count = 0.0f;
    for (int di = 0; di < 2; ++di)
      for (int dj = 0; dj < 2; ++dj)
        for (int dk = 0; dk < 2; ++dk) {
          const int fi = 2 * i + di, fj = 2 * j + dj, fk = 2 * k + dk;
          if (fi < fd.n0 && fj < fd.n1 && fk < fd.n2) {
            total = total + residual_cell(uniform, info, ghost, fi, fj, fk, cell_load(c, F, fi, fj, fk, false),
                                          cell_load(c, F, fi, fj, fk, true), load);
            count = count + 1.0f;
          }
        }
    cell_store(c, C, i, j, k, true, total / count);
    cell_store(c, C, i, j, k, false, 0.0f);
  }
}

// prolong_add_kernel (multigrid.py:63-68): each CTA adds the coarse correction to the fine planes it holds.
__device__ void cluster_prolong(const ClusterCtx& c, const LevelView& F, const LevelView& C) {
  const Dims fd = dims_of(F.info), cd = dims_of(C.info);
  int lo, hi;
  my_planes(c, F, lo, hi);
  const int cells = (hi - lo) * fd.n1 * fd.n2;
  for (int idx = threadIdx.x; idx < cells; idx += BOTTOM_THREADS) {
    const int a = idx / (fd.n1 * fd.n2), rem = idx - a * (fd.n1 * fd.n2), j = rem / fd.n2, k = rem - j * fd.n2;
    const int i = lo + a;
    const F3 g = prolong_point(i, j, k);  // sample_index_space (sample.py:10-29) on the coarse level
    const float x = clampf_(g[0], 0.0f, (float)(cd.n0 - 1)), y = clampf_(g[1], 0.0f, (float)(cd.n1 - 1)),
                z = clampf_(g[2], 0.0f, (float)(cd.n2 - 1));
    const int i0 = (int)x, j0 = (int)y, k0 = (int)z;
    const int i1 = imin_(i0 + 1, cd.n0 - 1), j1 = imin_(j0 + 1, cd.n1 - 1), k1 = imin_(k0 + 1, cd.n2 - 1);
    const float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
    auto cq = [&](int a2, int b2, int k2) { return cell_load(c, C, a2, b2, k2, false); };
    const float c00 = lerpf_(cq(i0, j0, k0), cq(i1, j0, k0), tx);
    const float c10 = lerpf_(cq(i0, j1, k0), cq(i1, j1, k0), tx);
    const float c01 = lerpf_(cq(i0, j0, k1), cq(i1, j0, k1), tx);
    const float c11 = lerpf_(cq(i0, j1, k1), cq(i1, j1, k1), tx);
    const int at_q = local_index(F, c.rank, i, j, k, false);  // a plane this CTA holds
    c.smem[at_q] = c.smem[at_q] + lerpf_(lerpf_(c00, c10, ty), lerpf_(c01, c11, ty), tz);
  }
}

// A barrier for the level just processed: the cluster for split levels, CTA 0's block for single ones.
__device__ __forceinline__ void level_barrier(const ClusterCtx& c, bool cluster_wide) {
  if (cluster_wide) c.cluster.sync();
  else if (c.rank == 0) __syncthreads();
}

__global__ void __launch_bounds__(BOTTOM_THREADS) k_cluster_solve(ClusterArgs b) {
  extern __shared__ float smem[];
  ClusterCtx c{cg::this_cluster(), smem, (int)cg::this_cluster().block_rank()};
  {  // the first level's pressure and right-hand side, each CTA its planes
    const LevelView& L = b.lv[0];
    int lo, hi;
    my_planes(c, L, lo, hi);
    const int n1 = L.info.dims[1], n2 = L.info.dims[2];
    const int cells = (hi - lo) * n1 * n2;
    const long base = (long)lo * n1 * n2;
    float* q = smem + L.offset;
    float* rhs = q + L.planes * n1 * n2;
    for (int idx = threadIdx.x; idx < cells; idx += BOTTOM_THREADS) {
      q[idx] = L.q[base + idx];
      rhs[idx] = L.rhs[base + idx];
    }
  }
  c.cluster.sync();
  const int last = b.count - 1;
  for (int l = 0; l < last; ++l) {  // down: smooth, then residual and restriction into the next level
    const LevelView& F = b.lv[l];
    const LevelView& C = b.lv[l + 1];
    cluster_smooth(c, F, b.sweeps, 1.0f);
    cluster_restrict(c, F, C, F.single != 0);
    level_barrier(c, F.single == 0);
  }
  {  // the coarsest solve (multigrid.py:132-136)
    const LevelView& L = b.lv[last];
    const int longest = imax_(L.info.dims[0], imax_(L.info.dims[1], L.info.dims[2]));
    cluster_smooth(c, L, imax_(COARSEST_SWEEPS, COARSEST_SWEEPS_PER_CELL * longest), 1.5f);
  }
  for (int l = last - 1; l >= 0; --l) {  // up: prolong the coarse correction, smooth
    const LevelView& F = b.lv[l];
    const LevelView& C = b.lv[l + 1];
    if (F.single == 0 && C.single) c.cluster.sync();  // the single part is done before its correction is read
    cluster_prolong(c, F, C);
    level_barrier(c, F.single == 0);
    cluster_smooth(c, F, b.sweeps, 1.0f);
  }
  c.cluster.sync();
  for (int l = 0; l < b.count; ++l) {  // every level's pressure (and the coarse right-hand sides) back out
    const LevelView& L = b.lv[l];
    int lo, hi;
    my_planes(c, L, lo, hi);
    const int n1 = L.info.dims[1], n2 = L.info.dims[2];
    const int cells = (hi - lo) * n1 * n2;
    const long base = (long)lo * n1 * n2;
    const float* q = smem + L.offset;
    const float* rhs = q + L.planes * n1 * n2;
    for (int idx = threadIdx.x; idx < cells; idx += BOTTOM_THREADS) {
      L.q[base + idx] = q[idx];
      if (l > 0) L.rhs[base + idx] = rhs[idx];
    }
  }
  c.cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// ---- the one-block coarse solve (alternative bottom: every level in one CTA's shared memory) --------------

struct BlockArgs {
  int count;
  int sweeps;
  PlumeLevel lv[BOTTOM_MAX_LEVELS];
  int offset[BOTTOM_MAX_LEVELS];
  int coef_offset[BOTTOM_MAX_LEVELS];  // a level with overhanging cells: its CellCoef table's float offset (else -1)
  int f64_offset;  // k_block_solve<true, ...>: the coarsest level's double copy, from this float offset
};

// The stencil of one cell of a level with overhanging cells (fill_hi < 1), as neighbor_sum and relaxed compute
// it: the six couplings in neighbor_sum's order (x-, x+, y-, y+, z-, z+; a ghost's coupling, or 0 for a closed
// face, where the neighbour is outside the level), their sum sc added in that order, and the source scale
// vc = (cell_volume * cell_m) * cell_m. The one-block solve builds these once per launch for its non-uniform
// levels, so each sweep's update is loads, products and sums, without neighbor_sum's seven divisions.
struct CellCoef {
  float c[6];
  float sc, vc;
};

__device__ __forceinline__ CellCoef cell_coef(const PlumeGridInfo& info, int i, int j, int k) {
  const int c[3] = {i, j, k};
  CellCoef out;
  float sc = 0.0f;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    float area = 1.0f;
#pragma unroll
    for (int other = 0; other < 3; ++other)
      if (other != axis) area = area * cell_fill(info, other, c[other]);
    const float own = cell_fill(info, axis, c[axis]);
    float tc[2];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int step = side == 0 ? -1 : 1;
      const int n = c[axis] + step;
      if (n >= 0 && n < info.dims[axis]) tc[side] = area / (0.5f * (own + cell_fill(info, axis, n)));
      else if ((step < 0 && info.open_lo[axis] == 1) || (step > 0 && info.open_hi[axis] == 1))
        tc[side] = area / (0.5f * own + info.ghost_gap);
      else tc[side] = 0.0f;
      out.c[2 * axis + side] = tc[side];
    }
    sc = (sc + tc[0]) + tc[1];
  }
  out.sc = sc;
  out.vc = cell_volume(info, i, j, k) * info.cell_m * info.cell_m;
  return out;
}

// neighbor_sum's sq from a cell's table entry: the in-level neighbours' coupling * pressure, 0 for the rest,
// added in its order.
__device__ __forceinline__ float coef_sum(const CellCoef& e, const float* q, const Dims& d, int i, int j, int k) {
  const int c[3] = {i, j, k}, n[3] = {d.n0, d.n1, d.n2}, stride[3] = {d.n1 * d.n2, d.n2, 1};
  const int own = at(d, i, j, k);
  float sq = 0.0f;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    const float t0 = c[axis] > 0 ? e.c[2 * axis] * q[own - stride[axis]] : 0.0f;
    const float t1 = c[axis] < n[axis] - 1 ? e.c[2 * axis + 1] * q[own + stride[axis]] : 0.0f;
    sq = (sq + t0) + t1;
  }
  return sq;
}

// The coarsest level's sweeps in double (the defect-correction solve's correction cycles; no reference
// counterpart): q and rhs widened into `dq`/`drhs`, the red-black sweeps of relaxed_f64 over the whole block,
// q rounded back to float.
__device__ __forceinline__ void coarsest_f64(const PlumeGridInfo& info, float* q, const float* rhs, int sweeps,
                                             double relaxation, double* dq, double* drhs) {
  const Dims d = dims_of(info);
  const int n = d.n0 * d.n1 * d.n2;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    dq[idx] = q[idx];
    drhs[idx] = rhs[idx];
  }
  __syncthreads();
  auto load = [&](int a, int b, int c) { return dq[at(d, a, b, c)]; };
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
        const int i = idx / (d.n1 * d.n2), r = idx - i * d.n1 * d.n2, j = r / d.n2, k = r - j * d.n2;
        if (((i + j + k) & 1) != color) continue;
        double out;
        if (relaxed_f64(info, i, j, k, dq[idx], drhs[idx], relaxation, load, out)) dq[idx] = out;
      }
      __syncthreads();
    }
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) q[idx] = (float)dq[idx];
  __syncthreads();
}

// The coarsest level in double when it is not inside the one-block solve: one block, arrays in global memory.
__global__ void __launch_bounds__(BOTTOM_THREADS) k_coarsest_f64(PlumeGridInfo info, float* q, const float* rhs,
                                                                 int sweeps) {
  wait_for_previous_grid();
  extern __shared__ double staged[];
  const int n = info.dims[0] * info.dims[1] * info.dims[2];
  coarsest_f64(info, q, rhs, sweeps, 1.5, staged, staged + n);
}

// Visits the index triples (i, j, c) of p = start, start + stride, ... in an (n0, n1, nc) box without a
// division per step: one division at the start, then the stride's own (di, dj, dc) added with carries.
struct Walk {
  int i, j, c, di, dj, dc, n1, nc;
  __device__ Walk(int start, int stride, int n1_, int nc_) : n1(n1_), nc(nc_) {
    const int plane = n1 * nc;
    i = start / plane;
    int r = start - i * plane;
    j = r / nc;
    c = r - j * nc;
    di = stride / plane;
    r = stride - di * plane;
    dj = r / nc;
    dc = r - dj * nc;
  }
  __device__ __forceinline__ void next() {
    c += dc;
    if (c >= nc) {
      c -= nc;
      ++j;
    }
    j += dj;
    if (j >= n1) {
      j -= n1;
      ++i;
    }
    i += di;
  }
};

// The cells of one colour that a thread updates in the one-block solve, with everything about them that stays
// fixed through a smoothing call held in registers: the cell's and its six neighbours' shared-memory indices
// (16 bits each, 0xffff for a neighbour outside the level), and the coupling total sc and the source term
// (cell_m * cell_m) * rhs of relaxed_uniform. A sweep pass is then seven shared loads, the sums and the update: the same float operations as relaxed_uniform, with
// an interior cell's sum (((((a + b) + c) + d) + e) + f) taken as ((((((0 + a) + b) + c) + d) + e) + f), equal
// in value (0 + a == a up to the sign of a zero).
constexpr int STENCIL_SLOTS = 2;
constexpr unsigned NO_CELL = 0xffffu;

struct StencilSlot {
  unsigned own_and_x0, x1_y0, y1_z0, z1;  // pairs of 16-bit indices
  float sc, source;
};

__device__ __forceinline__ unsigned pack16(unsigned lo, unsigned hi) { return (lo & 0xffffu) | (hi << 16); }

__device__ __forceinline__ StencilSlot stencil_slot(const PlumeGridInfo& info, const Dims& d, float ghost, const float* q,
                                                    const float* rhs, int p, int pairs_k, int color) {
  StencilSlot slot;
  slot.own_and_x0 = NO_CELL;
  const int i = p / (d.n1 * pairs_k), r = p - i * (d.n1 * pairs_k);
  const int j = r / pairs_k, k = 2 * (r - j * pairs_k) + ((i + j + color) & 1);
  if (k >= d.n2) return slot;
  const int c[3] = {i, j, k};
  const int stride[3] = {d.n1 * d.n2, d.n2, 1};
  const int own = at(d, i, j, k);
  unsigned nb[6];
  float sc = 0.0f;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {  // neighbor_sum_uniform's couplings, in its order
    float tc0 = 0.0f, tc1 = 0.0f;
    nb[2 * axis] = nb[2 * axis + 1] = NO_CELL;
    if (c[axis] > 0) {
      nb[2 * axis] = own - stride[axis];
      tc0 = 1.0f;
    } else if (info.open_lo[axis] == 1) {
      tc0 = ghost;
    }
    if (c[axis] < info.dims[axis] - 1) {
      nb[2 * axis + 1] = own + stride[axis];
      tc1 = 1.0f;
    } else if (info.open_hi[axis] == 1) {
      tc1 = ghost;
    }
    sc = (sc + tc0) + tc1;
  }
  if (sc == 0.0f) return slot;  // no coupling at all: relaxed_uniform leaves the cell alone
  slot.own_and_x0 = pack16(own, nb[0]);
  slot.x1_y0 = pack16(nb[1], nb[2]);
  slot.y1_z0 = pack16(nb[3], nb[4]);
  slot.z1 = nb[5];
  slot.sc = sc;
  slot.source = info.cell_m * info.cell_m * rhs[own];
  return slot;
}

__device__ __forceinline__ float neighbour16(const float* q, unsigned index) { return index == NO_CELL ? 0.0f : q[index]; }

__device__ __forceinline__ void relax_slot(float* q, const StencilSlot& slot, float relaxation) {
  if ((slot.own_and_x0 & 0xffffu) == NO_CELL) return;
  const float a = neighbour16(q, slot.own_and_x0 >> 16), b = neighbour16(q, slot.x1_y0 & 0xffffu);
  const float c = neighbour16(q, slot.x1_y0 >> 16), e = neighbour16(q, slot.y1_z0 & 0xffffu);
  const float f = neighbour16(q, slot.y1_z0 >> 16), g = neighbour16(q, slot.z1);
  const float sq = (((((0.0f + a) + b) + c) + e) + f) + g;
  const float target = (sq - slot.source) / slot.sc;
  float* own = q + (slot.own_and_x0 & 0xffffu);
  *own = *own + relaxation * (target - *own);
}

// `sweeps` red-black sweeps of a uniform level from register-held stencils: `lanes` threads (one warp or the
// whole block) with at most STENCIL_SLOTS cells of each colour each. Returns false, having done nothing, when
// the level does not fit that.
__device__ __forceinline__ bool stencil_smooth(const PlumeGridInfo& info, float* q, const float* rhs, int sweeps, float relaxation) {
  const Dims d = dims_of(info);
  const int pairs_k = (d.n2 + 1) / 2;
  const int pairs = d.n0 * d.n1 * pairs_k;
  const bool one_warp = pairs <= 32 * STENCIL_SLOTS;
  const int lanes = one_warp ? 32 : BOTTOM_THREADS;
  if (!is_uniform(info) || pairs > lanes * STENCIL_SLOTS || d.n0 * d.n1 * d.n2 >= (int)NO_CELL) return false;
  if (!one_warp || threadIdx.x < 32) {
    const float ghost = ghost_coupling(info);
    StencilSlot slot[2][STENCIL_SLOTS];
#pragma unroll
    for (int color = 0; color < 2; ++color)
#pragma unroll
      for (int n = 0; n < STENCIL_SLOTS; ++n) {
        const int p = threadIdx.x + n * lanes;
        if (p < pairs) slot[color][n] = stencil_slot(info, d, ghost, q, rhs, p, pairs_k, color);
        else slot[color][n].own_and_x0 = NO_CELL;
      }
    for (int s = 0; s < sweeps; ++s)
#pragma unroll
      for (int color = 0; color < 2; ++color) {
#pragma unroll
        for (int n = 0; n < STENCIL_SLOTS; ++n) relax_slot(q, slot[color][n], relaxation);
        if (one_warp) __syncwarp();
        else __syncthreads();
      }
  }
  __syncthreads();
  return true;
}

// block_smooth of a level with overhanging cells from its CellCoef table: relaxed's operations, the couplings
// read from the table. Out of line, so that the uniform levels' register stencils keep their registers.
__device__ __noinline__ void table_smooth(Dims d, float* q, const float* rhs, int sweeps, float relaxation,
                                          const CellCoef* coef) {
  const int pairs_k = (d.n2 + 1) / 2;
  const int pairs = d.n0 * d.n1 * pairs_k;
  const bool one_warp = pairs <= BOTTOM_WARP_PAIRS;
  if (!one_warp || threadIdx.x < 32) {
    for (int s = 0; s < sweeps; ++s)
      for (int color = 0; color < 2; ++color) {
        const int stride = one_warp ? 32 : BOTTOM_THREADS;
        Walk w((int)threadIdx.x, stride, d.n1, pairs_k);
        for (int p = threadIdx.x; p < pairs; p += stride, w.next()) {
          const int i = w.i, j = w.j;
          const int k = 2 * w.c + ((i + j + color) & 1);
          if (k >= d.n2) continue;
          const int idx = at(d, i, j, k);
          const CellCoef& e = coef[idx];
          if (e.sc == 0.0f) continue;
          const float sq = coef_sum(e, q, d, i, j, k);
          const float source = e.vc * rhs[idx];
          const float target = (sq - source) / e.sc;
          q[idx] = q[idx] + relaxation * (target - q[idx]);
        }
        if (one_warp) __syncwarp();
        else __syncthreads();
      }
  }
  __syncthreads();
}

// residual_at of a level with overhanging cells from its CellCoef table.
__device__ __noinline__ float table_residual(const CellCoef* coef, const float* q, const float* rhs, Dims d, int i, int j,
                                             int k) {
  const int f = at(d, i, j, k);
  const CellCoef& e = coef[f];
  return rhs[f] - divide(coef_sum(e, q, d, i, j, k) - e.sc * q[f], divisor(e.vc));
}

__device__ __forceinline__ void block_smooth(const PlumeGridInfo& info, float* q, const float* rhs, int sweeps, float relaxation,
                                             const CellCoef* coef = nullptr) {
  if (coef) return table_smooth(dims_of(info), q, rhs, sweeps, relaxation, coef);
  if (stencil_smooth(info, q, rhs, sweeps, relaxation)) return;
  const Dims d = dims_of(info);
  const int pairs_k = (d.n2 + 1) / 2;
  const int pairs = d.n0 * d.n1 * pairs_k;
  auto load = [&](int a, int b, int c) { return q[at(d, a, b, c)]; };
  const bool uniform = is_uniform(info);
  const float ghost = ghost_coupling(info);
  const bool one_warp = pairs <= BOTTOM_WARP_PAIRS;
  if (!one_warp || threadIdx.x < 32) {
    for (int s = 0; s < sweeps; ++s)
      for (int color = 0; color < 2; ++color) {
        const int stride = one_warp ? 32 : BOTTOM_THREADS;
        Walk w((int)threadIdx.x, stride, d.n1, pairs_k);
        for (int p = threadIdx.x; p < pairs; p += stride, w.next()) {
          const int i = w.i, j = w.j;
          const int k = 2 * w.c + ((i + j + color) & 1);
          if (k >= d.n2) continue;
          const int idx = at(d, i, j, k);
          float out;
          if (relax_cell(uniform, info, ghost, i, j, k, q[idx], rhs[idx], relaxation, load, out)) q[idx] = out;
        }
        if (one_warp) __syncwarp();
        else __syncthreads();
      }
  }
  __syncthreads();
}

// TABLES: some level has overhanging cells (CellCoef tables in b.coef_offset); without, the uniform levels'
// code is compiled alone.
template <bool COARSE_F64, bool TABLES>
__global__ void __launch_bounds__(BOTTOM_THREADS) k_block_solve(BlockArgs b) {
  wait_for_previous_grid();
  extern __shared__ float smem[];
  const int t = threadIdx.x;
  {
    const Dims d = dims_of(b.lv[0].info);
    const int n = d.n0 * d.n1 * d.n2;
    float* q = smem + b.offset[0];
    for (int idx = t; idx < n; idx += BOTTOM_THREADS) {
      q[idx] = b.lv[0].q[idx];
      q[n + idx] = b.lv[0].rhs[idx];
    }
  }
  auto coef_of = [&](int l) -> CellCoef* {
    if constexpr (TABLES) return b.coef_offset[l] >= 0 ? reinterpret_cast<CellCoef*>(smem + b.coef_offset[l]) : nullptr;
    else return nullptr;
  };
  for (int l = 0; TABLES && l < b.count; ++l) {
    CellCoef* table = coef_of(l);
    if (!table) continue;
    const Dims d = dims_of(b.lv[l].info);
    Walk w(t, BOTTOM_THREADS, d.n1, d.n2);
    for (int idx = t; idx < d.n0 * d.n1 * d.n2; idx += BOTTOM_THREADS, w.next())
      table[idx] = cell_coef(b.lv[l].info, w.i, w.j, w.c);
  }
  __syncthreads();
  for (int l = 0; l + 1 < b.count; ++l) {
    const PlumeGridInfo& info = b.lv[l].info;
    const Dims fd = dims_of(info), cd = dims_of(b.lv[l + 1].info);
    float* q = smem + b.offset[l];
    float* rhs = q + fd.n0 * fd.n1 * fd.n2;
    float* cq = smem + b.offset[l + 1];
    float* crhs = cq + cd.n0 * cd.n1 * cd.n2;
    const CellCoef* table = coef_of(l);
    block_smooth(info, q, rhs, b.sweeps, 1.0f, table);
    auto load = [&](int a, int bb, int c) { return q[at(fd, a, bb, c)]; };
    const bool uniform = is_uniform(info);
    const float ghost = ghost_coupling(info);
    const int coarse_cells = cd.n0 * cd.n1 * cd.n2;
    Walk w(t, BOTTOM_THREADS, cd.n1, cd.n2);
    for (int idx = t; idx < coarse_cells; idx += BOTTOM_THREADS, w.next()) {
      const int i = w.i, j = w.j, k = w.c;
      float total = 0.0f, count = 0.0f;
      for (int di = 0; di < 2; ++di)
        for (int dj = 0; dj < 2; ++dj)
          for (int dk = 0; dk < 2; ++dk) {
            const int fi = 2 * i + di, fj = 2 * j + dj, fk = 2 * k + dk;
            if (fi < fd.n0 && fj < fd.n1 && fk < fd.n2) {
              const int f = at(fd, fi, fj, fk);
              if (table) {
                total = total + table_residual(table, q, rhs, fd, fi, fj, fk);
              } else {
                total = total + residual_cell(uniform, info, ghost, fi, fj, fk, q[f], rhs[f], load);
              }
              count = count + 1.0f;
            }
          }
      crhs[idx] = total / count;
      cq[idx] = 0.0f;
    }
    __syncthreads();
  }
  {
    const PlumeGridInfo& info = b.lv[b.count - 1].info;
    const Dims d = dims_of(info);
    float* q = smem + b.offset[b.count - 1];
    const int longest = imax_(d.n0, imax_(d.n1, d.n2));
    const int n = d.n0 * d.n1 * d.n2;
    const int sweeps = imax_(COARSEST_SWEEPS, COARSEST_SWEEPS_PER_CELL * longest);
    if constexpr (COARSE_F64) {
      double* staged = reinterpret_cast<double*>(smem + b.f64_offset);
      coarsest_f64(info, q, q + n, sweeps, 1.5, staged, staged + n);
    } else {
      block_smooth(info, q, q + n, sweeps, 1.5f, coef_of(b.count - 1));
    }
  }
  for (int l = b.count - 2; l >= 0; --l) {
    const PlumeGridInfo& info = b.lv[l].info;
    const Dims fd = dims_of(info), cd = dims_of(b.lv[l + 1].info);
    float* q = smem + b.offset[l];
    const float* cq = smem + b.offset[l + 1];
    const int n = fd.n0 * fd.n1 * fd.n2;
    Walk w(t, BOTTOM_THREADS, fd.n1, fd.n2);
    for (int idx = t; idx < n; idx += BOTTOM_THREADS, w.next())
      q[idx] = q[idx] + sample_plain(cq, cd, prolong_point(w.i, w.j, w.c));
    __syncthreads();
    block_smooth(info, q, q + n, b.sweeps, 1.0f, coef_of(l));
  }
  for (int l = 0; l < b.count; ++l) {
    const Dims d = dims_of(b.lv[l].info);
    const int n = d.n0 * d.n1 * d.n2;
    const float* q = smem + b.offset[l];
    for (int idx = t; idx < n; idx += BOTTOM_THREADS) {
      b.lv[l].q[idx] = q[idx];
      if (l > 0) b.lv[l].rhs[idx] = q[n + idx];
    }
  }
}

// ---- host side --------------------------------------------------------------------------------------------

static long cells_of(const PlumeGridInfo& info) { return (long)info.dims[0] * info.dims[1] * info.dims[2]; }

static dim3 tile_grid(const PlumeGridInfo& info) {
  return dim3((info.dims[2] + TILE_K - 1) / TILE_K, (info.dims[1] + TILE_J - 1) / TILE_J,
              (info.dims[0] + TILE_I - 1) / TILE_I);
}

static bool pdl_enabled() {
  static const bool enabled = std::getenv("PLUME_B200_NO_PDL") == nullptr;
  return enabled;
}

// Launches a solve kernel, with programmatic dependent launch unless PLUME_B200_NO_PDL is set.
template <class... Params, class... Args>
static int launch_solve_kernel(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                               const char* what, Args... args) {
  cudaLaunchConfig_t config = {};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = smem;
  config.stream = st;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = pdl_enabled() ? 1 : 0;
  int status = runtime_status(what, cudaLaunchKernelEx(&config, kernel, static_cast<Params>(args)...));
  if (status != PLUME_OK) return status;
  return launch_status(what);
}

// A level's pressure lives in two arrays: sweeps alternate between them. `cur` holds the current values.
struct Pressure {
  float* cur;
  float* other;
  void flip() { std::swap(cur, other); }
};

static bool uniform_level(const PlumeGridInfo& info) {
  return info.fill_hi[0] == 1.0f && info.fill_hi[1] == 1.0f && info.fill_hi[2] == 1.0f;
}

template <bool PROLONG>
static void launch_tiled(const PlumeGridInfo& info, Pressure& q, const float* rhs, float relaxation,
                         const float* coarse_q, Dims cd, cudaStream_t st) {
  if (uniform_level(info))
    k_rb_sweep<PROLONG, true><<<tile_grid(info), SWEEP_THREADS, 0, st>>>(info, q.cur, q.other, rhs, relaxation, coarse_q, cd);
  else
    k_rb_sweep<PROLONG, false><<<tile_grid(info), SWEEP_THREADS, 0, st>>>(info, q.cur, q.other, rhs, relaxation, coarse_q, cd);
}

// Levels of at least this many cells (q and rhs over 64 MB) sweep two planes per thread (k_rb_colour_pair).
// PLUME_PAIR_MIN_CELLS overrides the threshold (for measurements).
static const long RB_PAIR_MIN_CELLS = [] {
  const char* v = getenv("PLUME_PAIR_MIN_CELLS");
  return v ? atol(v) : 1L << 23;
}();
// Smaller levels with rows of a multiple of four cells sweep four cells of a row per thread (k_rb_colour4);
// PLUME_COLOUR4=0 keeps one cell per thread.
static const bool g_colour4 = [] {
  const char* v = getenv("PLUME_COLOUR4");
  return !(v && v[0] == '0');
}();

static int colour_sweep(const PlumeGridInfo& info, float* q, const float* rhs, float relaxation, cudaStream_t st) {
  const Dims d = dims_of(info);
  if (cells_of(info) >= RB_PAIR_MIN_CELLS) {
    const dim3 grid(((d.n2 + 1) / 2 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, (d.n0 + 1) / 2);
    for (int color = 0; color < 2; ++color) {
      int status = uniform_level(info) ? launch_solve_kernel(k_rb_colour_pair<true>, grid, cell_block(), 0, st,
                                                             "red-black colour", info, q, rhs, color, relaxation)
                                       : launch_solve_kernel(k_rb_colour_pair<false>, grid, cell_block(), 0, st,
                                                             "red-black colour", info, q, rhs, color, relaxation);
      if (status != PLUME_OK) return status;
    }
    return PLUME_OK;
  }
  if (g_colour4 && d.n2 % 4 == 0 && (((uintptr_t)q | (uintptr_t)rhs) & 15) == 0) {
    const dim3 grid((d.n2 / 4 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, d.n0);
    for (int color = 0; color < 2; ++color) {
      int status = uniform_level(info) ? launch_solve_kernel(k_rb_colour4<true>, grid, cell_block(), 0, st,
                                                             "red-black colour", info, q, rhs, color, relaxation)
                                       : launch_solve_kernel(k_rb_colour4<false>, grid, cell_block(), 0, st,
                                                             "red-black colour", info, q, rhs, color, relaxation);
      if (status != PLUME_OK) return status;
    }
    return PLUME_OK;
  }
  const dim3 grid(((d.n2 + 1) / 2 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, d.n0);
  for (int color = 0; color < 2; ++color) {
    const float* none = nullptr;
    int status = uniform_level(info)
                     ? launch_solve_kernel(k_rb_colour<true>, grid, cell_block(), 0, st, "red-black colour", info, q, rhs,
                                           color, relaxation, none, Dims{1, 1, 1})
                     : launch_solve_kernel(k_rb_colour<false>, grid, cell_block(), 0, st, "red-black colour", info, q,
                                           rhs, color, relaxation, none, Dims{1, 1, 1});
    if (status != PLUME_OK) return status;
  }
  return PLUME_OK;
}

// The split top level's prolongation takes both colours of a row's four half indices per thread when the
// coarse rows hold a multiple of four cells (k_prolong_add_split8); PLUME_PROLONG8=0 keeps k_prolong_add_split4.
// Measured on B200 at 256x384x256, 4 V-cycles: the solve 3.094 -> 3.020 ms, every value unchanged.
static const bool g_prolong8 = [] {
  const char* v = getenv("PLUME_PROLONG8");
  return !(v && v[0] == '0');
}();

// The top level's split arrays: q then rhs, each 2 * nx * ny * H floats.
struct SplitTop {
  float* q;
  float* rhs;
  int H;
};

// Half-row length of the split arrays: (nz + 1) / 2 cells, padded to a multiple of four for 16-byte loads.
static int split_H(const PlumeGridInfo& info) { return ((info.dims[2] + 1) / 2 + 3) / 4 * 4; }

static long split_floats(const PlumeGridInfo& info) {
  return 2L * info.dims[0] * info.dims[1] * split_H(info);
}

static int split_sweeps(const PlumeGridInfo& info, const SplitTop& sp, int sweeps, const float* coarse_q,
                        const PlumeGridInfo* coarse, cudaStream_t st) {
  const Dims d = dims_of(info);
  if (coarse) {
    const Dims cd = dims_of(*coarse);
    const bool rows4 = g_prolong8 && cd.n2 % 4 == 0 && ((uintptr_t)coarse_q & 15) == 0;
    int status = rows4 ? launch_solve_kernel(k_prolong_add_split8, dim3((sp.H / 4 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, d.n0),
                                             cell_block(), 0, st, "prolong (split)", cd, d, sp.H, coarse_q, sp.q)
                       : launch_solve_kernel(k_prolong_add_split4, dim3((sp.H / 4 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, 2 * d.n0),
                                             cell_block(), 0, st, "prolong (split)", cd, d, sp.H, coarse_q, sp.q);
    if (status != PLUME_OK) return status;
  }
  const dim3 grid((sp.H / 4 + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, d.n0);
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      int status = launch_solve_kernel(k_rb_split4, grid, cell_block(), 0, st, "red-black colour (split)", info,
                                       sp.H, sp.q, (const float*)sp.rhs, color, 1.0f);
      if (status != PLUME_OK) return status;
    }
  return PLUME_OK;
}

// `sweeps` full sweeps; when `coarse` is given its correction is prolonged first (folded into the first tiled
// sweep on large levels).
static int sweeps_with_prolong(const PlumeGridInfo& info, Pressure& q, const float* rhs, int sweeps, float relaxation,
                               const float* coarse_q, const PlumeGridInfo* coarse, cudaStream_t st) {
  int s = 0;
  const bool tiled = cells_of(info) >= g_tiled_min_cells;
  if (coarse) {
    const Dims cd = dims_of(*coarse);
    if (sweeps == 0 || !tiled) {
      const Dims fd = dims_of(info);
      int status = launch_solve_kernel(k_prolong_add, cell_grid(fd.n0, fd.n1, fd.n2), cell_block(), 0, st, "prolong",
                                       cd, fd, coarse_q, q.cur);
      if (status != PLUME_OK) return status;
    } else {
      launch_tiled<true>(info, q, rhs, relaxation, coarse_q, cd, st);
      int status = launch_status("red-black sweep with prolongation");
      if (status != PLUME_OK) return status;
      q.flip();
      s = 1;
    }
  }
  for (; s < sweeps; ++s) {
    if (tiled) {
      launch_tiled<false>(info, q, rhs, relaxation, nullptr, Dims{1, 1, 1}, st);
      int status = launch_status("red-black sweep");
      if (status != PLUME_OK) return status;
      q.flip();
    } else {
      int status = colour_sweep(info, q.cur, rhs, relaxation, st);
      if (status != PLUME_OK) return status;
    }
  }
  return PLUME_OK;
}

// Sweeps on `q` with `scratch` as the second array; the result always ends in `q`.
int red_black_sweeps(const PlumeGridInfo& info, float* q, float* scratch, const float* rhs, int sweeps,
                     float relaxation, cudaStream_t st) {
  Pressure p{q, scratch};
  int status = sweeps_with_prolong(info, p, rhs, sweeps, relaxation, nullptr, nullptr, st);
  if (status != PLUME_OK || p.cur == q) return status;
  return runtime_status("pressure copy-back", cudaMemcpyAsync(q, p.cur, sizeof(float) * (size_t)cells_of(info),
                                                              cudaMemcpyDeviceToDevice, st));
}

// The first level from which the rest of the hierarchy runs in one cluster launch (count when none fits),
// and that launch's per-CTA shared memory.
// With coarse_f64 the one-block solve is used (it holds the double copy of the coarsest level after the
// float arrays, 8-byte aligned).
static int bottom_kind(int coarse_f64) { return coarse_f64 ? 0 : g_bottom_kind; }

static size_t f64_staging_offset(size_t float_bytes) { return (float_bytes + 7) / 8 * 8; }

static bool overhangs(const PlumeGridInfo& info) {
  return info.fill_hi[0] != 1.0f || info.fill_hi[1] != 1.0f || info.fill_hi[2] != 1.0f;
}

// The one-block solve's shared memory after its q and rhs arrays (`bytes`): a CellCoef table per level with
// overhanging cells, each from a 16-byte boundary. With `offsets`, the tables' float offsets (-1: none).
static size_t coef_bytes(const PlumeLevel* levels, int count, size_t bytes, int* offsets = nullptr) {
  for (int l = 0; l < count; ++l) {
    if (offsets) offsets[l] = -1;
    if (!overhangs(levels[l].info)) continue;
    bytes = (bytes + 15) / 16 * 16;
    if (offsets) offsets[l] = (int)(bytes / sizeof(float));
    bytes += sizeof(CellCoef) * (size_t)cells_of(levels[l].info);
  }
  return bytes;
}

static int bottom_start(const PlumeLevel* levels, int count, size_t* smem_bytes, int coarse_f64) {
  for (int first = 0; first < count; ++first) {
    if (count - first > BOTTOM_MAX_LEVELS || cells_of(levels[first].info) > g_bottom_max_cells) continue;
    size_t bytes = 0;
    for (int l = first; l < count; ++l) {
      const PlumeGridInfo& info = levels[l].info;
      const bool single = bottom_kind(coarse_f64) == 0 || cells_of(info) <= SINGLE_MAX_CELLS;
      const long planes = single ? info.dims[0] : (info.dims[0] + CLUSTER - 1) / CLUSTER;
      bytes += 2 * sizeof(float) * (size_t)planes * info.dims[1] * info.dims[2];
    }
    if (bottom_kind(coarse_f64) == 0) bytes = coef_bytes(levels + first, count - first, bytes);
    if (coarse_f64) bytes = f64_staging_offset(bytes) + 2 * sizeof(double) * (size_t)cells_of(levels[count - 1].info);
    if (bytes > BOTTOM_MAX_SMEM) continue;
    *smem_bytes = bytes;
    return first;
  }
  return count;
}

// Lets the coarse solves use up to BOTTOM_MAX_SMEM of shared memory (once per device, outside any capture).
static int prepare_bottom() {
  static std::mutex mutex;
  static bool configured[64] = {};
  int device = 0;
  int status = runtime_status("current device", cudaGetDevice(&device));
  if (status != PLUME_OK) return status;
  std::lock_guard<std::mutex> lock(mutex);
  if (device >= 0 && device < 64 && !configured[device]) {
    status = runtime_status("coarse solve shared memory",
                            cudaFuncSetAttribute(k_cluster_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)BOTTOM_MAX_SMEM));
    for (auto kernel : {k_block_solve<false, false>, k_block_solve<true, false>, k_block_solve<false, true>,
                        k_block_solve<true, true>})
      if (status == PLUME_OK)
        status = runtime_status("coarse solve shared memory",
                                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)BOTTOM_MAX_SMEM));
    if (status == PLUME_OK)
      status = runtime_status("coarse solve shared memory",
                              cudaFuncSetAttribute(k_coarsest_f64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)BOTTOM_MAX_SMEM));
    if (status != PLUME_OK) return status;
    configured[device] = true;
  }
  return PLUME_OK;
}

static int launch_bottom(const PlumeLevel* levels, int count, int sweeps, size_t smem, cudaStream_t st,
                         int coarse_f64) {
  int status = prepare_bottom();
  if (status != PLUME_OK) return status;
  if (bottom_kind(coarse_f64) == 0) {
    BlockArgs b{};
    b.count = count;
    b.sweeps = sweeps;
    int offset = 0;
    for (int l = 0; l < count; ++l) {
      b.lv[l] = levels[l];
      b.offset[l] = offset;
      offset += 2 * (int)cells_of(levels[l].info);
    }
    const size_t table_end = coef_bytes(levels, count, sizeof(float) * (size_t)offset, b.coef_offset);
    b.f64_offset = (int)(f64_staging_offset(table_end) / sizeof(float));
    bool tables = false;
    for (int l = 0; l < count; ++l) tables = tables || b.coef_offset[l] >= 0;
    auto kernel = coarse_f64 ? (tables ? k_block_solve<true, true> : k_block_solve<true, false>)
                             : (tables ? k_block_solve<false, true> : k_block_solve<false, false>);
    return launch_solve_kernel(kernel, dim3(1), dim3(BOTTOM_THREADS),
                               smem, st, "coarse-level block solve", b);
  }
  ClusterArgs b{};
  b.count = count;
  b.sweeps = sweeps;
  int offset = 0;
  for (int l = 0; l < count; ++l) {
    LevelView& L = b.lv[l];
    L.info = levels[l].info;
    L.q = levels[l].q;
    L.rhs = levels[l].rhs;
    L.single = cells_of(L.info) <= SINGLE_MAX_CELLS ? 1 : 0;
    L.planes = L.single ? L.info.dims[0] : (L.info.dims[0] + CLUSTER - 1) / CLUSTER;
    L.offset = offset;
    offset += 2 * L.planes * L.info.dims[1] * L.info.dims[2];
  }
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(CLUSTER, 1, 1);
  config.blockDim = dim3(BOTTOM_THREADS, 1, 1);
  config.dynamicSmemBytes = smem;
  config.stream = st;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeClusterDimension;
  attribute[0].val.clusterDim.x = CLUSTER;
  attribute[0].val.clusterDim.y = 1;
  attribute[0].val.clusterDim.z = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  status = runtime_status("coarse-level cluster solve", cudaLaunchKernelEx(&config, k_cluster_solve, b));
  if (status != PLUME_OK) return status;
  return launch_status("coarse-level cluster solve");
}

// One V-cycle below `index` (multigrid.py:130-147). Every level keeps its pressure in q and uses its residual
// array as the sweeps' second array; the residual itself is never stored (k_residual_restrict).
static int v_cycle(const PlumeLevel* levels, int count, int index, Pressure& q, int bottom, size_t smem, int sweeps,
                   cudaStream_t st, int coarse_f64, const SplitTop* split = nullptr) {
  const PlumeLevel& lv = levels[index];
  if (index == 0 && split) {  // the top level in split storage (never the bottom or the coarsest level)
    int status = split_sweeps(lv.info, *split, sweeps, nullptr, nullptr, st);
    if (status != PLUME_OK) return status;
    const PlumeLevel& coarse = levels[1];
    const Dims cd = dims_of(coarse.info);
    constexpr int V = PLUME_RESTRICT_CELLS;
    const dim3 grid(((cd.n2 + V - 1) / V + TZ - 1) / TZ, (cd.n1 + TY - 1) / TY, cd.n0);
    status = uniform_level(lv.info)
                 ? launch_solve_kernel(k_residual_restrict_split<V, true>, grid, cell_block(), 0, st,
                                       "residual and restriction (split)", lv.info, split->H, (const float*)split->q,
                                       (const float*)split->rhs, cd, coarse.rhs, coarse.q)
                 : launch_solve_kernel(k_residual_restrict_split<V, false>, grid, cell_block(), 0, st,
                                       "residual and restriction (split)", lv.info, split->H, (const float*)split->q,
                                       (const float*)split->rhs, cd, coarse.rhs, coarse.q);
    if (status != PLUME_OK) return status;
    Pressure coarse_q{coarse.q, coarse.residual};
    if ((status = v_cycle(levels, count, 1, coarse_q, bottom, smem, sweeps, st, coarse_f64)) != PLUME_OK) return status;
    if (coarse_q.cur != coarse.q) {
      status = runtime_status("coarse pressure copy",
                              cudaMemcpyAsync(coarse.q, coarse_q.cur, sizeof(float) * cd.n0 * cd.n1 * cd.n2,
                                              cudaMemcpyDeviceToDevice, st));
      if (status != PLUME_OK) return status;
    }
    return split_sweeps(lv.info, *split, sweeps, coarse.q, &coarse.info, st);
  }
  if (index == bottom) {
    PlumeLevel first[BOTTOM_MAX_LEVELS];
    for (int l = bottom; l < count && l - bottom < BOTTOM_MAX_LEVELS; ++l) first[l - bottom] = levels[l];
    first[0].q = q.cur;
    return launch_bottom(first, count - bottom, sweeps, smem, st, coarse_f64);
  }
  if (index == count - 1) {
    const int longest = std::max(lv.info.dims[0], std::max(lv.info.dims[1], lv.info.dims[2]));
    if (coarse_f64) {
      const size_t bytes = 2 * sizeof(double) * (size_t)cells_of(lv.info);
      if (bytes > BOTTOM_MAX_SMEM) return fail(PLUME_ERR_INVALID, "coarsest level too large for the double solve");
      int status = prepare_bottom();
      if (status != PLUME_OK) return status;
      return launch_solve_kernel(k_coarsest_f64, dim3(1), dim3(BOTTOM_THREADS), bytes, st, "coarsest double solve",
                                 lv.info, q.cur, lv.rhs, std::max(COARSEST_SWEEPS, COARSEST_SWEEPS_PER_CELL * longest));
    }
    return sweeps_with_prolong(lv.info, q, lv.rhs, std::max(COARSEST_SWEEPS, COARSEST_SWEEPS_PER_CELL * longest), 1.5f,
                               nullptr, nullptr, st);
  }
  int status = sweeps_with_prolong(lv.info, q, lv.rhs, sweeps, 1.0f, nullptr, nullptr, st);
  if (status != PLUME_OK) return status;
  const PlumeLevel& coarse = levels[index + 1];
  const Dims cd = dims_of(coarse.info);
  if ((status = launch_solve_kernel(k_residual_restrict, cell_grid(cd.n0, cd.n1, cd.n2), cell_block(), 0, st,
                                    "residual and restriction", lv.info, q.cur, lv.rhs, cd, coarse.rhs, coarse.q)) !=
      PLUME_OK)
    return status;
  Pressure coarse_q{coarse.q, coarse.residual};
  if ((status = v_cycle(levels, count, index + 1, coarse_q, bottom, smem, sweeps, st, coarse_f64)) != PLUME_OK)
    return status;
  if (coarse_q.cur != coarse.q) {  // an odd number of coarsest sweeps left the result in the second array
    status = runtime_status("coarse pressure copy", cudaMemcpyAsync(coarse.q, coarse_q.cur, sizeof(float) * cd.n0 * cd.n1 * cd.n2,
                                                                    cudaMemcpyDeviceToDevice, st));
    if (status != PLUME_OK) return status;
  }
  return sweeps_with_prolong(lv.info, q, lv.rhs, sweeps, 1.0f, coarse.q, &coarse.info, st);
}

// Whether the top level runs split: scratch given, at least two levels with level 0 above the bottom solve,
// uniform couplings, swept by colour (not tiled) and at least g_split_min_cells cells.
static bool use_split(const PlumeLevel* levels, int count, int bottom, const float* scratch) {
  const PlumeGridInfo& info = levels[0].info;
  return scratch && ((uintptr_t)scratch & 15) == 0 && count >= 2 && bottom > 0 && uniform_level(info) &&
         cells_of(info) >= g_split_min_cells && cells_of(info) < g_tiled_min_cells;
}

static int multigrid_direct(const PlumeLevel* levels, int count, int cycles, int sweeps, cudaStream_t st,
                            int coarse_f64, float* split_scratch = nullptr) {
  size_t smem = 0;
  const int bottom = bottom_start(levels, count, &smem, coarse_f64);
  if (use_split(levels, count, bottom, split_scratch)) {
    const PlumeGridInfo& info = levels[0].info;
    const Dims d = dims_of(info);
    SplitTop sp{split_scratch, split_scratch + split_floats(info), split_H(info)};
    const dim3 grid((sp.H + TZ - 1) / TZ, (d.n1 + TY - 1) / TY, d.n0);
    int status = launch_solve_kernel(k_split_layout<true>, grid, cell_block(), 0, st, "pressure to split storage", d,
                                     sp.H, (const float*)levels[0].q, sp.q);
    if (status != PLUME_OK) return status;
    if ((status = launch_solve_kernel(k_split_layout<true>, grid, cell_block(), 0, st, "divergence to split storage",
                                      d, sp.H, (const float*)levels[0].rhs, sp.rhs)) != PLUME_OK)
      return status;
    Pressure unused{levels[0].q, levels[0].residual};
    for (int c = 0; c < cycles; ++c)
      if ((status = v_cycle(levels, count, 0, unused, bottom, smem, sweeps, st, coarse_f64, &sp)) != PLUME_OK)
        return status;
    return launch_solve_kernel(k_split_layout<false>, grid, cell_block(), 0, st, "pressure from split storage", d,
                               sp.H, (const float*)sp.q, levels[0].q);
  }
  Pressure q{levels[0].q, levels[0].residual};
  for (int c = 0; c < cycles; ++c) {
    int status = v_cycle(levels, count, 0, q, bottom, smem, sweeps, st, coarse_f64);
    if (status != PLUME_OK) return status;
  }
  if (q.cur == levels[0].q) return PLUME_OK;
  return runtime_status("pressure copy-back", cudaMemcpyAsync(levels[0].q, q.cur, sizeof(float) * (size_t)cells_of(levels[0].info),
                                                              cudaMemcpyDeviceToDevice, st));
}

}  // namespace plume

namespace plume {

// ---- replaying the solve as a CUDA graph -----------------------------------------------------------------
// The launch sequence of a solve depends only on the levels (geometry and arrays), the cycle and sweep
// counts and the strategy, so it is captured once into a graph (on a private stream: capture records and
// runs nothing) and replayed on the caller's stream, which saves the per-launch cost of its ~30 launches per
// V-cycle, most of them short.
struct GraphKey {
  int device;
  int count, cycles, sweeps, kind, coarse_f64;
  long tiled, bottom, split_min;
  float* split;
  PlumeLevel levels[16];
  bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
};

struct GraphEntry {
  GraphKey key;
  uint64_t hash;
  cudaGraphExec_t exec;
  size_t kernels;  // kernel nodes in the graph
};

static uint64_t key_hash(const GraphKey& key) {  // FNV-1a over the key's bytes
  uint64_t h = 1469598103934665603ull;
  const unsigned char* bytes = reinterpret_cast<const unsigned char*>(&key);
  for (size_t i = 0; i < sizeof(GraphKey); ++i) h = (h ^ bytes[i]) * 1099511628211ull;
  return h;
}

static std::mutex g_graph_mutex;
static std::vector<GraphEntry> g_graphs;
static cudaStream_t g_capture_stream[64] = {};
static bool g_use_graphs = true;
constexpr size_t MAX_GRAPHS = 1024;  // one per live level hierarchy (batched runs hold many)

static int graph_for(const GraphKey& key, const PlumeLevel* levels, cudaGraphExec_t* out, size_t* kernels) {
  const uint64_t hash = key_hash(key);
  for (const GraphEntry& e : g_graphs)
    if (e.hash == hash && e.key == key) {
      *out = e.exec;
      *kernels = e.kernels;
      return PLUME_OK;
    }
  cudaStream_t& cap = g_capture_stream[key.device];
  int status = PLUME_OK;
  if (!cap) status = runtime_status("capture stream", cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  if (status != PLUME_OK) return status;
  // one-time function attributes are set outside the capture: run the smallest possible warm-up first
  status = runtime_status("begin capture", cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  if (status != PLUME_OK) return status;
  set_launch_counting(false);
  const int run = multigrid_direct(levels, key.count, key.cycles, key.sweeps, cap, key.coarse_f64, key.split);
  set_launch_counting(true);
  cudaGraph_t graph = nullptr;
  status = runtime_status("end capture", cudaStreamEndCapture(cap, &graph));
  if (run != PLUME_OK || status != PLUME_OK) {
    if (graph) cudaGraphDestroy(graph);
    return run != PLUME_OK ? run : status;
  }
  size_t nodes = 0, kernel_nodes = 0;
  if (cudaGraphGetNodes(graph, nullptr, &nodes) == cudaSuccess && nodes > 0) {
    std::vector<cudaGraphNode_t> list(nodes);
    if (cudaGraphGetNodes(graph, list.data(), &nodes) == cudaSuccess)
      for (cudaGraphNode_t node : list) {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(node, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernel_nodes;
      }
  }
  cudaGraphExec_t exec = nullptr;
  status = runtime_status("instantiate graph", cudaGraphInstantiate(&exec, graph, 0));
  cudaGraphDestroy(graph);
  if (status != PLUME_OK) return status;
  if (g_graphs.size() >= MAX_GRAPHS) {
    cudaGraphExecDestroy(g_graphs.front().exec);
    g_graphs.erase(g_graphs.begin());
  }
  g_graphs.push_back(GraphEntry{key, hash, exec, kernel_nodes});
  *out = exec;
  *kernels = kernel_nodes;
  return PLUME_OK;
}

int multigrid_cycles(const PlumeLevel* levels, int count, int cycles, int sweeps, cudaStream_t st, int coarse_f64,
                     float* split_scratch) {
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  int device = 0;
  if (!g_use_graphs || count > 16 || cudaStreamIsCapturing(st, &capturing) != cudaSuccess ||
      capturing != cudaStreamCaptureStatusNone || cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64)
    return multigrid_direct(levels, count, cycles, sweeps, st, coarse_f64, split_scratch);
  GraphKey key;
  std::memset(&key, 0, sizeof(key));
  key.device = device;
  key.count = count;
  key.cycles = cycles;
  key.sweeps = sweeps;
  key.kind = g_bottom_kind;
  key.coarse_f64 = coarse_f64;
  key.tiled = g_tiled_min_cells;
  key.bottom = g_bottom_max_cells;
  key.split_min = g_split_min_cells;
  key.split = split_scratch;
  std::memcpy(key.levels, levels, sizeof(PlumeLevel) * count);
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  {  // the coarse solve's shared-memory attribute must be set before its first capture
    size_t smem = 0;
    if (bottom_start(levels, count, &smem, coarse_f64) < count || coarse_f64) {
      int prepared = prepare_bottom();
      if (prepared != PLUME_OK) return prepared;
    }
  }
  cudaGraphExec_t exec = nullptr;
  size_t kernels = 0;
  int status = graph_for(key, levels, &exec, &kernels);
  if (status != PLUME_OK) return status;
  status = runtime_status("graph launch", cudaGraphLaunch(exec, st));
  if (status == PLUME_OK) count_launches(kernels);
  return status;
}

}  // namespace plume

extern "C" int plume_use_graphs(int32_t enable) {
  plume::g_use_graphs = enable != 0;
  return PLUME_OK;
}

extern "C" int plume_tune_solver(long long tiled_min_cells, long long bottom_max_cells, int32_t bottom_kind) {
  if (tiled_min_cells < 1 || bottom_max_cells < 0 || bottom_kind < 0 || bottom_kind > 1)
    return plume::fail(PLUME_ERR_INVALID, "tune_solver: thresholds must be positive, bottom_kind 0 or 1");
  plume::g_tiled_min_cells = (long)tiled_min_cells;
  plume::g_bottom_max_cells = (long)bottom_max_cells;
  plume::g_bottom_kind = bottom_kind;
  return PLUME_OK;
}

extern "C" int plume_tune_split(long long min_cells) {
  if (min_cells < 1) return plume::fail(PLUME_ERR_INVALID, "tune_split: min_cells must be positive");
  plume::g_split_min_cells = (long)min_cells;
  return PLUME_OK;
}

extern "C" long long plume_split_min_cells(void) { return plume::g_split_min_cells; }

extern "C" long long plume_split_scratch_floats(const PlumeGridInfo* info) {
  if (!info || info->dims[0] < 1 || info->dims[1] < 1 || info->dims[2] < 1)
    return plume::fail(PLUME_ERR_INVALID, "split_scratch_floats: bad dims");
  return 2 * plume::split_floats(*info);
}

extern "C" int plume_solver_tuning(long long* tiled_min_cells, long long* bottom_max_cells, int32_t* bottom_kind) {
  if (!tiled_min_cells || !bottom_max_cells || !bottom_kind)
    return plume::fail(PLUME_ERR_INVALID, "solver_tuning: null output");
  *tiled_min_cells = plume::g_tiled_min_cells;
  *bottom_max_cells = plume::g_bottom_max_cells;
  *bottom_kind = plume::g_bottom_kind;
  return PLUME_OK;
}
