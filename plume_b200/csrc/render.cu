// Volume-render kernels of libplume_b200.so for sm_100a: the light volume (shadow march), the normal field
// and the camera ray march of chadmv/plume (src/plume/render/*), with their C ABI.
#include <algorithm>

#include "common.cuh"

namespace plume {

__device__ __forceinline__ void slab_range(F3 origin, F3 dir, F3 bmin, F3 bmax, float& t0out, float& t1out) {
  float t_enter = -1.0e30f, t_exit = 1.0e30f;  // raymarch.py:55-69
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (fabsf(dir[a]) < 1.0e-12f) {
      if (origin[a] < bmin[a] || origin[a] > bmax[a]) {
        t0out = 1.0f;
        t1out = 0.0f;
        return;
      }
    } else {
      float t0 = (bmin[a] - origin[a]) / dir[a];
      float t1 = (bmax[a] - origin[a]) / dir[a];
      t_enter = fmax_(t_enter, fmin_(t0, t1));
      t_exit = fmin_(t_exit, fmax_(t0, t1));
    }
  }
  t0out = t_enter;
  t1out = t_exit;
}

// ---- empty-space skipping ------------------------------------------------------------------------------------
// A brick map holds, for each 4x4x4 brick of cells, the largest smoke value of the brick and of the next cell
// past it on each axis: every corner a trilinear sample with lower corner in the brick can blend. When that
// is <= 0, every corner is <= 0, their blend is <= 0 (each weighted term is), max(sample, 0) is +0 and the
// sample adds exactly nothing: skipping it changes no bit of the result.
constexpr int BRICK = 4;

__host__ __device__ __forceinline__ Dims brick_dims(const Dims& d) {
  return Dims{(d.n0 + BRICK - 1) / BRICK, (d.n1 + BRICK - 1) / BRICK, (d.n2 + BRICK - 1) / BRICK};
}

// How many samples after the one at index-space point g stay in g's brick, for a march that advances `delta`
// cells per sample on each axis (returned as a float, possibly negative or huge; the caller floors and caps it).
// A sample's brick is that of its clamped lower corner, so on each axis the first brick reaches to -inf and the
// last to +inf. Samples nearer than `margin` cells to a brick face are not counted: the margin bounds twice the
// float error of a computed sample point against the exact line through the march, so every counted sample,
// as computed, lies in the brick.
__device__ __forceinline__ float samples_in_brick(const Dims& d, F3 g, F3 delta, float margin) {
  const int n[3] = {d.n0, d.n1, d.n2};
  float count = 3.0e38f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (delta[a] == 0.0f) continue;
    const int b = (int)fminf(fmaxf(g[a], 0.0f), (float)(n[a] - 1)) / BRICK;
    float room;
    if (delta[a] > 0.0f) {
      if (b == (n[a] - 1) / BRICK) continue;
      room = (float)((b + 1) * BRICK) - g[a];
    } else {
      if (b == 0) continue;
      room = g[a] - (float)(b * BRICK);
    }
    count = fminf(count, (room - margin) / fabsf(delta[a]));
  }
  return count;
}

// samples_in_brick with the divisions by |delta| replaced by products with their reciprocals `per_cell`
// (computed once per march). The count may move by a few ulps, far inside the margin, so every sample it
// counts still lies in the brick.
__device__ __forceinline__ float samples_in_brick_by(const Dims& d, F3 g, F3 delta, F3 per_cell, float margin) {
  const int n[3] = {d.n0, d.n1, d.n2};
  float count = 3.0e38f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (delta[a] == 0.0f) continue;
    const int b = (int)fminf(fmaxf(g[a], 0.0f), (float)(n[a] - 1)) / BRICK;
    float room;
    if (delta[a] > 0.0f) {
      if (b == (n[a] - 1) / BRICK) continue;
      room = (float)((b + 1) * BRICK) - g[a];
    } else {
      if (b == 0) continue;
      room = g[a] - (float)(b * BRICK);
    }
    count = fminf(count, (room - margin) * per_cell[a]);
  }
  return count;
}

// Index of the sample a march continues from after the sample `s` in an empty brick: past every later sample
// that `samples_in_brick` places in the same brick, and at most `end`.
__device__ __forceinline__ int past_brick(int s, int end, float count) {
  return count >= 1.0f ? s + (int)fminf(count, (float)(end - s)) : s;
}

template <class T>
__global__ void k_brick_max(Dims d, const T* __restrict__ f, float* __restrict__ bricks) {
  const Dims b = brick_dims(d);
  const int bi = blockIdx.z, bj = blockIdx.y * blockDim.y + threadIdx.y, bk = blockIdx.x * blockDim.x + threadIdx.x;
  if (bj >= b.n1 || bk >= b.n2) return;
  float best = -3.0e38f;
  for (int i = bi * BRICK; i <= imin_(bi * BRICK + BRICK, d.n0 - 1); ++i)
    for (int j = bj * BRICK; j <= imin_(bj * BRICK + BRICK, d.n1 - 1); ++j)
      for (int k = bk * BRICK; k <= imin_(bk * BRICK + BRICK, d.n2 - 1); ++k) best = fmaxf(best, ldg_f(f + at(d, i, j, k)));
  bricks[at(b, bi, bj, bk)] = best;
}

// light_volume_kernel (light_volume.py:18-33): each lit cell marches toward the light in at most half-cell
// steps to the box edge and gets exp(-opacity * column * cell_m). With `bricks`, samples whose corners are all
// <= 0 add exactly 0: the march steps over the whole run of them that lies in one brick.
//
// With `march_cells`, only the cells a camera march of the same smoke can read get their value: a march sample
// reads the light at its eight corners only when its alpha is > 0, so when one of those corners holds smoke
// > 0; the corners of every sample that reads cell c lie in {c-1, c, c+1}^3. So c is read only if one of those
// 27 cells holds smoke > 0 (tested first through the bricks of the lower corners {c-1, c}^3, which hold the
// largest smoke of every such corner). Every other cell gets 1.
//
// Arithmetic: the trilinear blends are fma(t, b - a, a) and the column adds each sample with one fma, one
// rounding fewer than light_volume_kernel's lerp and multiply-add, so the light agrees with the reference's to
// about an ulp of the column (held to 1e-5 relative); the empty-space skipping and the march_cells form change
// no bit of it.
__device__ __forceinline__ float lerp_fma(float a, float b, float t) { return __fmaf_rn(t, b - a, a); }

template <class T>
__device__ __forceinline__ float sample_fma(const T* __restrict__ f, const Dims& d, const Axis1& x, const Axis1& y,
                                            const Axis1& z) {
  const T* p = f + (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  const float c00 = lerp_fma(ldg_f(p), ldg_f(p + x.step), x.t);
  const float c10 = lerp_fma(ldg_f(p + y.step), ldg_f(p + x.step + y.step), x.t);
  const float c01 = lerp_fma(ldg_f(p + z.step), ldg_f(p + x.step + z.step), x.t);
  const float c11 = lerp_fma(ldg_f(p + y.step + z.step), ldg_f(p + x.step + y.step + z.step), x.t);
  return lerp_fma(lerp_fma(c00, c10, y.t), lerp_fma(c01, c11, y.t), z.t);
}

// Whether a camera march of this smoke reads the light at cell (i, j, k) (the march_cells test above).
template <class T>
__device__ __forceinline__ bool read_by_march(const Dims& d, const T* __restrict__ smoke, const float* __restrict__ bricks,
                                              int i, int j, int k) {
  const Dims bd = brick_dims(d);
  bool read = false;
  for (int a = imax_(i - 1, 0); a <= i; ++a)
    for (int b = imax_(j - 1, 0); b <= j; ++b)
      for (int c = imax_(k - 1, 0); c <= k; ++c) read |= __ldg(bricks + at(bd, a / BRICK, b / BRICK, c / BRICK)) > 0.0f;
  if (!read) return false;
  read = false;
  for (int a = imax_(i - 1, 0); a <= imin_(i + 1, d.n0 - 1); ++a)
    for (int b = imax_(j - 1, 0); b <= imin_(j + 1, d.n1 - 1); ++b)
      for (int c = imax_(k - 1, 0); c <= imin_(k + 1, d.n2 - 1); ++c) read |= ldg_f(smoke + at(d, a, b, c)) > 0.0f;
  return read;
}

// The light of one cell: its march toward the light.
template <class T>
__device__ __forceinline__ float light_at(const Dims& d, const T* __restrict__ smoke, F3 toward, float cell_m,
                                          float opacity, const float* __restrict__ bricks, int i, int j, int k) {
  const Dims bd = brick_dims(d);
  const F3 half = f3(0.5f, 0.5f, 0.5f);
  F3 start = add3(f3((float)i, (float)j, (float)k), half);
  F3 box_max = f3((float)d.n0, (float)d.n1, (float)d.n2);
  float t0, length;
  slab_range(start, toward, f3(0.0f, 0.0f, 0.0f), box_max, t0, length);
  int steps = (int)ceilf(length / 0.5f);
  float column = 0.0f;
  if (steps > 0) {
    float step = length / (float)steps;
    // the computed points (i, j, k) + toward * ((s + 0.5) * step), from the cell's lower corner, are within
    // (2 * length + 2 * extent) * 2^-24 cells of the exact line
    const float extent = (float)(imax_(imax_(d.n0, d.n1), d.n2) + 1);
    const float margin = (4.0f * length + 4.0f * extent) * 5.9604645e-8f + 1.0e-3f;
    const F3 delta = mul3(toward, step);
    const F3 per_cell = f3(1.0f / fabsf(delta[0]), 1.0f / fabsf(delta[1]), 1.0f / fabsf(delta[2]));
    const F3 corner = f3((float)i, (float)j, (float)k);
    int occupied = -1;  // the last brick of the map found holding smoke: its samples need no look-up
    for (int s = 0; s < steps; ++s) {
      const float t = ((float)s + 0.5f) * step;
      const F3 g = f3(__fmaf_rn(toward[0], t, corner[0]), __fmaf_rn(toward[1], t, corner[1]),
                      __fmaf_rn(toward[2], t, corner[2]));
      // the sample's axes; a sample's brick is that of its clamped lower corner (x.i0, y.i0, z.i0)
      const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
      if (bricks) {
        const int brick = at(bd, x.i0 / BRICK, y.i0 / BRICK, z.i0 / BRICK);
        if (brick != occupied) {
          if (__ldg(bricks + brick) <= 0.0f) {
            s = past_brick(s, steps - 1, samples_in_brick_by(d, g, delta, per_cell, margin));
            continue;
          }
          occupied = brick;
        }
      }
      column = __fmaf_rn(fmax_(sample_fma(smoke, d, x, y, z), 0.0f), step, column);
    }
  }
  return exp_f(-opacity * column * cell_m);
}

// A block of 32 x 8 threads covers 32 cells along z of LIGHT_ROWS * 8 rows of one x-plane; each warp takes
// LIGHT_ROWS rows. The warp first gives every cell that no march reads its 1 and queues the others in shared
// memory in row order, then marches the queue 32 cells at a time, so its lanes stay busy where only part of a
// row is lit. Measured on B200 at 256x384x256 (14% of the cells lit): 5.83 ms at 4 rows, 5.85 at 2, 6.15 at 8,
// where more rows per warp leave fewer, longer blocks to balance over the SMs.
constexpr int LIGHT_ROWS = 4;

template <class T>
__global__ void __launch_bounds__(256, 5) k_light_volume(Dims d, const T* __restrict__ smoke, F3 toward, float cell_m,
                                                      float opacity, float* __restrict__ light,
                                                      const float* __restrict__ bricks, int march_cells) {
  __shared__ unsigned short queue[8][LIGHT_ROWS * 32];
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int i = blockIdx.z, k = blockIdx.x * 32 + lane, j0 = (blockIdx.y * 8 + warp) * LIGHT_ROWS;
  int count = 0;
#pragma unroll 1
  for (int r = 0; r < LIGHT_ROWS; ++r) {
    const int j = j0 + r;
    bool lit = j < d.n1 && k < d.n2;
    if (lit && march_cells && !read_by_march(d, smoke, bricks, i, j, k)) {
      light[at(d, i, j, k)] = 1.0f;
      lit = false;
    }
    const unsigned vote = __ballot_sync(0xffffffffu, lit);
    if (lit) queue[warp][count + __popc(vote & ((1u << lane) - 1u))] = (unsigned short)(r * 32 + lane);
    count += __popc(vote);
  }
  __syncwarp();
#pragma unroll 1
  for (int b = 0; b < count; b += 32) {
    if (b + lane < count) {
      const int e = queue[warp][b + lane], j = j0 + e / 32, kk = blockIdx.x * 32 + e % 32;
      light[at(d, i, j, kk)] = light_at(d, smoke, toward, cell_m, opacity, bricks, i, j, kk);
    }
  }
}

// blur_axis_kernel (normal_field.py:12-22); weights in constant memory.
constexpr int MAX_BLUR_TAPS = 129;
__constant__ float c_weights[MAX_BLUR_TAPS];

template <class T>
__global__ void k_blur_axis(Dims d, const T* __restrict__ src, float* __restrict__ dst, int radius, int axis) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.n1 || k >= d.n2) return;
  const int cell[3] = {i, j, k};
  const int n[3] = {d.n0, d.n1, d.n2};
  float total = 0.0f;
  for (int o = -radius; o <= radius; ++o) {
    int c[3] = {i, j, k};
    c[axis] = imin_(imax_(cell[axis] + o, 0), n[axis] - 1);
    total = total + c_weights[o + radius] * ldg_f(src + at(d, c[0], c[1], c[2]));
  }
  dst[at(d, i, j, k)] = total;
}

// gradient_kernel (normal_field.py:25-38): per-cell central differences, one-sided at the edges; AoS output.
__global__ void k_gradient(Dims d, const float* __restrict__ src, float* __restrict__ gradient) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.n1 || k >= d.n2) return;
  const int cell[3] = {i, j, k};
  const int n[3] = {d.n0, d.n1, d.n2};
  float r[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[a] = imax_(cell[a] - 1, 0);
    hi[a] = imin_(cell[a] + 1, n[a] - 1);
    float span = (float)(hi[a] - lo[a]);
    if (span > 0.0f) r[a] = (__ldg(src + at(d, hi[0], hi[1], hi[2])) - __ldg(src + at(d, lo[0], lo[1], lo[2]))) / span;
  }
  float* out = gradient + (size_t)at(d, i, j, k) * 3;
  out[0] = r[0];
  out[1] = r[1];
  out[2] = r[2];
}

__device__ __forceinline__ F3 sample_vec(const float* __restrict__ f, const Dims& d, F3 g) {
  float x = clampf_(g[0], 0.0f, (float)(d.n0 - 1));
  float y = clampf_(g[1], 0.0f, (float)(d.n1 - 1));
  float z = clampf_(g[2], 0.0f, (float)(d.n2 - 1));
  int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  int i1 = imin_(i0 + 1, d.n0 - 1), j1 = imin_(j0 + 1, d.n1 - 1), k1 = imin_(k0 + 1, d.n2 - 1);
  float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
  auto ld = [&](int i, int j, int k) {
    const float* q = f + (size_t)at(d, i, j, k) * 3;
    return f3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
  };
  F3 c00 = lerp3(ld(i0, j0, k0), ld(i1, j0, k0), tx);
  F3 c10 = lerp3(ld(i0, j1, k0), ld(i1, j1, k0), tx);
  F3 c01 = lerp3(ld(i0, j0, k1), ld(i1, j0, k1), tx);
  F3 c11 = lerp3(ld(i0, j1, k1), ld(i1, j1, k1), tx);
  return lerp3(lerp3(c00, c10, ty), lerp3(c01, c11, ty), tz);
}

// The camera march's brick map: over each brick and the next cell past it on each axis (every corner a sample
// with lower corner in the brick can blend), 0 when the smoke is <= 0 and the temperature cannot glow, 1 when
// the smoke is <= 0 but the temperature may glow, 2 otherwise. The temperature cannot glow when its largest
// value is below glow_start by more than the rounding of three lerps (16 ulps), or when it is one value
// <= glow_start: a blend of equal corners is exactly that value. A sample in a class-0 brick has alpha 0 and
// glow 0 (adds exactly nothing); one in a class-1 brick has alpha 0.
template <class T>
__global__ void k_march_bricks(Dims d, const T* __restrict__ smoke, const T* __restrict__ temperature,
                               float glow_start, float* __restrict__ bricks) {
  const Dims b = brick_dims(d);
  const int bi = blockIdx.z, bj = blockIdx.y * blockDim.y + threadIdx.y, bk = blockIdx.x * blockDim.x + threadIdx.x;
  if (bj >= b.n1 || bk >= b.n2) return;
  float most = -3.0e38f, hot = -3.0e38f, cold = 3.0e38f;
  for (int i = bi * BRICK; i <= imin_(bi * BRICK + BRICK, d.n0 - 1); ++i)
    for (int j = bj * BRICK; j <= imin_(bj * BRICK + BRICK, d.n1 - 1); ++j)
      for (int k = bk * BRICK; k <= imin_(bk * BRICK + BRICK, d.n2 - 1); ++k) {
        const size_t c = at(d, i, j, k);
        most = fmaxf(most, ldg_f(smoke + c));
        const float t = ldg_f(temperature + c);
        hot = fmaxf(hot, t);
        cold = fminf(cold, t);
      }
  const bool dark = (hot + fabsf(hot) * 9.5367432e-7f < glow_start) || (cold == hot && hot <= glow_start);
  bricks[at(b, bi, bj, bk)] = most > 0.0f ? 2.0f : (dark ? 0.0f : 1.0f);
}

struct MarchArgs {
  PlumeGridInfo info;
  PlumeViewParams view;
  PlumeLookParams look;
  Dims d, dg, dl;
};

// raymarch_kernel (raymarch.py:86-140): one thread per pixel, 256 consecutive pixels of the image per block.
// Terms that are exactly zero are not evaluated: with no smoke at a sample (all eight corners <= 0 in the
// brick map, or a blend <= 0) alpha is exactly 0, so the exp, the light or gradient sample and the
// transmittance update are skipped (they would add +0 or multiply by 1); with no glow the pow is skipped (it
// would add +0); a run of samples in a brick with neither smoke nor glow is stepped over whole. Every result
// bit is unchanged.
template <class T>
__global__ void __launch_bounds__(256, 4) k_raymarch(MarchArgs a, const T* __restrict__ smoke, const T* __restrict__ temperature,
                           const float* __restrict__ gradient, const float* __restrict__ light, float* __restrict__ image,
                           int height, int width, const float* __restrict__ bricks) {
  const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
  if (pixel >= height * width) return;
  const int px = pixel % width, py = pixel / width;
  const PlumeViewParams& view = a.view;
  const PlumeLookParams& look = a.look;
  const PlumeGridInfo& info = a.info;
  F3 right = f3(view.right[0], view.right[1], view.right[2]);
  F3 up = f3(view.up[0], view.up[1], view.up[2]);
  F3 toward = f3(view.toward[0], view.toward[1], view.toward[2]);
  float plane_x = view.left_m + ((float)px + 0.5f) * view.pixel_m;  // pixel_ray (raymarch.py:72-83)
  float plane_y = view.top_m - ((float)py + 0.5f) * view.pixel_m;
  F3 origin = add3(add3(mul3(right, plane_x), mul3(up, plane_y)), mul3(toward, 1.0e4f));
  F3 direction = f3(-toward[0], -toward[1], -toward[2]);
  if (view.perspective == 1) {
    origin = f3(view.eye[0], view.eye[1], view.eye[2]);
    direction = normalize3(sub3(add3(mul3(right, plane_x), mul3(up, plane_y)), toward));
  }
  F3 box_origin = f3(info.origin_m[0], info.origin_m[1], info.origin_m[2]);
  F3 box_max = add3(box_origin, mul3(f3((float)info.dims[0], (float)info.dims[1], (float)info.dims[2]), info.cell_m));
  float s0, s1;
  slab_range(origin, direction, box_origin, box_max, s0, s1);
  if (view.perspective == 1) s0 = fmax_(s0, 0.0f);
  float tr = 1.0f, heat = 0.0f, shade_sum = 0.0f;
  F3 normal_sum = f3(0.0f, 0.0f, 0.0f);
  if (s1 > s0) {
    float length = s1 - s0;
    int steps = (int)ceilf(length / (0.5f * info.cell_m));
    float step_m = length / (float)steps;
    const Dims bd = brick_dims(a.d);
    // The computed points origin + direction * (s0 + (s + 0.5) * step_m) lie within
    // (3 |t| + 2 |box coordinate| + |box origin|) * 2^-24 / cell_m + 2 |g| * 2^-24 cells of the exact line; the
    // margin is over twice that.
    float box_far = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) box_far = fmaxf(box_far, fmaxf(fabsf(box_origin[c]), fabsf(box_max[c])));
    const float cells_far = (float)imax_(imax_(a.d.n0, a.d.n1), a.d.n2);
    const float margin = (8.0f * fmaxf(fabsf(s0), fabsf(s1)) + 6.0f * box_far) * 5.9604645e-8f / info.cell_m +
                         cells_far * 9.5367432e-7f + 1.0e-3f;
    const F3 delta = mul3(direction, step_m / info.cell_m);
    const Divisor cell = divisor(info.cell_m);  // (position - origin) / cell_m: a product when cell_m is 2^-e
    for (int s = 0; s < steps; ++s) {
      F3 position = add3(origin, mul3(direction, s0 + ((float)s + 0.5f) * step_m));
      F3 g = sub3(divide3(sub3(position, box_origin), cell), f3(0.5f, 0.5f, 0.5f));
      bool empty = false;
      if (bricks) {
        const int i0 = (int)fminf(fmaxf(g[0], 0.0f), (float)(a.d.n0 - 1));
        const int j0 = (int)fminf(fmaxf(g[1], 0.0f), (float)(a.d.n1 - 1));
        const int k0 = (int)fminf(fmaxf(g[2], 0.0f), (float)(a.d.n2 - 1));
        const float kind = __ldg(bricks + at(bd, i0 / BRICK, j0 / BRICK, k0 / BRICK));
        if (kind == 0.0f) {
          s = past_brick(s, steps - 1, samples_in_brick(a.d, g, delta, margin));
          continue;
        }
        empty = kind == 1.0f;
      }
      const float density = empty ? 0.0f : fmax_(sample_index_space(smoke, a.d, g), 0.0f);
      const float alpha = density > 0.0f ? 1.0f - exp_f(-look.opacity_per_density * density * step_m) : 0.0f;
      const float glow = fmax_(sample_index_space(temperature, a.d, g) - look.glow_start_k, 0.0f);
      if (glow > 0.0f) heat = heat + glow * step_m * pow_f(tr, look.smoke_hides_heat);
      if (alpha > 0.0f) {
        if (look.shade_layout == 1) {
          float lit = look.shade_fill + (1.0f - look.shade_fill) * sample_index_space(light, a.dl, g);
          shade_sum = shade_sum + tr * alpha * lit;
        } else {
          F3 slope = sample_vec(gradient, a.dg, g);
          if (len3(slope) > 1.0e-9f) normal_sum = sub3(normal_sum, mul3(normalize3(slope), tr * alpha));
        }
        tr = tr * (1.0f - alpha);
      }
    }
  }
  float thickness = 1.0f - tr;
  float* out = image + ((size_t)py * width + px) * 5;
  out[0] = heat;
  out[1] = thickness;
  if (look.shade_layout == 1) {
    out[2] = shade_sum;
    out[3] = 0.0f;
    out[4] = 0.0f;
    return;
  }
  F3 facing = f3(0.0f, 0.0f, 1.0f);
  F3 normal = facing;
  F3 cam = f3(dot3(normal_sum, right), dot3(normal_sum, up), dot3(normal_sum, toward));
  if (len3(cam) > 1.0e-9f) {
    normal = normalize3(cam);
    normal = f3(normal[0], normal[1], fabsf(normal[2]));
    float weight = clampf_(thickness / look.normal_fade_thickness, 0.0f, 1.0f);
    normal = normalize3(lerp3(facing, normal, weight));
  }
  out[2] = normal[0];
  out[3] = normal[1];
  out[4] = normal[2];
}

static bool valid_shape(const int32_t* s) {
  return s && s[0] >= 1 && s[1] >= 1 && s[2] >= 1 && (long long)s[0] * s[1] * s[2] * 3 < (1LL << 31);
}

}  // namespace plume

using namespace plume;

extern "C" long long plume_brick_floats(const int32_t shape[3]) {
  if (!valid_shape(shape)) return fail(PLUME_ERR_INVALID, "brick_floats: bad shape");
  const Dims b = brick_dims(Dims{shape[0], shape[1], shape[2]});
  return (long long)b.n0 * b.n1 * b.n2;
}

namespace plume {

template <class T>
static int light_volume(const Dims& d, const T* smoke, F3 toward, float cell_m, float opacity, float* light,
                        float* bricks, int march_cells, cudaStream_t st) {
  if (bricks) {
    const Dims b = brick_dims(d);
    k_brick_max<T><<<cell_grid(b.n0, b.n1, b.n2), cell_block(), 0, st>>>(d, smoke, bricks);
    int status = launch_status("smoke brick map");
    if (status != PLUME_OK) return status;
  }
  const dim3 grid((d.n2 + 31) / 32, (d.n1 + 8 * LIGHT_ROWS - 1) / (8 * LIGHT_ROWS), d.n0);
  k_light_volume<T><<<grid, dim3(32, 8), 0, st>>>(d, smoke, toward, cell_m, opacity, light, bricks, march_cells);
  return launch_status("light volume");
}

template <class T>
static int normal_field(const Dims& d, const T* smoke, float* blurred, float* scratch, float* gradient, int radius,
                        cudaStream_t st) {
  k_blur_axis<T><<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(d, smoke, blurred, radius, 0);
  int status = launch_status("blur");
  if (status != PLUME_OK) return status;
  k_blur_axis<float><<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(d, blurred, scratch, radius, 1);
  if ((status = launch_status("blur")) != PLUME_OK) return status;
  k_blur_axis<float><<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(d, scratch, blurred, radius, 2);
  if ((status = launch_status("blur")) != PLUME_OK) return status;
  k_gradient<<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(d, blurred, gradient);
  return launch_status("gradient");
}

template <class T>
static int brick_max(const Dims& d, const T* field, float* bricks, cudaStream_t st) {
  const Dims b = brick_dims(d);
  k_brick_max<T><<<cell_grid(b.n0, b.n1, b.n2), cell_block(), 0, st>>>(d, field, bricks);
  return launch_status("brick map");
}

template <class T>
static int raymarch(const MarchArgs& a, const T* smoke, const T* temperature, const float* gradient, const float* light,
                    float* image, int height, int width, float* bricks, cudaStream_t st) {
  if (bricks) {  // the brick map of exactly the smoke and temperature being marched
    const Dims b = brick_dims(a.d);
    k_march_bricks<T><<<cell_grid(b.n0, b.n1, b.n2), cell_block(), 0, st>>>(a.d, smoke, temperature,
                                                                             a.look.glow_start_k, bricks);
    int status = launch_status("march brick map");
    if (status != PLUME_OK) return status;
  }
  const long pixels = (long)height * width;
  k_raymarch<T><<<(int)((pixels + 255) / 256), 256, 0, st>>>(a, smoke, temperature, gradient, light, image, height,
                                                              width, bricks);
  return launch_status("raymarch");
}

// Returns the call for the storage code (its arrays of float, bfloat16 or half).
#define PLUME_BY_STORAGE(storage, call_f32, call_bf16, call_f16, what) \
  switch (storage) {                                                 \
    case PLUME_STORAGE_F32: return call_f32;                           \
    case PLUME_STORAGE_BF16: return call_bf16;                         \
    case PLUME_STORAGE_F16: return call_f16;                           \
  }                                                                    \
  return fail(PLUME_ERR_INVALID, "%s: storage %d", what, storage);

}  // namespace plume

static int light_volume_call(const int32_t shape[3], const void* smoke, int32_t storage, const float toward_light[3],
                             float cell_m, float opacity_per_density, float* light, float* bricks, int march_cells,
                             void* stream) {
  const Dims d{shape[0], shape[1], shape[2]};
  const F3 toward = f3(toward_light[0], toward_light[1], toward_light[2]);
  cudaStream_t st = as_stream(stream);
  PLUME_BY_STORAGE(storage,
                   light_volume(d, static_cast<const float*>(smoke), toward, cell_m, opacity_per_density, light, bricks,
                                march_cells, st),
                   light_volume(d, static_cast<const __nv_bfloat16*>(smoke), toward, cell_m, opacity_per_density, light,
                                bricks, march_cells, st),
                   light_volume(d, static_cast<const __half*>(smoke), toward, cell_m, opacity_per_density, light, bricks,
                                march_cells, st),
                   "light_volume")
}

extern "C" int plume_light_volume(const int32_t shape[3], const void* smoke, int32_t storage, const float toward_light[3],
                                  float cell_m, float opacity_per_density, float* light, float* bricks, void* stream) {
  if (!valid_shape(shape) || !smoke || !toward_light || !light) return fail(PLUME_ERR_INVALID, "light_volume: bad argument");
  return light_volume_call(shape, smoke, storage, toward_light, cell_m, opacity_per_density, light, bricks, 0, stream);
}

extern "C" int plume_march_light_volume(const int32_t shape[3], const void* smoke, int32_t storage,
                                        const float toward_light[3], float cell_m, float opacity_per_density,
                                        float* light, float* bricks, void* stream) {
  if (!valid_shape(shape) || !smoke || !toward_light || !light || !bricks)
    return fail(PLUME_ERR_INVALID, "march_light_volume: bad argument");
  return light_volume_call(shape, smoke, storage, toward_light, cell_m, opacity_per_density, light, bricks, 1, stream);
}

extern "C" int plume_normal_field(const int32_t shape[3], const void* smoke, int32_t storage, float* blurred,
                                  float* scratch, float* gradient, const float* weights_host, int32_t radius,
                                  void* stream) {
  if (!valid_shape(shape) || !smoke || !blurred || !scratch || !gradient || !weights_host || radius < 0 ||
      2 * radius + 1 > MAX_BLUR_TAPS)
    return fail(PLUME_ERR_INVALID, "normal_field: bad argument");
  cudaStream_t st = as_stream(stream);
  int weights = runtime_status("blur weights", cudaMemcpyToSymbolAsync(c_weights, weights_host, sizeof(float) * (2 * radius + 1),
                                                                      0, cudaMemcpyHostToDevice, st));
  if (weights != PLUME_OK) return weights;
  const Dims d{shape[0], shape[1], shape[2]};
  PLUME_BY_STORAGE(storage, normal_field(d, static_cast<const float*>(smoke), blurred, scratch, gradient, radius, st),
                   normal_field(d, static_cast<const __nv_bfloat16*>(smoke), blurred, scratch, gradient, radius, st),
                   normal_field(d, static_cast<const __half*>(smoke), blurred, scratch, gradient, radius, st),
                   "normal_field")
}

extern "C" int plume_brick_max(const int32_t shape[3], const void* field, int32_t storage, float* bricks, void* stream) {
  if (!valid_shape(shape) || !field || !bricks) return fail(PLUME_ERR_INVALID, "brick_max: bad argument");
  const Dims d{shape[0], shape[1], shape[2]};
  cudaStream_t st = as_stream(stream);
  PLUME_BY_STORAGE(storage, brick_max(d, static_cast<const float*>(field), bricks, st),
                   brick_max(d, static_cast<const __nv_bfloat16*>(field), bricks, st),
                   brick_max(d, static_cast<const __half*>(field), bricks, st), "brick_max")
}

extern "C" int plume_raymarch(const PlumeGridInfo* info, const void* smoke, const void* temperature, int32_t storage,
                              const float* gradient, const int32_t gradient_shape[3], const float* light,
                              const int32_t light_shape[3], const PlumeViewParams* view, const PlumeLookParams* look,
                              float* image, int32_t height, int32_t width, float* bricks, void* stream) {
  if (!info || !smoke || !temperature || !gradient || !light || !view || !look || !image || height < 1 || width < 1 ||
      (long long)height * width >= (1LL << 31) || !valid_shape(info->dims) || !valid_shape(gradient_shape) || !valid_shape(light_shape))
    return fail(PLUME_ERR_INVALID, "raymarch: bad argument");
  MarchArgs a;
  a.info = *info;
  a.view = *view;
  a.look = *look;
  a.d = Dims{info->dims[0], info->dims[1], info->dims[2]};
  a.dg = Dims{gradient_shape[0], gradient_shape[1], gradient_shape[2]};
  a.dl = Dims{light_shape[0], light_shape[1], light_shape[2]};
  cudaStream_t st = as_stream(stream);
  PLUME_BY_STORAGE(storage,
                   raymarch(a, static_cast<const float*>(smoke), static_cast<const float*>(temperature), gradient, light,
                            image, height, width, bricks, st),
                   raymarch(a, static_cast<const __nv_bfloat16*>(smoke), static_cast<const __nv_bfloat16*>(temperature),
                            gradient, light, image, height, width, bricks, st),
                   raymarch(a, static_cast<const __half*>(smoke), static_cast<const __half*>(temperature), gradient,
                            light, image, height, width, bricks, st),
                   "raymarch")
}
