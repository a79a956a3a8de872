// The adjoint (reverse-mode derivative) of the smoke path of the fluid step and of the thickness render, for
// fitting a smoke source field to a target thickness image. The smoke path is: a source field added to the
// smoke, MacCormack advection of the smoke by a given velocity (advect.py:59-68), the smoke budget's rescale
// (conserve.py:45-52) and dissipation (dissipate.py:10-15); the render is the ray march's thickness channel
// (raymarch.py:86-140). With the velocity independent of the smoke (no smoke weight in the buoyancy), these
// are exactly the operators a smoke source field acts through, so the derivative is the loss's gradient.
//
// Each adjoint kernel recomputes its forward pass's traces and branches and then transposes it:
//   - a trilinear sample becomes a scatter of the incoming derivative to its eight corners with the same
//     weights (atomic adds: several samples share a corner);
//   - MacCormack's clamp passes the derivative to the clamped value's corner (the first of equal corners in the
//     reference's min/max order) when it clamps, else through the correction hat + (data - back) / 2;
//   - the smoke budget's factor is a function of three totals, which adds uniform terms to the data, hat and
//     next derivatives;
//   - the march's thickness 1 - prod(exp(-k rho_s ds)) has d thickness / d rho_s = k ds * transmittance for every
//     sample with rho_s > 0.
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace plume {

constexpr int ADJ_THREADS = 256;
static int adj_blocks(long n) { return (int)((n + ADJ_THREADS - 1) / ADJ_THREADS); }

// The eight corners and weights of sample_index_space at g (sim/sample.py:10-29), in the reference's corner
// order (x fastest within (y, z) pairs as the lerps pair them).
struct Corners {
  int idx[8];
  float w[8];
};

__device__ __forceinline__ Corners corners_of(const Dims& d, F3 g) {
  const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
  const int base = (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  Corners c;
  // c00 = lerp(a000, a100, tx), c10 = lerp(a010, a110), c01 = lerp(a001, a101), c11 = lerp(a011, a111);
  // result = lerp(lerp(c00, c10, ty), lerp(c01, c11, ty), tz)
  const float wx[2] = {x.one_minus_t, x.t}, wy[2] = {y.one_minus_t, y.t}, wz[2] = {z.one_minus_t, z.t};
  const int sx[2] = {0, x.step}, sy[2] = {0, y.step}, sz[2] = {0, z.step};
  int n = 0;
  for (int kz = 0; kz < 2; ++kz)
    for (int ky = 0; ky < 2; ++ky)
      for (int kx = 0; kx < 2; ++kx) {
        c.idx[n] = base + sx[kx] + sy[ky] + sz[kz];
        c.w[n] = (wx[kx] * wy[ky]) * wz[kz];
        ++n;
      }
  return c;
}

__device__ __forceinline__ void scatter(float* __restrict__ target, const Corners& c, float value) {
  if (value == 0.0f) return;
#pragma unroll
  for (int n = 0; n < 8; ++n)
    if (c.w[n] != 0.0f) atomicAdd(target + c.idx[n], c.w[n] * value);
}

// The clamp range of the forward sample and the corner each bound came from (sample.py:32-50: the min and max
// run over a000, a001, a010, a011, a100, a101, a110, a111; a tie keeps the earlier corner).
__device__ __forceinline__ void range_corners(const float* __restrict__ f, const Dims& d, F3 g, int& lo_idx,
                                              int& hi_idx, float& lo, float& hi) {
  const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
  const int base = (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  const int order[8] = {base,
                        base + z.step,
                        base + y.step,
                        base + y.step + z.step,
                        base + x.step,
                        base + x.step + z.step,
                        base + x.step + y.step,
                        base + x.step + y.step + z.step};
  lo = hi = __ldg(f + order[0]);
  lo_idx = hi_idx = order[0];
#pragma unroll
  for (int n = 1; n < 8; ++n) {
    const float v = __ldg(f + order[n]);
    if (v < lo) {
      lo = v;
      lo_idx = order[n];
    }
    if (v > hi) {
      hi = v;
      hi_idx = order[n];
    }
  }
}

// smoke[corner + (i, j, k)] += scale * source[i, j, k] inside the grid.
__global__ void k_add_source(float* __restrict__ smoke, Dims d, const float* __restrict__ source, Dims s, int3 corner,
                             float scale) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)s.n0 * s.n1 * s.n2) return;
  const int k = (int)(idx % s.n2), j = (int)((idx / s.n2) % s.n1), i = (int)(idx / ((long)s.n1 * s.n2));
  const int gi = corner.x + i, gj = corner.y + j, gk = corner.z + k;
  if (gi < 0 || gj < 0 || gk < 0 || gi >= d.n0 || gj >= d.n1 || gk >= d.n2) return;
  const int c = at(d, gi, gj, gk);
  smoke[c] = smoke[c] + scale * source[idx];
}

// grad[i, j, k] += scale * a_smoke[corner + (i, j, k)] (the adjoint of k_add_source for its source).
__global__ void k_source_grad(const float* __restrict__ a_smoke, Dims d, float* __restrict__ grad, Dims s,
                              int3 corner, float scale) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)s.n0 * s.n1 * s.n2) return;
  const int k = (int)(idx % s.n2), j = (int)((idx / s.n2) % s.n1), i = (int)(idx / ((long)s.n1 * s.n2));
  const int gi = corner.x + i, gj = corner.y + j, gk = corner.z + k;
  if (gi < 0 || gj < 0 || gk < 0 || gi >= d.n0 || gj >= d.n1 || gk >= d.n2) return;
  grad[idx] = grad[idx] + scale * a_smoke[at(d, gi, gj, gk)];
}

// MacCormack adjoint, part 1 (per cell of the advected cell-centred field): the clamp's branch, the correction's
// own terms, and the backward sample's transpose into a_hat. a_data and a_hat must start as the derivatives
// already known for them (atomically accumulated).
__global__ void k_mac_adjoint_correct(PlumeGridInfo info, Vel vel, const float* __restrict__ data,
                                      const float* __restrict__ hat, const float* __restrict__ a_next,
                                      float* __restrict__ a_data, float* __restrict__ a_hat, float dt_over_cell,
                                      float outside) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = dims_of(info);
  if (j >= d.n1 || k >= d.n2) return;
  const int c = at(d, i, j, k);
  const float g_next = a_next[c];
  if (g_next == 0.0f) return;
  const F3 offset = f3(0.5f, 0.5f, 0.5f);
  const F3 p = add3(f3((float)i, (float)j, (float)k), offset);
  const F3 vp = velocity_at_node(vel, p);
  const F3 src = trace_from(vel, p, vp, dt_over_cell);
  const F3 back_src = trace_from(vel, p, vp, -dt_over_cell);
  const bool src_outside = is_outside_open_face(src, info);
  const bool back_outside = is_outside_open_face(back_src, info);
  const F3 gb = sub3(back_src, offset);
  const float back = back_outside ? outside : sample_index_space(hat, d, gb);
  const float corrected = __ldg(hat + c) + 0.5f * (__ldg(data + c) - back);
  float lo = outside, hi = outside;
  int lo_idx = -1, hi_idx = -1;
  if (!src_outside) range_corners(data, d, sub3(src, offset), lo_idx, hi_idx, lo, hi);
  if (corrected < lo) {  // clampf_: x < lo ? lo : (x > hi ? hi : x)
    if (lo_idx >= 0) atomicAdd(a_data + lo_idx, g_next);
    return;
  }
  if (corrected > hi) {
    if (hi_idx >= 0) atomicAdd(a_data + hi_idx, g_next);
    return;
  }
  atomicAdd(a_hat + c, g_next);
  atomicAdd(a_data + c, 0.5f * g_next);
  if (!back_outside) scatter(a_hat, corners_of(d, gb), -0.5f * g_next);
}

// MacCormack adjoint, part 2: the forward sample's transpose, a_data += sample^T(a_hat).
__global__ void k_mac_adjoint_forward(PlumeGridInfo info, Vel vel, const float* __restrict__ a_hat,
                                      float* __restrict__ a_data, float dt_over_cell) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = dims_of(info);
  if (j >= d.n1 || k >= d.n2) return;
  const float g = a_hat[at(d, i, j, k)];
  if (g == 0.0f) return;
  const F3 offset = f3(0.5f, 0.5f, 0.5f);
  const F3 p = add3(f3((float)i, (float)j, (float)k), offset);
  const F3 src = trace_from(vel, p, velocity_at_node(vel, p), dt_over_cell);
  if (is_outside_open_face(src, info)) return;
  scatter(a_data, corners_of(d, sub3(src, offset)), g);
}

// sum_i a[i] * b[i] in double, per block of ADJ_THREADS, then the blocks in order on one thread.
__global__ void k_dot_partials(const float* __restrict__ a, const float* __restrict__ b, long n, double* __restrict__ partial) {
  __shared__ double slot[ADJ_THREADS];
  double value = 0.0;
  for (long i = (long)blockIdx.x * ADJ_THREADS + threadIdx.x; i < n; i += (long)gridDim.x * ADJ_THREADS)
    value = value + (double)a[i] * (double)b[i];
  slot[threadIdx.x] = value;
  __syncthreads();
  for (int h = ADJ_THREADS / 2; h >= 1; h >>= 1) {
    if ((int)threadIdx.x < h) slot[threadIdx.x] = slot[threadIdx.x] + slot[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = slot[0];
}

// The smoke budget's adjoint coefficients from its three totals (before, semi-Lagrangian, MacCormack) and
// G = sum a_out * next (next before scaling): factor = held / mc with held = max(sl, min(mc, before)); the
// derivatives of the scaled output add uniform terms c_data to a_data, c_hat to a_hat and c_next to a_next.
// coeffs = {factor, c_data, c_hat, c_next}.
__global__ void k_budget_adjoint_coeffs(const double* __restrict__ totals, const double* __restrict__ partial, int blocks,
                                        double* __restrict__ coeffs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double g = 0.0;
  for (int b = 0; b < blocks; ++b) g = g + partial[b];
  const double before = totals[0], sl = totals[1], mc = totals[2];
  double factor = 1.0, c_data = 0.0, c_hat = 0.0, c_next = 0.0;
  if (mc > 0.0) {
    const double inner = mc < before ? mc : before;
    const double held = sl > inner ? sl : inner;
    factor = (double)(float)(held / mc);
    if (sl > inner) {  // held = sl
      c_hat = g / mc;
      c_next = -g * sl / (mc * mc);
    } else if (!(mc < before)) {  // held = before
      c_data = g / mc;
      c_next = -g * before / (mc * mc);
    }  // held = mc: factor is 1 around here
  }
  coeffs[0] = factor;
  coeffs[1] = c_data;
  coeffs[2] = c_hat;
  coeffs[3] = c_next;
}

// a_next_pre = keep * factor * a_out + keep * c_next (a_out: derivative of the dissipated, scaled smoke);
// a_data += c_data; a_hat = c_hat (a_hat starts here). Dissipation's keep enters as a_out * keep.
__global__ void k_budget_adjoint_apply(const float* __restrict__ a_out, long n, const double* __restrict__ coeffs,
                                       float keep, float* __restrict__ a_next, float* __restrict__ a_data,
                                       float* __restrict__ a_hat) {
  const double factor = coeffs[0], c_data = coeffs[1], c_hat = coeffs[2], c_next = coeffs[3];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double a = (double)a_out[i] * (double)keep;
    a_next[i] = (float)(a * factor + c_next * (double)keep);
    a_data[i] = (float)c_data * keep;
    a_hat[i] = (float)c_hat * keep;
  }
}

// The ortho thickness march (raymarch.py:86-140, thickness channel only) and its adjoint for
// loss = sum over pixels (thickness - target)^2: writes thickness and scatters d loss / d smoke into a_smoke
// (k_loss_sum adds the squared errors to *loss).
__global__ void k_thickness_adjoint(PlumeGridInfo info, PlumeViewParams view, float opacity,
                                    const float* __restrict__ smoke, const float* __restrict__ target, int height,
                                    int width, float* __restrict__ thickness_out, double* __restrict__ loss,
                                    float* __restrict__ a_smoke) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= width || py >= height) return;
  const Dims d = dims_of(info);
  const F3 right = f3(view.right[0], view.right[1], view.right[2]);
  const F3 up = f3(view.up[0], view.up[1], view.up[2]);
  const F3 toward = f3(view.toward[0], view.toward[1], view.toward[2]);
  const float plane_x = view.left_m + ((float)px + 0.5f) * view.pixel_m;
  const float plane_y = view.top_m - ((float)py + 0.5f) * view.pixel_m;
  const F3 origin = add3(add3(mul3(right, plane_x), mul3(up, plane_y)), mul3(toward, 1.0e4f));
  const F3 direction = f3(-toward[0], -toward[1], -toward[2]);
  const F3 box_origin = f3(info.origin_m[0], info.origin_m[1], info.origin_m[2]);
  const F3 box_max = add3(box_origin, mul3(f3((float)d.n0, (float)d.n1, (float)d.n2), info.cell_m));
  float t_enter = -1.0e30f, t_exit = 1.0e30f;
  bool miss = false;
  for (int a = 0; a < 3; ++a) {  // slab_range (raymarch.py:55-69)
    if (fabsf(direction[a]) < 1.0e-12f) {
      if (origin[a] < box_origin[a] || origin[a] > box_max[a]) miss = true;
    } else {
      const float t0 = (box_origin[a] - origin[a]) / direction[a], t1 = (box_max[a] - origin[a]) / direction[a];
      t_enter = fmax_(t_enter, fmin_(t0, t1));
      t_exit = fmin_(t_exit, fmax_(t0, t1));
    }
  }
  float tr = 1.0f;
  int steps = 0;
  float step_m = 0.0f;
  if (!miss && t_exit > t_enter) {
    const float length = t_exit - t_enter;
    steps = (int)ceilf(length / (0.5f * info.cell_m));
    step_m = length / (float)steps;
    for (int s = 0; s < steps; ++s) {
      const F3 position = add3(origin, mul3(direction, t_enter + ((float)s + 0.5f) * step_m));
      const F3 g = sub3(div3(sub3(position, box_origin), info.cell_m), f3(0.5f, 0.5f, 0.5f));
      const float density = fmax_(sample_index_space(smoke, d, g), 0.0f);
      if (density > 0.0f) tr = tr * (1.0f - (1.0f - exp_f(-opacity * density * step_m)));
    }
  }
  const float thickness = 1.0f - tr;
  const long pixel = (long)py * width + px;
  thickness_out[pixel] = thickness;
  const float error = thickness - target[pixel];
  const float a_rho = 2.0f * error * opacity * step_m * tr;
  if (a_rho == 0.0f) return;
  for (int s = 0; s < steps; ++s) {
    const F3 position = add3(origin, mul3(direction, t_enter + ((float)s + 0.5f) * step_m));
    const F3 g = sub3(div3(sub3(position, box_origin), info.cell_m), f3(0.5f, 0.5f, 0.5f));
    if (sample_index_space(smoke, d, g) > 0.0f) scatter(a_smoke, corners_of(d, g), a_rho);
  }
}

// ---- the velocity path (no reference counterpart) ------------------------------------------------------------
// The derivatives with respect to the advecting velocity and the forces, for gradients with respect to the
// buoyancy and drag scalars. Traces are recomputed with the forward kernels' functions; the linearisation is
// that of the reference's formulas (trace: advect.py:16-21, samples: sample.py:10-82).

// sample_index_space at g and its gradient with respect to g (index units): along an axis where the clamp holds
// the coordinate at an end the sample does not move, so that component is 0.
__device__ __forceinline__ float sample_and_gradient(const float* __restrict__ f, const Dims& d, F3 g, F3& grad) {
  const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
  const float* p = f + (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  const float a000 = p[0], a100 = p[x.step], a010 = p[y.step], a110 = p[x.step + y.step];
  const float a001 = p[z.step], a101 = p[x.step + z.step], a011 = p[y.step + z.step];
  const float a111 = p[x.step + y.step + z.step];
  const float c00 = lerp_w(a000, a100, x), c10 = lerp_w(a010, a110, x);
  const float c01 = lerp_w(a001, a101, x), c11 = lerp_w(a011, a111, x);
  const float e0 = lerp_w(c00, c10, y), e1 = lerp_w(c01, c11, y);
  const bool free_x = g[0] >= 0.0f && g[0] <= (float)(d.n0 - 1);
  const bool free_y = g[1] >= 0.0f && g[1] <= (float)(d.n1 - 1);
  const bool free_z = g[2] >= 0.0f && g[2] <= (float)(d.n2 - 1);
  grad[0] = free_x ? lerp_w(lerp_w(a100 - a000, a110 - a010, y), lerp_w(a101 - a001, a111 - a011, y), z) : 0.0f;
  grad[1] = free_y ? lerp_w(c10 - c00, c11 - c01, z) : 0.0f;
  grad[2] = free_z ? e1 - e0 : 0.0f;
  return lerp_w(e0, e1, z);
}

__device__ __forceinline__ F3 component_offset(int c) {
  return f3(c == 0 ? 0.0f : 0.5f, c == 1 ? 0.0f : 0.5f, c == 2 ? 0.0f : 0.5f);
}

// Scatters a velocity derivative w (one value per component) at point m to the components' trilinear corners.
__device__ __forceinline__ void scatter_velocity(float* const a_vel[3], const Vel& vel, F3 m, F3 w) {
  const Dims dims[3] = {vel.du, vel.dv, vel.dw};
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (w[c] != 0.0f) scatter(a_vel[c], corners_of(dims[c], sub3(m, component_offset(c))), w[c]);
}

// The adjoint of end = p - tau V(mid), mid = p - tau/2 V(p) (trace, advect.py:16-21) for d loss / d end = lambda:
// the velocity's derivative at mid, and through mid's own dependence on V(p), at p.
__device__ __forceinline__ void trace_adjoint(const Vel& vel, F3 p, float tau, F3 lambda, float* const a_vel[3]) {
  if (lambda[0] == 0.0f && lambda[1] == 0.0f && lambda[2] == 0.0f) return;
  const F3 vp = velocity_at_node(vel, p);
  const F3 mid = sub3(p, mul3(vp, 0.5f * tau));
  const float* arrays[3] = {vel.u, vel.v, vel.w};
  const Dims dims[3] = {vel.du, vel.dv, vel.dw};
  F3 jac[3];  // jac[c][a] = d V_c / d x_a at mid
#pragma unroll
  for (int c = 0; c < 3; ++c) sample_and_gradient(arrays[c], dims[c], sub3(mid, component_offset(c)), jac[c]);
  const F3 a_vm = mul3(lambda, -tau);
  scatter_velocity(a_vel, vel, mid, a_vm);
  F3 a_mid = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int c = 0; c < 3; ++c) a_mid = add3(a_mid, mul3(jac[c], a_vm[c]));
  scatter_velocity(a_vel, vel, p, mul3(a_mid, -0.5f * tau));
}

struct AdjField {
  const float* data;   // the field before advection
  const float* hat;    // its forward semi-Lagrangian values
  Dims d;
  F3 offset;
  float outside;
  int uses_outside;
};

// MacCormack adjoint, part 1 for any field (cells or faces): the clamp's branch, the correction's own terms, the
// backward sample's transpose into a_hat and, with a_vel, the backward trace's velocity derivative.
__global__ void k_mac_adj_correct(PlumeGridInfo info, Vel vel, AdjField fd, const float* __restrict__ a_next,
                                  float* __restrict__ a_data, float* __restrict__ a_hat, float* a_u, float* a_v,
                                  float* a_w, float dt_over_cell) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = fd.d;
  if (j >= d.n1 || k >= d.n2) return;
  const int c = at(d, i, j, k);
  const float g_next = a_next[c];
  if (g_next == 0.0f) return;
  const F3 p = add3(f3((float)i, (float)j, (float)k), fd.offset);
  const F3 vp = velocity_at_node(vel, p);
  const F3 src = trace_from(vel, p, vp, dt_over_cell);
  const F3 back_src = trace_from(vel, p, vp, -dt_over_cell);
  const bool src_outside = fd.uses_outside == 1 && is_outside_open_face(src, info);
  const bool back_outside = fd.uses_outside == 1 && is_outside_open_face(back_src, info);
  const F3 gb = sub3(back_src, fd.offset);
  const float back = back_outside ? fd.outside : sample_index_space(fd.hat, d, gb);
  const float corrected = __ldg(fd.hat + c) + 0.5f * (__ldg(fd.data + c) - back);
  float lo = fd.outside, hi = fd.outside;
  int lo_idx = -1, hi_idx = -1;
  if (!src_outside) range_corners(fd.data, d, sub3(src, fd.offset), lo_idx, hi_idx, lo, hi);
  if (corrected < lo) {
    if (lo_idx >= 0) atomicAdd(a_data + lo_idx, g_next);
    return;
  }
  if (corrected > hi) {
    if (hi_idx >= 0) atomicAdd(a_data + hi_idx, g_next);
    return;
  }
  atomicAdd(a_hat + c, g_next);
  atomicAdd(a_data + c, 0.5f * g_next);
  if (back_outside) return;
  const float a_back = -0.5f * g_next;
  scatter(a_hat, corners_of(d, gb), a_back);
  if (!a_u) return;
  F3 grad;
  sample_and_gradient(fd.hat, d, gb, grad);
  float* a_vel[3] = {a_u, a_v, a_w};
  trace_adjoint(vel, p, -dt_over_cell, mul3(grad, a_back), a_vel);
}

// MacCormack adjoint, part 2: the forward sample's transpose, a_data += sample^T(a_hat), and with a_vel the
// forward trace's velocity derivative.
__global__ void k_mac_adj_forward(PlumeGridInfo info, Vel vel, AdjField fd, const float* __restrict__ a_hat,
                                  float* __restrict__ a_data, float* a_u, float* a_v, float* a_w, float dt_over_cell) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = fd.d;
  if (j >= d.n1 || k >= d.n2) return;
  const float g = a_hat[at(d, i, j, k)];
  if (g == 0.0f) return;
  const F3 p = add3(f3((float)i, (float)j, (float)k), fd.offset);
  const F3 src = trace_from(vel, p, velocity_at_node(vel, p), dt_over_cell);
  if (fd.uses_outside == 1 && is_outside_open_face(src, info)) return;
  const F3 gs = sub3(src, fd.offset);
  scatter(a_data, corners_of(d, gs), g);
  if (!a_u) return;
  F3 grad;
  sample_and_gradient(fd.data, d, gs, grad);
  float* a_vel[3] = {a_u, a_v, a_w};
  trace_adjoint(vel, p, dt_over_cell, mul3(grad, g), a_vel);
}

// Block sums of a per-thread double into *out (one atomic per block).
__device__ __forceinline__ void block_add(double value, double* out) {
  __shared__ double slot[ADJ_THREADS];
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  slot[t] = value;
  __syncthreads();
  for (int h = ADJ_THREADS / 2; h >= 1; h >>= 1) {
    if (t < h) slot[t] = slot[t] + slot[t + h];
    __syncthreads();
  }
  if (t == 0 && slot[0] != 0.0) atomicAdd(out, slot[0]);
}

// buoyancy_kernel's adjoint (forces.py:13-23) for v += g (hb (T - Ta) / Ta - ws s) dt with T, s averaged over
// the face's two cells: a_T, a_s receive a_v's share; *grad_hb += sum a_v g (T - Ta) / Ta dt. a_v is unchanged.
__global__ void k_buoyancy_adjoint(PlumeGridInfo info, const float* __restrict__ a_v, const float* __restrict__ smoke,
                                   const float* __restrict__ temperature, float* __restrict__ a_smoke,
                                   float* __restrict__ a_temperature, float gravity, float heat_buoyancy,
                                   float smoke_weight, float ambient, float dt, double* grad_hb) {
  const int ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (j <= ny && k < nz) {
    const float a = a_v[(i * (ny + 1) + j) * nz + k];
    if (a != 0.0f) {
      const int below = imax_(j - 1, 0), above = imin_(j, ny - 1);
      const int cb = (i * ny + below) * nz + k, ca = (i * ny + above) * nz + k;
      const float heat = 0.5f * (temperature[cb] + temperature[ca]);
      const float a_heat = a * gravity * dt * heat_buoyancy / ambient;
      atomicAdd(a_temperature + cb, 0.5f * a_heat);
      atomicAdd(a_temperature + ca, 0.5f * a_heat);
      if (smoke_weight != 0.0f && a_smoke) {
        const float a_density = -a * gravity * dt * smoke_weight;
        atomicAdd(a_smoke + cb, 0.5f * a_density);
        atomicAdd(a_smoke + ca, 0.5f * a_density);
      }
      part = (double)a * (double)gravity * (double)dt * ((double)heat - (double)ambient) / (double)ambient;
    }
  }
  block_add(part, grad_hb);
}

// drag_kernel's adjoint (forces.py:34-48) for f = wind + (f_before - wind) keep over the three face arrays
// (blockIdx.z segments as the face kernels): *grad_drag += sum a_f (f_before - wind) (-dt keep) (keep =
// exp(-drag dt)), then a_f *= keep.
__global__ void k_drag_adjoint(PlumeGridInfo info, float* __restrict__ a_u, float* __restrict__ a_v,
                               float* __restrict__ a_w, const float* __restrict__ u, const float* __restrict__ v,
                               const float* __restrict__ w, float3 wind, float keep, float dt, double* grad_drag) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  int slab = blockIdx.z, axis = 0;
  if (slab >= nx + 1) {
    slab -= nx + 1;
    axis = 1;
    if (slab >= nx) {
      slab -= nx;
      axis = 2;
    }
  }
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n1 = ny + (axis == 1), n2 = nz + (axis == 2);
  double part = 0.0;
  if (j < n1 && k < n2) {
    const long c = ((long)slab * n1 + j) * n2 + k;
    float* a = axis == 0 ? a_u : (axis == 1 ? a_v : a_w);
    const float* f = axis == 0 ? u : (axis == 1 ? v : w);
    const float target = axis == 0 ? wind.x : (axis == 1 ? wind.y : wind.z);
    const float g = a[c];
    part = (double)g * ((double)f[c] - (double)target) * (-(double)dt * (double)keep);
    a[c] = g * keep;
  }
  block_add(part, grad_drag);
}

// ---- vorticity confinement's adjoint (vorticity.py:17-84) ----------------------------------------------------
// Forward, per cell: centre velocity c = face averages; curl w = central differences of c (one-sided at the
// edges); spin s = |w|; g = central differences of s; N = g / |g|; push = sigma (N x w) with sigma =
// strength * cell_m (zero where |g| < 1e-12); each face adds dt/2 (push of the cell below + of the cell above),
// the cells clamped into the grid. The adjoint runs those steps backwards, each difference's transpose as a
// gather over the cells whose stencil holds this one, so no atomics are needed.

// The transpose of one axis's central difference D(c') = (x[hi(c')] - x[lo(c')]) / (span(c') h), hi/lo
// clamped into 0..n-1 (vorticity.py:25-35): d/dx[t] of sum over c' of e[c'] D(c').
__device__ __forceinline__ float difference_adjoint(const float* __restrict__ e, long at_t, long stride, int t, int n,
                                                    float h) {
  if (n < 2) return 0.0f;
  auto span = [&](int c) { return (float)(imin_(c + 1, n - 1) - imax_(c - 1, 0)) * h; };
  float total = 0.0f;
  if (t >= 1) total += __ldg(e + at_t - stride) / span(t - 1);  // t is the upper point of cell t - 1
  if (t <= n - 2) total -= __ldg(e + at_t + stride) / span(t + 1);  // the lower point of cell t + 1
  if (t == n - 1) total += __ldg(e + at_t) / span(t);  // an edge cell is its own upper (or lower) point
  if (t == 0) total -= __ldg(e + at_t) / span(t);
  return total;
}

// Curl and spin of the velocity before confinement (the forward's values, recomputed).
__global__ void k_conf_adj_curl(PlumeGridInfo info, Vel vel, float* __restrict__ wx, float* __restrict__ wy,
                                float* __restrict__ wz, float* __restrict__ spin) {
  const int n[3] = {info.dims[0], info.dims[1], info.dims[2]};
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n[1] || k >= n[2]) return;
  auto centre = [&](int a, int b, int c) {
    return f3(0.5f * (__ldg(vel.u + at(vel.du, a, b, c)) + __ldg(vel.u + at(vel.du, a + 1, b, c))),
              0.5f * (__ldg(vel.v + at(vel.dv, a, b, c)) + __ldg(vel.v + at(vel.dv, a, b + 1, c))),
              0.5f * (__ldg(vel.w + at(vel.dw, a, b, c)) + __ldg(vel.w + at(vel.dw, a, b, c + 1))));
  };
  const int cell[3] = {i, j, k};
  F3 d[3];
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[axis] = imax_(cell[axis] - 1, 0);
    hi[axis] = imin_(cell[axis] + 1, n[axis] - 1);
    const float span = (float)(hi[axis] - lo[axis]);
    d[axis] = span == 0.0f ? f3(0.0f, 0.0f, 0.0f)
                           : div3(sub3(centre(hi[0], hi[1], hi[2]), centre(lo[0], lo[1], lo[2])), span * info.cell_m);
  }
  const long c = ((long)i * n[1] + j) * n[2] + k;
  const F3 w = f3(d[1][2] - d[2][1], d[2][0] - d[0][2], d[0][1] - d[1][0]);
  wx[c] = w[0];
  wy[c] = w[1];
  wz[c] = w[2];
  spin[c] = len3(w);
}

// The push's adjoint at each cell: the push derivative gathered from the faces beside the cell, then through
// push = sigma (N x w) and N = g / |g|: writes d/dg (ga) and the direct part of d/dw (wa), and adds
// d loss / d strength = sum over cells of pbar . cell_m (N x w).
__global__ void k_conf_adj_push(PlumeGridInfo info, const float* __restrict__ a_u, const float* __restrict__ a_v,
                                const float* __restrict__ a_w, const float* __restrict__ wx,
                                const float* __restrict__ wy, const float* __restrict__ wz,
                                const float* __restrict__ spin, float* __restrict__ gax, float* __restrict__ gay,
                                float* __restrict__ gaz, float* __restrict__ wax, float* __restrict__ way,
                                float* __restrict__ waz, float strength, float dt, double* grad_strength) {
  const int n[3] = {info.dims[0], info.dims[1], info.dims[2]};
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (j < n[1] && k < n[2]) {
    const int cell[3] = {i, j, k};
    const Dims cd{n[0], n[1], n[2]};
    const long c = ((long)i * n[1] + j) * n[2] + k;
    // pbar: face t of the axis feeds cells max(t-1, 0) and min(t, n-1) with weight dt/2 each
    const float* a_face[3] = {a_u, a_v, a_w};
    F3 pbar;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      const Dims fd{n[0] + (axis == 0), n[1] + (axis == 1), n[2] + (axis == 2)};
      int up[3] = {i, j, k};
      up[axis] += 1;
      const float lo_face = __ldg(a_face[axis] + at(fd, i, j, k));
      const float hi_face = __ldg(a_face[axis] + at(fd, up[0], up[1], up[2]));
      float total = lo_face + hi_face;
      if (cell[axis] == 0) total += lo_face;
      if (cell[axis] == n[axis] - 1) total += hi_face;
      pbar[axis] = 0.5f * dt * total;
    }
    F3 g = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      int lo[3] = {i, j, k}, hi[3] = {i, j, k};
      lo[axis] = imax_(cell[axis] - 1, 0);
      hi[axis] = imin_(cell[axis] + 1, n[axis] - 1);
      const float span = (float)(hi[axis] - lo[axis]);
      if (span > 0.0f)
        g[axis] = (__ldg(spin + at(cd, hi[0], hi[1], hi[2])) - __ldg(spin + at(cd, lo[0], lo[1], lo[2]))) /
                  (span * info.cell_m);
    }
    const float length = len3(g);
    F3 ga = f3(0.0f, 0.0f, 0.0f), wa = f3(0.0f, 0.0f, 0.0f);
    if (length >= 1.0e-12f) {
      const F3 w = f3(__ldg(wx + c), __ldg(wy + c), __ldg(wz + c));
      const F3 nrm = div3(g, length);
      const float sigma = strength * info.cell_m;
      const F3 nbar = mul3(cross3(w, pbar), sigma);
      wa = mul3(cross3(pbar, nrm), sigma);
      ga = div3(sub3(nbar, mul3(nrm, dot3(nrm, nbar))), length);
      const F3 nw = cross3(nrm, w);
      part = (double)info.cell_m * ((double)pbar[0] * nw[0] + (double)pbar[1] * nw[1] + (double)pbar[2] * nw[2]);
    }
    gax[c] = ga[0];
    gay[c] = ga[1];
    gaz[c] = ga[2];
    wax[c] = wa[0];
    way[c] = wa[1];
    waz[c] = wa[2];
  }
  block_add(part, grad_strength);
}

// The spin's adjoint: sbar = the transposed differences of ga; w's derivative += sbar w / s (s > 0).
__global__ void k_conf_adj_spin(PlumeGridInfo info, const float* __restrict__ gax, const float* __restrict__ gay,
                                const float* __restrict__ gaz, const float* __restrict__ wx,
                                const float* __restrict__ wy, const float* __restrict__ wz,
                                const float* __restrict__ spin, float* __restrict__ wax, float* __restrict__ way,
                                float* __restrict__ waz) {
  const int n[3] = {info.dims[0], info.dims[1], info.dims[2]};
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n[1] || k >= n[2]) return;
  const long plane = (long)n[1] * n[2], c = i * plane + (long)j * n[2] + k;
  const float h = info.cell_m;
  const float sbar = difference_adjoint(gax, c, plane, i, n[0], h) + difference_adjoint(gay, c, n[2], j, n[1], h) +
                     difference_adjoint(gaz, c, 1, k, n[2], h);
  const float s = __ldg(spin + c);
  if (s > 0.0f && sbar != 0.0f) {
    const float scale = sbar / s;
    wax[c] += scale * __ldg(wx + c);
    way[c] += scale * __ldg(wy + c);
    waz[c] += scale * __ldg(wz + c);
  }
}

// The curl's adjoint: the centre velocity's derivative from w's (wa) through the transposed differences:
// cbar_x = D_z^T(wa_y) - D_y^T(wa_z), cbar_y = D_x^T(wa_z) - D_z^T(wa_x), cbar_z = D_y^T(wa_x) - D_x^T(wa_y).
__global__ void k_conf_adj_curlT(PlumeGridInfo info, const float* __restrict__ wax, const float* __restrict__ way,
                                 const float* __restrict__ waz, float* __restrict__ cbx, float* __restrict__ cby,
                                 float* __restrict__ cbz) {
  const int n[3] = {info.dims[0], info.dims[1], info.dims[2]};
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n[1] || k >= n[2]) return;
  const long plane = (long)n[1] * n[2], c = i * plane + (long)j * n[2] + k;
  const float h = info.cell_m;
  auto dx = [&](const float* e) { return difference_adjoint(e, c, plane, i, n[0], h); };
  auto dy = [&](const float* e) { return difference_adjoint(e, c, n[2], j, n[1], h); };
  auto dz = [&](const float* e) { return difference_adjoint(e, c, 1, k, n[2], h); };
  cbx[c] = dz(way) - dy(waz);
  cby[c] = dx(waz) - dz(wax);
  cbz[c] = dy(wax) - dx(way);
}

// The centre velocity's adjoint onto the faces: face t of an axis averages into cells t - 1 and t.
__global__ void k_conf_adj_faces(PlumeGridInfo info, float* __restrict__ a_u, float* __restrict__ a_v,
                                 float* __restrict__ a_w, const float* __restrict__ cbx, const float* __restrict__ cby,
                                 const float* __restrict__ cbz) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  int slab = blockIdx.z, axis = 0;
  if (slab >= nx + 1) {
    slab -= nx + 1;
    axis = 1;
    if (slab >= nx) {
      slab -= nx;
      axis = 2;
    }
  }
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n1 = ny + (axis == 1), n2 = nz + (axis == 2);
  if (j >= n1 || k >= n2) return;
  const int face[3] = {slab, j, k};
  const int n[3] = {nx, ny, nz};
  const Dims cd{nx, ny, nz};
  const float* cb = axis == 0 ? cbx : (axis == 1 ? cby : cbz);
  float* a = axis == 0 ? a_u : (axis == 1 ? a_v : a_w);
  const int t = face[axis];
  float total = 0.0f;
  if (t >= 1) {
    int b[3] = {slab, j, k};
    b[axis] -= 1;
    total += __ldg(cb + at(cd, b[0], b[1], b[2]));
  }
  if (t <= n[axis] - 1) total += __ldg(cb + at(cd, slab, j, k));
  a[((long)slab * n1 + j) * n2 + k] += 0.5f * total;
}

}  // namespace plume

using namespace plume;

#define ADJ_CHECK(cond, what) \
  do {                        \
    if (!(cond)) return fail(PLUME_ERR_INVALID, "%s", what); \
  } while (0)

extern "C" int plume_add_source(float* smoke, const int32_t shape[3], const float* source, const int32_t source_shape[3],
                                const int32_t corner[3], float scale, void* stream) {
  ADJ_CHECK(smoke && shape && source && source_shape && corner, "add_source: null argument");
  const Dims s{source_shape[0], source_shape[1], source_shape[2]};
  k_add_source<<<adj_blocks((long)s.n0 * s.n1 * s.n2), ADJ_THREADS, 0, as_stream(stream)>>>(
      smoke, Dims{shape[0], shape[1], shape[2]}, source, s, make_int3(corner[0], corner[1], corner[2]), scale);
  return launch_status("add source");
}

extern "C" int plume_source_grad(const float* a_smoke, const int32_t shape[3], float* grad, const int32_t source_shape[3],
                                 const int32_t corner[3], float scale, void* stream) {
  ADJ_CHECK(a_smoke && shape && grad && source_shape && corner, "source_grad: null argument");
  const Dims s{source_shape[0], source_shape[1], source_shape[2]};
  k_source_grad<<<adj_blocks((long)s.n0 * s.n1 * s.n2), ADJ_THREADS, 0, as_stream(stream)>>>(
      a_smoke, Dims{shape[0], shape[1], shape[2]}, grad, s, make_int3(corner[0], corner[1], corner[2]), scale);
  return launch_status("source gradient");
}

extern "C" int plume_smoke_adjoint(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                   const float* data, const float* hat, const float* next_pre, const double* totals,
                                   float dt_over_cell, float keep, const float* a_out, float* a_next, float* a_hat,
                                   float* a_data, double* partial, double* coeffs, void* stream) {
  ADJ_CHECK(info && u && v && w && data && hat && next_pre && totals && a_out && a_next && a_hat && a_data && partial &&
                coeffs && a_data != a_out,
            "smoke_adjoint: bad argument");
  cudaStream_t st = as_stream(stream);
  const Dims d = dims_of(*info);
  const long n = (long)d.n0 * d.n1 * d.n2;
  const int blocks = (int)std::min<long>(adj_blocks(n), 1024);
  k_dot_partials<<<blocks, ADJ_THREADS, 0, st>>>(a_out, next_pre, n, partial);
  int status = launch_status("adjoint dot");
  if (status != PLUME_OK) return status;
  k_budget_adjoint_coeffs<<<1, 32, 0, st>>>(totals, partial, blocks, coeffs);
  if ((status = launch_status("budget adjoint coefficients")) != PLUME_OK) return status;
  k_budget_adjoint_apply<<<blocks, ADJ_THREADS, 0, st>>>(a_out, n, coeffs, keep, a_next, a_data, a_hat);
  if ((status = launch_status("budget adjoint")) != PLUME_OK) return status;
  const Vel vel = make_vel(u, v, w, info->dims);
  k_mac_adjoint_correct<<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(*info, vel, data, hat, a_next, a_data, a_hat,
                                                                              dt_over_cell, 0.0f);
  if ((status = launch_status("MacCormack adjoint (correction)")) != PLUME_OK) return status;
  k_mac_adjoint_forward<<<cell_grid(d.n0, d.n1, d.n2), cell_block(), 0, st>>>(*info, vel, a_hat, a_data, dt_over_cell);
  return launch_status("MacCormack adjoint (forward sample)");
}

// *loss += sum over pixels (thickness - target)^2 in double, in one fixed order: one block, each thread a fixed
// stride of pixels, then a halving tree, so the same images give the same loss bit for bit on every run.
__global__ void __launch_bounds__(1024) k_loss_sum(const float* __restrict__ thickness, const float* __restrict__ target,
                                                   long n, double* __restrict__ loss) {
  __shared__ double slot[1024];
  double value = 0.0;
  for (long i = threadIdx.x; i < n; i += 1024) {
    const float error = thickness[i] - target[i];
    value = value + (double)error * (double)error;
  }
  slot[threadIdx.x] = value;
  __syncthreads();
  for (int h = 512; h >= 1; h >>= 1) {
    if ((int)threadIdx.x < h) slot[threadIdx.x] = slot[threadIdx.x] + slot[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = *loss + slot[0];
}

extern "C" int plume_thickness_adjoint(const PlumeGridInfo* info, const PlumeViewParams* view, float opacity,
                                       const float* smoke, const float* target, int32_t height, int32_t width,
                                       float* thickness, double* loss, float* a_smoke, void* stream) {
  ADJ_CHECK(info && view && smoke && target && thickness && loss && a_smoke && height >= 1 && width >= 1 &&
                view->perspective == 0,
            "thickness_adjoint: bad argument (orthographic views only)");
  dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
  k_thickness_adjoint<<<grid, block, 0, as_stream(stream)>>>(*info, *view, opacity, smoke, target, height, width,
                                                             thickness, loss, a_smoke);
  int status = launch_status("thickness adjoint");
  if (status != PLUME_OK) return status;
  k_loss_sum<<<1, 1024, 0, as_stream(stream)>>>(thickness, target, (long)height * width, loss);
  return launch_status("thickness loss");
}

extern "C" int plume_maccormack_adjoint(const PlumeGridInfo* info, const int32_t shape[3], const float offset[3],
                                       const float* data, const float* hat, const float* u, const float* v,
                                       const float* w, const float* a_next, float* a_data, float* a_hat, float* a_u,
                                       float* a_v, float* a_w, float dt_over_cell, float outside, int32_t uses_outside,
                                       void* stream) {
  ADJ_CHECK(info && shape && offset && data && hat && u && v && w && a_next && a_data && a_hat,
            "maccormack_adjoint: null argument");
  ADJ_CHECK((a_u == nullptr) == (a_v == nullptr) && (a_v == nullptr) == (a_w == nullptr),
            "maccormack_adjoint: give all three velocity adjoints or none");
  cudaStream_t st = as_stream(stream);
  AdjField fd{data, hat, Dims{shape[0], shape[1], shape[2]}, f3(offset[0], offset[1], offset[2]), outside,
              uses_outside};
  const Vel vel = make_vel(u, v, w, info->dims);
  const dim3 grid = cell_grid(fd.d.n0, fd.d.n1, fd.d.n2);
  k_mac_adj_correct<<<grid, cell_block(), 0, st>>>(*info, vel, fd, a_next, a_data, a_hat, a_u, a_v, a_w, dt_over_cell);
  int status = launch_status("MacCormack adjoint (correction, velocity)");
  if (status != PLUME_OK) return status;
  k_mac_adj_forward<<<grid, cell_block(), 0, st>>>(*info, vel, fd, a_hat, a_data, a_u, a_v, a_w, dt_over_cell);
  return launch_status("MacCormack adjoint (forward sample, velocity)");
}

extern "C" int plume_buoyancy_adjoint(const PlumeGridInfo* info, const float* a_v, const float* smoke,
                                      const float* temperature, float* a_smoke, float* a_temperature, float gravity,
                                      float heat_buoyancy, float smoke_weight, float ambient_k, float dt,
                                      double* grad_heat_buoyancy, void* stream) {
  ADJ_CHECK(info && a_v && smoke && temperature && a_temperature && grad_heat_buoyancy,
            "buoyancy_adjoint: null argument");
  const int nx = info->dims[0], ny = info->dims[1], nz = info->dims[2];
  k_buoyancy_adjoint<<<cell_grid(nx, ny + 1, nz), cell_block(), 0, as_stream(stream)>>>(
      *info, a_v, smoke, temperature, a_smoke, a_temperature, gravity, heat_buoyancy, smoke_weight, ambient_k, dt,
      grad_heat_buoyancy);
  return launch_status("buoyancy adjoint");
}

extern "C" int plume_drag_adjoint(const PlumeGridInfo* info, float* a_u, float* a_v, float* a_w, const float* u,
                                  const float* v, const float* w, const float wind[3], float keep, float dt,
                                  double* grad_drag, void* stream) {
  ADJ_CHECK(info && a_u && a_v && a_w && u && v && w && wind && grad_drag, "drag_adjoint: null argument");
  const int nx = info->dims[0], ny = info->dims[1], nz = info->dims[2];
  const dim3 grid((nz + 1 + TZ - 1) / TZ, (ny + 1 + TY - 1) / TY, (nx + 1) + nx + nx);
  k_drag_adjoint<<<grid, cell_block(), 0, as_stream(stream)>>>(*info, a_u, a_v, a_w, u, v, w,
                                                              make_float3(wind[0], wind[1], wind[2]), keep, dt,
                                                              grad_drag);
  return launch_status("drag adjoint");
}

extern "C" int plume_budget_adjoint(const PlumeGridInfo* info, const float* next_pre, const double* totals, float keep,
                                   const float* a_out, float* a_next, float* a_data, float* a_hat, double* partial,
                                   double* coeffs, void* stream) {
  ADJ_CHECK(info && next_pre && totals && a_out && a_next && a_data && a_hat && partial && coeffs,
            "budget_adjoint: null argument");
  cudaStream_t st = as_stream(stream);
  const Dims d = dims_of(*info);
  const long n = (long)d.n0 * d.n1 * d.n2;
  const int blocks = (int)std::min<long>(adj_blocks(n), 1024);
  k_dot_partials<<<blocks, ADJ_THREADS, 0, st>>>(a_out, next_pre, n, partial);
  int status = launch_status("adjoint dot");
  if (status != PLUME_OK) return status;
  k_budget_adjoint_coeffs<<<1, 32, 0, st>>>(totals, partial, blocks, coeffs);
  if ((status = launch_status("budget adjoint coefficients")) != PLUME_OK) return status;
  k_budget_adjoint_apply<<<blocks, ADJ_THREADS, 0, st>>>(a_out, n, coeffs, keep, a_next, a_data, a_hat);
  return launch_status("budget adjoint");
}

extern "C" int plume_confinement_adjoint(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                         float* a_u, float* a_v, float* a_w, float strength, float dt, float* scratch,
                                         double* grad_strength, void* stream) {
  ADJ_CHECK(info && u && v && w && a_u && a_v && a_w && scratch && grad_strength,
            "confinement_adjoint: null argument");
  ADJ_CHECK(info->dims[0] >= 1 && info->dims[1] >= 1 && info->dims[2] >= 1, "confinement_adjoint: bad dims");
  cudaStream_t st = as_stream(stream);
  const Dims d = dims_of(*info);
  const long n = (long)d.n0 * d.n1 * d.n2;
  float* wx = scratch;  // curl (3), spin, d/dg (3), d/dw (3); d/dg's arrays then hold d/d centre velocity
  float *wy = wx + n, *wz = wy + n, *spin = wz + n, *gax = spin + n, *gay = gax + n, *gaz = gay + n;
  float *wax = gaz + n, *way = wax + n, *waz = way + n;
  const dim3 grid = cell_grid(d.n0, d.n1, d.n2);
  k_conf_adj_curl<<<grid, cell_block(), 0, st>>>(*info, make_vel(u, v, w, info->dims), wx, wy, wz, spin);
  int status = launch_status("confinement adjoint (curl)");
  if (status != PLUME_OK) return status;
  k_conf_adj_push<<<grid, cell_block(), 0, st>>>(*info, a_u, a_v, a_w, wx, wy, wz, spin, gax, gay, gaz, wax, way, waz,
                                                 strength, dt, grad_strength);
  if ((status = launch_status("confinement adjoint (push)")) != PLUME_OK) return status;
  k_conf_adj_spin<<<grid, cell_block(), 0, st>>>(*info, gax, gay, gaz, wx, wy, wz, spin, wax, way, waz);
  if ((status = launch_status("confinement adjoint (spin)")) != PLUME_OK) return status;
  k_conf_adj_curlT<<<grid, cell_block(), 0, st>>>(*info, wax, way, waz, gax, gay, gaz);
  if ((status = launch_status("confinement adjoint (curl transpose)")) != PLUME_OK) return status;
  const dim3 faces((d.n2 + 1 + TZ - 1) / TZ, (d.n1 + 1 + TY - 1) / TY, (d.n0 + 1) + d.n0 + d.n0);
  k_conf_adj_faces<<<faces, cell_block(), 0, st>>>(*info, a_u, a_v, a_w, gax, gay, gaz);
  return launch_status("confinement adjoint (faces)");
}

extern "C" long plume_confinement_adjoint_scratch_floats(const PlumeGridInfo* info) {
  return info ? 10L * info->dims[0] * info->dims[1] * info->dims[2] : -1;
}
