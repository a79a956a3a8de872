// Compute kernels of the live viewer (chadmv/plume src/plume/view/*): everything the viewer computes on the
// device between a kept frame and the window's display bytes. The window itself (imgui + OpenGL) is not part of
// this library; these kernels produce the bytes it would show.
//   - the look: a raw march image to display bytes by view (viewport.py:78-113);
//   - the centre ray's depth where the thickness first passes a threshold (viewport.py:116-140);
//   - the slice plane: cell-centre velocity, its curl, its length, and the plane coloured over the volume's
//     display bytes (slice_plane.py:104-137, vorticity.py:17-45);
//   - the six boundary layers of the smoke (live_run.py:42-57);
//   - the frame cache's float32 <-> float16 casts (frame_cache.py:26-50).
// Arithmetic is float32 in the reference's order (built with -fmad=false).
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace plume {

constexpr int VIEW_CHANNELS = 5;
constexpr float VIEW_NO_SMOKE = 1e-12f;  // sheet/shade.py:20
constexpr float SLICE_DIM = 0.4f;        // slice_plane.py:35

struct LookInputsC {  // viewport.py:50-59
  int view;
  int shade_layout;
  float heat_divisor, shade_divisor, shade_depth, ambient;
  float toward_light[3];
  float background[3];
};

__device__ __forceinline__ F3 table_lookup(const float* __restrict__ table, int n, float value) {
  const float position = clampf_(value, 0.0f, 1.0f) * (float)(n - 1);
  const int low = imin_((int)position, n - 2);
  const float t = position - (float)low;
  const float* a = table + 3 * low;
  const float* b = a + 3;
  return f3(lerpf_(a[0], b[0], t), lerpf_(a[1], b[1], t), lerpf_(a[2], b[2], t));
}

__device__ __forceinline__ uint8_t view_byte(float value) {  // viewport.py:72-74
  return (uint8_t)(int)clampf_(floorf(value * 255.0f + 0.5f), 0.0f, 255.0f);
}

__device__ __forceinline__ uint8_t srgb_byte(const uint8_t* __restrict__ table, int n, float linear) {
  return table[(int)(clampf_(linear, 0.0f, 1.0f) * (float)(n - 1) + 0.5f)];
}

__global__ void k_look(const float* __restrict__ raw, int height, int width, const float* __restrict__ smoke_ramp,
                       const float* __restrict__ emission_ramp, int ramp_n, const uint8_t* __restrict__ srgb, int srgb_n,
                       LookInputsC in, uint8_t* __restrict__ out) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= width || py >= height) return;
  const float* r = raw + ((long)py * width + px) * VIEW_CHANNELS;
  const float heat = clampf_(r[0] / in.heat_divisor, 0.0f, 1.0f);
  const float thickness = clampf_(r[1], 0.0f, 1.0f);
  const F3 normal = f3(r[2], r[3], r[4]);
  float shade = 0.0f, light = 1.0f;
  if (in.shade_layout == 1) {
    if (thickness > VIEW_NO_SMOKE) shade = clampf_(r[2] / thickness / in.shade_divisor, 0.0f, 1.0f);
    light = 1.0f - in.shade_depth * (1.0f - shade);
  } else {
    const F3 toward = f3(in.toward_light[0], in.toward_light[1], in.toward_light[2]);
    light = in.ambient + (1.0f - in.ambient) * fmax_(0.0f, dot3(normal, toward));
  }
  uint8_t* o = out + ((long)py * width + px) * 4;
  if (in.view == 0) {
    const F3 ramp = table_lookup(smoke_ramp, ramp_n, heat);
    const F3 smoke = f3(ramp[0] * light, ramp[1] * light, ramp[2] * light);
    const F3 glow = table_lookup(emission_ramp, ramp_n, heat);
    for (int c = 0; c < 3; ++c) {
      const float linear = (in.background[c] * (1.0f - thickness) + smoke[c] * thickness) + glow[c];
      o[c] = srgb_byte(srgb, srgb_n, linear);
    }
  } else {
    float gray = heat;
    if (in.view == 2) gray = thickness;
    else if (in.view == 3) gray = shade;
    F3 color = f3(gray, gray, gray);
    if (in.view == 3 && in.shade_layout == 0) color = mul3(add3(normal, f3(1.0f, 1.0f, 1.0f)), 0.5f);
    for (int c = 0; c < 3; ++c) o[c] = view_byte(color[c]);
  }
  o[3] = 255;
}

__device__ __forceinline__ void view_slab(F3 origin, F3 dir, F3 bmin, F3 bmax, float& t0out, float& t1out) {
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

// viewport.py:116-140 center_depth_kernel (one thread).
__global__ void k_center_depth(const float* __restrict__ smoke, PlumeGridInfo info, F3 origin, F3 direction,
                               float opacity, float threshold, float* __restrict__ result) {
  const Dims d = dims_of(info);
  const F3 box_origin = f3(info.origin_m[0], info.origin_m[1], info.origin_m[2]);
  const F3 box_max = add3(box_origin, mul3(f3((float)d.n0, (float)d.n1, (float)d.n2), info.cell_m));
  float s0, s1;
  view_slab(origin, direction, box_origin, box_max, s0, s1);
  const float start = fmax_(s0, 0.0f);
  float found = -1.0f;
  if (s1 > start) {
    const float length = s1 - start;
    const int steps = (int)ceilf(length / (0.5f * info.cell_m));
    const float step_m = length / (float)steps;
    float transmittance = 1.0f;
    for (int s = 0; s < steps; ++s) {
      const float distance = start + ((float)s + 0.5f) * step_m;
      const F3 g = sub3(div3(sub3(add3(origin, mul3(direction, distance)), box_origin), info.cell_m), f3(0.5f, 0.5f, 0.5f));
      const float density = fmax_(sample_index_space(smoke, d, g), 0.0f);
      transmittance = transmittance * exp_f(-opacity * density * step_m);
      if (found < 0.0f && 1.0f - transmittance >= threshold) found = distance;
    }
  }
  *result = found;
}

// vorticity.py:17-22 center_velocity_kernel: (nx, ny, nz, 3) cell-centre velocity.
__global__ void k_center_velocity(PlumeGridInfo info, const float* __restrict__ u, const float* __restrict__ v,
                                  const float* __restrict__ w, float* __restrict__ out) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = dims_of(info);
  if (j >= d.n1 || k >= d.n2) return;
  const Vel vel = make_vel(u, v, w, info.dims);
  float* o = out + (long)at(d, i, j, k) * 3;
  o[0] = 0.5f * (__ldg(vel.u + at(vel.du, i, j, k)) + __ldg(vel.u + at(vel.du, i + 1, j, k)));
  o[1] = 0.5f * (__ldg(vel.v + at(vel.dv, i, j, k)) + __ldg(vel.v + at(vel.dv, i, j + 1, k)));
  o[2] = 0.5f * (__ldg(vel.w + at(vel.dw, i, j, k)) + __ldg(vel.w + at(vel.dw, i, j, k + 1)));
}

// vorticity.py:25-45 curl_kernel over a cell-centred vector field (central differences, one-sided at edges).
__global__ void k_curl_centers(PlumeGridInfo info, const float* __restrict__ centers, float* __restrict__ curl) {
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims d = dims_of(info);
  if (j >= d.n1 || k >= d.n2) return;
  const int cell[3] = {i, j, k};
  const int n[3] = {d.n0, d.n1, d.n2};
  F3 g[3];
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[axis] = imax_(cell[axis] - 1, 0);
    hi[axis] = imin_(cell[axis] + 1, n[axis] - 1);
    const float span = (float)(hi[axis] - lo[axis]);
    if (span == 0.0f) {
      g[axis] = f3(0.0f, 0.0f, 0.0f);
    } else {
      const float* a = centers + (long)at(d, hi[0], hi[1], hi[2]) * 3;
      const float* b = centers + (long)at(d, lo[0], lo[1], lo[2]) * 3;
      g[axis] = div3(sub3(f3(a[0], a[1], a[2]), f3(b[0], b[1], b[2])), span * info.cell_m);
    }
  }
  float* o = curl + (long)at(d, i, j, k) * 3;
  o[0] = g[1][2] - g[2][1];
  o[1] = g[2][0] - g[0][2];
  o[2] = g[0][1] - g[1][0];
}

// slice_plane.py:104-107 speed_kernel: |v| of a (cells, 3) vector field.
__global__ void k_speed(const float* __restrict__ vectors, long cells, float* __restrict__ out) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const float* p = vectors + c * 3;
  out[c] = len3(f3(p[0], p[1], p[2]));
}

// slice_plane.py:110-137 slice_kernel: colours the pixels whose ray meets the plane axis = coordinate inside the
// domain by the field there; dims the rest of the display bytes in place.
__global__ void k_slice(PlumeViewParams view, PlumeGridInfo info, int axis, float coordinate_m,
                        const float* __restrict__ values, float low, float high, const float* __restrict__ ramp,
                        int ramp_n, uint8_t* __restrict__ image, int height, int width) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= width || py >= height) return;
  const F3 right = f3(view.right[0], view.right[1], view.right[2]);
  const F3 up = f3(view.up[0], view.up[1], view.up[2]);
  const F3 toward = f3(view.toward[0], view.toward[1], view.toward[2]);
  const float plane_x = view.left_m + ((float)px + 0.5f) * view.pixel_m;  // pixel_ray (raymarch.py:72-83)
  const float plane_y = view.top_m - ((float)py + 0.5f) * view.pixel_m;
  F3 origin = add3(add3(mul3(right, plane_x), mul3(up, plane_y)), mul3(toward, 1.0e4f));
  F3 direction = f3(-toward[0], -toward[1], -toward[2]);
  if (view.perspective == 1) {
    origin = f3(view.eye[0], view.eye[1], view.eye[2]);
    direction = normalize3(sub3(add3(mul3(right, plane_x), mul3(up, plane_y)), toward));
  }
  bool hit = false;
  F3 position = f3(0.0f, 0.0f, 0.0f);
  if (fabsf(direction[axis]) > 1.0e-9f) {
    const float distance = (coordinate_m - origin[axis]) / direction[axis];
    if (view.perspective == 0 || distance > 0.0f) {
      position = add3(origin, mul3(direction, distance));
      hit = true;
      for (int other = 0; other < 3; ++other) {
        const float extent = (float)info.dims[other] * info.cell_m;
        if (other != axis && (position[other] < info.origin_m[other] || position[other] > info.origin_m[other] + extent))
          hit = false;
      }
    }
  }
  uint8_t* o = image + ((long)py * width + px) * 4;
  if (hit) {
    const F3 box_origin = f3(info.origin_m[0], info.origin_m[1], info.origin_m[2]);
    const F3 g = sub3(div3(sub3(position, box_origin), info.cell_m), f3(0.5f, 0.5f, 0.5f));
    const F3 color = table_lookup(ramp, ramp_n, (sample_index_space(values, dims_of(info), g) - low) / (high - low));
    o[0] = view_byte(color[0]);
    o[1] = view_byte(color[1]);
    o[2] = view_byte(color[2]);
  } else {
    for (int c = 0; c < 3; ++c) o[c] = view_byte((float)o[c] / 255.0f * SLICE_DIM);
  }
}

// live_run.py:42-57 boundary_layer_kernel: layers[face][a][b], faces x low, x high, y low, y high, z low, z high;
// a, b the face's other two axes in x, y, z order; 0 past a face's size.
__global__ void k_boundary_layers(const float* __restrict__ smoke, Dims d, int side, float* __restrict__ layers) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 6L * side * side) return;
  const int b = (int)(idx % side), a = (int)((idx / side) % side), face = (int)(idx / ((long)side * side));
  const int axis = face / 2;
  const int first = imin_((axis + 1) % 3, (axis + 2) % 3), second = imax_((axis + 1) % 3, (axis + 2) % 3);
  const int n[3] = {d.n0, d.n1, d.n2};
  if (a >= n[first] || b >= n[second]) {
    layers[idx] = 0.0f;
    return;
  }
  int cell[3] = {0, 0, 0};
  cell[axis] = (face % 2) * (n[axis] - 1);
  cell[first] = a;
  cell[second] = b;
  layers[idx] = smoke[at(d, cell[0], cell[1], cell[2])];
}

// frame_cache.py:26-50: float32 -> float16 (round to nearest even) and back.
__global__ void k_narrow(const float* __restrict__ src, __half* __restrict__ dst, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = __float2half_rn(src[i]);
}
__global__ void k_widen(const __half* __restrict__ src, float* __restrict__ dst, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = __half2float(src[i]);
}

}  // namespace plume

using namespace plume;

#define VIEW_CHECK(cond, what) \
  do {                         \
    if (!(cond)) return fail(PLUME_ERR_INVALID, "%s", what); \
  } while (0)

extern "C" int plume_view_look(const float* raw, int32_t height, int32_t width, const float* smoke_ramp,
                               const float* emission_ramp, int32_t ramp_n, const uint8_t* srgb, int32_t srgb_n,
                               const PlumeLookInputs* inputs, uint8_t* out, void* stream) {
  VIEW_CHECK(raw && smoke_ramp && emission_ramp && srgb && inputs && out && height >= 1 && width >= 1 && ramp_n >= 2 &&
                 srgb_n >= 2 && inputs->view >= 0 && inputs->view <= 3,
             "view_look: bad argument");
  LookInputsC in;
  in.view = inputs->view;
  in.shade_layout = inputs->shade_layout;
  in.heat_divisor = inputs->heat_divisor;
  in.shade_divisor = inputs->shade_divisor;
  in.shade_depth = inputs->shade_depth;
  in.ambient = inputs->ambient;
  for (int c = 0; c < 3; ++c) {
    in.toward_light[c] = inputs->toward_light[c];
    in.background[c] = inputs->background[c];
  }
  dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
  k_look<<<grid, block, 0, as_stream(stream)>>>(raw, height, width, smoke_ramp, emission_ramp, ramp_n, srgb, srgb_n,
                                                in, out);
  return launch_status("look");
}

extern "C" int plume_view_center_depth(const float* smoke, const PlumeGridInfo* info, const float origin[3],
                                       const float direction[3], float opacity_per_density, float threshold,
                                       float* result, void* stream) {
  VIEW_CHECK(smoke && info && origin && direction && result, "view_center_depth: bad argument");
  k_center_depth<<<1, 1, 0, as_stream(stream)>>>(smoke, *info, f3(origin[0], origin[1], origin[2]),
                                                 f3(direction[0], direction[1], direction[2]), opacity_per_density,
                                                 threshold, result);
  return launch_status("center depth");
}

extern "C" int plume_view_center_velocity(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                          float* centers, void* stream) {
  VIEW_CHECK(info && u && v && w && centers, "view_center_velocity: bad argument");
  k_center_velocity<<<cell_grid(info->dims[0], info->dims[1], info->dims[2]), cell_block(), 0, as_stream(stream)>>>(
      *info, u, v, w, centers);
  return launch_status("center velocity");
}

extern "C" int plume_view_curl(const PlumeGridInfo* info, const float* centers, float* curl, void* stream) {
  VIEW_CHECK(info && centers && curl && centers != curl, "view_curl: bad argument");
  k_curl_centers<<<cell_grid(info->dims[0], info->dims[1], info->dims[2]), cell_block(), 0, as_stream(stream)>>>(
      *info, centers, curl);
  return launch_status("curl of centres");
}

extern "C" int plume_view_speed(const float* vectors, long long cells, float* out, void* stream) {
  VIEW_CHECK(vectors && out && cells >= 1, "view_speed: bad argument");
  k_speed<<<(int)((cells + 255) / 256), 256, 0, as_stream(stream)>>>(vectors, (long)cells, out);
  return launch_status("speed");
}

extern "C" int plume_view_slice(const PlumeViewParams* view, const PlumeGridInfo* info, int32_t axis,
                                float coordinate_m, const float* values, float low, float high, const float* ramp,
                                int32_t ramp_n, uint8_t* image, int32_t height, int32_t width, void* stream) {
  VIEW_CHECK(view && info && values && ramp && image && axis >= 0 && axis <= 2 && ramp_n >= 2 && height >= 1 &&
                 width >= 1,
             "view_slice: bad argument");
  dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
  k_slice<<<grid, block, 0, as_stream(stream)>>>(*view, *info, axis, coordinate_m, values, low, high, ramp, ramp_n,
                                                 image, height, width);
  return launch_status("slice");
}

extern "C" int plume_view_boundary_layers(const float* smoke, const int32_t shape[3], float* layers, void* stream) {
  VIEW_CHECK(smoke && shape && layers && shape[0] >= 1 && shape[1] >= 1 && shape[2] >= 1, "view_boundary_layers: bad argument");
  const Dims d{shape[0], shape[1], shape[2]};
  const int side = std::max(d.n0, std::max(d.n1, d.n2));
  const long n = 6L * side * side;
  k_boundary_layers<<<(int)((n + 255) / 256), 256, 0, as_stream(stream)>>>(smoke, d, side, layers);
  return launch_status("boundary layers");
}

extern "C" int plume_view_narrow(const float* src, void* dst, long long count, void* stream) {
  VIEW_CHECK(src && dst && count >= 0, "view_narrow: bad argument");
  if (count == 0) return PLUME_OK;
  if (count == 0) return PLUME_OK;
  k_narrow<<<(int)std::min<long long>((count + 255) / 256, 148 * 16), 256, 0, as_stream(stream)>>>(
      src, static_cast<__half*>(dst), (long)count);
  return launch_status("narrow");
}

extern "C" int plume_view_widen(const void* src, float* dst, long long count, void* stream) {
  VIEW_CHECK(src && dst && count >= 0, "view_widen: bad argument");
  if (count == 0) return PLUME_OK;
  if (count == 0) return PLUME_OK;
  k_widen<<<(int)std::min<long long>((count + 255) / 256, 148 * 16), 256, 0, as_stream(stream)>>>(
      static_cast<const __half*>(src), dst, (long)count);
  return launch_status("widen");
}
