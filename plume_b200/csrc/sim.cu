// Fluid-step kernels of libplume_b200.so for sm_100a, and their C ABI (include/plume_b200.h).
//
// Each kernel cites the Warp kernel(s) of chadmv/plume whose result it produces (paths relative to that
// project). Kernels are gathers with one thread per output element, so results never depend on scheduling;
// the only reduction (the smoke budget) adds in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "advect.cuh"
#include "poisson.cuh"

namespace plume {

static thread_local char g_error[512] = "";

int fail(int status, const char* fmt, ...) {
  va_list args;
  va_start(args, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, args);
  va_end(args);
  return status;
}

static unsigned long long g_launches = 0;  // kernels enqueued by this library (host-side count)
static thread_local bool g_counting = true;  // off while a graph is being captured (its replays are counted)

void count_launches(unsigned long long n) { __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED); }
void set_launch_counting(bool on) { g_counting = on; }

int launch_status(const char* what) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fail(PLUME_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(err));
  if (g_counting) count_launches(1);
  return PLUME_OK;
}

int runtime_status(const char* what, cudaError_t err) {
  if (err != cudaSuccess) return fail(PLUME_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(err));
  return PLUME_OK;
}

static bool valid_dims(const int* d) {
  if (d[0] < 1 || d[1] < 1 || d[2] < 1) return false;
  long long n = (long long)(d[0] + 1) * (d[1] + 1) * (d[2] + 1);
  return n < (1LL << 31);
}

#define CHECK_ARG(cond, ...) \
  do {                       \
    if (!(cond)) return fail(PLUME_ERR_INVALID, __VA_ARGS__); \
  } while (0)

#define CHECK_LAUNCH(what)                  \
  do {                                      \
    int _s = launch_status(what);           \
    if (_s != PLUME_OK) return _s;          \
  } while (0)

// ---- emitters: sim/emitters.py -----------------------------------------------------------------------------

struct EmitterSet {
  int count;
  PlumeEmitter e[PLUME_MAX_EMITTERS];
};

__device__ __forceinline__ F3 v3(const float* a) { return f3(a[0], a[1], a[2]); }

__device__ __forceinline__ float soft_edge(float distance, float extent, float softness) {  // emitters.py:41-50
  float inner = extent * (1.0f - softness);
  if (distance <= inner) return 1.0f;
  if (distance >= extent) return 0.0f;
  float t = (distance - inner) / (extent - inner);
  return 1.0f - t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ float coverage(const PlumeEmitter& e, F3 x, int seed) {  // emitters.py:53-67
  F3 offset = sub3(x, v3(e.center_m));
  float amount = 0.0f;
  if (e.shape == 0) {
    amount = soft_edge(len3(offset), e.radius_m, e.edge_softness);
  } else {
    amount = soft_edge(fabsf(offset[0]), e.half_size_m[0], e.edge_softness) *
             soft_edge(fabsf(offset[1]), e.half_size_m[1], e.edge_softness) *
             soft_edge(fabsf(offset[2]), e.half_size_m[2], e.edge_softness);
  }
  if (amount > 0.0f && e.noise_strength > 0.0f) {
    float breakup = 1.0f + e.noise_strength * value_noise(seed, e.stream, div3(x, e.noise_scale_m));
    amount = amount * fmax_(breakup, 0.0f);
  }
  return fmin_(amount, 1.0f);
}

__device__ __forceinline__ float blend_factor(float amount, float dt) {  // emitters.py:70-77
  const float reference = 1.0f / 80.0f;
  return 1.0f - pow_f(1.0f - amount, dt / reference);
}

__device__ __forceinline__ F3 world_position(const PlumeGridInfo& info, F3 index) {
  return add3(v3(info.origin_m), mul3(index, info.cell_m));
}

// emit_scalars_kernel (emitters.py:90-102) over the cells, then emit_velocity_kernel (:105-121) over the
// three face arrays, within a box of cells (`lo`, `n`) that contains every cell and face an active emitter can
// cover (coverage is 0 outside each emitter's reach). blockIdx.z segments: n[0] cell slices, then n[0]+1 u
// slices, n[0] v slices, n[0] w slices.
template <class T>
__global__ void k_emit(PlumeGridInfo info, T* __restrict__ smoke, T* __restrict__ temperature, T* __restrict__ u,
                       T* __restrict__ v, T* __restrict__ w, EmitterSet set, int seed, float time_s, float dt, int3 lo,
                       int3 n) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  int slab = blockIdx.z;
  int part = 0;
  if (slab >= n.x) { slab -= n.x; part = 1; }
  if (part == 1 && slab >= n.x + 1) { slab -= n.x + 1; part = 2; }
  if (part == 2 && slab >= n.x) { slab -= n.x; part = 3; }
  const int i = lo.x + slab;
  const int j = lo.y + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = lo.z + blockIdx.x * blockDim.x + threadIdx.x;
  if (part == 0) {
    if (i >= nx || j >= ny || k >= nz || j >= lo.y + n.y || k >= lo.z + n.z) return;
    F3 x = world_position(info, add3(f3((float)i, (float)j, (float)k), f3(0.5f, 0.5f, 0.5f)));
    const int c = (i * ny + j) * nz + k;
    for (int e_index = 0; e_index < set.count; ++e_index) {
      const PlumeEmitter& e = set.e[e_index];
      if (!(time_s >= e.start_s && time_s < e.end_s)) continue;
      float amount = coverage(e, x, seed);
      if (amount > 0.0f) {
        st_f(smoke + c, ld_f(smoke + c) + e.smoke_per_s * amount * dt);
        st_f(temperature + c, lerpf_(ld_f(temperature + c), e.temperature_k, blend_factor(amount, dt)));
      }
    }
    return;
  }
  const int axis = part - 1;
  T* comp = axis == 0 ? u : (axis == 1 ? v : w);
  const int n0 = nx + (axis == 0), n1 = ny + (axis == 1), n2 = nz + (axis == 2);
  if (i >= n0 || j >= n1 || k >= n2 || j > lo.y + n.y || k > lo.z + n.z) return;
  F3 offset = axis == 0 ? f3(0.0f, 0.5f, 0.5f) : (axis == 1 ? f3(0.5f, 0.0f, 0.5f) : f3(0.5f, 0.5f, 0.0f));
  F3 x = world_position(info, add3(f3((float)i, (float)j, (float)k), offset));
  const int c = (i * n1 + j) * n2 + k;
  for (int e_index = 0; e_index < set.count; ++e_index) {
    const PlumeEmitter& e = set.e[e_index];
    if (!(time_s >= e.start_s && time_s < e.end_s)) continue;
    float amount = coverage(e, x, seed);
    if (amount > 0.0f) {
      F3 target = v3(e.velocity_mps);
      if (e.outward == 1) {
        F3 away = sub3(x, v3(e.center_m));
        if (len3(away) > 0.0f) target = mul3(normalize3(away), len3(v3(e.velocity_mps)));
      }
      st_f(comp + c, lerpf_(ld_f(comp + c), target[axis], blend_factor(amount, dt)));
    }
  }
}

// The adjoint of k_emit for the temperature and velocity blends (no reference counterpart): each blend
// T = lerp(T, target, b) passes (1 - b) of the derivative back; the smoke's addition passes it unchanged. Same
// box and segments as k_emit.
__global__ void k_emit_adjoint(PlumeGridInfo info, float* __restrict__ a_temperature, float* __restrict__ a_u,
                               float* __restrict__ a_v, float* __restrict__ a_w, EmitterSet set, int seed, float time_s,
                               float dt, int3 lo, int3 n) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  int slab = blockIdx.z;
  int part = 0;
  if (slab >= n.x) { slab -= n.x; part = 1; }
  if (part == 1 && slab >= n.x + 1) { slab -= n.x + 1; part = 2; }
  if (part == 2 && slab >= n.x) { slab -= n.x; part = 3; }
  const int i = lo.x + slab;
  const int j = lo.y + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = lo.z + blockIdx.x * blockDim.x + threadIdx.x;
  F3 x;
  float* target;
  if (part == 0) {
    if (i >= nx || j >= ny || k >= nz || j >= lo.y + n.y || k >= lo.z + n.z) return;
    x = world_position(info, add3(f3((float)i, (float)j, (float)k), f3(0.5f, 0.5f, 0.5f)));
    target = a_temperature + (i * ny + j) * nz + k;
  } else {
    const int axis = part - 1;
    const int n0 = nx + (axis == 0), n1 = ny + (axis == 1), n2 = nz + (axis == 2);
    if (i >= n0 || j >= n1 || k >= n2 || j > lo.y + n.y || k > lo.z + n.z) return;
    const F3 offset = axis == 0 ? f3(0.0f, 0.5f, 0.5f) : (axis == 1 ? f3(0.5f, 0.0f, 0.5f) : f3(0.5f, 0.5f, 0.0f));
    x = world_position(info, add3(f3((float)i, (float)j, (float)k), offset));
    target = (axis == 0 ? a_u : (axis == 1 ? a_v : a_w)) + (i * n1 + j) * n2 + k;
  }
  float keep = 1.0f;
  for (int e_index = 0; e_index < set.count; ++e_index) {
    const PlumeEmitter& e = set.e[e_index];
    if (!(time_s >= e.start_s && time_s < e.end_s)) continue;
    const float amount = coverage(e, x, seed);
    if (amount > 0.0f) keep = keep * (1.0f - blend_factor(amount, dt));
  }
  if (keep != 1.0f) *target = *target * keep;
}

// The cells (inclusive index range per axis) that can lie within reach of the emitters, with a 2-cell margin
// for rounding; false when none is inside the grid.
static bool emitter_box(const PlumeGridInfo& info, const PlumeEmitter* e, int count, int lo[3], int hi[3]) {
  for (int a = 0; a < 3; ++a) {
    lo[a] = info.dims[a];
    hi[a] = -1;
  }
  for (int n = 0; n < count; ++n)
    for (int a = 0; a < 3; ++a) {
      const double reach = e[n].shape == 0 ? (double)e[n].radius_m : (double)e[n].half_size_m[a];
      const double first = ((double)e[n].center_m[a] - reach - (double)info.origin_m[a]) / (double)info.cell_m;
      const double last = ((double)e[n].center_m[a] + reach - (double)info.origin_m[a]) / (double)info.cell_m;
      lo[a] = std::min(lo[a], (int)std::max(-1.0, std::floor(first) - 2.0));
      hi[a] = std::max(hi[a], (int)std::min((double)info.dims[a] + 1.0, std::ceil(last) + 2.0));
    }
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::max(lo[a], 0);
    hi[a] = std::min(hi[a], info.dims[a] - 1);
    if (hi[a] < lo[a]) return false;
  }
  return true;
}

template <class T>
static int launch_emit(const PlumeGridInfo& info, T* smoke, T* temperature, T* u, T* v, T* w,
                       const PlumeEmitter* emitters, int count, int seed, float time_s, float dt, cudaStream_t st) {
  // Emitters inactive at time_s change nothing; skip them on the host (the kernel re-checks).
  std::vector<PlumeEmitter> active;
  for (int n = 0; n < count; ++n)
    if (time_s >= emitters[n].start_s && time_s < emitters[n].end_s) active.push_back(emitters[n]);
  for (size_t first = 0; first < active.size(); first += PLUME_MAX_EMITTERS) {
    EmitterSet set;
    set.count = (int)std::min<size_t>(PLUME_MAX_EMITTERS, active.size() - first);
    for (int n = 0; n < set.count; ++n) set.e[n] = active[first + n];
    int lo[3], hi[3];
    if (!emitter_box(info, set.e, set.count, lo, hi)) continue;
    const int3 box_lo = make_int3(lo[0], lo[1], lo[2]);
    const int3 box_n = make_int3(hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1);
    dim3 grid((box_n.z + 1 + TZ - 1) / TZ, (box_n.y + 1 + TY - 1) / TY, box_n.x + (box_n.x + 1) + box_n.x + box_n.x);
    k_emit<<<grid, cell_block(), 0, st>>>(info, smoke, temperature, u, v, w, set, seed, time_s, dt, box_lo, box_n);
    CHECK_LAUNCH("emit");
  }
  return PLUME_OK;
}

// ---- streaming kernels: several x-planes per thread -----------------------------------------------------
// The one-pass stencil kernels of the step (buoyancy, curl, push, face forces, divergence, gradient) handle
// PLANES x-planes per thread with every load issued before any store, so more bytes are in flight per SM than
// with one element per thread. Each element's arithmetic is unchanged. PLUME_STREAM_PLANES = 1, 2 or 4
// (default 4) selects the count.
static int stream_planes() {
  static const int n = [] {
    const char* v = getenv("PLUME_STREAM_PLANES");
    const int p = v ? atoi(v) : 4;
    return p == 1 || p == 2 ? p : 4;
  }();
  return n;
}

// Calls f(std::integral_constant<int, P>) with P the streaming kernels' planes per thread.
template <class F>
static int with_planes(F f) {
  switch (stream_planes()) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    default: return f(std::integral_constant<int, 4>{});
  }
}

static dim3 cell_grid_planes(int n0, int n1, int n2, int planes) {
  return dim3((n2 + TZ - 1) / TZ, (n1 + TY - 1) / TY, (n0 + planes - 1) / planes);
}

// ---- buoyancy: forces.py:13-23 -----------------------------------------------------------------------------
template <class T, int PLANES>
__global__ void k_buoyancy(PlumeGridInfo info, T* __restrict__ v, const T* __restrict__ smoke,
                           const T* __restrict__ temperature, float gravity, float heat_buoyancy, float smoke_weight,
                           float ambient, float dt) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i0 = blockIdx.z * PLANES, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > ny || k >= nz) return;
  const int below = imax_(j - 1, 0), above = imin_(j, ny - 1);
  const long cell_plane = (long)ny * nz, face_plane = (long)(ny + 1) * nz;
  float tb[PLANES], ta[PLANES], sb[PLANES], sa[PLANES], vv[PLANES];
#pragma unroll
  for (int p = 0; p < PLANES; ++p) {
    if (i0 + p >= nx) break;
    const long cb = (i0 + p) * cell_plane + below * nz + k, ca = (i0 + p) * cell_plane + above * nz + k;
    tb[p] = ldg_f(temperature + cb);
    ta[p] = ldg_f(temperature + ca);
    sb[p] = ldg_f(smoke + cb);
    sa[p] = ldg_f(smoke + ca);
    vv[p] = ld_f(v + (i0 + p) * face_plane + (long)j * nz + k);
  }
#pragma unroll
  for (int p = 0; p < PLANES; ++p) {
    if (i0 + p >= nx) break;
    float heat = 0.5f * (tb[p] + ta[p]);
    float density = 0.5f * (sb[p] + sa[p]);
    float lift = heat_buoyancy * (heat - ambient) / ambient - smoke_weight * density;
    st_f(v + (i0 + p) * face_plane + (long)j * nz + k, vv[p] + gravity * lift * dt);
  }
}

template <class T>
static int launch_buoyancy(const PlumeGridInfo& info, T* v, const T* smoke, const T* temperature, float gravity,
                           float heat_buoyancy, float smoke_weight, float ambient, float dt, cudaStream_t st) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  return with_planes([&](auto P) {
    constexpr int PL = decltype(P)::value;
    k_buoyancy<T, PL><<<cell_grid_planes(nx, ny + 1, nz, PL), cell_block(), 0, st>>>(
        info, v, smoke, temperature, gravity, heat_buoyancy, smoke_weight, ambient, dt);
    return launch_status("buoyancy");
  });
}

// ---- vorticity confinement: vorticity.py:17-84 -------------------------------------------------------------
template <class T>
__device__ __forceinline__ F3 center_velocity(const VelT<T>& vel, int i, int j, int k) {  // vorticity.py:17-22
  return f3(0.5f * (ldg_f(vel.u + at(vel.du, i, j, k)) + ldg_f(vel.u + at(vel.du, i + 1, j, k))),
            0.5f * (ldg_f(vel.v + at(vel.dv, i, j, k)) + ldg_f(vel.v + at(vel.dv, i, j + 1, k))),
            0.5f * (ldg_f(vel.w + at(vel.dw, i, j, k)) + ldg_f(vel.w + at(vel.dw, i, j, k + 1))));
}

// curl_kernel (vorticity.py:38-45) with the centre velocities of center_velocity_kernel computed in place.
// With `spin` (the step's scratch), |curl| of the cell is stored as well, computed as push_at would compute it
// from the stored components (the same floats), so the push reads one value per neighbour instead of three and
// a square root.
template <class T>
__device__ __forceinline__ void curl_at(const PlumeGridInfo& info, const VelT<T>& vel, float* __restrict__ cx,
                                        float* __restrict__ cy, float* __restrict__ cz, float* __restrict__ spin,
                                        int i, int j, int k) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int cell[3] = {i, j, k};
  const int n[3] = {nx, ny, nz};
  F3 d[3];
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {  // central_difference (vorticity.py:25-35)
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[axis] = imax_(cell[axis] - 1, 0);
    hi[axis] = imin_(cell[axis] + 1, n[axis] - 1);
    float span = (float)(hi[axis] - lo[axis]);
    if (span == 0.0f) {
      d[axis] = f3(0.0f, 0.0f, 0.0f);
    } else {
      d[axis] = divide3(sub3(center_velocity(vel, hi[0], hi[1], hi[2]), center_velocity(vel, lo[0], lo[1], lo[2])),
                        divisor(span * info.cell_m));
    }
  }
  const int c = (i * ny + j) * nz + k;
  const F3 curl = f3(d[1][2] - d[2][1], d[2][0] - d[0][2], d[0][1] - d[1][0]);
  cx[c] = curl[0];
  cy[c] = curl[1];
  cz[c] = curl[2];
  if (spin) spin[c] = len3(curl);
}

template <class T, int PLANES>
__global__ void k_curl(PlumeGridInfo info, VelT<T> vel, float* __restrict__ cx, float* __restrict__ cy,
                       float* __restrict__ cz, float* __restrict__ spin) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i0 = blockIdx.z * PLANES, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny || k >= nz) return;
#pragma unroll
  for (int p = 0; p < PLANES; ++p)
    if (i0 + p < nx) curl_at(info, vel, cx, cy, cz, spin, i0 + p, j, k);
}

__device__ __forceinline__ F3 load3(const float* __restrict__ x, const float* __restrict__ y,
                                    const float* __restrict__ z, int c) {
  return f3(__ldg(x + c), __ldg(y + c), __ldg(z + c));
}

// confinement_push_kernel (vorticity.py:53-71); SPIN: |curl| read from k_curl's `spin` array.
template <bool SPIN>
__device__ __forceinline__ void push_at(const PlumeGridInfo& info, const float* __restrict__ cx,
                                        const float* __restrict__ cy, const float* __restrict__ cz,
                                        const float* __restrict__ spin, float* __restrict__ px,
                                        float* __restrict__ py, float* __restrict__ pz, float strength, int i, int j,
                                        int k) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const Dims d{nx, ny, nz};
  const int cell[3] = {i, j, k};
  const int n[3] = {nx, ny, nz};
  F3 toward = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[axis] = imax_(cell[axis] - 1, 0);
    hi[axis] = imin_(cell[axis] + 1, n[axis] - 1);
    float span = (float)(hi[axis] - lo[axis]);
    if (span > 0.0f) {
      const int at_hi = at(d, hi[0], hi[1], hi[2]), at_lo = at(d, lo[0], lo[1], lo[2]);
      float spin_hi = SPIN ? __ldg(spin + at_hi) : len3(load3(cx, cy, cz, at_hi));
      float spin_lo = SPIN ? __ldg(spin + at_lo) : len3(load3(cx, cy, cz, at_lo));
      toward[axis] = divide(spin_hi - spin_lo, divisor(span * info.cell_m));
    }
  }
  const int c = at(d, i, j, k);
  float length = len3(toward);
  if (length < 1.0e-12f) {
    px[c] = 0.0f;
    py[c] = 0.0f;
    pz[c] = 0.0f;
    return;
  }
  F3 push = mul3(cross3(div3(toward, length), load3(cx, cy, cz, c)), strength * info.cell_m);
  px[c] = push[0];
  py[c] = push[1];
  pz[c] = push[2];
}

// push_at from values loaded beforehand: the spin of the two neighbours on each axis (clamped) and the curl.
__device__ __forceinline__ F3 push_from(const PlumeGridInfo& info, int i, int j, int k, const float* spin_lo,
                                        const float* spin_hi, F3 curl, float strength) {
  const int cell[3] = {i, j, k};
  const int n[3] = {info.dims[0], info.dims[1], info.dims[2]};
  F3 toward = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    const int lo = imax_(cell[axis] - 1, 0), hi = imin_(cell[axis] + 1, n[axis] - 1);
    float span = (float)(hi - lo);
    if (span > 0.0f) toward[axis] = divide(spin_hi[axis] - spin_lo[axis], divisor(span * info.cell_m));
  }
  float length = len3(toward);
  if (length < 1.0e-12f) return f3(0.0f, 0.0f, 0.0f);
  return mul3(cross3(div3(toward, length), curl), strength * info.cell_m);
}

template <int PLANES, bool SPIN>
__global__ void k_push(PlumeGridInfo info, const float* __restrict__ cx, const float* __restrict__ cy,
                       const float* __restrict__ cz, const float* __restrict__ spin, float* __restrict__ px,
                       float* __restrict__ py, float* __restrict__ pz, float strength) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i0 = blockIdx.z * PLANES, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny || k >= nz) return;
  if constexpr (SPIN) {
    // every plane's spins and curl loaded before any push is stored (the loads do not wait on the stores)
    const Dims d{nx, ny, nz};
    float lo[PLANES][3], hi[PLANES][3];
    F3 curl[PLANES];
#pragma unroll
    for (int p = 0; p < PLANES; ++p) {
      const int i = imin_(i0 + p, nx - 1);
      lo[p][0] = __ldg(spin + at(d, imax_(i - 1, 0), j, k));
      hi[p][0] = __ldg(spin + at(d, imin_(i + 1, nx - 1), j, k));
      lo[p][1] = __ldg(spin + at(d, i, imax_(j - 1, 0), k));
      hi[p][1] = __ldg(spin + at(d, i, imin_(j + 1, ny - 1), k));
      lo[p][2] = __ldg(spin + at(d, i, j, imax_(k - 1, 0)));
      hi[p][2] = __ldg(spin + at(d, i, j, imin_(k + 1, nz - 1)));
      curl[p] = load3(cx, cy, cz, at(d, i, j, k));
    }
#pragma unroll
    for (int p = 0; p < PLANES; ++p) {
      if (i0 + p >= nx) break;
      const F3 push = push_from(info, i0 + p, j, k, lo[p], hi[p], curl[p], strength);
      const int c = at(d, i0 + p, j, k);
      px[c] = push[0];
      py[c] = push[1];
      pz[c] = push[2];
    }
  } else {
#pragma unroll
    for (int p = 0; p < PLANES; ++p)
      if (i0 + p < nx) push_at<SPIN>(info, cx, cy, cz, spin, px, py, pz, strength, i0 + p, j, k);
  }
}

// ---- turbulence: turbulence.py:26-53 -----------------------------------------------------------------------
constexpr int TURBULENCE_STREAM = 1 << 24;

__device__ __forceinline__ float potential(int seed, int component, F3 p, float pattern_time) {
  float slice_lo = floorf(pattern_time);
  float blend = fade(pattern_time - slice_lo);
  int first = TURBULENCE_STREAM + 3 * (int)slice_lo + component;
  return lerpf_(value_noise(seed, first, p), value_noise(seed, first + 3, p), blend);
}

struct FaceForces {
  int confinement;  // add the averaged push (add_face_push_kernel, vorticity.py:74-84)
  const float* push[3];
  int turbulence;   // turbulence_kernel (turbulence.py:35-53)
  int seed;
  float scale_m, strength, pattern_time;
  int drag;         // drag_kernel (forces.py:34-37)
  float wind[3];
  float keep;
  float dt;
};

// One pass over the three face arrays applying, per face and in the reference's order, the confinement push,
// the turbulence push and drag. blockIdx.z segments: nx+1 u slices, nx v slices, nx w slices.
// The push of the two cells beside face (i, j, k) along AXIS (add_face_push_kernel's neighbours, clamped).
template <int AXIS>
__device__ __forceinline__ void face_push_pair(const PlumeGridInfo& info, int i, int j, int k, const FaceForces& ff,
                                               float& below, float& above) {
  const int index = AXIS == 0 ? i : (AXIS == 1 ? j : k);
  const int lo = imax_(index - 1, 0), hi = imin_(index, info.dims[AXIS] - 1);
  const Dims d{info.dims[0], info.dims[1], info.dims[2]};
  const int at_lo = AXIS == 0 ? at(d, lo, j, k) : (AXIS == 1 ? at(d, i, lo, k) : at(d, i, j, lo));
  const int at_hi = AXIS == 0 ? at(d, hi, j, k) : (AXIS == 1 ? at(d, i, hi, k) : at(d, i, j, hi));
  below = __ldg(ff.push[AXIS] + at_lo);
  above = __ldg(ff.push[AXIS] + at_hi);
}

// `below` and `above`: the face's face_push_pair (read only with the confinement push).
template <int AXIS>
__device__ __forceinline__ float face_forces_value(const PlumeGridInfo& info, float value, int i, int j, int k,
                                                   const FaceForces& ff, float below, float above) {
  if (ff.confinement) {
    float average = 0.5f * (below + above);
    value = value + average * ff.dt;
  }
  if (ff.turbulence) {
    const F3 offset = AXIS == 0 ? f3(0.0f, 0.5f, 0.5f) : (AXIS == 1 ? f3(0.5f, 0.0f, 0.5f) : f3(0.5f, 0.5f, 0.0f));
    const F3 face = add3(f3((float)i, (float)j, (float)k), offset);
    constexpr int B = (AXIS + 1) % 3, C = (AXIS + 2) % 3;
    const F3 half_b = f3(B == 0 ? 0.5f : 0.0f, B == 1 ? 0.5f : 0.0f, B == 2 ? 0.5f : 0.0f);
    const F3 half_c = f3(C == 0 ? 0.5f : 0.0f, C == 1 ? 0.5f : 0.0f, C == 2 ? 0.5f : 0.0f);
    float to_lattice = info.cell_m / ff.scale_m;
    float c_plus = potential(ff.seed, C, mul3(add3(face, half_b), to_lattice), ff.pattern_time);
    float c_minus = potential(ff.seed, C, mul3(sub3(face, half_b), to_lattice), ff.pattern_time);
    float b_plus = potential(ff.seed, B, mul3(add3(face, half_c), to_lattice), ff.pattern_time);
    float b_minus = potential(ff.seed, B, mul3(sub3(face, half_c), to_lattice), ff.pattern_time);
    float curl = ((c_plus - c_minus) - (b_plus - b_minus)) / to_lattice;
    value = value + ff.strength * curl * ff.dt;
  }
  if (ff.drag) value = ff.wind[AXIS] + (value - ff.wind[AXIS]) * ff.keep;
  return value;
}

// The face kernels' blockIdx.z: groups of PLANES x-planes of u (nx + 1 planes), then of v, then of w.
template <int PLANES>
__device__ __forceinline__ void face_planes(const PlumeGridInfo& info, int& axis, int& i0) {
  const int nx = info.dims[0];
  const int gu = (nx + 1 + PLANES - 1) / PLANES, gv = (nx + PLANES - 1) / PLANES;
  int z = blockIdx.z;
  axis = 0;
  if (z >= gu) {
    z -= gu;
    axis = 1;
    if (z >= gv) {
      z -= gv;
      axis = 2;
    }
  }
  i0 = z * PLANES;
}

static dim3 face_grid(const PlumeGridInfo& info, int planes) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  return dim3((nz + 1 + TZ - 1) / TZ, (ny + 1 + TY - 1) / TY,
              (nx + 1 + planes - 1) / planes + 2 * ((nx + planes - 1) / planes));
}

// confinement push, turbulence and drag on PLANES faces per thread, every face loaded before any is stored
template <int AXIS, int PLANES, class T>
__device__ __forceinline__ void face_forces_planes(const PlumeGridInfo& info, T* __restrict__ f, int i0, int j, int k,
                                                   const FaceForces& ff) {
  const Dims d = {info.dims[0] + (AXIS == 0), info.dims[1] + (AXIS == 1), info.dims[2] + (AXIS == 2)};
  if (j >= d.n1 || k >= d.n2) return;
  const long plane = (long)d.n1 * d.n2, at_jk = (long)j * d.n2 + k;
  float value[PLANES], below[PLANES] = {}, above[PLANES] = {};
#pragma unroll
  for (int p = 0; p < PLANES; ++p)  // every face and push value loaded before any face is stored
    if (i0 + p < d.n0) {
      value[p] = ld_f(f + (i0 + p) * plane + at_jk);
      if (ff.confinement) face_push_pair<AXIS>(info, i0 + p, j, k, ff, below[p], above[p]);
    }
#pragma unroll
  for (int p = 0; p < PLANES; ++p)
    if (i0 + p < d.n0)
      st_f(f + (i0 + p) * plane + at_jk, face_forces_value<AXIS>(info, value[p], i0 + p, j, k, ff, below[p], above[p]));
}

template <class T, int PLANES>
__global__ void k_face_forces(PlumeGridInfo info, T* __restrict__ u, T* __restrict__ v, T* __restrict__ w,
                              FaceForces ff) {
  int axis, i0;
  face_planes<PLANES>(info, axis, i0);
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (axis == 0) face_forces_planes<0, PLANES>(info, u, i0, j, k, ff);
  else if (axis == 1) face_forces_planes<1, PLANES>(info, v, i0, j, k, ff);
  else face_forces_planes<2, PLANES>(info, w, i0, j, k, ff);
}

template <class T>
static int launch_face_forces(const PlumeGridInfo& info, T* u, T* v, T* w, const FaceForces& ff, const char* what,
                              cudaStream_t st) {
  return with_planes([&](auto P) {
    constexpr int PL = decltype(P)::value;
    k_face_forces<T, PL><<<face_grid(info, PL), cell_block(), 0, st>>>(info, u, v, w, ff);
    return launch_status(what);
  });
}

// `spin`, when given, is nx*ny*nz floats of scratch for |curl| (the step passes its divergence array, which
// the projection overwrites later).
template <class T>
static int launch_confinement_push(const PlumeGridInfo& info, const T* u, const T* v, const T* w,
                                   float* const curl[3], float* const push[3], float strength, int apply,
                                   cudaStream_t st, float* spin = nullptr) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  VelT<T> vel = make_vel(u, v, w, info.dims);
  if (!apply) spin = nullptr;
  return with_planes([&](auto P) {
    constexpr int PL = decltype(P)::value;
    const dim3 grid = cell_grid_planes(nx, ny, nz, PL);
    k_curl<T, PL><<<grid, cell_block(), 0, st>>>(info, vel, curl[0], curl[1], curl[2], spin);
    CHECK_LAUNCH("curl");
    if (!apply) return PLUME_OK;
    if (spin)
      k_push<PL, true><<<grid, cell_block(), 0, st>>>(info, curl[0], curl[1], curl[2], spin, push[0], push[1],
                                                      push[2], strength);
    else
      k_push<PL, false><<<grid, cell_block(), 0, st>>>(info, curl[0], curl[1], curl[2], nullptr, push[0], push[1],
                                                       push[2], strength);
    return launch_status("confinement push");
  });
}

// ---- advection: advect.py -----------------------------------------------------------------------------------
//
// Every trace starts at a sample position p = index + offset, where each velocity component's trilinear
// weights are 0 or 1/2: velocity_at_node blends only the corners with a non-zero weight (6 to 9 loads instead
// of 24; the same values, up to the sign of a zero). The forward and backward traces of one element share
// that first sample, and fields with the same positions (smoke and temperature) share whole traces.

// Up to two fields sampled at the same positions (same shape and offset, e.g. smoke and temperature).
// `range`, when set, holds per element the (lo, hi) clamp bounds the forward pass found (two values of the
// storage type: the bounds are stored values, so they keep every bit), so the correction does not trace
// forward a second time.
template <class T>
struct FieldDesc {
  const T* data[2];
  T* hat[2];
  T* next[2];
  pair_t<T>* range[2];
  float outside[2];
  int fields;
  Dims d;
  F3 offset;
  int uses_outside;
};

// Up to three groups (the three velocity components) in one launch (blockIdx.z segments).
template <class T>
struct FieldSet {
  FieldDesc<T> f[3];
  int count;
};

// Where a launch's groups sit on the MAC grid, when the host can tell (layout_of): on the velocity
// components' faces, group g holding component g, or on cell centres. The first velocity sample of every trace
// is then formed from its corners with the weights known in advance: 1/2 between two corners, and one corner
// alone where the clamp meets a wall (only along the axis in which the sample sits half a cell from the
// element). The float operations and their order are velocity_at_node's, so the values are the same.
enum AdvectLayout { LAYOUT_ANY = 0, LAYOUT_FACES = 1, LAYOUT_CELLS = 2 };

template <int G>
struct GroupIndex {
  static constexpr int value = G;
};

// velocity_at_node (sample.py:74-82 at p = index + offset) for element (i, j, k) of group G.
template <int LAYOUT, int G, class T>
__device__ __forceinline__ F3 node_velocity(const VelT<T>& vel, int i, int j, int k, F3 p) {
  if constexpr (LAYOUT == LAYOUT_ANY) {
    return velocity_at_node(vel, p);
  } else if constexpr (LAYOUT == LAYOUT_CELLS) {  // p = (i + 1/2, j + 1/2, k + 1/2): u, v, w halfway along x, y, z
    const T* u = vel.u + at(vel.du, i, j, k);
    const T* v = vel.v + at(vel.dv, i, j, k);
    const T* w = vel.w + at(vel.dw, i, j, k);
    return f3(lerpf_(ldg_f(u), ldg_f(u + vel.du.n1 * vel.du.n2), 0.5f), lerpf_(ldg_f(v), ldg_f(v + vel.dv.n2), 0.5f),
              lerpf_(ldg_f(w), ldg_f(w + 1), 0.5f));
  } else if constexpr (G == 0) {  // a u face, p = (i, j + 1/2, k + 1/2): v and w halfway along x except at the walls
    const int nx = vel.dv.n0, i0 = imax_(i - 1, 0);
    const bool wall = i == 0 || i == nx;
    const int sv = vel.dv.n1 * vel.dv.n2, sw = vel.dw.n1 * vel.dw.n2;
    auto along_x = [&](const T* q, int s) { return wall ? ldg_f(q) : lerpf_(ldg_f(q), ldg_f(q + s), 0.5f); };
    const T* v = vel.v + at(vel.dv, i0, j, k);
    const T* w = vel.w + at(vel.dw, i0, j, k);
    return f3(ldg_f(vel.u + at(vel.du, i, j, k)), lerpf_(along_x(v, sv), along_x(v + vel.dv.n2, sv), 0.5f),
              lerpf_(along_x(w, sw), along_x(w + 1, sw), 0.5f));
  } else if constexpr (G == 1) {  // a v face, p = (i + 1/2, j, k + 1/2): u and w halfway along y except at the walls
    const int ny = vel.du.n1, j0 = imax_(j - 1, 0);
    const bool wall = j == 0 || j == ny;
    const int su = vel.du.n1 * vel.du.n2;
    const T* u = vel.u + at(vel.du, i, j0, k);
    const T* w = vel.w + at(vel.dw, i, j0, k);
    auto u_x = [&](const T* q) { return lerpf_(ldg_f(q), ldg_f(q + su), 0.5f); };
    const float u_lo = u_x(u);
    const float u_at = wall ? u_lo : lerpf_(u_lo, u_x(u + vel.du.n2), 0.5f);
    auto w_y = [&](const T* q) { return wall ? ldg_f(q) : lerpf_(ldg_f(q), ldg_f(q + vel.dw.n2), 0.5f); };
    return f3(u_at, ldg_f(vel.v + at(vel.dv, i, j, k)), lerpf_(w_y(w), w_y(w + 1), 0.5f));
  } else {  // a w face, p = (i + 1/2, j + 1/2, k): u and v halfway along z except at the walls
    const int nz = vel.du.n2, k0 = imax_(k - 1, 0);
    const bool wall = k == 0 || k == nz;
    const int su = vel.du.n1 * vel.du.n2;
    const T* u = vel.u + at(vel.du, i, j, k0);
    const T* v = vel.v + at(vel.dv, i, j, k0);
    auto u_x = [&](const T* q) { return lerpf_(ldg_f(q), ldg_f(q + su), 0.5f); };
    auto v_y = [&](const T* q) { return lerpf_(ldg_f(q), ldg_f(q + vel.dv.n2), 0.5f); };
    const float u_lo = u_x(u), v_lo = v_y(v);
    return f3(wall ? u_lo : lerpf_(u_lo, u_x(u + 1), 0.5f), wall ? v_lo : lerpf_(v_lo, v_y(v + 1), 0.5f),
              ldg_f(vel.w + at(vel.dw, i, j, k)));
  }
}

// semi_lagrangian_kernel (advect.py:24-31): the forward pass into `hat` (or, for plain semi-Lagrangian
// advection, into `next`).
// Calls body(group, slab, GroupIndex<g>) with the group of `set` that blockIdx.z falls in, as a constant index
// into the kernel parameters (each group's body is compiled on its own, with its descriptor at fixed parameter
// offsets).
template <class T, class Body>
__device__ __forceinline__ void for_group(const FieldSet<T>& set, Body body) {
  int slab = blockIdx.z;
  if (slab < set.f[0].d.n0 || set.count == 1) return body(set.f[0], slab, GroupIndex<0>{});
  slab -= set.f[0].d.n0;
  if (slab < set.f[1].d.n0 || set.count == 2) return body(set.f[1], slab, GroupIndex<1>{});
  body(set.f[2], slab - set.f[1].d.n0, GroupIndex<2>{});
}

// FIELDS: the group's field count when fixed at compile time, 0 to read it from the descriptor.
template <int FIELDS, int LAYOUT, int G, class T>
__device__ __forceinline__ void advect_forward_at(const PlumeGridInfo& info, const VelT<T>& vel, const FieldDesc<T>& fd,
                                                  int slab, float dt_over_cell, int write_next) {
  const int i = slab, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= fd.d.n1 || k >= fd.d.n2) return;
  const int c = at(fd.d, i, j, k);
  const F3 p = add3(f3((float)i, (float)j, (float)k), fd.offset);
  const F3 src = trace_from(vel, p, node_velocity<LAYOUT, G>(vel, i, j, k, p), dt_over_cell);
  const bool outside = fd.uses_outside == 1 && is_outside_open_face(src, info);
  const F3 g = sub3(src, fd.offset);
  // every field sampled before any result is stored: the second field's loads do not wait on the first's stores
  constexpr int MAXF = FIELDS ? FIELDS : 2;
  const int count = FIELDS ? FIELDS : fd.fields;
  float value[MAXF], lo[MAXF], hi[MAXF];
#pragma unroll
  for (int n = 0; n < MAXF; ++n) {
    if (n >= count) break;
    value[n] = lo[n] = hi[n] = fd.outside[n];
    if (!outside) value[n] = sample_with_range(fd.data[n], fd.d, g, lo[n], hi[n]);
  }
#pragma unroll
  for (int n = 0; n < MAXF; ++n) {
    if (n >= count) break;
    st_f((write_next ? fd.next[n] : fd.hat[n]) + c, value[n]);
    if (fd.range[n]) fd.range[n][c] = make_pair_t<T>(lo[n], hi[n]);
  }
}

// FIELDS: every group of the launch holds this many fields (1: the velocity components, 2: smoke and
// temperature), a count the compiler then knows; 0 reads each group's count. Measured on B200, as kernels of
// their own: velocity advection -3.5%, scalar advection -4%.
// LAYOUT: an AdvectLayout the host found for every group of the launch.
// 32 registers (8 blocks of 256 a SM): without the bound the shared velocity axes take 40-43 and the lower
// occupancy costs more than the sharing saves. Measured on B200 with the bound: velocity advection -2.2%.
template <class T, int FIELDS, int LAYOUT>
__global__ void __launch_bounds__(256, 8) k_advect_forward(PlumeGridInfo info, VelT<T> vel, FieldSet<T> set, float dt_over_cell, int write_next) {
  for_group(set, [&](const FieldDesc<T>& fd, int slab, auto group) {
    advect_forward_at<FIELDS, LAYOUT, decltype(group)::value>(info, vel, fd, slab, dt_over_cell, write_next);
  });
}

// maccormack_correct_kernel (advect.py:34-50) with the backward pass (advect.py:64) evaluated in place:
// back = sample(hat, trace(p, -dt)), corrected = hat + (data - back) / 2, clamped to the range of the eight
// values the forward sample blended.
template <int FIELDS, int LAYOUT, int G, class T, bool STORED_RANGE>
__device__ __forceinline__ void advect_correct_at(const PlumeGridInfo& info, const VelT<T>& vel, const FieldDesc<T>& fd,
                                                  int slab, float dt_over_cell) {
  const int i = slab, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= fd.d.n1 || k >= fd.d.n2) return;
  const int c = at(fd.d, i, j, k);
  const F3 p = add3(f3((float)i, (float)j, (float)k), fd.offset);
  const F3 vp = node_velocity<LAYOUT, G>(vel, i, j, k, p);
  const F3 back_src = trace_from(vel, p, vp, -dt_over_cell);
  const bool back_outside = fd.uses_outside == 1 && is_outside_open_face(back_src, info);
  const F3 gb = sub3(back_src, fd.offset);
  F3 gs = f3(0.0f, 0.0f, 0.0f);
  bool source_outside = false;
  if (!STORED_RANGE) {
    const F3 source = trace_from(vel, p, vp, dt_over_cell);
    source_outside = fd.uses_outside == 1 && is_outside_open_face(source, info);
    gs = sub3(source, fd.offset);
  }
  // every field corrected before any is stored: the second field's loads do not wait on the first's store
  constexpr int MAXF = FIELDS ? FIELDS : 2;
  const int count = FIELDS ? FIELDS : fd.fields;
  float result[MAXF];
#pragma unroll
  for (int n = 0; n < MAXF; ++n) {
    if (n >= count) break;
    const float back = back_outside ? fd.outside[n] : sample_index_space(fd.hat[n], fd.d, gb);
    const float corrected = ldg_f(fd.hat[n] + c) + 0.5f * (ldg_f(fd.data[n] + c) - back);
    float lo = fd.outside[n], hi = fd.outside[n];
    if (STORED_RANGE) {
      const pair_t<T> r = fd.range[n][c];
      lo = to_f<T>(r.x);
      hi = to_f<T>(r.y);
    } else if (!source_outside) {
      sample_with_range(fd.data[n], fd.d, gs, lo, hi);
    }
    result[n] = clampf_(corrected, lo, hi);
  }
#pragma unroll
  for (int n = 0; n < MAXF; ++n) {
    if (n >= count) break;
    st_f(fd.next[n] + c, result[n]);
  }
}

// With a stored range, 32 registers as in the forward pass. Tracing forward again needs more: it spills at 32
// and at 40, so those forms get 48.
template <class T, bool STORED_RANGE, int FIELDS, int LAYOUT>
__global__ void __launch_bounds__(256, STORED_RANGE ? 8 : 5) k_advect_correct(PlumeGridInfo info, VelT<T> vel, FieldSet<T> set, float dt_over_cell) {
  for_group(set, [&](const FieldDesc<T>& fd, int slab, auto group) {
    advect_correct_at<FIELDS, LAYOUT, decltype(group)::value, T, STORED_RANGE>(info, vel, fd, slab, dt_over_cell);
  });
}

// The AdvectLayout of a launch: LAYOUT_FACES when its three groups are the velocity components' faces in
// order, LAYOUT_CELLS when every group sits at the cell centres, LAYOUT_ANY otherwise.
template <class T>
static int layout_of(const PlumeGridInfo& info, const FieldSet<T>& set) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  auto is = [](const FieldDesc<T>& f, Dims d, float ox, float oy, float oz) {
    return f.d.n0 == d.n0 && f.d.n1 == d.n1 && f.d.n2 == d.n2 && f.offset[0] == ox && f.offset[1] == oy &&
           f.offset[2] == oz;
  };
  if (set.count == 3 && is(set.f[0], Dims{nx + 1, ny, nz}, 0.0f, 0.5f, 0.5f) &&
      is(set.f[1], Dims{nx, ny + 1, nz}, 0.5f, 0.0f, 0.5f) && is(set.f[2], Dims{nx, ny, nz + 1}, 0.5f, 0.5f, 0.0f))
    return LAYOUT_FACES;
  for (int n = 0; n < set.count; ++n)
    if (!is(set.f[n], Dims{nx, ny, nz}, 0.5f, 0.5f, 0.5f)) return LAYOUT_ANY;
  return LAYOUT_CELLS;
}

// The compiled forms: the velocity components on their faces (one field a group), smoke and temperature or a
// single scalar at the cell centres, and the general kernels for any other launch.
template <class T>
using ForwardKernel = void (*)(PlumeGridInfo, VelT<T>, FieldSet<T>, float, int);
template <class T>
using CorrectKernel = void (*)(PlumeGridInfo, VelT<T>, FieldSet<T>, float);

template <class T>
static ForwardKernel<T> forward_kernel(int fields, int layout) {
  if (layout == LAYOUT_FACES && fields == 1) return k_advect_forward<T, 1, LAYOUT_FACES>;
  if (layout == LAYOUT_CELLS && fields == 1) return k_advect_forward<T, 1, LAYOUT_CELLS>;
  if (layout == LAYOUT_CELLS && fields == 2) return k_advect_forward<T, 2, LAYOUT_CELLS>;
  return fields == 1 ? k_advect_forward<T, 1, LAYOUT_ANY>
                     : (fields == 2 ? k_advect_forward<T, 2, LAYOUT_ANY> : k_advect_forward<T, 0, LAYOUT_ANY>);
}

template <class T, bool STORED_RANGE>
static CorrectKernel<T> correct_kernel(int fields, int layout) {
  if (layout == LAYOUT_FACES && fields == 1) return k_advect_correct<T, STORED_RANGE, 1, LAYOUT_FACES>;
  if (layout == LAYOUT_CELLS && fields == 1) return k_advect_correct<T, STORED_RANGE, 1, LAYOUT_CELLS>;
  if (layout == LAYOUT_CELLS && fields == 2) return k_advect_correct<T, STORED_RANGE, 2, LAYOUT_CELLS>;
  return fields == 1 ? k_advect_correct<T, STORED_RANGE, 1, LAYOUT_ANY>
                     : (fields == 2 ? k_advect_correct<T, STORED_RANGE, 2, LAYOUT_ANY>
                                    : k_advect_correct<T, STORED_RANGE, 0, LAYOUT_ANY>);
}

template <class T>
static int launch_advect(const PlumeGridInfo& info, const VelT<T>& vel, const FieldSet<T>& set, float dt_over_cell,
                         bool maccormack, cudaStream_t st) {
  int slabs = 0, n1 = 0, n2 = 0;
  for (int n = 0; n < set.count; ++n) {
    slabs += set.f[n].d.n0;
    n1 = std::max(n1, set.f[n].d.n1);
    n2 = std::max(n2, set.f[n].d.n2);
  }
  dim3 grid((n2 + TZ - 1) / TZ, (n1 + TY - 1) / TY, slabs);
  int fields = set.f[0].fields;  // the groups' common field count, or 0 when they differ
  for (int n = 1; n < set.count; ++n)
    if (set.f[n].fields != fields) fields = 0;
  const int layout = layout_of(info, set);
  const ForwardKernel<T> forward = forward_kernel<T>(fields, layout);
  if (!maccormack) {
    forward<<<grid, cell_block(), 0, st>>>(info, vel, set, dt_over_cell, 1);
    CHECK_LAUNCH("semi-Lagrangian advection");
    return PLUME_OK;
  }
  forward<<<grid, cell_block(), 0, st>>>(info, vel, set, dt_over_cell, 0);
  CHECK_LAUNCH("MacCormack forward pass");
  const CorrectKernel<T> correct =
      set.f[0].range[0] ? correct_kernel<T, true>(fields, layout) : correct_kernel<T, false>(fields, layout);
  correct<<<grid, cell_block(), 0, st>>>(info, vel, set, dt_over_cell);
  CHECK_LAUNCH("MacCormack correction");
  return PLUME_OK;
}

template <class T>
static FieldDesc<T> single_field(const T* data, T* hat, T* next, Dims d, F3 offset, float outside, int uses_outside) {
  FieldDesc<T> f{};
  f.data[0] = data;
  f.hat[0] = hat;
  f.next[0] = next;
  f.outside[0] = outside;
  f.fields = 1;
  f.d = d;
  f.offset = offset;
  f.uses_outside = uses_outside;
  return f;
}

// ---- pressure: pressure.py ----------------------------------------------------------------------------------

// zero_closed_faces_kernel (pressure.py:21-28) on the two boundary planes of each face array.
template <class T>
__global__ void k_zero_walls(PlumeGridInfo info, T* __restrict__ u, T* __restrict__ v, T* __restrict__ w) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int axis = blockIdx.z / 2, side = blockIdx.z % 2;
  const bool closed = side == 0 ? info.open_lo[axis] == 0 : info.open_hi[axis] == 0;
  if (!closed) return;
  const int a = blockIdx.y * blockDim.y + threadIdx.y, b = blockIdx.x * blockDim.x + threadIdx.x;
  const int plane = side == 0 ? 0 : info.dims[axis];
  if (axis == 0) {
    if (a < ny && b < nz) st_f(u + (plane * ny + a) * nz + b, 0.0f);
  } else if (axis == 1) {
    if (a < nx && b < nz) st_f(v + (a * (ny + 1) + plane) * nz + b, 0.0f);
  } else {
    if (a < nx && b < ny) st_f(w + (a * ny + b) * (nz + 1) + plane, 0.0f);
  }
}

template <class T, int PLANES>
__global__ void k_divergence(PlumeGridInfo info, const T* __restrict__ u, const T* __restrict__ v,
                             const T* __restrict__ w, float* __restrict__ div) {  // pressure.py:31-36
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int i0 = blockIdx.z * PLANES, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny || k >= nz) return;
#pragma unroll
  for (int p = 0; p < PLANES; ++p) {
    const int i = i0 + p;
    if (i >= nx) break;
    float flux = (ldg_f(u + ((i + 1) * ny + j) * nz + k) - ldg_f(u + (i * ny + j) * nz + k)) +
                 (ldg_f(v + (i * (ny + 1) + j + 1) * nz + k) - ldg_f(v + (i * (ny + 1) + j) * nz + k)) +
                 (ldg_f(w + (i * ny + j) * (nz + 1) + k + 1) - ldg_f(w + (i * ny + j) * (nz + 1) + k));
    div[(i * ny + j) * nz + k] = divide(flux, divisor(info.cell_m));
  }
}

// subtract_gradient_kernel (pressure.py:95-116) over the three face arrays (blockIdx.z segments).
// The face's pressure difference (q_above - q_below); false for a closed wall face, which is left alone.
template <int AXIS>
__device__ __forceinline__ bool gradient_at(const PlumeGridInfo& info, const float* __restrict__ q, int i, int j, int k,
                                            float& q_above, float& q_below) {
  const Dims d = dims_of(info);
  const int index = AXIS == 0 ? i : (AXIS == 1 ? j : k);
  const int below = AXIS == 0 ? at(d, i - 1, j, k) : (AXIS == 1 ? at(d, i, j - 1, k) : at(d, i, j, k - 1));
  q_above = 0.0f;
  q_below = 0.0f;
  if (index == 0) {
    if (info.open_lo[AXIS] == 0) return false;
    q_above = __ldg(q + at(d, i, j, k));
  } else if (index == info.dims[AXIS]) {
    if (info.open_hi[AXIS] == 0) return false;
    q_below = __ldg(q + below);
  } else {
    q_above = __ldg(q + at(d, i, j, k));
    q_below = __ldg(q + below);
  }
  return true;
}

template <int AXIS, int PLANES, class T>
__device__ __forceinline__ void subtract_gradient_planes(const PlumeGridInfo& info, T* __restrict__ f,
                                                         const float* __restrict__ q, int i0, int j, int k) {
  const Dims d = {info.dims[0] + (AXIS == 0), info.dims[1] + (AXIS == 1), info.dims[2] + (AXIS == 2)};
  if (j >= d.n1 || k >= d.n2) return;
  const long plane = (long)d.n1 * d.n2, at_jk = (long)j * d.n2 + k;
  float value[PLANES], above[PLANES], below[PLANES];
  bool apply[PLANES];
#pragma unroll
  for (int p = 0; p < PLANES; ++p) {
    apply[p] = i0 + p < d.n0 && gradient_at<AXIS>(info, q, i0 + p, j, k, above[p], below[p]);
    if (apply[p]) value[p] = ld_f(f + (i0 + p) * plane + at_jk);
  }
#pragma unroll
  for (int p = 0; p < PLANES; ++p)
    if (apply[p]) st_f(f + (i0 + p) * plane + at_jk, value[p] - divide(above[p] - below[p], divisor(info.cell_m)));
}

template <class T, int PLANES>
__global__ void k_subtract_gradient(PlumeGridInfo info, T* __restrict__ u, T* __restrict__ v, T* __restrict__ w,
                                    const float* __restrict__ q) {
  int axis, i0;
  face_planes<PLANES>(info, axis, i0);
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (axis == 0) subtract_gradient_planes<0, PLANES>(info, u, q, i0, j, k);
  else if (axis == 1) subtract_gradient_planes<1, PLANES>(info, v, q, i0, j, k);
  else subtract_gradient_planes<2, PLANES>(info, w, q, i0, j, k);
}

template <class T>
static int launch_divergence(const PlumeGridInfo& info, const T* u, const T* v, const T* w, float* div,
                             cudaStream_t st) {
  return with_planes([&](auto P) {
    constexpr int PL = decltype(P)::value;
    k_divergence<T, PL><<<cell_grid_planes(info.dims[0], info.dims[1], info.dims[2], PL), cell_block(), 0, st>>>(
        info, u, v, w, div);
    return launch_status("divergence");
  });
}

template <class T>
static int launch_subtract_gradient(const PlumeGridInfo& info, T* u, T* v, T* w, const float* q, cudaStream_t st) {
  return with_planes([&](auto P) {
    constexpr int PL = decltype(P)::value;
    k_subtract_gradient<T, PL><<<face_grid(info, PL), cell_block(), 0, st>>>(info, u, v, w, q);
    return launch_status("subtract gradient");
  });
}

// ---- residual (multigrid.py:36-43), for callers that inspect it ---------------------------------------------
__global__ void k_residual(PlumeGridInfo info, const float* __restrict__ q, const float* __restrict__ rhs,
                           float* __restrict__ res) {
  const int ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny || k >= nz) return;
  const Dims d{info.dims[0], ny, nz};
  auto load = [&](int a, int b, int c) { return __ldg(q + at(d, a, b, c)); };
  const int idx = (i * ny + j) * nz + k;
  res[idx] = residual_at(info, i, j, k, __ldg(q + idx), __ldg(rhs + idx), load);
}

// ---- the defect-correction solve's residual (no reference counterpart) --------------------------------------
// r = rhs - A q evaluated in double (residual_f64), stored as float for the correction cycle, with the block
// sums of r^2 and rhs^2 (double, a halving tree over the block's 256 threads); k_norm_finish adds the block
// partials in a fixed order, so the norms are the same on every run. With `q_lo`, the pressure is the
// unevaluated sum q + q_lo of two floats (the refinement's compensated iterate).
constexpr int NORM_THREADS = TZ * TY;

__global__ void k_residual_f64(PlumeGridInfo info, const float* __restrict__ q, const float* __restrict__ q_lo,
                               const float* __restrict__ rhs, float* __restrict__ res, double* __restrict__ partial) {
  __shared__ double rr[NORM_THREADS], bb[NORM_THREADS];
  const int ny = info.dims[1], nz = info.dims[2];
  const int i = blockIdx.z, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  double r = 0.0, b = 0.0;
  if (j < ny && k < nz) {
    const Dims d{info.dims[0], ny, nz};
    auto value = [&](int c) { return (double)__ldg(q + c) + (q_lo ? (double)__ldg(q_lo + c) : 0.0); };
    auto load = [&](int a, int bb_, int c) { return value(at(d, a, bb_, c)); };
    const int idx = (i * ny + j) * nz + k;
    b = __ldg(rhs + idx);
    r = residual_f64(info, i, j, k, value(idx), b, load);
    res[idx] = (float)r;
  }
  rr[t] = r * r;
  bb[t] = b * b;
  __syncthreads();
  for (int half = NORM_THREADS / 2; half > 0; half /= 2) {
    if (t < half) {
      rr[t] = rr[t] + rr[t + half];
      bb[t] = bb[t] + bb[t + half];
    }
    __syncthreads();
  }
  if (t == 0) {
    const long block = blockIdx.x + (long)gridDim.x * (blockIdx.y + (long)gridDim.y * blockIdx.z);
    partial[2 * block] = rr[0];
    partial[2 * block + 1] = bb[0];
  }
}

__global__ void k_norm_finish(const double* __restrict__ partial, long blocks, double* __restrict__ norms) {
  __shared__ double rr[NORM_THREADS], bb[NORM_THREADS];
  const int t = threadIdx.x;
  double r = 0.0, b = 0.0;
  for (long n = t; n < blocks; n += NORM_THREADS) {
    r = r + partial[2 * n];
    b = b + partial[2 * n + 1];
  }
  rr[t] = r;
  bb[t] = b;
  __syncthreads();
  for (int half = NORM_THREADS / 2; half > 0; half /= 2) {
    if (t < half) {
      rr[t] = rr[t] + rr[t + half];
      bb[t] = bb[t] + bb[t + half];
    }
    __syncthreads();
  }
  if (t == 0) {
    norms[0] = rr[0];
    norms[1] = bb[0];
  }
}

// q += e; with q_lo, (q, q_lo) += e as a float pair: the rounding error of q + e (Knuth's two-sum) joins
// q_lo, then the pair is renormalised so that q is the float nearest q + q_lo.
__global__ void k_add_into(float* __restrict__ q, float* __restrict__ q_lo, const float* __restrict__ e, long n) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const float a = q[idx], b = e[idx];
  const float s = a + b;
  if (!q_lo) {
    q[idx] = s;
    return;
  }
  const float bv = s - a;
  const float err = (a - (s - bv)) + (b - bv);
  const float lo = q_lo[idx] + err;
  const float hi = s + lo;
  q[idx] = hi;
  q_lo[idx] = lo - (hi - s);
}

static long norm_blocks(const PlumeGridInfo& info) {
  const dim3 g = cell_grid(info.dims[0], info.dims[1], info.dims[2]);
  return (long)g.x * g.y * g.z;
}

// ---- smoke budget: conserve.py:33-52 + reduce.py:12-38 ------------------------------------------------------
// Line totals along x in float (reduce.py:12-25); lines added in double in blocks of 256 by a halving tree,
// then the block partials in order on one thread. The CPU oracle adds in the same order.
constexpr int SUM_BLOCK = 256;

template <class T>
__global__ void k_line_partials(Dims d, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ c,
                                double* __restrict__ partial, int blocks) {
  __shared__ double slot[SUM_BLOCK];
  const T* src = blockIdx.y == 0 ? a : (blockIdx.y == 1 ? b : c);
  const long line = (long)blockIdx.x * SUM_BLOCK + threadIdx.x;
  const long lines = (long)d.n1 * d.n2;
  double value = 0.0;
  if (line < lines) {
    float total = 0.0f;
    for (int i = 0; i < d.n0; ++i) total = total + ldg_f(src + (long)i * lines + line);
    value = (double)total;
  }
  slot[threadIdx.x] = value;
  __syncthreads();
  for (int h = SUM_BLOCK / 2; h >= 1; h >>= 1) {
    if ((int)threadIdx.x < h) slot[threadIdx.x] = slot[threadIdx.x] + slot[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.y * blocks + blockIdx.x] = slot[0];
}

// totals[0..2] = before, semi-Lagrangian, MacCormack; factor = held / MacCormack (1 when MacCormack <= 0).
// One warp per total (threadIdx.y): the lanes load 32 block partials at a time and every lane adds them in
// block order from the shuffles, the same additions in the same order as one thread walking the partials.
// Measured on B200 at 128x192x128 (96 partials per total), cold under ncu: 13.0-16.7 us on one thread,
// 3.7-5.0 us this way; the scalar advection phase went from 0.176 to 0.172 ms (1.154 to 1.137 ms at
// 256x384x256).
__global__ void k_budget_factor(const double* __restrict__ partial, int blocks, float* factor, double* totals_out,
                                int want_factor) {
  __shared__ double t[3];
  const int which = threadIdx.y, lane = threadIdx.x;
  double total = 0.0;
  for (int base = 0; base < blocks; base += 32) {
    const double mine = base + lane < blocks ? partial[which * blocks + base + lane] : 0.0;
    const int count = blocks - base < 32 ? blocks - base : 32;
    for (int l = 0; l < count; ++l) total = total + __shfl_sync(0xffffffffu, mine, l);
  }
  if (lane == 0) t[which] = total;
  __syncthreads();
  if (threadIdx.x != 0 || threadIdx.y != 0) return;
  if (totals_out) {
    totals_out[0] = t[0];
    totals_out[1] = t[1];
    totals_out[2] = t[2];
  }
  if (!want_factor) return;
  const double before = t[0], sl = t[1], mc = t[2];
  const double held = sl > (mc < before ? mc : before) ? sl : (mc < before ? mc : before);
  *factor = mc > 0.0 ? (float)(held / mc) : 1.0f;
}

template <class T>
__global__ void k_scale(T* __restrict__ f, long n, const float* __restrict__ factor) {  // conserve.py:27-30
  const float s = *factor;
  for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x)
    st_f(f + idx, ld_f(f + idx) * s);
}

static int sum_blocks(const Dims& d) { return (int)(((long)d.n1 * d.n2 + SUM_BLOCK - 1) / SUM_BLOCK); }

template <class T>
static int launch_triple_sum(const Dims& d, const T* a, const T* b, const T* c, double* sums, float* factor,
                             double* totals_out, cudaStream_t st) {
  const int blocks = sum_blocks(d);
  k_line_partials<T><<<dim3(blocks, 3), SUM_BLOCK, 0, st>>>(d, a, b, c, sums, blocks);
  CHECK_LAUNCH("line sums");
  k_budget_factor<<<1, dim3(32, 3), 0, st>>>(sums, blocks, factor, totals_out, factor != nullptr);
  CHECK_LAUNCH("budget factor");
  return PLUME_OK;
}

// Which advections of plume_step run the fused march (advect.cu): bit 0 the velocity, bit 1 smoke and
// temperature; the others run the two-pass kernels (hat and the clamp ranges through global memory, the
// reference's blend arithmetic). Measured on B200 at 256x384x256: velocity 2.25 ms fused against 2.60 ms two-pass,
// smoke and temperature 1.27 ms fused against 1.13 ms two-pass.
static int g_fused_advection = 1;

static int grid_stride_blocks(long n) {
  long b = (n + 255) / 256;
  return (int)std::min<long>(b, 148L * 16);
}

// ---- the scalar epilogue: conserve scale + dissipation (conserve.py:50-52, dissipate.py:10-15) -------------
// With storage narrower than float, the conserve scale is rounded to storage before dissipation, as the
// reference's separate passes do.
template <class T>
__global__ void k_scalar_finish(T* __restrict__ smoke, T* __restrict__ temperature, long n,
                                const float* __restrict__ factor, int dissipate, float smoke_keep, float heat_keep,
                                float ambient) {
  const float s = *factor;
  for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    float value = to_f<T>(from_f<T>(ld_f(smoke + idx) * s));
    if (dissipate) {
      value = value * smoke_keep;
      if (temperature) st_f(temperature + idx, ambient + (ld_f(temperature + idx) - ambient) * heat_keep);
    }
    st_f(smoke + idx, value);
  }
}

template <class T>
__global__ void k_dissipate(T* __restrict__ smoke, T* __restrict__ temperature, long n, float smoke_keep,
                            float heat_keep, float ambient) {  // dissipate.py:10-15
  for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    st_f(smoke + idx, ld_f(smoke + idx) * smoke_keep);
    st_f(temperature + idx, ambient + (ld_f(temperature + idx) - ambient) * heat_keep);
  }
}

// ---- grid speed: step_cap.py:50-55 (max is exact in any order) ----------------------------------------------
template <class T>
__global__ void k_abs_max(const T* __restrict__ a, long na, const T* __restrict__ b, long nb, const T* __restrict__ c,
                          long nc, unsigned int* __restrict__ out) {
  float best = 0.0f;
  const long total = na + nb + nc;
  for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    float value = idx < na ? ldg_f(a + idx) : (idx < na + nb ? ldg_f(b + idx - na) : ldg_f(c + idx - na - nb));
    best = fmax_(best, fabsf(value));
  }
  for (int off = 16; off >= 1; off >>= 1) best = fmax_(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(best));  // non-negative floats order as ints
}

}  // namespace plume

using namespace plume;

// ---- C ABI -------------------------------------------------------------------------------------------------

extern "C" const char* plume_last_error(void) { return g_error; }
extern "C" int plume_abi_version(void) { return 1; }
extern "C" unsigned long long plume_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

extern "C" int plume_advect_semi_lagrangian(const PlumeGridInfo* info, const int32_t shape[3], const float* src,
                                            float* dst, const float* u, const float* v, const float* w,
                                            float dt_over_cell, const float offset[3], float outside,
                                            int32_t uses_outside, void* stream) {
  CHECK_ARG(info && shape && src && dst && u && v && w && offset, "semi_lagrangian: null argument");
  CHECK_ARG(valid_dims(info->dims) && valid_dims(shape), "semi_lagrangian: bad dims");
  FieldSet<float> set{};
  set.count = 1;
  set.f[0] = single_field<float>(src, nullptr, dst, Dims{shape[0], shape[1], shape[2]},
                                 f3(offset[0], offset[1], offset[2]), outside, uses_outside);
  return launch_advect(*info, make_vel(u, v, w, info->dims), set, dt_over_cell, false, as_stream(stream));
}

extern "C" int plume_advect_maccormack(const PlumeGridInfo* info, const int32_t shape[3], const float* data,
                                       float* hat, float* next, const float* u, const float* v, const float* w,
                                       float dt_over_cell, const float offset[3], float outside, int32_t uses_outside,
                                       void* stream) {
  CHECK_ARG(info && shape && data && hat && next && u && v && w && offset, "maccormack: null argument");
  CHECK_ARG(valid_dims(info->dims) && valid_dims(shape), "maccormack: bad dims");
  FieldSet<float> set{};
  set.count = 1;
  set.f[0] = single_field<float>(data, hat, next, Dims{shape[0], shape[1], shape[2]},
                                 f3(offset[0], offset[1], offset[2]), outside, uses_outside);
  return launch_advect(*info, make_vel(u, v, w, info->dims), set, dt_over_cell, true, as_stream(stream));
}

extern "C" int plume_emit(const PlumeGridInfo* info, float* smoke, float* temperature, float* u, float* v, float* w,
                          const PlumeEmitter* emitters, int32_t count, int32_t seed, float time_s, float dt,
                          void* stream) {
  CHECK_ARG(info && smoke && temperature && u && v && w, "emit: null argument");
  CHECK_ARG(count >= 0 && (count == 0 || emitters), "emit: bad emitter list");
  CHECK_ARG(valid_dims(info->dims), "emit: bad dims");
  return launch_emit(*info, smoke, temperature, u, v, w, emitters, count, seed, time_s, dt, as_stream(stream));
}

extern "C" int plume_emit_adjoint(const PlumeGridInfo* info, float* a_temperature, float* a_u, float* a_v, float* a_w,
                                  const PlumeEmitter* emitters, int32_t count, int32_t seed, float time_s, float dt,
                                  void* stream) {
  CHECK_ARG(info && a_temperature && a_u && a_v && a_w, "emit_adjoint: null argument");
  CHECK_ARG(count >= 0 && (count == 0 || emitters), "emit_adjoint: bad emitter list");
  CHECK_ARG(valid_dims(info->dims), "emit_adjoint: bad dims");
  cudaStream_t st = as_stream(stream);
  std::vector<PlumeEmitter> active;
  for (int n = 0; n < count; ++n)
    if (time_s >= emitters[n].start_s && time_s < emitters[n].end_s) active.push_back(emitters[n]);
  for (size_t first = 0; first < active.size(); first += PLUME_MAX_EMITTERS) {
    EmitterSet set;
    set.count = (int)std::min<size_t>(PLUME_MAX_EMITTERS, active.size() - first);
    for (int n = 0; n < set.count; ++n) set.e[n] = active[first + n];
    int lo[3], hi[3];
    if (!emitter_box(*info, set.e, set.count, lo, hi)) continue;
    const int3 box_lo = make_int3(lo[0], lo[1], lo[2]);
    const int3 box_n = make_int3(hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1);
    dim3 grid((box_n.z + 1 + TZ - 1) / TZ, (box_n.y + 1 + TY - 1) / TY, box_n.x + (box_n.x + 1) + box_n.x + box_n.x);
    k_emit_adjoint<<<grid, cell_block(), 0, st>>>(*info, a_temperature, a_u, a_v, a_w, set, seed, time_s, dt, box_lo,
                                                   box_n);
    CHECK_LAUNCH("emit adjoint");
  }
  return PLUME_OK;
}

extern "C" int plume_buoyancy(const PlumeGridInfo* info, float* v, const float* smoke, const float* temperature,
                              float gravity, float heat_buoyancy, float smoke_weight, float ambient_k, float dt,
                              void* stream) {
  CHECK_ARG(info && v && smoke && temperature, "buoyancy: null argument");
  CHECK_ARG(valid_dims(info->dims), "buoyancy: bad dims");
  return launch_buoyancy<float>(*info, v, smoke, temperature, gravity, heat_buoyancy, smoke_weight, ambient_k, dt,
                                as_stream(stream));
}

extern "C" int plume_drag(const PlumeGridInfo* info, float* u, float* v, float* w, const float wind[3], float keep,
                          void* stream) {
  CHECK_ARG(info && u && v && w && wind, "drag: null argument");
  CHECK_ARG(valid_dims(info->dims), "drag: bad dims");
  FaceForces ff{};
  ff.drag = 1;
  ff.wind[0] = wind[0];
  ff.wind[1] = wind[1];
  ff.wind[2] = wind[2];
  ff.keep = keep;
  return launch_face_forces<float>(*info, u, v, w, ff, "drag", as_stream(stream));
}

extern "C" int plume_confinement(const PlumeGridInfo* info, float* u, float* v, float* w, float* curl_xyz[3],
                                 float* push_xyz[3], float strength, float dt, int32_t apply, void* stream) {
  CHECK_ARG(info && u && v && w && curl_xyz && curl_xyz[0] && curl_xyz[1] && curl_xyz[2], "confinement: null argument");
  CHECK_ARG(!apply || (push_xyz && push_xyz[0] && push_xyz[1] && push_xyz[2]), "confinement: null push");
  CHECK_ARG(valid_dims(info->dims), "confinement: bad dims");
  cudaStream_t st = as_stream(stream);
  int status = launch_confinement_push(*info, u, v, w, curl_xyz, push_xyz, strength, apply, st);
  if (status != PLUME_OK || !apply) return status;
  FaceForces ff{};
  ff.confinement = 1;
  ff.push[0] = push_xyz[0];
  ff.push[1] = push_xyz[1];
  ff.push[2] = push_xyz[2];
  ff.dt = dt;
  return launch_face_forces<float>(*info, u, v, w, ff, "add face push", st);
}

extern "C" int plume_turbulence(const PlumeGridInfo* info, float* u, float* v, float* w, int32_t seed, float scale_m,
                                float strength, float pattern_time, float dt, void* stream) {
  CHECK_ARG(info && u && v && w, "turbulence: null argument");
  CHECK_ARG(valid_dims(info->dims), "turbulence: bad dims");
  FaceForces ff{};
  ff.turbulence = 1;
  ff.seed = seed;
  ff.scale_m = scale_m;
  ff.strength = strength;
  ff.pattern_time = pattern_time;
  ff.dt = dt;
  return launch_face_forces<float>(*info, u, v, w, ff, "turbulence", as_stream(stream));
}

extern "C" int plume_divergence(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                float* divergence, void* stream) {
  CHECK_ARG(info && u && v && w && divergence, "divergence: null argument");
  CHECK_ARG(valid_dims(info->dims), "divergence: bad dims");
  return launch_divergence<float>(*info, u, v, w, divergence, as_stream(stream));
}

namespace plume {
// zero_closed_faces_kernel x 3 + divergence_kernel (pressure.py:144-150).
template <class T>
static int project_begin(const PlumeGridInfo& info, T* u, T* v, T* w, float* divergence, cudaStream_t st) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const int m = std::max(nx, ny) + 1, n = std::max(ny, nz) + 1;
  k_zero_walls<T><<<dim3((n + TZ - 1) / TZ, (m + TY - 1) / TY, 6), cell_block(), 0, st>>>(info, u, v, w);
  CHECK_LAUNCH("zero closed faces");
  return launch_divergence<T>(info, u, v, w, divergence, st);
}
}  // namespace plume

extern "C" int plume_project_begin(const PlumeGridInfo* info, float* u, float* v, float* w, float* divergence,
                                   void* stream) {
  CHECK_ARG(info && u && v && w && divergence, "project: null argument");
  CHECK_ARG(valid_dims(info->dims), "project: bad dims");
  return project_begin(*info, u, v, w, divergence, as_stream(stream));
}

extern "C" int plume_subtract_gradient(const PlumeGridInfo* info, float* u, float* v, float* w, const float* q,
                                       void* stream) {
  CHECK_ARG(info && u && v && w && q, "subtract_gradient: null argument");
  CHECK_ARG(valid_dims(info->dims), "subtract_gradient: bad dims");
  return launch_subtract_gradient<float>(*info, u, v, w, q, as_stream(stream));
}

extern "C" int plume_red_black_sweeps(const PlumeGridInfo* info, float* q, float* scratch, const float* rhs,
                                      int32_t sweeps, float relaxation, void* stream) {
  CHECK_ARG(info && q && scratch && rhs && sweeps >= 0 && scratch != q, "red_black_sweeps: bad argument");
  CHECK_ARG(valid_dims(info->dims), "red_black_sweeps: bad dims");
  return red_black_sweeps(*info, q, scratch, rhs, sweeps, relaxation, as_stream(stream));
}

extern "C" int plume_multigrid(const PlumeLevel* levels, int32_t level_count, int32_t cycles, int32_t sweeps,
                               void* stream) {
  CHECK_ARG(levels && level_count >= 1 && cycles >= 0 && sweeps >= 0, "multigrid: bad argument");
  for (int l = 0; l < level_count; ++l)
    CHECK_ARG(levels[l].q && levels[l].rhs && levels[l].residual && levels[l].residual != levels[l].q &&
                  valid_dims(levels[l].info.dims),
              "multigrid: bad level %d", l);
  return multigrid_cycles(levels, level_count, cycles, sweeps, as_stream(stream));
}

extern "C" int plume_multigrid_split(const PlumeLevel* levels, int32_t level_count, int32_t cycles, int32_t sweeps,
                                     float* scratch, void* stream) {
  CHECK_ARG(levels && level_count >= 1 && cycles >= 0 && sweeps >= 0 && scratch, "multigrid_split: bad argument");
  for (int l = 0; l < level_count; ++l)
    CHECK_ARG(levels[l].q && levels[l].rhs && levels[l].residual && levels[l].residual != levels[l].q &&
                  valid_dims(levels[l].info.dims),
              "multigrid_split: bad level %d", l);
  return multigrid_cycles(levels, level_count, cycles, sweeps, as_stream(stream), 0, scratch);
}

extern "C" int plume_residual(const PlumeGridInfo* info, const float* q, const float* rhs, float* residual,
                              void* stream) {
  CHECK_ARG(info && q && rhs && residual, "residual: null argument");
  CHECK_ARG(valid_dims(info->dims), "residual: bad dims");
  const int nx = info->dims[0], ny = info->dims[1], nz = info->dims[2];
  k_residual<<<cell_grid(nx, ny, nz), cell_block(), 0, as_stream(stream)>>>(*info, q, rhs, residual);
  return launch_status("residual");
}

extern "C" long long plume_norm_scratch_doubles(const PlumeGridInfo* info) {
  if (!info || !valid_dims(info->dims)) return fail(PLUME_ERR_INVALID, "norm_scratch_doubles: bad dims");
  return 2 * (long long)norm_blocks(*info);
}

extern "C" int plume_residual_f64(const PlumeGridInfo* info, const float* q, const float* q_lo, const float* rhs,
                                  float* residual, double* scratch, double* norms, void* stream) {
  CHECK_ARG(info && q && rhs && residual && scratch && norms, "residual_f64: null argument");
  CHECK_ARG(valid_dims(info->dims), "residual_f64: bad dims");
  cudaStream_t st = as_stream(stream);
  const int nx = info->dims[0], ny = info->dims[1], nz = info->dims[2];
  k_residual_f64<<<cell_grid(nx, ny, nz), cell_block(), 0, st>>>(*info, q, q_lo, rhs, residual, scratch);
  int status = launch_status("residual (double)");
  if (status != PLUME_OK) return status;
  k_norm_finish<<<1, NORM_THREADS, 0, st>>>(scratch, norm_blocks(*info), norms);
  return launch_status("residual norms");
}

extern "C" int plume_multigrid_correct(const PlumeLevel* levels, int32_t level_count, int32_t sweeps, float* pressure,
                                       float* pressure_lo, void* stream) {
  CHECK_ARG(levels && level_count >= 1 && sweeps >= 0 && pressure && pressure_lo != pressure,
            "multigrid_correct: bad argument");
  for (int l = 0; l < level_count; ++l)
    CHECK_ARG(levels[l].q && levels[l].rhs && levels[l].residual && levels[l].residual != levels[l].q &&
                  levels[l].q != pressure && levels[l].q != pressure_lo && valid_dims(levels[l].info.dims),
              "multigrid_correct: bad level %d", l);
  cudaStream_t st = as_stream(stream);
  const long n = (long)levels[0].info.dims[0] * levels[0].info.dims[1] * levels[0].info.dims[2];
  int status = runtime_status("correction clear", cudaMemsetAsync(levels[0].q, 0, sizeof(float) * n, st));
  if (status != PLUME_OK) return status;
  if ((status = multigrid_cycles(levels, level_count, 1, sweeps, st, 1)) != PLUME_OK) return status;
  k_add_into<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pressure, pressure_lo, levels[0].q, n);
  return launch_status("correction add");
}

extern "C" long long plume_advect_scratch_floats(const PlumeGridInfo* info) {
  if (!info || !valid_dims(info->dims)) return fail(PLUME_ERR_INVALID, "advect_scratch_floats: bad dims");
  const long long nx = info->dims[0], ny = info->dims[1], nz = info->dims[2];
  // the clamp ranges of the two-pass advection, or the colour-split solve's q and rhs (rows padded to 4)
  const long long ranges = 2 * ((nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1));
  const long long split = 4 * nx * ny * (((nz + 1) / 2 + 3) / 4 * 4);
  return ranges > split ? ranges : split;
}

extern "C" int plume_smoke_scratch_doubles(const PlumeGridInfo* info) {
  if (!info || !valid_dims(info->dims)) return fail(PLUME_ERR_INVALID, "smoke_scratch_doubles: bad dims");
  return 3 * sum_blocks(dims_of(*info));
}

extern "C" int plume_triple_sum(const int32_t shape[3], const float* a, const float* b, const float* c, double* sums,
                                double* totals_out, void* stream) {
  CHECK_ARG(shape && a && b && c && sums && totals_out, "triple_sum: null argument");
  CHECK_ARG(valid_dims(shape), "triple_sum: bad dims");
  return launch_triple_sum(Dims{shape[0], shape[1], shape[2]}, a, b, c, sums, nullptr, totals_out, as_stream(stream));
}

extern "C" int plume_smoke_budget(const PlumeGridInfo* info, const float* data, const float* hat, float* next,
                                  double* sums, float* factor, double* totals_out, void* stream) {
  CHECK_ARG(info && data && hat && next && sums && factor, "smoke_budget: null argument");
  CHECK_ARG(valid_dims(info->dims), "smoke_budget: bad dims");
  cudaStream_t st = as_stream(stream);
  const Dims d = dims_of(*info);
  int status = launch_triple_sum(d, data, hat, next, sums, factor, totals_out, st);
  if (status != PLUME_OK) return status;
  const long n = (long)d.n0 * d.n1 * d.n2;
  k_scale<<<grid_stride_blocks(n), 256, 0, st>>>(next, n, factor);
  return launch_status("smoke budget scale");
}

extern "C" int plume_use_fused_advection(int32_t mask) {
  CHECK_ARG(mask >= 0 && mask <= 3, "use_fused_advection: mask %d (bit 0 velocity, bit 1 scalars)", mask);
  g_fused_advection = mask;
  return PLUME_OK;
}

extern "C" long long plume_maccormack_scratch_floats(const PlumeGridInfo* info) {
  if (!info || !valid_dims(info->dims)) return fail(PLUME_ERR_INVALID, "maccormack_scratch_floats: bad dims");
  return mac_partial_floats(*info);
}

extern "C" int plume_maccormack_velocity(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                         float* u_next, float* v_next, float* w_next, float dt_over_cell,
                                         void* stream) {
  CHECK_ARG(info && u && v && w && u_next && v_next && w_next, "maccormack_velocity: null argument");
  CHECK_ARG(valid_dims(info->dims), "maccormack_velocity: bad dims");
  CHECK_ARG(u_next != u && v_next != v && w_next != w, "maccormack_velocity: next must not alias data");
  return launch_mac_velocity<float>(*info, u, v, w, u_next, v_next, w_next, dt_over_cell, as_stream(stream));
}

extern "C" int plume_maccormack_scalars(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                                        const float* smoke, const float* temperature, float* smoke_next,
                                        float* temperature_next, float dt_over_cell, float smoke_outside,
                                        float heat_outside, int32_t uses_outside, float* scratch, double* sums,
                                        double* totals_out, void* stream) {
  CHECK_ARG(info && u && v && w && smoke && temperature && smoke_next && temperature_next && scratch && sums,
            "maccormack_scalars: null argument");
  CHECK_ARG(valid_dims(info->dims), "maccormack_scalars: bad dims");
  CHECK_ARG(smoke_next != smoke && temperature_next != temperature, "maccormack_scalars: next must not alias data");
  cudaStream_t st = as_stream(stream);
  int status = launch_mac_scalars<float>(*info, u, v, w, smoke, temperature, smoke_next, temperature_next,
                                         smoke_outside, heat_outside, uses_outside, scratch, sums, 0, 1.0f, 0.0f,
                                         dt_over_cell, st);
  if (status != PLUME_OK || !totals_out) return status;
  k_budget_factor<<<1, dim3(32, 3), 0, st>>>(sums, sum_blocks(dims_of(*info)), nullptr, totals_out, 0);
  return launch_status("maccormack_scalars: totals");
}

extern "C" int plume_dissipate(const PlumeGridInfo* info, float* smoke, float* temperature, float smoke_keep,
                               float heat_keep, float ambient_k, void* stream) {
  CHECK_ARG(info && smoke && temperature, "dissipate: null argument");
  CHECK_ARG(valid_dims(info->dims), "dissipate: bad dims");
  const long n = (long)info->dims[0] * info->dims[1] * info->dims[2];
  k_dissipate<<<grid_stride_blocks(n), 256, 0, as_stream(stream)>>>(smoke, temperature, n, smoke_keep, heat_keep,
                                                                    ambient_k);
  return launch_status("dissipate");
}

namespace plume {
template <class T>
static int grid_speed(const PlumeGridInfo& info, const void* u, const void* v, const void* w, float* speed,
                      cudaStream_t st) {
  const long nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const long na = (nx + 1) * ny * nz, nb = nx * (ny + 1) * nz, nc = nx * ny * (nz + 1);
  int status = runtime_status("grid speed reset", cudaMemsetAsync(speed, 0, sizeof(float), st));
  if (status != PLUME_OK) return status;
  k_abs_max<T><<<grid_stride_blocks(na + nb + nc), 256, 0, st>>>(static_cast<const T*>(u), na, static_cast<const T*>(v),
                                                                 nb, static_cast<const T*>(w), nc,
                                                                 reinterpret_cast<unsigned int*>(speed));
  return launch_status("grid speed");
}
}  // namespace plume

extern "C" int plume_grid_speed(const PlumeGridInfo* info, const void* u, const void* v, const void* w, int32_t storage,
                                float* speed, void* stream) {
  CHECK_ARG(info && u && v && w && speed, "grid_speed: null argument");
  CHECK_ARG(valid_dims(info->dims), "grid_speed: bad dims");
  cudaStream_t st = as_stream(stream);
  switch (storage) {
    case PLUME_STORAGE_F32: return grid_speed<float>(*info, u, v, w, speed, st);
    case PLUME_STORAGE_BF16: return grid_speed<__nv_bfloat16>(*info, u, v, w, speed, st);
    case PLUME_STORAGE_F16: return grid_speed<__half>(*info, u, v, w, speed, st);
  }
  return fail(PLUME_ERR_INVALID, "grid_speed: storage %d", storage);
}

namespace plume {

// Stepper.step (stepper.py:28-44) with the fields stored as T.
template <class T>
static int step(const PlumeStepState* s, const PlumeStepParams* p, void* stream) {
  cudaStream_t st = as_stream(stream);
  const PlumeGridInfo& info = s->info;
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  T* const ud = static_cast<T*>(s->u.data);
  T* const vd = static_cast<T*>(s->v.data);
  T* const wd = static_cast<T*>(s->w.data);
  T* const sd = static_cast<T*>(s->smoke.data);
  T* const td = static_cast<T*>(s->temperature.data);
  int status;
  int phase = 0;
  auto mark = [&]() -> int {  // phase boundary event, when the caller asked for them
    if (!p->phase_events) return PLUME_OK;
    return runtime_status("phase event", cudaEventRecord(reinterpret_cast<cudaEvent_t>(p->phase_events[phase++]), st));
  };
  if ((status = mark()) != PLUME_OK) return status;
  // emit, buoyancy (stepper.py:32-34)
  if ((status = launch_emit<T>(info, sd, td, ud, vd, wd, p->emitters, p->emitter_count, p->seed, p->time_s, p->dt,
                               st)) != PLUME_OK)
    return status;
  if ((status = launch_buoyancy<T>(info, vd, sd, td, p->gravity, p->heat_buoyancy, p->smoke_weight, p->ambient_k, p->dt,
                                   st)) != PLUME_OK)
    return status;
  // confinement, turbulence, drag (stepper.py:35-40): one face pass after the push is known
  FaceForces ff{};
  ff.dt = p->dt;
  if (p->confinement != 0.0f) {
    float* curl[3] = {s->curl[0], s->curl[1], s->curl[2]};
    float* push[3] = {s->push[0], s->push[1], s->push[2]};
    if ((status = launch_confinement_push<T>(info, ud, vd, wd, curl, push, p->confinement, 1, st, s->divergence)) !=
        PLUME_OK)
      return status;
    ff.confinement = 1;
    ff.push[0] = s->push[0];
    ff.push[1] = s->push[1];
    ff.push[2] = s->push[2];
  }
  if (p->turbulence_strength != 0.0f) {
    ff.turbulence = 1;
    ff.seed = p->seed;
    ff.scale_m = p->turbulence_scale_m;
    ff.strength = p->turbulence_strength;
    ff.pattern_time = p->turbulence_pattern_time;
  }
  if (p->apply_drag) {
    ff.drag = 1;
    ff.wind[0] = p->wind[0];
    ff.wind[1] = p->wind[1];
    ff.wind[2] = p->wind[2];
    ff.keep = p->drag_keep;
  }
  if (ff.confinement || ff.turbulence || ff.drag) {
    if ((status = launch_face_forces<T>(info, ud, vd, wd, ff, "face forces", st)) != PLUME_OK) return status;
  }
  if ((status = mark()) != PLUME_OK) return status;
  // advect velocity (stepper.py:46-52)
  if (s->advect_scratch && (g_fused_advection & 1)) {
    if ((status = launch_mac_velocity<T>(info, ud, vd, wd, static_cast<T*>(s->u.next), static_cast<T*>(s->v.next),
                                         static_cast<T*>(s->w.next), p->dt_over_cell, st)) != PLUME_OK)
      return status;
  } else {
    FieldSet<T> set{};
    set.count = 3;
    set.f[0] = single_field<T>(ud, static_cast<T*>(s->u.hat), static_cast<T*>(s->u.next), Dims{nx + 1, ny, nz},
                               f3(0.0f, 0.5f, 0.5f), 0.0f, 0);
    set.f[1] = single_field<T>(vd, static_cast<T*>(s->v.hat), static_cast<T*>(s->v.next), Dims{nx, ny + 1, nz},
                               f3(0.5f, 0.0f, 0.5f), 0.0f, 0);
    set.f[2] = single_field<T>(wd, static_cast<T*>(s->w.hat), static_cast<T*>(s->w.next), Dims{nx, ny, nz + 1},
                               f3(0.5f, 0.5f, 0.0f), 0.0f, 0);
    if (s->advect_scratch) {  // clamp ranges: u's, v's, w's, back to back
      pair_t<T>* r = reinterpret_cast<pair_t<T>*>(s->advect_scratch);
      set.f[0].range[0] = r;
      set.f[1].range[0] = r + (size_t)(nx + 1) * ny * nz;
      set.f[2].range[0] = r + (size_t)(nx + 1) * ny * nz + (size_t)nx * (ny + 1) * nz;
    }
    if ((status = launch_advect<T>(info, make_vel<T>(ud, vd, wd, info.dims), set, p->dt_over_cell, true, st)) !=
        PLUME_OK)
      return status;
  }
  if ((status = mark()) != PLUME_OK) return status;
  T* u = static_cast<T*>(s->u.next);  // after the swap
  T* v = static_cast<T*>(s->v.next);
  T* w = static_cast<T*>(s->w.next);
  // project (stepper.py:42, pressure.py:144-154)
  if ((status = project_begin<T>(info, u, v, w, s->divergence, st)) != PLUME_OK) return status;
  if ((status = mark()) != PLUME_OK) return status;
  if (p->solver == 0) {
    if ((status = multigrid_cycles(s->levels, s->level_count, p->solver_iterations, p->multigrid_sweeps, st, 0,
                                   s->advect_scratch)) != PLUME_OK)
      return status;
  } else if ((status = red_black_sweeps(info, s->pressure, s->levels[0].residual, s->divergence, p->solver_iterations,
                                        1.5f, st)) != PLUME_OK) {
    return status;
  }
  if ((status = mark()) != PLUME_OK) return status;
  if ((status = launch_subtract_gradient<T>(info, u, v, w, s->pressure, st)) != PLUME_OK) return status;
  if ((status = mark()) != PLUME_OK) return status;
  // advect smoke and temperature (stepper.py:54-60): the smoke budget holds smoke.next before its swap
  const long n = (long)nx * ny * nz;
  if (s->advect_scratch && (g_fused_advection & 2)) {
    // one pass: smoke and temperature advected together, temperature dissipated as it is stored, the smoke
    // line sums of data, hat and next from the march; then the held factor and the smoke's scale + dissipation
    if ((status = launch_mac_scalars<T>(info, u, v, w, sd, td, static_cast<T*>(s->smoke.next),
                                        static_cast<T*>(s->temperature.next), 0.0f, p->ambient_k, 1,
                                        s->advect_scratch, s->sums, p->apply_dissipation, p->heat_keep, p->ambient_k,
                                        p->dt_over_cell, st)) != PLUME_OK)
      return status;
    k_budget_factor<<<1, dim3(32, 3), 0, st>>>(s->sums, sum_blocks(dims_of(info)), s->factor, nullptr, 1);
    CHECK_LAUNCH("budget factor");
    k_scalar_finish<T><<<grid_stride_blocks(n), 256, 0, st>>>(static_cast<T*>(s->smoke.next), nullptr, n, s->factor,
                                                              p->apply_dissipation, p->smoke_keep, 1.0f,
                                                              p->ambient_k);
    CHECK_LAUNCH("scale and dissipate");
    return mark();
  }
  {
    VelT<T> vel = make_vel<T>(u, v, w, info.dims);
    FieldSet<T> set{};
    set.count = 1;  // smoke and temperature share positions: one trace serves both
    set.f[0] = single_field<T>(sd, static_cast<T*>(s->smoke.hat), static_cast<T*>(s->smoke.next), Dims{nx, ny, nz},
                               f3(0.5f, 0.5f, 0.5f), 0.0f, 1);
    set.f[0].data[1] = td;
    set.f[0].hat[1] = static_cast<T*>(s->temperature.hat);
    set.f[0].next[1] = static_cast<T*>(s->temperature.next);
    set.f[0].outside[1] = p->ambient_k;
    set.f[0].fields = 2;
    if (s->advect_scratch) {
      pair_t<T>* r = reinterpret_cast<pair_t<T>*>(s->advect_scratch);
      set.f[0].range[0] = r;
      set.f[0].range[1] = r + (size_t)nx * ny * nz;
    }
    if ((status = launch_advect<T>(info, vel, set, p->dt_over_cell, true, st)) != PLUME_OK) return status;
  }
  if ((status = launch_triple_sum<T>(dims_of(info), sd, static_cast<const T*>(s->smoke.hat),
                                     static_cast<const T*>(s->smoke.next), s->sums, s->factor, nullptr, st)) != PLUME_OK)
    return status;
  // scale + dissipate (stepper.py:44) on the advected buffers
  k_scalar_finish<T><<<grid_stride_blocks(n), 256, 0, st>>>(static_cast<T*>(s->smoke.next),
                                                            static_cast<T*>(s->temperature.next), n, s->factor,
                                                            p->apply_dissipation, p->smoke_keep, p->heat_keep,
                                                            p->ambient_k);
  CHECK_LAUNCH("scale and dissipate");
  return mark();
}

}  // namespace plume

extern "C" int plume_step(const PlumeStepState* s, const PlumeStepParams* p, void* stream) {
  CHECK_ARG(s && p, "step: null argument");
  CHECK_ARG(valid_dims(s->info.dims), "step: bad dims");
  CHECK_ARG(s->u.data && s->u.hat && s->u.next && s->v.data && s->v.hat && s->v.next && s->w.data && s->w.hat &&
                s->w.next && s->smoke.data && s->smoke.hat && s->smoke.next && s->temperature.data &&
                s->temperature.hat && s->temperature.next && s->pressure && s->divergence && s->sums && s->factor,
            "step: null buffer");
  CHECK_ARG(s->levels && s->level_count >= 1 && s->levels[0].q == s->pressure && s->levels[0].rhs == s->divergence &&
                s->levels[0].residual && s->levels[0].residual != s->pressure,
            "step: levels must start at the grid's pressure and divergence, with a second pressure array");
  CHECK_ARG(p->confinement == 0.0f || (s->curl[0] && s->curl[1] && s->curl[2] && s->push[0] && s->push[1] && s->push[2]),
            "step: confinement scratch missing");
  switch (s->storage) {
    case PLUME_STORAGE_F32: return step<float>(s, p, stream);
    case PLUME_STORAGE_BF16: return step<__nv_bfloat16>(s, p, stream);
    case PLUME_STORAGE_F16: return step<__half>(s, p, stream);
  }
  return fail(PLUME_ERR_INVALID, "step: storage %d", s->storage);
}

// ---- the smoke budget without caller scratch --------------------------------------------------------------
// Some callers cannot allocate device memory at the moment they run the budget: a host engine that hands
// this library only the field arrays it owns, with its own allocator locked or budgeted, or code running
// inside a region where any cudaMalloc would synchronise the device or is forbidden. For them,
// plume_smoke_budget_static keeps its partial sums and its factor in one fixed array that lives in the
// library's own device memory (allocated when the library's module loads on a device, held until the
// process exits).
namespace plume {

constexpr long STATIC_BUDGET_MAX_LINES = 1L << 20;  // ny * nz: every (y, z) line summed along x
constexpr long STATIC_BUDGET_BLOCKS = STATIC_BUDGET_MAX_LINES / SUM_BLOCK;
// 3 totals' partials, then one slot whose first 4 bytes hold the float factor: 3 * 4096 + 1 doubles (96 KiB)
static __device__ __align__(256) double g_budget_scratch[3 * STATIC_BUDGET_BLOCKS + 1];

constexpr int MAX_DEVICES = 64;
static std::mutex g_scratch_mutex;
static double* g_scratch_address[MAX_DEVICES] = {};

// The array's device address on the current device. The name g_budget_scratch, used in host code, is only a
// host-side stand-in and must never be passed to a kernel; the real address is looked up once per device.
static int static_budget_scratch(double** out) {
  int device = 0;
  int status = runtime_status("static smoke budget: current device", cudaGetDevice(&device));
  if (status != PLUME_OK) return status;
  if (device < 0 || device >= MAX_DEVICES) return fail(PLUME_ERR_INVALID, "static smoke budget: device %d", device);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_address[device] == nullptr) {
    void* address = nullptr;
    status = runtime_status("static smoke budget: cudaGetSymbolAddress",
                            cudaGetSymbolAddress(&address, g_budget_scratch));
    if (status != PLUME_OK) return status;
    g_scratch_address[device] = static_cast<double*>(address);
  }
  *out = g_scratch_address[device];
  return PLUME_OK;
}

}  // namespace plume

extern "C" int plume_smoke_budget_static(const PlumeGridInfo* info, const float* data, const float* hat, float* next,
                                         double* totals_out, void* stream) {
  CHECK_ARG(info && data && hat && next, "smoke_budget_static: null argument");
  CHECK_ARG(valid_dims(info->dims), "smoke_budget_static: bad dims");
  const Dims d = dims_of(*info);
  const long lines = (long)d.n1 * d.n2;
  CHECK_ARG(lines <= STATIC_BUDGET_MAX_LINES,
            "smoke_budget_static: ny * nz = %ld lines exceeds the fixed scratch for %ld lines; use "
            "plume_smoke_budget with caller scratch", lines, STATIC_BUDGET_MAX_LINES);
  double* scratch = nullptr;
  int status = static_budget_scratch(&scratch);
  if (status != PLUME_OK) return status;
  // Nothing in the array needs clearing: each call writes every partial it reads, and the factor, before use.
  float* factor = reinterpret_cast<float*>(scratch + 3 * STATIC_BUDGET_BLOCKS);
  cudaStream_t st = as_stream(stream);
  status = launch_triple_sum(d, data, hat, next, scratch, factor, totals_out, st);
  if (status != PLUME_OK) return status;
  const long n = (long)d.n0 * d.n1 * d.n2;
  k_scale<<<grid_stride_blocks(n), 256, 0, st>>>(next, n, factor);
  return launch_status("static smoke budget scale");
}
