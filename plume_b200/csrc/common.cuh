// Device helpers shared by the sim and render kernels of libplume_b200.so (sm_100a).
//
// Arithmetic contract: every expression keeps the reference's order of IEEE float operations (the library is
// compiled with -fmad=false, so no multiply-add is contracted), lerp(a, b, t) = a*(1-t) + b*t, float->int
// conversions truncate, and min/max/clamp are plain comparisons. With that, every operator without exp/pow
// gives the same floats as the FP32 restatement of chadmv/plume's Warp kernels. exp and pow are evaluated
// in double and rounded once to float (within 1 ulp of the C library's expf/powf the reference calls).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/plume_b200.h"

namespace plume {

// ---- status reporting (defined in sim.cu) -----------------------------------------------------------------
int fail(int status, const char* fmt, ...);
int launch_status(const char* what);                   // after a kernel launch: checks it and counts it
int runtime_status(const char* what, cudaError_t err);  // after any other runtime call
void count_launches(unsigned long long n);             // kernels enqueued another way (graph replays)
void set_launch_counting(bool on);

// ---- small vector type -----------------------------------------------------------------------------------
struct F3 {
  float c[3];
  __host__ __device__ __forceinline__ float& operator[](int a) { return c[a]; }
  __host__ __device__ __forceinline__ const float& operator[](int a) const { return c[a]; }
};
__host__ __device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{{x, y, z}}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return f3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return f3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
__device__ __forceinline__ F3 mul3(F3 a, float s) { return f3(a[0] * s, a[1] * s, a[2] * s); }
__device__ __forceinline__ F3 div3(F3 a, float s) { return f3(a[0] / s, a[1] / s, a[2] / s); }

// x / d where d is often a power of two (a grid spacing such as 1/64 m, its square, a child count). When d is
// a positive power of two whose reciprocal is a normal float, x * (1/d) multiplies by an exact 2^-e, so the
// product is the correctly rounded quotient: the same float as the IEEE division (this library never flushes
// subnormals), without the division's instruction sequence. Any other d divides.
struct Divisor {
  float d, inv;
  bool pow2;
};
__device__ __forceinline__ Divisor divisor(float d) {
  const unsigned bits = __float_as_uint(d), e = bits >> 23;  // sign bit 0 checked below, so e is the exponent
  const bool pow2 = (bits & 0x807fffffu) == 0u && e >= 1u && e <= 253u;
  return Divisor{d, __uint_as_float((254u - (pow2 ? e : 127u)) << 23), pow2};
}
__device__ __forceinline__ float divide(float x, const Divisor& q) { return q.pow2 ? x * q.inv : x / q.d; }
__device__ __forceinline__ F3 divide3(F3 a, const Divisor& q) {
  return f3(divide(a[0], q), divide(a[1], q), divide(a[2], q));
}
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ float len3(F3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ F3 normalize3(F3 a) { return div3(a, len3(a)); }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return f3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
__device__ __forceinline__ float fmin_(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ int imin_(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax_(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ float clampf_(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ float lerpf_(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ F3 lerp3(F3 a, F3 b, float t) {
  return f3(lerpf_(a[0], b[0], t), lerpf_(a[1], b[1], t), lerpf_(a[2], b[2], t));
}
__device__ __forceinline__ float exp_f(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float pow_f(float x, float y) { return (float)pow((double)x, (double)y); }

// ---- arrays ------------------------------------------------------------------------------------------------
struct Dims {
  int n0, n1, n2;
};
__device__ __forceinline__ int at(const Dims& d, int i, int j, int k) { return (i * d.n1 + j) * d.n2 + k; }
__host__ __device__ __forceinline__ Dims dims_of(const PlumeGridInfo& info) {
  return Dims{info.dims[0], info.dims[1], info.dims[2]};
}

// ---- field storage ----------------------------------------------------------------------------------------
// Velocity, smoke and temperature may be stored as float, bfloat16 or half (PLUME_STORAGE_*); every kernel
// loads them as float, computes in float and rounds once to the storage type (round to nearest even) when it
// stores. Pressure, divergence and all scratch stay float.
template <class T>
__device__ __forceinline__ float to_f(T x);
template <>
__device__ __forceinline__ float to_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <>
__device__ __forceinline__ float to_f<__half>(__half x) { return __half2float(x); }

template <class T>
__device__ __forceinline__ T from_f(float x);
template <>
__device__ __forceinline__ float from_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <>
__device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }

// read-only (non-coherent) load of an element that no thread of the kernel writes
template <class T>
__device__ __forceinline__ float ldg_f(const T* p) { return to_f<T>(__ldg(p)); }
// load / store of an element the kernel also writes
template <class T>
__device__ __forceinline__ float ld_f(const T* p) { return to_f<T>(*p); }
template <class T>
__device__ __forceinline__ void st_f(T* p, float x) { *p = from_f<T>(x); }

// A pair of values of the storage type (a clamp range): float2, __nv_bfloat162 or __half2.
template <class T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<__nv_bfloat16> { using type = __nv_bfloat162; };
template <> struct Pair<__half> { using type = __half2; };
template <class T>
using pair_t = typename Pair<T>::type;

template <class T>
__device__ __forceinline__ pair_t<T> make_pair_t(float lo, float hi) {
  pair_t<T> r;
  r.x = from_f<T>(lo);
  r.y = from_f<T>(hi);
  return r;
}

// One axis of a trilinear sample: the clamped position's lower index, the step to the upper corner (0 at the
// far edge) and the weights, computed once per axis. The clamp uses min/max, which differs from the reference's
// comparisons only in the sign of a zero (the same values follow).
struct Axis1 {
  int i0;
  int step;
  float t, one_minus_t;
};

__device__ __forceinline__ Axis1 axis_of(float g, int n, int stride) {
  const float x = fminf(fmaxf(g, 0.0f), (float)(n - 1));
  Axis1 a;
  a.i0 = (int)x;
  a.step = a.i0 < n - 1 ? stride : 0;
  a.t = x - (float)a.i0;
  a.one_minus_t = 1.0f - a.t;
  return a;
}

// lerp(a, b, t) = a*(1-t) + b*t with (1-t) precomputed: the same float operations.
__device__ __forceinline__ float lerp_w(float a, float b, const Axis1& w) { return a * w.one_minus_t + b * w.t; }

// Trilinear sample at continuous index g, clamped to the array (sim/sample.py:10-29).
template <class T>
__device__ __forceinline__ float sample_index_space(const T* __restrict__ f, const Dims& d, F3 g) {
  const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
  const T* p = f + (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  const float c00 = lerp_w(ldg_f(p), ldg_f(p + x.step), x);
  const float c10 = lerp_w(ldg_f(p + y.step), ldg_f(p + x.step + y.step), x);
  const float c01 = lerp_w(ldg_f(p + z.step), ldg_f(p + x.step + z.step), x);
  const float c11 = lerp_w(ldg_f(p + y.step + z.step), ldg_f(p + x.step + y.step + z.step), x);
  return lerp_w(lerp_w(c00, c10, y), lerp_w(c01, c11, y), z);
}

// The value and the min/max of the eight values a trilinear sample blends (sample.py:10-50), from one set
// of loads: MacCormack's forward pass and its clamp bounds read the same corners. The min/max run in the
// reference's corner order.
template <class T>
__device__ __forceinline__ float sample_with_range(const T* __restrict__ f, const Dims& d, F3 g, float& lo, float& hi) {
  const Axis1 x = axis_of(g[0], d.n0, d.n1 * d.n2), y = axis_of(g[1], d.n1, d.n2), z = axis_of(g[2], d.n2, 1);
  const T* p = f + (x.i0 * d.n1 + y.i0) * d.n2 + z.i0;
  const float a000 = ldg_f(p), a100 = ldg_f(p + x.step);
  const float a010 = ldg_f(p + y.step), a110 = ldg_f(p + x.step + y.step);
  const float a001 = ldg_f(p + z.step), a101 = ldg_f(p + x.step + z.step);
  const float a011 = ldg_f(p + y.step + z.step), a111 = ldg_f(p + x.step + y.step + z.step);
  lo = fmin_(fmin_(fmin_(fmin_(fmin_(fmin_(fmin_(a000, a000), a001), a010), a011), a100), a101), a110);
  lo = fmin_(lo, a111);
  hi = fmax_(fmax_(fmax_(fmax_(fmax_(fmax_(fmax_(a000, a000), a001), a010), a011), a100), a101), a110);
  hi = fmax_(hi, a111);
  const float c00 = lerp_w(a000, a100, x), c10 = lerp_w(a010, a110, x);
  const float c01 = lerp_w(a001, a101, x), c11 = lerp_w(a011, a111, x);
  return lerp_w(lerp_w(c00, c10, y), lerp_w(c01, c11, y), z);
}

__device__ __forceinline__ bool is_outside_open_face(F3 p, const PlumeGridInfo& info) {  // sample.py:53-61
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (p[a] < 0.0f && info.open_lo[a] == 1) return true;
    if (p[a] > (float)info.dims[a] && info.open_hi[a] == 1) return true;
  }
  return false;
}

template <class T>
struct VelT {
  const T* __restrict__ u;
  const T* __restrict__ v;
  const T* __restrict__ w;
  Dims du, dv, dw;
};
using Vel = VelT<float>;

template <class T>
__host__ __device__ __forceinline__ VelT<T> make_vel(const T* u, const T* v, const T* w, const int* dims) {
  VelT<T> r;
  r.u = u;
  r.v = v;
  r.w = w;
  r.du = Dims{dims[0] + 1, dims[1], dims[2]};
  r.dv = Dims{dims[0], dims[1] + 1, dims[2]};
  r.dw = Dims{dims[0], dims[1], dims[2] + 1};
  return r;
}

template <class T>
__device__ __forceinline__ F3 velocity_at(const VelT<T>& vel, F3 p) {  // sample.py:74-82
  // The three extents from one set of cell counts (make_vel's), so that the axes two components share (the
  // same coordinate and extent: x of v and w, y of u and w, z of u and v) are visibly one computation.
  const int nx = vel.dv.n0, ny = vel.du.n1, nz = vel.du.n2;
  const Dims du{nx + 1, ny, nz}, dv{nx, ny + 1, nz}, dw{nx, ny, nz + 1};
  return f3(sample_index_space(vel.u, du, sub3(p, f3(0.0f, 0.5f, 0.5f))),
            sample_index_space(vel.v, dv, sub3(p, f3(0.5f, 0.0f, 0.5f))),
            sample_index_space(vel.w, dw, sub3(p, f3(0.5f, 0.5f, 0.0f))));
}

// Midpoint backtrace (advect.py:16-21); a negative dt_over_cell traces forward.
template <class T>
__device__ __forceinline__ F3 trace(const VelT<T>& vel, F3 p, float dt_over_cell) {
  F3 mid = sub3(p, mul3(velocity_at(vel, p), 0.5f * dt_over_cell));
  return sub3(p, mul3(velocity_at(vel, mid), dt_over_cell));
}

// ---- advection traces (advect.py:16-21) shared by the forward kernels and their adjoints --------------------
// Every trace starts at a sample position p = index + offset, where each velocity component's trilinear
// weights are 0 or 1/2: velocity_at_node blends only the corners with a non-zero weight (the same values, up
// to the sign of a zero).
// Trilinear sample that skips the corners whose weight is exactly 0 (sample.py:10-29 otherwise unchanged).
template <class T>
__device__ __forceinline__ float sample_sparse(const T* __restrict__ f, const Dims& d, F3 g) {
  float x = clampf_(g[0], 0.0f, (float)(d.n0 - 1));
  float y = clampf_(g[1], 0.0f, (float)(d.n1 - 1));
  float z = clampf_(g[2], 0.0f, (float)(d.n2 - 1));
  const int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  const int i1 = imin_(i0 + 1, d.n0 - 1), j1 = imin_(j0 + 1, d.n1 - 1), k1 = imin_(k0 + 1, d.n2 - 1);
  const float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
  auto along_x = [&](int j, int k) {
    const float a = ldg_f(f + at(d, i0, j, k));
    return tx == 0.0f ? a : lerpf_(a, ldg_f(f + at(d, i1, j, k)), tx);
  };
  const float c00 = along_x(j0, k0);
  const float y0 = ty == 0.0f ? c00 : lerpf_(c00, along_x(j1, k0), ty);
  if (tz == 0.0f) return y0;
  const float c01 = along_x(j0, k1);
  const float y1 = ty == 0.0f ? c01 : lerpf_(c01, along_x(j1, k1), ty);
  return lerpf_(y0, y1, tz);
}

template <class T>
__device__ __forceinline__ F3 velocity_at_node(const VelT<T>& vel, F3 p) {  // velocity_at (sample.py:74-82) at p
  return f3(sample_sparse(vel.u, vel.du, sub3(p, f3(0.0f, 0.5f, 0.5f))),
            sample_sparse(vel.v, vel.dv, sub3(p, f3(0.5f, 0.0f, 0.5f))),
            sample_sparse(vel.w, vel.dw, sub3(p, f3(0.5f, 0.5f, 0.0f))));
}

// trace (advect.py:16-21) given the velocity at p.
template <class T>
__device__ __forceinline__ F3 trace_from(const VelT<T>& vel, F3 p, F3 vp, float dt_over_cell) {
  F3 mid = sub3(p, mul3(vp, 0.5f * dt_over_cell));
  return sub3(p, mul3(velocity_at(vel, mid), dt_over_cell));
}

// ---- value noise (sim/noise.py) ----------------------------------------------------------------------------
constexpr uint32_t LATTICE_OFFSET = 1048576u;

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {  // lowbias32 (noise.py:13-21)
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ float lattice_value(int seed, int stream, int i, int j, int k) {  // noise.py:24-32
  uint32_t h = hash_u32((uint32_t)seed + LATTICE_OFFSET);
  h = hash_u32(h ^ ((uint32_t)stream + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)i + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)j + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)k + LATTICE_OFFSET));
  const float scale = 2.0f / 16777215.0f;
  return (float)(h >> 8) * scale - 1.0f;
}

__device__ __forceinline__ float fade(float t) { return t * t * (3.0f - 2.0f * t); }

__device__ __forceinline__ float value_noise(int seed, int stream, F3 p) {  // noise.py:40-57
  float fx = floorf(p[0]), fy = floorf(p[1]), fz = floorf(p[2]);
  int i = (int)fx, j = (int)fy, k = (int)fz;
  float tx = fade(p[0] - fx), ty = fade(p[1] - fy), tz = fade(p[2] - fz);
  float c00 = lerpf_(lattice_value(seed, stream, i, j, k), lattice_value(seed, stream, i + 1, j, k), tx);
  float c10 = lerpf_(lattice_value(seed, stream, i, j + 1, k), lattice_value(seed, stream, i + 1, j + 1, k), tx);
  float c01 = lerpf_(lattice_value(seed, stream, i, j, k + 1), lattice_value(seed, stream, i + 1, j, k + 1), tx);
  float c11 = lerpf_(lattice_value(seed, stream, i, j + 1, k + 1),
                     lattice_value(seed, stream, i + 1, j + 1, k + 1), tx);
  return lerpf_(lerpf_(c00, c10, ty), lerpf_(c01, c11, ty), tz);
}

// ---- launch geometry ---------------------------------------------------------------------------------------
// Cell-parallel kernels use 256-thread blocks of 32 (z, the contiguous axis) x 8 (y), one x-slice per z-block.
constexpr int TZ = 32, TY = 8;
inline dim3 cell_grid(int n0, int n1, int n2) { return dim3((n2 + TZ - 1) / TZ, (n1 + TY - 1) / TY, n0); }
inline dim3 cell_block() { return dim3(TZ, TY, 1); }

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace plume
