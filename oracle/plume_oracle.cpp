// CPU restatement of the reference's fluid step and volume render -- TEST INFRASTRUCTURE ONLY.
//
// This file is the parity oracle: tests, the smoke check and the CPU-baseline leg of the benchmark call it
// through ctypes (oracle/oracle.py). No product code path links or calls it.
//
// It restates, operator by operator and in the same order of floating-point operations, the Warp kernels of
// chadmv/plume (paths below are relative to that project):
//   src/plume/sim/sample.py, advect.py, emitters.py, noise.py, forces.py, vorticity.py, turbulence.py,
//   pressure.py, multigrid.py, conserve.py, reduce.py, dissipate.py, step_cap.py,
//   src/plume/render/light_volume.py, normal_field.py, raymarch.py.
// Every function is templated on the field type T: T = float is the FP32 parity oracle, T = double is the
// FP64 "plain method" used for error bounds. Arithmetic is plain IEEE (build with -ffp-contract=off, no
// -ffast-math); exp and pow are the C library's at precision T; lerp(a, b, t) = a*(1-t) + b*t.
// Pinned: in FP32 this file reproduces the reference's own raw-frame SHA-256 digests (Warp 1.19 CPU, Linux,
// tests/render/test_raw_frame_digest.py:178-182) byte for byte in both channel layouts.
// Loops over cells run under OpenMP when it is enabled; every cell is independent within a pass, so the
// thread count never changes a result.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class T> struct V3 {
  T c[3];
  T& operator[](int a) { return c[a]; }
  const T& operator[](int a) const { return c[a]; }
};
template <class T> V3<T> mk(T x, T y, T z) { return V3<T>{{x, y, z}}; }
template <class T> V3<T> add(V3<T> a, V3<T> b) { return mk(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <class T> V3<T> sub(V3<T> a, V3<T> b) { return mk(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <class T> V3<T> mul(V3<T> a, T s) { return mk(a[0] * s, a[1] * s, a[2] * s); }
template <class T> V3<T> divs(V3<T> a, T s) { return mk(a[0] / s, a[1] / s, a[2] / s); }
template <class T> T dot(V3<T> a, V3<T> b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <class T> T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> V3<T> normalize(V3<T> a) { return divs(a, length(a)); }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
  return mk(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
template <class T> T tmin(T a, T b) { return a < b ? a : b; }
template <class T> T tmax(T a, T b) { return a > b ? a : b; }
inline int imin(int a, int b) { return a < b ? a : b; }
inline int imax(int a, int b) { return a > b ? a : b; }
template <class T> T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class T> T lerp(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <class T> V3<T> lerp3(V3<T> a, V3<T> b, T t) {
  return mk(lerp(a[0], b[0], t), lerp(a[1], b[1], t), lerp(a[2], b[2], t));
}
// exp and pow at the field's own precision (expf/powf for float, as Warp's CPU kernels call them).
template <class T> T exp_t(T x) { return std::exp(x); }
template <class T> T pow_t(T x, T y) { return std::pow(x, y); }

// ---- plain C views handed in through ctypes ------------------------------------------------------------

struct OInfo {  // GridInfo (sim/grid.py:21-33), every real in double; rounded to T on entry
  int dims[3];
  double cell_m;
  double origin_m[3];
  int open_lo[3];
  int open_hi[3];
  double fill_hi[3];
  double ghost_gap;
};

template <class T> struct Info {
  int dims[3];
  T cell_m;
  V3<T> origin;
  int open_lo[3], open_hi[3];
  V3<T> fill_hi;
  T ghost_gap;
  explicit Info(const OInfo& o) {
    for (int a = 0; a < 3; ++a) {
      dims[a] = o.dims[a];
      origin[a] = (T)o.origin_m[a];
      open_lo[a] = o.open_lo[a];
      open_hi[a] = o.open_hi[a];
      fill_hi[a] = (T)o.fill_hi[a];
    }
    cell_m = (T)o.cell_m;
    ghost_gap = (T)o.ghost_gap;
  }
};

template <class E> struct A3 {  // C-ordered (n0, n1, n2) array, n2 contiguous
  E* p;
  int n[3];
  E& at(int i, int j, int k) const { return p[((size_t)i * n[1] + j) * n[2] + k]; }
  size_t size() const { return (size_t)n[0] * n[1] * n[2]; }
};
template <class E> A3<E> a3(void* p, const int* shape) { return A3<E>{(E*)p, {shape[0], shape[1], shape[2]}}; }

// ---- sampling: sim/sample.py -----------------------------------------------------------------------------

template <class T> T sample_index_space(const A3<T>& f, V3<T> g) {  // sample.py:10-29
  T x = clampv(g[0], T(0), (T)(f.n[0] - 1));
  T y = clampv(g[1], T(0), (T)(f.n[1] - 1));
  T z = clampv(g[2], T(0), (T)(f.n[2] - 1));
  int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  int i1 = imin(i0 + 1, f.n[0] - 1), j1 = imin(j0 + 1, f.n[1] - 1), k1 = imin(k0 + 1, f.n[2] - 1);
  T tx = x - (T)i0, ty = y - (T)j0, tz = z - (T)k0;
  T c00 = lerp(f.at(i0, j0, k0), f.at(i1, j0, k0), tx);
  T c10 = lerp(f.at(i0, j1, k0), f.at(i1, j1, k0), tx);
  T c01 = lerp(f.at(i0, j0, k1), f.at(i1, j0, k1), tx);
  T c11 = lerp(f.at(i0, j1, k1), f.at(i1, j1, k1), tx);
  return lerp(lerp(c00, c10, ty), lerp(c01, c11, ty), tz);
}

template <class T> V3<T> sample_vec(const A3<T>& f, V3<T> g) {  // the same blend on a (n0,n1,n2,3) array
  T x = clampv(g[0], T(0), (T)(f.n[0] - 1));
  T y = clampv(g[1], T(0), (T)(f.n[1] - 1));
  T z = clampv(g[2], T(0), (T)(f.n[2] - 1));
  int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  int i1 = imin(i0 + 1, f.n[0] - 1), j1 = imin(j0 + 1, f.n[1] - 1), k1 = imin(k0 + 1, f.n[2] - 1);
  T tx = x - (T)i0, ty = y - (T)j0, tz = z - (T)k0;
  auto at = [&](int i, int j, int k) {
    const T* q = f.p + (((size_t)i * f.n[1] + j) * f.n[2] + k) * 3;
    return mk(q[0], q[1], q[2]);
  };
  V3<T> c00 = lerp3(at(i0, j0, k0), at(i1, j0, k0), tx);
  V3<T> c10 = lerp3(at(i0, j1, k0), at(i1, j1, k0), tx);
  V3<T> c01 = lerp3(at(i0, j0, k1), at(i1, j0, k1), tx);
  V3<T> c11 = lerp3(at(i0, j1, k1), at(i1, j1, k1), tx);
  return lerp3(lerp3(c00, c10, ty), lerp3(c01, c11, ty), tz);
}

template <class T> void range_index_space(const A3<T>& f, V3<T> g, T& lo, T& hi) {  // sample.py:32-50
  T x = clampv(g[0], T(0), (T)(f.n[0] - 1));
  T y = clampv(g[1], T(0), (T)(f.n[1] - 1));
  T z = clampv(g[2], T(0), (T)(f.n[2] - 1));
  int i0 = (int)x, j0 = (int)y, k0 = (int)z;
  lo = f.at(i0, j0, k0);
  hi = lo;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        T v = f.at(imin(i0 + di, f.n[0] - 1), imin(j0 + dj, f.n[1] - 1), imin(k0 + dk, f.n[2] - 1));
        lo = tmin(lo, v);
        hi = tmax(hi, v);
      }
}

template <class T> bool is_outside_open_face(V3<T> p, const Info<T>& info) {  // sample.py:53-61
  for (int a = 0; a < 3; ++a) {
    if (p[a] < T(0) && info.open_lo[a] == 1) return true;
    if (p[a] > (T)info.dims[a] && info.open_hi[a] == 1) return true;
  }
  return false;
}

template <class T>
T sample_field(const A3<T>& f, V3<T> p, V3<T> offset, const Info<T>& info, T outside, int uses_outside) {
  if (uses_outside == 1 && is_outside_open_face(p, info)) return outside;  // sample.py:64-71
  return sample_index_space(f, sub(p, offset));
}

template <class T> struct Vel {
  A3<T> u, v, w;
};

template <class T> V3<T> velocity_at(const Vel<T>& vel, V3<T> p) {  // sample.py:74-82
  return mk(sample_index_space(vel.u, sub(p, mk(T(0), T(0.5), T(0.5)))),
            sample_index_space(vel.v, sub(p, mk(T(0.5), T(0), T(0.5)))),
            sample_index_space(vel.w, sub(p, mk(T(0.5), T(0.5), T(0)))));
}

// ---- advection: sim/advect.py -----------------------------------------------------------------------------

template <class T> V3<T> trace(const Vel<T>& vel, V3<T> p, T dt_over_cell) {  // advect.py:16-21
  V3<T> mid = sub(p, mul(velocity_at(vel, p), T(0.5) * dt_over_cell));
  return sub(p, mul(velocity_at(vel, mid), dt_over_cell));
}

template <class T>
void semi_lagrangian(const A3<T>& src, const A3<T>& dst, const Vel<T>& vel, const Info<T>& info, T dt_over_cell,
                     V3<T> offset, T outside, int uses_outside) {  // advect.py:24-31
#pragma omp parallel for schedule(static)
  for (int i = 0; i < src.n[0]; ++i)
    for (int j = 0; j < src.n[1]; ++j)
      for (int k = 0; k < src.n[2]; ++k) {
        V3<T> p = add(mk((T)i, (T)j, (T)k), offset);
        dst.at(i, j, k) = sample_field(src, trace(vel, p, dt_over_cell), offset, info, outside, uses_outside);
      }
}

template <class T>
void maccormack_correct(const A3<T>& orig, const A3<T>& hat, const A3<T>& back, const A3<T>& dst,
                        const Vel<T>& vel, const Info<T>& info, T dt_over_cell, V3<T> offset, T outside,
                        int uses_outside) {  // advect.py:34-50
#pragma omp parallel for schedule(static)
  for (int i = 0; i < orig.n[0]; ++i)
    for (int j = 0; j < orig.n[1]; ++j)
      for (int k = 0; k < orig.n[2]; ++k) {
        V3<T> p = add(mk((T)i, (T)j, (T)k), offset);
        T corrected = hat.at(i, j, k) + T(0.5) * (orig.at(i, j, k) - back.at(i, j, k));
        V3<T> source = trace(vel, p, dt_over_cell);
        T lo = outside, hi = outside;
        if (uses_outside == 0 || !is_outside_open_face(source, info)) range_index_space(orig, sub(source, offset), lo, hi);
        dst.at(i, j, k) = clampv(corrected, lo, hi);
      }
}

// ---- noise: sim/noise.py ----------------------------------------------------------------------------------

constexpr uint32_t LATTICE_OFFSET = 1048576u;

inline uint32_t hash_u32(uint32_t x) {  // noise.py:13-21 (lowbias32)
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

template <class T> T lattice_value(int seed, int stream, int i, int j, int k) {  // noise.py:24-32
  uint32_t h = hash_u32((uint32_t)seed + LATTICE_OFFSET);
  h = hash_u32(h ^ ((uint32_t)stream + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)i + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)j + LATTICE_OFFSET));
  h = hash_u32(h ^ ((uint32_t)k + LATTICE_OFFSET));
  const T scale = T(2) / T(16777215);
  return (T)(h >> 8) * scale - T(1);
}

template <class T> T fade(T t) { return t * t * (T(3) - T(2) * t); }  // noise.py:35-37

template <class T> T value_noise(int seed, int stream, V3<T> p) {  // noise.py:40-57
  T fx = std::floor(p[0]), fy = std::floor(p[1]), fz = std::floor(p[2]);
  int i = (int)fx, j = (int)fy, k = (int)fz;
  T tx = fade(p[0] - fx), ty = fade(p[1] - fy), tz = fade(p[2] - fz);
  T c00 = lerp(lattice_value<T>(seed, stream, i, j, k), lattice_value<T>(seed, stream, i + 1, j, k), tx);
  T c10 = lerp(lattice_value<T>(seed, stream, i, j + 1, k), lattice_value<T>(seed, stream, i + 1, j + 1, k), tx);
  T c01 = lerp(lattice_value<T>(seed, stream, i, j, k + 1), lattice_value<T>(seed, stream, i + 1, j, k + 1), tx);
  T c11 = lerp(lattice_value<T>(seed, stream, i, j + 1, k + 1),
               lattice_value<T>(seed, stream, i + 1, j + 1, k + 1), tx);
  return lerp(lerp(c00, c10, ty), lerp(c01, c11, ty), tz);
}

// ---- emitters: sim/emitters.py ----------------------------------------------------------------------------

struct OEmitter {  // EmitterParams (emitters.py:23-38)
  int shape;
  double center_m[3];
  double radius_m;
  double half_size_m[3];
  double edge_softness;
  double start_s, end_s;
  double smoke_per_s;
  double temperature_k;
  double velocity_mps[3];
  int outward;
  double noise_scale_m, noise_strength;
  int stream;
};

template <class T> struct Emitter {
  int shape;
  V3<T> center;
  T radius;
  V3<T> half;
  T softness, start, end, smoke_per_s, temperature;
  V3<T> velocity;
  int outward;
  T noise_scale, noise_strength;
  int stream;
  explicit Emitter(const OEmitter& o) {
    shape = o.shape;
    for (int a = 0; a < 3; ++a) {
      center[a] = (T)o.center_m[a];
      half[a] = (T)o.half_size_m[a];
      velocity[a] = (T)o.velocity_mps[a];
    }
    radius = (T)o.radius_m;
    softness = (T)o.edge_softness;
    start = (T)o.start_s;
    end = (T)o.end_s;
    smoke_per_s = (T)o.smoke_per_s;
    temperature = (T)o.temperature_k;
    outward = o.outward;
    noise_scale = (T)o.noise_scale_m;
    noise_strength = (T)o.noise_strength;
    stream = o.stream;
  }
};

template <class T> T soft_edge(T distance, T extent, T softness) {  // emitters.py:41-50
  T inner = extent * (T(1) - softness);
  if (distance <= inner) return T(1);
  if (distance >= extent) return T(0);
  T t = (distance - inner) / (extent - inner);
  return T(1) - t * t * (T(3) - T(2) * t);
}

template <class T> T coverage(const Emitter<T>& e, V3<T> x, int seed) {  // emitters.py:53-67
  V3<T> offset = sub(x, e.center);
  T amount = T(0);
  if (e.shape == 0) {
    amount = soft_edge(length(offset), e.radius, e.softness);
  } else {
    amount = soft_edge(std::fabs(offset[0]), e.half[0], e.softness) *
             soft_edge(std::fabs(offset[1]), e.half[1], e.softness) *
             soft_edge(std::fabs(offset[2]), e.half[2], e.softness);
  }
  if (amount > T(0) && e.noise_strength > T(0)) {
    T breakup = T(1) + e.noise_strength * value_noise(seed, e.stream, divs(x, e.noise_scale));
    amount = amount * tmax(breakup, T(0));
  }
  return tmin(amount, T(1));
}

template <class T> T blend_factor(T amount, T dt) {  // emitters.py:70-77 (BLEND_REFERENCE_S = 1/80 s)
  const T reference = T(1) / T(80);
  return T(1) - pow_t(T(1) - amount, dt / reference);
}

template <class T> bool is_active(const Emitter<T>& e, T time_s) { return time_s >= e.start && time_s < e.end; }

template <class T> V3<T> world_position(const Info<T>& info, V3<T> index) { return add(info.origin, mul(index, info.cell_m)); }

template <class T>
void emit_scalars(const A3<T>& smoke, const A3<T>& temperature, const std::vector<Emitter<T>>& ems,
                  const Info<T>& info, int seed, T time_s, T dt) {  // emitters.py:90-102
#pragma omp parallel for schedule(static)
  for (int i = 0; i < smoke.n[0]; ++i)
    for (int j = 0; j < smoke.n[1]; ++j)
      for (int k = 0; k < smoke.n[2]; ++k) {
        V3<T> x = world_position(info, add(mk((T)i, (T)j, (T)k), mk(T(0.5), T(0.5), T(0.5))));
        for (const Emitter<T>& e : ems) {
          if (!is_active(e, time_s)) continue;
          T amount = coverage(e, x, seed);
          if (amount > T(0)) {
            smoke.at(i, j, k) = smoke.at(i, j, k) + e.smoke_per_s * amount * dt;
            temperature.at(i, j, k) = lerp(temperature.at(i, j, k), e.temperature, blend_factor(amount, dt));
          }
        }
      }
}

template <class T>
void emit_velocity(const A3<T>& comp, int axis, V3<T> offset, const std::vector<Emitter<T>>& ems,
                   const Info<T>& info, int seed, T time_s, T dt) {  // emitters.py:105-121
#pragma omp parallel for schedule(static)
  for (int i = 0; i < comp.n[0]; ++i)
    for (int j = 0; j < comp.n[1]; ++j)
      for (int k = 0; k < comp.n[2]; ++k) {
        V3<T> x = world_position(info, add(mk((T)i, (T)j, (T)k), offset));
        for (const Emitter<T>& e : ems) {
          if (!is_active(e, time_s)) continue;
          T amount = coverage(e, x, seed);
          if (amount > T(0)) {
            V3<T> target = e.velocity;
            if (e.outward == 1) {
              V3<T> away = sub(x, e.center);
              if (length(away) > T(0)) target = mul(normalize(away), length(e.velocity));
            }
            comp.at(i, j, k) = lerp(comp.at(i, j, k), target[axis], blend_factor(amount, dt));
          }
        }
      }
}

// ---- forces: sim/forces.py --------------------------------------------------------------------------------

template <class T>
void buoyancy(const A3<T>& v, const A3<T>& smoke, const A3<T>& temperature, const Info<T>& info, T gravity,
              T heat_buoyancy, T smoke_weight, T ambient, T dt) {  // forces.py:13-23
#pragma omp parallel for schedule(static)
  for (int i = 0; i < v.n[0]; ++i)
    for (int j = 0; j < v.n[1]; ++j)
      for (int k = 0; k < v.n[2]; ++k) {
        int below = imax(j - 1, 0), above = imin(j, info.dims[1] - 1);
        T heat = T(0.5) * (temperature.at(i, below, k) + temperature.at(i, above, k));
        T density = T(0.5) * (smoke.at(i, below, k) + smoke.at(i, above, k));
        T lift = heat_buoyancy * (heat - ambient) / ambient - smoke_weight * density;
        v.at(i, j, k) = v.at(i, j, k) + gravity * lift * dt;
      }
}

template <class T> void drag(const A3<T>& f, T wind, T keep) {  // forces.py:34-37
#pragma omp parallel for schedule(static)
  for (int i = 0; i < f.n[0]; ++i)
    for (int j = 0; j < f.n[1]; ++j)
      for (int k = 0; k < f.n[2]; ++k) f.at(i, j, k) = wind + (f.at(i, j, k) - wind) * keep;
}

// ---- vorticity confinement: sim/vorticity.py --------------------------------------------------------------

template <class T> struct VecField {  // (n0, n1, n2, 3)
  T* p;
  int n[3];
  V3<T> get(int i, int j, int k) const {
    const T* q = p + (((size_t)i * n[1] + j) * n[2] + k) * 3;
    return mk(q[0], q[1], q[2]);
  }
  void set(int i, int j, int k, V3<T> v) const {
    T* q = p + (((size_t)i * n[1] + j) * n[2] + k) * 3;
    q[0] = v[0];
    q[1] = v[1];
    q[2] = v[2];
  }
};

template <class T> void center_velocity(const Vel<T>& vel, const VecField<T>& center) {  // vorticity.py:17-22
#pragma omp parallel for schedule(static)
  for (int i = 0; i < center.n[0]; ++i)
    for (int j = 0; j < center.n[1]; ++j)
      for (int k = 0; k < center.n[2]; ++k)
        center.set(i, j, k, mk(T(0.5) * (vel.u.at(i, j, k) + vel.u.at(i + 1, j, k)),
                               T(0.5) * (vel.v.at(i, j, k) + vel.v.at(i, j + 1, k)),
                               T(0.5) * (vel.w.at(i, j, k) + vel.w.at(i, j, k + 1))));
}

template <class T> V3<T> central_difference(const VecField<T>& f, int c[3], int axis, const Info<T>& info) {
  int lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};  // vorticity.py:25-35
  lo[axis] = imax(c[axis] - 1, 0);
  hi[axis] = imin(c[axis] + 1, info.dims[axis] - 1);
  T span = (T)(hi[axis] - lo[axis]);
  if (span == T(0)) return mk(T(0), T(0), T(0));
  return divs(sub(f.get(hi[0], hi[1], hi[2]), f.get(lo[0], lo[1], lo[2])), span * info.cell_m);
}

template <class T> void curl_pass(const VecField<T>& center, const VecField<T>& curl, const Info<T>& info) {
#pragma omp parallel for schedule(static)  // vorticity.py:38-45
  for (int i = 0; i < center.n[0]; ++i)
    for (int j = 0; j < center.n[1]; ++j)
      for (int k = 0; k < center.n[2]; ++k) {
        int c[3] = {i, j, k};
        V3<T> dx = central_difference(center, c, 0, info);
        V3<T> dy = central_difference(center, c, 1, info);
        V3<T> dz = central_difference(center, c, 2, info);
        curl.set(i, j, k, mk(dy[2] - dz[1], dz[0] - dx[2], dx[1] - dy[0]));
      }
}

template <class T>
void confinement_push(const VecField<T>& curl, const VecField<T>& push, const Info<T>& info, T strength) {
#pragma omp parallel for schedule(static)  // vorticity.py:53-71
  for (int i = 0; i < curl.n[0]; ++i)
    for (int j = 0; j < curl.n[1]; ++j)
      for (int k = 0; k < curl.n[2]; ++k) {
        int c[3] = {i, j, k};
        V3<T> toward = mk(T(0), T(0), T(0));
        for (int a = 0; a < 3; ++a) {
          int lo[3] = {i, j, k}, hi[3] = {i, j, k};
          lo[a] = imax(c[a] - 1, 0);
          hi[a] = imin(c[a] + 1, info.dims[a] - 1);
          T span = (T)(hi[a] - lo[a]);
          if (span > T(0))
            toward[a] = (length(curl.get(hi[0], hi[1], hi[2])) - length(curl.get(lo[0], lo[1], lo[2]))) /
                        (span * info.cell_m);
        }
        T len = length(toward);
        if (len < (T)1.0e-12) {
          push.set(i, j, k, mk(T(0), T(0), T(0)));
          continue;
        }
        push.set(i, j, k, mul(cross(divs(toward, len), curl.get(i, j, k)), strength * info.cell_m));
      }
}

template <class T>
void add_face_push(const A3<T>& f, const VecField<T>& push, int axis, const Info<T>& info, T dt) {
#pragma omp parallel for schedule(static)  // vorticity.py:74-84
  for (int i = 0; i < f.n[0]; ++i)
    for (int j = 0; j < f.n[1]; ++j)
      for (int k = 0; k < f.n[2]; ++k) {
        int b[3] = {i, j, k}, a[3] = {i, j, k};
        b[axis] = imax(b[axis] - 1, 0);
        a[axis] = imin(a[axis], info.dims[axis] - 1);
        T average = T(0.5) * (push.get(b[0], b[1], b[2])[axis] + push.get(a[0], a[1], a[2])[axis]);
        f.at(i, j, k) = f.at(i, j, k) + average * dt;
      }
}

// ---- turbulence: sim/turbulence.py ------------------------------------------------------------------------

constexpr int TURBULENCE_STREAM = 1 << 24;

template <class T> T potential(int seed, int component, V3<T> p, T pattern_time) {  // turbulence.py:26-32
  T slice_lo = std::floor(pattern_time);
  T blend = fade(pattern_time - slice_lo);
  int first = TURBULENCE_STREAM + 3 * (int)slice_lo + component;
  return lerp(value_noise(seed, first, p), value_noise(seed, first + 3, p), blend);
}

template <class T>
void turbulence(const A3<T>& f, int axis, V3<T> offset, const Info<T>& info, int seed, T scale_m, T strength,
                T pattern_time, T dt) {  // turbulence.py:35-53
#pragma omp parallel for schedule(static)
  for (int i = 0; i < f.n[0]; ++i)
    for (int j = 0; j < f.n[1]; ++j)
      for (int k = 0; k < f.n[2]; ++k) {
        V3<T> face = add(mk((T)i, (T)j, (T)k), offset);
        int b = (axis + 1) % 3, c = (axis + 2) % 3;
        V3<T> half_b = mk(T(0), T(0), T(0)), half_c = mk(T(0), T(0), T(0));
        half_b[b] = T(0.5);
        half_c[c] = T(0.5);
        T to_lattice = info.cell_m / scale_m;
        T c_plus = potential(seed, c, mul(add(face, half_b), to_lattice), pattern_time);
        T c_minus = potential(seed, c, mul(sub(face, half_b), to_lattice), pattern_time);
        T b_plus = potential(seed, b, mul(add(face, half_c), to_lattice), pattern_time);
        T b_minus = potential(seed, b, mul(sub(face, half_c), to_lattice), pattern_time);
        T curl = ((c_plus - c_minus) - (b_plus - b_minus)) / to_lattice;
        f.at(i, j, k) = f.at(i, j, k) + strength * curl * dt;
      }
}

// ---- pressure: sim/pressure.py ----------------------------------------------------------------------------

template <class T> void zero_closed_faces(const A3<T>& f, int axis, const Info<T>& info) {  // pressure.py:21-28
#pragma omp parallel for schedule(static)
  for (int i = 0; i < f.n[0]; ++i)
    for (int j = 0; j < f.n[1]; ++j)
      for (int k = 0; k < f.n[2]; ++k) {
        int idx[3] = {i, j, k};
        int index = idx[axis];
        if (index == 0 && info.open_lo[axis] == 0) f.at(i, j, k) = T(0);
        if (index == info.dims[axis] && info.open_hi[axis] == 0) f.at(i, j, k) = T(0);
      }
}

template <class T> void divergence(const Vel<T>& vel, const A3<T>& div, const Info<T>& info) {  // pressure.py:31-36
#pragma omp parallel for schedule(static)
  for (int i = 0; i < div.n[0]; ++i)
    for (int j = 0; j < div.n[1]; ++j)
      for (int k = 0; k < div.n[2]; ++k) {
        T flux = (vel.u.at(i + 1, j, k) - vel.u.at(i, j, k)) + (vel.v.at(i, j + 1, k) - vel.v.at(i, j, k)) +
                 (vel.w.at(i, j, k + 1) - vel.w.at(i, j, k));
        div.at(i, j, k) = flux / info.cell_m;
      }
}

template <class T> T cell_fill(const Info<T>& info, int axis, int index) {  // pressure.py:39-44
  if (index == info.dims[axis] - 1) return info.fill_hi[axis];
  return T(1);
}

template <class T> T cell_volume(const Info<T>& info, const int c[3]) {  // pressure.py:47-49
  return cell_fill(info, 0, c[0]) * cell_fill(info, 1, c[1]) * cell_fill(info, 2, c[2]);
}

// pressure.py:52-69: (coupling * neighbour pressure, coupling) of one neighbour
template <class T> void neighbor_term(const A3<T>& q, const int c[3], int axis, int step, const Info<T>& info, T& tq, T& tc) {
  T area = T(1);
  for (int other = 0; other < 3; ++other)
    if (other != axis) area = area * cell_fill(info, other, c[other]);
  T own = cell_fill(info, axis, c[axis]);
  int n[3] = {c[0], c[1], c[2]};
  n[axis] = n[axis] + step;
  if (n[axis] >= 0 && n[axis] < info.dims[axis]) {
    T coupling = area / (T(0.5) * (own + cell_fill(info, axis, n[axis])));
    tq = coupling * q.at(n[0], n[1], n[2]);
    tc = coupling;
    return;
  }
  if ((step < 0 && info.open_lo[axis] == 1) || (step > 0 && info.open_hi[axis] == 1)) {
    tq = T(0);
    tc = area / (T(0.5) * own + info.ghost_gap);
    return;
  }
  tq = T(0);
  tc = T(0);
}

template <class T> void neighbor_sum(const A3<T>& q, const int c[3], const Info<T>& info, T& sq, T& sc) {
  sq = T(0);  // pressure.py:72-77
  sc = T(0);
  for (int axis = 0; axis < 3; ++axis) {
    T aq, ac, bq, bc;
    neighbor_term(q, c, axis, -1, info, aq, ac);
    neighbor_term(q, c, axis, 1, info, bq, bc);
    sq = (sq + aq) + bq;
    sc = (sc + ac) + bc;
  }
}

template <class T> void red_black_sweep(const A3<T>& q, const A3<T>& rhs, const Info<T>& info, int color, T relaxation) {
#pragma omp parallel for schedule(static)  // pressure.py:80-92
  for (int i = 0; i < q.n[0]; ++i)
    for (int j = 0; j < q.n[1]; ++j)
      for (int k = ((i + j + color) & 1); k < q.n[2]; k += 2) {
        int c[3] = {i, j, k};
        T sq, sc;
        neighbor_sum(q, c, info, sq, sc);
        if (sc == T(0)) continue;
        T source = cell_volume(info, c) * info.cell_m * info.cell_m * rhs.at(i, j, k);
        T target = (sq - source) / sc;
        q.at(i, j, k) = q.at(i, j, k) + relaxation * (target - q.at(i, j, k));
      }
}

template <class T> void red_black_sweeps(const A3<T>& q, const A3<T>& rhs, const Info<T>& info, int sweeps, T relaxation) {
  for (int s = 0; s < sweeps; ++s)  // pressure.py:135-141
    for (int color = 0; color < 2; ++color) red_black_sweep(q, rhs, info, color, relaxation);
}

template <class T> void subtract_gradient(const A3<T>& f, const A3<T>& q, int axis, const Info<T>& info) {
#pragma omp parallel for schedule(static)  // pressure.py:95-116
  for (int i = 0; i < f.n[0]; ++i)
    for (int j = 0; j < f.n[1]; ++j)
      for (int k = 0; k < f.n[2]; ++k) {
        int face[3] = {i, j, k};
        int index = face[axis];
        int below[3] = {i, j, k};
        below[axis] = index - 1;
        T q_above = T(0), q_below = T(0);
        if (index == 0) {
          if (info.open_lo[axis] == 0) continue;
          q_above = q.at(i, j, k);
        } else if (index == info.dims[axis]) {
          if (info.open_hi[axis] == 0) continue;
          q_below = q.at(below[0], below[1], below[2]);
        } else {
          q_above = q.at(i, j, k);
          q_below = q.at(below[0], below[1], below[2]);
        }
        f.at(i, j, k) = f.at(i, j, k) - (q_above - q_below) / info.cell_m;
      }
}

// ---- multigrid: sim/multigrid.py --------------------------------------------------------------------------

template <class T> void residual(const A3<T>& q, const A3<T>& rhs, const A3<T>& res, const Info<T>& info) {
#pragma omp parallel for schedule(static)  // multigrid.py:36-43
  for (int i = 0; i < q.n[0]; ++i)
    for (int j = 0; j < q.n[1]; ++j)
      for (int k = 0; k < q.n[2]; ++k) {
        int c[3] = {i, j, k};
        T sq, sc;
        neighbor_sum(q, c, info, sq, sc);
        T scale = cell_volume(info, c) * info.cell_m * info.cell_m;
        res.at(i, j, k) = rhs.at(i, j, k) - (sq - sc * q.at(i, j, k)) / scale;
      }
}

template <class T> void restrict_avg(const A3<T>& fine, const A3<T>& coarse) {  // multigrid.py:46-60
#pragma omp parallel for schedule(static)
  for (int i = 0; i < coarse.n[0]; ++i)
    for (int j = 0; j < coarse.n[1]; ++j)
      for (int k = 0; k < coarse.n[2]; ++k) {
        T total = T(0), count = T(0);
        for (int di = 0; di < 2; ++di)
          for (int dj = 0; dj < 2; ++dj)
            for (int dk = 0; dk < 2; ++dk) {
              int fi = 2 * i + di, fj = 2 * j + dj, fk = 2 * k + dk;
              if (fi < fine.n[0] && fj < fine.n[1] && fk < fine.n[2]) {
                total = total + fine.at(fi, fj, fk);
                count = count + T(1);
              }
            }
        coarse.at(i, j, k) = total / count;
      }
}

template <class T> void prolong_add(const A3<T>& coarse, const A3<T>& fine) {  // multigrid.py:63-68
#pragma omp parallel for schedule(static)
  for (int i = 0; i < fine.n[0]; ++i)
    for (int j = 0; j < fine.n[1]; ++j)
      for (int k = 0; k < fine.n[2]; ++k) {
        V3<T> g = sub(mul(mk((T)i, (T)j, (T)k), T(0.5)), mk(T(0.25), T(0.25), T(0.25)));
        fine.at(i, j, k) = fine.at(i, j, k) + sample_index_space(coarse, g);
      }
}

constexpr int COARSEST_SWEEPS = 20;  // multigrid.py:24-33
constexpr int COARSEST_SWEEPS_PER_CELL = 4;

template <class T> struct Level {
  Info<T> info;
  A3<T> q, rhs, res;
};

template <class T> void v_cycle(std::vector<Level<T>>& levels, size_t index, int sweeps) {  // multigrid.py:130-147
  Level<T>& lv = levels[index];
  if (index == levels.size() - 1) {
    int longest = std::max(lv.q.n[0], std::max(lv.q.n[1], lv.q.n[2]));
    int n = std::max(COARSEST_SWEEPS, COARSEST_SWEEPS_PER_CELL * longest);
    red_black_sweeps(lv.q, lv.rhs, lv.info, n, T(1.5));
    return;
  }
  red_black_sweeps(lv.q, lv.rhs, lv.info, sweeps, T(1));
  residual(lv.q, lv.rhs, lv.res, lv.info);
  Level<T>& coarse = levels[index + 1];
  restrict_avg(lv.res, coarse.rhs);
  std::memset(coarse.q.p, 0, coarse.q.size() * sizeof(T));
  v_cycle(levels, index + 1, sweeps);
  prolong_add(coarse.q, lv.q);
  red_black_sweeps(lv.q, lv.rhs, lv.info, sweeps, T(1));
}

// ---- reductions: sim/reduce.py, sim/conserve.py, sim/step_cap.py -----------------------------------------

// Each (j, k) line is summed along x in T, in order (reduce.py:12-25). The lines are then added in double in
// a fixed order shared with the device reduction: blocks of 256 consecutive lines (line index j*nz + k), each
// folded by a halving tree (slot s += slot s + h for h = 128, 64, ..., 1), then the block partials in order.
template <class T> double fixed_order_total(const A3<T>& a) {
  const int ny = a.n[1], nz = a.n[2];
  const long lines = (long)ny * nz;
  const long blocks = (lines + 255) / 256;
  std::vector<double> partial(blocks);
#pragma omp parallel for schedule(static)
  for (long b = 0; b < blocks; ++b) {
    double slot[256];
    for (int s = 0; s < 256; ++s) {
      long line = b * 256 + s;
      double v = 0.0;
      if (line < lines) {
        int j = (int)(line / nz), k = (int)(line % nz);
        T total = T(0);
        for (int i = 0; i < a.n[0]; ++i) total = total + a.at(i, j, k);
        v = (double)total;
      }
      slot[s] = v;
    }
    for (int h = 128; h >= 1; h >>= 1)
      for (int s = 0; s < h; ++s) slot[s] = slot[s] + slot[s + h];
    partial[b] = slot[0];
  }
  double total = 0.0;
  for (long b = 0; b < blocks; ++b) total = total + partial[b];
  return total;
}

template <class T> void scale_field(const A3<T>& f, T factor) {  // conserve.py:27-30
#pragma omp parallel for schedule(static)
  for (long n = 0; n < (long)f.size(); ++n) f.p[n] = f.p[n] * factor;
}

template <class T> void dissipate_fields(const A3<T>& smoke, const A3<T>& temperature, T smoke_keep, T heat_keep, T ambient) {
#pragma omp parallel for schedule(static)  // dissipate.py:10-15
  for (long n = 0; n < (long)smoke.size(); ++n) {
    smoke.p[n] = smoke.p[n] * smoke_keep;
    temperature.p[n] = ambient + (temperature.p[n] - ambient) * heat_keep;
  }
}

template <class T> T abs_max(const A3<T>& f) {  // step_cap.py:50-55 (max is exact in any order)
  T best = T(0);
#pragma omp parallel for reduction(max : best) schedule(static)
  for (long n = 0; n < (long)f.size(); ++n) {
    T v = std::fabs(f.p[n]);
    if (v > best) best = v;
  }
  return best;
}

// ---- render: render/raymarch.py, light_volume.py, normal_field.py ----------------------------------------

template <class T> void slab_range(V3<T> origin, V3<T> dir, V3<T> bmin, V3<T> bmax, T& t0out, T& t1out) {
  T t_enter = (T)-1.0e30, t_exit = (T)1.0e30;  // raymarch.py:55-69
  for (int a = 0; a < 3; ++a) {
    if (std::fabs(dir[a]) < (T)1.0e-12) {
      if (origin[a] < bmin[a] || origin[a] > bmax[a]) {
        t0out = T(1);
        t1out = T(0);
        return;
      }
    } else {
      T t0 = (bmin[a] - origin[a]) / dir[a];
      T t1 = (bmax[a] - origin[a]) / dir[a];
      t_enter = tmax(t_enter, tmin(t0, t1));
      t_exit = tmin(t_exit, tmax(t0, t1));
    }
  }
  t0out = t_enter;
  t1out = t_exit;
}

template <class T>
void light_volume(const A3<T>& smoke, V3<T> toward, T cell_m, T opacity, const A3<T>& light) {  // light_volume.py:18-33
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < smoke.n[0]; ++i)
    for (int j = 0; j < smoke.n[1]; ++j)
      for (int k = 0; k < smoke.n[2]; ++k) {
        V3<T> half = mk(T(0.5), T(0.5), T(0.5));
        V3<T> start = add(mk((T)i, (T)j, (T)k), half);
        V3<T> box_max = mk((T)smoke.n[0], (T)smoke.n[1], (T)smoke.n[2]);
        T t0, len;
        slab_range(start, toward, mk(T(0), T(0), T(0)), box_max, t0, len);
        int steps = (int)std::ceil(len / T(0.5));
        T column = T(0);
        if (steps > 0) {
          T step = len / (T)steps;
          for (int s = 0; s < steps; ++s) {
            V3<T> pos = add(start, mul(toward, ((T)s + T(0.5)) * step));
            column = column + tmax(sample_index_space(smoke, sub(pos, half)), T(0)) * step;
          }
        }
        light.at(i, j, k) = exp_t(-opacity * column * cell_m);
      }
}

template <class T> void blur_axis(const A3<T>& src, const A3<T>& dst, const T* weights, int radius, int axis) {
#pragma omp parallel for schedule(static)  // normal_field.py:12-22
  for (int i = 0; i < src.n[0]; ++i)
    for (int j = 0; j < src.n[1]; ++j)
      for (int k = 0; k < src.n[2]; ++k) {
        int c[3] = {i, j, k};
        T total = T(0);
        for (int o = -radius; o <= radius; ++o) {
          int n[3] = {i, j, k};
          n[axis] = std::min(std::max(c[axis] + o, 0), src.n[axis] - 1);
          total = total + weights[o + radius] * src.at(n[0], n[1], n[2]);
        }
        dst.at(i, j, k) = total;
      }
}

template <class T> void gradient_pass(const A3<T>& src, const VecField<T>& grad) {  // normal_field.py:25-38
#pragma omp parallel for schedule(static)
  for (int i = 0; i < src.n[0]; ++i)
    for (int j = 0; j < src.n[1]; ++j)
      for (int k = 0; k < src.n[2]; ++k) {
        int c[3] = {i, j, k};
        V3<T> r = mk(T(0), T(0), T(0));
        for (int a = 0; a < 3; ++a) {
          int lo[3] = {i, j, k}, hi[3] = {i, j, k};
          lo[a] = imax(c[a] - 1, 0);
          hi[a] = imin(c[a] + 1, src.n[a] - 1);
          T span = (T)(hi[a] - lo[a]);
          if (span > T(0)) r[a] = (src.at(hi[0], hi[1], hi[2]) - src.at(lo[0], lo[1], lo[2])) / span;
        }
        grad.set(i, j, k, r);
      }
}

struct OView {  // ViewParams (raymarch.py:30-42)
  double right[3], up[3], toward[3];
  double left_m, top_m, pixel_m;
  int perspective;
  double eye[3];
};
struct OLook {  // LookParams (raymarch.py:45-52)
  double opacity_per_density, glow_start_k, smoke_hides_heat, normal_fade_thickness;
  int shade_layout;
  double shade_fill;
};

template <class T>
void raymarch(const A3<T>& smoke, const A3<T>& temperature, const A3<T>& grad3, const A3<T>& light,
              const Info<T>& info, const OView& ov, const OLook& ol, T* image, int height, int width) {
  V3<T> right = mk((T)ov.right[0], (T)ov.right[1], (T)ov.right[2]);  // raymarch.py:86-140
  V3<T> up = mk((T)ov.up[0], (T)ov.up[1], (T)ov.up[2]);
  V3<T> toward = mk((T)ov.toward[0], (T)ov.toward[1], (T)ov.toward[2]);
  V3<T> eye = mk((T)ov.eye[0], (T)ov.eye[1], (T)ov.eye[2]);
  const T left_m = (T)ov.left_m, top_m = (T)ov.top_m, pixel_m = (T)ov.pixel_m;
  const T opacity = (T)ol.opacity_per_density, glow_start = (T)ol.glow_start_k, hides = (T)ol.smoke_hides_heat;
  const T fade_thickness = (T)ol.normal_fade_thickness, fill = (T)ol.shade_fill;
  const T far_m = (T)1.0e4;
#pragma omp parallel for schedule(dynamic, 1)
  for (int py = 0; py < height; ++py)
    for (int px = 0; px < width; ++px) {
      T plane_x = left_m + ((T)px + T(0.5)) * pixel_m;
      T plane_y = top_m - ((T)py + T(0.5)) * pixel_m;
      V3<T> origin = add(add(mul(right, plane_x), mul(up, plane_y)), mul(toward, far_m));
      V3<T> direction = mk(-toward[0], -toward[1], -toward[2]);
      if (ov.perspective == 1) {
        origin = eye;
        direction = normalize(sub(add(mul(right, plane_x), mul(up, plane_y)), toward));
      }
      V3<T> box_max = add(info.origin, mul(mk((T)info.dims[0], (T)info.dims[1], (T)info.dims[2]), info.cell_m));
      T s0, s1;
      slab_range(origin, direction, info.origin, box_max, s0, s1);
      if (ov.perspective == 1) s0 = tmax(s0, T(0));
      T tr = T(1), heat = T(0), shade_sum = T(0);
      V3<T> normal_sum = mk(T(0), T(0), T(0));
      if (s1 > s0) {
        T len = s1 - s0;
        int steps = (int)std::ceil(len / (T(0.5) * info.cell_m));
        T step_m = len / (T)steps;
        for (int s = 0; s < steps; ++s) {
          V3<T> position = add(origin, mul(direction, s0 + ((T)s + T(0.5)) * step_m));
          V3<T> g = sub(divs(sub(position, info.origin), info.cell_m), mk(T(0.5), T(0.5), T(0.5)));
          T density = tmax(sample_index_space(smoke, g), T(0));
          T alpha = T(1) - exp_t(-opacity * density * step_m);
          T glow = tmax(sample_index_space(temperature, g) - glow_start, T(0));
          heat = heat + glow * step_m * pow_t(tr, hides);
          if (ol.shade_layout == 1) {
            T lit = fill + (T(1) - fill) * sample_index_space(light, g);
            shade_sum = shade_sum + tr * alpha * lit;
          } else {
            V3<T> slope = sample_vec(grad3, g);
            if (alpha > T(0) && length(slope) > (T)1.0e-9)
              normal_sum = sub(normal_sum, mul(normalize(slope), tr * alpha));
          }
          tr = tr * (T(1) - alpha);
        }
      }
      T thickness = T(1) - tr;
      T* out = image + ((size_t)py * width + px) * 5;
      out[0] = heat;
      out[1] = thickness;
      if (ol.shade_layout == 1) {
        out[2] = shade_sum;
        out[3] = T(0);
        out[4] = T(0);
        continue;
      }
      V3<T> facing = mk(T(0), T(0), T(1));
      V3<T> normal = facing;
      V3<T> cam = mk(dot(normal_sum, right), dot(normal_sum, up), dot(normal_sum, toward));
      if (length(cam) > (T)1.0e-9) {
        normal = normalize(cam);
        normal = mk(normal[0], normal[1], std::fabs(normal[2]));
        T weight = clampv(thickness / fade_thickness, T(0), T(1));
        normal = normalize(lerp3(facing, normal, weight));
      }
      out[2] = normal[0];
      out[3] = normal[1];
      out[4] = normal[2];
    }
}

template <class T> V3<T> v3d(const double* d) { return mk((T)d[0], (T)d[1], (T)d[2]); }

template <class T> Vel<T> vel_of(void* u, void* v, void* w, const int* dims) {
  int su[3] = {dims[0] + 1, dims[1], dims[2]}, sv[3] = {dims[0], dims[1] + 1, dims[2]},
      sw[3] = {dims[0], dims[1], dims[2] + 1};
  return Vel<T>{a3<T>(u, su), a3<T>(v, sv), a3<T>(w, sw)};
}

template <class T> std::vector<Emitter<T>> emitters_of(const OEmitter* e, int count) {
  std::vector<Emitter<T>> out;
  for (int n = 0; n < count; ++n) out.emplace_back(e[n]);
  return out;
}

}  // namespace

// ---- C ABI (ctypes) ------------------------------------------------------------------------------------
// Every entry point exists as _f32 (T = float) and _f64 (T = double). Arrays are C-contiguous; `shape` is
// the array's own (n0, n1, n2); face arrays take the grid's `dims` and derive their shapes.

#define PLUME_ORACLE_BOTH(DECL) DECL(f32, float) DECL(f64, double)

#define DECL_ADVECT(S, T)                                                                                       \
  extern "C" void oracle_semi_lagrangian_##S(const OInfo* oi, const int* shape, void* src, void* dst, void* u,  \
                                             void* v, void* w, double dt_over_cell, const double* offset,     \
                                             double outside, int uses_outside) {                              \
    Info<T> info(*oi);                                                                                         \
    semi_lagrangian(a3<T>(src, shape), a3<T>(dst, shape), vel_of<T>(u, v, w, oi->dims), info,                \
                    (T)dt_over_cell, v3d<T>(offset), (T)outside, uses_outside);                               \
  }                                                                                                            \
  extern "C" void oracle_maccormack_##S(const OInfo* oi, const int* shape, void* data, void* hat, void* back,   \
                                        void* next, void* u, void* v, void* w, double dt_over_cell,            \
                                        const double* offset, double outside, int uses_outside) {              \
    Info<T> info(*oi);                                                                                         \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    T dtc = (T)dt_over_cell;                                                                                   \
    semi_lagrangian(a3<T>(data, shape), a3<T>(hat, shape), vel, info, dtc, v3d<T>(offset), (T)outside,       \
                    uses_outside);                                                                             \
    semi_lagrangian(a3<T>(hat, shape), a3<T>(back, shape), vel, info, (T)(-dtc), v3d<T>(offset), (T)outside, \
                    uses_outside);                                                                             \
    maccormack_correct(a3<T>(data, shape), a3<T>(hat, shape), a3<T>(back, shape), a3<T>(next, shape), vel,   \
                       info, dtc, v3d<T>(offset), (T)outside, uses_outside);                                   \
  }
PLUME_ORACLE_BOTH(DECL_ADVECT)

#define DECL_EMIT(S, T)                                                                                         \
  extern "C" void oracle_emit_##S(const OInfo* oi, void* smoke, void* temperature, void* u, void* v, void* w,    \
                                  const OEmitter* ems, int count, int seed, double time_s, double dt) {         \
    Info<T> info(*oi);                                                                                         \
    auto e = emitters_of<T>(ems, count);                                                                       \
    emit_scalars(a3<T>(smoke, oi->dims), a3<T>(temperature, oi->dims), e, info, seed, (T)time_s, (T)dt);      \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    const A3<T>* comps[3] = {&vel.u, &vel.v, &vel.w};                                                          \
    const V3<T> offs[3] = {mk(T(0), T(0.5), T(0.5)), mk(T(0.5), T(0), T(0.5)), mk(T(0.5), T(0.5), T(0))};     \
    for (int a = 0; a < 3; ++a) emit_velocity(*comps[a], a, offs[a], e, info, seed, (T)time_s, (T)dt);        \
  }
PLUME_ORACLE_BOTH(DECL_EMIT)

#define DECL_FORCES(S, T)                                                                                       \
  extern "C" void oracle_buoyancy_##S(const OInfo* oi, void* v, void* smoke, void* temperature, double gravity, \
                                      double heat_buoyancy, double smoke_weight, double ambient, double dt) {  \
    Info<T> info(*oi);                                                                                         \
    int sv[3] = {oi->dims[0], oi->dims[1] + 1, oi->dims[2]};                                                   \
    buoyancy(a3<T>(v, sv), a3<T>(smoke, oi->dims), a3<T>(temperature, oi->dims), info, (T)gravity,            \
             (T)heat_buoyancy, (T)smoke_weight, (T)ambient, (T)dt);                                            \
  }                                                                                                            \
  extern "C" void oracle_drag_##S(const int* shape, void* f, double wind, double keep) {                       \
    drag(a3<T>(f, shape), (T)wind, (T)keep);                                                                   \
  }                                                                                                            \
  extern "C" void oracle_confinement_##S(const OInfo* oi, void* u, void* v, void* w, void* center, void* curl,  \
                                         void* push, double strength, double dt, int apply) {                  \
    Info<T> info(*oi);                                                                                         \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    VecField<T> c{(T*)center, {oi->dims[0], oi->dims[1], oi->dims[2]}};                                        \
    VecField<T> cu{(T*)curl, {oi->dims[0], oi->dims[1], oi->dims[2]}};                                         \
    VecField<T> pu{(T*)push, {oi->dims[0], oi->dims[1], oi->dims[2]}};                                         \
    center_velocity(vel, c);                                                                                   \
    curl_pass(c, cu, info);                                                                                    \
    if (!apply) return;                                                                                        \
    confinement_push(cu, pu, info, (T)strength);                                                               \
    add_face_push(vel.u, pu, 0, info, (T)dt);                                                                  \
    add_face_push(vel.v, pu, 1, info, (T)dt);                                                                  \
    add_face_push(vel.w, pu, 2, info, (T)dt);                                                                  \
  }                                                                                                            \
  extern "C" void oracle_turbulence_##S(const OInfo* oi, void* u, void* v, void* w, int seed, double scale_m,   \
                                        double strength, double pattern_time, double dt) {                     \
    Info<T> info(*oi);                                                                                         \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    const A3<T>* comps[3] = {&vel.u, &vel.v, &vel.w};                                                          \
    const V3<T> offs[3] = {mk(T(0), T(0.5), T(0.5)), mk(T(0.5), T(0), T(0.5)), mk(T(0.5), T(0.5), T(0))};     \
    for (int a = 0; a < 3; ++a)                                                                                \
      turbulence(*comps[a], a, offs[a], info, seed, (T)scale_m, (T)strength, (T)pattern_time, (T)dt);         \
  }
PLUME_ORACLE_BOTH(DECL_FORCES)

#define DECL_PRESSURE(S, T)                                                                                     \
  extern "C" void oracle_zero_closed_faces_##S(const OInfo* oi, void* u, void* v, void* w) {                    \
    Info<T> info(*oi);                                                                                         \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    zero_closed_faces(vel.u, 0, info);                                                                         \
    zero_closed_faces(vel.v, 1, info);                                                                         \
    zero_closed_faces(vel.w, 2, info);                                                                         \
  }                                                                                                            \
  extern "C" void oracle_divergence_##S(const OInfo* oi, void* u, void* v, void* w, void* div) {               \
    Info<T> info(*oi);                                                                                         \
    divergence(vel_of<T>(u, v, w, oi->dims), a3<T>(div, oi->dims), info);                                     \
  }                                                                                                            \
  extern "C" void oracle_red_black_sweeps_##S(const OInfo* oi, void* q, void* rhs, int sweeps, double relax) {  \
    Info<T> info(*oi);                                                                                         \
    red_black_sweeps(a3<T>(q, oi->dims), a3<T>(rhs, oi->dims), info, sweeps, (T)relax);                       \
  }                                                                                                            \
  extern "C" void oracle_subtract_gradient_##S(const OInfo* oi, void* u, void* v, void* w, void* q) {           \
    Info<T> info(*oi);                                                                                         \
    Vel<T> vel = vel_of<T>(u, v, w, oi->dims);                                                                 \
    A3<T> qa = a3<T>(q, oi->dims);                                                                             \
    subtract_gradient(vel.u, qa, 0, info);                                                                     \
    subtract_gradient(vel.v, qa, 1, info);                                                                     \
    subtract_gradient(vel.w, qa, 2, info);                                                                     \
  }                                                                                                            \
  extern "C" void oracle_residual_##S(const OInfo* oi, void* q, void* rhs, void* res) {                        \
    Info<T> info(*oi);                                                                                         \
    residual(a3<T>(q, oi->dims), a3<T>(rhs, oi->dims), a3<T>(res, oi->dims), info);                           \
  }                                                                                                            \
  extern "C" void oracle_multigrid_##S(int nlevels, const OInfo* infos, void** q, void** rhs, void** res,      \
                                       int cycles, int sweeps) {                                               \
    std::vector<Level<T>> levels;                                                                              \
    for (int l = 0; l < nlevels; ++l)                                                                          \
      levels.push_back(Level<T>{Info<T>(infos[l]), a3<T>(q[l], infos[l].dims), a3<T>(rhs[l], infos[l].dims),  \
                                a3<T>(res[l], infos[l].dims)});                                                \
    for (int c = 0; c < cycles; ++c) v_cycle(levels, 0, sweeps);                                              \
  }
PLUME_ORACLE_BOTH(DECL_PRESSURE)

#define DECL_SCALARS(S, T)                                                                                      \
  extern "C" double oracle_total_##S(const int* shape, void* f) { return fixed_order_total(a3<T>(f, shape)); }  \
  extern "C" void oracle_scale_##S(const int* shape, void* f, double factor) {                                 \
    scale_field(a3<T>(f, shape), (T)factor);                                                                   \
  }                                                                                                            \
  extern "C" void oracle_dissipate_##S(const int* shape, void* smoke, void* temperature, double smoke_keep,    \
                                       double heat_keep, double ambient) {                                     \
    dissipate_fields(a3<T>(smoke, shape), a3<T>(temperature, shape), (T)smoke_keep, (T)heat_keep, (T)ambient);\
  }                                                                                                            \
  extern "C" double oracle_abs_max_##S(const int* shape, void* f) { return (double)abs_max(a3<T>(f, shape)); }
PLUME_ORACLE_BOTH(DECL_SCALARS)

#define DECL_RENDER(S, T)                                                                                       \
  extern "C" void oracle_light_volume_##S(const int* shape, void* smoke, const double* toward, double cell_m,   \
                                          double opacity, void* light) {                                       \
    light_volume(a3<T>(smoke, shape), v3d<T>(toward), (T)cell_m, (T)opacity, a3<T>(light, shape));            \
  }                                                                                                            \
  extern "C" void oracle_normal_field_##S(const int* shape, void* smoke, void* blurred, void* scratch,          \
                                          void* gradient, const void* weights, int radius) {                   \
    A3<T> s = a3<T>(smoke, shape), b = a3<T>(blurred, shape), c = a3<T>(scratch, shape);                       \
    const T* wts = (const T*)weights;                                                                          \
    blur_axis(s, b, wts, radius, 0);                                                                           \
    blur_axis(b, c, wts, radius, 1);                                                                           \
    blur_axis(c, b, wts, radius, 2);                                                                           \
    gradient_pass(b, VecField<T>{(T*)gradient, {shape[0], shape[1], shape[2]}});                              \
  }                                                                                                            \
  extern "C" void oracle_raymarch_##S(const OInfo* oi, void* smoke, void* temperature, void* gradient,          \
                                      const int* gshape, void* light, const int* lshape, const OView* view,    \
                                      const OLook* look, void* image, int height, int width) {                 \
    Info<T> info(*oi);                                                                                         \
    raymarch(a3<T>(smoke, oi->dims), a3<T>(temperature, oi->dims), a3<T>(gradient, gshape),                  \
             a3<T>(light, lshape), info, *view, *look, (T*)image, height, width);                              \
  }
PLUME_ORACLE_BOTH(DECL_RENDER)

extern "C" int oracle_threads(int wanted) {
#ifdef _OPENMP
  if (wanted > 0) omp_set_num_threads(wanted);
  return omp_get_max_threads();
#else
  (void)wanted;
  return 1;
#endif
}
