// Fused clamped-MacCormack advection for sm_100a: forward trace, backward trace and limiter in one pass.
//
// Reference: advect_maccormack and its kernels (src/plume/sim/advect.py:16-68) with the sampling functions of
// src/plume/sim/sample.py:10-82. The reference makes three full-grid passes per field (semi-Lagrangian into
// `hat`, semi-Lagrangian of `hat` backward into `back`, then the clamped correction) and re-reads the
// velocity for every trace. Here one kernel does all three for the three velocity components, and another for
// smoke and temperature together:
//
// - A block owns a tile of TY x TZ elements in (y, z) and marches along x over a segment of planes. The
//   velocity components (and, for the scalars, smoke and temperature) of the planes the traces can reach are
//   staged in shared memory: a ring of planes, each plane the tile plus two cells on every side, with indices
//   clamped at the array edges (edge replication). Every trilinear sample then reads 8 shared-memory words at
//   fixed offsets from one index.
// - `hat` (the forward semi-Lagrangian value) is computed for the tile plus a one-cell ring in (y, z), one
//   plane ahead of the correction, into a ring of hat planes in shared memory; it never goes to HBM. The
//   correction traces backward and samples that ring, so HBM sees each input read once and `next` written once.
// - A trace is only taken from shared memory when it stays inside the staged planes: |v| dt / dx < REACH at
//   the element and at the midpoint. Otherwise that element's hat, or its backward sample, is evaluated from
//   global memory with the same arithmetic (clamped indices), so results do not depend on which path ran.
//
// Arithmetic: positions, traces and the limiter keep the reference's float operations and their order. The
// trilinear blends use lerp(a, b, t) = fma(t, b - a, a) (one rounding fewer than a*(1-t) + b*t); values agree
// with the reference to about an ulp. With edge replication the lower clamp of each coordinate is the only
// clamp needed: a coordinate above n-1 blends two equal values, which the fma form returns exactly, and the
// min/max range covers the same corner values as range_index_space (sample.py:33-50), whose corners are
// those of the coordinate clamped into [0, n-1].
//
// The smoke budget's line totals (reduce.py:12-25) come out of the scalar march: each thread walks its
// (y, z) line along x and adds data, hat and next in float, per segment; k_segment_lines adds the segments of
// each line in order and the lines in double. Temperature's dissipation (dissipate.py:10-15) is applied as
// it is stored.
#include <algorithm>
#include <cstdlib>

#include "advect.cuh"

namespace plume {
namespace mac {

// Tile height: 8 rows (256 threads, four blocks per SM). Measured on B200 at 256x384x256, velocity advection:
// 2.25 ms at 8 rows, 2.31 ms at 16 (512 threads, two blocks per SM).
#ifndef PLUME_MAC_TY
#define PLUME_MAC_TY 8
#endif
constexpr int TY = PLUME_MAC_TY, TZ = 32, NT = TY * TZ;   // tile of one block: TY x 32 elements per plane
constexpr int BLOCKS_PER_SM = 1024 / NT;                // 512 threads: 2 blocks per SM, 256: 4
// Plane strides are padded to a multiple of 32 floats, so that samples in neighbouring planes of the same row
// and column fall in the same bank only for the same lane position (planes 720 floats apart would put lanes 16
// columns apart in one bank).
constexpr int pad32(int n) { return (n + 31) / 32 * 32; }
constexpr int RZ = TZ + 4, RY = TY + 4, RP = pad32(RY * RZ);  // staged plane: rows j0-2..j0+TY+1, cols k0-2..k0+TZ+1
constexpr int HZ = TZ + 2, HY = TY + 2, HP = pad32(HY * HZ);  // hat plane: rows j0-1..j0+TY, cols k0-1..k0+TZ
constexpr int HALO = HY * HZ - NT;                        // the hat plane's one-cell ring (84 elements at TY 8)
constexpr int VR = 8;                                     // velocity ring: planes i-1..i+2 in use, i+3 landing
constexpr int SR = 4;                                     // smoke/temperature ring: planes i..i+2, i+3 landing
constexpr int HR = 4;                                     // hat ring: planes i-1..i+1 read, i+2 written next
constexpr float REACH = 0.98f;                            // trace reach (cells) served from shared memory
constexpr int RPN = RY * RZ;                              // staged elements per plane
constexpr int STAGE_PER_THREAD = (RPN + NT - 1) / NT;

__device__ __forceinline__ float lerpm(float a, float b, float t) { return __fmaf_rn(t, b - a, a); }

// One axis of a sample: the coordinate clamped below at 0 (as sample.py's clamp), its floor and fraction.
struct Ax {
  int i;
  float t;
};
__device__ __forceinline__ Ax split(float g) {
  const float x = fmaxf(g, 0.0f);
  const float f = floorf(x);
  return Ax{(int)f, x - f};
}

// The 8 corners in the order a[dx + 2 dy + 4 dz].
__device__ __forceinline__ float blend8(const float* a, float tx, float ty, float tz) {
  const float c00 = lerpm(a[0], a[1], tx), c10 = lerpm(a[2], a[3], tx);
  const float c01 = lerpm(a[4], a[5], tx), c11 = lerpm(a[6], a[7], tx);
  return lerpm(lerpm(c00, c10, ty), lerpm(c01, c11, ty), tz);
}

__device__ __forceinline__ void range8(const float* a, float& lo, float& hi) {
  lo = fminf(fminf(fminf(a[0], a[1]), fminf(a[2], a[3])), fminf(fminf(a[4], a[5]), fminf(a[6], a[7])));
  hi = fmaxf(fmaxf(fmaxf(a[0], a[1]), fmaxf(a[2], a[3])), fmaxf(fmaxf(a[4], a[5]), fmaxf(a[6], a[7])));
}

// Corners from a ring of R staged planes; `inplane` = y * RZ + z - rowbase (the staged row and column).
template <int R, int S>
__device__ __forceinline__ void ring_corners(const float* ring, int x, int inplane, float* a) {
  const float* p0 = ring + (x & (R - 1)) * S + inplane;
  const float* p1 = ring + ((x + 1) & (R - 1)) * S + inplane;
  a[0] = p0[0];
  a[1] = p1[0];
  a[2] = p0[RZ];
  a[3] = p1[RZ];
  a[4] = p0[1];
  a[5] = p1[1];
  a[6] = p0[RZ + 1];
  a[7] = p1[RZ + 1];
}

// Corners from global memory, indices clamped to the array as sample.py does.
template <class T>
__device__ __forceinline__ void global_corners(const T* __restrict__ f, const Dims& d, int x, int y, int z, float* a) {
  const int x0 = imin_(x, d.n0 - 1), x1 = imin_(x + 1, d.n0 - 1);
  const int y0 = imin_(y, d.n1 - 1), y1 = imin_(y + 1, d.n1 - 1);
  const int z0 = imin_(z, d.n2 - 1), z1 = imin_(z + 1, d.n2 - 1);
  a[0] = ldg_f(f + at(d, x0, y0, z0));
  a[1] = ldg_f(f + at(d, x1, y0, z0));
  a[2] = ldg_f(f + at(d, x0, y1, z0));
  a[3] = ldg_f(f + at(d, x1, y1, z0));
  a[4] = ldg_f(f + at(d, x0, y0, z1));
  a[5] = ldg_f(f + at(d, x1, y0, z1));
  a[6] = ldg_f(f + at(d, x0, y1, z1));
  a[7] = ldg_f(f + at(d, x1, y1, z1));
}

template <class T>
struct Args {
  PlumeGridInfo info;
  const T* vel[3];      // u, v, w: the velocity the traces follow (and, for G < 3, the advected field)
  const T* field[2];    // smoke, temperature (the scalar march)
  T* next[3];           // u, v, w next (velocity march) or smoke, temperature next (scalar march)
  float outside[2];     // the scalars' values beyond open faces
  int uses_outside;
  float dt;             // dt / cell_m
  int seg_len;          // planes per block along x
  int segs[4];          // segments per group (u, v, w; or the cells)
  float* partials;      // scalar march: float line sums [3][segs][ny * nz] (data, hat, next of smoke)
  int dissipate;        // scalar march: temperature = ambient + (T - ambient) * heat_keep on store
  float heat_keep, ambient;
};

// Position offset of group G's elements (u, v, w faces; 3 = cell centres).
template <int G>
__device__ __forceinline__ F3 offset_of() {
  return f3(G == 0 ? 0.0f : 0.5f, G == 1 ? 0.0f : 0.5f, G == 2 ? 0.0f : 0.5f);
}

__device__ __forceinline__ Dims group_dims(const PlumeGridInfo& info, int g) {
  return Dims{info.dims[0] + (g == 0), info.dims[1] + (g == 1), info.dims[2] + (g == 2)};
}

__device__ __forceinline__ float maxabs3(F3 v) { return fmaxf(fmaxf(fabsf(v[0]), fabsf(v[1])), fabsf(v[2])); }

// ---- velocity at a point (sample.py:74-82), from the staged ring or from global memory --------------------
// The three components' axes are split once: x of v and w, y of u and w, z of u and v are the same
// coordinate minus 1/2.
template <int S>
__device__ __forceinline__ F3 ring_velocity(const float* vring, int rowbase, F3 m) {
  const Ax x0 = split(m[0]), x1 = split(m[0] - 0.5f);
  const Ax y0 = split(m[1]), y1 = split(m[1] - 0.5f);
  const Ax z0 = split(m[2]), z1 = split(m[2] - 0.5f);
  float a[8];
  ring_corners<VR, S>(vring, x0.i, y1.i * RZ + z1.i - rowbase, a);
  const float u = blend8(a, x0.t, y1.t, z1.t);
  ring_corners<VR, S>(vring + VR * S, x1.i, y0.i * RZ + z1.i - rowbase, a);
  const float v = blend8(a, x1.t, y0.t, z1.t);
  ring_corners<VR, S>(vring + 2 * VR * S, x1.i, y1.i * RZ + z0.i - rowbase, a);
  const float w = blend8(a, x1.t, y1.t, z0.t);
  return f3(u, v, w);
}

template <class T>
__device__ __forceinline__ F3 global_velocity(const Args<T>& A, F3 m) {
  const int nx = A.info.dims[0], ny = A.info.dims[1], nz = A.info.dims[2];
  const Ax x0 = split(m[0]), x1 = split(m[0] - 0.5f);
  const Ax y0 = split(m[1]), y1 = split(m[1] - 0.5f);
  const Ax z0 = split(m[2]), z1 = split(m[2] - 0.5f);
  float a[8];
  global_corners(A.vel[0], Dims{nx + 1, ny, nz}, x0.i, y1.i, z1.i, a);
  const float u = blend8(a, x0.t, y1.t, z1.t);
  global_corners(A.vel[1], Dims{nx, ny + 1, nz}, x1.i, y0.i, z1.i, a);
  const float v = blend8(a, x1.t, y0.t, z1.t);
  global_corners(A.vel[2], Dims{nx, ny, nz + 1}, x1.i, y1.i, z0.i, a);
  const float w = blend8(a, x1.t, y1.t, z0.t);
  return f3(u, v, w);
}

// ---- velocity at an element's own position (velocity_at at p = index + offset) ----------------------------
// Each component's trilinear weights there are 0 or 1/2: the component sampled on its own faces is read
// directly; for the others, the axis of the component sits half a cell above (corners c, c+1) and the axis of
// the element's group half a cell below (corners c-1, c), blended at 1/2 in the reference's axis order.
// Cells: each component sits half a cell above along its own axis. At the walls the clamp of sample.py keeps
// one corner; the staged ring's edge replication and the global path's clamped indices both give that value.
template <int G, int C>
struct Node {
  // direction of the half-cell shift of component C's sample along each axis: +1 above, -1 below, 0 none
  static constexpr int shift(int axis) {
    return G == 3 ? (axis == C ? 1 : 0) : (G == C ? 0 : (axis == C ? 1 : (axis == G ? -1 : 0)));
  }
  static constexpr int sx = shift(0), sy = shift(1), sz = shift(2);
};

// blend of one component at the element from a corner accessor load(dx, dy, dz)
template <int G, int C, class Load>
__device__ __forceinline__ float node_component(Load load) {
  using N = Node<G, C>;
  constexpr int ax0 = N::sx < 0 ? -1 : 0, ax1 = N::sx > 0 ? 1 : 0;
  constexpr int ay0 = N::sy < 0 ? -1 : 0, ay1 = N::sy > 0 ? 1 : 0;
  constexpr int az0 = N::sz < 0 ? -1 : 0, az1 = N::sz > 0 ? 1 : 0;
  auto along_x = [&](int dy, int dz) {
    const float a = load(ax0, dy, dz);
    if constexpr (N::sx == 0) return a;
    else return lerpm(a, load(ax1, dy, dz), 0.5f);
  };
  auto along_y = [&](int dz) {
    const float c0 = along_x(ay0, dz);
    if constexpr (N::sy == 0) return c0;
    else return lerpm(c0, along_x(ay1, dz), 0.5f);
  };
  const float y0 = along_y(az0);
  if constexpr (N::sz == 0) return y0;
  else return lerpm(y0, along_y(az1), 0.5f);
}

// The velocity ring's plane stride: padded to a multiple of 32 floats in the velocity march; the scalar march
// keeps it unpadded so that two blocks still fit in one SM's shared memory.
template <int G>
struct Stride {
  static constexpr int value = G == 3 ? RPN : RP;
};

template <int G>
__device__ __forceinline__ F3 ring_node(const float* vring, int x, int inplane) {
  constexpr int S = Stride<G>::value;
  auto ring = [&](const float* r) {
    return [=](int dx, int dy, int dz) { return r[((x + dx) & (VR - 1)) * S + inplane + dy * RZ + dz]; };
  };
  return f3(node_component<G, 0>(ring(vring)), node_component<G, 1>(ring(vring + VR * S)),
            node_component<G, 2>(ring(vring + 2 * VR * S)));
}

template <int G, class T>
__device__ __forceinline__ F3 global_node(const Args<T>& A, int x, int y, int z) {
  const int nx = A.info.dims[0], ny = A.info.dims[1], nz = A.info.dims[2];
  auto global = [&](const T* f, Dims d) {
    return [=](int dx, int dy, int dz) {
      const int a = imin_(imax_(x + dx, 0), d.n0 - 1), b = imin_(imax_(y + dy, 0), d.n1 - 1);
      const int c = imin_(imax_(z + dz, 0), d.n2 - 1);
      return ldg_f(f + at(d, a, b, c));
    };
  };
  return f3(node_component<G, 0>(global(A.vel[0], Dims{nx + 1, ny, nz})),
            node_component<G, 1>(global(A.vel[1], Dims{nx, ny + 1, nz})),
            node_component<G, 2>(global(A.vel[2], Dims{nx, ny, nz + 1})));
}

// ---- the forward (semi-Lagrangian) value and its clamp range at one element --------------------------------
template <int G>
struct Fields {
  static constexpr int count = G == 3 ? 2 : 1;
};

// Evaluated from global memory: the whole trace, every sample through clamped indices.
template <int G, class T>
__device__ __noinline__ void hat_global(const Args<T>& A, int x, int y, int z, float* hat, float* lo, float* hi) {
  constexpr int F = Fields<G>::count;
  const F3 off = offset_of<G>();
  const F3 p = add3(f3((float)x, (float)y, (float)z), off);
  const F3 vp = global_node<G>(A, x, y, z);
  const F3 mid = sub3(p, mul3(vp, 0.5f * A.dt));
  const F3 src = sub3(p, mul3(global_velocity(A, mid), A.dt));
  const bool outside = G == 3 && A.uses_outside == 1 && is_outside_open_face(src, A.info);
  const F3 g = sub3(src, off);
  const Ax gx = split(g[0]), gy = split(g[1]), gz = split(g[2]);
  for (int f = 0; f < F; ++f) {
    if (outside) {
      hat[f] = lo[f] = hi[f] = A.outside[f];
      continue;
    }
    float a[8];
    const T* src_field = G == 3 ? A.field[f] : A.vel[G];
    global_corners(src_field, group_dims(A.info, G), gx.i, gy.i, gz.i, a);
    hat[f] = blend8(a, gx.t, gy.t, gz.t);
    range8(a, lo[f], hi[f]);
  }
}

// From the staged rings when the trace stays inside them, else hat_global.
template <int G, class T>
__device__ __forceinline__ void hat_at(const Args<T>& A, const float* vring, const float* sring, int rowbase, int x, int y,
                                       int z, float* hat, float* lo, float* hi) {
  constexpr int F = Fields<G>::count;
  const F3 off = offset_of<G>();
  const F3 p = add3(f3((float)x, (float)y, (float)z), off);
  const int inplane = y * RZ + z - rowbase;
  const F3 vp = ring_node<G>(vring, x, inplane);
  bool fast = maxabs3(vp) * fabsf(A.dt) < REACH;
  F3 src = p;
  if (fast) {
    const F3 mid = sub3(p, mul3(vp, 0.5f * A.dt));
    const F3 vm = ring_velocity<Stride<G>::value>(vring, rowbase, mid);
    fast = maxabs3(vm) * fabsf(A.dt) < REACH;
    src = sub3(p, mul3(vm, A.dt));
  }
  if (!fast) {
    hat_global<G>(A, x, y, z, hat, lo, hi);
    return;
  }
  const bool outside = G == 3 && A.uses_outside == 1 && is_outside_open_face(src, A.info);
  const F3 g = sub3(src, off);
  const Ax gx = split(g[0]), gy = split(g[1]), gz = split(g[2]);
  const int gin = gy.i * RZ + gz.i - rowbase;
#pragma unroll
  for (int f = 0; f < F; ++f) {
    if (outside) {
      hat[f] = lo[f] = hi[f] = A.outside[f];
      continue;
    }
    float a[8];
    if constexpr (G == 3) ring_corners<SR, RPN>(sring + f * SR * RPN, gx.i, gin, a);
    else ring_corners<VR, RP>(vring + G * VR * RP, gx.i, gin, a);
    hat[f] = blend8(a, gx.t, gy.t, gz.t);
    range8(a, lo[f], hi[f]);
  }
}

// ---- the backward sample of hat (the reference's `back`) ---------------------------------------------------
// From the hat ring when the backward trace stays inside it, else each corner's hat from wherever it is: the
// ring for corners inside the staged hat planes, hat_global for the rest.
template <int G, class T>
__device__ __noinline__ void back_global(const Args<T>& A, const float* hring, int hbase, int j0, int k0, int plane_lo,
                                         int x, int y, int z, float* back) {
  constexpr int F = Fields<G>::count;
  const F3 off = offset_of<G>();
  const Dims gd = group_dims(A.info, G);
  const F3 p = add3(f3((float)x, (float)y, (float)z), off);
  const F3 vp = global_node<G>(A, x, y, z);
  const F3 mid = sub3(p, mul3(vp, 0.5f * -A.dt));
  const F3 bsrc = sub3(p, mul3(global_velocity(A, mid), -A.dt));
  if (G == 3 && A.uses_outside == 1 && is_outside_open_face(bsrc, A.info)) {
    for (int f = 0; f < F; ++f) back[f] = A.outside[f];
    return;
  }
  const F3 g = sub3(bsrc, off);
  const Ax gx = split(g[0]), gy = split(g[1]), gz = split(g[2]);
  float a[F][8];
  for (int c = 0; c < 8; ++c) {
    const int cx = imin_(gx.i + (c & 1), gd.n0 - 1), cy = imin_(gy.i + ((c >> 1) & 1), gd.n1 - 1);
    const int cz = imin_(gz.i + (c >> 2), gd.n2 - 1);
    const bool staged = cx >= plane_lo && cx <= plane_lo + 2 && cy >= j0 - 1 && cy <= j0 + TY && cz >= k0 - 1 &&
                        cz <= k0 + TZ;
    if (staged) {
      for (int f = 0; f < F; ++f) a[f][c] = hring[(f * HR + (cx & (HR - 1))) * HP + cy * HZ + cz - hbase];
    } else {
      float h[F], lo[F], hi[F];
      hat_global<G>(A, cx, cy, cz, h, lo, hi);
      for (int f = 0; f < F; ++f) a[f][c] = h[f];
    }
  }
  for (int f = 0; f < F; ++f) back[f] = blend8(a[f], gx.t, gy.t, gz.t);
}

// ---- staging ------------------------------------------------------------------------------------------------
// Each thread stages the plane elements e = t, t + NT, ... (while e < RPN); its offsets inside a plane of each
// array shape are fixed for the whole march.
struct StageOffsets {
  int off[3][STAGE_PER_THREAD];  // per array shape: u and the cells share (ny, nz); v (ny+1, nz); w (ny, nz+1)
};

template <class T>
__device__ __forceinline__ void stage_plane(const T* __restrict__ src, const Dims& d, int shape, int plane,
                                            float* ring_plane, const StageOffsets& so) {
  const int pc = imin_(imax_(plane, 0), d.n0 - 1);
  const T* base = src + (size_t)pc * d.n1 * d.n2;
#pragma unroll
  for (int n = 0; n < STAGE_PER_THREAD; ++n) {
    const int e = threadIdx.x + n * NT;
    if (e < RPN) {
      if constexpr (sizeof(T) == 4) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(ring_plane + e);
        const size_t from = __cvta_generic_to_global(base + so.off[shape][n]);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(from));
      } else {
        ring_plane[e] = ldg_f(base + so.off[shape][n]);
      }
    }
  }
}

__device__ __forceinline__ void stage_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---- the march -----------------------------------------------------------------------------------------------
template <class T, int G>
__device__ __forceinline__ void march(const Args<T>& A, int seg, float* sm) {
  constexpr int F = Fields<G>::count;
  const int nx = A.info.dims[0], ny = A.info.dims[1], nz = A.info.dims[2];
  const Dims gd = group_dims(A.info, G);
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TY;
  if (j0 >= gd.n1 || k0 >= gd.n2) return;  // a tile past this group's extent (the v and w end rows)
  const int s = seg * A.seg_len;
  if (s >= gd.n0) return;
  const int e = imin_(s + A.seg_len, gd.n0);

  constexpr int VS = Stride<G>::value;                 // velocity ring plane stride
  float* vring = sm;                                  // [3][VR][VS]
  float* sring = vring + 3 * VR * VS;                 // [2][SR][RPN] (scalar march)
  float* hring = sring + (G == 3 ? 2 * SR * RPN : 0);  // [F][HR][HP]
  const int t = threadIdx.x, ty = t / TZ, tz = t % TZ;
  const int rowbase = (j0 - 2) * RZ + (k0 - 2), hbase = (j0 - 1) * HZ + (k0 - 1);

  // staging offsets inside one plane of each array shape (edge-clamped)
  StageOffsets so;
  {
    const Dims shapes[3] = {Dims{0, ny, nz}, Dims{0, ny + 1, nz}, Dims{0, ny, nz + 1}};
#pragma unroll
    for (int sh = 0; sh < 3; ++sh)
#pragma unroll
      for (int n = 0; n < STAGE_PER_THREAD; ++n) {
        const int el = imin_(t + n * NT, RPN - 1), r = el / RZ, q = el % RZ;
        const int y = imin_(imax_(j0 - 2 + r, 0), shapes[sh].n1 - 1);
        const int z = imin_(imax_(k0 - 2 + q, 0), shapes[sh].n2 - 1);
        so.off[sh][n] = y * shapes[sh].n2 + z;
      }
  }
  const Dims vd[3] = {Dims{nx + 1, ny, nz}, Dims{nx, ny + 1, nz}, Dims{nx, ny, nz + 1}};
  const Dims cd{nx, ny, nz};
  auto stage_velocity = [&](int plane) {
#pragma unroll
    for (int c = 0; c < 3; ++c) stage_plane(A.vel[c], vd[c], c, plane, vring + (c * VR + (plane & (VR - 1))) * VS, so);
  };
  auto stage_scalars = [&](int plane) {
    if constexpr (G == 3) {
#pragma unroll
      for (int f = 0; f < 2; ++f) stage_plane(A.field[f], cd, 0, plane, sring + (f * SR + (plane & (SR - 1))) * RPN, so);
    }
  };

  // this thread's tile element, and its element of the hat plane's ring (t < HALO)
  const int tj = j0 + ty, tk = k0 + tz;
  const bool valid = tj < gd.n1 && tk < gd.n2;
  const int cj = imin_(tj, gd.n1 - 1), ck = imin_(tk, gd.n2 - 1);
  int hj, hk;  // position in the hat plane (0..HY-1, 0..HZ-1)
  if (t < HZ) {
    hj = 0;
    hk = t;
  } else if (t < 2 * HZ) {
    hj = HY - 1;
    hk = t - HZ;
  } else if (t < 2 * HZ + TY) {
    hj = 1 + t - 2 * HZ;
    hk = 0;
  } else {
    hj = 1 + t - 2 * HZ - TY;
    hk = HZ - 1;
  }
  const bool has_halo = t < HALO;
  const int rj = imin_(imax_(j0 - 1 + hj, 0), gd.n1 - 1), rk = imin_(imax_(k0 - 1 + hk, 0), gd.n2 - 1);
  const int tile_h = (ty + 1) * HZ + (tz + 1), ring_h = hj * HZ + hk;

  float range_lo[F], range_hi[F], own_hat[F];
  float sum_data = 0.0f, sum_hat = 0.0f, sum_next = 0.0f;

  // The hat plane x (clamped to the array), this thread's two elements; the tile element's range and hat
  // are kept for its correction.
  auto hat_plane = [&](int x, float* keep_lo, float* keep_hi, float* keep_hat) {
    const int xc = imin_(imax_(x, 0), gd.n0 - 1);
    float h[F], lo[F], hi[F];
    hat_at<G>(A, vring, sring, rowbase, xc, cj, ck, h, lo, hi);
#pragma unroll
    for (int f = 0; f < F; ++f) {
      hring[(f * HR + (x & (HR - 1))) * HP + tile_h] = h[f];
      keep_lo[f] = lo[f];
      keep_hi[f] = hi[f];
      keep_hat[f] = h[f];
    }
    if (has_halo) {
      hat_at<G>(A, vring, sring, rowbase, xc, rj, rk, h, lo, hi);
#pragma unroll
      for (int f = 0; f < F; ++f) hring[(f * HR + (x & (HR - 1))) * HP + ring_h] = h[f];
    }
  };
  // hat plane `to` copied from plane `from` (the array's edge planes, replicated); each thread copies the
  // elements it wrote itself
  auto copy_hat_plane = [&](int from, int to) {
#pragma unroll
    for (int f = 0; f < F; ++f) {
      hring[(f * HR + (to & (HR - 1))) * HP + tile_h] = hring[(f * HR + (from & (HR - 1))) * HP + tile_h];
      if (has_halo) hring[(f * HR + (to & (HR - 1))) * HP + ring_h] = hring[(f * HR + (from & (HR - 1))) * HP + ring_h];
    }
  };

  // prologue: planes s-2..s+2 of the velocity (and s-2..s+1 of the scalars), hat planes s-1 and s
  for (int p = s - 2; p <= s + 2; ++p) stage_velocity(p);
  for (int p = s - 2; p <= s + 1; ++p) stage_scalars(p);
  stage_commit();
  stage_wait();
  __syncthreads();
  {
    float lo[F], hi[F], h[F];
    if (s == 0) {
      hat_plane(0, range_lo, range_hi, own_hat);
      copy_hat_plane(0, -1);
    } else {
      hat_plane(s - 1, lo, hi, h);
      hat_plane(s, range_lo, range_hi, own_hat);
    }
  }
  if (G == 3) {
    __syncthreads();  // the scalar ring's slot of plane s-2 is free
    stage_scalars(s + 2);
    stage_commit();
    stage_wait();
  }
  if (G == 3 && valid) sum_hat = own_hat[0];
  __syncthreads();

  const size_t plane_stride = (size_t)gd.n1 * gd.n2;
  for (int i = s; i < e; ++i) {
    // planes i+3 start landing while hat plane i+1 is computed
    stage_velocity(i + 3);
    stage_scalars(i + 3);
    stage_commit();
    float next_lo[F] = {}, next_hi[F] = {}, next_hat[F] = {};
    if (i + 1 <= gd.n0 - 1) {
      hat_plane(i + 1, next_lo, next_hi, next_hat);
      if (G == 3 && valid && i + 1 < e) sum_hat += next_hat[0];
    } else {
      copy_hat_plane(i, i + 1);
    }
    stage_wait();
    __syncthreads();

    if (valid) {
      // the correction (advect.py:34-50, 64): back = hat sampled along the backward trace
      const F3 off = offset_of<G>();
      const F3 p = add3(f3((float)i, (float)tj, (float)tk), off);
      const int inplane = tj * RZ + tk - rowbase;
      const F3 vp = ring_node<G>(vring, i, inplane);
      bool fast = maxabs3(vp) * fabsf(A.dt) < REACH;
      float back[F];
      if (fast) {
        const F3 mid = sub3(p, mul3(vp, 0.5f * -A.dt));
        const F3 vm = ring_velocity<VS>(vring, rowbase, mid);
        fast = maxabs3(vm) * fabsf(A.dt) < REACH;
        if (fast) {
          const F3 bsrc = sub3(p, mul3(vm, -A.dt));
          if (G == 3 && A.uses_outside == 1 && is_outside_open_face(bsrc, A.info)) {
#pragma unroll
            for (int f = 0; f < F; ++f) back[f] = A.outside[f];
          } else {
            const F3 g = sub3(bsrc, off);
            const Ax gx = split(g[0]), gy = split(g[1]), gz = split(g[2]);
            const int gin = gy.i * HZ + gz.i - hbase;
#pragma unroll
            for (int f = 0; f < F; ++f) {
              const float* h0 = hring + (f * HR + (gx.i & (HR - 1))) * HP + gin;
              const float* h1 = hring + (f * HR + ((gx.i + 1) & (HR - 1))) * HP + gin;
              const float a[8] = {h0[0], h1[0], h0[HZ], h1[HZ], h0[1], h1[1], h0[HZ + 1], h1[HZ + 1]};
              back[f] = blend8(a, gx.t, gy.t, gz.t);
            }
          }
        }
      }
      if (!fast) back_global<G>(A, hring, hbase, j0, k0, i - 1, i, tj, tk, back);
      const size_t out = (size_t)i * plane_stride + (size_t)tj * gd.n2 + tk;
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const float data = G == 3 ? ldg_f(A.field[f] + out) : vring[(G * VR + (i & (VR - 1))) * VS + inplane];
        const float corrected = own_hat[f] + 0.5f * (data - back[f]);
        float value = clampf_(corrected, range_lo[f], range_hi[f]);
        if (G == 3 && f == 0) {
          sum_data += data;
          sum_next += value;
        }
        if (G == 3 && f == 1 && A.dissipate) value = A.ambient + (to_f<T>(from_f<T>(value)) - A.ambient) * A.heat_keep;
        st_f(A.next[G == 3 ? f : G] + out, value);
      }
    }
#pragma unroll
    for (int f = 0; f < F; ++f) {
      range_lo[f] = next_lo[f];
      range_hi[f] = next_hi[f];
      own_hat[f] = next_hat[f];
    }
  }
  if (G == 3 && valid) {
    const size_t lines = (size_t)ny * nz, line = (size_t)tj * nz + tk;
    const int segs = A.segs[3];
    A.partials[(size_t)(0 * segs + seg) * lines + line] = sum_data;
    A.partials[(size_t)(1 * segs + seg) * lines + line] = sum_hat;
    A.partials[(size_t)(2 * segs + seg) * lines + line] = sum_next;
  }
}

// MINB: resident blocks per SM the kernel is compiled for (4 at 256 threads: at most 64 registers a thread;
// 3: 80; 2: 128).
template <class T, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_mac_velocity(Args<T> A) {
  extern __shared__ float sm[];
  int z = blockIdx.z;
  if (z < A.segs[0]) return march<T, 0>(A, z, sm);
  z -= A.segs[0];
  if (z < A.segs[1]) return march<T, 1>(A, z, sm);
  march<T, 2>(A, z - A.segs[1], sm);
}

template <class T, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_mac_scalars(Args<T> A) {
  extern __shared__ float sm[];
  march<T, 3>(A, blockIdx.z, sm);
}

// Line totals from the segment sums (in segment order, float), then 256 lines per block added in double by a
// halving tree, as k_line_partials lays them out: partial[f * blocks + block].
constexpr int LINE_BLOCK = 256;
__global__ void k_segment_lines(const float* __restrict__ seg_sums, int segs, long lines, double* __restrict__ partial,
                                int blocks) {
  __shared__ double slot[LINE_BLOCK];
  const int f = blockIdx.y;
  const long line = (long)blockIdx.x * LINE_BLOCK + threadIdx.x;
  double value = 0.0;
  if (line < lines) {
    float total = 0.0f;
    for (int s = 0; s < segs; ++s) total = total + seg_sums[((long)f * segs + s) * lines + line];
    value = (double)total;
  }
  slot[threadIdx.x] = value;
  __syncthreads();
  for (int h = LINE_BLOCK / 2; h >= 1; h >>= 1) {
    if ((int)threadIdx.x < h) slot[threadIdx.x] = slot[threadIdx.x] + slot[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[f * blocks + blockIdx.x] = slot[0];
}

constexpr size_t VELOCITY_SMEM = sizeof(float) * (3 * VR * RP + HR * HP);
constexpr size_t SCALAR_SMEM = sizeof(float) * (3 * VR * RPN + 2 * SR * RPN + 2 * HR * HP);

// Segments along x: enough blocks for about six waves of the resident blocks, each segment at least 8 planes.
static int segments(int n0, long tiles, int groups) {
  const long target = 6L * BLOCKS_PER_SM * 148;
  long segs = (target + tiles * groups - 1) / (tiles * groups);
  segs = std::max(1L, std::min(segs, (long)std::max(1, n0 / 8)));
  return (int)segs;
}

static int env_int(const char* name) {
  const char* v = getenv(name);
  return v ? atoi(v) : 0;
}

// Blocks per SM the march kernels run with (PLUME_MAC_BLOCKS = 1 selects the 128-register form).
// Blocks per SM the marches are compiled for: PLUME_MAC_BLOCKS = 2, 3 or 4 (the default, BLOCKS_PER_SM).
static int blocks_per_sm() {
  static const int b = [] {
    const int v = env_int("PLUME_MAC_BLOCKS");
    return v == 2 || v == 3 ? v : BLOCKS_PER_SM;
  }();
  return b;
}


template <class Kernel>
static int configure(Kernel k, size_t smem, bool& done) {
  if (done) return PLUME_OK;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return runtime_status("fused advection: shared memory", err);
  done = true;
  return PLUME_OK;
}

}  // namespace mac

int mac_segments_for_scalars(const PlumeGridInfo& info) {
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  const long tiles = (long)((ny + mac::TY - 1) / mac::TY) * ((nz + mac::TZ - 1) / mac::TZ);
  int segs = mac::env_int("PLUME_MAC_SCALAR_SEGS");
  if (segs <= 0) segs = mac::segments(nx, tiles, 1);
  segs = std::max(1, std::min(segs, nx));
  const int len = (nx + segs - 1) / segs;
  return (nx + len - 1) / len;  // every segment non-empty
}

long long mac_partial_floats(const PlumeGridInfo& info) {
  return 3LL * mac_segments_for_scalars(info) * info.dims[1] * info.dims[2];
}

template <class T>
int launch_mac_velocity(const PlumeGridInfo& info, const T* u, const T* v, const T* w, T* u_next, T* v_next,
                        T* w_next, float dt_over_cell, cudaStream_t st) {
  static bool configured[5] = {};
  const int bps = mac::blocks_per_sm();
  auto kernel = bps == 2 ? mac::k_mac_velocity<T, 2> : (bps == 3 ? mac::k_mac_velocity<T, 3> : mac::k_mac_velocity<T, 4>);
  int status = mac::configure(kernel, mac::VELOCITY_SMEM, configured[bps]);
  if (status != PLUME_OK) return status;
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  mac::Args<T> A{};
  A.info = info;
  A.vel[0] = u;
  A.vel[1] = v;
  A.vel[2] = w;
  A.next[0] = u_next;
  A.next[1] = v_next;
  A.next[2] = w_next;
  A.dt = dt_over_cell;
  const int jt = (ny + 1 + mac::TY - 1) / mac::TY, kt = (nz + 1 + mac::TZ - 1) / mac::TZ;
  int segs = mac::env_int("PLUME_MAC_VELOCITY_SEGS");
  if (segs <= 0) segs = mac::segments(nx, (long)jt * kt, 3);
  segs = std::max(1, std::min(segs, nx));
  A.seg_len = (nx + segs - 1) / segs;
  for (int g = 0; g < 3; ++g) A.segs[g] = (nx + (g == 0) + A.seg_len - 1) / A.seg_len;
  const dim3 grid(kt, jt, A.segs[0] + A.segs[1] + A.segs[2]);
  kernel<<<grid, mac::NT, mac::VELOCITY_SMEM, st>>>(A);
  return launch_status("fused velocity advection");
}

template <class T>
int launch_mac_scalars(const PlumeGridInfo& info, const T* u, const T* v, const T* w, const T* smoke,
                       const T* temperature, T* smoke_next, T* temperature_next, float smoke_outside,
                       float heat_outside, int uses_outside, float* seg_sums, double* line_partials, int dissipate,
                       float heat_keep, float ambient, float dt_over_cell, cudaStream_t st) {
  static bool configured[5] = {};
  const int bps = mac::blocks_per_sm();
  auto kernel = bps == 2 ? mac::k_mac_scalars<T, 2> : (bps == 3 ? mac::k_mac_scalars<T, 3> : mac::k_mac_scalars<T, 4>);
  int status = mac::configure(kernel, mac::SCALAR_SMEM, configured[bps]);
  if (status != PLUME_OK) return status;
  const int nx = info.dims[0], ny = info.dims[1], nz = info.dims[2];
  mac::Args<T> A{};
  A.info = info;
  A.vel[0] = u;
  A.vel[1] = v;
  A.vel[2] = w;
  A.field[0] = smoke;
  A.field[1] = temperature;
  A.next[0] = smoke_next;
  A.next[1] = temperature_next;
  A.outside[0] = smoke_outside;
  A.outside[1] = heat_outside;
  A.uses_outside = uses_outside;
  A.dt = dt_over_cell;
  const int segs = mac_segments_for_scalars(info);
  A.seg_len = (nx + segs - 1) / segs;
  A.segs[3] = segs;
  A.partials = seg_sums;
  A.dissipate = dissipate;
  A.heat_keep = heat_keep;
  A.ambient = ambient;
  const dim3 grid((nz + mac::TZ - 1) / mac::TZ, (ny + mac::TY - 1) / mac::TY, segs);
  kernel<<<grid, mac::NT, mac::SCALAR_SMEM, st>>>(A);
  status = launch_status("fused scalar advection");
  if (status != PLUME_OK) return status;
  const long lines = (long)ny * nz;
  const int blocks = (int)((lines + mac::LINE_BLOCK - 1) / mac::LINE_BLOCK);
  mac::k_segment_lines<<<dim3(blocks, 3), mac::LINE_BLOCK, 0, st>>>(seg_sums, segs, lines, line_partials, blocks);
  return launch_status("smoke budget line sums");
}

#define PLUME_MAC_INSTANTIATE(T)                                                                              \
  template int launch_mac_velocity<T>(const PlumeGridInfo&, const T*, const T*, const T*, T*, T*, T*, float,   \
                                      cudaStream_t);                                                           \
  template int launch_mac_scalars<T>(const PlumeGridInfo&, const T*, const T*, const T*, const T*, const T*,  \
                                     T*, T*, float, float, int, float*, double*, int, float, float, float,     \
                                     cudaStream_t);
PLUME_MAC_INSTANTIATE(float)
PLUME_MAC_INSTANTIATE(__nv_bfloat16)
PLUME_MAC_INSTANTIATE(__half)

}  // namespace plume
