// Sheet assembly and the numbers file on the device (chadmv/plume src/plume/sheet/*, src/plume/report/numbers.py),
// so that a run's raw frames never leave the GPU until they are 8-bit sheet frames.
//
// Raw frames arrive as one (frames, height, width, 5) float32 array. The steps, each a kernel:
//   - the content box: the largest heat of any frame, then the union of pixels any frame shows (crop.py:29-43);
//   - bicubic resampling of the crop square (resample.py:16-41), restating the two-pass separable filter the
//     reference gets from Pillow: the caller passes, per output index and pass, the first source index, the
//     window length and the normalised weights; each pass accumulates in double and stores float32, and the
//     horizontal pass covers only the rows the vertical pass reads. Padding with the layout's empty pixel is
//     done on the fly. The vertical pass also applies the resampled frame's clamps, in double;
//   - Gaussian blurs in double along one axis with the edge extended (soften.py:27-49), the normal layout's
//     renormalisation (soften.py:52-60), the shade layout's thin-pixel easing (shade.py:22-42);
//   - maxima for the heat and shade divisors, quantisation to bytes (quantize.py:20-39), the gutter check
//     (assemble.py:70-73), packing into the sheet (pack.py:13-20);
//   - per-frame integer tallies for the numbers file (numbers.py:80-100).
// Every float64 expression keeps the reference's numpy order of operations (the library builds with
// -fmad=false); the one exception is the frame-wide sums of the easing step, added here in a fixed order
// rather than numpy's pairwise order.
#include <cstdint>

#include "common.cuh"

namespace plume {

constexpr int RAW_CHANNELS = 5;
constexpr int HEAT_CH = 0, THICK_CH = 1, SHADE_CH = 2;
constexpr double CONTENT_LEVEL = 0.5 / 255.0;  // crop.py:10
constexpr double FRAME_MEAN_WEIGHT = 1.0 / 255.0, NO_SMOKE = 1e-12;  // shade.py:17-20
constexpr int SHEET_THREADS = 256;

// Order-preserving keys for atomic max of floats and doubles.
__device__ __forceinline__ unsigned int float_key(float v) {
  const unsigned int b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__device__ __forceinline__ unsigned long long double_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_double(unsigned long long k) {
  return __longlong_as_double((long long)((k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k));
}

static int sheet_blocks(long n) { return (int)((n + SHEET_THREADS - 1) / SHEET_THREADS); }

// ---- content box ---------------------------------------------------------------------------------------------
__global__ void k_heat_key(const float* __restrict__ raw, long pixels, unsigned int* __restrict__ key) {
  unsigned int best = 0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x)
    best = max(best, float_key(raw[p * RAW_CHANNELS + HEAT_CH]));
  for (int off = 16; off >= 1; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(key, best);
}

// box = (left, top, right, bottom), right/bottom exclusive; starts as (width, height, 0, 0).
__global__ void k_content_union(const float* __restrict__ raw, int frames, int height, int width,
                                const unsigned int* __restrict__ heat_key, int* __restrict__ box) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)height * width) return;
  const double heat_max = (double)key_float(*heat_key);
  bool covered = false;
  for (int f = 0; f < frames && !covered; ++f) {
    const float* px = raw + ((long)f * height * width + p) * RAW_CHANNELS;
    covered = (double)px[THICK_CH] >= CONTENT_LEVEL || (heat_max > 0.0 && (double)px[HEAT_CH] >= CONTENT_LEVEL * heat_max);
  }
  if (!covered) return;
  const int y = (int)(p / width), x = (int)(p % width);
  atomicMin(box + 0, x);
  atomicMin(box + 1, y);
  atomicMax(box + 2, x + 1);
  atomicMax(box + 3, y + 1);
}

// ---- bicubic resampling ------------------------------------------------------------------------------------
struct Taps {
  const int* first;
  const int* count;
  const double* weights;
  int ksize;
};

struct PadSpec {
  int height, width, pad;
  float empty[RAW_CHANNELS];
};

// temp[f][c][r][xx]: the horizontal pass over padded rows row_first + r.
__global__ void k_resample_rows(const float* __restrict__ raw, int frames, PadSpec ps, Taps h, int row_first, int rows,
                                int out, float* __restrict__ temp) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)frames * RAW_CHANNELS * rows * out;
  if (idx >= total) return;
  const int xx = (int)(idx % out);
  long rest = idx / out;
  const int r = (int)(rest % rows);
  rest /= rows;
  const int c = (int)(rest % RAW_CHANNELS);
  const int f = (int)(rest / RAW_CHANNELS);
  const int rr = row_first + r - ps.pad;
  const bool row_inside = rr >= 0 && rr < ps.height;
  const int first = h.first[xx], count = h.count[xx];
  const double* w = h.weights + (long)xx * h.ksize;
  double acc = 0.0;
  for (int x = 0; x < count; ++x) {
    const int cc = first + x - ps.pad;
    const float v = (row_inside && cc >= 0 && cc < ps.width)
                        ? raw[(((long)f * ps.height + rr) * ps.width + cc) * RAW_CHANNELS + c]
                        : ps.empty[c];
    acc = acc + (double)v * w[x];
  }
  temp[idx] = (float)acc;
}

// The vertical pass for all five channels of one output pixel, then the resampled frame's clamps (thickness
// to [0, 1], heat to >= 0, in the shade layout shade to [0, thickness]); frame is (frames, out, out, 5) double.
__global__ void k_resample_columns(const float* __restrict__ temp, int frames, Taps v, int rows, int out,
                                   int shade_layout, double* __restrict__ frame) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)frames * out * out) return;
  const int xx = (int)(idx % out);
  const int yy = (int)((idx / out) % out);
  const int f = (int)(idx / ((long)out * out));
  const int first = v.first[yy], count = v.count[yy];
  const double* w = v.weights + (long)yy * v.ksize;
  double value[RAW_CHANNELS];
  for (int c = 0; c < RAW_CHANNELS; ++c) {
    const float* plane = temp + ((long)f * RAW_CHANNELS + c) * rows * out;
    double acc = 0.0;
    for (int y = 0; y < count; ++y) acc = acc + (double)plane[(long)(first + y) * out + xx] * w[y];
    value[c] = (double)(float)acc;  // Pillow stores the pass as float32; the reference then widens to double
  }
  value[THICK_CH] = value[THICK_CH] < 0.0 ? 0.0 : (value[THICK_CH] > 1.0 ? 1.0 : value[THICK_CH]);
  value[HEAT_CH] = value[HEAT_CH] > 0.0 ? value[HEAT_CH] : 0.0;  // np.maximum(heat, 0)
  if (shade_layout)
    value[SHADE_CH] = value[SHADE_CH] < 0.0 ? 0.0 : (value[SHADE_CH] > value[THICK_CH] ? value[THICK_CH] : value[SHADE_CH]);
  double* out_px = frame + idx * RAW_CHANNELS;
  for (int c = 0; c < RAW_CHANNELS; ++c) out_px[c] = value[c];
}

// ---- blurs and per-pixel passes in double ---------------------------------------------------------------------
// One axis (0 rows, 1 columns) of a Gaussian blur of `channels` interleaved planes of (frames, size, size),
// edges extended: result = sum over taps of weight * neighbour, added in tap order (soften.py:40-49).
__global__ void k_blur_f64(const double* __restrict__ src, double* __restrict__ dst, int frames, int size,
                           int channels, int stride, int offset, const double* __restrict__ weights, int radius,
                           int axis) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)frames * size * size * channels) return;
  const int c = (int)(idx % channels);
  const long pixel = idx / channels;
  const int x = (int)(pixel % size), y = (int)((pixel / size) % size), f = (int)(pixel / ((long)size * size));
  double result = 0.0;
  for (int o = 0; o <= 2 * radius; ++o) {
    int yy = y, xx = x;
    if (axis == 0) yy = min(max(y + o - radius, 0), size - 1);
    else xx = min(max(x + o - radius, 0), size - 1);
    result = result + weights[o] * src[(((long)f * size + yy) * size + xx) * stride + offset + c];
  }
  dst[pixel * stride + offset + c] = result;
}

// soften.py:52-60: normals to unit length with |z|, or facing the camera where they vanish.
__global__ void k_renormalize(double* __restrict__ frame, long pixels) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pixels) return;
  double* n = frame + p * RAW_CHANNELS + 2;
  const double x = n[0], y = n[1], z = fabs(n[2]);
  const double length = sqrt((x * x + y * y) + z * z);
  if (length > 1e-6) {
    const double d = length > 1e-6 ? length : 1e-6;
    n[0] = x / d;
    n[1] = y / d;
    n[2] = z / d;
  } else {
    n[0] = 0.0;
    n[1] = 0.0;
    n[2] = 1.0;
  }
}

// Per-frame sums of thickness and shade-times-thickness, in a fixed order (one block per frame).
__global__ void k_frame_sums(const double* __restrict__ frame, int size, double* __restrict__ sums) {
  __shared__ double st[SHEET_THREADS], ss[SHEET_THREADS];
  const int f = blockIdx.x;
  const long pixels = (long)size * size;
  const double* base = frame + (long)f * pixels * RAW_CHANNELS;
  double t = 0.0, s = 0.0;
  for (long p = threadIdx.x; p < pixels; p += SHEET_THREADS) {
    t = t + base[p * RAW_CHANNELS + THICK_CH];
    s = s + base[p * RAW_CHANNELS + SHADE_CH];
  }
  st[threadIdx.x] = t;
  ss[threadIdx.x] = s;
  __syncthreads();
  for (int h = SHEET_THREADS / 2; h >= 1; h >>= 1) {
    if ((int)threadIdx.x < h) {
      st[threadIdx.x] = st[threadIdx.x] + st[threadIdx.x + h];
      ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[2 * f] = st[0];
    sums[2 * f + 1] = ss[0];
  }
}

// shade.py:37-42 given `blurred`, a frame-shaped array whose thickness and shade-times-thickness channels hold
// those planes blurred by the neighbourhood Gaussian.
__global__ void k_ease(double* __restrict__ frame, const double* __restrict__ blurred, int frames, int size,
                       const double* __restrict__ sums, double fade_thickness) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)frames * size * size) return;
  const int f = (int)(p / ((long)size * size));
  const double total = sums[2 * f], weighted_total = sums[2 * f + 1];
  const double mean = total > 0.0 ? weighted_total / total : 0.0;
  double* px = frame + p * RAW_CHANNELS;
  const double thickness = px[THICK_CH], weighted = px[SHADE_CH];
  const double* b = blurred + p * RAW_CHANNELS;
  const double neighborhood = (b[SHADE_CH] + FRAME_MEAN_WEIGHT * mean) / (b[THICK_CH] + FRAME_MEAN_WEIGHT);
  const bool has_smoke = thickness > NO_SMOKE;
  double own = has_smoke ? weighted / thickness : 0.0;
  own = own < 0.0 ? 0.0 : (own > 1.0 ? 1.0 : own);
  double weight = thickness / fade_thickness;
  weight = weight < 0.0 ? 0.0 : (weight > 1.0 ? 1.0 : weight);
  px[SHADE_CH] = neighborhood + weight * (own - neighborhood);
}

// Largest value of one channel over all frames, only where thickness >= floor (floor -inf: everywhere).
__global__ void k_channel_max(const double* __restrict__ frame, long pixels, int channel, double floor,
                              unsigned long long* __restrict__ key, int* __restrict__ any) {
  unsigned long long best = 0;
  bool found = false;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x) {
    const double* px = frame + p * RAW_CHANNELS;
    if (px[THICK_CH] >= floor) {
      found = true;
      const unsigned long long k = double_key(px[channel]);
      best = k > best ? k : best;
    }
  }
  for (int off = 16; off >= 1; off >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, off);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(key, best);
  if (found) atomicOr(any, 1);
}

// ---- quantisation, gutter, packing, numbers ---------------------------------------------------------------------
__device__ __forceinline__ unsigned char to_byte(double v) {  // clip(floor(v * 255 + 0.5), 0, 255)
  const double r = floor(v * 255.0 + 0.5);
  return (unsigned char)(r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r));
}

__global__ void k_quantize(const double* __restrict__ frame, long pixels, double heat_divisor, double shade_divisor,
                           int shade_layout, unsigned char* __restrict__ rgba) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pixels) return;
  const double* px = frame + p * RAW_CHANNELS;
  unsigned char* o = rgba + p * 4;
  o[0] = heat_divisor > 0.0 ? to_byte(px[HEAT_CH] / heat_divisor) : 0;
  o[1] = to_byte(px[THICK_CH]);
  if (shade_layout) {
    o[2] = to_byte(px[SHADE_CH] / shade_divisor);
    o[3] = 255;
    return;
  }
  o[2] = to_byte((px[2] + 1.0) * 0.5);
  o[3] = to_byte((px[3] + 1.0) * 0.5);
  if (o[0] == 0 && o[1] == 0) {
    o[2] = 128;
    o[3] = 128;
  }
}

// Sets *touched when any frame has a non-zero R or G byte within `gutter` pixels of its edge.
__global__ void k_gutter(const unsigned char* __restrict__ rgba, int frames, int size, int gutter, int* __restrict__ touched) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)frames * size * size) return;
  const int x = (int)(p % size), y = (int)((p / size) % size);
  const bool ring = x < gutter || y < gutter || x >= size - gutter || y >= size - gutter;
  if (ring && (rgba[p * 4] != 0 || rgba[p * 4 + 1] != 0)) atomicOr(touched, 1);
}

__global__ void k_pack(const unsigned char* __restrict__ rgba, int frames, int size, int columns, int rows,
                       unsigned char* __restrict__ sheet) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long width = (long)columns * size;
  if (idx >= (long)rows * size * width) return;
  const long sy = idx / width, sx = idx % width;
  const int row = (int)(sy / size), column = (int)(sx / size);
  const int index = row * columns + column;
  uint32_t value = 0;
  if (index < frames) {
    const long src = ((long)index * size + sy % size) * size + sx % size;
    value = reinterpret_cast<const uint32_t*>(rgba)[src];
  }
  reinterpret_cast<uint32_t*>(sheet)[idx] = value;
}

// Per frame: covered count, box of covered pixels (left, top, right, bottom; right/bottom exclusive), byte
// sums of heat and thickness over covered pixels, byte sum of thickness over all pixels, largest heat byte.
constexpr int MEASURE_FIELDS = 9;
__global__ void k_measure(const unsigned char* __restrict__ rgba, int frames, int size, int covered_level,
                          long long* __restrict__ stats) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)frames * size * size) return;
  const int f = (int)(p / ((long)size * size));
  const int x = (int)(p % size), y = (int)((p / size) % size);
  const unsigned char heat = rgba[p * 4], thick = rgba[p * 4 + 1];
  long long* s = stats + (long)f * MEASURE_FIELDS;
  if (thick) atomicAdd(reinterpret_cast<unsigned long long*>(s + 7), (unsigned long long)thick);
  if (heat) atomicMax(s + 8, (long long)heat);
  if (thick < covered_level) return;
  atomicAdd(reinterpret_cast<unsigned long long*>(s + 0), 1ull);
  atomicMin(s + 1, (long long)x);
  atomicMin(s + 2, (long long)y);
  atomicMax(s + 3, (long long)x + 1);
  atomicMax(s + 4, (long long)y + 1);
  atomicAdd(reinterpret_cast<unsigned long long*>(s + 5), (unsigned long long)heat);
  atomicAdd(reinterpret_cast<unsigned long long*>(s + 6), (unsigned long long)thick);
}

__global__ void k_measure_init(long long* stats, int frames, int size) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= frames) return;
  long long* s = stats + (long)f * MEASURE_FIELDS;
  s[0] = 0;
  s[1] = size;
  s[2] = size;
  s[3] = 0;
  s[4] = 0;
  s[5] = 0;
  s[6] = 0;
  s[7] = 0;
  s[8] = 0;
}

__global__ void k_box_init(int* box, int width, int height, unsigned int* key) {
  box[0] = width;
  box[1] = height;
  box[2] = 0;
  box[3] = 0;
  *key = 0;
}

__global__ void k_key_init(unsigned long long* key, int* any) {
  *key = 0;
  *any = 0;
}

__global__ void k_key_decode(const unsigned long long* key, const int* any, double* out) {
  out[0] = *any && *key ? key_double(*key) : 0.0;
  out[1] = *any ? 1.0 : 0.0;
}

}  // namespace plume

using namespace plume;

#define SHEET_CHECK(cond, what) \
  do {                          \
    if (!(cond)) return fail(PLUME_ERR_INVALID, "%s", what); \
  } while (0)

extern "C" int plume_sheet_content_box(const float* raw, int32_t frames, int32_t height, int32_t width,
                                       uint32_t* heat_key, int32_t* box, void* stream) {
  SHEET_CHECK(raw && heat_key && box && frames >= 1 && height >= 1 && width >= 1, "sheet_content_box: bad argument");
  cudaStream_t st = as_stream(stream);
  k_box_init<<<1, 1, 0, st>>>(box, width, height, heat_key);
  int status = launch_status("content box init");
  if (status != PLUME_OK) return status;
  const long pixels = (long)frames * height * width;
  k_heat_key<<<std::min(sheet_blocks(pixels), 148 * 8), SHEET_THREADS, 0, st>>>(raw, pixels, heat_key);
  if ((status = launch_status("heat max")) != PLUME_OK) return status;
  k_content_union<<<sheet_blocks((long)height * width), SHEET_THREADS, 0, st>>>(raw, frames, height, width, heat_key, box);
  return launch_status("content union");
}

extern "C" int plume_sheet_resample(const float* raw, int32_t frames, int32_t height, int32_t width, int32_t pad,
                                    const float empty[5], const int32_t* h_first, const int32_t* h_count,
                                    const double* h_weights, int32_t h_ksize, const int32_t* v_first,
                                    const int32_t* v_count, const double* v_weights, int32_t v_ksize, int32_t row_first,
                                    int32_t rows, int32_t out, int32_t shade_layout, float* temp, double* frame,
                                    void* stream) {
  SHEET_CHECK(raw && empty && h_first && h_count && h_weights && v_first && v_count && v_weights && temp && frame &&
                  frames >= 1 && height >= 1 && width >= 1 && pad >= 0 && rows >= 1 && out >= 1 && h_ksize >= 1 &&
                  v_ksize >= 1,
              "sheet_resample: bad argument");
  cudaStream_t st = as_stream(stream);
  PadSpec ps;
  ps.height = height;
  ps.width = width;
  ps.pad = pad;
  for (int c = 0; c < RAW_CHANNELS; ++c) ps.empty[c] = empty[c];
  const long horizontal = (long)frames * RAW_CHANNELS * rows * out;
  k_resample_rows<<<sheet_blocks(horizontal), SHEET_THREADS, 0, st>>>(raw, frames, ps, Taps{h_first, h_count, h_weights, h_ksize},
                                                                    row_first, rows, out, temp);
  int status = launch_status("resample rows");
  if (status != PLUME_OK) return status;
  k_resample_columns<<<sheet_blocks((long)frames * out * out), SHEET_THREADS, 0, st>>>(
      temp, frames, Taps{v_first, v_count, v_weights, v_ksize}, rows, out, shade_layout, frame);
  return launch_status("resample columns");
}

extern "C" int plume_sheet_blur(const double* src, double* dst, double* scratch, int32_t frames, int32_t size,
                                int32_t channels, int32_t stride, int32_t offset, const double* weights, int32_t radius,
                                void* stream) {
  SHEET_CHECK(src && dst && scratch && weights && frames >= 1 && size >= 1 && channels >= 1 && stride >= channels &&
                  offset >= 0 && offset + channels <= stride && radius >= 0,
              "sheet_blur: bad argument");
  cudaStream_t st = as_stream(stream);
  const long n = (long)frames * size * size * channels;
  k_blur_f64<<<sheet_blocks(n), SHEET_THREADS, 0, st>>>(src, scratch, frames, size, channels, stride, offset, weights,
                                                        radius, 0);
  int status = launch_status("blur rows");
  if (status != PLUME_OK) return status;
  k_blur_f64<<<sheet_blocks(n), SHEET_THREADS, 0, st>>>(scratch, dst, frames, size, channels, stride, offset, weights,
                                                        radius, 1);
  return launch_status("blur columns");
}

extern "C" int plume_sheet_renormalize(double* frame, int32_t frames, int32_t size, void* stream) {
  SHEET_CHECK(frame && frames >= 1 && size >= 1, "sheet_renormalize: bad argument");
  const long pixels = (long)frames * size * size;
  k_renormalize<<<sheet_blocks(pixels), SHEET_THREADS, 0, as_stream(stream)>>>(frame, pixels);
  return launch_status("renormalize");
}

extern "C" int plume_sheet_ease(double* frame, const double* blurred, double* sums, int32_t frames, int32_t size,
                                double fade_thickness, void* stream) {
  SHEET_CHECK(frame && blurred && sums && frames >= 1 && size >= 1 && fade_thickness > 0.0, "sheet_ease: bad argument");
  cudaStream_t st = as_stream(stream);
  k_frame_sums<<<frames, SHEET_THREADS, 0, st>>>(frame, size, sums);
  int status = launch_status("frame sums");
  if (status != PLUME_OK) return status;
  k_ease<<<sheet_blocks((long)frames * size * size), SHEET_THREADS, 0, st>>>(frame, blurred, frames, size, sums,
                                                                             fade_thickness);
  return launch_status("ease thin pixels");
}

extern "C" int plume_sheet_channel_max(const double* frame, int32_t frames, int32_t size, int32_t channel, double floor,
                                       unsigned long long* key, int32_t* any, double* out, void* stream) {
  SHEET_CHECK(frame && key && any && out && frames >= 1 && size >= 1 && channel >= 0 && channel < RAW_CHANNELS,
              "sheet_channel_max: bad argument");
  cudaStream_t st = as_stream(stream);
  k_key_init<<<1, 1, 0, st>>>(key, any);
  int status = launch_status("channel max init");
  if (status != PLUME_OK) return status;
  const long pixels = (long)frames * size * size;
  k_channel_max<<<std::min(sheet_blocks(pixels), 148 * 8), SHEET_THREADS, 0, st>>>(frame, pixels, channel, floor, key, any);
  if ((status = launch_status("channel max")) != PLUME_OK) return status;
  k_key_decode<<<1, 1, 0, st>>>(key, any, out);
  return launch_status("channel max decode");
}

extern "C" int plume_sheet_quantize(const double* frame, int32_t frames, int32_t size, double heat_divisor,
                                    double shade_divisor, int32_t shade_layout, int32_t gutter, uint8_t* rgba,
                                    int32_t* touched, void* stream) {
  SHEET_CHECK(frame && rgba && touched && frames >= 1 && size >= 1 && gutter >= 0, "sheet_quantize: bad argument");
  cudaStream_t st = as_stream(stream);
  const long pixels = (long)frames * size * size;
  k_quantize<<<sheet_blocks(pixels), SHEET_THREADS, 0, st>>>(frame, pixels, heat_divisor, shade_divisor, shade_layout,
                                                            rgba);
  int status = launch_status("quantize");
  if (status != PLUME_OK) return status;
  status = runtime_status("gutter flag", cudaMemsetAsync(touched, 0, sizeof(int32_t), st));
  if (status != PLUME_OK) return status;
  k_gutter<<<sheet_blocks(pixels), SHEET_THREADS, 0, st>>>(rgba, frames, size, gutter, touched);
  return launch_status("gutter");
}

extern "C" int plume_sheet_pack(const uint8_t* rgba, int32_t frames, int32_t size, int32_t columns, uint8_t* sheet,
                                void* stream) {
  SHEET_CHECK(rgba && sheet && frames >= 1 && size >= 1 && columns >= 1, "sheet_pack: bad argument");
  const int rows = (frames + columns - 1) / columns;
  const long n = (long)rows * size * columns * size;
  k_pack<<<sheet_blocks(n), SHEET_THREADS, 0, as_stream(stream)>>>(rgba, frames, size, columns, rows, sheet);
  return launch_status("pack");
}

extern "C" int plume_sheet_measure(const uint8_t* rgba, int32_t frames, int32_t size, int32_t covered_level,
                                   long long* stats, void* stream) {
  SHEET_CHECK(rgba && stats && frames >= 1 && size >= 1, "sheet_measure: bad argument");
  cudaStream_t st = as_stream(stream);
  k_measure_init<<<(frames + 127) / 128, 128, 0, st>>>(stats, frames, size);
  int status = launch_status("measure init");
  if (status != PLUME_OK) return status;
  k_measure<<<sheet_blocks((long)frames * size * size), SHEET_THREADS, 0, st>>>(rgba, frames, size, covered_level, stats);
  return launch_status("measure");
}
