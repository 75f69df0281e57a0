// ref_shim.h -- OpenCL C compatibility layer used to compile the reference's
// own OpenCL kernels (PyOpenCL27C/Pipe/*.c, PyOpenCL27C/Shaders/*.c) as C++
// for the CPU, so that they can serve as a parity reference for the oracle.
// TEST INFRASTRUCTURE ONLY (see oracle/build_ref.py).
//
// Work-items run one at a time (or one work-group per OpenMP thread); the
// harness sets the ids below before each call.  `__local` variables become
// thread-local namespace-scope arrays that the harness can preload.
// Float conventions match the oracle: no contraction (-ffp-contract=off),
// min/max/clamp = fminf/fmaxf, fast_normalize = v * (1/sqrt(dot(v,v))),
// fast_length = sqrt(dot(v,v)).
#pragma once
#include <math.h>
#include <stdint.h>
#include <limits.h>

namespace cl_shim {

typedef unsigned short ushort;
typedef unsigned char uchar;
typedef unsigned int uint;

extern thread_local int g_group[2];
extern thread_local int g_local[2];
extern thread_local int g_global[2];
inline int get_group_id(int d) { return g_group[d]; }
inline int get_local_id(int d) { return g_local[d]; }
inline int get_global_id(int d) { return g_global[d]; }
#define CLK_GLOBAL_MEM_FENCE 1
#define CLK_LOCAL_MEM_FENCE 2
// Kernels run one work-item at a time need no barrier.  Kernels whose
// barrier is meant to order the whole launch run one thread per work-item,
// and the harness points g_barrier at a barrier across all of them.
extern thread_local void (*g_barrier)();
inline void barrier(int) { if (g_barrier) g_barrier(); }
inline int atomic_inc(volatile int *p) { return __atomic_fetch_add((int *)p, 1, __ATOMIC_RELAXED); }

struct int3;
struct float2 {
  float x, y;
};
struct int2 {
  int x, y;
};
struct float3 {
  union {
    struct { float x, y, z; };
    struct { float s0, s1, s2; };
  };
  float pad_;
  float3() = default;
  float3(float s) : pad_(0) { x = s; y = s; z = s; }   // OpenCL scalar-to-vector broadcast
};
struct int3 {
  union {
    struct { int x, y, z; };
    struct { int s0, s1, s2; };
  };
  int pad_;
};
struct ushort3 {
  ushort x, y, z, pad_;
};
static_assert(sizeof(float3) == 16, "OpenCL float3 occupies 16 bytes");
static_assert(sizeof(int3) == 16, "OpenCL int3 occupies 16 bytes");

inline float2 make_float2(float a, float b) { float2 r; r.x = a; r.y = b; return r; }
inline int2 make_int2(int a, int b) { int2 r; r.x = a; r.y = b; return r; }
inline float3 make_float3(float a, float b, float c) { float3 r; r.x = a; r.y = b; r.z = c; r.pad_ = 0; return r; }
inline int3 make_int3(int a, int b, int c) { int3 r; r.x = a; r.y = b; r.z = c; r.pad_ = 0; return r; }
inline ushort3 make_ushort3(ushort a, ushort b, ushort c) { ushort3 r; r.x = a; r.y = b; r.z = c; r.pad_ = 0; return r; }

// float2 arithmetic
inline float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
inline float2 operator/(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }
inline float2 operator+(float2 a, float s) { return make_float2(a.x + s, a.y + s); }
inline float2 operator-(float2 a, float s) { return make_float2(a.x - s, a.y - s); }
inline float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
inline float2 operator/(float2 a, float s) { return make_float2(a.x / s, a.y / s); }
inline float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
inline float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
inline float2 &operator+=(float2 &a, float2 b) { a = a + b; return a; }
inline float2 &operator-=(float2 &a, float2 b) { a = a - b; return a; }
inline float2 &operator*=(float2 &a, float s) { a = a * s; return a; }
inline float2 &operator/=(float2 &a, float s) { a = a / s; return a; }

// float3 arithmetic
inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator+(float3 a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
inline float3 operator-(float3 a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator/(float s, float3 a) { return make_float3(s / a.x, s / a.y, s / a.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
inline float3 &operator-=(float3 &a, float3 b) { a = a - b; return a; }
inline float3 &operator*=(float3 &a, float3 b) { a = a * b; return a; }
inline float3 &operator*=(float3 &a, float s) { a = a * s; return a; }
inline float3 &operator/=(float3 &a, float s) { a = a / s; return a; }
inline float3 &operator+=(float3 &a, float s) { a = a + s; return a; }

// comparisons give OpenCL masks (-1 true, 0 false)
inline int3 operator>(float3 a, float s) { return make_int3(a.x > s ? -1 : 0, a.y > s ? -1 : 0, a.z > s ? -1 : 0); }
inline int3 operator<(float3 a, float s) { return make_int3(a.x < s ? -1 : 0, a.y < s ? -1 : 0, a.z < s ? -1 : 0); }
inline int3 operator>=(int3 a, int s) { return make_int3(a.x >= s ? -1 : 0, a.y >= s ? -1 : 0, a.z >= s ? -1 : 0); }
inline int3 operator<(int3 a, int s) { return make_int3(a.x < s ? -1 : 0, a.y < s ? -1 : 0, a.z < s ? -1 : 0); }
inline bool all(int3 m) { return m.x < 0 && m.y < 0 && m.z < 0; }

// built-ins
inline float dot(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float3 fabs(float3 a) { return make_float3(::fabsf(a.x), ::fabsf(a.y), ::fabsf(a.z)); }
inline float fabs(float a) { return ::fabsf(a); }
inline float min(float a, float b) { return ::fminf(a, b); }
inline float max(float a, float b) { return ::fmaxf(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float clamp(float x, float lo, float hi) { return ::fminf(::fmaxf(x, lo), hi); }
inline float floor(float x) { return ::floorf(x); }
inline float ceil(float x) { return ::ceilf(x); }
inline float sqrt(float x) { return ::sqrtf(x); }
inline float3 sqrt(float3 a) { return make_float3(::sqrtf(a.x), ::sqrtf(a.y), ::sqrtf(a.z)); }
inline int abs(int x) { return x < 0 ? (int)(0u - (unsigned)x) : x; }
inline float round(float x) { return ::roundf(x); }
inline float3 cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float3 operator*(int s, float3 a) { return (float)s * a; }
inline float3 fast_normalize(float3 v) { return v * (1.0f / ::sqrtf(dot(v, v))); }
inline float fast_length(float3 v) { return ::sqrtf(dot(v, v)); }
inline float3 max(float3 a, float s) { return make_float3(::fmaxf(a.x, s), ::fmaxf(a.y, s), ::fmaxf(a.z, s)); }
inline int cvt_int(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x <= -2147483648.0f) return INT_MIN;
  return (int)x;
}
inline int3 convert_int3(float3 a) { return make_int3(cvt_int(a.x), cvt_int(a.y), cvt_int(a.z)); }
inline ushort convert_ushort(float x) {
  int v = cvt_int(x);
  return (ushort)(v < 0 ? 0 : (v > 65535 ? 65535 : v));
}
inline ushort convert_ushort_sat(float x) { return convert_ushort(x); }

// A u16 buffer element whose implicit conversion from float (a store such as
// `Ro[i] = x * y`, undefined out of range in C) is pinned as convert_ushort's
// truncate-and-saturate.  Kernels whose stores rely on it see `ushort` as this
// type (build_ref.py gives them a one-line prelude).
struct sat_u16 {
  unsigned short v;
  operator float() const { return (float)v; }
  sat_u16 &operator=(float x) { v = convert_ushort(x); return *this; }
};
static_assert(sizeof(sat_u16) == 2, "sat_u16 aliases a u16 buffer");
inline float3 convert_float3(ushort3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }

// for the normal-mapped mip material (Shaders_src/av_draw_normmap_mip.c)
struct uchar3 {
  uchar x, y, z, pad_;   // OpenCL uchar3 occupies 4 bytes
};
static_assert(sizeof(uchar3) == 4, "OpenCL uchar3 occupies 4 bytes");
inline float3 convert_float3(uchar3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
inline float2 fabs(float2 a) { return make_float2(::fabsf(a.x), ::fabsf(a.y)); }
// log2 correctly rounded (the convention pinned for the library and the
// oracle): the double result rounded once to float
inline float log2(float x) { return (float)::log2((double)x); }
// exp2 correctly rounded (the double result rounded once), half_sqrt as the
// correctly rounded square root: conventions where OpenCL leaves the
// precision to the device
inline float exp2(float x) { return (float)::exp2((double)x); }
inline float half_sqrt(float x) { return ::sqrtf(x); }
// pown(x, n) = x^n for integer n, by repeated squaring of |n| then, for
// negative n, the reciprocal (OpenCL leaves its rounding to the device)
inline float pown(float x, int n) {
  unsigned k = n < 0 ? 0u - (unsigned)n : (unsigned)n;
  float r = 1.0f, b = x;
  while (k) {
    if (k & 1u) r *= b;
    b *= b;
    k >>= 1;
  }
  return n < 0 ? 1.0f / r : r;
}

}  // namespace cl_shim
