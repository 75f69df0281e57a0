// raster.cuh -- device-side arithmetic of the rasterizer hot path (sm_100a).
//
// Every float operation is written out in the reference's order and compiled
// with -fmad=false (no contraction), IEEE division and square root, so that
// coverage, triangle ids and depth are bit-identical to the reference's
// kernels run serially.  Conventions where OpenCL leaves a choice:
//   dot = (a.x*b.x + a.y*b.y) + a.z*b.z; min/max/clamp = fminf/fmaxf;
//   float->int truncates, saturates, NaN -> 0 (cvt.rzi); fast_normalize =
//   v * (1/sqrt(dot)); convert_ushort = truncate then saturate; log2 =
//   own correctly rounded series (axr_log2f).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace axr {

// F_MULTI: av_draw_multi.c's 4-way blend with the next three groups' textures;
// F_NORMAL: the normal-mapped materials (av_draw_normmap.c, with F_ALPHA
// av_draw_normmap_alpha.c, with F_MIP av_draw_normmap_mip.c)
enum { F_MIP = 1, F_ALPHA = 2, F_SHADOW = 4, F_CULL = 8, F_MULTI = 16, F_NORMAL = 32 };
constexpr int TILE = 16;
constexpr int SMALL_THRESH = 6;
constexpr unsigned FULL = 0xffffffffu;

struct GroupDev {
  const float *xyz, *vn, *uv, *li;
  const ushort4 *tex;     // texels as (R, G, B, 0): one 8-byte load per bilinear tap
  const uint8_t *amask;   // alpha mask, one byte per texel (nearest-texel tests)
  const uint8_t *aquad;   // per texel the 4 taps of its bilinear footprint as bits
  int alen;
  int ntris, tri_base, tex_size, flags;
  float mip_bias;
  int enabled;
  int pad_;
  // F_NORMAL: normal map (R, G, B, unused) with one texel per texel of the
  // texture or chain; the specular powers (int)exp2(12 (1 - roughness)) and
  // (int)sqrt of it; the metal switch
  const uchar4 *nm;
  int spec_pow, spec_pow2, is_metal;
  int pad2_;
};

struct ViewDev {
  int w, h;
  float pos[3], vv[9];
  float sscale, cax, cay;
};

struct ShadowDev {
  const float *map;
  int dim;
  float scale;
  float pos[3], vv[9];
};

struct LightDev {
  float lint[3], ldir[3], amb;
};

// ------------------------------------------------------------ scalars

__device__ __forceinline__ int f2i(float x) { return __float2int_rz(x); }
// t = max(0, min(1, t)) with min/max = fminf/fmaxf, so NaN (0/0 on one-pixel
// spans) gives 1.  Written with an explicit NaN branch because the compiler
// may otherwise fold the clamp into a saturate, which maps NaN to 0.
__device__ __forceinline__ float clamp_t(float t) { return t != t ? 1.0f : fmaxf(0.f, fminf(1.f, t)); }
__device__ __forceinline__ int iabs_(int x) { return x < 0 ? (int)(0u - (unsigned)x) : x; }
__device__ __forceinline__ float clampf_(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ uint16_t u16sat(float x) {
  int v = f2i(x);
  v = v < 0 ? 0 : v;
  v = v > 65535 ? 65535 : v;
  return (uint16_t)v;
}

// log2 by exponent extraction and ln(m) = 2*atanh((m-1)/(m+1)) summed in
// double (plain IEEE operations only), rounded once to float.
__device__ __forceinline__ float axr_log2f(float x) {
  if (x != x) return x;
  if (x < 0.0f) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return __int_as_float(0xff800000);
  if (isinf(x)) return x;
  uint32_t u = __float_as_uint(x);
  int e;
  if ((u >> 23) == 0) {
    u = __float_as_uint(x * 16777216.0f);
    e = (int)(u >> 23) - 127 - 24;
  } else {
    e = (int)(u >> 23) - 127;
  }
  uint32_t man = u & 0x7fffffu;
  double m = 1.0 + (double)man / 8388608.0;
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  double term = s, sum = s;
  // atanh series s + s^3/3 + ... + s^19/19, the divisions as products with the
  // reciprocals (same constants and order as the oracle's orc_log2f)
  const double inv[9] = {1.0 / 3, 1.0 / 5, 1.0 / 7, 1.0 / 9, 1.0 / 11, 1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19};
#pragma unroll
  for (int k = 1; k <= 9; k++) {
    term = term * s2;
    sum = sum + term * inv[k - 1];
  }
  double r = (double)e + sum * 2.8853900817779268;
  return (float)r;
}

// Correctly rounded n/d from y = RN(1/d) (Markstein's theorem, "Computation
// of elementary functions on the IBM RISC System/6000", IBM J. R&D 1990):
// q = RN(n*y), r = n - d*q (exact with a fused multiply-add), RN(q + r*y) is
// RN(n/d) when nothing overflows or underflows.  span_recip returns y, or 0
// when d is outside [2^-60, 2^60] (zero, denormal, huge, inf, NaN) and the
// caller must divide; quot_by_recip also divides when |n| is outside that
// range, so every quotient equals the IEEE division bit for bit.
__device__ __forceinline__ float span_recip(float d) {
  float a = fabsf(d);
  return (a >= 8.6736174e-19f && a <= 1.1529215e18f) ? __frcp_rn(d) : 0.f;
}
// y of span_recip(d) when, in addition, every quotient (ax - cx2) / d of the
// span's pixels (integer ax >= lo >= 0) can take the reciprocal path: then
// |ax - cx2| <= 2^60 and it is 0 or >= 2^-60 (for |cx2| >= 2^-36 the exact
// difference is a multiple of ulp(cx2) >= 2^-59; for smaller cx2 it is
// either cx2 itself, when ax = 0 and cx2 = 0, or at least 1 - 2^-36).
// Returns 0 when a pixel might need the true division.
__device__ __forceinline__ float span_recip_exact(float d, float cx2, int lo) {
  float y = span_recip(d);
  float a = fabsf(cx2);
  bool ok = a <= 0x1p59f && (a >= 0x1p-36f || cx2 == 0.f || lo > 0);
  return ok ? y : 0.f;
}

// The quotient of quot_by_recip when the operands are known to be in range.
__device__ __forceinline__ float quot_fast(float n, float d, float y) {
  float q = __fmul_rn(n, y);
  float r = __fmaf_rn(-d, q, n);
  return __fmaf_rn(r, y, q);
}

// t = clamp(n / d, 0, 1) of a pixel of a span queued by span_queue_form.
// The operands are in range there (finite, d and y nonzero), so the
// quotient is never NaN and the clamp needs no NaN rule.
__device__ __forceinline__ float span_t(float n, float d, float y) {
  return fmaxf(0.f, fminf(1.f, quot_fast(n, d, y)));
}

// The (cx2, d, y) a span with first pixel lo is queued with, so that every
// pixel x of it takes t = span_t(x - cx2, d, y).  Usually (cx2, d, RN(1/d)).
// d = cx1 - cx2 = +-0 means cx1 and cx2 are equal (or both zero), so the
// span is the one pixel lo: its n / d is an infinity of sign sign(n) xor
// sign(d), clamped to 1 or 0, or NaN for n = 0, clamped to 1; that t is
// fixed here as cx2 = lo - 1 (t = 1) or lo + 1 (t = 0) with d = y = 1.
// Returns false when a pixel might need the true division (a reciprocal out
// of the safe range with d != 0, which real scenes almost never produce):
// the span's own lane then draws it with the true cx2 and d.
__device__ __forceinline__ bool span_queue_form(float cx2, float d, int lo, float &qx, float &qd, float &qy) {
  qx = cx2;
  qd = d;
  qy = span_recip_exact(d, cx2, lo);
  if (qy != 0.f) return true;
  if (d != 0.f) return false;
  float n = (float)lo - cx2;
  bool one = n == 0.f || ((__float_as_uint(n) ^ __float_as_uint(d)) & 0x80000000u) == 0u;
  qx = (float)lo - (one ? 1.f : -1.f);
  qd = 1.f;
  qy = 1.f;
  return true;
}

__device__ __forceinline__ float quot_by_recip(float n, float d, float y) {
  float an = fabsf(n);
  if (y != 0.f && an <= 1.1529215e18f && (an >= 8.6736174e-19f || n == 0.f)) {
    float q = __fmul_rn(n, y);
    float r = __fmaf_rn(-d, q, n);
    return __fmaf_rn(r, y, q);
  }
  return n / d;
}

// ------------------------------------------------------------ order keys
// 64-bit visibility word: high = monotone depth key, low = ~order, so that
// atomicMin keeps the smallest depth and, on equal depth, the fragment that
// the serial reference would have drawn last.  order 0 = prior contents.

__device__ __forceinline__ uint32_t depth_key(float z) {
  uint32_t u = __float_as_uint(z);
  if ((u & 0x7fffffffu) == 0) u = 0;                  // -0 compares equal to +0
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0u;      // NaN depth: nothing passes
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ uint32_t make_order(int phase, uint32_t gtri, int half) {
  return 1u + (((uint32_t)phase << 31) | (gtri << 1) | (uint32_t)half);
}
__device__ __forceinline__ uint64_t frag_key(float tz, uint32_t ord) {
  return ((uint64_t)depth_key(tz) << 32) | (uint64_t)(0xffffffffu - ord);
}

// ------------------------------------------------------------ vectors

struct V2 { float x, y; };
struct V3 { float x, y, z; };
__device__ __forceinline__ V3 ld3(const float *__restrict__ p) { return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }
__device__ __forceinline__ V2 ld2(const float *__restrict__ p) { return V2{__ldg(p), __ldg(p + 1)}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 mul3(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 smul3(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 div3(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 neg3(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V2 sub2(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ V2 add2(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ V2 mul2(V2 a, float s) { return V2{a.x * s, a.y * s}; }
__device__ __forceinline__ V2 smul2(float s, V2 a) { return V2{s * a.x, s * a.y}; }
__device__ __forceinline__ V2 div2(V2 a, float s) { return V2{a.x / s, a.y / s}; }
__device__ __forceinline__ V2 neg2(V2 a) { return V2{-a.x, -a.y}; }
__device__ __forceinline__ V3 fast_normalize(V3 v) { return mul3(v, 1.0f / sqrtf(dot3(v, v))); }

// Attribute bundle interpolated along the two active edges (the AVSL
// `currvert*` values): UV, light I, normal N, world position PXYZ, all * z.
// FULL=false carries UV only (alpha test in the visibility pass).
template <bool FULL>
struct Attr {
  V2 uv;
  V3 li, n, p;
};
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_sub(Attr<FULL> a, Attr<FULL> b) {
  Attr<FULL> r; r.uv = sub2(a.uv, b.uv);
  if (FULL) { r.li = sub3(a.li, b.li); r.n = sub3(a.n, b.n); r.p = sub3(a.p, b.p); }
  return r;
}
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_add(Attr<FULL> a, Attr<FULL> b) {
  Attr<FULL> r; r.uv = add2(a.uv, b.uv);
  if (FULL) { r.li = add3(a.li, b.li); r.n = add3(a.n, b.n); r.p = add3(a.p, b.p); }
  return r;
}
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_mul(Attr<FULL> a, float s) {
  Attr<FULL> r; r.uv = mul2(a.uv, s);
  if (FULL) { r.li = mul3(a.li, s); r.n = mul3(a.n, s); r.p = mul3(a.p, s); }
  return r;
}
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_smul(float s, Attr<FULL> a) {
  Attr<FULL> r; r.uv = smul2(s, a.uv);
  if (FULL) { r.li = smul3(s, a.li); r.n = smul3(s, a.n); r.p = smul3(s, a.p); }
  return r;
}
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_neg(Attr<FULL> a) {
  Attr<FULL> r; r.uv = neg2(a.uv);
  if (FULL) { r.li = neg3(a.li); r.n = neg3(a.n); r.p = neg3(a.p); }
  return r;
}
template <bool FULL> __device__ __forceinline__ Attr<FULL> a_load(const GroupDev &g, int tri, int k, float z) {
  Attr<FULL> a;
  size_t vi = (size_t)tri * 3 + k;
  a.uv = mul2(ld2(g.uv + vi * 2), z);
  if (FULL) {
    a.li = mul3(ld3(g.li + vi * 3), z);
    a.n = mul3(ld3(g.vn + vi * 3), z);
    a.p = mul3(ld3(g.xyz + vi * 3), z);
  }
  return a;
}

// ------------------------------------------------------------ setup

// trisetup.c:29-80 / trisetup_cull.c:49-54: returns 0 rejected, 1 small, 2 large
__device__ __forceinline__ int project_persp(const GroupDev &g, int tri, const ViewDev &v, float sx[3], float sy[3],
                                             float sz[3]) {
  V3 vp{v.pos[0], v.pos[1], v.pos[2]};
  V3 svd{v.vv[0], v.vv[1], v.vv[2]}, svx{v.vv[3], v.vv[4], v.vv[5]}, svy{v.vv[6], v.vv[7], v.vv[8]};
  V3 x[3];
  float dd[3], dx[3], dy[3];
  const float *p = g.xyz + (size_t)tri * 9;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    x[k] = sub3(ld3(p + 3 * k), vp);
    dd[k] = dot3(x[k], svd);
    dx[k] = dot3(x[k], svx);
    dy[k] = dot3(x[k], svy);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    dd[k] = 1.0f / dd[k];
    dx[k] = dx[k] * dd[k];
    dy[k] = dy[k] * dd[k];
  }
  bool yes = dd[0] > 0 && dd[1] > 0 && dd[2] > 0 && fabsf(dx[0]) < v.cax && fabsf(dx[1]) < v.cax &&
             fabsf(dx[2]) < v.cax && fabsf(dy[0]) < v.cay && fabsf(dy[1]) < v.cay && fabsf(dy[2]) < v.cay;
  if (g.flags & F_CULL) {
    const float *n = g.vn + (size_t)tri * 9;
    if (dot3(ld3(n), x[0]) < -0.0f && dot3(ld3(n + 3), x[1]) < -0.0f && dot3(ld3(n + 6), x[2]) < -0.0f) yes = false;
  }
  float hw = (float)(v.w / 2), hh = (float)(v.h / 2);
  int dix[3], diy[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    dx[k] = dx[k] * -v.sscale + hw;
    dy[k] = dy[k] * v.sscale + hh;
    dix[k] = f2i(dx[k]);
    diy[k] = f2i(dy[k]);
    sx[k] = dx[k]; sy[k] = dy[k]; sz[k] = dd[k];
  }
  int maxX = max(dix[0], max(dix[1], dix[2])), minX = min(dix[0], min(dix[1], dix[2]));
  int maxY = max(diy[0], max(diy[1], diy[2])), minY = min(diy[0], min(diy[1], diy[2]));
  long long dimx = (long long)maxX - minX, dimy = (long long)maxY - minY;
  if (dimx == 0 || dimx > 2LL * v.w) yes = false;
  if (dimy == 0 || dimy > 2LL * v.h) yes = false;
  if (maxX < 0 || maxY < 0 || minX > v.w || minY > v.h) yes = false;
  if (!yes) return 0;
  return ((dimx > dimy ? dimx : dimy) < SMALL_THRESH * TILE) ? 1 : 2;
}

// trisetupOrtho.c:20-59
__device__ __forceinline__ bool project_ortho(const GroupDev &g, int tri, const ShadowDev &s, float bias, int ix[3],
                                              int iy[3], float z[3]) {
  V3 vp{s.pos[0], s.pos[1], s.pos[2]};
  V3 svd{s.vv[0], s.vv[1], s.vv[2]}, svx{s.vv[3], s.vv[4], s.vv[5]}, svy{s.vv[6], s.vv[7], s.vv[8]};
  const float *p = g.xyz + (size_t)tri * 9;
  bool yes = true;
  float half = (float)(s.dim / 2);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    V3 x = sub3(ld3(p + 3 * k), vp);
    float dd = dot3(x, svd);
    float dx = dot3(x, svx);
    float dy = dot3(x, svy);
    dd = dd + bias;
    dd = 1.0f / dd;
    dx = dx * s.scale + half;
    dy = dy * -s.scale + half;
    ix[k] = f2i(dx);
    iy[k] = f2i(dy);
    z[k] = dd;
    if (!(dd > 0) || ix[k] < -120 || ix[k] >= s.dim + 120 || iy[k] < -120 || iy[k] >= s.dim + 120) yes = false;
  }
  return yes;
}

// per-triangle mip level of av_draw_normmap_mip.c:26-59
struct MipSel {
  float fmip;
  int mip, len_mip, len_mip2, start_mip, start_mip2;
};

// Applies the UV/PXYZ round trip (/z then *z) of the mip setup to vertices
// 1..3 and returns the level; edge lengths from the (sorted) screen coords,
// computed in int on the direct path (ix/iy) and in float on the tiled path.
template <bool FULL>
__device__ __forceinline__ MipSel mip_setup(Attr<FULL> a[3], const float z[3], bool small, const int *ix,
                                            const int *iy, const float *x, const float *y, int num_mip,
                                            float mip_bias) {
  V2 uv1 = div2(a[0].uv, z[0]), uv2 = div2(a[1].uv, z[1]), uv3 = div2(a[2].uv, z[2]);
  V3 p1, p2, p3;
  if (FULL) { p1 = div3(a[0].p, z[0]); p2 = div3(a[1].p, z[1]); p3 = div3(a[2].p, z[2]); }
  V2 d1 = sub2(uv2, uv1), d2 = sub2(uv3, uv1), d3 = sub2(uv3, uv2);
  float l1, l2, l3;
  if (small) {
    l1 = (float)((iy[1] - iy[0]) * (iy[1] - iy[0]) + (ix[1] - ix[0]) * (ix[1] - ix[0]));
    l2 = (float)((iy[2] - iy[0]) * (iy[2] - iy[0]) + (ix[2] - ix[0]) * (ix[2] - ix[0]));
    l3 = (float)((iy[2] - iy[1]) * (iy[2] - iy[1]) + (ix[2] - ix[1]) * (ix[2] - ix[1]));
  } else {
    l1 = (y[1] - y[0]) * (y[1] - y[0]) + (x[1] - x[0]) * (x[1] - x[0]);
    l2 = (y[2] - y[0]) * (y[2] - y[0]) + (x[2] - x[0]) * (x[2] - x[0]);
    l3 = (y[2] - y[1]) * (y[2] - y[1]) + (x[2] - x[1]) * (x[2] - x[1]);
  }
  V2 s1 = div2(d1, l1), s2 = div2(d2, l2), s3 = div2(d3, l3);
  float dt = fmaxf(fabsf(s1.x), fmaxf(fabsf(s1.y), fmaxf(fabsf(s2.x), fabsf(s2.y))));
  dt = fmaxf(dt, fmaxf(fabsf(s3.x), fabsf(s3.y)));
  float fmip = fmaxf(0.f, fminf((float)(num_mip - 1), fabsf(axr_log2f(dt)) / 2.0f + mip_bias));
  MipSel m;
  m.mip = f2i(fmip);
  m.fmip = fmip - (float)m.mip;
  m.len_mip = 1 << m.mip;
  m.len_mip2 = m.len_mip << 1;
  int start = 0;
  for (int i = 0; i < m.mip; i++) start += (1 << i) * (1 << i);
  m.start_mip = start;
  m.start_mip2 = start + m.len_mip * m.len_mip;
  a[0].uv = mul2(uv1, z[0]); a[1].uv = mul2(uv2, z[1]); a[2].uv = mul2(uv3, z[2]);
  if (FULL) { a[0].p = mul3(p1, z[0]); a[1].p = mul3(p2, z[1]); a[2].p = mul3(p3, z[2]); }
  return m;
}

// The attribute round trip mip_setup makes (uv and position divided by the
// vertex z, then multiplied back), for callers that have the mip level
// already: the interpolants must be these values, bit for bit.
template <bool FULL>
__device__ __forceinline__ void mip_attr_roundtrip(Attr<FULL> a[3], const float z[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    V2 uv = div2(a[k].uv, z[k]);
    a[k].uv = mul2(uv, z[k]);
    if (FULL) {
      V3 p = div3(a[k].p, z[k]);
      a[k].p = mul3(p, z[k]);
    }
  }
}

// bilinear taps of av_draw_base.c:29-42 at side `len`, texel offset `start`
struct Taps {
  int tex, tex10, tex01, tex11;
  float texr1, texr2, texi1, texi2;
};
__device__ __forceinline__ Taps make_taps(V2 uvi, float tz, int len, int start) {
  Taps q;
  float rx = (uvi.x * tz) * (float)len;
  float ry = (uvi.y * tz) * (float)len;
  int t1 = f2i(rx);
  rx -= (float)t1;
  t1 = iabs_(t1) & (len - 1);
  int t2 = f2i(ry);
  ry -= (float)t2;
  t2 = iabs_(t2) & (len - 1);
  int t1n = min(t1 + 1, len - 1), t2n = min(t2 + 1, len - 1);
  q.tex = start + t1 + len * t2;
  q.tex10 = start + t1n + len * t2;
  q.tex01 = start + t1 + len * t2n;
  q.tex11 = start + t1n + len * t2n;
  q.texr1 = rx; q.texr2 = ry;
  q.texi1 = 1 - rx; q.texi2 = 1 - ry;
  return q;
}
// bilinear R, G, B of av_draw_base.c:50-55 (same products and sums per channel)
__device__ __forceinline__ V3 bilerp_rgb(const Taps &q, const ushort4 *__restrict__ T) {
  ushort4 a = __ldg(T + q.tex), b = __ldg(T + q.tex10), c = __ldg(T + q.tex01), d = __ldg(T + q.tex11);
  float w00 = q.texi1 * q.texi2, w10 = q.texr1 * q.texi2, w01 = q.texi1 * q.texr2, w11 = q.texr1 * q.texr2;
  V3 r;
  r.x = w00 * (float)a.x + w10 * (float)b.x + w01 * (float)c.x + w11 * (float)d.x;
  r.y = w00 * (float)a.y + w10 * (float)b.y + w01 * (float)c.y + w11 * (float)d.y;
  r.z = w00 * (float)a.z + w10 * (float)b.z + w01 * (float)c.z + w11 * (float)d.z;
  return r;
}
// bilinear boolean alpha of av_draw_alpha.c:95-96 from the packed footprint:
// bit 0 = tap (t1,t2), bit 1 = (t1+1,t2), bit 2 = (t1,t2+1), bit 3 = (t1+1,t2+1)
__device__ __forceinline__ float bilerp_quad(const Taps &q, const uint8_t *__restrict__ Q) {
  unsigned m = __ldg(Q + q.tex);
  return q.texi1 * q.texi2 * (float)(m & 1) + q.texr1 * q.texi2 * (float)((m >> 1) & 1) +
         q.texi1 * q.texr2 * (float)((m >> 2) & 1) + q.texr1 * q.texr2 * (float)((m >> 3) & 1);
}
__device__ __forceinline__ float bilerp_u16(const Taps &q, const uint16_t *__restrict__ T) {
  return q.texi1 * q.texi2 * (float)__ldg(T + q.tex) + q.texr1 * q.texi2 * (float)__ldg(T + q.tex10) +
         q.texi1 * q.texr2 * (float)__ldg(T + q.tex01) + q.texr1 * q.texr2 * (float)__ldg(T + q.tex11);
}
__device__ __forceinline__ float bilerp_bool(const Taps &q, const uint8_t *__restrict__ T) {
  return q.texi1 * q.texi2 * (float)(__ldg(T + q.tex) != 0) + q.texr1 * q.texi2 * (float)(__ldg(T + q.tex10) != 0) +
         q.texi1 * q.texr2 * (float)(__ldg(T + q.tex01) != 0) + q.texr1 * q.texr2 * (float)(__ldg(T + q.tex11) != 0);
}

}  // namespace axr
