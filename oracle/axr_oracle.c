/*
 * axr_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see axr_oracle.h).
 *
 * Compiled with -O2 -ffp-contract=off -fno-fast-math (x86-64 SSE): every
 * float operation below is one IEEE-754 single rounding, in source order.
 * Conventions pinned where the OpenCL source leaves them to the compiler:
 *   - dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, no fused multiply-add
 *   - min/max/clamp on floats = fminf/fmaxf (NaN -> the other operand)
 *   - float->int truncates toward zero, saturates, NaN -> 0 (f2i)
 *   - fast_normalize(v) = v * (1/sqrtf(dot(v,v))), fast_length(v) = sqrtf(dot(v,v))
 *   - convert_ushort = truncate, then saturate to [0, 65535]
 *   - log2 = orc_log2f (correctly rounded, own series evaluation)
 */
#include "axr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TILE 16
#define SMALL_THRESH 6

/* ------------------------------------------------------------------ */
/* scalar helpers                                                      */
/* ------------------------------------------------------------------ */

static inline int f2i(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x <= -2147483648.0f) return INT_MIN;
  return (int)x;
}
static inline int iabs(int x) { return x < 0 ? (int)(0u - (unsigned)x) : x; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline float fclampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static inline uint16_t u16sat(float x) {
  int v = f2i(x);
  if (v < 0) v = 0;
  if (v > 65535) v = 65535;
  return (uint16_t)v;
}

typedef struct { float x, y; } f2;
typedef struct { float x, y, z; } f3;

static inline f3 f3ld(const float *p) { f3 r = {p[0], p[1], p[2]}; return r; }
static inline f2 f2ld(const float *p) { f2 r = {p[0], p[1]}; return r; }
static inline float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline f3 f3sub(f3 a, f3 b) { f3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline f3 f3add(f3 a, f3 b) { f3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline f3 f3mul(f3 a, float s) { f3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline f3 f3smul(float s, f3 a) { f3 r = {s * a.x, s * a.y, s * a.z}; return r; }
static inline f3 f3div(f3 a, float s) { f3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static inline f3 f3neg(f3 a) { f3 r = {-a.x, -a.y, -a.z}; return r; }
static inline f2 f2sub(f2 a, f2 b) { f2 r = {a.x - b.x, a.y - b.y}; return r; }
static inline f2 f2add(f2 a, f2 b) { f2 r = {a.x + b.x, a.y + b.y}; return r; }
static inline f2 f2mul(f2 a, float s) { f2 r = {a.x * s, a.y * s}; return r; }
static inline f2 f2smul(float s, f2 a) { f2 r = {s * a.x, s * a.y}; return r; }
static inline f2 f2div(f2 a, float s) { f2 r = {a.x / s, a.y / s}; return r; }
static inline f2 f2neg(f2 a) { f2 r = {-a.x, -a.y}; return r; }
static inline f3 fast_normalize(f3 v) { return f3mul(v, 1.0f / sqrtf(dot3(v, v))); }

/* log2 by exponent extraction and the atanh series
 *   ln(m) = 2 * (s + s^3/3 + s^5/5 + ...),  s = (m-1)/(m+1)
 * with m reduced to [sqrt(1/2), sqrt(2)), evaluated in double with plain
 * IEEE operations (so the same source gives the same bits on any IEEE
 * machine without contraction) and rounded once to float. */
float orc_log2f(float x) {
  if (x != x) return x;
  if (x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (isinf(x)) return INFINITY;
  union { float f; uint32_t u; } v; v.f = x;
  int e;
  uint32_t man;
  if ((v.u >> 23) == 0) {            /* subnormal: scale by 2^24 */
    v.f = x * 16777216.0f;
    e = (int)(v.u >> 23) - 127 - 24;
  } else {
    e = (int)(v.u >> 23) - 127;
  }
  man = v.u & 0x7fffffu;
  double m = 1.0 + (double)man / 8388608.0;
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  double term = s, sum = s;
  /* atanh series s + s^3/3 + ... + s^19/19, the divisions as products with the
     reciprocals (same constants and order as the CUDA side's axr_log2f) */
  static const double inv[9] = {1.0 / 3, 1.0 / 5, 1.0 / 7, 1.0 / 9, 1.0 / 11, 1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19};
  for (int k = 1; k <= 9; k++) {
    term = term * s2;
    sum = sum + term * inv[k - 1];
  }
  double r = (double)e + sum * 2.8853900817779268; /* 2/ln(2) */
  return (float)r;
}

/* ------------------------------------------------------------------ */
/* triangle setup: PyOpenCL27C/Pipe/trisetup.c:29-80, trisetup_cull.c:49-54 */
/* ------------------------------------------------------------------ */

static int setup_persp_tri(const orc_group *g, const orc_frame *f, int i,
                           float sx[3], float sy[3], float sz[3]) {
  f3 vp = {f->pos[0], f->pos[1], f->pos[2]};
  f3 svd = f3ld(f->vv), svx = f3ld(f->vv + 3), svy = f3ld(f->vv + 6);
  f3 x[3];
  float dd[3], dx[3], dy[3];
  for (int k = 0; k < 3; k++) {
    x[k] = f3sub(f3ld(g->xyz + (size_t)(i * 3 + k) * 3), vp);
    dd[k] = dot3(x[k], svd);
    dx[k] = dot3(x[k], svx);
    dy[k] = dot3(x[k], svy);
  }
  for (int k = 0; k < 3; k++) {
    dd[k] = 1.0f / dd[k];
    dx[k] = dx[k] * dd[k];
    dy[k] = dy[k] * dd[k];
  }
  int yes = 0;
  if (dd[0] > 0 && dd[1] > 0 && dd[2] > 0 &&
      fabsf(dx[0]) < f->cax && fabsf(dx[1]) < f->cax && fabsf(dx[2]) < f->cax &&
      fabsf(dy[0]) < f->cay && fabsf(dy[1]) < f->cay && fabsf(dy[2]) < f->cay)
    yes = 1;
  if (g->flags & ORC_CULL) {
    f3 n0 = f3ld(g->vn + (size_t)(i * 3 + 0) * 3);
    f3 n1 = f3ld(g->vn + (size_t)(i * 3 + 1) * 3);
    f3 n2 = f3ld(g->vn + (size_t)(i * 3 + 2) * 3);
    if (dot3(n0, x[0]) < -0.0f && dot3(n1, x[1]) < -0.0f && dot3(n2, x[2]) < -0.0f) yes = 0;
  }
  float hw = (float)(f->w / 2), hh = (float)(f->h / 2);
  int dix[3], diy[3];
  for (int k = 0; k < 3; k++) {
    dx[k] = dx[k] * -f->sscale + hw;
    dy[k] = dy[k] * f->sscale + hh;
    dix[k] = f2i(dx[k]);
    diy[k] = f2i(dy[k]);
  }
  int maxX = imax(dix[0], imax(dix[1], dix[2])), minX = imin(dix[0], imin(dix[1], dix[2]));
  int maxY = imax(diy[0], imax(diy[1], diy[2])), minY = imin(diy[0], imin(diy[1], diy[2]));
  long long dimx = (long long)maxX - minX, dimy = (long long)maxY - minY;
  if (dimx == 0 || dimx > 2LL * f->w) yes = 0;
  if (dimy == 0 || dimy > 2LL * f->h) yes = 0;
  if (maxX < 0 || maxY < 0 || minX > f->w || minY > f->h) yes = 0;
  for (int k = 0; k < 3; k++) { sx[k] = dx[k]; sy[k] = dy[k]; sz[k] = dd[k]; }
  if (!yes) return 0;
  return ((dimx > dimy ? dimx : dimy) < SMALL_THRESH * TILE) ? 1 : 2;
}

void orc_setup_persp(const orc_group *g, const orc_frame *f, uint8_t *cls,
                     float *sp, float *zz) {
  for (int i = 0; i < g->ntris; i++) {
    float sx[3], sy[3], sz[3];
    int c = setup_persp_tri(g, f, i, sx, sy, sz);
    cls[i] = (uint8_t)c;
    for (int k = 0; k < 3; k++) {
      sp[(i * 3 + k) * 2] = sx[k];
      sp[(i * 3 + k) * 2 + 1] = sy[k];
      zz[i * 3 + k] = sz[k];
    }
  }
}

/* ------------------------------------------------------------------ */
/* fragment shading                                                    */
/* ------------------------------------------------------------------ */

/* per-draw context handed to the fragment core */
typedef struct {
  const orc_frame *f;
  const orc_group *g;
  const orc_alpha *alpha;      /* mask sampled by the alpha test, or NULL */
  const orc_shadow *sh;
  int nsh;
  int gid_base;
  int num_mip;                 /* mip materials */
  float fmip;                  /* per-triangle mip fraction */
  int mip, len_mip, len_mip2, start_mip, start_mip2;
  f3 tangent, bitangent;       /* normal-mapped materials: per-triangle frame */
  int spec_pow, spec_pow2;     /* (int)exp2(12 (1 - roughness)), (int)half_sqrt of it */
} shade_ctx;

/* attribute bundle interpolated along the two active edges
 * (Templates.py "currvert*1/2"); PXYZ is the world position */
typedef struct { f2 uv; f3 li, n, p; } attrs;

static inline attrs at_lerp_dummy(void) { attrs a; memset(&a, 0, sizeof a); return a; }

/* bilinear taps of av_draw_base.c:29-42 at side length len (power of two),
 * texel offset `start` */
typedef struct { int tex, tex10, tex01, tex11; float texr1, texr2, texi1, texi2; } taps;

static inline taps make_taps(f2 uvi, float tz, int len, int start) {
  taps q;
  f2 texr12 = f2mul(f2mul(uvi, tz), (float)len);
  int tex1 = f2i(texr12.x);
  texr12.x -= (float)tex1;
  tex1 = iabs(tex1) & (len - 1);
  int tex2 = f2i(texr12.y);
  texr12.y -= (float)tex2;
  tex2 = iabs(tex2) & (len - 1);
  q.tex = start + tex1 + len * tex2;
  q.tex10 = start + imin(tex1 + 1, len - 1) + len * tex2;
  q.tex01 = start + tex1 + len * imin(tex2 + 1, len - 1);
  q.tex11 = start + imin(tex1 + 1, len - 1) + len * imin(tex2 + 1, len - 1);
  q.texr1 = texr12.x; q.texr2 = texr12.y;
  q.texi1 = 1 - q.texr1; q.texi2 = 1 - q.texr2;
  return q;
}

static inline float bilerp_u16(const taps *q, const uint16_t *T) {
  return q->texi1 * q->texi2 * (float)T[q->tex] + q->texr1 * q->texi2 * (float)T[q->tex10] +
         q->texi1 * q->texr2 * (float)T[q->tex01] + q->texr1 * q->texr2 * (float)T[q->tex11];
}
static inline float bilerp_bool(const taps *q, const uint8_t *T) {
  return q->texi1 * q->texi2 * (float)(T[q->tex] != 0) + q->texr1 * q->texi2 * (float)(T[q->tex10] != 0) +
         q->texi1 * q->texr2 * (float)(T[q->tex01] != 0) + q->texr1 * q->texr2 * (float)(T[q->tex11] != 0);
}

/* double-cascade 5-tap count: av_alpha_max.c:53-84 (shDist 2) */
static float shadow_light(const shade_ctx *c, f3 p) {
  int shadow = 0;
  for (int k = 0; k < c->nsh && k < 2; k++) {
    const orc_shadow *s = &c->sh[k];
    int wS = s->dim / 2;
    f3 sp = {s->pos[0], s->pos[1], s->pos[2]};
    f3 pos = f3sub(p, sp);
    float depth = dot3(pos, f3ld(s->vv));
    int sx = f2i(dot3(pos, f3ld(s->vv + 3)) * s->scale) + wS;
    int sy = f2i(dot3(pos, f3ld(s->vv + 6)) * -s->scale) + wS;
    if (sx >= 2 && sx < 2 * wS - 2 && sy >= 2 && sy < 2 * wS - 2) {
      const float *SD = s->map;
      if (SD[2 * wS * sy + sx] < depth) shadow += 1;
      if (SD[2 * wS * (sy + 2) + sx] < depth) shadow += 1;
      if (SD[2 * wS * (sy - 2) + sx] < depth) shadow += 1;
      if (SD[2 * wS * sy + (sx + 2)] < depth) shadow += 1;
      if (SD[2 * wS * sy + (sx - 2)] < depth) shadow += 1;
    }
  }
  shadow = imin(5, shadow);
  float light = (float)shadow * c->f->amb + (float)(5 - shadow);
  light *= 0.2f;
  return light;
}

/* av_draw_multi.c:30-105: the 4-way terrain blend.  This group's texture and
 * the next three groups' (Ops0.py:533-545 binds TR[tn+1..tn+3]) are sampled
 * at the same bilinear taps (side lenT of this group); blend weights m, n, o
 * come from the world height and the normal; no shadow lookup (light = 1).
 * The blended texel is converted to u16 before the lighting product, and
 * the product's implicit conversion to u16 is pinned as convert_ushort's. */
static void multi_core(const shade_ctx *c, size_t pix, float t, float tz, f2 uvi, const attrs *a1,
                       const attrs *a2) {
  const orc_frame *f = c->f;
  const orc_group *g = c->g;
  float omt = 1 - t;
  taps q = make_taps(uvi, tz, g->tex_size, 0);
  float tr[4], tg[4], tb[4];
  for (int k = 0; k < 4; k++) {
    tr[k] = bilerp_u16(&q, g[k].tr);
    tg[k] = bilerp_u16(&q, g[k].tg);
    tb[k] = bilerp_u16(&q, g[k].tb);
  }
  f3 col = f3mul(f3add(f3smul(omt, a2->li), f3smul(t, a1->li)), tz);
  f3 norm = fast_normalize(f3mul(f3add(f3smul(omt, a2->n), f3smul(t, a1->n)), tz));
  f3 lint = {f->lint[0], f->lint[1], f->lint[2]};
  f3 ldir = {f->ldir[0], f->ldir[1], f->ldir[2]};
  f3 dirCol = f3smul(fmaxf(0.f, dot3(norm, ldir)), lint);
  f3 cpos = f3mul(f3add(f3smul(omt, a2->p), f3smul(t, a1->p)), tz);
  float m = (cpos.y - 15.f) / 4.f;
  m = fclampf(m, 0.f, 1.f);
  float ny = fmaxf(0.f, fabsf(norm.y) - 0.33f) * 1.5f;
  m -= 1.5f * (ny * ny - 0.4f);
  m = fclampf(m, 0.f, 1.f);
  f3 qv = f3div(cpos, 3.f);
  float threshy = 16.f + 2.f * fabsf(qv.x - roundf(qv.x)) + 2.f * fabsf(qv.z - roundf(qv.z));
  float n = fclampf((cpos.y - threshy) / 2.f, 0.f, 4.f);
  n = n * n * n;
  n += 1.5f * (ny * ny - 0.4f);
  n = fclampf(n, 0.f, 32.f);
  float o = fclampf((5.f - cpos.y) / 4.f, 0.f, 1.f);
  if (m + n + o > 1.f) {   /* each weight divides by the sum of the updated ones */
    n = n / (n + m + o);
    m = m / (n + m + o);
    o = o / (n + m + o);
  }
  float w1 = 1 - m - n - o;
  float light = 1;
  f->ro[pix] = u16sat((float)u16sat(m * tr[1] + n * tr[2] + o * tr[3] + w1 * tr[0]) * (light * dirCol.x + col.x));
  f->go[pix] = u16sat((float)u16sat(m * tg[1] + n * tg[2] + o * tg[3] + w1 * tg[0]) * (light * dirCol.y + col.y));
  f->bo[pix] = u16sat((float)u16sat(m * tb[1] + n * tb[2] + o * tb[3] + w1 * tb[0]) * (light * dirCol.z + col.z));
}

/* ---- normal-mapped materials (av_draw_normmap.c, _alpha.c, _mip.c) ---- */

/* pown(x, n) for n >= 0 by repeated squaring (the convention pinned where
 * OpenCL leaves pown's rounding to the device) */
static inline float pown_rs(float x, int n) {
  unsigned k = n < 0 ? 0u - (unsigned)n : (unsigned)n;
  float r = 1.0f, b = x;
  while (k) {
    if (k & 1u) r *= b;
    b *= b;
    k >>= 1;
  }
  return n < 0 ? 1.0f / r : r;
}

/* sampleShadow, which the reference calls but defines nowhere, as this
 * library defines it: the five taps of one cascade (centre, +-2 texels in x
 * and y) at the truncated map position, counted where the map is nearer
 * than `depth`, only when the centre lies in [2, 2 wS - 2) on both axes;
 * the shadowed fraction is count * 0.2 */
static float sample_shadow5(const orc_shadow *s, float depth, float sfx, float sfy) {
  int wS = s->dim / 2;
  int sx = f2i(sfx), sy = f2i(sfy), n = 0;
  if (sx >= 2 && sx < 2 * wS - 2 && sy >= 2 && sy < 2 * wS - 2) {
    const float *SD = s->map;
    int r = 2 * wS;
    if (SD[r * sy + sx] < depth) n += 1;
    if (SD[r * (sy + 2) + sx] < depth) n += 1;
    if (SD[r * (sy - 2) + sx] < depth) n += 1;
    if (SD[r * sy + (sx + 2)] < depth) n += 1;
    if (SD[r * sy + (sx - 2)] < depth) n += 1;
  }
  return (float)n * 0.2f;
}

/* bilinear normal-map texel (R, G, B bytes) at the taps, as the sources'
 * texi1*texi2*convert_float3(NM[tex]) + ... */
static inline f3 bilerp_nm(const taps *q, const uint8_t *NM) {
  const uint8_t *a = NM + 4 * (size_t)q->tex, *b = NM + 4 * (size_t)q->tex10;
  const uint8_t *cc = NM + 4 * (size_t)q->tex01, *d = NM + 4 * (size_t)q->tex11;
  float w00 = q->texi1 * q->texi2, w10 = q->texr1 * q->texi2, w01 = q->texi1 * q->texr2, w11 = q->texr1 * q->texr2;
  f3 r;
  r.x = w00 * (float)a[0] + w10 * (float)b[0] + w01 * (float)cc[0] + w11 * (float)d[0];
  r.y = w00 * (float)a[1] + w10 * (float)b[1] + w01 * (float)cc[1] + w11 * (float)d[1];
  r.z = w00 * (float)a[2] + w10 * (float)b[2] + w01 * (float)cc[2] + w11 * (float)d[2];
  return r;
}

/* av_draw_normmap.c:47-149 (_alpha.c shares it after its alpha test) and
 * av_draw_normmap_mip.c:73-160 for a fragment that passed the depth test */
static void normal_core(const shade_ctx *c, size_t pix, float t, float tz, f2 uvi, const attrs *a1,
                        const attrs *a2) {
  const orc_frame *f = c->f;
  const orc_group *g = c->g;
  const int mip = (g->flags & ORC_MIP) != 0;
  float omt = 1 - t;
  float outR, outG, outB;
  f3 tg;
  taps q = make_taps(uvi, tz, mip ? c->len_mip : g->tex_size, mip ? c->start_mip : 0);
  outR = bilerp_u16(&q, g->tr);
  outG = bilerp_u16(&q, g->tg);
  outB = bilerp_u16(&q, g->tb);
  tg = bilerp_nm(&q, g->nm);
  if (mip) {
    taps q2 = make_taps(uvi, tz, c->len_mip2, c->start_mip2);
    float fm = c->fmip, ofm = 1 - c->fmip;
    outR = ofm * outR + fm * bilerp_u16(&q2, g->tr);
    outG = ofm * outG + fm * bilerp_u16(&q2, g->tg);
    outB = ofm * outB + fm * bilerp_u16(&q2, g->tb);
    tg = f3add(f3smul(ofm, tg), f3smul(fm, bilerp_nm(&q2, g->nm)));
  }
  float light = 1;
  if (c->nsh > 0) {
    const orc_shadow *sh = &c->sh[0];
    f3 sp = {sh->pos[0], sh->pos[1], sh->pos[2]};
    f3 pos = f3sub(f3mul(f3add(f3smul(omt, a2->p), f3smul(t, a1->p)), tz), sp);
    float depth = dot3(pos, f3ld(sh->vv));
    float wS = (float)(sh->dim / 2);
    float sfx = (dot3(pos, f3ld(sh->vv + 3)) * sh->scale) + wS;
    float sfy = (dot3(pos, f3ld(sh->vv + 6)) * -sh->scale) + wS;
    light = 1 - sample_shadow5(sh, depth, sfx, sfy);
  } else {
    light = 1 - 0.f;
  }
  f3 col = f3mul(f3add(f3smul(omt, a2->li), f3smul(t, a1->li)), tz);
  f3 norm = fast_normalize(f3mul(f3add(f3smul(omt, a2->n), f3smul(t, a1->n)), tz));
  tg = f3sub(f3mul(f3div(tg, 255.f), 2.f), (f3){1.f, 1.f, 1.f});
  tg = fast_normalize(tg);
  norm = fast_normalize(f3add(f3add(f3smul(tg.z, norm), f3smul(-tg.y, c->tangent)), f3smul(-tg.x, c->bitangent)));
  f3 vp = {f->pos[0], f->pos[1], f->pos[2]};
  f3 lint = {f->lint[0], f->lint[1], f->lint[2]};
  f3 ldir = {f->ldir[0], f->ldir[1], f->ldir[2]};
  f3 pos = f3mul(f3add(f3smul(omt, a2->p), f3smul(t, a1->p)), tz);
  f3 spec;
  if (mip) {
    f3 a = f3sub(pos, vp);
    f3 h = fast_normalize(f3add(fast_normalize(a), ldir));
    float theta = fmaxf(0.f, dot3(h, norm));
    float mf = (float)c->mip + c->fmip;
    int sp = f2i(1.f * (mf * mf));
    spec = f3smul(((pown_rs(theta, sp) * 256.f) * light) * 2.f, lint);
    spec = f3mul(spec, (float)(sp + 1) / (2.f * 3.1416f));
  } else {
    f3 a = fast_normalize(f3sub(pos, vp));
    f3 h = fast_normalize(f3add(a, ldir));
    float theta = fmaxf(0.f, dot3(h, norm));
    int sp = c->spec_pow;
    spec = f3smul(((pown_rs(theta, sp) * 256.f) * 4.f) * light, lint);
    spec = f3mul(spec, (float)(sp + 2) / (8.f * 3.1416f));
    a = f3sub(pos, vp);
    float nd = dot3(a, norm);
    f3 refl = fast_normalize(f3sub(a, f3smul(2.f * nd, norm)));
    f3 up = {0.f, 1.f, 0.f};
    theta = fmaxf(0.f, dot3(refl, up));
    f3 sky = {0.1f, 0.3f, 0.5f};
    spec = f3add(spec, f3smul((pown_rs(theta, 2) * 128.f) * (float)(1 + g->is_metal), sky));
    theta = fmaxf(0.f, dot3(fast_normalize(a), refl));
    f3 grey = {0.2f, 0.2f, 0.2f};
    spec = f3add(spec, f3smul(pown_rs(theta, c->spec_pow2) * 256.f, grey));
    if (g->is_metal) {
      spec.x *= (float)g->tr[q.tex] / 1024.f;
      spec.y *= (float)g->tg[q.tex] / 1024.f;
      spec.z *= (float)g->tb[q.tex] / 1024.f;
      light = 0.f;
      col.x = col.y = col.z = 0.f;
    }
  }
  f3 dirCol = f3smul(fmaxf(0.f, dot3(norm, ldir)), lint);
  f->ro[pix] = u16sat(spec.x + outR * (light * dirCol.x + col.x));
  f->go[pix] = u16sat(spec.y + outG * (light * dirCol.y + col.y));
  f->bo[pix] = u16sat(spec.z + outB * (light * dirCol.z + col.z));
}

/* One fragment at (cy, ax) with edge interpolants a1 (edge 1) and a2
 * (edge 2).  `zcur` points at the depth sample the test reads (the global
 * depth buffer in the serial model).  Returns 1 if it wrote. */
static int fragment(const shade_ctx *c, int tri, int cy, int ax, float t, float tz,
                    const attrs *a1, const attrs *a2) {
  const orc_frame *f = c->f;
  const orc_group *g = c->g;
  int flags = g->flags;
  size_t pix = (size_t)f->w * cy + ax;
  float omt = 1 - t;
  f2 uvi = f2add(f2smul(omt, a2->uv), f2smul(t, a1->uv));
  taps q;
  int have_q = 0;
  int base_len = (flags & ORC_MIP) ? (1 << c->num_mip) : g->tex_size;
  if (flags & ORC_ALPHA) {
    /* av_draw_alpha.c:80-97: bilinear bool alpha at base-level taps */
    q = make_taps(uvi, tz, base_len, 0);
    have_q = 1;
    float ca = bilerp_bool(&q, c->alpha->mask);
    if (!(ca > 0.5f)) return 0;
  }
  /* Templates.py:74-91 + AVSL.py:238-239: `depth >= tz` (later wins ties) */
  if (!(f->db[pix] >= tz)) return 0;
  f->db[pix] = tz;
  if ((flags & ORC_MULTI) && !(flags & ORC_ALPHA)) {
    multi_core(c, pix, t, tz, uvi, a1, a2);
    f->tri_id[pix] = c->gid_base + tri;
    f->cov[pix] = 1;
    return 1;
  }
  if (flags & ORC_NORMAL) {
    normal_core(c, pix, t, tz, uvi, a1, a2);
    f->tri_id[pix] = c->gid_base + tri;
    f->cov[pix] = 1;
    return 1;
  }
  float outR, outG, outB;
  if (flags & ORC_MIP) {
    /* av_draw_normmap_mip.c:73-123 */
    taps q1 = make_taps(uvi, tz, c->len_mip, c->start_mip);
    outR = bilerp_u16(&q1, g->tr);
    outG = bilerp_u16(&q1, g->tg);
    outB = bilerp_u16(&q1, g->tb);
    taps q2 = make_taps(uvi, tz, c->len_mip2, c->start_mip2);
    float fm = c->fmip, ofm = 1 - c->fmip;
    outR = ofm * outR + fm * bilerp_u16(&q2, g->tr);
    outG = ofm * outG + fm * bilerp_u16(&q2, g->tg);
    outB = ofm * outB + fm * bilerp_u16(&q2, g->tb);
  } else {
    if (!have_q) q = make_taps(uvi, tz, g->tex_size, 0);
    outR = bilerp_u16(&q, g->tr);
    outG = bilerp_u16(&q, g->tg);
    outB = bilerp_u16(&q, g->tb);
  }
  float light = 1;
  if (flags & ORC_SHADOW) {
    f3 p = f3mul(f3add(f3smul(omt, a2->p), f3smul(t, a1->p)), tz);
    light = shadow_light(c, p);
  }
  /* av_draw_base.c:44-55 */
  f3 col = f3mul(f3add(f3smul(omt, a2->li), f3smul(t, a1->li)), tz);
  f3 norm = fast_normalize(f3mul(f3add(f3smul(omt, a2->n), f3smul(t, a1->n)), tz));
  f3 lint = {f->lint[0], f->lint[1], f->lint[2]};
  f3 ldir = {f->ldir[0], f->ldir[1], f->ldir[2]};
  f3 dirCol = f3smul(fmaxf(0.f, dot3(norm, ldir)), lint);
  float oml = 1 - light;
  f->ro[pix] = u16sat(outR * (light * (dirCol.x + col.x) + oml * col.x));
  f->go[pix] = u16sat(outG * (light * (dirCol.y + col.y) + oml * col.y));
  f->bo[pix] = u16sat(outB * (light * (dirCol.z + col.z) + oml * col.z));
  f->tri_id[pix] = c->gid_base + tri;
  f->cov[pix] = 1;
  return 1;
}

/* ------------------------------------------------------------------ */
/* per-triangle raster state (Templates.py:38-72, 210-247)             */
/* ------------------------------------------------------------------ */

typedef struct {
  float x[4], y[4], z[4];   /* sorted vertices 1..3 (index 0..2) and vertex 4 (3) */
  attrs v[4];               /* attribute * z, sorted, and vertex 4 */
} tri_setup;

static inline attrs attrs_load(const orc_group *g, int i, int k, float z) {
  attrs a;
  size_t vi = (size_t)i * 3 + k;
  a.uv = f2mul(f2ld(g->uv + vi * 2), z);
  a.li = f3mul(f3ld(g->li + vi * 3), z);
  a.n = f3mul(f3ld(g->vn + vi * 3), z);
  a.p = f3mul(f3ld(g->xyz + vi * 3), z);
  return a;
}

static inline attrs attrs_sub(attrs a, attrs b) {
  attrs r; r.uv = f2sub(a.uv, b.uv); r.li = f3sub(a.li, b.li); r.n = f3sub(a.n, b.n); r.p = f3sub(a.p, b.p); return r;
}
static inline attrs attrs_add(attrs a, attrs b) {
  attrs r; r.uv = f2add(a.uv, b.uv); r.li = f3add(a.li, b.li); r.n = f3add(a.n, b.n); r.p = f3add(a.p, b.p); return r;
}
static inline attrs attrs_mul(attrs a, float s) {
  attrs r; r.uv = f2mul(a.uv, s); r.li = f3mul(a.li, s); r.n = f3mul(a.n, s); r.p = f3mul(a.p, s); return r;
}
static inline attrs attrs_smul(float s, attrs a) {
  attrs r; r.uv = f2smul(s, a.uv); r.li = f3smul(s, a.li); r.n = f3smul(s, a.n); r.p = f3smul(s, a.p); return r;
}
static inline attrs attrs_neg(attrs a) {
  attrs r; r.uv = f2neg(a.uv); r.li = f3neg(a.li); r.n = f3neg(a.n); r.p = f3neg(a.p); return r;
}

/* the AVSL sort: three conditional swaps on y (AVSL.py:109-129) */
#define SWAPV(a, b) do { float _t = (a); (a) = (b); (b) = _t; } while (0)
#define SWAPA(a, b) do { attrs _t = (a); (a) = (b); (b) = _t; } while (0)

static void sort3(float *x, float *y, float *z, attrs *v) {
  if (y[0] > y[1]) { SWAPV(y[0], y[1]); SWAPV(x[0], x[1]); SWAPV(z[0], z[1]); SWAPA(v[0], v[1]); }
  if (y[1] > y[2]) { SWAPV(y[1], y[2]); SWAPV(x[1], x[2]); SWAPV(z[1], z[2]); SWAPA(v[1], v[2]); }
  if (y[0] > y[1]) { SWAPV(y[0], y[1]); SWAPV(x[0], x[1]); SWAPV(z[0], z[1]); SWAPA(v[0], v[1]); }
}

/* mip selection of av_draw_normmap_mip.c:26-59, evaluated after the sort
 * and after vertex 4.  `x`,`y` hold the sorted screen coordinates (ints
 * converted to float on the direct path); edge lengths are computed in int
 * on the direct path and in float on the tiled path. */
static void mip_setup(shade_ctx *c, tri_setup *s, int small, const int *ix, const int *iy) {
  float z1 = s->z[0], z2 = s->z[1], z3 = s->z[2];
  f2 uv1 = f2div(s->v[0].uv, z1), uv2 = f2div(s->v[1].uv, z2), uv3 = f2div(s->v[2].uv, z3);
  f3 p1 = f3div(s->v[0].p, z1), p2 = f3div(s->v[1].p, z2), p3 = f3div(s->v[2].p, z3);
  f2 dUV1 = f2sub(uv2, uv1), dUV2 = f2sub(uv3, uv1), dUV3 = f2sub(uv3, uv2);
  float l1, l2, l3;
  if (small) {
    l1 = (float)((iy[1] - iy[0]) * (iy[1] - iy[0]) + (ix[1] - ix[0]) * (ix[1] - ix[0]));
    l2 = (float)((iy[2] - iy[0]) * (iy[2] - iy[0]) + (ix[2] - ix[0]) * (ix[2] - ix[0]));
    l3 = (float)((iy[2] - iy[1]) * (iy[2] - iy[1]) + (ix[2] - ix[1]) * (ix[2] - ix[1]));
  } else {
    float *x = s->x, *y = s->y;
    l1 = (y[1] - y[0]) * (y[1] - y[0]) + (x[1] - x[0]) * (x[1] - x[0]);
    l2 = (y[2] - y[0]) * (y[2] - y[0]) + (x[2] - x[0]) * (x[2] - x[0]);
    l3 = (y[2] - y[1]) * (y[2] - y[1]) + (x[2] - x[1]) * (x[2] - x[1]);
  }
  f2 su1 = f2div(dUV1, l1), su2 = f2div(dUV2, l2), su3 = f2div(dUV3, l3);
  su1.x = fabsf(su1.x); su1.y = fabsf(su1.y);
  su2.x = fabsf(su2.x); su2.y = fabsf(su2.y);
  su3.x = fabsf(su3.x); su3.y = fabsf(su3.y);
  float dt = fmaxf(su1.x, fmaxf(su1.y, fmaxf(su2.x, su2.y)));
  dt = fmaxf(dt, fmaxf(su3.x, su3.y));
  float fmip = fmaxf(0.f, fminf((float)(c->num_mip - 1), fabsf(orc_log2f(dt)) / 2 + c->g->mip_bias));
  int mip = f2i(fmip);
  fmip -= (float)mip;
  c->fmip = fmip;
  c->mip = mip;
  c->len_mip = 1 << mip;
  c->len_mip2 = c->len_mip << 1;
  int start = 0;
  for (int i = 0; i < mip; i++) start += (1 << i) * (1 << i);
  c->start_mip = start;
  c->start_mip2 = start + c->len_mip * c->len_mip;
  s->v[0].uv = f2mul(uv1, z1); s->v[1].uv = f2mul(uv2, z2); s->v[2].uv = f2mul(uv3, z3);
  s->v[0].p = f3mul(p1, z1); s->v[1].p = f3mul(p2, z2); s->v[2].p = f3mul(p3, z3);
}

/* shader_setup of the normal-mapped sources (av_draw_normmap.c:24-38): the
 * tangent frame from the sorted vertices' uv and position divided by z,
 * before they are multiplied back.  Called before the mip setup, which
 * divides the same values; without ORC_MIP this setup makes the round trip
 * itself. */
static void normal_setup(shade_ctx *c, tri_setup *s) {
  float z1 = s->z[0], z2 = s->z[1], z3 = s->z[2];
  f2 uv1 = f2div(s->v[0].uv, z1), uv2 = f2div(s->v[1].uv, z2), uv3 = f2div(s->v[2].uv, z3);
  f3 p1 = f3div(s->v[0].p, z1), p2 = f3div(s->v[1].p, z2), p3 = f3div(s->v[2].p, z3);
  f2 dUV1 = f2sub(uv2, uv1), dUV2 = f2sub(uv3, uv1);
  f3 dPos1 = f3sub(p2, p1), dPos2 = f3sub(p3, p1);
  float rdet = 1.f / (dUV1.x * dUV2.y - dUV1.y * dUV2.x);
  c->tangent = fast_normalize(f3mul(f3sub(f3mul(dPos1, dUV2.y), f3mul(dPos2, dUV1.y)), rdet));
  c->bitangent = fast_normalize(f3mul(f3sub(f3mul(dPos2, dUV1.x), f3mul(dPos1, dUV2.x)), rdet));
  if (!(c->g->flags & ORC_MIP)) {
    s->v[0].uv = f2mul(uv1, z1); s->v[1].uv = f2mul(uv2, z2); s->v[2].uv = f2mul(uv3, z3);
    s->v[0].p = f3mul(p1, z1); s->v[1].p = f3mul(p2, z2); s->v[2].p = f3mul(p3, z3);
  }
}

/* ------------------------------------------------------------------ */
/* direct raster of small triangles: Templates.py:210-323              */
/* rows restricted to [row0, row1) (strip-parallel baseline)           */
/* ------------------------------------------------------------------ */

static void draw_small_tri(shade_ctx *c, int tri, const float sp[6], const float sz[3],
                           int row0, int row1) {
  const orc_frame *f = c->f;
  const orc_group *g = c->g;
  tri_setup s;
  int ix[3], iy[3];
  for (int k = 0; k < 3; k++) {
    s.z[k] = sz[k];
    s.v[k] = attrs_load(g, tri, k, sz[k]);
    ix[k] = f2i(sp[k * 2]);
    iy[k] = f2i(sp[k * 2 + 1]);
  }
  /* integer sort (Templates.py:230-239) */
  float fz[3] = {s.z[0], s.z[1], s.z[2]};
#define SWAPI(a, b) do { int _t = (a); (a) = (b); (b) = _t; } while (0)
  if (iy[0] > iy[1]) { SWAPI(iy[0], iy[1]); SWAPI(ix[0], ix[1]); SWAPV(fz[0], fz[1]); SWAPA(s.v[0], s.v[1]); }
  if (iy[1] > iy[2]) { SWAPI(iy[1], iy[2]); SWAPI(ix[1], ix[2]); SWAPV(fz[1], fz[2]); SWAPA(s.v[1], s.v[2]); }
  if (iy[0] > iy[1]) { SWAPI(iy[0], iy[1]); SWAPI(ix[0], ix[1]); SWAPV(fz[0], fz[1]); SWAPA(s.v[0], s.v[1]); }
  int x1 = ix[0], x2 = ix[1], x3 = ix[2], y1 = iy[0], y2 = iy[1], y3 = iy[2];
  float z1 = fz[0], z2 = fz[1], z3 = fz[2];
  s.z[0] = z1; s.z[1] = z2; s.z[2] = z3;
  if (y1 >= row1 || y3 < row0) {
    /* rows y1..y3 miss the strip: nothing to draw (rows only grow/shrink
     * monotonically inside each half) */
    return;
  }
  float ydiff1 = (float)(y2 - y1) / (float)(y3 - y1);
  float x4 = (float)x1 + ydiff1 * (float)(x3 - x1);
  float z4 = z1 + ydiff1 * (z3 - z1);
  attrs v4 = attrs_add(s.v[0], attrs_smul(ydiff1, attrs_sub(s.v[2], s.v[0])));
  s.v[3] = v4;
  if (g->flags & ORC_NORMAL) normal_setup(c, &s);
  if (g->flags & ORC_MIP) {
    s.x[0] = (float)x1; s.x[1] = (float)x2; s.x[2] = (float)x3;
    s.y[0] = (float)y1; s.y[1] = (float)y2; s.y[2] = (float)y3;
    int sx[3] = {x1, x2, x3}, sy[3] = {y1, y2, y3};
    mip_setup(c, &s, 1, sx, sy);
  }
  attrs a1v = s.v[0], a2v = s.v[1], a3v = s.v[2];

  /* bottom half (Templates.py:251-285) */
  ydiff1 = 1 / (float)(y2 - y1);
  float slope1 = (float)(x2 - x1) * ydiff1;
  float slope2 = (x4 - (float)x1) * ydiff1;
  float slopez1 = (z2 - z1) * ydiff1;
  float slopez2 = (z4 - z1) * ydiff1;
  attrs sa1 = attrs_mul(attrs_sub(a2v, a1v), ydiff1);
  attrs sa2 = attrs_mul(attrs_sub(v4, a1v), ydiff1);
  float cx1 = (float)x1, cx2 = (float)x1, cz1 = z1, cz2 = z1;
  attrs c1 = a1v, c2 = a1v;
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPA(sa1, sa2);
  }
  for (int cy = y1; cy <= y2; cy++) {
    if (cy >= row0 && cy < row1) {
      for (int ax = f2i(cx2); (float)ax <= cx1; ax++) {
        if (cy >= 0 && cy < f->h && ax >= 0 && ax < f->w) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          fragment(c, tri, cy, ax, t, tz, &c1, &c2);
        }
      }
    }
    cx1 += slope1; cx2 += slope2; cz1 += slopez1; cz2 += slopez2;
    c1 = attrs_add(c1, sa1); c2 = attrs_add(c2, sa2);
  }

  /* top half (Templates.py:287-320) */
  ydiff1 = 1 / (float)(y3 - y2);
  slope1 = (float)(x3 - x2) * ydiff1;
  slope2 = ((float)x3 - x4) * ydiff1;
  slopez1 = (z3 - z2) * ydiff1;
  slopez2 = (z3 - z4) * ydiff1;
  sa1 = attrs_mul(attrs_neg(attrs_sub(a2v, a3v)), ydiff1);
  sa2 = attrs_mul(attrs_neg(attrs_sub(v4, a3v)), ydiff1);
  cx1 = (float)x3; cx2 = (float)x3; cz1 = z3; cz2 = z3;
  c1 = a3v; c2 = a3v;
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPA(sa1, sa2);
  }
  for (int cy = y3; cy >= y2; cy--) {
    if (cy >= row0 && cy < row1) {
      for (int ax = f2i(cx1); (float)ax <= cx2; ax++) {
        if (cy >= 0 && cy < f->h && ax >= 0 && ax < f->w) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          fragment(c, tri, cy, ax, t, tz, &c1, &c2);
        }
      }
    }
    cx1 -= slope1; cx2 -= slope2; cz1 -= slopez1; cz2 -= slopez2;
    c1 = attrs_sub(c1, sa1); c2 = attrs_sub(c2, sa2);
  }
}

/* ------------------------------------------------------------------ */
/* tiled raster of a large triangle inside one tile: Templates.py:4-185 */
/* ------------------------------------------------------------------ */

static void draw_tiled_tri(shade_ctx *c, int tri, int bx, const float sp[6], const float sz[3]) {
  const orc_frame *f = c->f;
  const orc_group *g = c->g;
  int wc = f->w / TILE;
  int tileX = bx % wc;
  int tileY = f2i((float)bx / ((float)f->w / 16.f));
  float xMin = (float)tileX * 16.f;
  float xMax = ((float)tileX + 1.f) * 16.f - 1.f;
  float yMin = (float)tileY * 16.f;
  float yMax = ((float)tileY + 1.f) * 16.f - 1.f;

  tri_setup s;
  for (int k = 0; k < 3; k++) {
    s.x[k] = sp[k * 2];
    s.y[k] = sp[k * 2 + 1];
    s.z[k] = sz[k];
    s.v[k] = attrs_load(g, tri, k, sz[k]);
  }
  sort3(s.x, s.y, s.z, s.v);
  float x1 = s.x[0], x2 = s.x[1], x3 = s.x[2];
  float y1 = s.y[0], y2 = s.y[1], y3 = s.y[2];
  float z1 = s.z[0], z2 = s.z[1], z3 = s.z[2];
  float ydiff1 = (y2 - y1) / (y3 - y1);
  float x4 = x1 + ydiff1 * (x3 - x1);
  float z4 = z1 + ydiff1 * (z3 - z1);
  attrs v4 = attrs_add(s.v[0], attrs_smul(ydiff1, attrs_sub(s.v[2], s.v[0])));
  s.v[3] = v4;
  if (g->flags & ORC_NORMAL) normal_setup(c, &s);
  if (g->flags & ORC_MIP) mip_setup(c, &s, 0, NULL, NULL);
  attrs a1v = s.v[0], a2v = s.v[1], a3v = s.v[2];

  /* bottom half (Templates.py:93-138) */
  ydiff1 = 1 / (y2 - y1);
  float slope1 = (x2 - x1) * ydiff1;
  float slope2 = (x4 - x1) * ydiff1;
  float slopez1 = (z2 - z1) * ydiff1;
  float slopez2 = (z4 - z1) * ydiff1;
  attrs sa1 = attrs_mul(attrs_sub(a2v, a1v), ydiff1);
  attrs sa2 = attrs_mul(attrs_sub(v4, a1v), ydiff1);
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPA(sa1, sa2);
  }
  int cy = f2i(fclampf(y1, yMin, yMax));
  float dy = (float)cy - y1;
  float cx1 = x1 + dy * slope1;
  float cx2 = x1 + dy * slope2;
  float cz1 = z1 + dy * slopez1;
  float cz2 = z1 + dy * slopez2;
  attrs c1 = attrs_add(a1v, attrs_smul(dy, sa1));
  attrs c2 = attrs_add(a1v, attrs_smul(dy, sa2));
  if (y2 > yMin) {
    for (; (float)cy <= fclampf(y2, yMin, yMax); cy++) {
      if (cx2 < xMax && cx1 > xMin) {
        for (int ax = f2i(fclampf(cx2, xMin, xMax)); (float)ax <= fclampf(cx1, xMin, xMax); ax++) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          fragment(c, tri, cy, ax, t, tz, &c1, &c2);
        }
      }
      cx1 += slope1; cx2 += slope2; cz1 += slopez1; cz2 += slopez2;
      c1 = attrs_add(c1, sa1); c2 = attrs_add(c2, sa2);
    }
  }

  /* top half (Templates.py:140-182) */
  ydiff1 = 1 / (y3 - y2);
  slope1 = (x3 - x2) * ydiff1;
  slope2 = (x3 - x4) * ydiff1;
  slopez1 = (z3 - z2) * ydiff1;
  slopez2 = (z3 - z4) * ydiff1;
  sa1 = attrs_mul(attrs_neg(attrs_sub(a2v, a3v)), ydiff1);
  sa2 = attrs_mul(attrs_neg(attrs_sub(v4, a3v)), ydiff1);
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPA(sa1, sa2);
  }
  cy = f2i(fclampf(y3, yMin, yMax));
  dy = (float)cy - y3;
  cx1 = x3 + dy * slope1;
  cx2 = x3 + dy * slope2;
  cz1 = z3 + dy * slopez1;
  cz2 = z3 + dy * slopez2;
  c1 = attrs_add(a3v, attrs_smul(dy, sa1));
  c2 = attrs_add(a3v, attrs_smul(dy, sa2));
  if (y2 < yMax) {
    for (; (float)cy >= fclampf(y2, yMin, yMax); cy--) {
      if (cx1 < xMax && cx2 > xMin) {
        for (int ax = f2i(fclampf(cx1, xMin, xMax)); (float)ax <= fclampf(cx2, xMin, xMax); ax++) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          fragment(c, tri, cy, ax, t, tz, &c1, &c2);
        }
      }
      cx1 -= slope1; cx2 -= slope2; cz1 -= slopez1; cz2 -= slopez2;
      c1 = attrs_sub(c1, sa1); c2 = attrs_sub(c2, sa2);
    }
  }
}

/* ------------------------------------------------------------------ */
/* coarse binning: PyOpenCL27C/Pipe/coarse.c:17-125                   */
/* ------------------------------------------------------------------ */

typedef struct { int32_t *v; int n, cap; } ivec;

static void ivec_push(ivec *a, int32_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 16;
    a->v = (int32_t *)realloc(a->v, sizeof(int32_t) * (size_t)a->cap);
  }
  a->v[a->n++] = x;
}

/* calls emit(tile, arg) for every bin entry coarse.c makes for one triangle */
typedef void (*emit_fn)(int tile, int tri, void *arg);

static void coarse_tri(const float sp[6], int wc, int hc, int tri, emit_fn emit, void *arg) {
  float x[3], y[3];
  for (int k = 0; k < 3; k++) {
    x[k] = sp[k * 2] / 16.f - 0.5f;
    y[k] = sp[k * 2 + 1] / 16.f - 0.5f;
  }
  float x1 = x[0], x2 = x[1], x3 = x[2], y1 = y[0], y2 = y[1], y3 = y[2];
  if (y1 > y2) { SWAPV(y1, y2); SWAPV(x1, x2); }
  if (y2 > y3) { SWAPV(y2, y3); SWAPV(x2, x3); }
  if (y1 > y2) { SWAPV(y1, y2); SWAPV(x1, x2); }
  float x4 = (x1 + ((y2 - y1) / (y3 - y1)) * (x3 - x1));
  float y4 = y2;
  float slope1 = (x2 - x1) / (y2 - y1);
  float slope2 = (x4 - x1) / (y4 - y1);
  float cx1 = x1, cx2 = x1;
  if (slope1 < slope2) SWAPV(slope1, slope2);
  float sbias = 1.f + floorf(y1) - y1;
  float wcm1 = (float)wc - 1;
  if (y1 != y2) {
    for (int cy = f2i(floorf(y1)); (float)cy <= ceilf(y2); cy++) {
      float mx1 = cx1 + sbias * slope1;
      if (slope1 < 0) mx1 -= slope1;
      float mx2 = cx2 + sbias * slope2;
      if (slope2 > 0) mx2 -= slope2;
      mx1 = fminf(mx1, wcm1);
      mx2 = fmaxf(mx2, 0.f);
      if (cy >= 0 && cy < hc) {
        for (int ax = f2i(floorf(mx2)); (float)ax <= ceilf(mx1); ax++) emit(wc * cy + ax, tri, arg);
      }
      cx1 += slope1;
      cx2 += slope2;
    }
  }
  slope1 = (x3 - x2) / (y3 - y2);
  slope2 = (x3 - x4) / (y3 - y4);
  cx1 = x3; cx2 = x3;
  if (slope1 < slope2) SWAPV(slope1, slope2);
  sbias = y3 - floorf(y3);
  if (y2 != y3) {
    for (int cy = f2i(ceilf(y3)); (float)cy >= floorf(y2); cy--) {
      float mx1 = cx1 - sbias * slope1;
      if (slope1 < 0) mx1 += slope1;
      float mx2 = cx2 - sbias * slope2;
      if (slope2 > 0) mx2 += slope2;
      mx2 = fminf(mx2, wcm1);
      mx1 = fmaxf(mx1, 0.f);
      if (cy >= 0 && cy < hc) {
        for (int ax = f2i(floorf(mx1)); (float)ax <= ceilf(mx2); ax++) emit(wc * cy + ax, tri, arg);
      }
      cx1 -= slope1;
      cx2 -= slope2;
    }
  }
}

static void emit_bin(int tile, int tri, void *arg) { ivec_push(&((ivec *)arg)[tile], tri); }
static void emit_count(int tile, int tri, void *arg) { (void)tri; ((int32_t *)arg)[tile] += 1; }

/* ------------------------------------------------------------------ */
/* drawAll orchestration: Ops0.py:471-648                               */
/* ------------------------------------------------------------------ */

typedef struct {
  uint8_t *cls;
  float *sp, *zz;
} setup_out;

static void setup_group(const orc_group *g, const orc_frame *f, setup_out *o, int nthreads) {
  o->cls = (uint8_t *)malloc((size_t)g->ntris + 1);
  o->sp = (float *)malloc(sizeof(float) * ((size_t)g->ntris * 6 + 1));
  o->zz = (float *)malloc(sizeof(float) * ((size_t)g->ntris * 3 + 1));
  (void)nthreads;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 0; i < g->ntris; i++) {
    float sx[3], sy[3], sz[3];
    int cl = setup_persp_tri(g, f, i, sx, sy, sz);
    o->cls[i] = (uint8_t)cl;
    for (int k = 0; k < 3; k++) {
      o->sp[(size_t)i * 6 + k * 2] = sx[k];
      o->sp[(size_t)i * 6 + k * 2 + 1] = sy[k];
      o->zz[(size_t)i * 3 + k] = sz[k];
    }
  }
}

static void init_ctx(shade_ctx *c, const orc_frame *f, const orc_group *g, int gid_base,
                     const orc_alpha *alphas, int nalpha, const orc_shadow *sh, int nsh) {
  memset(c, 0, sizeof *c);
  c->f = f;
  c->g = g;
  c->gid_base = gid_base;
  c->alpha = NULL;
  if ((g->flags & ORC_ALPHA) && g->alpha_index >= 0 && g->alpha_index < nalpha) c->alpha = &alphas[g->alpha_index];
  c->sh = sh;
  c->nsh = nsh;
  c->num_mip = (g->flags & ORC_MIP) ? g->tex_size : 0;
  if (g->flags & ORC_NORMAL) {
    /* av_draw_normmap.c:127: int specPow = exp2(12*(1.f - roughness)), with
     * exp2 correctly rounded; the third specular term's power is
     * (int)half_sqrt((float)specPow), half_sqrt correctly rounded */
    float e = 12.f * (1.f - g->roughness);
    c->spec_pow = f2i((float)exp2((double)e));
    c->spec_pow2 = f2i(sqrtf((float)c->spec_pow));
  }
}

int orc_draw_all(orc_frame *f, const orc_group *g, int ng, const uint8_t *mask,
                 const orc_alpha *alphas, int nalpha,
                 const orc_shadow *shadows, int nshadow, int nthreads) {
  if (f->w % TILE != 0) return -1;
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    if ((g[tn].flags & ORC_ALPHA) && (g[tn].alpha_index < 0 || g[tn].alpha_index >= nalpha)) return -2;
    if ((g[tn].flags & ORC_SHADOW) && nshadow < 1) return -3;
    if ((g[tn].flags & ORC_MULTI) && !(g[tn].flags & ORC_ALPHA) && tn + 3 >= ng) return -4;
  }
  if (nthreads < 1) nthreads = 1;
  size_t npix = (size_t)f->w * f->h;
  for (size_t p = 0; p < npix; p++) { f->tri_id[p] = -1; f->cov[p] = 0; }
  int wc = f->w / TILE, hc = f->h / TILE;
  setup_out *so = (setup_out *)calloc((size_t)ng, sizeof(setup_out));
  int *base = (int *)calloc((size_t)ng + 1, sizeof(int));
  for (int tn = 0; tn < ng; tn++) base[tn + 1] = base[tn] + g[tn].ntris;
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    setup_group(&g[tn], f, &so[tn], nthreads);
  }

  /* small triangles: every material, in index order (Ops0.py:501-569).
   * The OpenMP build splits the screen into row strips; every strip walks
   * every small triangle in order and keeps only its rows, so the result
   * is the serial one. */
  int nstrips = nthreads > 1 ? nthreads * 4 : 1;
  if (nstrips > f->h) nstrips = f->h > 0 ? f->h : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
  for (int st = 0; st < nstrips; st++) {
    int r0 = (int)((long long)f->h * st / nstrips);
    int r1 = (int)((long long)f->h * (st + 1) / nstrips);
    if (nstrips == 1) { r0 = INT_MIN; r1 = INT_MAX; }
    for (int tn = 0; tn < ng; tn++) {
      if (mask && mask[tn]) continue;
      shade_ctx c;
      init_ctx(&c, f, &g[tn], base[tn], alphas, nalpha, shadows, nshadow);
      for (int i = 0; i < g[tn].ntris; i++) {
        if (so[tn].cls[i] != 1) continue;
        draw_small_tri(&c, i, so[tn].sp + (size_t)i * 6, so[tn].zz + (size_t)i * 3, r0, r1);
      }
    }
  }

  /* large triangles, per material: coarse bins then the tiled draw
   * (Ops0.py:572-646) */
  ivec *bins = (ivec *)calloc((size_t)wc * hc + 1, sizeof(ivec));
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    for (int t = 0; t < wc * hc; t++) bins[t].n = 0;
    for (int i = 0; i < g[tn].ntris; i++) {
      if (so[tn].cls[i] != 2) continue;
      coarse_tri(so[tn].sp + (size_t)i * 6, wc, hc, i, emit_bin, bins);
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) if (nthreads > 1)
    for (int bx = 0; bx < wc * hc; bx++) {
      shade_ctx c;
      init_ctx(&c, f, &g[tn], base[tn], alphas, nalpha, shadows, nshadow);
      for (int k = 0; k < bins[bx].n; k++) {
        int i = bins[bx].v[k];
        draw_tiled_tri(&c, i, bx, so[tn].sp + (size_t)i * 6, so[tn].zz + (size_t)i * 3);
      }
    }
  }
  for (int t = 0; t < wc * hc; t++) free(bins[t].v);
  free(bins);
  for (int tn = 0; tn < ng; tn++) { free(so[tn].cls); free(so[tn].sp); free(so[tn].zz); }
  free(so);
  free(base);
  return 0;
}

long orc_coarse_counts(const orc_group *g, const orc_frame *f, int32_t *tile_counts) {
  int wc = f->w / TILE, hc = f->h / TILE;
  memset(tile_counts, 0, sizeof(int32_t) * (size_t)wc * hc);
  setup_out so;
  setup_group(g, f, &so, 1);
  for (int i = 0; i < g->ntris; i++)
    if (so.cls[i] == 2) coarse_tri(so.sp + (size_t)i * 6, wc, hc, i, emit_count, tile_counts);
  long total = 0;
  for (int t = 0; t < wc * hc; t++) total += tile_counts[t];
  free(so.cls); free(so.sp); free(so.zz);
  return total;
}

/* ------------------------------------------------------------------ */
/* shadow depth pass                                                   */
/* ------------------------------------------------------------------ */

/* trisetupOrtho.c:20-59 */
static int setup_ortho_tri(const orc_group *g, const orc_shadow *s, float bias, int i,
                           int ix[3], int iy[3], float z[3]) {
  f3 vp = {s->pos[0], s->pos[1], s->pos[2]};
  f3 svd = f3ld(s->vv), svx = f3ld(s->vv + 3), svy = f3ld(s->vv + 6);
  int dim = s->dim;
  int yes = 1;
  for (int k = 0; k < 3; k++) {
    f3 x = f3sub(f3ld(g->xyz + (size_t)(i * 3 + k) * 3), vp);
    float dd = dot3(x, svd);
    float dx = dot3(x, svx);
    float dy = dot3(x, svy);
    dd += bias;
    dd = 1 / dd;
    dx = dx * s->scale + (float)(dim / 2);
    dy = dy * -s->scale + (float)(dim / 2);
    ix[k] = f2i(dx);
    iy[k] = f2i(dy);
    z[k] = dd;
    if (!(dd > 0) || ix[k] < -120 || ix[k] >= dim + 120 || iy[k] < -120 || iy[k] >= dim + 120) yes = 0;
  }
  return yes;
}

/* drawmin.c:25-115 and drawminalpha.c:23-158, rows limited to [row0,row1) */
static void draw_shadow_tri(float *F, int wF, int hF, const int ix[3], const int iy[3], const float iz[3],
                            const orc_group *g, int tri, const orc_alpha *al, int row0, int row1) {
  int x1 = ix[0], x2 = ix[1], x3 = ix[2], y1 = iy[0], y2 = iy[1], y3 = iy[2];
  float z1 = iz[0], z2 = iz[1], z3 = iz[2];
  f2 uv1 = {0, 0}, uv2 = {0, 0}, uv3 = {0, 0};
  if (al) {
    uv1 = f2mul(f2ld(g->uv + ((size_t)tri * 3 + 0) * 2), z1);
    uv2 = f2mul(f2ld(g->uv + ((size_t)tri * 3 + 1) * 2), z2);
    uv3 = f2mul(f2ld(g->uv + ((size_t)tri * 3 + 2) * 2), z3);
  }
  f2 ft;
  if (y1 > y2) { SWAPI(y1, y2); SWAPI(x1, x2); SWAPV(z1, z2); ft = uv1; uv1 = uv2; uv2 = ft; }
  if (y2 > y3) { SWAPI(y2, y3); SWAPI(x2, x3); SWAPV(z2, z3); ft = uv2; uv2 = uv3; uv3 = ft; }
  if (y1 > y2) { SWAPI(y1, y2); SWAPI(x1, x2); SWAPV(z1, z2); ft = uv1; uv1 = uv2; uv2 = ft; }
  if (!((y1 < hF) && (y3 >= 0))) return;
  if (y1 >= row1 || y3 < row0) return;
  float q = (float)(y2 - y1) / (float)(y3 - y1);
  int x4 = f2i((float)x1 + q * (float)(x3 - x1));
  int y4 = y2;
  float z4 = z1 + q * (z3 - z1);
  float u1 = uv1.x, u2 = uv2.x, u3 = uv3.x, v1 = uv1.y, v2 = uv2.y, v3 = uv3.y;
  float u4 = u1 + q * (u3 - u1);
  float v4 = v1 + q * (v3 - v1);
  int lenT = al ? al->len : 1;
  float lm1 = (float)(lenT - 1);

  float slope1 = (float)(x2 - x1) / (float)(y2 - y1);
  float slope2 = (float)(x4 - x1) / (float)(y4 - y1);
  float slopeu1 = (u2 - u1) / (float)(y2 - y1);
  float slopev1 = (v2 - v1) / (float)(y2 - y1);
  float slopeu2 = (u4 - u1) / (float)(y4 - y1);
  float slopev2 = (v4 - v1) / (float)(y4 - y1);
  float slopez1 = (z2 - z1) / (float)(y2 - y1);
  float slopez2 = (z4 - z1) / (float)(y4 - y1);
  float cx1 = (float)x1, cx2 = (float)x1, cz1 = z1, cz2 = z1;
  float cu1 = u1, cv1 = v1, cu2 = u1, cv2 = v1;
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPV(slopeu1, slopeu2); SWAPV(slopev1, slopev2);
  }
  for (int cy = y1; cy <= y2; cy++) {
    if (cy >= row0 && cy < row1) {
      int axe = f2i(cx1);
      for (int ax = f2i(cx2); ax <= axe; ax++) {
        if (cy >= 0 && cy < hF && ax >= 0 && ax < wF) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          size_t pix = (size_t)wF * cy + ax;
          if (F[pix] > tz) {
            if (al) {
              int tex1 = f2i((((1 - t) * cu2 + t * cu1) * tz) * lm1);
              tex1 = iabs(tex1) & (lenT - 1);
              int tex2 = f2i((lm1 * ((1 - t) * cv2 + t * cv1)) * tz);
              tex2 = iabs(tex2) & (lenT - 1);
              tex2 *= lenT;
              if (al->mask[tex1 + tex2]) F[pix] = tz;
            } else {
              F[pix] = tz;
            }
          }
        }
      }
    }
    cx1 += slope1; cx2 += slope2; cz1 += slopez1; cz2 += slopez2;
    cu1 += slopeu1; cv1 += slopev1; cu2 += slopeu2; cv2 += slopev2;
  }
  slope1 = (float)(x3 - x2) / (float)(y3 - y2);
  slope2 = (float)(x3 - x4) / (float)(y3 - y4);
  slopeu1 = (u3 - u2) / (float)(y3 - y2);
  slopev1 = (v3 - v2) / (float)(y3 - y2);
  slopeu2 = (u3 - u4) / (float)(y3 - y4);
  slopev2 = (v3 - v4) / (float)(y3 - y4);
  slopez1 = (z3 - z2) / (float)(y3 - y2);
  slopez2 = (z3 - z4) / (float)(y3 - y4);
  cx1 = (float)x3; cx2 = (float)x3; cz1 = z3; cz2 = z3;
  cu1 = u3; cv1 = v3; cu2 = u3; cv2 = v3;
  if (slope1 < slope2) {
    SWAPV(slope1, slope2); SWAPV(slopez1, slopez2); SWAPV(slopeu1, slopeu2); SWAPV(slopev1, slopev2);
  }
  for (int cy = y3; cy > y2; cy--) {
    if (cy >= row0 && cy < row1) {
      int axe = f2i(cx2);
      for (int ax = f2i(cx1); ax <= axe; ax++) {
        if (cy >= 0 && cy < hF && ax >= 0 && ax < wF) {
          float t = ((float)ax - cx2) / (cx1 - cx2);
          t = fmaxf(0.f, fminf(1.f, t));
          float tz = 1 / ((1 - t) * cz2 + t * cz1);
          size_t pix = (size_t)wF * cy + ax;
          if (F[pix] > tz) {
            if (al) {
              int tex1 = f2i((((1 - t) * cu2 + t * cu1) * tz) * lm1);
              tex1 = iabs(tex1) & (lenT - 1);
              int tex2 = f2i((lm1 * ((1 - t) * cv2 + t * cv1)) * tz);
              tex2 = iabs(tex2) & (lenT - 1);
              tex2 *= lenT;
              if (al->mask[tex1 + tex2]) F[pix] = tz;
            } else {
              F[pix] = tz;
            }
          }
        }
      }
    }
    cx1 -= slope1; cx2 -= slope2; cz1 -= slopez1; cz2 -= slopez2;
    cu1 -= slopeu1; cv1 -= slopev1; cu2 -= slopeu2; cv2 -= slopev2;
  }
}

int orc_shadow_map(orc_shadow *s, const orc_group *g, int ng, const uint8_t *cast,
                   const orc_alpha *alphas, int nalpha, float bias, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  for (int tn = 0; tn < ng; tn++) {
    if (!cast[tn]) continue;
    if ((g[tn].flags & ORC_ALPHA) && (g[tn].alpha_index < 0 || g[tn].alpha_index >= nalpha)) return -2;
  }
  int dim = s->dim;
  for (int tn = 0; tn < ng; tn++) {
    if (!cast[tn]) continue;
    const orc_group *gg = &g[tn];
    int nt = gg->ntris;
    int *ok = (int *)malloc(sizeof(int) * ((size_t)nt + 1));
    int *ix = (int *)malloc(sizeof(int) * ((size_t)nt * 3 + 1));
    int *iy = (int *)malloc(sizeof(int) * ((size_t)nt * 3 + 1));
    float *iz = (float *)malloc(sizeof(float) * ((size_t)nt * 3 + 1));
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
    for (int i = 0; i < nt; i++) ok[i] = setup_ortho_tri(gg, s, bias, i, ix + 3 * i, iy + 3 * i, iz + 3 * i);
    const orc_alpha *al = (gg->flags & ORC_ALPHA) ? &alphas[gg->alpha_index] : NULL;
    /* depth-min is order independent; strips keep the per-pixel min */
    int nstrips = nthreads > 1 ? nthreads * 4 : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
    for (int st = 0; st < nstrips; st++) {
      int r0 = (int)((long long)dim * st / nstrips);
      int r1 = (int)((long long)dim * (st + 1) / nstrips);
      if (nstrips == 1) { r0 = INT_MIN; r1 = INT_MAX; }
      for (int i = 0; i < nt; i++)
        if (ok[i]) draw_shadow_tri(s->map, dim, dim, ix + 3 * i, iy + 3 * i, iz + 3 * i, gg, i, al, r0, r1);
    }
    free(ok); free(ix); free(iy); free(iz);
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* clear and gamma                                                     */
/* ------------------------------------------------------------------ */

void orc_clear_depth(float *f, int w, int h, int lenP) {
  /* clearzb.c:10-22: each of lenP x lenP work-items clears a (w/lenP)x(h/lenP) block */
  int bw = w / lenP, bh = h / lenP;
  for (int cy = 0; cy < bh * lenP; cy++)
    for (int cx = 0; cx < bw * lenP; cx++) f[(size_t)w * cy + cx] = 65535.f;
}

void orc_gamma(uint16_t *r, uint16_t *g, uint16_t *b, int w, int h, float exposure) {
  /* Post/gamma.c:38-52 */
  size_t n = (size_t)w * h;
  float e8 = 8 * exposure;
  for (size_t p = 0; p < n; p++) {
    float jx = sqrtf(e8 * (float)r[p]) / 1.1f;
    float jy = sqrtf(e8 * (float)g[p]) / 1.1f;
    float jz = sqrtf(e8 * (float)b[p]) / 1.1f;
    float m = fmaxf(jx, fmaxf(jy, jz)) / 255.f;
    if (m > 1.f) {
      float sm = sqrtf(m);
      jx = jx / sm; jy = jy / sm; jz = jz / sm;
    }
    r[p] = (uint16_t)f2i(fminf(255.f, jx));
    g[p] = (uint16_t)f2i(fminf(255.f, jy));
    b[p] = (uint16_t)f2i(fminf(255.f, jz));
  }
}


/* ------------------------------------------------------------------ */
/* vertex stage                                                        */
/* ------------------------------------------------------------------ */

static inline f3 f3max(f3 a, float s) { f3 r = {fmaxf(a.x, s), fmaxf(a.y, s), fmaxf(a.z, s)}; return r; }
static inline float fast_length(f3 v) { return sqrtf(dot3(v, v)); }
static inline void f3st(float *p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

void orc_transform(float *xyz, float *vn, const float old_rm[9], const float rot_mat[9],
                   const float origin[3], int start, int end) {
  /* vert.c:3-28 with OldR = rows of oldRM and RR = rows of rotMat^T
   * (CLDraw.rotate, Ops.py:481-497) */
  f3 oldr[3], rr[3], o = f3ld(origin);
  for (int i = 0; i < 3; i++) {
    oldr[i] = f3ld(old_rm + 3 * i);
    rr[i].x = rot_mat[i]; rr[i].y = rot_mat[3 + i]; rr[i].z = rot_mat[6 + i];
  }
  for (int v = start; v < end; v++) {
    f3 p = f3sub(f3ld(xyz + 3 * (size_t)v), o);
    f3 q = {dot3(p, oldr[0]), dot3(p, oldr[1]), dot3(p, oldr[2])};
    f3 r = {dot3(q, rr[0]), dot3(q, rr[1]), dot3(q, rr[2])};
    f3st(xyz + 3 * (size_t)v, f3add(r, o));
    f3 n = f3ld(vn + 3 * (size_t)v);
    f3 m = {dot3(n, oldr[0]), dot3(n, oldr[1]), dot3(n, oldr[2])};
    f3 l = {dot3(m, rr[0]), dot3(m, rr[1]), dot3(m, rr[2])};
    f3st(vn + 3 * (size_t)v, l);
  }
}

void orc_translate(float *xyz, const float c[3], int start, int end) {
  /* vert.c:29-36 */
  f3 o = f3ld(c);
  for (int v = start; v < end; v++) f3st(xyz + 3 * (size_t)v, f3add(f3ld(xyz + 3 * (size_t)v), o));
}

void orc_vert_light(const float *xyz, const float *vn, float *li, int nv,
                    const float *dir_int, const float *dir_dir, int nd,
                    const float *pint, const float *ppos, int np,
                    const float *sint, const float *sdir, const float *spos, int ns, float amb) {
  /* vert.c:38-88; light 0 is the primary light, shaded per pixel */
  for (int v = 0; v < nv; v++) {
    f3 x = f3ld(xyz + 3 * (size_t)v), n = f3ld(vn + 3 * (size_t)v);
    f3 light = {0.f, 0.f, 0.f};
    for (int i = 1; i < nd; i++) {   /* vert.c:57-60 */
      float s = fmaxf(0.f, dot3(n, f3ld(dir_dir + 3 * i)) + 0.5f) * 0.66f;
      light = f3add(light, f3smul(s, f3ld(dir_int + 3 * i)));
    }
    for (int i = 0; i < np; i++) {   /* vert.c:61-66 */
      f3 pl = f3sub(x, f3ld(ppos + 3 * i));
      if (dot3(n, pl) > 0.f) {
        float fl = fast_length(pl);
        float s = dot3(n, fast_normalize(pl)) / (1.f + fl * fl);
        light = f3add(light, f3smul(s, f3ld(pint + 3 * i)));
      }
    }
    for (int i = 0; i < ns; i++) {   /* vert.c:67-82 */
      f3 pl = f3sub(x, f3ld(spos + 3 * i)), sd = f3ld(sdir + 3 * i);
      if (dot3(sd, pl) > 0.f && dot3(n, pl) > 0.f) {
        f3 u = fast_normalize(pl);
        float fl = fast_length(pl);
        float s = dot3(n, u) * dot3(u, sd) / (1.5f + fl * fl);
        light = f3add(light, f3smul(s, f3ld(sint + 3 * i)));
      }
    }
    f3st(li + 3 * (size_t)v, f3max(light, amb));   /* vert.c:83-86 */
  }
}


/* ------------------------------------------------------------------ */
/* post effects                                                        */
/* ------------------------------------------------------------------ */

static inline f3 f3cross(f3 a, f3 b) {
  f3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}

void orc_ssao(uint16_t *r, uint16_t *g, uint16_t *b, const float *db, int w, int h, float sscale,
              const float *rnd) {
  /* ssao.c:6-97 over the (h/16) x (w/16) work-groups of 16 x 16 (Ops.py:973-983) */
  const float radius = 1.f, bias = 0.002f;
  size_t n = (size_t)w * h;
  int w2 = w / 2, h2 = h / 2;
  for (int cy = 0; cy < h / 16 * 16; cy++)
    for (int cx = 0; cx < w / 16 * 16; cx++) {
      size_t pix = (size_t)w * cy + cx;
      float ao = 0.f;
      float d = db[pix];
      f3 pv = {((float)cx + 0.5f - (float)w2) / sscale, (-((float)cy + 0.5f - (float)h2)) / sscale, 1.f};
      f3 pos = f3smul(d, pv);
      size_t ix = pix + 1, iy = pix + (size_t)w;
      float dx = ix < n ? db[ix] : 65535.f;
      float dy = iy < n ? db[iy] : 65535.f;
      const int rx = 1, ry = 1;
      f3 xv = {((float)cx + 0.5f + (float)rx - (float)w2) / sscale, (-((float)cy + 0.5f - (float)h2)) / sscale, 1.f};
      f3 yv = {((float)cx + 0.5f - (float)w2) / sscale, (-((float)cy + 0.5f + (float)ry - (float)h2)) / sscale, 1.f};
      f3 px = f3smul(dx, xv), py = f3smul(dy, yv);
      f3 norm = f3smul((float)(rx * ry), fast_normalize(f3cross(f3sub(pos, px), f3sub(pos, py))));
      for (int i = 0; i < 16; i++) {
        f3 sv = {rnd[(7 * i + 13 * ((cx * 3) & 7) + 17 * ((cy * 7) & 7)) & 31],
                 rnd[(7 * i + 1 + 13 * ((cx * 7) & 7) + 17 * ((cy * 5) & 7)) & 31],
                 rnd[(7 * i + 2 + 13 * ((cx * 5) & 7) + 17 * ((cy * 3) & 7)) & 31]};
        sv = f3sub(f3mul(sv, 2.f), (f3){1.f, 1.f, 1.f});
        sv = fast_normalize(sv);
        if (dot3(sv, norm) < 0) sv = f3sub(sv, f3mul(f3smul(2.f, norm), dot3(sv, norm)));
        float rlen = rnd[(7 * i + 3 + 13 * ((cx * 3) & 7) + 17 * ((cy * 3) & 7)) & 31];
        sv = f3mul(sv, rlen * rlen * radius);
        sv = f3add(sv, pos);
        float sz = sv.z;
        float sx = (sv.x / sz * sscale) + (float)w2;
        float sy = (-sv.y / sz * sscale) + (float)h2;
        if (sx >= 0 && sx < (float)w && sy >= 0 && sy < (float)h) {
          float sampd = db[(size_t)w * f2i(sy) + f2i(sx)];
          float disct = fclampf(2.f - (d - sampd), 0.f, 1.f);
          ao += disct * ((sampd < sz - bias) ? 1.f : 0.f);
        }
      }
      ao /= 16.f;
      if (d > 6000) ao = 0;
      ao = fclampf(ao * 2.f, 0.f, 1.f);
      r[pix] = u16sat((1 - ao) * (float)r[pix]);
      g[pix] = u16sat((1 - ao) * (float)g[pix]);
      b[pix] = u16sat((1 - ao) * (float)b[pix]);
    }
}

void orc_dof(const uint16_t *r, const uint16_t *g, const uint16_t *b, const float *db, int w, int h,
             float focus, uint16_t *r2, uint16_t *g2, uint16_t *b2) {
  /* dof.c:4-69 over the (h/16) x (w/16) work-groups of 16 x 16 (Ops.py:985-995) */
  const float maxcoc = 4.f, aperture = 4.f;
  for (int iy = 0; iy < h / 16 * 16; iy++)
    for (int ix = 0; ix < w / 16 * 16; ix++) {
      float cx = (float)ix + 0.5f, cy = (float)iy + 0.5f;
      float d = db[(size_t)w * iy + ix];
      float coc = aperture * fabsf(d - focus) / focus / d;
      float dofR = 0, dofG = 0, dofB = 0, nsamples = 0;
      float radius = fminf(maxcoc, coc);
      for (int sy = f2i(floorf(cy - radius)); (float)sy < ceilf(cy + radius); sy++)
        for (int sx = f2i(floorf(cx - radius)); (float)sx < ceilf(cx + radius); sx++) {
          float cover = (1.f - fmaxf(cx - radius - (float)sx, 0.f)) * (1.f - fmaxf(cy - radius - (float)sy, 0.f));
          cover *= fminf(cx + radius - (float)sx, 1.f) * fminf(cy + radius - (float)sy, 1.f);
          if (sx < 0 || sx >= w || sy < 0 || sy >= h) continue;
          float ecoc = db[(size_t)w * sy + sx];
          ecoc = aperture * fabsf(ecoc - focus) / focus / ecoc;
          ecoc = fminf(maxcoc, ecoc);
          if (radius > ecoc) cover *= ecoc / radius;
          size_t q = (size_t)w * sy + sx;
          dofR += (float)r[q] * cover;
          dofG += (float)g[q] * cover;
          dofB += (float)b[q] * cover;
          nsamples += cover;
        }
      dofR /= nsamples; dofG /= nsamples; dofB /= nsamples;
      size_t pix = (size_t)w * iy + ix;
      r2[pix] = u16sat(dofR); g2[pix] = u16sat(dofG); b2[pix] = u16sat(dofB);
    }
}

static const float BLOOM_W[9] = {0.00816f, 0.01384f, 0.02207f, 0.03306f, 0.04654f,
                                 0.06157f, 0.07654f, 0.08941f, 0.09815f};   /* taps 9..1 */

void orc_bloom(uint16_t *r, uint16_t *g, uint16_t *b, int w, int h) {
  int wf = w / 2, hf = h / 2;
  size_t hn = (size_t)wf * (hf + 8);               /* 8 zero rows past the end */
  uint16_t *br[3], *hb[3], *vb[3];
  uint16_t *fr[3] = {r, g, b};
  for (int k = 0; k < 3; k++) {
    br[k] = (uint16_t *)calloc(hn, 2);
    hb[k] = (uint16_t *)calloc(hn, 2);
    vb[k] = (uint16_t *)calloc(hn, 2);
  }
  /* blur.c:22-34: bright pass at half resolution (the 4 taps of row 2cy at
   * columns 2cx, 2cx+1, 2cx+1, 2cx+2 as the source indexes them) */
  for (int cy = 0; cy < hf - 2; cy++)
    for (int cx = 0; cx < wf; cx++) {
      int y1 = imin(wf * (hf - 1) * 4, wf * cy * 4 + 1);
      int x1 = imin(wf * 2 - 1, cx * 2 + 1);
      float c[3];
      for (int k = 0; k < 3; k++) {
        const uint16_t *f = fr[k];
        c[k] = (float)(f[wf * cy * 4 + cx * 2] / 4 + f[y1 + cx * 2] / 4 + f[wf * cy * 4 + x1] / 4 + f[y1 + x1] / 4);
      }
      float lum = (float)(0.3626 * (double)c[0] + 0.5152 * (double)c[1] + 0.1222 * (double)c[2]);
      for (int k = 0; k < 3; k++) br[k][(size_t)wf * cy + cx] = u16sat(c[k] * lum / 256.f / 256.f);
    }
  /* blur.c:38-66: horizontal 19-tap blur of the bright pass */
  for (int cy = 0; cy < hf - 1; cy++)
    for (int cx = 0; cx < wf; cx++)
      for (int k = 0; k < 3; k++) {
        const uint16_t *row = br[k] + (size_t)wf * cy;
        float a = 0.f;
        for (int d = 9; d >= 1; d--)
          if (cx > d - 1) a = a + BLOOM_W[9 - d] * (float)row[cx - d];
        a += 0.10125f * (float)row[cx];
        for (int d = 1; d <= 9; d++)
          if (cx < wf - d) a = a + BLOOM_W[9 - d] * (float)row[cx + d];
        a /= 0.9f;
        hb[k][(size_t)wf * cy + cx] = u16sat(a);
      }
  /* blur2.c:22-50: vertical 19-tap blur; the lower taps are bounded by the
   * half width, as the source writes it, so rows past the buffer read 0 */
  for (int cy = 0; cy < hf - 1; cy++)
    for (int cx = 0; cx < wf; cx++)
      for (int k = 0; k < 3; k++) {
        const uint16_t *col = hb[k] + cx;
        float a = 0.f;
        for (int d = 9; d >= 1; d--)
          if (cy > d - 1) a = a + BLOOM_W[9 - d] * (float)col[(size_t)wf * (cy - d)];
        a += 0.10125f * (float)col[(size_t)wf * cy];
        for (int d = 1; d <= 9; d++)
          if (cy < wf - d) a = a + BLOOM_W[9 - d] * (float)(cy + d < hf + 8 ? col[(size_t)wf * (cy + d)] : 0);
        a /= 0.9f;
        vb[k][(size_t)wf * cy + cx] = u16sat(a);
      }
  /* blur2.c:54-79: bilinear upsample added to the full-resolution frame */
  int W2 = wf * 2, H2 = hf * 2, lenT = wf;
  for (int cy = 0; cy < H2; cy++)
    for (int cx = 0; cx < W2; cx++) {
      float texr1 = (float)cx / 2.f;
      int tex1 = f2i(texr1);
      texr1 -= (float)tex1;
      float texr2 = (float)cy / 2.f;
      int tex2 = f2i(texr2);
      texr2 -= (float)tex2;
      int tex = tex1 + lenT * tex2;
      int tex10 = imin(tex1 + 1, lenT - 1) + lenT * tex2;
      int tex01 = tex1 + lenT * imin(tex2 + 1, H2 / 2 - 2);
      int tex11 = imin(tex1 + 1, lenT - 1) + lenT * imin(tex2 + 1, H2 / 2 - 2);
      float texi1 = 1 - texr1, texi2 = 1 - texr2;
      for (int k = 0; k < 3; k++) {
        const uint16_t *T = vb[k];
        uint16_t *f = fr[k] + (size_t)w * cy + cx;
        *f = u16sat((float)*f + (texi1 * texi2 * (float)T[tex] + texr1 * texi2 * (float)T[tex10] +
                                 texi1 * texr2 * (float)T[tex01] + texr1 * texr2 * (float)T[tex11]));
      }
    }
  for (int k = 0; k < 3; k++) { free(br[k]); free(hb[k]); free(vb[k]); }
}
