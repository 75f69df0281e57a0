// kernels.cuh -- CUDA kernels of the rasterizer hot path (sm_100a).
//
// Frame = visibility then shading:
//   k_init_keys    one 64-bit visibility word per pixel from the depth buffer
//   k_setup        per triangle: projection, rejection, small/large split
//                  (trisetup.c), warp-ballot compaction into two lists
//   k_raster_small persistent; warps take 32 small triangles, each lane walks
//                  its rows (drawSmall, Templates.py:250-323) and the warp
//                  fills the queued spans pixel-parallel; fragment = 64-bit
//                  atomicMin(depth key | ~order) in the L2-resident buffer.
//                  Opaque and alpha-tested materials run as separate
//                  specialisations (the opaque one needs far fewer registers)
//   k_coarse       per large triangle: tile binning of coarse.c, written as
//                  (triangle, tile) units with warp-scan offsets
//   k_raster_tiled persistent over units: per-tile restart of the tiled
//                  `draw` (Templates.py:93-185), same span queue
//   k_shade        per pixel: decode the winner, replay its row interpolants
//                  and shade once (bilinear/trilinear, alpha, shadow)
// The packed key makes the result independent of scheduling: smallest depth
// wins, equal depths go to the later fragment of the reference's serial
// order (small pass < large pass, material, triangle, bottom < top half).
#pragma once
#include "raster.cuh"

namespace axr {

struct DrawParams {
  const GroupDev *groups;
  int ngroups;
  int total_tris;
  ViewDev view;
  LightDev light;
  ShadowDev sh[2];
  int nsh;
  uint64_t *keys;
  uint16_t *ro, *go, *bo;
  float *db;
  uint32_t *small_list;  // opaque small triangles from the front, alpha-tested from the back
  uint32_t *items;       // row chunks of small triangles: (list position << 2 | chunk), same two ends
  uint32_t *large_list;
  uint2 *units;          // opaque (triangle, tile) units from the front, alpha-tested from the back
  uint32_t *ctr;         // see CTR_*
  uint32_t cap_list, cap_units;
  int min_chunk;         // rows per small-triangle work item (at least; tuning knob)
  int claim_k;           // claim_size's k for the short queues (0: 32 items per claim)
  float2 *mipc;          // per triangle of a mip group: (mip fraction, mip level), written by
                         // the setup, read by the shade; null: the shade computes them
};

enum {
  CTR_SMALL = 0, CTR_SMALL_A, CTR_LARGE, CTR_UNITS, CTR_UNITS_A, CTR_WORK_SMALL, CTR_WORK_SMALL_A, CTR_WORK_LARGE,
  CTR_WORK_UNITS, CTR_WORK_UNITS_A, CTR_OVERFLOW, CTR_SH_LIST, CTR_SH_LIST_A, CTR_SH_WORK, CTR_SH_WORK_A,
  CTR_UNITS_RESERVED, CTR_LIMIT, CTR_ITEMS, CTR_ITEMS_A, CTR_SH_ITEMS, CTR_SH_ITEMS_A,
  // tiled shadow pass: unit queue overflowed (the per-caster path drew the
  // map), units the map needed, non-empty tiles, tiles claimed (opaque, alpha)
  CTR_SH_OVERFLOW, CTR_SH_UNITS_NEED, CTR_SH_TILES, CTR_SH_TILE_WORK, CTR_SH_TILE_WORK_A, CTR_SH_ITEMS_TILED,
  CTR_N = 32
};

// Every data-dependent loop is bounded by construction (rows of a small
// triangle < 2*96, of a tile unit <= 2*16, of a shadow triangle <= 2*(dim+240)
// because of the setup rejections).  As a second line of defence each one
// also stops after LOOP_LIMIT rounds and records that in ctr[CTR_LIMIT],
// which the host reports as an error.
constexpr int LOOP_LIMIT = 1 << 16;


// ------------------------------------------------------------ helpers

__device__ __forceinline__ int find_group(const GroupDev *__restrict__ gs, int ng, uint32_t gtri) {
  int lo = 0, hi = ng - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((uint32_t)gs[mid].tri_base <= gtri) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// count of x in [ax0, ...] with (float)x <= bound, clipped to [0, w)
__device__ __forceinline__ void span_clip(int ax0, float bound, int w, int &lo, int &cnt) {
  lo = ax0 < 0 ? 0 : ax0;
  if (bound != bound) { cnt = 0; return; }
  float fb = floorf(bound);
  int hi = fb >= (float)(w - 1) ? w - 1 : f2i(fb);
  cnt = hi >= lo ? hi - lo + 1 : 0;
}

// A small triangle's rows (bottom half y1..y2, then top half y3..y2, both
// inclusive) are cut into at most MAX_CHUNKS chunks of at least MIN_CHUNK
// rows, so that large "small" triangles spread over several lanes; a lane
// replays the row accumulation up to its chunk, which keeps every
// interpolant bit-identical to the serial walk.
constexpr int MIN_CHUNK = 12;   // default of DrawParams::min_chunk
constexpr int CHUNK_BITS = 3;   // work item = list position << CHUNK_BITS | chunk
constexpr int MAX_CHUNKS = 1 << CHUNK_BITS;
__device__ __forceinline__ int small_rows(int y1, int y3) { return y3 - y1 + 2; }
// Items a warp claims at a time in a persistent loop over n work items:
// one per lane, unless that leaves warps of the launch without work (short
// queues: the alpha-tested triangles and casters, the large triangles);
// then fewer, so that every warp gets about `k` claims.  The value is the
// same for every warp.  On the 1080p scene this took the alpha-tested
// tiled raster from 133 to 100 us and the alpha casters from 103 to 92 us;
// the opaque rasterizers stay at 32 (fewer per claim made them slower).
// k = 0: always 32 -- the batched launches, whose warps move on to the
// next view's queue when one runs dry, so no warp idles.
__device__ __forceinline__ uint32_t claim_size(uint32_t n, uint32_t k) {
  if (k == 0) return 32u;
  uint32_t nw = gridDim.x * (blockDim.x >> 5) * k;
  uint32_t per = (n + nw - 1) / nw;
  return per < 1u ? 1u : (per > 32u ? 32u : per);
}

__device__ __forceinline__ int chunk_len(int rows, int min_chunk) {
  int c = (rows + MAX_CHUNKS - 1) / MAX_CHUNKS;
  return c < min_chunk ? min_chunk : c;
}

// ------------------------------------------------------------ keys / clear

__global__ void k_init_keys(const float *__restrict__ db, uint64_t *__restrict__ keys, int n, uint32_t *ctr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < CTR_N && blockIdx.x == 0) ctr[i] = 0;
  for (; i < n; i += gridDim.x * blockDim.x) keys[i] = ((uint64_t)depth_key(db[i]) << 32) | 0xffffffffull;
}

// clearzb.c:10-22 over lenP x lenP work-items of (w/lenP) x (h/lenP)
// blocks: columns [0, bw) of rows [0, bh) := 65535.  When bw == w those rows
// are one contiguous range, written with 16-byte stores.
__global__ void k_clear_depth(float *__restrict__ f, int w, int h, int lenP) {
  int bw = (w / lenP) * lenP, bh = (h / lenP) * lenP;
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  if (bw == w && ((uintptr_t)f & 15) == 0) {
    size_t n = (size_t)w * bh, n4 = n >> 2;
    const float4 v = make_float4(65535.f, 65535.f, 65535.f, 65535.f);
    for (size_t i = tid; i < n4; i += stride) reinterpret_cast<float4 *>(f)[i] = v;
    for (size_t i = (n4 << 2) + tid; i < n; i += stride) f[i] = 65535.f;
    return;
  }
  int n = bw * bh;
  for (int i = (int)tid; i < n; i += (int)stride) {
    int y = i / bw, x = i - y * bw;
    f[(size_t)w * y + x] = 65535.f;
  }
}

// Colour half of the current reference's clearZBuffer (Ops.py:939-946):
// every pixel of the three colour planes := (r, g, b); 16-byte stores when
// the planes are 16-byte aligned.
__global__ void k_fill_rgb(uint16_t *__restrict__ ro, uint16_t *__restrict__ go, uint16_t *__restrict__ bo, int n,
                           uint16_t r, uint16_t g, uint16_t b) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  size_t done = 0;
  if ((((uintptr_t)ro | (uintptr_t)go | (uintptr_t)bo) & 15) == 0) {
    size_t n8 = (size_t)n >> 3;
    uint32_t rr = r * 0x10001u, gg = g * 0x10001u, bb = b * 0x10001u;
    const uint4 vr = make_uint4(rr, rr, rr, rr), vg = make_uint4(gg, gg, gg, gg), vb = make_uint4(bb, bb, bb, bb);
    for (size_t i = tid; i < n8; i += stride) {
      reinterpret_cast<uint4 *>(ro)[i] = vr;
      reinterpret_cast<uint4 *>(go)[i] = vg;
      reinterpret_cast<uint4 *>(bo)[i] = vb;
    }
    done = n8 << 3;
  }
  for (size_t i = done + tid; i < (size_t)n; i += stride) {
    ro[i] = r;
    go[i] = g;
    bo[i] = b;
  }
}

// Post/gamma.c:38-52
__device__ __forceinline__ void gamma_px(uint16_t r, uint16_t g, uint16_t b, float e8, int &ro, int &go, int &bo) {
  float jx = sqrtf(e8 * (float)r) / 1.1f;
  float jy = sqrtf(e8 * (float)g) / 1.1f;
  float jz = sqrtf(e8 * (float)b) / 1.1f;
  float m = fmaxf(jx, fmaxf(jy, jz)) / 255.f;
  if (m > 1.f) {
    float sm = sqrtf(m);
    jx = jx / sm; jy = jy / sm; jz = jz / sm;
  }
  ro = f2i(fminf(255.f, jx));
  go = f2i(fminf(255.f, jy));
  bo = f2i(fminf(255.f, jz));
}

__global__ void k_gamma(uint16_t *r, uint16_t *g, uint16_t *b, int n, float exposure) {
  float e8 = 8 * exposure;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int x, y, z;
    gamma_px(r[i], g[i], b[i], e8, x, y, z);
    r[i] = (uint16_t)x; g[i] = (uint16_t)y; b[i] = (uint16_t)z;
  }
}

// Post/gamma.c's mapping packed as interleaved 8-bit RGB for display (the
// planes are left as they are): 3 bytes per pixel instead of 6 + 4.
__global__ void k_pack_rgb8(const uint16_t *__restrict__ r, const uint16_t *__restrict__ g,
                            const uint16_t *__restrict__ b, int n, float exposure, uint8_t *__restrict__ out) {
  float e8 = 8 * exposure;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int x, y, z;
    gamma_px(r[i], g[i], b[i], e8, x, y, z);
    out[3 * (size_t)i] = (uint8_t)x; out[3 * (size_t)i + 1] = (uint8_t)y; out[3 * (size_t)i + 2] = (uint8_t)z;
  }
}

// ------------------------------------------------------------ post effects
//
// Post/ssao.c and Post/dof.c over the (w/16*16) x (h/16*16) region their
// 16 x 16 work-groups cover (Ops.py:973-995); one thread a pixel, a block a
// 16 x 16 tile.  Arithmetic in source order, one IEEE rounding an operation.

struct SsaoParams {
  float rnd[32];      // the random table (entries 0..31 of the reference's 48)
  float sscale;
};

__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ssao.c:6-97 in place on the colour planes; the depth row past the buffer
// (read on the last row when h is a multiple of 16) reads 65535.  A pixel's
// 16 sample directions depend on it only through cx mod 8 and cy mod 8, so
// the block first builds the 64 x 16 normalised directions and length
// factors (stride 17 float4 per (cx, cy) class: conflict-free reads), with
// the same arithmetic as the per-pixel loop.  The two quotients by the
// sample depth share one reciprocal (quot_by_recip: still the IEEE quotient).
__global__ void __launch_bounds__(256) k_ssao(uint16_t *__restrict__ ro, uint16_t *__restrict__ go,
                                              uint16_t *__restrict__ bo, const float *__restrict__ F, int w, int h,
                                              SsaoParams S) {
  const float radius = 1.f, bias = 0.002f;
  __shared__ float rnd[32];                  // indexed per lane: staged out of the parameter space
  __shared__ float4 tab[64 * 17];
  if (threadIdx.x < 32) rnd[threadIdx.x] = S.rnd[threadIdx.x];
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * 16; e += blockDim.x) {
    int i = e & 15, mx = (e >> 4) & 7, my = e >> 7;
    int c3 = 13 * ((mx * 3) & 7), c7 = 13 * ((mx * 7) & 7), c5 = 13 * ((mx * 5) & 7);
    int y7 = 17 * ((my * 7) & 7), y5 = 17 * ((my * 5) & 7), y3 = 17 * ((my * 3) & 7);
    V3 sv{rnd[(7 * i + c3 + y7) & 31], rnd[(7 * i + 1 + c7 + y5) & 31], rnd[(7 * i + 2 + c5 + y3) & 31]};
    sv = fast_normalize(sub3(mul3(sv, 2.f), V3{1.f, 1.f, 1.f}));
    float rlen = rnd[(7 * i + 3 + c3 + y3) & 31];
    tab[(my * 8 + mx) * 17 + i] = make_float4(sv.x, sv.y, sv.z, rlen * rlen * radius);
  }
  __syncthreads();
  int cx = blockIdx.x * 16 + (threadIdx.x & 15), cy = blockIdx.y * 16 + (threadIdx.x >> 4);
  size_t n = (size_t)w * h, pix = (size_t)w * cy + cx;
  float w2 = (float)(w / 2), h2 = (float)(h / 2), ss = S.sscale;
  float d = F[pix];
  V3 pos = smul3(d, V3{((float)cx + 0.5f - w2) / ss, (-((float)cy + 0.5f - h2)) / ss, 1.f});
  float dx = pix + 1 < n ? F[pix + 1] : 65535.f;
  float dy = pix + w < n ? F[pix + w] : 65535.f;
  V3 px = smul3(dx, V3{((float)cx + 0.5f + 1.f - w2) / ss, (-((float)cy + 0.5f - h2)) / ss, 1.f});
  V3 py = smul3(dy, V3{((float)cx + 0.5f - w2) / ss, (-((float)cy + 0.5f + 1.f - h2)) / ss, 1.f});
  V3 norm = fast_normalize(cross3(sub3(pos, px), sub3(pos, py)));   // rx * ry = 1
  const float4 *T = tab + ((cy & 7) * 8 + (cx & 7)) * 17;
  float ao = 0.f;
#pragma unroll 4
  for (int i = 0; i < 16; i++) {
    float4 t = T[i];
    V3 sv{t.x, t.y, t.z};
    if (dot3(sv, norm) < 0) sv = sub3(sv, mul3(smul3(2.f, norm), dot3(sv, norm)));
    sv = add3(mul3(sv, t.w), pos);
    float sz = sv.z, y = span_recip(sz);
    float sx = (quot_by_recip(sv.x, sz, y) * ss) + w2;
    float sy = (quot_by_recip(-sv.y, sz, y) * ss) + h2;
    if (sx >= 0 && sx < (float)w && sy >= 0 && sy < (float)h) {
      float sampd = __ldg(F + (size_t)w * f2i(sy) + f2i(sx));
      float disct = fminf(fmaxf(2.f - (d - sampd), 0.f), 1.f);
      ao += disct * ((sampd < sz - bias) ? 1.f : 0.f);
    }
  }
  ao /= 16.f;
  if (d > 6000) ao = 0;
  ao = fminf(fmaxf(ao * 2.f, 0.f), 1.f);
  ro[pix] = u16sat((1 - ao) * (float)ro[pix]);
  go[pix] = u16sat((1 - ao) * (float)go[pix]);
  bo[pix] = u16sat((1 - ao) * (float)bo[pix]);
}

// dof.c:4-69: the circle-of-confusion gather into (r2, g2, b2).  The tile and
// a 4-pixel halo (the largest radius) are staged in shared memory with each
// source pixel's own circle of confusion.
constexpr int DOF_HALO = 4, DOF_SIDE = 16 + 2 * DOF_HALO;
__global__ void __launch_bounds__(256) k_dof(const uint16_t *__restrict__ ro, const uint16_t *__restrict__ go,
                                             const uint16_t *__restrict__ bo, const float *__restrict__ F, int w,
                                             int h, float focus, uint16_t *__restrict__ r2, uint16_t *__restrict__ g2,
                                             uint16_t *__restrict__ b2) {
  const float maxcoc = 4.f, aperture = 4.f;
  __shared__ float ecs[DOF_SIDE * DOF_SIDE];
  __shared__ ushort4 cs[DOF_SIDE * DOF_SIDE];
  int x0 = blockIdx.x * 16 - DOF_HALO, y0 = blockIdx.y * 16 - DOF_HALO;
  for (int k = threadIdx.x; k < DOF_SIDE * DOF_SIDE; k += blockDim.x) {
    int sx = x0 + k % DOF_SIDE, sy = y0 + k / DOF_SIDE;
    float e = 0.f;
    ushort4 c = make_ushort4(0, 0, 0, 0);
    if (sx >= 0 && sx < w && sy >= 0 && sy < h) {
      size_t q = (size_t)w * sy + sx;
      float f = F[q];
      e = fminf(maxcoc, aperture * fabsf(f - focus) / focus / f);
      c = make_ushort4(ro[q], go[q], bo[q], 0);
    }
    ecs[k] = e;
    cs[k] = c;
  }
  __syncthreads();
  int ix = blockIdx.x * 16 + (threadIdx.x & 15), iy = blockIdx.y * 16 + (threadIdx.x >> 4);
  float cx = (float)ix + 0.5f, cy = (float)iy + 0.5f;
  float d = F[(size_t)w * iy + ix];
  float coc = aperture * fabsf(d - focus) / focus / d;
  float dofR = 0, dofG = 0, dofB = 0, nsamples = 0;
  float radius = fminf(maxcoc, coc);
  float ylim = ceilf(cy + radius), xlim = ceilf(cx + radius);
  int sx0 = f2i(floorf(cx - radius));
  for (int sy = f2i(floorf(cy - radius)); (float)sy < ylim; sy++) {
    float wy0 = 1.f - fmaxf(cy - radius - (float)sy, 0.f), wy1 = fminf(cy + radius - (float)sy, 1.f);
    for (int sx = sx0; (float)sx < xlim; sx++) {
      float cover = (1.f - fmaxf(cx - radius - (float)sx, 0.f)) * wy0;
      cover *= fminf(cx + radius - (float)sx, 1.f) * wy1;
      if (sx < 0 || sx >= w || sy < 0 || sy >= h) continue;
      int k = (sy - y0) * DOF_SIDE + (sx - x0);
      float ecoc = ecs[k];
      if (radius > ecoc) cover *= ecoc / radius;
      ushort4 c = cs[k];
      dofR += (float)c.x * cover;
      dofG += (float)c.y * cover;
      dofB += (float)c.z * cover;
      nsamples += cover;
    }
  }
  dofR /= nsamples; dofG /= nsamples; dofB /= nsamples;
  size_t pix = (size_t)w * iy + ix;
  r2[pix] = u16sat(dofR); g2[pix] = u16sat(dofG); b2[pix] = u16sat(dofB);
}

// Post/blur.c + Post/blur2.c (CLDraw.blur): the bloom.  Four passes, each
// over the whole image before the next (the reference's barrier orders only
// its work-group; the launch-wide order is the one its phases are written
// for).  The half-resolution planes are wf x (hf + 8) with wf = w/2,
// hf = h/2: rows no pass writes, and the 8 rows the vertical blur reads past
// the image, stay 0.
struct BloomPlanes {
  uint16_t *br[3], *hb[3], *vb[3];   // bright pass, horizontal blur, vertical blur
};

__constant__ float c_bloom_w[9] = {0.00816f, 0.01384f, 0.02207f, 0.03306f, 0.04654f,
                                   0.06157f, 0.07654f, 0.08941f, 0.09815f};   // taps 9..1

// blur.c:22-34: rows [0, hf - 2) of the bright pass
__global__ void k_bloom_bright(const uint16_t *__restrict__ ro, const uint16_t *__restrict__ go,
                               const uint16_t *__restrict__ bo, int wf, int hf, BloomPlanes B) {
  int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y;
  if (cx >= wf || cy >= hf - 2) return;
  int y1 = min(wf * (hf - 1) * 4, wf * cy * 4 + 1);
  int x1 = min(wf * 2 - 1, cx * 2 + 1);
  int i0 = wf * cy * 4 + cx * 2, i1 = y1 + cx * 2, i2 = wf * cy * 4 + x1, i3 = y1 + x1;
  const uint16_t *f[3] = {ro, go, bo};
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; k++)
    c[k] = (float)((int)f[k][i0] / 4 + (int)f[k][i1] / 4 + (int)f[k][i2] / 4 + (int)f[k][i3] / 4);
  float lum = (float)(0.3626 * (double)c[0] + 0.5152 * (double)c[1] + 0.1222 * (double)c[2]);
#pragma unroll
  for (int k = 0; k < 3; k++) B.br[k][(size_t)wf * cy + cx] = u16sat(c[k] * lum / 256.f / 256.f);
}

// blur.c:38-66 (HORIZONTAL) and blur2.c:22-50 (vertical): the 19-tap blur
// of rows [0, hf - 1); the vertical lower taps are bounded by the half
// width, as blur2.c writes it
template <bool HORIZONTAL>
__global__ void k_bloom_blur(int wf, int hf, BloomPlanes B) {
  int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y;
  if (cx >= wf || cy >= hf - 1) return;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint16_t *src = HORIZONTAL ? B.br[k] : B.hb[k];
    const int pos = HORIZONTAL ? cx : cy;
    const size_t step = HORIZONTAL ? 1 : (size_t)wf;
    const uint16_t *c0 = src + (size_t)wf * cy + cx;
    float a = 0.f;
#pragma unroll
    for (int d = 9; d >= 1; d--)
      if (pos > d - 1) a = a + c_bloom_w[9 - d] * (float)c0[-(ptrdiff_t)(d * step)];
    a += 0.10125f * (float)c0[0];
#pragma unroll
    for (int d = 1; d <= 9; d++)
      if (pos < wf - d) a = a + c_bloom_w[9 - d] * (float)c0[d * step];
    a /= 0.9f;
    (HORIZONTAL ? B.hb[k] : B.vb[k])[(size_t)wf * cy + cx] = u16sat(a);
  }
}

// blur2.c:54-79: the vertical blur upsampled bilinearly and added to the
// frame's rows [0, 2 hf) and columns [0, 2 wf)
__global__ void k_bloom_add(uint16_t *__restrict__ ro, uint16_t *__restrict__ go, uint16_t *__restrict__ bo, int w,
                            int wf, int hf, BloomPlanes B) {
  int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y;
  if (cx >= 2 * wf || cy >= 2 * hf) return;
  const int lenT = wf;
  float texr1 = (float)cx / 2.f;
  int tex1 = f2i(texr1);
  texr1 -= (float)tex1;
  float texr2 = (float)cy / 2.f;
  int tex2 = f2i(texr2);
  texr2 -= (float)tex2;
  int t1n = min(tex1 + 1, lenT - 1), t2n = min(tex2 + 1, hf - 2);
  int tex = tex1 + lenT * tex2, tex10 = t1n + lenT * tex2, tex01 = tex1 + lenT * t2n, tex11 = t1n + lenT * t2n;
  float texi1 = 1 - texr1, texi2 = 1 - texr2;
  uint16_t *f[3] = {ro, go, bo};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint16_t *T = B.vb[k];
    uint16_t *p = f[k] + (size_t)w * cy + cx;
    *p = u16sat((float)*p + (texi1 * texi2 * (float)T[tex] + texr1 * texi2 * (float)T[tex10] +
                             texi1 * texr2 * (float)T[tex01] + texr1 * texr2 * (float)T[tex11]));
  }
}

// ------------------------------------------------------------ vertex stage
//
// Pipe/vert.c over a group's packed vertex arrays (3 floats a vertex).  A
// thread takes a quad of 4 consecutive vertices -- three aligned 16-byte
// words of each array (the arrays start 256-byte aligned, so vertex 4k
// starts a word) -- when the whole quad lies in [v0, v1); the partial quads
// at both ends go vertex by vertex.  The arithmetic is vert.c's, one IEEE
// rounding an operation in source order (no contraction).

struct VertXform {
  float oldr[9];   // rows of oldRM
  float rr[9];     // rows of rotMat transposed (CLDraw.rotate uploads rotMat.T)
  float o[3];      // origin (transform) or offset (Ttranslate)
};

struct VertLights {
  const float *dint, *ddir;           // directional lights; light 0 is shaded per pixel
  const float *pint, *ppos;           // point lights
  const float *sint, *sdir, *spos;    // spot lights
  int nd, np, ns;
  float amb;
};

__device__ __forceinline__ V3 rows3(const float *m, V3 v) {
  return V3{dot3(v, V3{m[0], m[1], m[2]}), dot3(v, V3{m[3], m[4], m[5]}), dot3(v, V3{m[6], m[7], m[8]})};
}

// vert.c:3-28 (transform)
__device__ __forceinline__ void xform_rotate(const VertXform &X, V3 &p, V3 &n) {
  V3 o{X.o[0], X.o[1], X.o[2]};
  p = add3(rows3(X.rr, rows3(X.oldr, sub3(p, o))), o);
  n = rows3(X.rr, rows3(X.oldr, n));
}

// vert.c:29-36 (Ttranslate)
__device__ __forceinline__ void xform_translate(const VertXform &X, V3 &p) { p = add3(p, V3{X.o[0], X.o[1], X.o[2]}); }

__device__ __forceinline__ V3 ldg3(const float *p, int i) { return ld3(p + 3 * i); }

__device__ __forceinline__ float fast_length(V3 v) { return sqrtf(dot3(v, v)); }

// vert.c:49-86 (vertL) for one vertex
__device__ __forceinline__ V3 vert_light_one(const VertLights &L, V3 x, V3 n) {
  V3 light{0.f, 0.f, 0.f};
  for (int i = 1; i < L.nd; i++) {
    float s = fmaxf(0.f, dot3(n, ldg3(L.ddir, i)) + 0.5f) * 0.66f;
    light = add3(light, smul3(s, ldg3(L.dint, i)));
  }
  for (int i = 0; i < L.np; i++) {
    V3 pl = sub3(x, ldg3(L.ppos, i));
    if (dot3(n, pl) > 0.f) {
      float fl = fast_length(pl);
      float s = dot3(n, fast_normalize(pl)) / (1.f + fl * fl);
      light = add3(light, smul3(s, ldg3(L.pint, i)));
    }
  }
  for (int i = 0; i < L.ns; i++) {
    V3 pl = sub3(x, ldg3(L.spos, i)), sd = ldg3(L.sdir, i);
    if (dot3(sd, pl) > 0.f && dot3(n, pl) > 0.f) {
      V3 u = fast_normalize(pl);
      float fl = fast_length(pl);
      float s = dot3(n, u) * dot3(u, sd) / (1.5f + fl * fl);
      light = add3(light, smul3(s, ldg3(L.sint, i)));
    }
  }
  return V3{fmaxf(light.x, L.amb), fmaxf(light.y, L.amb), fmaxf(light.z, L.amb)};
}

__device__ __forceinline__ void quad_ld(const float *a, int q, V3 v[4]) {
  const float4 *w = reinterpret_cast<const float4 *>(a) + 3 * (size_t)q;
  float4 w0 = w[0], w1 = w[1], w2 = w[2];
  v[0] = V3{w0.x, w0.y, w0.z}; v[1] = V3{w0.w, w1.x, w1.y};
  v[2] = V3{w1.z, w1.w, w2.x}; v[3] = V3{w2.y, w2.z, w2.w};
}

__device__ __forceinline__ void quad_st(float *a, int q, const V3 v[4]) {
  float4 *w = reinterpret_cast<float4 *>(a) + 3 * (size_t)q;
  w[0] = make_float4(v[0].x, v[0].y, v[0].z, v[1].x);
  w[1] = make_float4(v[1].y, v[1].z, v[2].x, v[2].y);
  w[2] = make_float4(v[2].z, v[3].x, v[3].y, v[3].z);
}

__device__ __forceinline__ V3 v_ld(const float *a, int v) { return V3{a[3 * (size_t)v], a[3 * (size_t)v + 1], a[3 * (size_t)v + 2]}; }
__device__ __forceinline__ void v_st(float *a, int v, V3 x) {
  a[3 * (size_t)v] = x.x; a[3 * (size_t)v + 1] = x.y; a[3 * (size_t)v + 2] = x.z;
}

// CLDraw.rotate (ROT) / CLDraw.translate over vertices [v0, v1)
template <bool ROT>
__global__ void k_vert_xform(float *__restrict__ xyz, float *__restrict__ vn, int v0, int v1, VertXform X) {
  int q1 = (v1 + 3) >> 2;
  for (int q = (v0 >> 2) + blockIdx.x * blockDim.x + threadIdx.x; q < q1; q += gridDim.x * blockDim.x) {
    int a = q << 2;
    if (a >= v0 && a + 4 <= v1) {
      V3 p[4], n[4];
      quad_ld(xyz, q, p);
      if (ROT) quad_ld(vn, q, n);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (ROT) xform_rotate(X, p[k], n[k]);
        else xform_translate(X, p[k]);
      }
      quad_st(xyz, q, p);
      if (ROT) quad_st(vn, q, n);
    } else {
      for (int v = max(a, v0); v < min(a + 4, v1); v++) {
        V3 p = v_ld(xyz, v), n;
        if (ROT) {
          n = v_ld(vn, v);
          xform_rotate(X, p, n);
          v_st(vn, v, n);
        } else {
          xform_translate(X, p);
        }
        v_st(xyz, v, p);
      }
    }
  }
}

// CLDraw.vertLight for one group's nv vertices, one vertex a thread (the
// light loops make it issue-bound, so the launch is one full wave of
// resident blocks striding over the vertices); positions are read only when
// point or spot lights exist.
__global__ void k_vert_light(const float *__restrict__ xyz, const float *__restrict__ vn, float *__restrict__ li,
                             int nv, VertLights L) {
  const bool pos = L.np + L.ns > 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    V3 x = pos ? ld3(xyz + 3 * (size_t)v) : V3{0.f, 0.f, 0.f};
    v_st(li, v, vert_light_one(L, x, ld3(vn + 3 * (size_t)v)));
  }
}

// ------------------------------------------------------------ setup

// one thread per triangle of every enabled group; lists hold global ids.
// `first`/`step` give the block's grid-stride over the triangles.
// One reservation per block and counter in a grid-stride loop that every
// thread of the block runs in step: warp w's totals v[k] (the same in all
// its lanes) become offsets out[k] into the counters ctr[idx[k]].  The
// counters are the same few addresses for the whole launch, so one
// atomicAdd per block instead of one per warp keeps them from serialising.
template <int K>
__device__ __forceinline__ void block_reserve(const uint32_t (&v)[K], const int (&idx)[K], uint32_t *ctr,
                                              uint32_t (&out)[K]) {
  __shared__ uint32_t part[32][K];
  __shared__ uint32_t base[K];
  const int w = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; k++) part[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x < K) {
    const int k = threadIdx.x;
    uint32_t run = 0;
    for (int i = 0; i < nw; i++) {
      uint32_t x = part[i][k];
      part[i][k] = run;
      run += x;
    }
    base[k] = run ? atomicAdd(&ctr[idx[k]], run) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) out[k] = base[k] + part[w][k];
}

// Writes the row-chunk work items of a block's triangles (or casters),
// sorted by their row count, longest first, into one region per kind and
// block (opaque items from the front of `items`, alpha-tested ones from the
// back).  A warp of the raster claims 32 consecutive items, so sorted items
// give it rows of about the same count, and fewer lanes idle while the
// longest item of the claim finishes.  The raster's results do not depend
// on the order.  Every thread of the block calls it in step; a thread adds
// the nch items of its list entry `pos` (chunk c has min(cl, rows - c cl)
// rows).
constexpr int LEN_BUCKETS = 16;
__device__ __forceinline__ void block_items(uint32_t *items, uint32_t cap_items, uint32_t *ctr, int ctr_o, int ctr_a,
                                            uint32_t pos, bool alpha, int rows, int cl, int nch) {
  __shared__ uint32_t hist[2][LEN_BUCKETS];
  __shared__ uint32_t bbase[2];
  for (int i = threadIdx.x; i < 2 * LEN_BUCKETS; i += blockDim.x) hist[i / LEN_BUCKETS][i % LEN_BUCKETS] = 0;
  __syncthreads();
  const int k = alpha ? 1 : 0;
  uint32_t rk[MAX_CHUNKS];
#pragma unroll
  for (int c = 0; c < MAX_CHUNKS; c++) {
    rk[c] = 0;
    if (c < nch) {
      int len = min(cl, rows - c * cl);
      rk[c] = atomicAdd(&hist[k][LEN_BUCKETS - 1 - min(len, LEN_BUCKETS - 1)], 1u);   // bucket 0: the longest
    }
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    uint32_t run = 0;
    for (int b = 0; b < LEN_BUCKETS; b++) {
      uint32_t x = hist[threadIdx.x][b];
      hist[threadIdx.x][b] = run;
      run += x;
    }
    bbase[threadIdx.x] = run ? atomicAdd(&ctr[threadIdx.x ? ctr_a : ctr_o], run) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < MAX_CHUNKS; c++) {
    if (c < nch) {
      int len = min(cl, rows - c * cl);
      uint32_t p = bbase[k] + hist[k][LEN_BUCKETS - 1 - min(len, LEN_BUCKETS - 1)] + rk[c];
      uint32_t item = (pos << CHUNK_BITS) | (uint32_t)c;
      if (!alpha) items[p] = item;
      else items[cap_items - 1 - p] = item;
    }
  }
  __syncthreads();   // the next call reuses hist and bbase
}

__device__ __forceinline__ void setup_phase(const DrawParams &P, const GroupDev *sg, int first, int step) {
  int lane = threadIdx.x & 31;
  for (int base = first; base < P.total_tris; base += step) {
    int t = base + threadIdx.x;
    int cls = 0;
    bool alpha = false;
    int iy0 = 0, iy1 = 0, iy2 = 0;
    if (t < P.total_tris) {
      int g = find_group(sg, P.ngroups, (uint32_t)t);
      const GroupDev &G = sg[g];
      if (G.enabled) {
        float sx[3], sy[3], sz[3];
        cls = project_persp(G, t - G.tri_base, P.view, sx, sy, sz);
        alpha = (G.flags & F_ALPHA) != 0;
        iy0 = f2i(sy[0]); iy1 = f2i(sy[1]); iy2 = f2i(sy[2]);
        if (P.mipc && cls == 2 && (G.flags & F_MIP)) {
          // a large triangle's mip level, once here instead of once per
          // shaded (winner, row) pair; it does not depend on the vertex order
          Attr<false> a[3];
          int ix[3], iy[3];
#pragma unroll
          for (int k = 0; k < 3; k++) {
            a[k] = a_load<false>(G, t - G.tri_base, k, sz[k]);
            ix[k] = f2i(sx[k]); iy[k] = f2i(sy[k]);
          }
          MipSel m = mip_setup<false>(a, sz, cls == 1, ix, iy, sx, sy, G.tex_size, G.mip_bias);
          P.mipc[t] = make_float2(m.fmip, (float)m.mip);
        }
      }
    }
    unsigned ms = __ballot_sync(FULL, cls == 1 && !alpha), ma = __ballot_sync(FULL, cls == 1 && alpha);
    unsigned ml = __ballot_sync(FULL, cls == 2);
    const uint32_t want[3] = {(uint32_t)__popc(ms), (uint32_t)__popc(ma), (uint32_t)__popc(ml)};
    const int idx[3] = {CTR_SMALL, CTR_SMALL_A, CTR_LARGE};
    uint32_t got[3];
    block_reserve<3>(want, idx, P.ctr, got);
    unsigned lt = (1u << lane) - 1;
    uint32_t pos = 0;
    if (cls == 1 && !alpha) { pos = got[0] + __popc(ms & lt); P.small_list[pos] = (uint32_t)t; }
    if (cls == 1 && alpha) { pos = got[1] + __popc(ma & lt); P.small_list[P.cap_list - 1 - pos] = (uint32_t)t; }
    if (cls == 2) P.large_list[got[2] + __popc(ml & lt)] = (uint32_t)t;
    // row chunks of the small triangles
    int rows = 0, cl = 1, nch = 0;
    if (cls == 1) {
      int y0 = min(iy0, min(iy1, iy2)), y3 = max(iy0, max(iy1, iy2));
      rows = small_rows(y0, y3);
      cl = chunk_len(rows, P.min_chunk);
      nch = (rows + cl - 1) / cl;
    }
    block_items(P.items, P.cap_list * MAX_CHUNKS, P.ctr, CTR_ITEMS, CTR_ITEMS_A, pos, alpha, rows, cl, nch);
  }
}

// 512 threads: block_items sorts the row-chunk items of 512 triangles at a
// time (small raster 242 -> 234 us on the 1080p frame against 256 threads,
// same setup time; the casters' setup is faster at 256).
constexpr int SETUP_THREADS = 512;
__global__ void __launch_bounds__(SETUP_THREADS) k_setup(DrawParams P) {
  __shared__ GroupDev sg[64];
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  setup_phase(P, sg, blockIdx.x * blockDim.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------------------ span queue

// One round of spans, one per lane, in structure-of-arrays form in shared
// memory; the warp then fills their pixels cooperatively.  d = cx1 - cx2 and
// rd = its reciprocal (or 0) are per span, so a pixel's t costs one multiply
// and two fused multiply-adds instead of a division.
template <bool ALPHA>
struct VisQ {
  float4 a[32];                  // cx2, d, 1/d (0: divide), cz1
  float4 b[32];                  // cz2, pixel address - first pixel number, x - first pixel number, order
  float4 c[ALPHA ? 32 : 1];      // u1, u2 (uv / z at the span's ends)
  int g[ALPHA ? 32 : 1];
  int r2l[32];                   // rank among the round's non-empty spans -> span
};

// Pixels of a round are numbered 0..total-1 in span (lane) order.  Returns
// the total, sets `pre` to this lane's first pixel number and fills the
// rank -> span table of the non-empty spans.
__device__ __forceinline__ int fill_prepare(int cnt, int lane, int *r2l, int &pre) {
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += v;
  }
  pre = incl - cnt;
  unsigned ne = __ballot_sync(FULL, cnt > 0);
  if (cnt > 0) r2l[__popc(ne & ((1u << lane) - 1u))] = lane;
  return __shfl_sync(FULL, incl, 31);
}

// Calls pix(span, p) for every pixel p < total, lane j taking pixels j,
// j + 32, ...  A pixel's span is the last non-empty span starting at or
// before it: its rank = (non-empty spans starting before the window, one
// ballot) + (starts inside the window up to this lane, from one OR-reduction
// of the start bits) - 1.
template <class F>
__device__ __forceinline__ void fill_windows(int total, int cnt, int pre, int lane, const int *r2l, F &&pix) {
  const unsigned upto = 0xffffffffu >> (31 - lane);
  for (int base = 0; base < total; base += 32) {
    int rel = pre - base;
    unsigned bit = (cnt > 0 && (unsigned)rel < 32u) ? (1u << rel) : 0u;
    unsigned starts = __reduce_or_sync(FULL, bit);
    int before = __popc(__ballot_sync(FULL, cnt > 0 && rel < 0));
    int p = base + lane;
    if (p < total) pix(r2l[before + __popc(starts & upto) - 1], p);
  }
}

// fill_windows for a pixel function in two stages: first(span, p) issues
// the pixel's dependent load and returns a state, second(state) consumes
// it.  Window k's second stage runs after window k + 1's first, so the
// load's latency overlaps the next window's lookup and arithmetic.
template <class St, class F1, class F2>
__device__ __forceinline__ void fill_windows2(int total, int cnt, int pre, int lane, const int *r2l, F1 &&first,
                                              F2 &&second) {
  const unsigned upto = 0xffffffffu >> (31 - lane);
  St cur;
  bool have = false;
  for (int base = 0; base < total; base += 32) {
    int rel = pre - base;
    unsigned bit = (cnt > 0 && (unsigned)rel < 32u) ? (1u << rel) : 0u;
    unsigned starts = __reduce_or_sync(FULL, bit);
    int before = __popc(__ballot_sync(FULL, cnt > 0 && rel < 0));
    int p = base + lane;
    St nxt;
    bool hn = p < total;
    if (hn) nxt = first(r2l[before + __popc(starts & upto) - 1], p);
    if (have) second(cur);
    cur = nxt;
    have = hn;
  }
  if (have) second(cur);
}

// One round of a span queue: numbering, the record's second half written
// with its address and x made relative to the span's first pixel number
// (the emitter keeps `pb` in registers until the numbering is known), then
// the pixel-parallel fill.
template <class Q, class F>
__device__ __forceinline__ void fill_round(Q &q, int lane, int cnt, float4 pb, F &&pix);
template <class St, class Q, class F1, class F2>
__device__ __forceinline__ void fill_round2(Q &q, int lane, int cnt, float4 pb, F1 &&first, F2 &&second) {
  int pre;
  int total = fill_prepare(cnt, lane, q.r2l, pre);
  if (total == 0) return;
  if (cnt) {
    pb.y = __int_as_float(__float_as_int(pb.y) - pre);
    pb.z = __int_as_float(__float_as_int(pb.z) - pre);
    q.b[lane] = pb;
  }
  __syncwarp();
  fill_windows2<St>(total, cnt, pre, lane, q.r2l, first, second);
  __syncwarp();
}
template <class Q, class F>
__device__ __forceinline__ void fill_round(Q &q, int lane, int cnt, float4 pb, F &&pix) {
  int pre;
  int total = fill_prepare(cnt, lane, q.r2l, pre);
  if (total == 0) return;
  if (cnt) {
    pb.y = __int_as_float(__float_as_int(pb.y) - pre);
    pb.z = __int_as_float(__float_as_int(pb.z) - pre);
    q.b[lane] = pb;
  }
  __syncwarp();
  fill_windows(total, cnt, pre, lane, q.r2l, pix);
  __syncwarp();
}

// Writes lane's span record: row offset cyw, first pixel lo, ends cx1 / cx2.
// Its second half goes to `pb`, which fill_round stores; a span that must be
// drawn by its own lane (span_queue_form: returns false) is stored whole.
template <bool ALPHA>
__device__ __forceinline__ bool vis_put(VisQ<ALPHA> &q, int lane, int cyw, int lo, uint32_t ord, float cx1, float cx2,
                                        float cz1, float cz2, V2 cu1, V2 cu2, int g, float4 &pb) {
  float qx, qd, qy;
  bool ok = span_queue_form(cx2, cx1 - cx2, lo, qx, qd, qy);
  q.a[lane] = make_float4(qx, qd, qy, cz1);
  pb = make_float4(cz2, __int_as_float(cyw + lo), __int_as_float(lo), __uint_as_float(ord));
  if (!ok) q.b[lane] = pb;
  if (ALPHA) {
    q.c[lane] = make_float4(cu1.x, cu1.y, cu2.x, cu2.y);
    q.g[lane] = g;
  }
  return ok;
}

// Per-fragment visibility: alpha test (av_draw_alpha.c:80-97) then the
// packed depth/order atomicMin.
// Pixel number p of span s (x = p + b.z, address = p + b.y).  The reciprocal
// of the interpolated 1/z is correctly rounded (__frcp_rn), i.e. 1.0f / x.
// DIV: a span its own lane draws, with the true division.
template <bool ALPHA, bool DIV = false>
__device__ __forceinline__ void vis_pixel(const DrawParams &P, const GroupDev *sg, const VisQ<ALPHA> &q, int s, int p) {
  const float4 a = q.a[s], b = q.b[s];
  float n = (float)(p + __float_as_int(b.z)) - a.x;
  float t = DIV ? clamp_t(n / a.y) : span_t(n, a.y, a.z);
  float tz = __frcp_rn((1 - t) * b.x + t * a.w);
  if (tz != tz) return;
  if (ALPHA) {
    const float4 c = q.c[s];
    const GroupDev &G = sg[q.g[s]];
    float omt = 1 - t;
    V2 uvi{omt * c.z + t * c.x, omt * c.w + t * c.y};
    Taps tp = make_taps(uvi, tz, G.alen, 0);
    if (!(bilerp_quad(tp, G.aquad) > 0.5f)) return;
  }
  atomicMin((unsigned long long *)&P.keys[(size_t)(p + __float_as_int(b.y))],
            (unsigned long long)frag_key(tz, __float_as_uint(b.w)));
}

// vis_pixel<true> in two stages for fill_windows2: the first stage takes
// the depth, the alpha footprint's weights and the order key, and issues
// the load of the packed mask quad; the second tests the bilinear alpha
// and resolves the visibility word.
struct AlphaFrag {
  unsigned long long key;
  uint32_t addr;
  unsigned m;          // the packed 2 x 2 mask quad (loaded in stage one)
  float r1, r2;        // bilinear fractions
  bool live;
};
__device__ __forceinline__ AlphaFrag vis_alpha_first(const DrawParams &P, const GroupDev *sg, const VisQ<true> &q,
                                                     int s, int p) {
  AlphaFrag f;
  const float4 a = q.a[s], b = q.b[s];
  float n = (float)(p + __float_as_int(b.z)) - a.x;
  float t = span_t(n, a.y, a.z);
  float tz = __frcp_rn((1 - t) * b.x + t * a.w);
  f.live = tz == tz;
  const float4 c = q.c[s];
  const GroupDev &G = sg[q.g[s]];
  float omt = 1 - t;
  V2 uvi{omt * c.z + t * c.x, omt * c.w + t * c.y};
  Taps tp = make_taps(uvi, tz, G.alen, 0);
  f.m = f.live ? (unsigned)__ldg(G.aquad + tp.tex) : 0u;
  f.r1 = tp.texr1;
  f.r2 = tp.texr2;
  f.key = frag_key(tz, __float_as_uint(b.w));
  f.addr = (uint32_t)(p + __float_as_int(b.y));
  return f;
}
__device__ __forceinline__ void vis_alpha_second(const DrawParams &P, const AlphaFrag &f) {
  if (!f.live) return;
  float i1 = 1 - f.r1, i2 = 1 - f.r2;
  float ca = i1 * i2 * (float)(f.m & 1) + f.r1 * i2 * (float)((f.m >> 1) & 1) + i1 * f.r2 * (float)((f.m >> 2) & 1) +
             f.r1 * f.r2 * (float)((f.m >> 3) & 1);
  if (!(ca > 0.5f)) return;
  atomicMin((unsigned long long *)&P.keys[f.addr], f.key);
}

// The lane's own span record, drawn by the lane alone with the true division.
template <bool ALPHA>
__device__ __forceinline__ void vis_serial(const DrawParams &P, const GroupDev *sg, const VisQ<ALPHA> &q, int lane,
                                           int cnt) {
  for (int j = 0; j < cnt; j++) vis_pixel<ALPHA, true>(P, sg, q, lane, j);
}

// PIPE: alpha-tested fragments through the two-stage pipeline (the small
// triangles' raster: 407 -> 390 us in the 1080p frame; the tiled raster,
// whose spans are at most 16 pixels, was 3 us slower with it).
template <bool ALPHA, bool PIPE = false>
__device__ __forceinline__ void vis_fill(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane, int cnt,
                                         float4 pb) {
  if constexpr (ALPHA && PIPE)
    fill_round2<AlphaFrag>(q, lane, cnt, pb, [&](int s, int p) { return vis_alpha_first(P, sg, q, s, p); },
                           [&](const AlphaFrag &f) { vis_alpha_second(P, f); });
  else
    fill_round(q, lane, cnt, pb, [&](int s, int p) { vis_pixel<ALPHA>(P, sg, q, s, p); });
}

// ------------------------------------------------------------ small triangles

template <bool ALPHA>
struct SmallLane {
  int g;
  float4 pb = make_float4(0.f, 0.f, 0.f, 0.f);   // second half of the last span record (fill_round stores it)
  uint32_t gtri;
  int x1, x2, x3, y1, y2, y3;
  float z1, z2, z3, x4, z4;
  V2 uv1, uv2, uv3, uv4;
  int half, cy;
  float s1, s2, sz1, sz2, cx1, cx2, cz1, cz2;
  V2 su1, su2, cu1, cu2;

  __device__ __forceinline__ void start_half0() {
    half = 0;
    float yd = 1.0f / (float)(y2 - y1);
    s1 = (float)(x2 - x1) * yd;
    s2 = (x4 - (float)x1) * yd;
    sz1 = (z2 - z1) * yd;
    sz2 = (z4 - z1) * yd;
    cx1 = cx2 = (float)x1;
    cz1 = cz2 = z1;
    if (ALPHA) {
      su1 = mul2(sub2(uv2, uv1), yd);
      su2 = mul2(sub2(uv4, uv1), yd);
      cu1 = cu2 = uv1;
    }
    if (s1 < s2) {
      float t = s1; s1 = s2; s2 = t;
      t = sz1; sz1 = sz2; sz2 = t;
      if (ALPHA) { V2 tv = su1; su1 = su2; su2 = tv; }
    }
    cy = y1;
  }
  // The second half's slopes are computed at set-up (see ShadowLane), so
  // that reaching the middle row during the walk costs a few copies.
  float hs1, hs2, hsz1, hsz2;
  V2 hsu1, hsu2;
  __device__ __forceinline__ void half1_slopes() {
    float yd = 1.0f / (float)(y3 - y2);
    hs1 = (float)(x3 - x2) * yd;
    hs2 = ((float)x3 - x4) * yd;
    hsz1 = (z3 - z2) * yd;
    hsz2 = (z3 - z4) * yd;
    if (ALPHA) {
      hsu1 = mul2(neg2(sub2(uv2, uv3)), yd);
      hsu2 = mul2(neg2(sub2(uv4, uv3)), yd);
    }
    if (hs1 < hs2) {
      float t = hs1; hs1 = hs2; hs2 = t;
      t = hsz1; hsz1 = hsz2; hsz2 = t;
      if (ALPHA) { V2 tv = hsu1; hsu1 = hsu2; hsu2 = tv; }
    }
  }
  __device__ __forceinline__ void start_half1() {
    half = 1;
    s1 = hs1; s2 = hs2; sz1 = hsz1; sz2 = hsz2;
    cx1 = cx2 = (float)x3;
    cz1 = cz2 = z3;
    if (ALPHA) {
      su1 = hsu1; su2 = hsu2;
      cu1 = cu2 = uv3;
    }
    cy = y3;
  }

  int left;   // rows left in this lane's chunk

  // advances one row without drawing (the replay up to a chunk's first row)
  __device__ __forceinline__ void skip_row() {
    if (half == 0) {
      cx1 += s1; cx2 += s2; cz1 += sz1; cz2 += sz2;
      if (ALPHA) { cu1 = add2(cu1, su1); cu2 = add2(cu2, su2); }
      cy++;
      if (cy > y2) start_half1();
    } else {
      cx1 -= s1; cx2 -= s2; cz1 -= sz1; cz2 -= sz2;
      if (ALPHA) { cu1 = sub2(cu1, su1); cu2 = sub2(cu2, su2); }
      cy--;
    }
  }

  __device__ __forceinline__ void init_chunk(const DrawParams &P, const GroupDev *sg, uint32_t t, int chunk) {
    init(P, sg, t);
    int rows = small_rows(y1, y3);
    int cl = chunk_len(rows, P.min_chunk);
    int first = chunk * cl;
    left = min(cl, rows - first);
    for (int r = 0; r < first; r++) skip_row();
  }

  __device__ __forceinline__ void init(const DrawParams &P, const GroupDev *sg, uint32_t t) {
    gtri = t;
    g = find_group(sg, P.ngroups, t);
    const GroupDev &G = sg[g];
    int tri = (int)(t - G.tri_base);
    float sx[3], sy[3], sz[3];
    project_persp(G, tri, P.view, sx, sy, sz);
    int ix[3], iy[3];
    float z[3];
    Attr<false> a[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      ix[k] = f2i(sx[k]); iy[k] = f2i(sy[k]); z[k] = sz[k];
      if (ALPHA) a[k] = a_load<false>(G, tri, k, sz[k]);
    }
#define SW(i, j) { int ti = iy[i]; iy[i] = iy[j]; iy[j] = ti; ti = ix[i]; ix[i] = ix[j]; ix[j] = ti; \
                   float tf = z[i]; z[i] = z[j]; z[j] = tf; if (ALPHA) { Attr<false> ta = a[i]; a[i] = a[j]; a[j] = ta; } }
    if (iy[0] > iy[1]) SW(0, 1);
    if (iy[1] > iy[2]) SW(1, 2);
    if (iy[0] > iy[1]) SW(0, 1);
#undef SW
    x1 = ix[0]; x2 = ix[1]; x3 = ix[2]; y1 = iy[0]; y2 = iy[1]; y3 = iy[2];
    z1 = z[0]; z2 = z[1]; z3 = z[2];
    float yd = (float)(y2 - y1) / (float)(y3 - y1);
    x4 = (float)x1 + yd * (float)(x3 - x1);
    z4 = z1 + yd * (z3 - z1);
    if (ALPHA) {
      uv4 = add2(a[0].uv, smul2(yd, sub2(a[2].uv, a[0].uv)));
      if (G.flags & F_MIP) mip_setup<false>(a, z, true, ix, iy, nullptr, nullptr, G.tex_size, G.mip_bias);
      uv1 = a[0].uv; uv2 = a[1].uv; uv3 = a[2].uv;
    }
    half1_slopes();
    start_half0();
  }

  // writes the current row's span into q[lane], advances; returns the span's
  // pixel count and sets `live` false after the last row
  __device__ __forceinline__ int emit(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane, bool &live) {
    int lo = 0, cnt = 0;
    if (cy >= 0 && cy < P.view.h) {
      if (half == 0) span_clip(f2i(cx2), cx1, P.view.w, lo, cnt);
      else span_clip(f2i(cx1), cx2, P.view.w, lo, cnt);
    }
    if (cnt && !vis_put<ALPHA>(q, lane, cy * P.view.w, lo, make_order(0, gtri, half), cx1, cx2, cz1, cz2, cu1, cu2,
                               g, pb)) {
      vis_serial<ALPHA>(P, sg, q, lane, cnt);
      cnt = 0;
    }
    skip_row();
    live = --left > 0;
    return cnt;
  }
};

template <bool ALPHA>
__device__ __forceinline__ void raster_small_loop(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane) {
  uint32_t n = P.ctr[ALPHA ? CTR_ITEMS_A : CTR_ITEMS];
  uint32_t cap_items = P.cap_list * MAX_CHUNKS;
  const uint32_t per = ALPHA ? claim_size(n, (uint32_t)P.claim_k) : 32u;
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&P.ctr[ALPHA ? CTR_WORK_SMALL_A : CTR_WORK_SMALL], per);
    base = __shfl_sync(FULL, base, 0);
    if (base >= n) break;
    SmallLane<ALPHA> L;
    bool live = (uint32_t)lane < per && base + lane < n;
    if (live) {
      uint32_t idx = base + lane;
      uint32_t item = P.items[ALPHA ? cap_items - 1 - idx : idx];
      uint32_t pos = item >> CHUNK_BITS;
      L.init_chunk(P, sg, P.small_list[ALPHA ? P.cap_list - 1 - pos : pos], (int)(item & (MAX_CHUNKS - 1)));
    }
    for (int round = 0; __any_sync(FULL, live); round++) {
      if (round == LOOP_LIMIT) {
        if (lane == 0) atomicOr(&P.ctr[CTR_LIMIT], 1u);
        break;
      }
      int cnt = 0;
      if (live) cnt = L.emit(P, sg, q, lane, live);
      vis_fill<ALPHA, true>(P, sg, q, lane, cnt, L.pb);
    }
  }
}

template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 6 : 8) k_raster_small(DrawParams P) {
  __shared__ GroupDev sg[64];
  __shared__ VisQ<ALPHA> qs[4];
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  raster_small_loop<ALPHA>(P, sg, qs[threadIdx.x >> 5], threadIdx.x & 31);
}

// ------------------------------------------------------------ coarse binning

// coarse.c:17-125 in tile units; calls emit(tile) for every bin entry
template <class F>
__device__ __forceinline__ void coarse_walk(const float sx[3], const float sy[3], int wc, int hc, F emit) {
  float x1 = sx[0] / 16.f - 0.5f, x2 = sx[1] / 16.f - 0.5f, x3 = sx[2] / 16.f - 0.5f;
  float y1 = sy[0] / 16.f - 0.5f, y2 = sy[1] / 16.f - 0.5f, y3 = sy[2] / 16.f - 0.5f;
  float t;
  if (y1 > y2) { t = y1; y1 = y2; y2 = t; t = x1; x1 = x2; x2 = t; }
  if (y2 > y3) { t = y2; y2 = y3; y3 = t; t = x2; x2 = x3; x3 = t; }
  if (y1 > y2) { t = y1; y1 = y2; y2 = t; t = x1; x1 = x2; x2 = t; }
  float x4 = (x1 + ((y2 - y1) / (y3 - y1)) * (x3 - x1));
  float y4 = y2;
  float s1 = (x2 - x1) / (y2 - y1);
  float s2 = (x4 - x1) / (y4 - y1);
  float cx1 = x1, cx2 = x1;
  if (s1 < s2) { t = s1; s1 = s2; s2 = t; }
  float sbias = 1.f + floorf(y1) - y1;
  float wcm1 = (float)wc - 1;
  int guard = 0;
  if (y1 != y2) {
    for (int cy = f2i(floorf(y1)); (float)cy <= ceilf(y2) && guard < LOOP_LIMIT; cy++, guard++) {
      float mx1 = cx1 + sbias * s1;
      if (s1 < 0) mx1 -= s1;
      float mx2 = cx2 + sbias * s2;
      if (s2 > 0) mx2 -= s2;
      mx1 = fminf(mx1, wcm1);
      mx2 = fmaxf(mx2, 0.f);
      if (cy >= 0 && cy < hc) {
        int a1 = f2i(floorf(mx2));
        float hb = ceilf(mx1);
        for (int ax = a1; (float)ax <= hb && ax < wc; ax++) emit(wc * cy + ax);
      }
      cx1 += s1;
      cx2 += s2;
    }
  }
  s1 = (x3 - x2) / (y3 - y2);
  s2 = (x3 - x4) / (y3 - y4);
  cx1 = x3; cx2 = x3;
  if (s1 < s2) { t = s1; s1 = s2; s2 = t; }
  sbias = y3 - floorf(y3);
  if (y2 != y3) {
    for (int cy = f2i(ceilf(y3)); (float)cy >= floorf(y2) && guard < 2 * LOOP_LIMIT; cy--, guard++) {
      float mx1 = cx1 - sbias * s1;
      if (s1 < 0) mx1 += s1;
      float mx2 = cx2 - sbias * s2;
      if (s2 > 0) mx2 += s2;
      mx2 = fminf(mx2, wcm1);
      mx1 = fmaxf(mx1, 0.f);
      if (cy >= 0 && cy < hc) {
        int a1 = f2i(floorf(mx1));
        float hb = ceilf(mx2);
        for (int ax = a1; (float)ax <= hb && ax < wc; ax++) emit(wc * cy + ax);
      }
      cx1 -= s1;
      cx2 -= s2;
    }
  }
}

// Opaque units fill the queue from the front, alpha-tested ones from the back.
__device__ __forceinline__ void coarse_loop(const DrawParams &P, const GroupDev *sg, int lane) {
  uint32_t n = P.ctr[CTR_LARGE];
  int wc = P.view.w / TILE, hc = P.view.h / TILE;
  const uint32_t per = claim_size(n, P.claim_k > 0 ? 1u : 0u);
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&P.ctr[CTR_WORK_LARGE], per);
    base = __shfl_sync(FULL, base, 0);
    if (base >= n) break;
    bool live = (uint32_t)lane < per && base + lane < n;
    float sx[3], sy[3], sz[3];
    uint32_t gt = 0;
    int cnt = 0;
    bool alpha = false;
    if (live) {
      gt = P.large_list[base + lane];
      const GroupDev &G = sg[find_group(sg, P.ngroups, gt)];
      alpha = (G.flags & F_ALPHA) != 0;
      project_persp(G, (int)(gt - G.tri_base), P.view, sx, sy, sz);
      coarse_walk(sx, sy, wc, hc, [&](int) { cnt++; });
    }
    int co = alpha ? 0 : cnt, ca = alpha ? cnt : 0;
    int io = co, ia = ca;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(FULL, io, o);
      int va = __shfl_up_sync(FULL, ia, o);
      if (lane >= o) { io += v; ia += va; }
    }
    uint32_t to = (uint32_t)__shfl_sync(FULL, io, 31), ta = (uint32_t)__shfl_sync(FULL, ia, 31);
    // Capacity is reserved for both kinds together, so the opaque units
    // (growing from the front) and the alpha units (from the back) never
    // meet; after an overflow the fallback kernel draws every large triangle.
    uint32_t oo = 0, oa = 0, fits = 1;
    if (lane == 31 && to + ta) {
      uint32_t r = atomicAdd(&P.ctr[CTR_UNITS_RESERVED], to + ta);
      if ((uint64_t)r + to + ta > (uint64_t)P.cap_units) {
        fits = 0;
        atomicOr(&P.ctr[CTR_OVERFLOW], 1u);
      } else {
        if (to) oo = atomicAdd(&P.ctr[CTR_UNITS], to);
        if (ta) oa = atomicAdd(&P.ctr[CTR_UNITS_A], ta);
      }
    }
    fits = __shfl_sync(FULL, fits, 31);
    oo = __shfl_sync(FULL, oo, 31) + (uint32_t)(io - co);
    oa = __shfl_sync(FULL, oa, 31) + (uint32_t)(ia - ca);
    if (live && cnt && fits) {
      {
        int k = 0;
        if (!alpha) {
          uint2 *u = P.units + oo;
          coarse_walk(sx, sy, wc, hc, [&](int tile) { u[k++] = make_uint2(gt, (uint32_t)tile); });
        } else {
          uint2 *u = P.units + (P.cap_units - 1 - oa);
          coarse_walk(sx, sy, wc, hc, [&](int tile) { *(u - k) = make_uint2(gt, (uint32_t)tile); k++; });
        }
      }
    }
  }
}

__global__ void __launch_bounds__(128) k_coarse(DrawParams P) {
  __shared__ GroupDev sg[64];
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  coarse_loop(P, sg, threadIdx.x & 31);
}

// ------------------------------------------------------------ tiled (large) raster

template <bool ALPHA>
struct TileLane {
  int g;
  float4 pb = make_float4(0.f, 0.f, 0.f, 0.f);   // second half of the last span record (fill_round stores it)
  uint32_t gtri;
  float x1, x2, x3, y1, y2, y3, z1, z2, z3, x4, z4;
  V2 uv1, uv2, uv3, uv4;
  float xMin, xMax, yMin, yMax;
  int half, cy;
  bool live_half;
  float ybound;
  float s1, s2, sz1, sz2, cx1, cx2, cz1, cz2;
  V2 su1, su2, cu1, cu2;

  __device__ __forceinline__ void start_half0() {
    half = 0;
    float yd = 1.0f / (y2 - y1);
    s1 = (x2 - x1) * yd;
    s2 = (x4 - x1) * yd;
    sz1 = (z2 - z1) * yd;
    sz2 = (z4 - z1) * yd;
    if (ALPHA) { su1 = mul2(sub2(uv2, uv1), yd); su2 = mul2(sub2(uv4, uv1), yd); }
    if (s1 < s2) {
      float t = s1; s1 = s2; s2 = t;
      t = sz1; sz1 = sz2; sz2 = t;
      if (ALPHA) { V2 tv = su1; su1 = su2; su2 = tv; }
    }
    cy = f2i(clampf_(y1, yMin, yMax));
    float dy = (float)cy - y1;
    cx1 = x1 + dy * s1; cx2 = x1 + dy * s2;
    cz1 = z1 + dy * sz1; cz2 = z1 + dy * sz2;
    if (ALPHA) { cu1 = add2(uv1, smul2(dy, su1)); cu2 = add2(uv1, smul2(dy, su2)); }
    ybound = clampf_(y2, yMin, yMax);
    live_half = (y2 > yMin) && ((float)cy <= ybound);
  }
  // The second half's slopes are computed at set-up (see ShadowLane), so
  // that the lanes reaching the middle row during the walk do less while
  // the others wait.
  float hs1, hs2, hsz1, hsz2;
  V2 hsu1, hsu2;
  __device__ __forceinline__ void half1_slopes() {
    float yd = 1.0f / (y3 - y2);
    hs1 = (x3 - x2) * yd;
    hs2 = (x3 - x4) * yd;
    hsz1 = (z3 - z2) * yd;
    hsz2 = (z3 - z4) * yd;
    if (ALPHA) { hsu1 = mul2(neg2(sub2(uv2, uv3)), yd); hsu2 = mul2(neg2(sub2(uv4, uv3)), yd); }
    if (hs1 < hs2) {
      float t = hs1; hs1 = hs2; hs2 = t;
      t = hsz1; hsz1 = hsz2; hsz2 = t;
      if (ALPHA) { V2 tv = hsu1; hsu1 = hsu2; hsu2 = tv; }
    }
  }
  __device__ __forceinline__ void start_half1() {
    half = 1;
    s1 = hs1; s2 = hs2; sz1 = hsz1; sz2 = hsz2;
    if (ALPHA) { su1 = hsu1; su2 = hsu2; }
    cy = f2i(clampf_(y3, yMin, yMax));
    float dy = (float)cy - y3;
    cx1 = x3 + dy * s1; cx2 = x3 + dy * s2;
    cz1 = z3 + dy * sz1; cz2 = z3 + dy * sz2;
    if (ALPHA) { cu1 = add2(uv3, smul2(dy, su1)); cu2 = add2(uv3, smul2(dy, su2)); }
    ybound = clampf_(y2, yMin, yMax);
    live_half = (y2 < yMax) && ((float)cy >= ybound);
  }

  // returns false if the unit has no rows at all
  __device__ __forceinline__ bool init(const DrawParams &P, const GroupDev *sg, uint2 unit) {
    gtri = unit.x;
    int bx = (int)unit.y;
    g = find_group(sg, P.ngroups, gtri);
    const GroupDev &G = sg[g];
    int tri = (int)(gtri - G.tri_base);
    float sx[3], sy[3], sz[3];
    project_persp(G, tri, P.view, sx, sy, sz);
    Attr<false> a[3];
    float x[3], y[3], z[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      x[k] = sx[k]; y[k] = sy[k]; z[k] = sz[k];
      if (ALPHA) a[k] = a_load<false>(G, tri, k, sz[k]);
    }
#define SW(i, j) { float tf = y[i]; y[i] = y[j]; y[j] = tf; tf = x[i]; x[i] = x[j]; x[j] = tf; \
                   tf = z[i]; z[i] = z[j]; z[j] = tf; if (ALPHA) { Attr<false> ta = a[i]; a[i] = a[j]; a[j] = ta; } }
    if (y[0] > y[1]) SW(0, 1);
    if (y[1] > y[2]) SW(1, 2);
    if (y[0] > y[1]) SW(0, 1);
#undef SW
    x1 = x[0]; x2 = x[1]; x3 = x[2]; y1 = y[0]; y2 = y[1]; y3 = y[2];
    z1 = z[0]; z2 = z[1]; z3 = z[2];
    float yd = (y2 - y1) / (y3 - y1);
    x4 = x1 + yd * (x3 - x1);
    z4 = z1 + yd * (z3 - z1);
    if (ALPHA) {
      uv4 = add2(a[0].uv, smul2(yd, sub2(a[2].uv, a[0].uv)));
      if (G.flags & F_MIP) mip_setup<false>(a, z, false, nullptr, nullptr, x, y, G.tex_size, G.mip_bias);
      uv1 = a[0].uv; uv2 = a[1].uv; uv3 = a[2].uv;
    }
    int wc = P.view.w / TILE;
    int tileX = bx % wc;
    int tileY = f2i((float)bx / ((float)P.view.w / 16.f));
    xMin = (float)tileX * 16.f;
    xMax = ((float)tileX + 1.f) * 16.f - 1.f;
    yMin = (float)tileY * 16.f;
    yMax = ((float)tileY + 1.f) * 16.f - 1.f;
    half1_slopes();
    start_half0();
    if (!live_half) start_half1();
    return live_half;
  }

  // queues the row's span, or draws it with the lane alone (span_queue_form);
  // returns the pixels queued
  __device__ __forceinline__ int put(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane, int lo,
                                     int cnt) {
    if (vis_put<ALPHA>(q, lane, cy * P.view.w, lo, make_order(1, gtri, half), cx1, cx2, cz1, cz2, cu1, cu2, g, pb))
      return cnt;
    vis_serial<ALPHA>(P, sg, q, lane, cnt);
    return 0;
  }

  __device__ __forceinline__ int emit(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane, bool &live) {
    int cnt = 0;
    if (half == 0) {
      if (cx2 < xMax && cx1 > xMin) {
        int lo = f2i(clampf_(cx2, xMin, xMax));
        int hi = f2i(floorf(clampf_(cx1, xMin, xMax)));
        cnt = hi >= lo ? hi - lo + 1 : 0;
        if (cnt) cnt = put(P, sg, q, lane, lo, cnt);
      }
      cx1 += s1; cx2 += s2; cz1 += sz1; cz2 += sz2;
      if (ALPHA) { cu1 = add2(cu1, su1); cu2 = add2(cu2, su2); }
      cy++;
      if ((float)cy > ybound) {
        start_half1();
        live = live_half;
      }
      return cnt;
    }
    if (cx1 < xMax && cx2 > xMin) {
      int lo = f2i(clampf_(cx1, xMin, xMax));
      int hi = f2i(floorf(clampf_(cx2, xMin, xMax)));
      cnt = hi >= lo ? hi - lo + 1 : 0;
      if (cnt) cnt = put(P, sg, q, lane, lo, cnt);
    }
    cx1 -= s1; cx2 -= s2; cz1 -= sz1; cz2 -= sz2;
    if (ALPHA) { cu1 = sub2(cu1, su1); cu2 = sub2(cu2, su2); }
    cy--;
    live = (float)cy >= ybound;
    return cnt;
  }
};

template <bool ALPHA>
__device__ __forceinline__ void raster_tiled_loop(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane) {
  if (P.ctr[CTR_OVERFLOW]) return;
  uint32_t n = P.ctr[ALPHA ? CTR_UNITS_A : CTR_UNITS];
  const uint32_t per = ALPHA ? claim_size(n, (uint32_t)P.claim_k) : 32u;
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&P.ctr[ALPHA ? CTR_WORK_UNITS_A : CTR_WORK_UNITS], per);
    base = __shfl_sync(FULL, base, 0);
    if (base >= n) break;
    TileLane<ALPHA> L;
    bool live = false;
    if ((uint32_t)lane < per && base + lane < n) {
      uint32_t idx = base + lane;
      live = L.init(P, sg, P.units[ALPHA ? P.cap_units - 1 - idx : idx]);
    }
    for (int round = 0; __any_sync(FULL, live); round++) {
      if (round == LOOP_LIMIT) {
        if (lane == 0) atomicOr(&P.ctr[CTR_LIMIT], 1u);
        break;
      }
      int cnt = 0;
      if (live) cnt = L.emit(P, sg, q, lane, live);
      vis_fill<ALPHA>(P, sg, q, lane, cnt, L.pb);
    }
  }
}

template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 6 : 8) k_raster_tiled(DrawParams P) {
  __shared__ GroupDev sg[64];
  __shared__ VisQ<ALPHA> qs[4];
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  raster_tiled_loop<ALPHA>(P, sg, qs[threadIdx.x >> 5], threadIdx.x & 31);
}

// Tile-unit queue overflow: every large triangle is rasterized here instead,
// one triangle per warp, its coarse tiles dealt round-robin to the lanes and
// each lane filling its tiles on its own (slow, same fragments).
template <bool ALPHA>
__device__ __forceinline__ void fallback_unit(const DrawParams &P, const GroupDev *sg, VisQ<ALPHA> &q, int lane,
                                              uint32_t gt, int tile) {
  TileLane<ALPHA> L;
  bool live = L.init(P, sg, make_uint2(gt, (uint32_t)tile));
  for (int round = 0; live && round < LOOP_LIMIT; round++) {
    int cnt = L.emit(P, sg, q, lane, live);   // the lane's own record: pixel j is x = lo + j
    if (cnt) q.b[lane] = L.pb;
    for (int j = 0; j < cnt; j++) vis_pixel<ALPHA>(P, sg, q, lane, j);
  }
}

__device__ __forceinline__ void fallback_loop(const DrawParams &P, const GroupDev *sg, VisQ<false> &qo, VisQ<true> &qa,
                                              int lane, int gw, int nw) {
  if (!P.ctr[CTR_OVERFLOW]) return;
  uint32_t n = P.ctr[CTR_LARGE];
  int wc = P.view.w / TILE, hc = P.view.h / TILE;
  for (uint32_t i = gw; i < n; i += nw) {
    uint32_t gt = P.large_list[i];
    const GroupDev &G = sg[find_group(sg, P.ngroups, gt)];
    bool alpha = (G.flags & F_ALPHA) != 0;
    float sx[3], sy[3], sz[3];
    project_persp(G, (int)(gt - G.tri_base), P.view, sx, sy, sz);
    int k = 0;
    coarse_walk(sx, sy, wc, hc, [&](int tile) {
      if ((k++ & 31) != lane) return;
      if (alpha) fallback_unit<true>(P, sg, qa, lane, gt, tile);
      else fallback_unit<false>(P, sg, qo, lane, gt, tile);
    });
  }
}

__global__ void __launch_bounds__(128) k_raster_tiled_fallback(DrawParams P) {
  __shared__ GroupDev sg[64];
  __shared__ VisQ<false> qo[4];
  __shared__ VisQ<true> qa[4];
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  int w = threadIdx.x >> 5;
  fallback_loop(P, sg, qo[w], qa[w], threadIdx.x & 31, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                (gridDim.x * blockDim.x) >> 5);
}

// ------------------------------------------------------------ shade

// double-cascade 5-tap count: av_alpha_max.c:53-84 (shDist 2)
__device__ __forceinline__ float shadow_light(const DrawParams &P, V3 p) {
  int shadow = 0;
  for (int k = 0; k < P.nsh; k++) {
    const ShadowDev &s = P.sh[k];
    int wS = s.dim / 2;
    V3 pos = sub3(p, V3{s.pos[0], s.pos[1], s.pos[2]});
    float depth = dot3(pos, V3{s.vv[0], s.vv[1], s.vv[2]});
    int sx = f2i(dot3(pos, V3{s.vv[3], s.vv[4], s.vv[5]}) * s.scale) + wS;
    int sy = f2i(dot3(pos, V3{s.vv[6], s.vv[7], s.vv[8]}) * -s.scale) + wS;
    if (sx >= 2 && sx < 2 * wS - 2 && sy >= 2 && sy < 2 * wS - 2) {
      const float *SD = s.map;
      int r = 2 * wS;
      if (__ldg(SD + r * sy + sx) < depth) shadow += 1;
      if (__ldg(SD + r * (sy + 2) + sx) < depth) shadow += 1;
      if (__ldg(SD + r * (sy - 2) + sx) < depth) shadow += 1;
      if (__ldg(SD + r * sy + (sx + 2)) < depth) shadow += 1;
      if (__ldg(SD + r * sy + (sx - 2)) < depth) shadow += 1;
    }
  }
  shadow = min(5, shadow);
  float light = (float)shadow * P.light.amb + (float)(5 - shadow);
  return light * 0.2f;
}

template <class A>
__device__ __forceinline__ void swap_(A &a, A &b) { A t = a; a = b; b = t; }

// The interpolants of winner `ord` on row cy: triangle set-up, mip level and
// the row accumulation (small triangles from their first row, large ones
// from the tile's first row), as the rasterizer walked them.
struct RowState {
  float cx1, cx2, cz1, cz2;
  Attr<true> c1, c2;
  float fmip;
  int mip, g;
  V3 tan, bit;   // F_NORMAL: the triangle's tangent frame
};

// shader_setup of the normal-mapped sources (av_draw_normmap.c:24-38): the
// tangent frame from the sorted vertices' uv and position divided by z
// (before the round trip multiplies them back)
__device__ __noinline__ void normal_frame(const Attr<true> a[3], const float z[3], V3 &tan, V3 &bit) {
  V2 uv1 = div2(a[0].uv, z[0]), uv2 = div2(a[1].uv, z[1]), uv3 = div2(a[2].uv, z[2]);
  V3 p1 = div3(a[0].p, z[0]), p2 = div3(a[1].p, z[1]), p3 = div3(a[2].p, z[2]);
  V2 dUV1 = sub2(uv2, uv1), dUV2 = sub2(uv3, uv1);
  V3 dPos1 = sub3(p2, p1), dPos2 = sub3(p3, p1);
  float rdet = 1.f / (dUV1.x * dUV2.y - dUV1.y * dUV2.x);
  tan = fast_normalize(mul3(sub3(mul3(dPos1, dUV2.y), mul3(dPos2, dUV1.y)), rdet));
  bit = fast_normalize(mul3(sub3(mul3(dPos2, dUV1.x), mul3(dPos1, dUV2.x)), rdet));
}

// Replays `steps` rows of the two edge chains (add: downwards, else upwards)
// and stores them in st: edge 0 the first chain (cx1, cz1, c1), edge 1 the
// second (cx2, cz2, c2), edge 2 both.  The chains are independent sequences
// of rounded additions, so two threads can each replay one of them and the
// results are those of one thread replaying both.
__device__ __forceinline__ void replay_edges(int edge, int steps, bool add, float cx1, float cx2, float cz1, float cz2,
                                             Attr<true> c1, Attr<true> c2, float s1, float s2, float sz1, float sz2,
                                             const Attr<true> &sa1, const Attr<true> &sa2, RowState &st) {
  if (edge == 2) {
    if (add) {
      for (int r = 0; r < steps; r++) {
        cx1 += s1; cx2 += s2; cz1 += sz1; cz2 += sz2; c1 = a_add(c1, sa1); c2 = a_add(c2, sa2);
      }
    } else {
      for (int r = 0; r < steps; r++) {
        cx1 -= s1; cx2 -= s2; cz1 -= sz1; cz2 -= sz2; c1 = a_sub(c1, sa1); c2 = a_sub(c2, sa2);
      }
    }
    st.cx1 = cx1; st.cx2 = cx2; st.cz1 = cz1; st.cz2 = cz2;
    st.c1 = c1; st.c2 = c2;
    return;
  }
  const bool e2 = edge != 0;
  float cx = e2 ? cx2 : cx1, cz = e2 ? cz2 : cz1, s = e2 ? s2 : s1, sz = e2 ? sz2 : sz1;
  Attr<true> c = e2 ? c2 : c1;
  const Attr<true> &sa = e2 ? sa2 : sa1;
  if (add) {
    for (int r = 0; r < steps; r++) { cx += s; cz += sz; c = a_add(c, sa); }
  } else {
    for (int r = 0; r < steps; r++) { cx -= s; cz -= sz; c = a_sub(c, sa); }
  }
  if (e2) { st.cx2 = cx; st.cz2 = cz; st.c2 = c; }
  else { st.cx1 = cx; st.cz1 = cz; st.c1 = c; }
}

// The row state of winner `ord` on row cy: the edge chain(s) `edge` selects
// (see replay_edges) and, for edge 0 or 2, the mip level, group and (NRM,
// F_NORMAL groups) the tangent frame.  NRM = false: draws without
// normal-mapped groups, whose shade then carries none of that code.
template <bool NRM = true>
__device__ __forceinline__ void shade_row_edge(const DrawParams &P, const GroupDev *sg, uint32_t ord, int cy, int edge,
                                               RowState &st) {
  uint32_t o = ord - 1;
  int phase = (int)(o >> 31);
  uint32_t gtri = (o >> 1) & 0x3fffffffu;
  int half = (int)(o & 1);
  int g = find_group(sg, P.ngroups, gtri);
  const GroupDev &G = sg[g];
  int tri = (int)(gtri - G.tri_base);
  float sx[3], sy[3], sz[3];
  project_persp(G, tri, P.view, sx, sy, sz);
  Attr<true> a[3];
  float z[3], x[3], y[3];
  int ix[3], iy[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    a[k] = a_load<true>(G, tri, k, sz[k]);
    z[k] = sz[k];
    x[k] = sx[k]; y[k] = sy[k];
    ix[k] = f2i(sx[k]); iy[k] = f2i(sy[k]);
  }
  const bool mip = (G.flags & F_MIP) != 0;
  const bool normal = NRM && (G.flags & F_NORMAL) != 0;
  MipSel ms;
  ms.fmip = 0; ms.mip = 0; ms.len_mip = 1; ms.len_mip2 = 2; ms.start_mip = 0; ms.start_mip2 = 1;
  float cx1, cx2, cz1, cz2;
  Attr<true> c1, c2;
  if (phase == 0) {
    // direct path: integer vertices (Templates.py:230-231)
    if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); swap_(a[0], a[1]); }
    if (iy[1] > iy[2]) { swap_(iy[1], iy[2]); swap_(ix[1], ix[2]); swap_(z[1], z[2]); swap_(a[1], a[2]); }
    if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); swap_(a[0], a[1]); }
    int x1 = ix[0], x2 = ix[1], x3 = ix[2], y1 = iy[0], y2 = iy[1], y3 = iy[2];
    float z1 = z[0], z2 = z[1], z3 = z[2];
    float yd = (float)(y2 - y1) / (float)(y3 - y1);
    float x4 = (float)x1 + yd * (float)(x3 - x1);
    float z4 = z1 + yd * (z3 - z1);
    Attr<true> a4 = a_add(a[0], a_smul(yd, a_sub(a[2], a[0])));
    if (normal) {
      if (edge != 1) normal_frame(a, z, st.tan, st.bit);
      if (!mip) mip_attr_roundtrip<true>(a, z);
    }
    if (mip) ms = mip_setup<true>(a, z, true, ix, iy, nullptr, nullptr, G.tex_size, G.mip_bias);
    float s1, s2, sz1, sz2;
    Attr<true> sa1, sa2;
    int n;
    if (half == 0) {
      float d = 1.0f / (float)(y2 - y1);
      s1 = (float)(x2 - x1) * d; s2 = (x4 - (float)x1) * d;
      sz1 = (z2 - z1) * d; sz2 = (z4 - z1) * d;
      sa1 = a_mul(a_sub(a[1], a[0]), d); sa2 = a_mul(a_sub(a4, a[0]), d);
      cx1 = cx2 = (float)x1; cz1 = cz2 = z1; c1 = c2 = a[0];
      n = cy - y1;
    } else {
      float d = 1.0f / (float)(y3 - y2);
      s1 = (float)(x3 - x2) * d; s2 = ((float)x3 - x4) * d;
      sz1 = (z3 - z2) * d; sz2 = (z3 - z4) * d;
      sa1 = a_mul(a_neg(a_sub(a[1], a[2])), d); sa2 = a_mul(a_neg(a_sub(a4, a[2])), d);
      cx1 = cx2 = (float)x3; cz1 = cz2 = z3; c1 = c2 = a[2];
      n = y3 - cy;
    }
    if (s1 < s2) { swap_(s1, s2); swap_(sz1, sz2); swap_(sa1, sa2); }
    replay_edges(edge, n, half == 0, cx1, cx2, cz1, cz2, c1, c2, s1, s2, sz1, sz2, sa1, sa2, st);
  } else {
    // tiled path: float vertices, per-tile restart (Templates.py:93-182)
    if (y[0] > y[1]) { swap_(y[0], y[1]); swap_(x[0], x[1]); swap_(z[0], z[1]); swap_(a[0], a[1]); }
    if (y[1] > y[2]) { swap_(y[1], y[2]); swap_(x[1], x[2]); swap_(z[1], z[2]); swap_(a[1], a[2]); }
    if (y[0] > y[1]) { swap_(y[0], y[1]); swap_(x[0], x[1]); swap_(z[0], z[1]); swap_(a[0], a[1]); }
    float x1 = x[0], x2 = x[1], x3 = x[2], y1 = y[0], y2 = y[1], y3 = y[2];
    float z1 = z[0], z2 = z[1], z3 = z[2];
    float yd = (y2 - y1) / (y3 - y1);
    float x4 = x1 + yd * (x3 - x1);
    float z4 = z1 + yd * (z3 - z1);
    Attr<true> a4 = a_add(a[0], a_smul(yd, a_sub(a[2], a[0])));
    if (normal) {
      if (edge != 1) normal_frame(a, z, st.tan, st.bit);
      if (!mip) mip_attr_roundtrip<true>(a, z);
    }
    if (mip) {
      if (P.mipc) {
        mip_attr_roundtrip<true>(a, z);
        float2 mc = P.mipc[gtri];
        ms.fmip = mc.x; ms.mip = (int)mc.y;
      } else {
        ms = mip_setup<true>(a, z, false, nullptr, nullptr, x, y, G.tex_size, G.mip_bias);
      }
    }
    int tileY = cy / TILE;
    float yMin = (float)tileY * 16.f, yMax = ((float)tileY + 1.f) * 16.f - 1.f;
    float s1, s2, sz1, sz2;
    Attr<true> sa1, sa2;
    if (half == 0) {
      float d = 1.0f / (y2 - y1);
      s1 = (x2 - x1) * d; s2 = (x4 - x1) * d;
      sz1 = (z2 - z1) * d; sz2 = (z4 - z1) * d;
      sa1 = a_mul(a_sub(a[1], a[0]), d); sa2 = a_mul(a_sub(a4, a[0]), d);
      if (s1 < s2) { swap_(s1, s2); swap_(sz1, sz2); swap_(sa1, sa2); }
      int cy0 = f2i(clampf_(y1, yMin, yMax));
      float dy = (float)cy0 - y1;
      cx1 = x1 + dy * s1; cx2 = x1 + dy * s2; cz1 = z1 + dy * sz1; cz2 = z1 + dy * sz2;
      c1 = a_add(a[0], a_smul(dy, sa1)); c2 = a_add(a[0], a_smul(dy, sa2));
      replay_edges(edge, cy - cy0, true, cx1, cx2, cz1, cz2, c1, c2, s1, s2, sz1, sz2, sa1, sa2, st);
    } else {
      float d = 1.0f / (y3 - y2);
      s1 = (x3 - x2) * d; s2 = (x3 - x4) * d;
      sz1 = (z3 - z2) * d; sz2 = (z3 - z4) * d;
      sa1 = a_mul(a_neg(a_sub(a[1], a[2])), d); sa2 = a_mul(a_neg(a_sub(a4, a[2])), d);
      if (s1 < s2) { swap_(s1, s2); swap_(sz1, sz2); swap_(sa1, sa2); }
      int cy0 = f2i(clampf_(y3, yMin, yMax));
      float dy = (float)cy0 - y3;
      cx1 = x3 + dy * s1; cx2 = x3 + dy * s2; cz1 = z3 + dy * sz1; cz2 = z3 + dy * sz2;
      c1 = a_add(a[2], a_smul(dy, sa1)); c2 = a_add(a[2], a_smul(dy, sa2));
      replay_edges(edge, cy0 - cy, false, cx1, cx2, cz1, cz2, c1, c2, s1, s2, sz1, sz2, sa1, sa2, st);
    }
  }
  if (edge != 1) { st.fmip = ms.fmip; st.mip = ms.mip; st.g = g; }
}

__device__ __forceinline__ void shade_row(const DrawParams &P, const GroupDev *sg, uint32_t ord, int cy, RowState &st) {
  shade_row_edge(P, sg, ord, cy, 2, st);
}

// av_draw_multi.c:30-105: the 4-way terrain blend of a F_MULTI group.  Its
// texture and the next three groups' (Ops0.py:533-545 binds TR[tn+1..tn+3])
// are sampled at the same bilinear taps; blend weights come from the world
// height and the normal; no shadow lookup.  The blended texel is converted
// to u16 before the lighting product, as the source does.
__device__ __forceinline__ void shade_multi(const DrawParams &P, const GroupDev *G, size_t pix, float t, float tz,
                                            V2 uvi, const RowState &st) {
  float omt = 1 - t;
  Taps q = make_taps(uvi, tz, G[0].tex_size, 0);
  V3 tx[4];
#pragma unroll
  for (int k = 0; k < 4; k++) tx[k] = bilerp_rgb(q, G[k].tex);
  V3 col = mul3(add3(smul3(omt, st.c2.li), smul3(t, st.c1.li)), tz);
  V3 nrm = fast_normalize(mul3(add3(smul3(omt, st.c2.n), smul3(t, st.c1.n)), tz));
  V3 ldir{P.light.ldir[0], P.light.ldir[1], P.light.ldir[2]};
  V3 lint{P.light.lint[0], P.light.lint[1], P.light.lint[2]};
  V3 dc = smul3(fmaxf(0.f, dot3(nrm, ldir)), lint);
  V3 cpos = mul3(add3(smul3(omt, st.c2.p), smul3(t, st.c1.p)), tz);
  float m = (cpos.y - 15.f) / 4.f;
  m = fminf(fmaxf(m, 0.f), 1.f);
  float ny = fmaxf(0.f, fabsf(nrm.y) - 0.33f) * 1.5f;
  m -= 1.5f * (ny * ny - 0.4f);
  m = fminf(fmaxf(m, 0.f), 1.f);
  V3 qv = div3(cpos, 3.f);
  float threshy = 16.f + 2.f * fabsf(qv.x - roundf(qv.x)) + 2.f * fabsf(qv.z - roundf(qv.z));
  float n = fminf(fmaxf((cpos.y - threshy) / 2.f, 0.f), 4.f);
  n = n * n * n;
  n += 1.5f * (ny * ny - 0.4f);
  n = fminf(fmaxf(n, 0.f), 32.f);
  float o = fminf(fmaxf((5.f - cpos.y) / 4.f, 0.f), 1.f);
  if (m + n + o > 1.f) {   // each weight divides by the sum of the updated ones
    n = n / (n + m + o);
    m = m / (n + m + o);
    o = o / (n + m + o);
  }
  float w1 = 1 - m - n - o;
  const float light = 1;
  P.ro[pix] = u16sat((float)u16sat(m * tx[1].x + n * tx[2].x + o * tx[3].x + w1 * tx[0].x) * (light * dc.x + col.x));
  P.go[pix] = u16sat((float)u16sat(m * tx[1].y + n * tx[2].y + o * tx[3].y + w1 * tx[0].y) * (light * dc.y + col.y));
  P.bo[pix] = u16sat((float)u16sat(m * tx[1].z + n * tx[2].z + o * tx[3].z + w1 * tx[0].z) * (light * dc.z + col.z));
  P.db[pix] = tz;
}

// pown(x, n), n >= 0, by repeated squaring (the convention pinned for
// OpenCL's pown, whose rounding the device chooses)
__device__ __forceinline__ float pown_rs(float x, int n) {
  unsigned k = n < 0 ? 0u - (unsigned)n : (unsigned)n;
  float r = 1.0f, b = x;
  while (k) {
    if (k & 1u) r *= b;
    b *= b;
    k >>= 1;
  }
  return n < 0 ? 1.0f / r : r;
}

// sampleShadow of the normal-mapped sources, which the reference calls but
// defines nowhere, as this library defines it: the five taps of one cascade
// (centre, +-2 texels in x and y) at the truncated map position, counted
// where the map is nearer than `depth`, only when the centre lies in
// [2, 2 wS - 2) on both axes; the shadowed fraction is count * 0.2.
__device__ __forceinline__ float sample_shadow5(const ShadowDev &s, float depth, float sfx, float sfy) {
  int wS = s.dim / 2;
  int sx = f2i(sfx), sy = f2i(sfy), n = 0;
  if (sx >= 2 && sx < 2 * wS - 2 && sy >= 2 && sy < 2 * wS - 2) {
    const float *SD = s.map;
    int r = 2 * wS;
    if (__ldg(SD + r * sy + sx) < depth) n += 1;
    if (__ldg(SD + r * (sy + 2) + sx) < depth) n += 1;
    if (__ldg(SD + r * (sy - 2) + sx) < depth) n += 1;
    if (__ldg(SD + r * sy + (sx + 2)) < depth) n += 1;
    if (__ldg(SD + r * sy + (sx - 2)) < depth) n += 1;
  }
  return (float)n * 0.2f;
}

// bilinear normal-map texel at the taps (texi1*texi2*convert_float3(NM[tex]) + ...)
__device__ __forceinline__ V3 bilerp_nm(const Taps &q, const uchar4 *__restrict__ NM) {
  uchar4 a = __ldg(NM + q.tex), b = __ldg(NM + q.tex10), c = __ldg(NM + q.tex01), d = __ldg(NM + q.tex11);
  float w00 = q.texi1 * q.texi2, w10 = q.texr1 * q.texi2, w01 = q.texi1 * q.texr2, w11 = q.texr1 * q.texr2;
  V3 r;
  r.x = w00 * (float)a.x + w10 * (float)b.x + w01 * (float)c.x + w11 * (float)d.x;
  r.y = w00 * (float)a.y + w10 * (float)b.y + w01 * (float)c.y + w11 * (float)d.y;
  r.z = w00 * (float)a.z + w10 * (float)b.z + w01 * (float)c.z + w11 * (float)d.z;
  return r;
}

// The normal-mapped fragment cores: av_draw_normmap.c:47-149 (its alpha
// variant after the visibility pass's alpha test) and, with F_MIP,
// av_draw_normmap_mip.c:73-160.  The light comes from the draw's first
// cascade (sample_shadow5), 1 without one.  Kept out of line so that the
// other materials keep their registers.
__device__ __noinline__ void shade_normal(const DrawParams &P, const GroupDev &G, size_t pix, float t, float tz,
                                          V2 uvi, const RowState &st, MipSel ms) {
  const bool mip = (G.flags & F_MIP) != 0;
  float omt = 1 - t;
  Taps q = make_taps(uvi, tz, mip ? ms.len_mip : G.tex_size, mip ? ms.start_mip : 0);
  V3 c = bilerp_rgb(q, G.tex);
  float outR = c.x, outG = c.y, outB = c.z;
  V3 tg = bilerp_nm(q, G.nm);
  if (mip) {
    Taps q2 = make_taps(uvi, tz, ms.len_mip2, ms.start_mip2);
    float ofm = 1 - ms.fmip;
    V3 c2 = bilerp_rgb(q2, G.tex);
    outR = ofm * outR + ms.fmip * c2.x;
    outG = ofm * outG + ms.fmip * c2.y;
    outB = ofm * outB + ms.fmip * c2.z;
    tg = add3(smul3(ofm, tg), smul3(ms.fmip, bilerp_nm(q2, G.nm)));
  }
  float light = 1;
  if (P.nsh > 0) {
    const ShadowDev &sh = P.sh[0];
    V3 pos = sub3(mul3(add3(smul3(omt, st.c2.p), smul3(t, st.c1.p)), tz), V3{sh.pos[0], sh.pos[1], sh.pos[2]});
    float depth = dot3(pos, V3{sh.vv[0], sh.vv[1], sh.vv[2]});
    float wS = (float)(sh.dim / 2);
    float sfx = (dot3(pos, V3{sh.vv[3], sh.vv[4], sh.vv[5]}) * sh.scale) + wS;
    float sfy = (dot3(pos, V3{sh.vv[6], sh.vv[7], sh.vv[8]}) * -sh.scale) + wS;
    light = 1 - sample_shadow5(sh, depth, sfx, sfy);
  } else {
    light = 1 - 0.f;
  }
  V3 col = mul3(add3(smul3(omt, st.c2.li), smul3(t, st.c1.li)), tz);
  V3 norm = fast_normalize(mul3(add3(smul3(omt, st.c2.n), smul3(t, st.c1.n)), tz));
  tg = sub3(mul3(div3(tg, 255.f), 2.f), V3{1.f, 1.f, 1.f});
  tg = fast_normalize(tg);
  norm = fast_normalize(add3(add3(smul3(tg.z, norm), smul3(-tg.y, st.tan)), smul3(-tg.x, st.bit)));
  V3 vp{P.view.pos[0], P.view.pos[1], P.view.pos[2]};
  V3 lint{P.light.lint[0], P.light.lint[1], P.light.lint[2]};
  V3 ldir{P.light.ldir[0], P.light.ldir[1], P.light.ldir[2]};
  V3 pos = mul3(add3(smul3(omt, st.c2.p), smul3(t, st.c1.p)), tz);
  V3 spec;
  if (mip) {
    V3 a = sub3(pos, vp);
    V3 h = fast_normalize(add3(fast_normalize(a), ldir));
    float theta = fmaxf(0.f, dot3(h, norm));
    float mf = (float)ms.mip + ms.fmip;
    int sp = f2i(1.f * (mf * mf));
    spec = smul3(((pown_rs(theta, sp) * 256.f) * light) * 2.f, lint);
    spec = mul3(spec, (float)(sp + 1) / (2.f * 3.1416f));
  } else {
    V3 a = fast_normalize(sub3(pos, vp));
    V3 h = fast_normalize(add3(a, ldir));
    float theta = fmaxf(0.f, dot3(h, norm));
    int sp = G.spec_pow;
    spec = smul3(((pown_rs(theta, sp) * 256.f) * 4.f) * light, lint);
    spec = mul3(spec, (float)(sp + 2) / (8.f * 3.1416f));
    a = sub3(pos, vp);
    float nd = dot3(a, norm);
    V3 refl = fast_normalize(sub3(a, smul3(2.f * nd, norm)));
    theta = fmaxf(0.f, dot3(refl, V3{0.f, 1.f, 0.f}));
    spec = add3(spec, smul3((pown_rs(theta, 2) * 128.f) * (float)(1 + G.is_metal), V3{0.1f, 0.3f, 0.5f}));
    theta = fmaxf(0.f, dot3(fast_normalize(a), refl));
    spec = add3(spec, smul3(pown_rs(theta, G.spec_pow2) * 256.f, V3{0.2f, 0.2f, 0.2f}));
    if (G.is_metal) {
      ushort4 tx = __ldg(G.tex + q.tex);
      spec.x *= (float)tx.x / 1024.f;
      spec.y *= (float)tx.y / 1024.f;
      spec.z *= (float)tx.z / 1024.f;
      light = 0.f;
      col = V3{0.f, 0.f, 0.f};
    }
  }
  V3 dc = smul3(fmaxf(0.f, dot3(norm, ldir)), lint);
  P.ro[pix] = u16sat(spec.x + outR * (light * dc.x + col.x));
  P.go[pix] = u16sat(spec.y + outG * (light * dc.y + col.y));
  P.bo[pix] = u16sat(spec.z + outB * (light * dc.z + col.z));
  P.db[pix] = tz;
}

// Shades pixel ax of row cy from its winner's row state.
template <bool NRM = true>
__device__ __forceinline__ void shade_from_row(const DrawParams &P, const GroupDev *sg, int ax, int cy,
                                               const RowState &st) {
  const GroupDev &G = sg[st.g];
  const bool mip = (G.flags & F_MIP) != 0;
  MipSel ms;
  ms.fmip = st.fmip; ms.mip = st.mip;
  ms.len_mip = 1 << ms.mip; ms.len_mip2 = ms.len_mip << 1;
  ms.start_mip = ((1 << (2 * ms.mip)) - 1) / 3;            // sum of 4^i for i < mip
  ms.start_mip2 = ms.start_mip + ms.len_mip * ms.len_mip;
  const float cx1 = st.cx1, cx2 = st.cx2, cz1 = st.cz1, cz2 = st.cz2;
  const Attr<true> c1 = st.c1, c2 = st.c2;
  float t = ((float)ax - cx2) / (cx1 - cx2);
  t = clamp_t(t);
  float tz = 1.0f / ((1 - t) * cz2 + t * cz1);
  float omt = 1 - t;
  V2 uvi = add2(smul2(omt, c2.uv), smul2(t, c1.uv));
  if (G.flags & F_MULTI) {                 // the group table clears F_MULTI on alpha-tested groups
    shade_multi(P, &G, (size_t)P.view.w * cy + ax, t, tz, uvi, st);
    return;
  }
  if (NRM && (G.flags & F_NORMAL)) {
    shade_normal(P, G, (size_t)P.view.w * cy + ax, t, tz, uvi, st, ms);
    return;
  }
  float outR, outG, outB;
  if (mip) {
    // av_draw_normmap_mip.c:73-123
    Taps q1 = make_taps(uvi, tz, ms.len_mip, ms.start_mip);
    V3 c1v = bilerp_rgb(q1, G.tex);
    outR = c1v.x; outG = c1v.y; outB = c1v.z;
    Taps q2 = make_taps(uvi, tz, ms.len_mip2, ms.start_mip2);
    float ofm = 1 - ms.fmip;
    V3 c2v = bilerp_rgb(q2, G.tex);
    outR = ofm * outR + ms.fmip * c2v.x;
    outG = ofm * outG + ms.fmip * c2v.y;
    outB = ofm * outB + ms.fmip * c2v.z;
  } else {
    Taps q = make_taps(uvi, tz, G.tex_size, 0);
    V3 cv = bilerp_rgb(q, G.tex);
    outR = cv.x; outG = cv.y; outB = cv.z;
  }
  float light = 1;
  if (G.flags & F_SHADOW) {
    V3 p = mul3(add3(smul3(omt, c2.p), smul3(t, c1.p)), tz);
    light = shadow_light(P, p);
  }
  V3 col = mul3(add3(smul3(omt, c2.li), smul3(t, c1.li)), tz);
  V3 nrm = fast_normalize(mul3(add3(smul3(omt, c2.n), smul3(t, c1.n)), tz));
  V3 ldir{P.light.ldir[0], P.light.ldir[1], P.light.ldir[2]};
  V3 lint{P.light.lint[0], P.light.lint[1], P.light.lint[2]};
  V3 dc = smul3(fmaxf(0.f, dot3(nrm, ldir)), lint);
  float oml = 1 - light;
  size_t pix = (size_t)P.view.w * cy + ax;
  P.ro[pix] = u16sat(outR * (light * (dc.x + col.x) + oml * col.x));
  P.go[pix] = u16sat(outG * (light * (dc.y + col.y) + oml * col.y));
  P.bo[pix] = u16sat(outB * (light * (dc.z + col.z) + oml * col.z));
  P.db[pix] = tz;
}

// Replays the winning fragment of pixel (ax, cy) and shades it.
__device__ __forceinline__ void shade_pixel(const DrawParams &P, const GroupDev *sg, int ax, int cy, uint64_t key) {
  uint32_t ord = 0xffffffffu - (uint32_t)key;
  if (ord == 0) return;
  RowState st;
  shade_row(P, sg, ord, cy, st);
  shade_from_row(P, sg, ax, cy, st);
}

// Shared memory of shade_tile for a block of NT threads (16 x NT/16 pixels).
template <int NT>
struct ShadeSmem {
  unsigned long long hkey[NT];   // open-addressing table of (winner, row) keys
  int hent[NT];                  // its entry numbers
  unsigned long long ekey[NT];   // entry -> key
  int nent;
  RowState rs[NT];
};

// Shades the 16 x (NT/16) pixels at (x0, y0): the block finds the distinct
// (winner, row) pairs among its pixels (a bounded open-addressing table in
// shared memory), two threads per pair set up the triangle and replay its
// row (one edge chain each), then every pixel shades from its pair's row
// state.  The arithmetic is shade_pixel's, done once per pair instead of once
// per pixel.
template <int NT, bool NRM = true>
__device__ __forceinline__ void shade_tile(const DrawParams &P, const GroupDev *sg, int x0, int y0, ShadeSmem<NT> &sm) {
  const unsigned long long EMPTY = ~0ull;
  int tid = threadIdx.x;
  int ax = x0 + (tid & 15), cy = y0 + (tid >> 4);
  bool in = ax < P.view.w && cy < P.view.h;
  uint32_t ord = in ? 0xffffffffu - (uint32_t)P.keys[(size_t)P.view.w * cy + ax] : 0u;
  bool valid = ord != 0;
  sm.hkey[tid] = EMPTY;
  if (tid == 0) sm.nent = 0;
  __syncthreads();
  int slot = 0;
  // the lanes of a warp with the same (winner, row) -- often a whole row of
  // the tile -- insert it once, through their first lane
  unsigned long long k = valid ? (((unsigned long long)ord << 32) | (uint32_t)cy) : EMPTY;
  const unsigned peers = __match_any_sync(FULL, k);
  const int leader = __ffs(peers) - 1;
  if (valid && (tid & 31) == leader) {
    uint32_t h = ((ord * 2654435761u) ^ ((uint32_t)cy * 40503u)) % NT;
    for (int i = 0; i < NT; i++) {       // at most NT keys: always finds a slot
      unsigned long long prev = atomicCAS(&sm.hkey[h], EMPTY, k);
      if (prev == EMPTY) {
        int e = atomicAdd(&sm.nent, 1);
        sm.hent[h] = e;
        sm.ekey[e] = k;
        slot = (int)h;
        break;
      }
      if (prev == k) {
        slot = (int)h;
        break;
      }
      h = (h + 1) % NT;
    }
  }
  slot = __shfl_sync(FULL, slot, leader);
  __syncthreads();
  int ne = sm.nent;
  for (int j = tid; j < 2 * ne; j += NT) {   // two threads a pair, one edge chain each
    unsigned long long k = sm.ekey[j >> 1];
    shade_row_edge<NRM>(P, sg, (uint32_t)(k >> 32), (int)(uint32_t)k, j & 1, sm.rs[j >> 1]);
  }
  __syncthreads();
  if (valid) shade_from_row<NRM>(P, sg, ax, cy, sm.rs[sm.hent[slot]]);
  __syncthreads();                       // the next tile reuses the shared memory
}


// one 256-thread block per 16x16 tile
// NRM: the draw has normal-mapped groups
template <bool NRM>
__global__ void __launch_bounds__(256, 4) k_shade(DrawParams P) {   // 64 registers: 4 blocks per SM
  __shared__ GroupDev sg[64];
  __shared__ ShadeSmem<256> sm;
  for (int i = threadIdx.x; i < P.ngroups; i += blockDim.x) sg[i] = P.groups[i];
  __syncthreads();
  shade_tile<256, NRM>(P, sg, blockIdx.x * TILE, blockIdx.y * TILE, sm);
}

__global__ void k_ids(const uint64_t *__restrict__ keys, int n, int32_t *tri_id, uint8_t *cov) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t ord = 0xffffffffu - (uint32_t)keys[i];
    int32_t id = ord == 0 ? -1 : (int32_t)(((ord - 1) >> 1) & 0x3fffffffu);
    if (tri_id) tri_id[i] = id;
    if (cov) cov[i] = ord != 0;
  }
}

// ------------------------------------------------------------ shadow depth pass

struct ShadowParams {
  const GroupDev *groups;
  int ngroups;
  int total_tris;
  ShadowDev sh;
  float *map;
  float bias;
  uint32_t *list;      // opaque casters from the front, alpha-tested from the back
  uint32_t cap_list;
  uint32_t *ctr;
  uint32_t *items;     // row chunks of the casters, same two ends (cap_list * MAX_CHUNKS);
                       // null: one work item per caster
  int min_chunk;       // rows per chunk (at least)
  int claim_k;         // claim_size's k (0: 32 items per claim)
  // tiled pass (rec != null): one record per caster at its list position,
  // per-tile unit counts (opaque [0, ntiles), alpha [ntiles, 2 ntiles)),
  // offsets, scatter cursors and claim counters (opaque, alpha per tile),
  // the non-empty tiles in order with the prefix of their block counts, units
  uint4 *rec;          // 2 per caster: sorted vertices, z, triangle, vertex order
  uint32_t *tcnt, *toff, *tcur, *tclaim, *tord, *hpre, *units;
  uint32_t cap_units;
  int ntx, ntiles;     // tiles per side, tiles
  int slice;           // units per block of a tile: a tile with n units gets ceil(n / slice) blocks
  int sort;            // 1: each tile's units front (nearest the light) first
};

// Rows per work item of a caster (at least).  Alpha-tested casters take
// half: their fragments cost more (the mask), so they balance better over
// shorter items (on the 1080p scene's cascades 102 -> 86 us at 6 rows
// against 12, while the opaque casters are fastest at 12).
__device__ __forceinline__ int shadow_min_chunk(const ShadowParams &S, bool alpha) {
  return alpha ? max(1, S.min_chunk >> 1) : S.min_chunk;
}

// rows = the caster's row count in the map (drawmin.c: y1..y2 up, y3..y2+1 down);
// g, ix, iy, z = its group and projected vertices (trisetupOrtho.c)
__device__ __forceinline__ void shadow_classify(const GroupDev *sg, const ShadowParams &S, int t, bool &ok, bool &alpha,
                                                int &rows, int &g, int ix[3], int iy[3], float z[3]) {
  ok = false;
  alpha = false;
  rows = 0;
  g = 0;
  if (t < S.total_tris) {
    g = find_group(sg, S.ngroups, (uint32_t)t);
    const GroupDev &G = sg[g];
    if (G.enabled) {
      ok = project_ortho(G, t - G.tri_base, S.sh, S.bias, ix, iy, z);
      alpha = (G.flags & F_ALPHA) != 0;
      rows = max(iy[0], max(iy[1], iy[2])) - min(iy[0], min(iy[1], iy[2])) + 1;
    }
  }
}

// Appends the casters of a warp to the list (opaque from the front,
// alpha-tested from the back) and their row chunks to the work items;
// returns the caster's list slot.
__device__ __forceinline__ uint32_t shadow_append(const ShadowParams &S, int t, bool ok, bool alpha, int rows,
                                                  int lane) {
  unsigned mo = __ballot_sync(FULL, ok && !alpha), ma = __ballot_sync(FULL, ok && alpha);
  const uint32_t want[2] = {(uint32_t)__popc(mo), (uint32_t)__popc(ma)};
  const int idx[2] = {CTR_SH_LIST, CTR_SH_LIST_A};
  uint32_t got[2];
  block_reserve<2>(want, idx, S.ctr, got);
  unsigned lt = (1u << lane) - 1;
  uint32_t pos = 0;
  if (ok && !alpha) { pos = got[0] + __popc(mo & lt); S.list[pos] = (uint32_t)t; }
  if (ok && alpha) { pos = got[1] + __popc(ma & lt); S.list[S.cap_list - 1 - pos] = (uint32_t)t; }
  uint32_t slot = alpha ? S.cap_list - 1 - pos : pos;
  if (!S.items) return slot;
  // row chunks of the casters, as for the small triangles of the view
  int cl = 1, nch = 0;
  if (ok) {
    cl = chunk_len(rows, shadow_min_chunk(S, alpha));
    nch = (rows + cl - 1) / cl;
  }
  block_items(S.items, S.cap_list * MAX_CHUNKS, S.ctr, CTR_SH_ITEMS, CTR_SH_ITEMS_A, pos, alpha, rows, cl, nch);
  return slot;
}

// ---- tiled shadow pass: caster records and tile binning

constexpr int STILE_LOG = 5;
constexpr int STILE = 1 << STILE_LOG;   // a map tile is STILE x STILE texels
constexpr int TROW = STILE + 1;         // row stride of a tile in shared memory (rows in different banks)
constexpr int SUB_LOG = 3;              // the tile's texel maxima are kept per 8 x 8 sub-block
constexpr int SUBS = STILE >> SUB_LOG;  // sub-blocks per tile side

// drawmin.c's vertex order: sorted by y with its three compare-and-swaps;
// perm packs which of the triangle's vertices became vertex k (2 bits each)
__device__ __forceinline__ int caster_sort(int ix[3], int iy[3], float z[3]) {
  int p0 = 0, p1 = 1, p2 = 2;
  if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); swap_(p0, p1); }
  if (iy[1] > iy[2]) { swap_(iy[1], iy[2]); swap_(ix[1], ix[2]); swap_(z[1], z[2]); swap_(p1, p2); }
  if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); swap_(p0, p1); }
  return p0 | (p1 << 2) | (p2 << 4);
}

__device__ __forceinline__ uint32_t pack_xy(int x, int y) { return ((uint32_t)x & 0xffffu) | ((uint32_t)y << 16); }
__device__ __forceinline__ int unpack_x(uint32_t w) { return (int)(int16_t)(w & 0xffffu); }
__device__ __forceinline__ int unpack_y(uint32_t w) { return (int)w >> 16; }

// The tiles a caster (sorted vertices) can write: rows y1..y3, and columns
// x_min..x_max widened by the drift of the accumulated edge positions (an
// addition rounds by at most |x| 2^-24, so `rows` of them stay below
// rows * X * 2^-23) and by one for the truncated split vertex x4; all
// clipped to the map.  False when nothing of the caster lies on the map.
__device__ __forceinline__ bool caster_tiles(const int x[3], int y1, int y3, int dim, int &tx0, int &tx1, int &ty0,
                                             int &ty1) {
  if (!(y1 < dim && y3 >= 0)) return false;
  int mn = min(x[0], min(x[1], x[2])), mx = max(x[0], max(x[1], x[2]));
  long long X = (long long)max(iabs_(mn), iabs_(mx)) + 2;
  long long rows = (long long)y3 - y1 + 1;
  int m = 1 + (int)((rows * X) >> 22);
  int c0 = mn - m, c1 = mx + m;
  if (c1 < 0 || c0 > dim - 1) return false;
  c0 = max(c0, 0);
  c1 = min(c1, dim - 1);
  tx0 = c0 >> STILE_LOG;
  tx1 = c1 >> STILE_LOG;
  ty0 = max(y1, 0) >> STILE_LOG;
  ty1 = min(y3, dim - 1) >> STILE_LOG;
  return true;
}

// Writes caster t's record at its list slot and, in the tiled pass, counts
// it in every tile it can write (opaque counts first, alpha-tested after them).
__device__ __forceinline__ void shadow_record(const ShadowParams &S, int t, int g, bool alpha, int ix[3], int iy[3],
                                              float z[3], uint32_t slot) {
  int perm = caster_sort(ix, iy, z);
  S.rec[2 * (size_t)slot] = make_uint4(pack_xy(ix[0], iy[0]), pack_xy(ix[1], iy[1]), pack_xy(ix[2], iy[2]),
                                       __float_as_uint(z[0]));
  S.rec[2 * (size_t)slot + 1] = make_uint4(__float_as_uint(z[1]), __float_as_uint(z[2]), (uint32_t)t,
                                           (uint32_t)perm | ((uint32_t)g << 8));
  int tx0, tx1, ty0, ty1;
  if (!S.tcnt || !caster_tiles(ix, iy[0], iy[2], S.sh.dim, tx0, tx1, ty0, ty1)) return;
  const uint32_t base = alpha ? (uint32_t)S.ntiles : 0u;
  for (int ty = ty0; ty <= ty1; ty++)
    for (int tx = tx0; tx <= tx1; tx++) {
      // lanes counting into the same tile add once (casters crowd into few tiles)
      uint32_t key = base + (uint32_t)(ty * S.ntx + tx);
      unsigned peers = __match_any_sync(__activemask(), key);
      if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&S.tcnt[key], (uint32_t)__popc(peers));
    }
}

__device__ __forceinline__ void shadow_setup_phase(const ShadowParams &S, const GroupDev *sg, int first, int step) {
  int lane = threadIdx.x & 31;
  for (int base = first; base < S.total_tris; base += step) {
    int t = base + threadIdx.x;
    bool ok, alpha;
    int rows, g, ix[3], iy[3];
    float z[3];
    shadow_classify(sg, S, t, ok, alpha, rows, g, ix, iy, z);
    uint32_t slot = shadow_append(S, t, ok, alpha, rows, lane);
    if (S.rec && ok) shadow_record(S, t, g, alpha, ix, iy, z, slot);
  }
}

__global__ void __launch_bounds__(256) k_shadow_setup(ShadowParams S) {
  __shared__ GroupDev sg[64];
  for (int i = threadIdx.x; i < S.ngroups; i += blockDim.x) sg[i] = S.groups[i];
  __syncthreads();
  shadow_setup_phase(S, sg, blockIdx.x * blockDim.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void atomic_min_depth(float *addr, float v) {
  if (v >= 0.f) atomicMin((int *)addr, __float_as_int(v));
  else atomicMax((unsigned int *)addr, __float_as_uint(v));
}

// The texel test of the tiled pass.  Every pixel of a span stores
// tz = RN(1 / v), v = RN(RN((1 - t) cz2) + RN(t cz1)), t in [0, 1]; when cz1
// and cz2 are positive, v <= max(cz1, cz2) (1 + 2^-24)^3, so tz stays above
// (1 / max) (1 - 2^-22).  The returned threshold is one more than the bits
// of a float below that (an approximate reciprocal, within 2 ulp, taken
// down by 2^-18): a texel whose bits are smaller already holds a depth no
// pixel of the span undercuts, so its min update would change nothing.
// Spans whose ends are not positive and within [2^-60, 2^60] get INT_MIN,
// which no texel is below.  (A NaN end makes every pixel's depth NaN, which
// is never stored.)
__device__ __forceinline__ int depth_floor_bits(float cz1, float cz2) {
  float hi = fmaxf(cz1, cz2), lo = fminf(cz1, cz2);
  if (!(lo > 0.f) || !(hi >= 0x1p-60f) || !(hi <= 0x1p60f)) return INT_MIN;
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(hi));
  return __float_as_int(__fmul_rn(r, 1.0f - 0x1p-18f)) + 1;
}

template <bool ALPHA>
struct ShadowQ {
  float4 a[32];                  // cx2, d, 1/d (0: divide), cz1
  float4 b[32];                  // cz2, texel address - first pixel number, x - first pixel number,
                                 // depth floor bits (tiled pass)
  float4 c[ALPHA ? 32 : 1];      // cu1, cv1, cu2, cv2
  int g[ALPHA ? 32 : 1];
  int r2l[32];
};

template <bool ALPHA>
struct ShadowLane {
  float4 pb = make_float4(0.f, 0.f, 0.f, 0.f);   // second half of the last span record (fill_round stores it)
  int x1, x2, x3, y1, y2, y3, x4;
  float z1, z2, z3, z4, u1, u2, u3, u4, v1, v2, v3, v4;
  int half, cy, g;
  float s1, s2, sz1, sz2, su1, su2, sv1, sv2;
  float cx1, cx2, cz1, cz2, cu1, cu2, cv1, cv2;

  // drawmin.c divides each slope by the row count; one reciprocal serves
  // them all (quot_by_recip: the same correctly rounded quotients)
  __device__ __forceinline__ void start_half0() {
    half = 0;
    float d = (float)(y2 - y1);
    float y = span_recip(d);
    s1 = quot_by_recip((float)(x2 - x1), d, y);
    s2 = quot_by_recip((float)(x4 - x1), d, y);
    if (ALPHA) {
      su1 = quot_by_recip(u2 - u1, d, y); sv1 = quot_by_recip(v2 - v1, d, y);
      su2 = quot_by_recip(u4 - u1, d, y); sv2 = quot_by_recip(v4 - v1, d, y);
    }
    sz1 = quot_by_recip(z2 - z1, d, y); sz2 = quot_by_recip(z4 - z1, d, y);
    cx1 = cx2 = (float)x1; cz1 = cz2 = z1;
    if (ALPHA) { cu1 = cu2 = u1; cv1 = cv2 = v1; }
    if (s1 < s2) {
      swap_(s1, s2); swap_(sz1, sz2);
      if (ALPHA) { swap_(su1, su2); swap_(sv1, sv2); }
    }
    cy = y1;
  }
  // The second half's slopes are computed with the first's, when the
  // caster is set up: a lane that reaches its caster's middle row during
  // the walk then only copies them, instead of stalling the warp's other
  // lanes for the divisions.
  float hs1, hs2, hsz1, hsz2, hsu1, hsv1, hsu2, hsv2;
  __device__ __forceinline__ void half1_slopes() {
    float d = (float)(y3 - y2);
    float y = span_recip(d);
    hs1 = quot_by_recip((float)(x3 - x2), d, y);
    hs2 = quot_by_recip((float)(x3 - x4), d, y);
    if (ALPHA) {
      hsu1 = quot_by_recip(u3 - u2, d, y); hsv1 = quot_by_recip(v3 - v2, d, y);
      hsu2 = quot_by_recip(u3 - u4, d, y); hsv2 = quot_by_recip(v3 - v4, d, y);
    }
    hsz1 = quot_by_recip(z3 - z2, d, y); hsz2 = quot_by_recip(z3 - z4, d, y);
    if (hs1 < hs2) {
      swap_(hs1, hs2); swap_(hsz1, hsz2);
      if (ALPHA) { swap_(hsu1, hsu2); swap_(hsv1, hsv2); }
    }
  }
  __device__ __forceinline__ void start_half1() {
    half = 1;
    s1 = hs1; s2 = hs2; sz1 = hsz1; sz2 = hsz2;
    if (ALPHA) { su1 = hsu1; sv1 = hsv1; su2 = hsu2; sv2 = hsv2; }
    cx1 = cx2 = (float)x3; cz1 = cz2 = z3;
    if (ALPHA) { cu1 = cu2 = u3; cv1 = cv2 = v3; }
    cy = y3;
  }

  __device__ __forceinline__ bool init(const ShadowParams &S, const GroupDev *sg, uint32_t t) {
    g = find_group(sg, S.ngroups, t);
    const GroupDev &G = sg[g];
    int tri = (int)(t - G.tri_base);
    int ix[3], iy[3];
    float z[3];
    project_ortho(G, tri, S.sh, S.bias, ix, iy, z);
    V2 uv[3] = {V2{0, 0}, V2{0, 0}, V2{0, 0}};
    if (ALPHA) {
#pragma unroll
      for (int k = 0; k < 3; k++) uv[k] = mul2(ld2(G.uv + ((size_t)tri * 3 + k) * 2), z[k]);
    }
    if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); if (ALPHA) swap_(uv[0], uv[1]); }
    if (iy[1] > iy[2]) { swap_(iy[1], iy[2]); swap_(ix[1], ix[2]); swap_(z[1], z[2]); if (ALPHA) swap_(uv[1], uv[2]); }
    if (iy[0] > iy[1]) { swap_(iy[0], iy[1]); swap_(ix[0], ix[1]); swap_(z[0], z[1]); if (ALPHA) swap_(uv[0], uv[1]); }
    x1 = ix[0]; x2 = ix[1]; x3 = ix[2]; y1 = iy[0]; y2 = iy[1]; y3 = iy[2];
    z1 = z[0]; z2 = z[1]; z3 = z[2];
    if (!((y1 < S.sh.dim) && (y3 >= 0))) return false;
    finish(uv);
    return true;
  }

  // drawmin.c:49-51 (split vertex) and the first half's slopes, from the
  // sorted vertices
  __device__ __forceinline__ void finish(const V2 uv[3]) {
    float q = (float)(y2 - y1) / (float)(y3 - y1);
    x4 = f2i((float)x1 + q * (float)(x3 - x1));
    z4 = z1 + q * (z3 - z1);
    if (ALPHA) {
      u1 = uv[0].x; u2 = uv[1].x; u3 = uv[2].x; v1 = uv[0].y; v2 = uv[1].y; v3 = uv[2].y;
      u4 = u1 + q * (u3 - u1);
      v4 = v1 + q * (v3 - v1);
    }
    half1_slopes();
    start_half0();
    left = y3 - y1 + 1;
  }

  // The caster of record r (the setup projected and sorted it).  Only
  // casters with rows on the map have units.
  __device__ __forceinline__ void init_rec(const ShadowParams &S, const GroupDev *sg, uint32_t r) {
    uint4 a = S.rec[2 * (size_t)r], b = S.rec[2 * (size_t)r + 1];
    x1 = unpack_x(a.x); y1 = unpack_y(a.x);
    x2 = unpack_x(a.y); y2 = unpack_y(a.y);
    x3 = unpack_x(a.z); y3 = unpack_y(a.z);
    z1 = __uint_as_float(a.w); z2 = __uint_as_float(b.x); z3 = __uint_as_float(b.y);
    g = (int)(b.w >> 8);
    V2 uv[3] = {V2{0, 0}, V2{0, 0}, V2{0, 0}};
    if (ALPHA) {
      const GroupDev &G = sg[g];
      size_t v0 = ((size_t)b.z - (size_t)G.tri_base) * 3;
      uv[0] = mul2(ld2(G.uv + (v0 + (b.w & 3)) * 2), z1);
      uv[1] = mul2(ld2(G.uv + (v0 + ((b.w >> 2) & 3)) * 2), z2);
      uv[2] = mul2(ld2(G.uv + (v0 + ((b.w >> 4) & 3)) * 2), z3);
    }
    finish(uv);
  }

  // Restricts the walk to the rows ty0..ty1 of a tile: replays the rows
  // before the first of them and leaves in `left` the rows up to the last
  // (rows outside the tile in between are skipped as they come).  The walk
  // visits bottom-half rows y1..y2 (positions 0..n0-1), then top-half rows
  // y3 down to y2 + 1.
  __device__ __forceinline__ bool clip_rows(int ty0, int ty1) {
    int n0 = y2 - y1 + 1;
    int a0 = max(y1, ty0) - y1, a1 = min(y2, ty1) - y1;
    int blo = max(y2 + 1, ty0), bhi = min(y3, ty1);
    bool ha = a0 <= a1, hb = blo <= bhi;
    if (!ha && !hb) return false;
    int first = ha ? a0 : n0 + (y3 - bhi);
    int last = hb ? n0 + (y3 - blo) : a1;
    for (int r = 0; r < first; r++) skip_row();
    left = last - first + 1;
    return true;
  }

  int left;      // rows left in this lane's chunk (a whole caster: y3 - y1 + 1)
  bool serial;   // emit_tile: the span just written needs the true division

  // advances one row without drawing (the replay up to a chunk's first row)
  __device__ __forceinline__ void skip_row() {
    if (half == 0) {
      cx1 += s1; cx2 += s2; cz1 += sz1; cz2 += sz2;
      if (ALPHA) { cu1 += su1; cv1 += sv1; cu2 += su2; cv2 += sv2; }
      cy++;
      if (cy > y2) start_half1();
    } else {
      cx1 -= s1; cx2 -= s2; cz1 -= sz1; cz2 -= sz2;
      if (ALPHA) { cu1 -= su1; cv1 -= sv1; cu2 -= su2; cv2 -= sv2; }
      cy--;
    }
  }

  // chunk `chunk` of the caster's rows: replays the accumulation up to its
  // first row, so every interpolant equals the serial walk's
  __device__ __forceinline__ bool init_chunk(const ShadowParams &S, const GroupDev *sg, uint32_t t, int chunk) {
    if (!init(S, sg, t)) return false;
    int rows = left;
    int cl = chunk_len(rows, shadow_min_chunk(S, ALPHA));
    int first = chunk * cl;
    if (first >= rows) return false;
    left = min(cl, rows - first);
    for (int r = 0; r < first; r++) skip_row();
    return true;
  }

  // sets `serial` when the span just written needs the true division (the
  // caller then draws it with this lane alone)
  __device__ __forceinline__ int emit(int dim, ShadowQ<ALPHA> &q, int lane, bool &live) {
    serial = false;
    int cnt = 0;
    if (cy >= 0 && cy < dim) {
      int a0 = half == 0 ? f2i(cx2) : f2i(cx1);
      int a1 = half == 0 ? f2i(cx1) : f2i(cx2);
      int lo = a0 < 0 ? 0 : a0, hi = a1 > dim - 1 ? dim - 1 : a1;
      cnt = hi >= lo ? hi - lo + 1 : 0;
      if (cnt) {
        float qx, qd, qy;
        serial = !span_queue_form(cx2, cx1 - cx2, lo, qx, qd, qy);
        q.a[lane] = make_float4(qx, qd, qy, cz1);
        pb = make_float4(cz2, __int_as_float(cy * dim + lo), __int_as_float(lo), 0.f);
        if (serial) q.b[lane] = pb;
        if (ALPHA) {
          q.c[lane] = make_float4(cu1, cv1, cu2, cv2);
          q.g[lane] = g;
        }
      }
    }
    skip_row();
    live = --left > 0;
    return cnt;
  }

  // emit() inside a tile: the current row lies in rows ty0..ty1; its span is
  // clipped to columns tx0..tx1 and written with its texel offset in the
  // tile and its depth floor.  Then advances to the next row in the tile.
  // A span whose depth floor lies above every texel it covers (by the
  // tile's sub-block maxima `smax`) is not queued.
  __device__ __forceinline__ int emit_tile(ShadowQ<ALPHA> &q, int lane, int tx0, int tx1, int ty0, int ty1,
                                           const int *smax, bool &live) {
    int a0 = half == 0 ? f2i(cx2) : f2i(cx1);
    int a1 = half == 0 ? f2i(cx1) : f2i(cx2);
    int lo = max(a0, tx0), hi = min(a1, tx1);
    int cnt = hi >= lo ? hi - lo + 1 : 0;
    int floor_bits = 0;
    if (cnt) {
      floor_bits = depth_floor_bits(cz1, cz2);
      const int *row = smax + ((cy - ty0) >> SUB_LOG) * SUBS;
      int m = INT_MIN;
      for (int bx = (lo - tx0) >> SUB_LOG; bx <= (hi - tx0) >> SUB_LOG; bx++) m = max(m, row[bx]);
      if (m < floor_bits) cnt = 0;
    }
    serial = false;
    if (cnt) {
      float qx, qd, qy;
      serial = !span_queue_form(cx2, cx1 - cx2, lo, qx, qd, qy);   // then the caller draws it with this lane alone
      q.a[lane] = make_float4(qx, qd, qy, cz1);
      pb = make_float4(cz2, __int_as_float((cy - ty0) * TROW + (lo - tx0)), __int_as_float(lo),
                       __int_as_float(floor_bits));
      if (serial) q.b[lane] = pb;
      if (ALPHA) {
        q.c[lane] = make_float4(cu1, cv1, cu2, cv2);
        q.g[lane] = g;
      }
    }
    skip_row();
    --left;
    while (left > 0 && (cy < ty0 || cy > ty1)) {
      skip_row();
      --left;
    }
    live = left > 0;
    return cnt;
  }
};

// drawmin.c:71-76 / drawminalpha.c:83-97 for pixel number p of span s: the
// depth tz, or false when nothing is written (NaN depth, alpha discard)
template <bool ALPHA, bool DIV = false, bool EZ = false>
__device__ __forceinline__ bool shadow_depth(const GroupDev *sg, const ShadowQ<ALPHA> &q, int s, int p, float4 b,
                                             float &tz, float cur = 0.f) {
  const float4 a = q.a[s];
  float n = (float)(p + __float_as_int(b.z)) - a.x;
  float t = DIV ? clamp_t(n / a.y) : span_t(n, a.y, a.z);
  tz = __frcp_rn((1 - t) * b.x + t * a.w);
  if (tz != tz) return false;
  if (EZ && !(cur > tz)) return false;
  if (ALPHA) {
    const float4 c = q.c[s];
    const GroupDev &G = sg[q.g[s]];
    int len = G.alen;
    float lm1 = (float)(len - 1);
    int t1 = f2i((((1 - t) * c.z + t * c.x) * tz) * lm1);
    t1 = iabs_(t1) & (len - 1);
    int t2 = f2i((lm1 * ((1 - t) * c.w + t * c.y)) * tz);
    t2 = iabs_(t2) & (len - 1);
    if (!__ldg(G.amask + t1 + t2 * len)) return false;
  }
  return true;
}

// drawmin.c:71-76 / drawminalpha.c:83-97 for one pixel of span s
template <bool ALPHA, bool DIV = false>
__device__ __forceinline__ void shadow_pixel(float *map, const GroupDev *sg, const ShadowQ<ALPHA> &q, int s, int p) {
  const float4 b = q.b[s];
  float *addr = map + (size_t)(p + __float_as_int(b.y));
  // alpha-tested casters read the texel first: one that already holds a
  // depth <= tz (most of them, behind the opaque casters) skips the mask
  // lookup.  Texels only decrease, so any value read bounds the final one.
  float cur = 0.f;
  if (ALPHA) cur = __ldcg(addr);
  float tz;
  if (shadow_depth<ALPHA, DIV, ALPHA>(sg, q, s, p, b, tz, cur)) atomic_min_depth(addr, tz);
}

template <bool ALPHA>
__device__ __forceinline__ void shadow_warp_loop(const ShadowParams &S, const GroupDev *sg, ShadowQ<ALPHA> &q, int lane,
                                                 int ctr_list, int ctr_work) {
  // work items: row chunks of the casters when S.items is given, else casters
  const bool chunked = S.items != nullptr;
  uint32_t n = chunked ? S.ctr[ALPHA ? CTR_SH_ITEMS_A : CTR_SH_ITEMS] : S.ctr[ctr_list];
  uint32_t cap_items = S.cap_list * MAX_CHUNKS;
  int dim = S.sh.dim;
  const uint32_t per = claim_size(n, (uint32_t)S.claim_k);
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&S.ctr[ctr_work], per);
    base = __shfl_sync(FULL, base, 0);
    if (base >= n) break;
    ShadowLane<ALPHA> L;
    bool live = false;
    if ((uint32_t)lane < per && base + lane < n) {
      uint32_t idx = base + lane;
      if (chunked) {
        uint32_t item = S.items[ALPHA ? cap_items - 1 - idx : idx];
        uint32_t pos = item >> CHUNK_BITS;
        live = L.init_chunk(S, sg, S.list[ALPHA ? S.cap_list - 1 - pos : pos], (int)(item & (MAX_CHUNKS - 1)));
      } else {
        live = L.init(S, sg, S.list[ALPHA ? S.cap_list - 1 - idx : idx]);
      }
    }
    for (int round = 0; __any_sync(FULL, live); round++) {
      if (round == LOOP_LIMIT) {
        if (lane == 0) atomicOr(&S.ctr[CTR_LIMIT], 1u);
        break;
      }
      int cnt = 0;
      if (live) {
        cnt = L.emit(dim, q, lane, live);
        if (L.serial) {   // a span the queue cannot take: this lane draws it
          for (int j = 0; j < cnt; j++) shadow_pixel<ALPHA, true>(S.map, sg, q, lane, j);
          cnt = 0;
        }
      }
      fill_round(q, lane, cnt, L.pb, [&](int s, int p) { shadow_pixel<ALPHA>(S.map, sg, q, s, p); });
    }
  }
}

// Blocks per SM: the opaque casters fit 9 in 56 registers and the
// alpha-tested ones 7 in 72, neither spilling (204 -> 199 and 84 -> 80 us
// per cascade against 8 and 6 blocks).
template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 7 : 9) k_shadow_raster(ShadowParams S) {
  __shared__ GroupDev sg[64];
  __shared__ ShadowQ<ALPHA> qs[4];
  for (int i = threadIdx.x; i < S.ngroups; i += blockDim.x) sg[i] = S.groups[i];
  __syncthreads();
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  shadow_warp_loop<ALPHA>(S, sg, qs[w], lane, ALPHA ? CTR_SH_LIST_A : CTR_SH_LIST, ALPHA ? CTR_SH_WORK_A : CTR_SH_WORK);
}

}  // namespace axr
