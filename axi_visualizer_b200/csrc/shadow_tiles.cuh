// shadow_tiles.cuh -- the tiled shadow depth pass (sm_100a).
//
// The map is cut into STILE x STILE tiles.  k_shadow_setup writes one record
// per caster and counts a unit in every tile the caster can write;
//   k_shadow_scan   (one block) places each tile's units contiguously,
//                   opaque casters first, orders the non-empty tiles by
//                   their unit count, largest first, and gives a tile of n
//                   units ceil(n / slice) blocks;
//   k_shadow_bin    scatters the units (record indices) to their tiles;
//   k_shadow_sort   (optional) orders each tile's opaque units front first
//                   (nearest the light), by 256 depth classes;
//   k_shadow_tiles  runs the blocks of every tile: a block holds the tile's
//                   texels in shared memory and its warps claim the tile's
//                   units 32 at a time (the blocks of one tile share the
//                   claim counter, so units go in list order); they
//                   rasterize them with the span queue of the per-caster
//                   path, rows and spans clipped to the tile, test each texel
//                   against the span's depth floor before the exact depth,
//                   and take the minimum with shared-memory atomics.  The
//                   tile is written back with coalesced stores (a tile with
//                   several blocks: a global min update of each texel that
//                   changed).
// The depth minimum is independent of the order of the fragments, so the map
// equals the per-caster path's (and drawmin.c's serial one) bit for bit.
// When the units do not fit the queue, the same launches run the
// per-caster path instead (k_shadow_bin and the tile loops do nothing) and
// the host grows the queue for the next pass.
#pragma once
#include "kernels.cuh"

namespace axr {

constexpr int SHADOW_TILED_MAX_DIM = 8192;   // at most 65536 tiles: one block scans them
constexpr int SCAN_THREADS = 1024;

// Exclusive prefix sum over the block (SCAN_THREADS threads); returns the total.
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t &excl, uint32_t *warp_sums) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t ws = warp_sums[lane], wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(FULL, wi, o);
      if (lane >= o) wi += u;
    }
    warp_sums[lane] = wi - ws;
    if (lane == 31) warp_sums[32] = wi;
  }
  __syncthreads();
  excl = warp_sums[w] + incl - v;
  uint32_t total = warp_sums[32];
  __syncthreads();
  return total;
}

// One block: tile offsets (opaque units of a tile, then its alpha-tested
// ones), scatter cursors, the queue check, the tile order (by
// floor(log2(units)), largest first) and the prefix of the tiles' block
// counts in that order.
__global__ void __launch_bounds__(SCAN_THREADS) k_shadow_scan(ShadowParams S) {
  __shared__ uint32_t warp_sums[33];
  __shared__ uint32_t hist[32], base[32];
  int n = S.ntiles;
  int per = (n + SCAN_THREADS - 1) / SCAN_THREADS;
  int t0 = threadIdx.x * per, t1 = min(t0 + per, n);
  uint32_t sum = 0;
  for (int t = t0; t < t1; t++) sum += S.tcnt[t] + S.tcnt[n + t];
  if (threadIdx.x < 32) hist[threadIdx.x] = 0;
  uint32_t excl;
  uint32_t total = block_scan(sum, excl, warp_sums);
  for (int t = t0; t < t1; t++) {
    uint32_t o = S.tcnt[t], a = S.tcnt[n + t];
    S.toff[t] = excl;
    S.tcur[2 * t] = excl;
    S.tcur[2 * t + 1] = excl + o;
    excl += o + a;
    if (o + a) atomicAdd(&hist[__clz(o + a)], 1u);   // class 0 = the largest tiles
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t h = hist[threadIdx.x], incl = h;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(FULL, incl, o);
      if ((int)threadIdx.x >= o) incl += u;
    }
    base[threadIdx.x] = incl - h;
    if (threadIdx.x == 31) hist[0] = incl;   // non-empty tiles (hist is not read again)
  }
  __syncthreads();
  const uint32_t ntl = hist[0];
  for (int t = t0; t < t1; t++) {
    uint32_t c = S.tcnt[t] + S.tcnt[n + t];
    if (c) S.tord[atomicAdd(&base[__clz(c)], 1u)] = (uint32_t)t;
  }
  __syncthreads();
  // blocks per tile in tile order
  const uint32_t slice = (uint32_t)S.slice;
  int per2 = ((int)ntl + SCAN_THREADS - 1) / SCAN_THREADS;
  int i0 = threadIdx.x * per2, i1 = min(i0 + per2, (int)ntl);
  uint32_t hs = 0;
  for (int i = i0; i < i1; i++) {
    uint32_t t = S.tord[i];
    hs += (S.tcnt[t] + S.tcnt[n + t] + slice - 1) / slice;
  }
  uint32_t hex;
  uint32_t items = block_scan(hs, hex, warp_sums);
  for (int i = i0; i < i1; i++) {
    S.hpre[i] = hex;
    uint32_t t = S.tord[i];
    hex += (S.tcnt[t] + S.tcnt[n + t] + slice - 1) / slice;
  }
  if (threadIdx.x == 0) {
    S.hpre[ntl] = items;
    S.ctr[CTR_SH_TILES] = ntl;
    S.ctr[CTR_SH_ITEMS_TILED] = items;
    S.ctr[CTR_SH_UNITS_NEED] = total;
    if (total > S.cap_units) S.ctr[CTR_SH_OVERFLOW] = 1;
  }
}

// Scatters every caster's units: the record index, once per tile it can write.
__global__ void __launch_bounds__(256) k_shadow_bin(ShadowParams S) {
  if (S.ctr[CTR_SH_OVERFLOW]) return;
  uint32_t no = S.ctr[CTR_SH_LIST], na = S.ctr[CTR_SH_LIST_A];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < no + na; i += gridDim.x * blockDim.x) {
    bool alpha = i >= no;
    uint32_t r = alpha ? S.cap_list - 1 - (i - no) : i;
    uint4 a = S.rec[2 * (size_t)r];
    int x[3] = {unpack_x(a.x), unpack_x(a.y), unpack_x(a.z)};
    int tx0, tx1, ty0, ty1;
    if (!caster_tiles(x, unpack_y(a.x), unpack_y(a.z), S.sh.dim, tx0, tx1, ty0, ty1)) continue;
    const int lane = threadIdx.x & 31;
    for (int ty = ty0; ty <= ty1; ty++)
      for (int tx = tx0; tx <= tx1; tx++) {
        // one cursor increment for all lanes scattering into the same tile
        uint32_t key = 2 * (uint32_t)(ty * S.ntx + tx) + (alpha ? 1 : 0);
        unsigned peers = __match_any_sync(__activemask(), key);
        int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (lane == leader) b = atomicAdd(&S.tcur[key], (uint32_t)__popc(peers));
        b = __shfl_sync(peers, b, leader);
        S.units[b + __popc(peers & ((1u << lane) - 1u))] = r;
      }
  }
}

constexpr int SORT_CAP = 2048;   // units sorted together (a tile's units in runs of this many)

// Front-first order of each tile's opaque units: the key is the caster's
// largest 1/depth (as bits; larger = nearer the light), in 256 classes over
// the run's own range.  The order only affects how many texels the depth
// floor skips, never the map.
__global__ void __launch_bounds__(256) k_shadow_sort(ShadowParams S) {
  __shared__ uint32_t su[SORT_CAP], sk[SORT_CAP], so[SORT_CAP];
  __shared__ uint32_t hist[256];
  __shared__ uint32_t kmin, kmax;
  if (S.ctr[CTR_SH_OVERFLOW]) return;
  const uint32_t ntl = S.ctr[CTR_SH_TILES];
  for (uint32_t i = blockIdx.x; i < ntl; i += gridDim.x) {
    uint32_t t = S.tord[i];
    uint32_t u0 = S.toff[t], n = S.tcur[2 * t] - u0;
    for (uint32_t r0 = 0; r0 < n; r0 += SORT_CAP) {
      uint32_t m = min((uint32_t)SORT_CAP, n - r0);
      if (threadIdx.x == 0) { kmin = 0xffffffffu; kmax = 0; }
      hist[threadIdx.x] = 0;
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
        uint32_t u = S.units[u0 + r0 + j];
        uint4 a = S.rec[2 * (size_t)u], b = S.rec[2 * (size_t)u + 1];
        uint32_t k = max(a.w, max(b.x, b.y));
        su[j] = u;
        sk[j] = k;
        atomicMin(&kmin, k);
        atomicMax(&kmax, k);
      }
      __syncthreads();
      uint32_t span = kmax - kmin;
      for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
        uint32_t c = span ? (uint32_t)(((uint64_t)(kmax - sk[j]) * 255u) / span) : 0u;
        sk[j] = c;
        atomicAdd(&hist[c], 1u);
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        uint32_t v[8], s8 = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) { v[q] = hist[threadIdx.x * 8 + q]; s8 += v[q]; }
        uint32_t incl = s8;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t u = __shfl_up_sync(FULL, incl, o);
          if ((int)threadIdx.x >= o) incl += u;
        }
        uint32_t e = incl - s8;
#pragma unroll
        for (int q = 0; q < 8; q++) { hist[threadIdx.x * 8 + q] = e; e += v[q]; }
      }
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) so[atomicAdd(&hist[sk[j]], 1u)] = su[j];
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) S.units[u0 + r0 + j] = so[j];
      __syncthreads();
    }
  }
}

// One texel of a tile: the depth-floor test, then drawmin.c's depth and the
// minimum in shared memory (the per-caster path's atomic_min_depth).
template <bool ALPHA, bool DIV = false>
__device__ __forceinline__ void tile_pixel(int *tile, const GroupDev *sg, const ShadowQ<ALPHA> &q, int s, int p) {
  const float4 b = q.b[s];
  int off = p + __float_as_int(b.y);
  if (tile[off] < __float_as_int(b.w)) return;
  float tz;
  if (!shadow_depth<ALPHA, DIV>(sg, q, s, p, b, tz)) return;
  if (tz >= 0.f) atomicMin(tile + off, __float_as_int(tz));
  else atomicMax((unsigned int *)(tile + off), __float_as_uint(tz));
}

// Upper bounds of the texel bits of each 8 x 8 sub-block of the tile, as
// of now.  Texels only decrease, so a bound read at any time stays one; the
// warp recomputes them from the tile before it culls.
__device__ __forceinline__ void refresh_smax(const int *tile, int *smax, int lane) {
  int sb = lane >> 1, half = lane & 1;
  const int *p = tile + ((sb / SUBS) * 8 + half * 4) * TROW + (sb % SUBS) * 8;
  int m = INT_MIN;
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 8; c++) m = max(m, p[r * TROW + c]);
  m = max(m, __shfl_xor_sync(FULL, m, 1));
  if (!half) smax[sb] = m;
  __syncwarp();
}

// True when record r's caster cannot lower any texel of the tile: the
// smallest depth any of its pixels can store lies above the maxima of all
// the sub-blocks its rows and (widened) columns touch.  Its 1/z
// interpolants stay below zmax (1 + (rows + 10) 2^-24) -- each of the at
// most `rows` accumulated additions and the split vertex's z round by 2^-24
// of their value -- and a pixel's 1/z below that times (1 + 2^-24)^3, so a
// pixel's depth is above (1 / zmax) (1 - (rows + 11) 2^-24); the bound used
// takes (2^-17 + rows 2^-22) off an approximate reciprocal of zmax.
__device__ __forceinline__ bool unit_hidden(const ShadowParams &S, uint32_t r, const int *smax, int tx0, int tx1,
                                            int ty0, int ty1) {
  uint4 a = S.rec[2 * (size_t)r], b = S.rec[2 * (size_t)r + 1];
  float zmax = fmaxf(__uint_as_float(a.w), fmaxf(__uint_as_float(b.x), __uint_as_float(b.y)));
  int x[3] = {unpack_x(a.x), unpack_x(a.y), unpack_x(a.z)};
  int y1 = unpack_y(a.x), y3 = unpack_y(a.z);
  int rows = y3 - y1 + 1;
  if (!(zmax >= 0x1p-60f) || !(zmax <= 0x1p60f) || rows > 65536) return false;
  float rz;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rz) : "f"(zmax));
  float f = 1.0f - 0x1p-17f - (float)rows * 0x1p-22f;
  int lb = __float_as_int(__fmul_rn(rz, f)) + 1;
  int cx0, cx1, cy0, cy1;
  if (!caster_tiles(x, y1, y3, S.sh.dim, cx0, cx1, cy0, cy1)) return true;   // nothing on the map
  // the caster's texels in this tile (columns widened as in caster_tiles)
  int mn = min(x[0], min(x[1], x[2])), mx = max(x[0], max(x[1], x[2]));
  long long X = (long long)max(iabs_(mn), iabs_(mx)) + 2;
  int m = 1 + (int)(((long long)rows * X) >> 22);
  int c0 = max(mn - m, tx0), c1 = min(mx + m, tx1), r0 = max(y1, ty0), r1 = min(y3, ty1);
  if (c0 > c1 || r0 > r1) return true;
  int bmax = INT_MIN;
  for (int by = (r0 - ty0) >> SUB_LOG; by <= (r1 - ty0) >> SUB_LOG; by++)
    for (int bx = (c0 - tx0) >> SUB_LOG; bx <= (c1 - tx0) >> SUB_LOG; bx++) bmax = max(bmax, smax[by * SUBS + bx]);
  return bmax < lb;
}

// A warp's share of one tile's units [u0, u0 + n): claimed 32 at a time from
// the tile's claim counter (shared by the tile's blocks); units whose caster
// cannot lower the tile are dropped, the rest queued until 32 are ready, one
// per lane, rows and spans clipped to the tile.
template <bool ALPHA>
__device__ __forceinline__ void tile_units(const ShadowParams &S, const GroupDev *sg, int *tile, int *smax,
                                           uint32_t *ready, ShadowQ<ALPHA> &q, int lane, uint32_t u0, uint32_t n,
                                           uint32_t *claim, int tx0, int tx1, int ty0, int ty1) {
  const unsigned below = (1u << lane) - 1u;
  int have = 0;
  bool more = true;
  while (true) {
    if (more && have < 32) refresh_smax(tile, smax, lane);
    while (more && have < 32) {
      uint32_t b = 0;
      if (lane == 0) b = atomicAdd(claim, 32u);
      b = __shfl_sync(FULL, b, 0);
      if (b >= n) {
        more = false;
        break;
      }
      uint32_t r = 0;
      bool keep = false;
      if (b + lane < n) {
        r = S.units[u0 + b + lane];
        keep = !unit_hidden(S, r, smax, tx0, tx1, ty0, ty1);
      }
      unsigned kept = __ballot_sync(FULL, keep);
      if (keep) ready[have + __popc(kept & below)] = r;
      have += __popc(kept);
      __syncwarp();
    }
    if (have == 0) break;
    int take = min(have, 32);
    ShadowLane<ALPHA> L;
    bool live = false;
    if (lane < take) {
      L.init_rec(S, sg, ready[lane]);
      live = L.clip_rows(ty0, ty1);
    }
    __syncwarp();
    if (lane < have - take) ready[lane] = ready[32 + lane];
    have -= take;
    __syncwarp();
    for (int round = 0; __any_sync(FULL, live); round++) {
      if (round == LOOP_LIMIT) {
        if (lane == 0) atomicOr(&S.ctr[CTR_LIMIT], 1u);
        break;
      }
      int cnt = 0;
      if (live) {
        cnt = L.emit_tile(q, lane, tx0, tx1, ty0, ty1, smax, live);
        if (L.serial) {   // a span the queue cannot take: this lane draws it
          for (int j = 0; j < cnt; j++) tile_pixel<ALPHA, true>(tile, sg, q, lane, j);
          cnt = 0;
        }
      }
      fill_round(q, lane, cnt, L.pb, [&](int s, int p) { tile_pixel<ALPHA>(tile, sg, q, s, p); });
    }
  }
}

constexpr int TILE_THREADS = 128;
constexpr int TEXELS_PER_THREAD = STILE * STILE / TILE_THREADS;

// ALPHA = false: every non-empty tile's opaque units; true: the alpha-tested
// units of the tiles that have some (after the opaque launch).  After an
// overflow of the unit queue the launch runs the per-caster path instead.
template <bool ALPHA>
__global__ void __launch_bounds__(TILE_THREADS, ALPHA ? 6 : 8) k_shadow_tiles(ShadowParams S) {
  __shared__ GroupDev sg[64];
  __shared__ int tile[STILE * TROW];
  __shared__ ShadowQ<ALPHA> qs[TILE_THREADS / 32];
  __shared__ int smax[TILE_THREADS / 32][SUBS * SUBS];
  __shared__ uint32_t ready[TILE_THREADS / 32][64];
  __shared__ uint32_t s_k;
  for (int i = threadIdx.x; i < S.ngroups; i += blockDim.x) sg[i] = S.groups[i];
  __syncthreads();
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (S.ctr[CTR_SH_OVERFLOW]) {
    shadow_warp_loop<ALPHA>(S, sg, qs[w], lane, ALPHA ? CTR_SH_LIST_A : CTR_SH_LIST, ALPHA ? CTR_SH_WORK_A : CTR_SH_WORK);
    return;
  }
  const uint32_t ntl = S.ctr[CTR_SH_TILES], nitems = S.ctr[CTR_SH_ITEMS_TILED];
  const int dim = S.sh.dim;
  while (true) {
    if (threadIdx.x == 0) s_k = atomicAdd(&S.ctr[ALPHA ? CTR_SH_TILE_WORK_A : CTR_SH_TILE_WORK], 1u);
    __syncthreads();
    uint32_t k = s_k;
    if (k >= nitems) break;
    // the tile of block k: the last position i with hpre[i] <= k
    uint32_t lo = 0, hi = ntl - 1;
    while (lo < hi) {
      uint32_t mid = (lo + hi + 1) >> 1;
      if (S.hpre[mid] <= k) lo = mid; else hi = mid - 1;
    }
    uint32_t t = S.tord[lo];
    bool alone = S.hpre[lo + 1] - S.hpre[lo] == 1;
    uint32_t u0 = ALPHA ? S.tcur[2 * t] : S.toff[t];          // after binning: end of the opaque units
    uint32_t n = ALPHA ? S.tcur[2 * t + 1] - u0 : S.tcur[2 * t] - u0;
    uint32_t *claim = S.tclaim + 2 * t + (ALPHA ? 1 : 0);
    // nothing left to claim (uniform: thread 0's read is shared after the barrier)
    if (threadIdx.x == 0) s_k = n == 0 || *(volatile uint32_t *)claim >= n;
    __syncthreads();
    if (s_k) {
      __syncthreads();
      continue;
    }
    int tx0 = (int)(t % (uint32_t)S.ntx) * STILE, ty0 = (int)(t / (uint32_t)S.ntx) * STILE;
    int tx1 = min(tx0 + STILE, dim) - 1, ty1 = min(ty0 + STILE, dim) - 1;
    int init[TEXELS_PER_THREAD];
#pragma unroll
    for (int j = 0; j < TEXELS_PER_THREAD; j++) {
      int i = threadIdx.x + j * TILE_THREADS;
      int x = tx0 + (i & (STILE - 1)), y = ty0 + (i >> STILE_LOG);
      init[j] = (x < dim && y < dim) ? __float_as_int(S.map[(size_t)y * dim + x]) : 0;
      tile[(i >> STILE_LOG) * TROW + (i & (STILE - 1))] = init[j];
    }
    __syncthreads();
    tile_units<ALPHA>(S, sg, tile, smax[w], ready[w], qs[w], lane, u0, n, claim, tx0, tx1, ty0, ty1);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < TEXELS_PER_THREAD; j++) {
      int i = threadIdx.x + j * TILE_THREADS;
      int x = tx0 + (i & (STILE - 1)), y = ty0 + (i >> STILE_LOG);
      int v = tile[(i >> STILE_LOG) * TROW + (i & (STILE - 1))];
      if (x < dim && y < dim) {
        float *dst = S.map + (size_t)y * dim + x;
        if (alone) *dst = __int_as_float(v);
        else if (v != init[j]) atomic_min_depth(dst, __int_as_float(v));
      }
    }
    __syncthreads();
  }
}

}  // namespace axr
