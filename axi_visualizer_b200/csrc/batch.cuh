// batch.cuh -- many views in one persistent launch (sm_100a).
//
// One cooperative kernel renders a batch of views of uneven size -- shaded
// perspective views (main view, cubemap faces) and depth-only orthographic
// views (shadow cascades) -- through five phases separated by grid barriers:
//   0 clear depth / visibility words / counters (and colour, where asked) of every view
//   1 triangle setup of every view (perspective and orthographic)
//   2 coarse binning, small-triangle raster and shadow-map raster
//   3 tiled raster of the large triangles' (triangle, tile) units
//   4 shading of every shaded view's pixels (sampling the batch's cascades)
// Work of all views shares each phase: warps move from one view's queue to
// the next, so small views fill the machine together with large ones.  The
// per-phase device functions are the ones the single-view kernels use, so a
// view rendered in a batch is bit-identical to the same view rendered alone.
#pragma once
#include "kernels.cuh"

namespace axr {

enum { VIEW_SHADED = 0, VIEW_DEPTH = 1, VIEW_SKIP = 2 };

constexpr int BATCH_TABLE = 64;   // group-table entries staged in shared memory

struct BatchView {
  int kind;
  int w, h;          // framebuffer, or map side
  int goff;          // first entry of the view's segment of the group tables
  int clear_rgb;     // shaded: colour planes := bg before drawing
  uint16_t bg[4];
  DrawParams dp;     // shaded views
  ShadowParams sp;   // depth views
};

struct BatchParams {
  const BatchView *views;
  int nviews;
  const GroupDev *groups_draw, *groups_shadow;
  int ngroups;
  uint32_t *bar;     // [0] arrivals, [1] generation, [2] barrier error, [3] blocks done,
                     // [4..15] six u64 globaltimer stamps: start, after phases 0-3, end
  uint32_t nblocks;    // blocks the grid barrier waits for
  long spin_limit;     // polls before a waiting block gives up
};

constexpr int BAR_WORDS = 16;

__device__ __forceinline__ void stamp(uint32_t *bar, int k) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    reinterpret_cast<uint64_t *>(bar + 4)[k] = t;
  }
}

constexpr long BARRIER_SPIN_LIMIT = 1L << 26;   // ~6 s of polling, then give up

// Grid-wide barrier of a cooperative launch (all blocks are co-resident).  A
// block that polls longer than spin_limit (BARRIER_SPIN_LIMIT by default)
// records an error and the kernel ends; returns false when the batch must
// stop.
__device__ __forceinline__ bool grid_sync(uint32_t *bar, uint32_t nblocks, long spin_limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t *vgen = bar + 1;
    uint32_t gen = *vgen;
    __threadfence();
    uint32_t arrived = atomicAdd(bar, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long it = 0;
      while (*vgen == gen) {
        if (++it > spin_limit) {
          atomicOr(bar + 2, 1u);
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    ok = *(volatile uint32_t *)(bar + 2) == 0;
  }
  __syncthreads();
  return ok;
}

union WarpQueue {
  VisQ<false> vo;
  VisQ<true> va;
  ShadowQ<false> so;
  ShadowQ<true> sa;
};

// ---- the phases, shared by the persistent kernel and the phased graph

__device__ __forceinline__ void load_tables(const BatchParams &B, GroupDev *sgd, GroupDev *sgs) {
  for (int i = threadIdx.x; i < B.ngroups; i += blockDim.x) {
    sgd[i] = B.groups_draw[i];
    sgs[i] = B.groups_shadow[i];
  }
  __syncthreads();
}

// phase 0: clears (clearzb.c regions) and visibility words, counters
__device__ __forceinline__ void batch_clear(const BatchParams &B, int tid, int step) {
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_SKIP) continue;
    if (tid < CTR_N) (V.kind == VIEW_SHADED ? V.dp.ctr : V.sp.ctr)[tid] = 0;
    if (V.kind == VIEW_SHADED) {
      int W = V.w, H = V.h, bw = (W / 4) * 4, bh = (H / 4) * 4;
      for (int i = tid; i < W * H; i += step) {
        int y = i / W, x = i - y * W;
        float d = V.dp.db[i];
        if (y < bh && x < bw) {
          d = 65535.f;
          V.dp.db[i] = d;
        } else if (V.clear_rgb) {
          d = 0.f;              // outside the clearzb.c region: the value of a new frame buffer
          V.dp.db[i] = d;
        }
        V.dp.keys[i] = ((uint64_t)depth_key(d) << 32) | 0xffffffffull;
        if (V.clear_rgb) {
          V.dp.ro[i] = V.bg[0];
          V.dp.go[i] = V.bg[1];
          V.dp.bo[i] = V.bg[2];
        }
      }
    } else {
      int D = V.w, bd = (D / 16) * 16;
      for (int i = tid; i < bd * bd; i += step) {
        int y = i / bd, x = i - y * bd;
        V.sp.map[(size_t)D * y + x] = 65535.f;
      }
    }
  }
}

// phase 1: setup of every view
__device__ __forceinline__ void batch_setup(const BatchParams &B, const GroupDev *sgd, const GroupDev *sgs, int first,
                                            int step) {
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_SHADED) setup_phase(V.dp, sgd + V.goff, first, step);
    else if (V.kind == VIEW_DEPTH) shadow_setup_phase(V.sp, sgs + V.goff, first, step);
  }
}

// phase 2 for one material kind: (opaque only) coarse units, then the depth
// maps' casters, then the small triangles of the shaded views
template <bool ALPHA>
__device__ __forceinline__ void batch_raster(const BatchParams &B, const GroupDev *sgd, const GroupDev *sgs,
                                             ShadowQ<ALPHA> &sq, VisQ<ALPHA> &vq, int lane) {
  if (!ALPHA)
    for (int v = 0; v < B.nviews; v++)
      if (B.views[v].kind == VIEW_SHADED) coarse_loop(B.views[v].dp, sgd + B.views[v].goff, lane);
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_DEPTH)
      shadow_warp_loop<ALPHA>(V.sp, sgs + V.goff, sq, lane, ALPHA ? CTR_SH_LIST_A : CTR_SH_LIST,
                              ALPHA ? CTR_SH_WORK_A : CTR_SH_WORK);
  }
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_SHADED) raster_small_loop<ALPHA>(V.dp, sgd + V.goff, vq, lane);
  }
}

// phase 4: shading, tile by tile (16 x NT/16 pixels per block and tile);
// NRM: some view draws a normal-mapped material (else the shade without
// that core, which runs with fewer registers)
template <int NT, bool NRM>
__device__ __forceinline__ void batch_shade(const BatchParams &B, const GroupDev *sgd, ShadeSmem<NT> &sm) {
  constexpr int TH = NT / 16;
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind != VIEW_SHADED) continue;
    int tw = (V.w + 15) / 16, th = (V.h + TH - 1) / TH;
    for (int t = blockIdx.x; t < tw * th; t += gridDim.x)
      shade_tile<NT, NRM>(V.dp, sgd + V.goff, (t % tw) * 16, (t / tw) * TH, sm);
  }
}

template <bool NRM>
__global__ void __launch_bounds__(128, 4) k_batch(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE], sgs[BATCH_TABLE];
  __shared__ union U { WarpQueue wq[4]; ShadeSmem<128> sh; } u;   // phases 2-3 / phase 4
  WarpQueue *wq = u.wq;
  load_tables(B, sgd, sgs);
  stamp(B.bar, 0);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int first = blockIdx.x * blockDim.x, step = gridDim.x * blockDim.x;
  const int tid = first + threadIdx.x;
  const int gw = tid >> 5, nw = step >> 5;
  WarpQueue &q = wq[w];

  batch_clear(B, tid, step);
  if (!grid_sync(B.bar, B.nblocks, B.spin_limit)) return;
  stamp(B.bar, 1);

  batch_setup(B, sgd, sgs, first, step);
  if (!grid_sync(B.bar, B.nblocks, B.spin_limit)) return;
  stamp(B.bar, 2);

  // phase 2: coarse units, small triangles, shadow maps (alpha-tested first)
  batch_raster<true>(B, sgd, sgs, q.sa, q.va, lane);
  batch_raster<false>(B, sgd, sgs, q.so, q.vo, lane);
  if (!grid_sync(B.bar, B.nblocks, B.spin_limit)) return;
  stamp(B.bar, 3);

  // phase 3: large triangles, tile by tile
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind != VIEW_SHADED) continue;
    raster_tiled_loop<true>(V.dp, sgd + V.goff, q.va, lane);
    raster_tiled_loop<false>(V.dp, sgd + V.goff, q.vo, lane);
    fallback_loop(V.dp, sgd + V.goff, q.vo, q.va, lane, gw, nw);
  }
  if (!grid_sync(B.bar, B.nblocks, B.spin_limit)) return;
  stamp(B.bar, 4);

  batch_shade<128, NRM>(B, sgd, u.sh);
  // the last block to finish stamps the end
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(B.bar + 3, 1u) == B.nblocks - 1) {
      uint64_t t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      reinterpret_cast<uint64_t *>(B.bar + 4)[5] = t;
    }
  }
}

// ---- phased form: the same phases as separate kernels, captured in one
// graph; each kernel runs at its own occupancy, and the alpha-tested
// rasterizers run on a parallel branch of the graph.  No grid barriers.

__global__ void __launch_bounds__(256) kb_clear(BatchParams B) {
  batch_clear(B, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(256) kb_setup(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE], sgs[BATCH_TABLE];
  load_tables(B, sgd, sgs);
  batch_setup(B, sgd, sgs, blockIdx.x * blockDim.x, gridDim.x * blockDim.x);
}

template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 6 : 8) kb_raster(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE], sgs[BATCH_TABLE];
  __shared__ union Q { ShadowQ<ALPHA> s; VisQ<ALPHA> v; } qs[4];
  load_tables(B, sgd, sgs);
  Q &q = qs[threadIdx.x >> 5];
  batch_raster<ALPHA>(B, sgd, sgs, q.s, q.v, threadIdx.x & 31);
}

template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 6 : 8) kb_tiled(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE], sgs[BATCH_TABLE];
  __shared__ VisQ<ALPHA> qs[4];
  load_tables(B, sgd, sgs);
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_SHADED) raster_tiled_loop<ALPHA>(V.dp, sgd + V.goff, qs[threadIdx.x >> 5], threadIdx.x & 31);
  }
}

__global__ void __launch_bounds__(128) kb_fallback(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE], sgs[BATCH_TABLE];
  __shared__ VisQ<false> qo[4];
  __shared__ VisQ<true> qa[4];
  load_tables(B, sgd, sgs);
  int w = threadIdx.x >> 5, tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int v = 0; v < B.nviews; v++) {
    const BatchView &V = B.views[v];
    if (V.kind == VIEW_SHADED)
      fallback_loop(V.dp, sgd + V.goff, qo[w], qa[w], threadIdx.x & 31, tid >> 5, (gridDim.x * blockDim.x) >> 5);
  }
}

template <bool NRM>
__global__ void __launch_bounds__(256, 4) kb_shade(BatchParams B) {
  __shared__ GroupDev sgd[BATCH_TABLE];
  __shared__ ShadeSmem<256> sm;
  for (int i = threadIdx.x; i < B.ngroups; i += blockDim.x) sgd[i] = B.groups_draw[i];
  __syncthreads();
  batch_shade<256, NRM>(B, sgd, sm);
}

}  // namespace axr
