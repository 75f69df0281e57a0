// axr.cu -- libaxr.so: handle, device memory and the C ABI of include/axr.h.
//
// Layout in HBM per handle: framebuffers as the reference keeps them (three
// uint16 planes and a float depth plane, [h][w]) plus one 64-bit visibility
// word per pixel; per material group the vertex streams (xyz, normal, uv,
// light I as packed float triplets/pairs, 3 vertices per triangle) and the
// texture planes (mip chain smallest level first); work queues sized by the
// triangle count (small/large lists) and a grow-only tile-unit queue.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <limits.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/axr.h"
#include "batch.cuh"
#include "shadow_tiles.cuh"

using namespace axr;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) return fail(AXR_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

struct Group {
  float *xyz = nullptr, *vn = nullptr, *uv = nullptr, *li = nullptr;
  ushort4 *tex = nullptr;     // interleaved (R, G, B, 0) texels
  int ntris = 0, tri_base = 0, tex_size = 0, mip_side = 0;
  long ntexels = 0;
  float mip_bias = 0.f;       // mipBias of the trilinear level selection (axr_set_mip_bias)
  int nmap = -1;              // normal map of the normal-mapped materials (axr_set_normal_material)
  float roughness = 0.f;
  int metal = 0;
};

struct NormalMap {
  uchar4 *texels = nullptr;   // (R, G, B, unused)
  long n = 0;
};

struct Alpha {
  uint8_t *mask = nullptr;
  uint8_t *quad = nullptr;    // 2x2 bilinear footprint of each texel as 4 bits
  int side = 0;
};

// A shadow map has its own stream, scratch (caster list, counters) and group
// table, so cascades render concurrently with each other and with the main
// view's visibility pass; ev_write orders the shade pass after the map's last
// writer, ev_read orders the next writer after the map's last reader.
struct Shadow {
  float *map = nullptr;
  int dim = 0;
  float scale = 1;
  float pos[3] = {0, 0, 0};
  float vv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  cudaStream_t st = nullptr;
  cudaEvent_t ev_write = nullptr, ev_read = nullptr;
  uint32_t *list = nullptr, *ctr = nullptr, *items = nullptr;
  uint32_t cap = 0;          // casters the list (and the records) hold
  bool items_ready = false;  // row-chunk items allocated (per-caster path)
  GroupDev *tab = nullptr;
  // tiled pass: caster records, tile offsets/cursors/order, units; the
  // per-tile counts sit right after the CTR_N counters (one clear for both)
  uint4 *rec = nullptr;
  uint32_t *tiles = nullptr, *units = nullptr;
  uint32_t cap_units = 0;
  int ntx = 0;
  int64_t overflows = 0;      // tiled passes that overflowed the unit queue
  uint32_t last_units = 0;    // units the last checked tiled pass needed
  uint32_t last_casters[2] = {0, 0};   // opaque, alpha-tested casters of the last checked pass
  // counters of the last two passes (pinned, each with its event), checked
  // once their pass has finished
  uint32_t *h_ring = nullptr;
  cudaEvent_t ev_ctr[2] = {nullptr, nullptr};
  bool pend[2] = {false, false};
  int last_slot = 1;
};

constexpr int MAX_GROUPS = 64;
constexpr int MAX_SHADOWS = 16;
// 3 * ntris + 3 stays an int: the vertex kernels round v_end up to a quad
constexpr int MAX_GROUP_TRIS = (INT_MAX - 3) / 3;

}  // namespace

struct axr_ctx {
  int device = 0, w = 0, h = 0, sms = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t s_alpha = nullptr;            // alpha-tested rasterizers of a drawAll
  cudaEvent_t ev_setup = nullptr, ev_coarse = nullptr, ev_alpha = nullptr;
  std::vector<Group> groups;
  std::vector<Alpha> alphas;
  std::vector<NormalMap> nmaps;
  int total_tris = 0;
  float sscale = 1, cax = 1, cay = 1;
  float pos[3] = {0, 0, 0};
  float vm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  float lint[3] = {1, 1, 1}, ldir[3] = {0, -1, 0};
  float amb = 0.2f;
  uint16_t *ro = nullptr, *go = nullptr, *bo = nullptr;
  float *db = nullptr;
  uint64_t *keys = nullptr;
  uint32_t *small_list = nullptr, *large_list = nullptr, *items = nullptr;
  float2 *mipc = nullptr;                    // per-triangle mip level of the last drawAll's setup
  uint32_t cap_list = 0;
  uint2 *units = nullptr;
  uint32_t cap_units = 0;
  uint32_t *ctr = nullptr;
  // counters of the last two drawAlls (pinned, each with its event); checked
  // without blocking once their frame has finished
  uint32_t *h_ring = nullptr;
  cudaEvent_t ev_ctr[2] = {nullptr, nullptr};
  bool pend[2] = {false, false};
  int last_slot = 1;
  uint32_t *h_ctr = nullptr;  // counters of the last checked drawAll (lastStats)
  GroupDev *d_groups = nullptr;
  Shadow shadows[MAX_SHADOWS];
  int64_t last_kernels = 0;
  // asynchronous frame read-back: two device staging slots, a copy stream
  struct ReadSlot {
    uint8_t *stage = nullptr;
    cudaEvent_t staged = nullptr, done = nullptr;
    int64_t seq = -1;
    bool busy = false;
  } rd[2];
  cudaStream_t s_copy = nullptr;
  int64_t read_seq = 0;
  // pinned staging of the per-call group tables: a host-to-device copy from
  // pageable memory would first synchronise its stream, i.e. wait for the
  // previous frame; a slot is reused only after the copy that read it ran
  struct Stage {
    GroupDev *h = nullptr;
    cudaEvent_t ev = nullptr;
    bool used = false;
  } stage[8];
  int stage_next = 0;
  // vertex stage: ev_geo follows the last geometry write on `stream`
  // (rotate/translate/copyTo), which shadow passes on their own streams wait
  // for; the light table of vertLight is staged through pinned memory
  cudaEvent_t ev_geo = nullptr;
  float *d_lights = nullptr, *h_lights = nullptr;
  size_t lights_cap = 0;
  cudaEvent_t ev_lights = nullptr;
  bool lights_used = false;
  uint16_t *post[3] = {nullptr, nullptr, nullptr};   // dof's gather target (SSRO/SSGO/SSBO)
  uint16_t *bloom = nullptr;                           // the bloom's 9 half-resolution planes
  int light_blocks = 4;                      // resident 256-thread blocks of k_vert_light per SM
  // launch accounting and optional per-kernel CUDA-event timing
  int64_t launches = 0;
  int min_chunk = MIN_CHUNK;
  // resident blocks per SM of the persistent rasterizers (their grids are
  // one full wave): small opaque / alpha, tiled opaque / alpha, casters
  // opaque / alpha
  int occ[6] = {8, 6, 8, 6, 8, 6};
  int shadow_mode = 0;                       // 0: per caster; tiled shadow pass where the map allows it
                                             // (2: units front first, 1: as binned)
  int shadow_slice = 512;                    // units per block of a tile in the tiled pass
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  struct Pending { const char *name; cudaEvent_t a, b; };
  std::vector<Pending> tpend;
  struct Acc { std::string name; double ms; int64_t n; };
  std::vector<Acc> tacc;
};

namespace {

// list positions travel in work items as position << CHUNK_BITS | chunk
constexpr uint32_t MAX_LIST = 0xffffffffu >> CHUNK_BITS;

int ensure_lists(axr_ctx *c) {
  uint32_t need = (uint32_t)std::max(c->total_tris, 1);
  if (need <= c->cap_list) return 0;
  if (need > MAX_LIST) return fail(AXR_EINVAL, "more than %u triangles", MAX_LIST);
  uint32_t cap = (uint32_t)std::max<uint64_t>(need, std::min<uint64_t>(2ull * c->cap_list, MAX_LIST));
  cudaStreamSynchronize(c->stream);
  cudaFree(c->small_list); cudaFree(c->large_list); cudaFree(c->items); cudaFree(c->mipc);
  c->small_list = c->large_list = c->items = nullptr;
  c->mipc = nullptr;
  c->cap_list = 0;
  if (cudaMalloc(&c->small_list, sizeof(uint32_t) * cap) != cudaSuccess ||
      cudaMalloc(&c->large_list, sizeof(uint32_t) * cap) != cudaSuccess ||
      cudaMalloc(&c->items, sizeof(uint32_t) * cap * MAX_CHUNKS) != cudaSuccess ||
      cudaMalloc(&c->mipc, sizeof(float2) * cap) != cudaSuccess)
    return fail(AXR_ENOMEM, "triangle lists of %u entries", cap);
  c->cap_list = cap;
  return 0;
}

int grow_units(axr_ctx *c, uint32_t need) {
  if (need <= c->cap_units) return 0;
  uint64_t cap = std::max<uint64_t>((uint64_t)need + need / 4, (uint64_t)c->cap_units * 2);
  if (cap > 0x7fffffffull) cap = 0x7fffffffull;
  cudaFree(c->units);
  c->units = nullptr;
  if (cudaMalloc(&c->units, sizeof(uint2) * cap) != cudaSuccess)
    return fail(AXR_ENOMEM, "tile-unit queue of %llu entries", (unsigned long long)cap);
  c->cap_units = (uint32_t)cap;
  return 0;
}

void collect_times(axr_ctx *c);

// Reads the counters of the last drawAll; grows the unit queue after an
// overflow (that frame was completed by the fallback kernel).
int sync_all(axr_ctx *c);

// Checks the counters of drawAll slot k: a raster loop at its safety limit is
// an error; an overflowed unit queue (that frame was completed by the
// fallback kernel) grows for the next frames.  blocking = wait for the frame;
// otherwise an unfinished frame is left for a later check.
int check_slot(axr_ctx *c, int k, bool blocking) {
  if (!c->pend[k]) return 0;
  if (blocking) {
    CK(cudaEventSynchronize(c->ev_ctr[k]));
  } else {
    cudaError_t e = cudaEventQuery(c->ev_ctr[k]);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return fail(AXR_ECUDA, "drawAll: %s", cudaGetErrorString(e));
  }
  c->pend[k] = false;
  const uint32_t *h = c->h_ring + k * CTR_N;
  memcpy(c->h_ctr, h, sizeof(uint32_t) * CTR_N);
  if (h[CTR_LIMIT]) return fail(AXR_ECUDA, "a raster loop reached its safety limit; the frame is incomplete");
  if (h[CTR_OVERFLOW] && h[CTR_UNITS_RESERVED] > c->cap_units) {
    CK(cudaStreamSynchronize(c->stream));   // frames in flight still use the old queue
    return grow_units(c, h[CTR_UNITS_RESERVED]);
  }
  return 0;
}

int grow_shadow_units(Shadow &sm, uint32_t need) {
  if (need <= sm.cap_units) return 0;
  uint64_t cap = std::max<uint64_t>((uint64_t)need + need / 4, (uint64_t)sm.cap_units * 2);
  if (cap > 0x7fffffffull) cap = 0x7fffffffull;
  cudaFree(sm.units);
  sm.units = nullptr;
  sm.cap_units = 0;
  if (cudaMalloc(&sm.units, sizeof(uint32_t) * cap) != cudaSuccess)
    return fail(AXR_ENOMEM, "shadow tile-unit queue of %llu entries", (unsigned long long)cap);
  sm.cap_units = (uint32_t)cap;
  return 0;
}

// Checks the counters of shadow pass slot k of map sm, as check_slot does
// for drawAll: a raster loop at its safety limit is an error; an overflowed
// unit queue (that pass was drawn by the per-caster path) grows.
int check_shadow_slot(Shadow &sm, int k, bool blocking) {
  if (!sm.pend[k]) return 0;
  if (blocking) {
    CK(cudaEventSynchronize(sm.ev_ctr[k]));
  } else {
    cudaError_t e = cudaEventQuery(sm.ev_ctr[k]);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return fail(AXR_ECUDA, "shadowMap: %s", cudaGetErrorString(e));
  }
  sm.pend[k] = false;
  const uint32_t *h = sm.h_ring + k * CTR_N;
  if (h[CTR_LIMIT]) return fail(AXR_ECUDA, "a shadow raster loop reached its safety limit; the map is incomplete");
  sm.last_units = h[CTR_SH_UNITS_NEED];
  sm.last_casters[0] = h[CTR_SH_LIST];
  sm.last_casters[1] = h[CTR_SH_LIST_A];
  if (h[CTR_SH_OVERFLOW]) sm.overflows++;
  if (h[CTR_SH_OVERFLOW] && h[CTR_SH_UNITS_NEED] > sm.cap_units) {
    CK(cudaStreamSynchronize(sm.st));   // passes in flight still use the old queue
    return grow_shadow_units(sm, h[CTR_SH_UNITS_NEED]);
  }
  return 0;
}

// Checks the shadow passes of every map, oldest first; without blocking,
// unfinished passes are left for a later check.
int settle_shadows(axr_ctx *c, bool blocking) {
  for (auto &sm : c->shadows) {
    if (!sm.h_ring) continue;
    int older = 1 - sm.last_slot;
    int rc = check_shadow_slot(sm, older, blocking);
    if (!rc && !sm.pend[older]) rc = check_shadow_slot(sm, sm.last_slot, blocking);
    if (rc) return rc;
  }
  return 0;
}

// Checks every drawAll and shadow pass that has finished, oldest first (no waiting).
int settle_ready(axr_ctx *c) {
  int older = 1 - c->last_slot;
  int rc = check_slot(c, older, false);
  if (!rc && !c->pend[older]) rc = check_slot(c, c->last_slot, false);
  if (!rc) rc = settle_shadows(c, false);
  return rc;
}

int settle(axr_ctx *c);

// Before queueing more work: checks finished frames without waiting (with
// per-kernel timing on, everything is synchronised as before).
int settle_next(axr_ctx *c) {
  if (!c->tpend.empty()) return settle(c);
  return settle_ready(c);
}

int settle(axr_ctx *c) {
  if (!c->tpend.empty()) {
    int rc = sync_all(c);
    if (rc) return rc;
    collect_times(c);
  }
  int rc = check_slot(c, 1 - c->last_slot, true);
  if (!rc) rc = check_slot(c, c->last_slot, true);
  if (!rc) rc = settle_shadows(c, true);
  return rc;
}

int check_ctx(axr_ctx *c) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  CK(cudaSetDevice(c->device));
  return 0;
}

cudaEvent_t ev_get(axr_ctx *c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Launches one kernel through `f`, counting it and, when timing is on,
// bracketing it with events on the handle's stream.
template <class F>
void launch(axr_ctx *c, cudaStream_t st, const char *name, F f) {
  cudaEvent_t a = nullptr;
  if (c->timing) {
    a = ev_get(c);
    cudaEventRecord(a, st);
  }
  f();
  c->launches++;
  if (c->timing) {
    cudaEvent_t b = ev_get(c);
    cudaEventRecord(b, st);
    c->tpend.push_back({name, a, b});
  }
}

// Waits for every stream of the handle.
int sync_all(axr_ctx *c) {
  CK(cudaStreamSynchronize(c->stream));
  if (c->s_alpha) CK(cudaStreamSynchronize(c->s_alpha));
  for (auto &sm : c->shadows)
    if (sm.st) CK(cudaStreamSynchronize(sm.st));
  return 0;
}

// Folds the finished event pairs into the per-kernel totals.
void collect_times(axr_ctx *c) {
  for (auto &p : c->tpend) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      bool found = false;
      for (auto &acc : c->tacc)
        if (acc.name == p.name) { acc.ms += ms; acc.n++; found = true; break; }
      if (!found) c->tacc.push_back({p.name, (double)ms, 1});
    }
    c->ev_pool.push_back(p.a);
    c->ev_pool.push_back(p.b);
  }
  c->tpend.clear();
}

template <class T>
int upload(axr_ctx *c, T **dst, const T *src, size_t n) {
  if (cudaMalloc(dst, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess)
    return fail(AXR_ENOMEM, "device allocation of %zu bytes", sizeof(T) * n);
  if (n) CK(cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, c->stream));
  return 0;
}

bool is_pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }

ViewDev make_view(const axr_ctx *c) {
  ViewDev v;
  v.w = c->w; v.h = c->h;
  memcpy(v.pos, c->pos, sizeof v.pos);
  memcpy(v.vv, c->vm, sizeof v.vv);
  v.sscale = c->sscale; v.cax = c->cax; v.cay = c->cay;
  return v;
}

int grid_for(axr_ctx *c, long n, int block, int per_sm) {
  long g = (n + block - 1) / block;
  long cap = (long)c->sms * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Builds the per-call group table (host copy).
// float -> int as the kernels convert (truncation, saturation, NaN -> 0)
int host_f2i(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x <= -2147483648.0f) return INT_MIN;
  return (int)x;
}

// The specular powers of av_draw_normmap.c:127-146 for a roughness, the same
// for every pixel of a draw: int specPow = exp2(12*(1.f - roughness)) and
// (int)half_sqrt((float)specPow), exp2 and half_sqrt correctly rounded
// (the double result rounded once; sqrtf).
void normal_powers(float roughness, int &p, int &p2) {
  float e = 12.f * (1.f - roughness);
  p = host_f2i((float)exp2((double)e));
  p2 = host_f2i(sqrtf((float)p));
}

int group_table(axr_ctx *c, const int32_t *flags, const int32_t *alpha_index, const uint8_t *enabled_mask,
                bool mask_means_enabled, int ngroups, GroupDev *tab) {
  memset(tab, 0, sizeof(GroupDev) * MAX_GROUPS);
  for (int g = 0; g < ngroups; g++) {
    const Group &G = c->groups[g];
    GroupDev &d = tab[g];
    d.xyz = G.xyz; d.vn = G.vn; d.uv = G.uv; d.li = G.li;
    d.tex = G.tex;
    d.ntris = G.ntris; d.tri_base = G.tri_base; d.tex_size = G.tex_size;
    d.flags = flags ? flags[g] : 0;
    d.mip_bias = G.mip_bias;
    bool on = true;
    if (enabled_mask) on = mask_means_enabled ? enabled_mask[g] != 0 : enabled_mask[g] == 0;
    d.enabled = on ? 1 : 0;
    if ((d.flags & F_MULTI) && (d.flags & F_ALPHA)) d.flags &= ~F_MULTI;   // the alpha material wins (Ops0.py:521-533)
    if (d.flags & F_MULTI) {
      // av_draw_multi.c samples this group's texture and the next three groups' at
      // this group's side (the reference has no mip or shadow lookup in it)
      d.flags &= ~(F_MIP | F_SHADOW);
      if (G.mip_side != 0) return fail(AXR_EINVAL, "group %d: the multi material needs a single-level texture", g);
      if (g + 3 >= ngroups)
        return fail(AXR_EINVAL, "group %d: the multi material blends the textures of groups %d..%d, which do not exist",
                    g, g + 1, g + 3);
      for (int k = 1; k <= 3; k++)
        if (c->groups[g + k].ntexels < (long)G.tex_size * G.tex_size)
          return fail(AXR_EINVAL, "group %d: texture of group %d has fewer than %d x %d texels", g, g + k,
                      G.tex_size, G.tex_size);
    }
    if (d.flags & F_NORMAL) {
      // av_draw_normmap*.c: the normal map is tapped at the texture's texel
      // indices; the alpha-tested variant has no mip level (Ops.py:772-805)
      if ((d.flags & F_MULTI) || ((d.flags & F_ALPHA) && (d.flags & F_MIP)))
        return fail(AXR_EINVAL, "group %d: the normal-mapped material combines with either alpha or mip, not multi", g);
      if (G.nmap < 0 || G.nmap >= (int)c->nmaps.size())
        return fail(AXR_ESTATE, "group %d: normal-mapped material with no normal map set", g);
      if (c->nmaps[G.nmap].n < G.ntexels)
        return fail(AXR_EINVAL, "group %d: normal map has %ld texels, the texture %ld", g, c->nmaps[G.nmap].n,
                    G.ntexels);
      d.nm = c->nmaps[G.nmap].texels;
      normal_powers(G.roughness, d.spec_pow, d.spec_pow2);
      d.is_metal = G.metal ? 1 : 0;
    }
    if ((d.flags & F_MIP) && G.mip_side == 0)
      return fail(AXR_EINVAL, "group %d: mip flag on a group added without a mip chain", g);
    if (!(d.flags & F_MIP) && G.mip_side != 0)
      return fail(AXR_EINVAL, "group %d: group has a mip chain but the mip flag is not set", g);
    if (d.flags & F_ALPHA) {
      int ai = alpha_index ? alpha_index[g] : 0;
      if (ai < 0 || ai >= (int)c->alphas.size())
        return fail(AXR_EINVAL, "group %d: alpha index %d out of range (%zu masks)", g, ai, c->alphas.size());
      int base_len = (d.flags & F_MIP) ? (1 << G.tex_size) : G.tex_size;
      if (c->alphas[ai].side != base_len)
        return fail(AXR_EINVAL, "group %d: alpha mask side %d differs from texture side %d", g, c->alphas[ai].side,
                    base_len);
      d.amask = c->alphas[ai].mask;
      d.aquad = c->alphas[ai].quad;
      d.alen = c->alphas[ai].side;
    }
  }
  return 0;
}

// Copies a group table to the device on stream s through the pinned ring.
int upload_table(axr_ctx *c, GroupDev *dst, const GroupDev *tab, int n, cudaStream_t s) {
  axr_ctx::Stage &st = c->stage[c->stage_next];
  c->stage_next = (c->stage_next + 1) % 8;
  if (!st.h) {
    if (cudaMallocHost(&st.h, sizeof(GroupDev) * MAX_GROUPS) != cudaSuccess) return fail(AXR_ENOMEM, "group table");
    CK(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
  } else if (st.used) {
    CK(cudaEventSynchronize(st.ev));
  }
  memcpy(st.h, tab, sizeof(GroupDev) * n);
  CK(cudaMemcpyAsync(dst, st.h, sizeof(GroupDev) * n, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(st.ev, s));
  st.used = true;
  return 0;
}

// Builds the per-call group table on the device.
int upload_groups(axr_ctx *c, const int32_t *flags, const int32_t *alpha_index, const uint8_t *enabled_mask,
                  bool mask_means_enabled, int ngroups) {
  GroupDev tab[MAX_GROUPS];
  int rc = group_table(c, flags, alpha_index, enabled_mask, mask_means_enabled, ngroups, tab);
  if (rc) return rc;
  rc = upload_table(c, c->d_groups, tab, std::max(ngroups, 1), c->stream);
  if (rc) return rc;
  return 0;
}

}  // namespace

extern "C" {

const char *axr_last_error(void) { return g_err.c_str(); }

int axr_create(int w, int h, int device, axr_ctx **out) {
  if (!out) return fail(AXR_EINVAL, "out is null");
  *out = nullptr;
  if (w <= 0 || h <= 0 || w % TILE != 0) return fail(AXR_EINVAL, "framebuffer %dx%d: width must be a positive multiple of 16", w, h);
  if ((long)w * h > (1L << 28)) return fail(AXR_EINVAL, "framebuffer %dx%d too large", w, h);
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(AXR_EINVAL, "device %d of %d", device, ndev);
  CK(cudaSetDevice(device));
  axr_ctx *c = new axr_ctx();
  c->device = device; c->w = w; c->h = h;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  {
    const void *kern[6] = {(const void *)k_raster_small<false>, (const void *)k_raster_small<true>,
                           (const void *)k_raster_tiled<false>, (const void *)k_raster_tiled<true>,
                           (const void *)k_shadow_raster<false>, (const void *)k_shadow_raster<true>};
    for (int k = 0; k < 6; k++) {
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern[k], 128, 0) == cudaSuccess && n > 0) c->occ[k] = n;
      else cudaGetLastError();
    }
  }
  size_t n = (size_t)w * h;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->s_alpha, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_setup, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_coarse, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_alpha, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc(&c->ro, n * 2) != cudaSuccess || cudaMalloc(&c->go, n * 2) != cudaSuccess ||
      cudaMalloc(&c->bo, n * 2) != cudaSuccess || cudaMalloc(&c->db, n * 4) != cudaSuccess ||
      cudaMalloc(&c->keys, n * 8) != cudaSuccess || cudaMalloc(&c->ctr, sizeof(uint32_t) * CTR_N) != cudaSuccess ||
      cudaMalloc(&c->d_groups, sizeof(GroupDev) * MAX_GROUPS) != cudaSuccess ||
      cudaMallocHost(&c->h_ctr, sizeof(uint32_t) * CTR_N) != cudaSuccess ||
      cudaMallocHost(&c->h_ring, sizeof(uint32_t) * CTR_N * 2) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_ctr[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_ctr[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_geo, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_lights, cudaEventDisableTiming) != cudaSuccess) {
    rc = fail(AXR_ENOMEM, "framebuffers for %dx%d", w, h);
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->light_blocks, k_vert_light, 256, 0);
  if (c->light_blocks < 1) c->light_blocks = 1;
  // initial tile-unit queue (grows after an overflow); AXR_UNIT_QUEUE overrides
  uint32_t units0 = 1u << 22;
  if (const char *e = getenv("AXR_UNIT_QUEUE")) {
    long v = atol(e);
    if (v >= 1 && v <= (1L << 30)) units0 = (uint32_t)v;
  }
  if (!rc) rc = grow_units(c, units0);
  if (rc) {
    axr_destroy(c);
    return rc;
  }
  // reference initial state: colour planes of ones (Ops0.py:111-113), depth cleared
  k_fill_rgb<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(c->ro, c->go, c->bo, (int)n, 1, 1, 1);
  k_clear_depth<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(c->db, w, h, 1);
  cudaMemsetAsync(c->keys, 0xff, n * 8, c->stream);
  cudaMemsetAsync(c->ctr, 0, sizeof(uint32_t) * CTR_N, c->stream);
  memset(c->h_ctr, 0, sizeof(uint32_t) * CTR_N);
  memset(c->h_ring, 0, sizeof(uint32_t) * CTR_N * 2);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    axr_destroy(c);
    return fail(AXR_ECUDA, "initialising framebuffers");
  }
  *out = c;
  return 0;
}

int axr_destroy(axr_ctx *c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &g : c->groups) {
    cudaFree(g.xyz); cudaFree(g.vn); cudaFree(g.uv); cudaFree(g.li);
    cudaFree(g.tex);
  }
  for (auto &a : c->alphas) { cudaFree(a.mask); cudaFree(a.quad); }
  for (auto &m : c->nmaps) cudaFree(m.texels);
  for (auto &sm : c->shadows) {
    if (sm.st) { cudaStreamSynchronize(sm.st); cudaStreamDestroy(sm.st); }
    if (sm.ev_write) cudaEventDestroy(sm.ev_write);
    if (sm.ev_read) cudaEventDestroy(sm.ev_read);
    cudaFree(sm.map); cudaFree(sm.list); cudaFree(sm.items); cudaFree(sm.ctr); cudaFree(sm.tab);
    cudaFree(sm.rec); cudaFree(sm.tiles); cudaFree(sm.units);
    if (sm.h_ring) cudaFreeHost(sm.h_ring);
    for (auto e : sm.ev_ctr)
      if (e) cudaEventDestroy(e);
  }
  if (c->s_alpha) { cudaStreamSynchronize(c->s_alpha); cudaStreamDestroy(c->s_alpha); }
  if (c->ev_setup) cudaEventDestroy(c->ev_setup);
  if (c->ev_coarse) cudaEventDestroy(c->ev_coarse);
  if (c->ev_alpha) cudaEventDestroy(c->ev_alpha);
  cudaFree(c->ro); cudaFree(c->go); cudaFree(c->bo); cudaFree(c->db); cudaFree(c->keys);
  cudaFree(c->small_list); cudaFree(c->large_list); cudaFree(c->items); cudaFree(c->units); cudaFree(c->mipc);
  cudaFree(c->ctr); cudaFree(c->d_groups);
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  if (c->h_ring) cudaFreeHost(c->h_ring);
  for (int k = 0; k < 2; k++) {
    if (c->ev_ctr[k]) cudaEventDestroy(c->ev_ctr[k]);
    auto &r = c->rd[k];
    if (r.done) cudaEventSynchronize(r.done);
    cudaFree(r.stage);
    if (r.staged) cudaEventDestroy(r.staged);
    if (r.done) cudaEventDestroy(r.done);
  }
  if (c->s_copy) { cudaStreamSynchronize(c->s_copy); cudaStreamDestroy(c->s_copy); }
  for (auto &st : c->stage) {
    if (st.ev) { cudaEventSynchronize(st.ev); cudaEventDestroy(st.ev); }
    if (st.h) cudaFreeHost(st.h);
  }
  for (auto &p : c->tpend) { c->ev_pool.push_back(p.a); c->ev_pool.push_back(p.b); }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->ev_geo) cudaEventDestroy(c->ev_geo);
  if (c->ev_lights) { cudaEventSynchronize(c->ev_lights); cudaEventDestroy(c->ev_lights); }
  cudaFree(c->d_lights);
  if (c->h_lights) cudaFreeHost(c->h_lights);
  for (auto p : c->post) cudaFree(p);
  cudaFree(c->bloom);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int axr_set_scale_cull(axr_ctx *c, float s, float cax, float cay) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  c->sscale = s; c->cax = cax; c->cay = cay;
  return 0;
}

int axr_add_texture_group(axr_ctx *c, const float *xyz, const float *uv, const float *vn, int ntris,
                          const uint16_t *r, const uint16_t *g, const uint16_t *b, long ntexels, int mip_side,
                          int *out_id) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!xyz || !uv || !vn || !r || !g || !b || ntris < 0) return fail(AXR_EINVAL, "null input or negative count");
  // vertex ranges (transform, translate, vertLight) are int vertex indices
  if (ntris > MAX_GROUP_TRIS) return fail(AXR_EINVAL, "a group holds at most %d triangles", MAX_GROUP_TRIS);
  if ((int)c->groups.size() >= MAX_GROUPS) return fail(AXR_EINVAL, "at most %d groups", MAX_GROUPS);
  if ((long)c->total_tris + ntris >= (1L << 30) - 1) return fail(AXR_EINVAL, "more than 2^30 triangles");
  Group G;
  G.ntris = ntris;
  G.tri_base = c->total_tris;
  G.ntexels = ntexels;
  G.mip_side = mip_side;
  if (mip_side > 0) {
    if (!is_pow2(mip_side)) return fail(AXR_EINVAL, "mip side %d is not a power of two", mip_side);
    long need = ((long)mip_side * mip_side * 4 - 1) / 3;
    if (ntexels != need) return fail(AXR_EINVAL, "mip chain of side %d needs %ld texels, got %ld", mip_side, need, ntexels);
    int lg = 0;
    while ((1 << lg) < mip_side) lg++;
    G.tex_size = lg;
    if (lg < 1) return fail(AXR_EINVAL, "mip side must be at least 2");
  } else {
    long side = 1;
    while (side * side < ntexels) side++;
    if (side * side != ntexels || !is_pow2(side)) return fail(AXR_EINVAL, "texture of %ld texels is not a power-of-two square", ntexels);
    G.tex_size = (int)side;
  }
  size_t nv = (size_t)ntris * 3;
  std::vector<ushort4> texels((size_t)ntexels);
  for (long k = 0; k < ntexels; k++) texels[k] = make_ushort4(r[k], g[k], b[k], 0);
  if ((rc = upload(c, &G.xyz, xyz, nv * 3)) || (rc = upload(c, &G.vn, vn, nv * 3)) || (rc = upload(c, &G.uv, uv, nv * 2)) ||
      (rc = upload(c, &G.tex, texels.data(), (size_t)ntexels)))
    return rc;
  if (cudaMalloc(&G.li, sizeof(float) * std::max<size_t>(nv * 3, 1)) != cudaSuccess) return fail(AXR_ENOMEM, "LI buffer");
  CK(cudaMemsetAsync(G.li, 0, sizeof(float) * nv * 3, c->stream));
  c->groups.push_back(G);
  c->total_tris += ntris;
  if ((rc = ensure_lists(c))) return rc;
  CK(cudaStreamSynchronize(c->stream));   // host arrays are borrowed only for the call
  if (out_id) *out_id = (int)c->groups.size() - 1;
  return 0;
}

int axr_set_vert_light(axr_ctx *c, int group, const float *li) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (group < 0 || group >= (int)c->groups.size() || !li) return fail(AXR_EINVAL, "group %d", group);
  CK(cudaMemcpyAsync(c->groups[group].li, li, sizeof(float) * 9 * (size_t)c->groups[group].ntris,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int axr_vert_light(axr_ctx *c, const uint8_t *mask, int ngroups, const float *dir_int, const float *dir_dir, int ndirs,
                   const float *point_int, const float *point_pos, int npoints, const float *spot_int,
                   const float *spot_dir, const float *spot_pos, int nspots, float amb) {
  int rc = check_ctx(c);
  if (rc) return rc;
  // the reference passes the counts as char / short / int (Ops.py:561,579,595)
  if (ngroups != (int)c->groups.size() || ndirs < 0 || ndirs > 127 || npoints < 0 || npoints > 32767 ||
      nspots < 0 || (ndirs && (!dir_int || !dir_dir)) || (npoints && (!point_int || !point_pos)) ||
      (nspots && (!spot_int || !spot_dir || !spot_pos)))
    return fail(AXR_EINVAL, "vert_light arguments");
  // table: dir int | dir dir | point int | point pos | spot int | spot dir | spot pos
  size_t nf = 3 * (2 * (size_t)ndirs + 2 * (size_t)npoints + 3 * (size_t)nspots);
  if (nf > c->lights_cap) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->lights_used) CK(cudaEventSynchronize(c->ev_lights));
    cudaFree(c->d_lights);
    if (c->h_lights) cudaFreeHost(c->h_lights);
    c->d_lights = c->h_lights = nullptr;
    c->lights_cap = 0;
    size_t cap = std::max<size_t>(nf, 1024);
    if (cudaMalloc(&c->d_lights, cap * 4) != cudaSuccess || cudaMallocHost(&c->h_lights, cap * 4) != cudaSuccess)
      return fail(AXR_ENOMEM, "light table of %zu floats", nf);
    c->lights_cap = cap;
  } else if (c->lights_used) {
    CK(cudaEventSynchronize(c->ev_lights));   // the copy that read the staging buffer last time
  }
  float *h = c->h_lights;
  const float *src[7] = {dir_int, dir_dir, point_int, point_pos, spot_int, spot_dir, spot_pos};
  const int cnt[7] = {ndirs, ndirs, npoints, npoints, nspots, nspots, nspots};
  size_t off[7], at = 0;
  for (int k = 0; k < 7; k++) {
    off[k] = at;
    if (cnt[k]) memcpy(h + at, src[k], sizeof(float) * 3 * cnt[k]);
    at += 3 * (size_t)cnt[k];
  }
  if (nf) CK(cudaMemcpyAsync(c->d_lights, h, nf * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaEventRecord(c->ev_lights, c->stream));
  c->lights_used = true;
  VertLights L;
  const float *d = c->d_lights;
  L.dint = d + off[0]; L.ddir = d + off[1]; L.pint = d + off[2]; L.ppos = d + off[3];
  L.sint = d + off[4]; L.sdir = d + off[5]; L.spos = d + off[6];
  L.nd = ndirs; L.np = npoints; L.ns = nspots; L.amb = amb;
  for (int g = 0; g < ngroups; g++) {
    if (mask && !mask[g]) continue;
    const Group &G = c->groups[g];
    int nv = G.ntris * 3;
    if (!nv) continue;
    launch(c, c->stream, "k_vert_light", [&] {
      k_vert_light<<<grid_for(c, nv, 256, c->light_blocks), 256, 0, c->stream>>>(G.xyz, G.vn, G.li, nv, L);
    });
  }
  CK(cudaGetLastError());
  c->amb = amb;
  return 0;
}

}  // extern "C"

namespace {

// A write of group geometry on the handle's stream: waits for every shadow
// pass in flight (they read the geometry on their own streams) and, after
// `body` has queued the write, marks it for the next shadow passes.
template <class F>
int geometry_write(axr_ctx *c, F body) {
  for (auto &sm : c->shadows)
    if (sm.st) CK(cudaStreamWaitEvent(c->stream, sm.ev_write, 0));
  int rc = body();
  if (rc) return rc;
  CK(cudaEventRecord(c->ev_geo, c->stream));
  return 0;
}

int vertex_range(axr_ctx *c, int group, int &v0, int &v1) {
  if (group < 0 || group >= (int)c->groups.size()) return fail(AXR_EINVAL, "group %d", group);
  int nv = c->groups[group].ntris * 3;
  if (v1 < 0) v1 = nv;
  if (v0 < 0 || v0 > v1 || v1 > nv) return fail(AXR_EINVAL, "vertices [%d, %d) outside group %d of %d", v0, v1, group, nv);
  return 0;
}

}  // namespace

extern "C" {

int axr_transform(axr_ctx *c, int group, const float *old_rm, const float *rot_mat, const float *origin, int v_start,
                  int v_end) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!old_rm || !rot_mat || !origin) return fail(AXR_EINVAL, "transform arguments");
  if ((rc = vertex_range(c, group, v_start, v_end))) return rc;
  VertXform X;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      X.oldr[3 * i + j] = old_rm[3 * i + j];
      X.rr[3 * i + j] = rot_mat[3 * j + i];
    }
  for (int k = 0; k < 3; k++) X.o[k] = origin[k];
  if (v_start == v_end) return 0;
  const Group &G = c->groups[group];
  return geometry_write(c, [&] {
    int nq = (v_end + 3) / 4 - v_start / 4;
    launch(c, c->stream, "k_vert_xform", [&] {
      k_vert_xform<true><<<grid_for(c, nq, 256, 8), 256, 0, c->stream>>>(G.xyz, G.vn, v_start, v_end, X);
    });
    CK(cudaGetLastError());
    return 0;
  });
}

int axr_translate(axr_ctx *c, int group, const float *coords, int v_start, int v_end) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!coords) return fail(AXR_EINVAL, "translate arguments");
  if ((rc = vertex_range(c, group, v_start, v_end))) return rc;
  VertXform X = {};
  for (int k = 0; k < 3; k++) X.o[k] = coords[k];
  if (v_start == v_end) return 0;
  const Group &G = c->groups[group];
  return geometry_write(c, [&] {
    int nq = (v_end + 3) / 4 - v_start / 4;
    launch(c, c->stream, "k_vert_translate", [&] {
      k_vert_xform<false><<<grid_for(c, nq, 256, 8), 256, 0, c->stream>>>(G.xyz, nullptr, v_start, v_end, X);
    });
    CK(cudaGetLastError());
    return 0;
  });
}

int axr_set_mip_bias(axr_ctx *c, int group, float bias) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (group < 0 || group >= (int)c->groups.size()) return fail(AXR_EINVAL, "group %d", group);
  if (!(bias == bias) || bias > 1e30f || bias < -1e30f) return fail(AXR_EINVAL, "mip bias is not a finite number");
  c->groups[group].mip_bias = bias;
  return 0;
}

int axr_get_vertices(axr_ctx *c, int group, float *xyz, float *vn, float *li) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (group < 0 || group >= (int)c->groups.size()) return fail(AXR_EINVAL, "group %d", group);
  const Group &G = c->groups[group];
  size_t n = (size_t)G.ntris * 9 * 4;
  if (xyz) CK(cudaMemcpyAsync(xyz, G.xyz, n, cudaMemcpyDeviceToHost, c->stream));
  if (vn) CK(cudaMemcpyAsync(vn, G.vn, n, cudaMemcpyDeviceToHost, c->stream));
  if (li) CK(cudaMemcpyAsync(li, G.li, n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int axr_copy_to(axr_ctx *c, int group, const float *xyz, const float *vn, int tri_start, int ntris) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (group < 0 || group >= (int)c->groups.size()) return fail(AXR_EINVAL, "group %d", group);
  Group &G = c->groups[group];
  if (tri_start < 0 || ntris < 0 || (long)tri_start + ntris > G.ntris) return fail(AXR_EINVAL, "range out of group");
  size_t off = (size_t)tri_start * 9, n = (size_t)ntris * 9;
  rc = geometry_write(c, [&] {
    if (xyz) CK(cudaMemcpyAsync(G.xyz + off, xyz, n * 4, cudaMemcpyHostToDevice, c->stream));
    if (vn) CK(cudaMemcpyAsync(G.vn + off, vn, n * 4, cudaMemcpyHostToDevice, c->stream));
    return 0;
  });
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));   // host arrays are borrowed only for the call
  return 0;
}

int axr_add_tex_alpha(axr_ctx *c, const uint8_t *mask, int side, int *out_id) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!mask || !is_pow2(side)) return fail(AXR_EINVAL, "alpha mask side %d is not a power of two", side);
  Alpha a;
  a.side = side;
  std::vector<uint8_t> b((size_t)side * side), q((size_t)side * side);
  for (size_t i = 0; i < b.size(); i++) b[i] = mask[i] ? 1 : 0;
  for (int t2 = 0; t2 < side; t2++)
    for (int t1 = 0; t1 < side; t1++) {
      int t1n = std::min(t1 + 1, side - 1), t2n = std::min(t2 + 1, side - 1);
      q[(size_t)side * t2 + t1] = (uint8_t)(b[(size_t)side * t2 + t1] | b[(size_t)side * t2 + t1n] << 1 |
                                            b[(size_t)side * t2n + t1] << 2 | b[(size_t)side * t2n + t1n] << 3);
    }
  if ((rc = upload(c, &a.mask, b.data(), b.size())) || (rc = upload(c, &a.quad, q.data(), q.size()))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->alphas.push_back(a);
  if (out_id) *out_id = (int)c->alphas.size() - 1;
  return 0;
}

int axr_add_normal_map(axr_ctx *c, const uint8_t *rgba, long ntexels, int *out_id) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!rgba || ntexels < 1) return fail(AXR_EINVAL, "normal map of %ld texels", ntexels);
  NormalMap m;
  m.n = ntexels;
  if ((rc = upload(c, &m.texels, reinterpret_cast<const uchar4 *>(rgba), (size_t)ntexels))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->nmaps.push_back(m);
  if (out_id) *out_id = (int)c->nmaps.size() - 1;
  return 0;
}

int axr_set_normal_material(axr_ctx *c, int group, int map, float roughness, int metal) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  if (group < 0 || group >= (int)c->groups.size()) return fail(AXR_EINVAL, "group %d out of range", group);
  if (map < -1 || map >= (int)c->nmaps.size()) return fail(AXR_EINVAL, "normal map %d out of range", map);
  Group &G = c->groups[group];
  G.nmap = map;
  G.roughness = roughness;
  G.metal = metal ? 1 : 0;
  return 0;
}

int axr_set_primary_light(axr_ctx *c, const float i[3], const float d[3]) {
  if (!c || !i || !d) return fail(AXR_EINVAL, "null argument");
  memcpy(c->lint, i, sizeof c->lint);
  memcpy(c->ldir, d, sizeof c->ldir);
  return 0;
}

int axr_set_pos(axr_ctx *c, const float p[3]) {
  if (!c || !p) return fail(AXR_EINVAL, "null argument");
  memcpy(c->pos, p, sizeof c->pos);
  return 0;
}

int axr_set_vm(axr_ctx *c, const float vm[9]) {
  if (!c || !vm) return fail(AXR_EINVAL, "null argument");
  memcpy(c->vm, vm, sizeof c->vm);
  return 0;
}

int axr_clear_zbuffer(axr_ctx *c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  launch(c, c->stream, "k_clear_depth", [&] { k_clear_depth<<<grid_for(c, (long)c->w * c->h, 256, 8), 256, 0, c->stream>>>(c->db, c->w, c->h, 4); });
  CK(cudaGetLastError());
  return 0;
}

int axr_clear_color(axr_ctx *c, int r, int g, int b) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (r < 0 || g < 0 || b < 0 || r > 65535 || g > 65535 || b > 65535)
    return fail(AXR_EINVAL, "colour (%d, %d, %d) outside [0, 65535]", r, g, b);
  long n = (long)c->w * c->h;
  launch(c, c->stream, "k_fill_rgb", [&] {
    k_fill_rgb<<<grid_for(c, n, 256, 8), 256, 0, c->stream>>>(c->ro, c->go, c->bo, (int)n, (uint16_t)r, (uint16_t)g,
                                                                (uint16_t)b);
  });
  CK(cudaGetLastError());
  return 0;
}

int axr_draw_all(axr_ctx *c, const int32_t *flags, const int32_t *alpha_index, const uint8_t *mask, int ngroups,
                 const int32_t *shadow_ids, int nshadow) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (ngroups != (int)c->groups.size()) return fail(AXR_EINVAL, "drawAll with %d groups, handle has %zu", ngroups, c->groups.size());
  if (nshadow < 0 || nshadow > 2) return fail(AXR_EINVAL, "at most two shadow cascades");
  if ((rc = settle_next(c))) return rc;
  DrawParams P;
  memset(&P, 0, sizeof P);
  bool any_shadow = false, any_alpha = false, any_normal = false;
  for (int g = 0; g < ngroups; g++) {
    if ((!mask || !mask[g]) && flags && (flags[g] & F_SHADOW)) any_shadow = true;
    if ((!mask || !mask[g]) && flags && (flags[g] & F_ALPHA)) any_alpha = true;
    if ((!mask || !mask[g]) && flags && (flags[g] & F_NORMAL)) any_normal = true;
  }
  P.nsh = nshadow;
  for (int k = 0; k < nshadow; k++) {
    int id = shadow_ids[k];
    if (id < 0 || id >= MAX_SHADOWS || !c->shadows[id].map) return fail(AXR_ESTATE, "shadow map %d does not exist", id);
    Shadow &s = c->shadows[id];
    P.sh[k].map = s.map; P.sh[k].dim = s.dim; P.sh[k].scale = s.scale;
    memcpy(P.sh[k].pos, s.pos, sizeof s.pos);
    memcpy(P.sh[k].vv, s.vv, sizeof s.vv);
  }
  if (any_shadow && nshadow == 0) return fail(AXR_ESTATE, "shadow materials drawn with no shadow map");
  if ((rc = upload_groups(c, flags, alpha_index, mask, false, ngroups))) return rc;
  P.groups = c->d_groups;
  P.ngroups = ngroups;
  P.total_tris = c->total_tris;
  P.view = make_view(c);
  memcpy(P.light.lint, c->lint, sizeof c->lint);
  memcpy(P.light.ldir, c->ldir, sizeof c->ldir);
  P.light.amb = c->amb;
  P.keys = c->keys; P.ro = c->ro; P.go = c->go; P.bo = c->bo; P.db = c->db;
  P.small_list = c->small_list; P.large_list = c->large_list; P.items = c->items;
  P.units = c->units; P.ctr = c->ctr;
  P.cap_list = c->cap_list; P.cap_units = c->cap_units;
  P.min_chunk = c->min_chunk;
  P.claim_k = 2;
  P.mipc = c->mipc;
  long npix = (long)c->w * c->h;
  cudaStream_t s = c->stream;
  int64_t nk = 0;
  cudaStream_t sa = c->s_alpha;
  launch(c, s, "k_init_keys", [&] { k_init_keys<<<grid_for(c, npix, 256, 16), 256, 0, s>>>(c->db, c->keys, (int)npix, c->ctr); }); nk++;
  if (c->total_tris > 0) {
    // visibility: opaque rasterizers on the main stream, alpha-tested ones
    // concurrently on a side stream (all of them atomicMin the same buffer)
    launch(c, s, "k_setup", [&] { k_setup<<<grid_for(c, c->total_tris, SETUP_THREADS, 8), SETUP_THREADS, 0, s>>>(P); }); nk++;
    if (any_alpha) {
      CK(cudaEventRecord(c->ev_setup, s));
      CK(cudaStreamWaitEvent(sa, c->ev_setup, 0));
      launch(c, sa, "k_raster_small_alpha", [&] { k_raster_small<true><<<c->sms * c->occ[1], 128, 0, sa>>>(P); }); nk++;
    }
    launch(c, s, "k_raster_small", [&] { k_raster_small<false><<<c->sms * c->occ[0], 128, 0, s>>>(P); }); nk++;
    launch(c, s, "k_coarse", [&] { k_coarse<<<c->sms * 4, 128, 0, s>>>(P); }); nk++;
    if (any_alpha) {
      CK(cudaEventRecord(c->ev_coarse, s));
      CK(cudaStreamWaitEvent(sa, c->ev_coarse, 0));
      launch(c, sa, "k_raster_tiled_alpha", [&] { k_raster_tiled<true><<<c->sms * c->occ[3], 128, 0, sa>>>(P); }); nk++;
    }
    launch(c, s, "k_raster_tiled", [&] { k_raster_tiled<false><<<c->sms * c->occ[2], 128, 0, s>>>(P); }); nk++;
    launch(c, s, "k_raster_tiled_fallback", [&] { k_raster_tiled_fallback<<<c->sms * 2, 128, 0, s>>>(P); }); nk++;
    if (any_alpha) {
      CK(cudaEventRecord(c->ev_alpha, sa));
      CK(cudaStreamWaitEvent(s, c->ev_alpha, 0));
    }
  }
  // shading samples the cascades: wait for their last writers
  for (int k = 0; k < nshadow; k++) CK(cudaStreamWaitEvent(s, c->shadows[shadow_ids[k]].ev_write, 0));
  dim3 sb(256), sgd((c->w + 15) / 16, (c->h + 15) / 16);   // a 16x16 tile per block
  if (any_normal)
    launch(c, s, "k_shade", [&] { k_shade<true><<<sgd, sb, 0, s>>>(P); });
  else
    launch(c, s, "k_shade", [&] { k_shade<false><<<sgd, sb, 0, s>>>(P); });
  nk++;
  for (int k = 0; k < nshadow; k++) CK(cudaEventRecord(c->shadows[shadow_ids[k]].ev_read, s));
  CK(cudaGetLastError());
  int slot = 1 - c->last_slot;
  if (c->pend[slot] && (rc = check_slot(c, slot, true))) return rc;   // the frame before last
  CK(cudaMemcpyAsync(c->h_ring + slot * CTR_N, c->ctr, sizeof(uint32_t) * CTR_N, cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(c->ev_ctr[slot], s));
  c->pend[slot] = true;
  c->last_slot = slot;
  c->last_kernels = nk;
  return 0;
}

int axr_get_frame(axr_ctx *c, uint16_t *r, uint16_t *g, uint16_t *b, float *depth) {
  int rc = check_ctx(c);
  if (rc) return rc;
  size_t n = (size_t)c->w * c->h;
  if (r) CK(cudaMemcpyAsync(r, c->ro, n * 2, cudaMemcpyDeviceToHost, c->stream));
  if (g) CK(cudaMemcpyAsync(g, c->go, n * 2, cudaMemcpyDeviceToHost, c->stream));
  if (b) CK(cudaMemcpyAsync(b, c->bo, n * 2, cudaMemcpyDeviceToHost, c->stream));
  if (depth) CK(cudaMemcpyAsync(depth, c->db, n * 4, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return settle(c);
}

int axr_read_frame_async(axr_ctx *c, uint16_t *r, uint16_t *g, uint16_t *b, float *depth, int64_t *ticket) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!ticket) return fail(AXR_EINVAL, "null ticket");
  if ((rc = settle_next(c))) return rc;
  size_t n = (size_t)c->w * c->h;
  if (!c->s_copy) CK(cudaStreamCreateWithFlags(&c->s_copy, cudaStreamNonBlocking));
  axr_ctx::ReadSlot &sl = c->rd[c->read_seq & 1];
  if (sl.busy) {                       // the read two calls ago still holds this slot
    CK(cudaEventSynchronize(sl.done));
    sl.busy = false;
  }
  if (!sl.stage) {
    if (cudaMalloc(&sl.stage, n * 10) != cudaSuccess) return fail(AXR_ENOMEM, "frame staging buffer");
    CK(cudaEventCreateWithFlags(&sl.staged, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  }
  // device copies on the render stream (ordered before the next frame's
  // writes), then the device-to-host copies on the copy stream
  uint16_t *sr = (uint16_t *)sl.stage, *sg = sr + n, *sb = sg + n;
  float *sd = (float *)(sb + n);
  cudaStream_t s = c->stream;
  if (r) CK(cudaMemcpyAsync(sr, c->ro, n * 2, cudaMemcpyDeviceToDevice, s));
  if (g) CK(cudaMemcpyAsync(sg, c->go, n * 2, cudaMemcpyDeviceToDevice, s));
  if (b) CK(cudaMemcpyAsync(sb, c->bo, n * 2, cudaMemcpyDeviceToDevice, s));
  if (depth) CK(cudaMemcpyAsync(sd, c->db, n * 4, cudaMemcpyDeviceToDevice, s));
  CK(cudaEventRecord(sl.staged, s));
  CK(cudaStreamWaitEvent(c->s_copy, sl.staged, 0));
  if (r) CK(cudaMemcpyAsync(r, sr, n * 2, cudaMemcpyDeviceToHost, c->s_copy));
  if (g) CK(cudaMemcpyAsync(g, sg, n * 2, cudaMemcpyDeviceToHost, c->s_copy));
  if (b) CK(cudaMemcpyAsync(b, sb, n * 2, cudaMemcpyDeviceToHost, c->s_copy));
  if (depth) CK(cudaMemcpyAsync(depth, sd, n * 4, cudaMemcpyDeviceToHost, c->s_copy));
  CK(cudaEventRecord(sl.done, c->s_copy));
  sl.busy = true;
  sl.seq = c->read_seq;
  *ticket = c->read_seq++;
  return 0;
}

int axr_read_frame_rgb8_async(axr_ctx *c, float exposure, uint8_t *rgb, int64_t *ticket) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!ticket || !rgb) return fail(AXR_EINVAL, "null argument");
  if ((rc = settle_next(c))) return rc;
  size_t n = (size_t)c->w * c->h;
  if (!c->s_copy) CK(cudaStreamCreateWithFlags(&c->s_copy, cudaStreamNonBlocking));
  axr_ctx::ReadSlot &sl = c->rd[c->read_seq & 1];
  if (sl.busy) {
    CK(cudaEventSynchronize(sl.done));
    sl.busy = false;
  }
  if (!sl.stage) {
    if (cudaMalloc(&sl.stage, n * 10) != cudaSuccess) return fail(AXR_ENOMEM, "frame staging buffer");
    CK(cudaEventCreateWithFlags(&sl.staged, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  }
  cudaStream_t s = c->stream;
  launch(c, s, "k_pack_rgb8", [&] {
    k_pack_rgb8<<<grid_for(c, (long)n, 256, 8), 256, 0, s>>>(c->ro, c->go, c->bo, (int)n, exposure, sl.stage);
  });
  CK(cudaGetLastError());
  CK(cudaEventRecord(sl.staged, s));
  CK(cudaStreamWaitEvent(c->s_copy, sl.staged, 0));
  CK(cudaMemcpyAsync(rgb, sl.stage, n * 3, cudaMemcpyDeviceToHost, c->s_copy));
  CK(cudaEventRecord(sl.done, c->s_copy));
  sl.busy = true;
  sl.seq = c->read_seq;
  *ticket = c->read_seq++;
  return 0;
}

int axr_wait_frame(axr_ctx *c, int64_t ticket) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (ticket < 0 || ticket >= c->read_seq) return fail(AXR_EINVAL, "no read with ticket %lld", (long long)ticket);
  axr_ctx::ReadSlot &sl = c->rd[ticket & 1];
  if (sl.seq == ticket && sl.busy) {   // (an older ticket finished before its slot was reused)
    CK(cudaEventSynchronize(sl.done));
    sl.busy = false;
  }
  return settle_next(c);
}

int axr_frame_done(axr_ctx *c, int64_t ticket) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  if (ticket < 0 || ticket >= c->read_seq) return fail(AXR_EINVAL, "no read with ticket %lld", (long long)ticket);
  axr_ctx::ReadSlot &sl = c->rd[ticket & 1];
  if (sl.seq != ticket || !sl.busy) return 1;
  cudaError_t e = cudaEventQuery(sl.done);
  if (e == cudaErrorNotReady) return 0;
  if (e != cudaSuccess) return fail(AXR_ECUDA, "frame read: %s", cudaGetErrorString(e));
  return 1;
}

int axr_get_ids(axr_ctx *c, int32_t *tri_id, uint8_t *cov) {
  int rc = check_ctx(c);
  if (rc) return rc;
  size_t n = (size_t)c->w * c->h;
  int32_t *dt = nullptr;
  uint8_t *dc = nullptr;
  if (cudaMalloc(&dt, n * 4) != cudaSuccess || cudaMalloc(&dc, n) != cudaSuccess) {
    cudaFree(dt);
    return fail(AXR_ENOMEM, "id buffers");
  }
  k_ids<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(c->keys, (int)n, dt, dc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && tri_id) e = cudaMemcpyAsync(tri_id, dt, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && cov) e = cudaMemcpyAsync(cov, dc, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dt);
  cudaFree(dc);
  if (e != cudaSuccess) return fail(AXR_ECUDA, "get_ids: %s", cudaGetErrorString(e));
  return settle(c);
}

int axr_set_frame(axr_ctx *c, const uint16_t *r, const uint16_t *g, const uint16_t *b, const float *depth) {
  int rc = check_ctx(c);
  if (rc) return rc;
  size_t n = (size_t)c->w * c->h;
  if (r) CK(cudaMemcpyAsync(c->ro, r, n * 2, cudaMemcpyHostToDevice, c->stream));
  if (g) CK(cudaMemcpyAsync(c->go, g, n * 2, cudaMemcpyHostToDevice, c->stream));
  if (b) CK(cudaMemcpyAsync(c->bo, b, n * 2, cudaMemcpyHostToDevice, c->stream));
  if (depth) CK(cudaMemcpyAsync(c->db, depth, n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int axr_gamma(axr_ctx *c, float ex) {
  int rc = check_ctx(c);
  if (rc) return rc;
  long n = (long)c->w * c->h;
  launch(c, c->stream, "k_gamma", [&] { k_gamma<<<grid_for(c, n, 256, 8), 256, 0, c->stream>>>(c->ro, c->go, c->bo, (int)n, ex); });
  CK(cudaGetLastError());
  return 0;
}

int axr_ssao(axr_ctx *c, const float *rnd, int n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!rnd || n < 32) return fail(AXR_EINVAL, "ssao needs a random table of at least 32 floats (got %d)", n);
  if (c->w < 16 || c->h < 16) return 0;          // no 16 x 16 work-group fits
  SsaoParams S;
  memcpy(S.rnd, rnd, sizeof S.rnd);
  S.sscale = c->sscale;
  dim3 grid(c->w / 16, c->h / 16);
  launch(c, c->stream, "k_ssao", [&] { k_ssao<<<grid, 256, 0, c->stream>>>(c->ro, c->go, c->bo, c->db, c->w, c->h, S); });
  CK(cudaGetLastError());
  return 0;
}

int axr_dof(axr_ctx *c, float focus) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (c->w < 16 || c->h < 16) return 0;
  size_t n = (size_t)c->w * c->h;
  for (auto &p : c->post)
    if (!p && cudaMalloc(&p, n * 2) != cudaSuccess) return fail(AXR_ENOMEM, "dof planes for %dx%d", c->w, c->h);
  dim3 grid(c->w / 16, c->h / 16);
  launch(c, c->stream, "k_dof", [&] {
    k_dof<<<grid, 256, 0, c->stream>>>(c->ro, c->go, c->bo, c->db, c->w, c->h, focus, c->post[0], c->post[1],
                                       c->post[2]);
  });
  // Ops.py:993-995 copies the gather back; rows below the covered region keep their colour
  size_t bytes = (size_t)c->w * (c->h / 16 * 16) * 2;
  uint16_t *dst[3] = {c->ro, c->go, c->bo};
  for (int k = 0; k < 3; k++) CK(cudaMemcpyAsync(dst[k], c->post[k], bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaGetLastError());
  return 0;
}

int axr_bloom(axr_ctx *c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  int wf = c->w / 2, hf = c->h / 2;
  if (hf < 3) return 0;                              // no row of the bright pass
  size_t plane = (size_t)wf * (hf + 8);
  if (!c->bloom) {
    if (cudaMalloc(&c->bloom, plane * 9 * 2) != cudaSuccess) return fail(AXR_ENOMEM, "bloom planes");
    CK(cudaMemsetAsync(c->bloom, 0, plane * 9 * 2, c->stream));   // rows no pass writes read 0
  }
  BloomPlanes B;
  for (int k = 0; k < 3; k++) {
    B.br[k] = c->bloom + plane * k;
    B.hb[k] = c->bloom + plane * (3 + k);
    B.vb[k] = c->bloom + plane * (6 + k);
  }
  int bx = (wf + 127) / 128;
  launch(c, c->stream, "k_bloom_bright", [&] {
    k_bloom_bright<<<dim3(bx, hf - 2), 128, 0, c->stream>>>(c->ro, c->go, c->bo, wf, hf, B);
  });
  launch(c, c->stream, "k_bloom_blur_h", [&] { k_bloom_blur<true><<<dim3(bx, hf - 1), 128, 0, c->stream>>>(wf, hf, B); });
  launch(c, c->stream, "k_bloom_blur_v", [&] { k_bloom_blur<false><<<dim3(bx, hf - 1), 128, 0, c->stream>>>(wf, hf, B); });
  int fx = (2 * wf + 127) / 128;
  launch(c, c->stream, "k_bloom_add", [&] {
    k_bloom_add<<<dim3(fx, 2 * hf), 128, 0, c->stream>>>(c->ro, c->go, c->bo, c->w, wf, hf, B);
  });
  CK(cudaGetLastError());
  return 0;
}

int axr_add_shadow_map(axr_ctx *c, int i, int size, float scale, float amb) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (i < 0 || i >= MAX_SHADOWS || size < 4 || size > 16384) return fail(AXR_EINVAL, "shadow map %d of size %d", i, size);
  Shadow &s = c->shadows[i];
  if (!s.st) {
    if (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev_write, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev_read, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev_ctr[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev_ctr[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&s.h_ring, sizeof(uint32_t) * 2 * CTR_N) != cudaSuccess ||
        cudaMalloc(&s.tab, sizeof(GroupDev) * MAX_GROUPS) != cudaSuccess)
      return fail(AXR_ENOMEM, "shadow map %d state", i);
  }
  if (s.map && s.dim != size) {
    CK(cudaStreamSynchronize(s.st));
    if ((rc = settle_shadows(c, true))) return rc;
    cudaFree(s.map); cudaFree(s.ctr); cudaFree(s.tiles);
    s.map = nullptr; s.ctr = s.tiles = nullptr;
  }
  CK(cudaStreamWaitEvent(s.st, s.ev_read, 0));
  if (!s.map) {
    // counters, then the per-tile unit counts and claim counters of the
    // tiled pass (opaque, alpha); tile offsets, cursors (2 per tile), order
    // and the prefix of blocks per tile
    s.ntx = (size + STILE - 1) / STILE;
    size_t nt = (size_t)s.ntx * s.ntx;
    if (cudaMalloc(&s.map, sizeof(float) * (size_t)size * size) != cudaSuccess ||
        cudaMalloc(&s.ctr, sizeof(uint32_t) * (CTR_N + 4 * nt)) != cudaSuccess ||
        cudaMalloc(&s.tiles, sizeof(uint32_t) * (5 * nt + 1)) != cudaSuccess)
      return fail(AXR_ENOMEM, "shadow map %dx%d", size, size);
  }
  s.dim = size;
  s.scale = scale;
  // a fresh map holds 65535 (Ops.py:1049)
  k_clear_depth<<<grid_for(c, (long)size * size, 256, 8), 256, 0, s.st>>>(s.map, size, size, 1);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(s.ev_write, s.st));
  c->amb = amb;
  return 0;
}

int axr_place_shadow_map(axr_ctx *c, int i, const float pos[3], const float vm[9], float amb) {
  if (!c || !pos || !vm) return fail(AXR_EINVAL, "null argument");
  if (i < 0 || i >= MAX_SHADOWS || !c->shadows[i].map) return fail(AXR_ESTATE, "shadow map %d does not exist", i);
  memcpy(c->shadows[i].pos, pos, sizeof(float) * 3);
  memcpy(c->shadows[i].vv, vm, sizeof(float) * 9);
  if (amb >= 0) c->amb = amb;
  return 0;
}

int axr_clear_shadow_map(axr_ctx *c, int i) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (i < 0 || i >= MAX_SHADOWS || !c->shadows[i].map) return fail(AXR_ESTATE, "shadow map %d does not exist", i);
  Shadow &s = c->shadows[i];
  CK(cudaStreamWaitEvent(s.st, s.ev_read, 0));
  launch(c, s.st, "k_clear_shadow", [&] { k_clear_depth<<<grid_for(c, (long)s.dim * s.dim, 256, 8), 256, 0, s.st>>>(s.map, s.dim, s.dim, 16); });
  CK(cudaGetLastError());
  CK(cudaEventRecord(s.ev_write, s.st));
  return 0;
}

int axr_shadow_map(axr_ctx *c, int i, const uint8_t *cast, const int32_t *flags, const int32_t *alpha_index, int ngroups,
                   float bias) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (i < 0 || i >= MAX_SHADOWS || !c->shadows[i].map) return fail(AXR_ESTATE, "shadow map %d does not exist", i);
  if (ngroups != (int)c->groups.size() || !cast) return fail(AXR_EINVAL, "shadowMap arguments");
  if ((rc = settle_next(c))) return rc;
  // alpha casters use the alpha mask's own side as lenT (drawminalpha.c:86-96)
  std::vector<int32_t> fl(ngroups, 0);
  for (int g = 0; g < ngroups; g++) fl[g] = flags ? (flags[g] & (F_ALPHA | F_MIP)) : 0;
  GroupDev tab[MAX_GROUPS];
  memset(tab, 0, sizeof tab);
  for (int g = 0; g < ngroups; g++) {
    const Group &G = c->groups[g];
    GroupDev &d = tab[g];
    d.xyz = G.xyz; d.uv = G.uv; d.ntris = G.ntris; d.tri_base = G.tri_base; d.tex_size = G.tex_size;
    d.flags = fl[g] & F_ALPHA;
    d.enabled = cast[g] ? 1 : 0;
    if (d.flags & F_ALPHA) {
      int ai = alpha_index ? alpha_index[g] : 0;
      if (ai < 0 || ai >= (int)c->alphas.size()) return fail(AXR_EINVAL, "group %d: alpha index %d", g, ai);
      d.amask = c->alphas[ai].mask;
      d.alen = c->alphas[ai].side;
    }
  }
  Shadow &sm = c->shadows[i];
  const bool tiled = c->shadow_mode >= 1 && sm.dim <= SHADOW_TILED_MAX_DIM;
  if (sm.cap < c->cap_list) {
    CK(cudaStreamSynchronize(sm.st));
    cudaFree(sm.list); cudaFree(sm.items); cudaFree(sm.rec);
    sm.list = sm.items = nullptr;
    sm.rec = nullptr;
    sm.items_ready = false;
    sm.cap = 0;
    if (cudaMalloc(&sm.list, sizeof(uint32_t) * c->cap_list) != cudaSuccess)
      return fail(AXR_ENOMEM, "caster list of shadow map %d", i);
    sm.cap = c->cap_list;
  }
  // caster records of the tiled pass
  if (tiled && !sm.rec && cudaMalloc(&sm.rec, 2 * sizeof(uint4) * sm.cap) != cudaSuccess)
    return fail(AXR_ENOMEM, "caster records of shadow map %d", i);
  if (tiled && !sm.units) {
    // initial tile-unit queue (grows after an overflow); AXR_SHADOW_UNIT_QUEUE overrides
    uint32_t units0 = sm.cap + sm.cap / 2 + 1024;
    if (const char *e = getenv("AXR_SHADOW_UNIT_QUEUE")) {
      long v = atol(e);
      if (v >= 1 && v <= (1L << 30)) units0 = (uint32_t)v;
    }
    if ((rc = grow_shadow_units(sm, units0))) return rc;
  }
  if (!tiled && !sm.items_ready) {
    if (cudaMalloc(&sm.items, sizeof(uint32_t) * sm.cap * MAX_CHUNKS) != cudaSuccess)
      return fail(AXR_ENOMEM, "row chunks of shadow map %d", i);
    sm.items_ready = true;
  }
  CK(cudaStreamWaitEvent(sm.st, sm.ev_read, 0));
  CK(cudaStreamWaitEvent(sm.st, c->ev_geo, 0));   // rotate / translate / copyTo queued before
  if ((rc = upload_table(c, sm.tab, tab, std::max(ngroups, 1), sm.st))) return rc;
  ShadowParams S;
  memset(&S, 0, sizeof S);
  S.groups = sm.tab; S.ngroups = ngroups; S.total_tris = c->total_tris;
  S.sh.map = sm.map; S.sh.dim = sm.dim; S.sh.scale = sm.scale;
  memcpy(S.sh.pos, sm.pos, sizeof sm.pos);
  memcpy(S.sh.vv, sm.vv, sizeof sm.vv);
  S.map = sm.map; S.bias = bias; S.list = sm.list; S.cap_list = sm.cap; S.ctr = sm.ctr;
  S.min_chunk = c->min_chunk;
  S.claim_k = 2;
  const size_t nt = (size_t)sm.ntx * sm.ntx;
  if (tiled) {
    S.rec = sm.rec;
    S.tcnt = sm.ctr + CTR_N; S.tclaim = sm.ctr + CTR_N + 2 * nt;
    S.toff = sm.tiles; S.tcur = sm.tiles + nt; S.tord = sm.tiles + 3 * nt; S.hpre = sm.tiles + 4 * nt;
    S.units = sm.units; S.cap_units = sm.cap_units;
    S.ntx = sm.ntx; S.ntiles = (int)nt;
    S.slice = c->shadow_slice; S.sort = c->shadow_mode == 2;
  } else {
    S.items = sm.items;
  }
  if (c->total_tris == 0) return 0;
  bool any_alpha = false;
  for (int g = 0; g < ngroups; g++)
    if (cast[g] && (tab[g].flags & F_ALPHA)) any_alpha = true;
  static_assert(CTR_SH_LIST_A == CTR_SH_LIST + 1 && CTR_SH_WORK == CTR_SH_LIST + 2 && CTR_SH_WORK_A == CTR_SH_LIST + 3,
                "shadow counters are contiguous");
  CK(cudaMemsetAsync(sm.ctr, 0, sizeof(uint32_t) * (CTR_N + (tiled ? 4 * nt : 0)), sm.st));
  cudaStream_t st = sm.st;
  launch(c, st, "k_shadow_setup", [&] { k_shadow_setup<<<grid_for(c, c->total_tris, 256, 16), 256, 0, st>>>(S); });
  if (tiled) {
    launch(c, st, "k_shadow_scan", [&] { k_shadow_scan<<<1, SCAN_THREADS, 0, st>>>(S); });
    launch(c, st, "k_shadow_bin", [&] { k_shadow_bin<<<c->sms * 8, 256, 0, st>>>(S); });
    if (S.sort) launch(c, st, "k_shadow_sort", [&] { k_shadow_sort<<<c->sms * 4, 256, 0, st>>>(S); });
    launch(c, st, "k_shadow_tiles", [&] { k_shadow_tiles<false><<<c->sms * 8, 128, 0, st>>>(S); });
    if (any_alpha)
      launch(c, st, "k_shadow_tiles_alpha", [&] { k_shadow_tiles<true><<<c->sms * 6, 128, 0, st>>>(S); });
  } else {
    launch(c, st, "k_shadow_raster", [&] { k_shadow_raster<false><<<c->sms * c->occ[4], 128, 0, st>>>(S); });
    if (any_alpha)
      launch(c, st, "k_shadow_raster_alpha", [&] { k_shadow_raster<true><<<c->sms * c->occ[5], 128, 0, st>>>(S); });
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(sm.ev_write, st));
  // the pass's counters to the ring (the slot before last is checked first)
  int slot = 1 - sm.last_slot;
  if (sm.pend[slot] && (rc = check_shadow_slot(sm, slot, true))) return rc;
  CK(cudaMemcpyAsync(sm.h_ring + slot * CTR_N, sm.ctr, sizeof(uint32_t) * CTR_N, cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(sm.ev_ctr[slot], st));
  sm.pend[slot] = true;
  sm.last_slot = slot;
  return 0;
}

int axr_shadow_stats(axr_ctx *c, int i, int64_t *out, int n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (i < 0 || i >= MAX_SHADOWS || !c->shadows[i].map) return fail(AXR_ESTATE, "shadow map %d does not exist", i);
  if (!out || n < 0) return fail(AXR_EINVAL, "shadowStats output");
  if ((rc = axr_sync(c))) return rc;
  const Shadow &s = c->shadows[i];
  const int64_t v[5] = {s.overflows, s.last_units, s.cap_units, s.last_casters[0], s.last_casters[1]};
  for (int k = 0; k < n && k < 5; k++) out[k] = v[k];
  return 0;
}

int axr_get_shadow_map(axr_ctx *c, int i, float *out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (i < 0 || i >= MAX_SHADOWS || !c->shadows[i].map) return fail(AXR_ESTATE, "shadow map %d does not exist", i);
  if (!out) return fail(AXR_EINVAL, "null output");
  Shadow &s = c->shadows[i];
  CK(cudaMemcpyAsync(out, s.map, sizeof(float) * (size_t)s.dim * s.dim, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return settle(c);
}

int axr_sync(axr_ctx *c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = sync_all(c))) return rc;
  return settle(c);
}

int axr_get_stream(axr_ctx *c, void **stream) {
  if (!c || !stream) return fail(AXR_EINVAL, "null argument");
  *stream = (void *)c->stream;
  return 0;
}

int axr_frame_device_ptrs(axr_ctx *c, void **r, void **g, void **b, void **depth, void **keys) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  if (r) *r = c->ro;
  if (g) *g = c->go;
  if (b) *b = c->bo;
  if (depth) *depth = c->db;
  if (keys) *keys = c->keys;
  return 0;
}

int axr_last_stats(axr_ctx *c, int64_t *kernels, int64_t *n_small, int64_t *n_large, int64_t *n_units) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = axr_sync(c))) return rc;
  if (kernels) *kernels = c->last_kernels;
  if (n_small) *n_small = (int64_t)c->h_ctr[CTR_SMALL] + c->h_ctr[CTR_SMALL_A];
  if (n_large) *n_large = c->h_ctr[CTR_LARGE];
  if (n_units) *n_units = c->h_ctr[CTR_UNITS_RESERVED];   // units the frame needed (queued or not)
  return 0;
}

int axr_last_queues(axr_ctx *c, int64_t *out, int n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out || n < 0) return fail(AXR_EINVAL, "lastQueues output");
  if ((rc = axr_sync(c))) return rc;
  const uint32_t *h = c->h_ctr;
  const int64_t v[5] = {h[CTR_SMALL], h[CTR_SMALL_A], h[CTR_LARGE], h[CTR_UNITS], h[CTR_UNITS_A]};
  for (int k = 0; k < n && k < 5; k++) out[k] = v[k];
  return 0;
}

int axr_launch_count(axr_ctx *c, int64_t *total) {
  if (!c || !total) return fail(AXR_EINVAL, "null argument");
  *total = c->launches;
  return 0;
}

int axr_set_kernel_timing(axr_ctx *c, int enable) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = axr_sync(c))) return rc;
  c->timing = enable != 0;
  c->tacc.clear();
  return 0;
}

int axr_kernel_times(axr_ctx *c, int max, char *names, int name_len, double *total_ms, int64_t *launches, int *n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = axr_sync(c))) return rc;
  int k = 0;
  for (auto &acc : c->tacc) {
    if (k >= max) break;
    if (names && name_len > 0) {
      strncpy(names + (size_t)k * name_len, acc.name.c_str(), name_len - 1);
      names[(size_t)k * name_len + name_len - 1] = 0;
    }
    if (total_ms) total_ms[k] = acc.ms;
    if (launches) launches[k] = acc.n;
    k++;
  }
  if (n) *n = k;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched multi-view rendering: one cooperative persistent launch per batch,
// captured once in a CUDA graph together with the uploads of the camera and
// material tables (from pinned host buffers) and the read-back of the work
// counters; every render replays the graph.
// ---------------------------------------------------------------------------

struct axr_batch {
  axr_ctx *c = nullptr;
  std::vector<axr_view_desc> desc;
  struct Buf {
    uint16_t *ro = nullptr, *go = nullptr, *bo = nullptr;
    float *db = nullptr, *map = nullptr;
    uint64_t *keys = nullptr;
    uint32_t *small = nullptr, *large = nullptr, *items = nullptr, *list = nullptr, *ctr = nullptr;
    uint2 *units = nullptr;
    uint32_t cap_units = 0;
  };
  std::vector<Buf> buf;
  uint32_t cap_list = 0;
  BatchView *d_views = nullptr, *h_views = nullptr;
  // material tables: one segment per distinct group range of the views, each
  // with tri_base counted from the range's first triangle
  GroupDev *d_gdraw = nullptr, *d_gshadow = nullptr, *h_gdraw = nullptr, *h_gshadow = nullptr;
  std::vector<int> goff;        // per view: first entry of its segment
  uint32_t *d_bar = nullptr, *h_bar = nullptr, *h_ctrs = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cs = nullptr;    // read-back copies
  cudaStream_t side = nullptr;  // phased form: the alpha-tested branch
  cudaEvent_t done = nullptr, read_done = nullptr, ev_fork = nullptr, ev_coarse = nullptr, ev_join = nullptr;
  int mode = AXR_BATCH_PERSISTENT;
  bool shade_nrm = true;   // the shade variant launched (and captured): with the normal-mapped core
  int phantom = 0;                  // fault injection: barrier waits for blocks never launched
  long spin_limit = BARRIER_SPIN_LIMIT;
  bool graph = false, pending = false, reads = false;
  int grid = 0, per_sm_max = 0, min_chunk = MIN_CHUNK;
  int64_t launches = 0, bytes = 0;
};

namespace {

void batch_free_buffers(axr_batch *b) {
  for (auto &x : b->buf) {
    cudaFree(x.ro); cudaFree(x.go); cudaFree(x.bo); cudaFree(x.db); cudaFree(x.map); cudaFree(x.keys);
    cudaFree(x.small); cudaFree(x.large); cudaFree(x.items); cudaFree(x.list); cudaFree(x.ctr); cudaFree(x.units);
  }
  b->buf.clear();
}

int batch_check_views(axr_ctx *c, const axr_view_desc *v, int n) {
  if (!v || n < 1 || n > 64) return fail(AXR_EINVAL, "a batch holds 1..64 views");
  for (int k = 0; k < n; k++) {
    if (v[k].kind == AXR_VIEW_SHADED || v[k].kind == AXR_VIEW_SKIP) {
      if (v[k].w <= 0 || v[k].h <= 0 || v[k].w % TILE || (long)v[k].w * v[k].h > (1L << 27))
        return fail(AXR_EINVAL, "view %d: shaded views need w a positive multiple of 16", k);
      if (v[k].ncascades < 0 || v[k].ncascades > 2) return fail(AXR_EINVAL, "view %d: at most two cascades", k);
      for (int j = 0; j < v[k].ncascades; j++) {
        int cv = v[k].cascades[j];
        if (cv < 0) {
          int m = -1 - cv;   // a shadow map of the handle (addShadowMap / shadowMap)
          if (m >= MAX_SHADOWS || !c->shadows[m].map)
            return fail(AXR_EINVAL, "view %d: handle shadow map %d does not exist", k, m);
        } else if (cv >= n || v[cv].kind != AXR_VIEW_DEPTH) {
          return fail(AXR_EINVAL, "view %d: cascade %d is not a depth view of the batch", k, cv);
        }
      }
    } else if (v[k].kind == AXR_VIEW_DEPTH) {
      if (v[k].w < 4 || v[k].w > 16384) return fail(AXR_EINVAL, "view %d: depth map side %d", k, v[k].w);
    } else {
      return fail(AXR_EINVAL, "view %d: unknown kind %d", k, v[k].kind);
    }
    for (int j = 0; j < 3; j++)
      if (v[k].clear_color && (v[k].bg[j] < 0 || v[k].bg[j] > 65535))
        return fail(AXR_EINVAL, "view %d: background colour outside [0, 65535]", k);
    int ng = (int)c->groups.size();
    if (v[k].group_count < 0 || v[k].group_first < 0 ||
        (v[k].group_count > 0 && (long)v[k].group_first + v[k].group_count > ng) ||
        (v[k].group_count == 0 && v[k].group_first != 0))
      return fail(AXR_EINVAL, "view %d: group range [%d, +%d) outside the handle's %d groups", k, v[k].group_first,
                  v[k].group_count, ng);
  }
  return 0;
}

// The group range [first, first + count) a view draws.
void view_range(const axr_ctx *c, const axr_view_desc &v, int &first, int &count) {
  first = v.group_count > 0 ? v.group_first : 0;
  count = v.group_count > 0 ? v.group_count : (int)c->groups.size();
}

template <class T>
bool dalloc(T **p, size_t n, int64_t &bytes) {
  if (cudaMalloc(p, n) != cudaSuccess) return false;
  bytes += (int64_t)n;
  return true;
}

int batch_alloc(axr_batch *b, uint32_t units_per_view) {
  axr_ctx *c = b->c;
  uint32_t cap = (uint32_t)std::max(c->total_tris, 1);
  if (cap > MAX_LIST) return fail(AXR_EINVAL, "more than %u triangles", MAX_LIST);
  b->cap_list = cap;
  b->buf.assign(b->desc.size(), axr_batch::Buf());
  int64_t &B = b->bytes;
  for (size_t k = 0; k < b->desc.size(); k++) {
    const axr_view_desc &v = b->desc[k];
    axr_batch::Buf &x = b->buf[k];
    bool ok = dalloc(&x.ctr, sizeof(uint32_t) * CTR_N, B);
    if (v.kind == AXR_VIEW_SHADED || v.kind == AXR_VIEW_SKIP) {
      size_t n = (size_t)v.w * v.h;
      ok = ok && dalloc(&x.ro, n * 2, B) && dalloc(&x.go, n * 2, B) && dalloc(&x.bo, n * 2, B) &&
           dalloc(&x.db, n * 4, B) && dalloc(&x.keys, n * 8, B) && dalloc(&x.small, 4ull * cap, B) &&
           dalloc(&x.large, 4ull * cap, B) && dalloc(&x.items, 4ull * cap * MAX_CHUNKS, B) &&
           dalloc(&x.units, sizeof(uint2) * (size_t)units_per_view, B);
      x.cap_units = units_per_view;
      if (ok) {   // a new frame buffer: colour planes of ones (Ops0.py:111-113), depth 0
        k_fill_rgb<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(x.ro, x.go, x.bo, (int)n, 1, 1, 1);
        ok = cudaGetLastError() == cudaSuccess && cudaMemsetAsync(x.db, 0, n * 4, c->stream) == cudaSuccess;
      }
    } else {
      size_t n = (size_t)v.w * v.w;
      ok = ok && dalloc(&x.map, n * 4, B) && dalloc(&x.list, 4ull * cap, B) &&
           dalloc(&x.items, 4ull * cap * MAX_CHUNKS, B);
      if (ok) {
        k_clear_depth<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(x.map, v.w, v.w, 1);
        ok = cudaGetLastError() == cudaSuccess;
      }
    }
    if (!ok) return fail(AXR_ENOMEM, "batch view %zu buffers", k);
  }
  return 0;
}

// Host-side view table of the current cameras and buffers.
void batch_fill_views(axr_batch *b) {
  axr_ctx *c = b->c;
  for (size_t k = 0; k < b->desc.size(); k++) {
    const axr_view_desc &v = b->desc[k];
    axr_batch::Buf &x = b->buf[k];
    BatchView &V = b->h_views[k];
    memset(&V, 0, sizeof V);
    V.kind = v.kind;
    V.w = v.w;
    V.h = v.kind == AXR_VIEW_DEPTH ? v.w : v.h;
    int gf, gn;
    view_range(c, v, gf, gn);
    int tris = 0;
    for (int g = gf; g < gf + gn; g++) tris += c->groups[g].ntris;
    V.goff = b->goff[k];
    V.clear_rgb = v.kind == AXR_VIEW_SHADED && v.clear_color;
    for (int j = 0; j < 3; j++) V.bg[j] = (uint16_t)v.bg[j];
    if (v.kind == AXR_VIEW_SHADED || v.kind == AXR_VIEW_SKIP) {
      DrawParams &P = V.dp;
      P.groups = b->d_gdraw + V.goff; P.ngroups = gn; P.total_tris = tris;
      P.view.w = v.w; P.view.h = v.h;
      memcpy(P.view.pos, v.pos, sizeof v.pos); memcpy(P.view.vv, v.vm, sizeof v.vm);
      P.view.sscale = v.scale; P.view.cax = v.cax; P.view.cay = v.cay;
      memcpy(P.light.lint, c->lint, sizeof c->lint); memcpy(P.light.ldir, c->ldir, sizeof c->ldir);
      P.light.amb = c->amb;
      P.nsh = v.ncascades;
      for (int j = 0; j < v.ncascades; j++) {
        int cv = v.cascades[j];
        if (cv < 0) {
          const Shadow &hm = c->shadows[-1 - cv];
          P.sh[j].map = hm.map; P.sh[j].dim = hm.dim; P.sh[j].scale = hm.scale;
          memcpy(P.sh[j].pos, hm.pos, sizeof hm.pos); memcpy(P.sh[j].vv, hm.vv, sizeof hm.vv);
        } else {
          const axr_view_desc &sv = b->desc[cv];
          P.sh[j].map = b->buf[cv].map; P.sh[j].dim = sv.w; P.sh[j].scale = sv.scale;
          memcpy(P.sh[j].pos, sv.pos, sizeof sv.pos); memcpy(P.sh[j].vv, sv.vm, sizeof sv.vm);
        }
      }
      P.keys = x.keys; P.ro = x.ro; P.go = x.go; P.bo = x.bo; P.db = x.db;
      P.small_list = x.small; P.items = x.items; P.large_list = x.large; P.units = x.units; P.ctr = x.ctr;
      P.cap_list = b->cap_list; P.cap_units = x.cap_units;
      P.min_chunk = b->min_chunk;
    } else {
      ShadowParams &S = V.sp;
      S.groups = b->d_gshadow + V.goff; S.ngroups = gn; S.total_tris = tris;
      S.sh.map = x.map; S.sh.dim = v.w; S.sh.scale = v.scale;
      memcpy(S.sh.pos, v.pos, sizeof v.pos); memcpy(S.sh.vv, v.vm, sizeof v.vm);
      S.map = x.map; S.bias = v.bias; S.list = x.list; S.cap_list = b->cap_list; S.ctr = x.ctr;
      S.items = x.items; S.min_chunk = b->min_chunk;
    }
  }
}

// Enqueues one batch render on the handle's stream (captured or direct).
int batch_enqueue(axr_batch *b) {
  axr_ctx *c = b->c;
  cudaStream_t s = c->stream;
  size_t nv = b->desc.size(), ng = BATCH_TABLE;
  CK(cudaMemcpyAsync(b->d_views, b->h_views, sizeof(BatchView) * nv, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(b->d_gdraw, b->h_gdraw, sizeof(GroupDev) * ng, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(b->d_gshadow, b->h_gshadow, sizeof(GroupDev) * ng, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(b->d_bar, 0, sizeof(uint32_t) * BAR_WORDS, s));
  BatchParams B;
  B.views = b->d_views; B.nviews = (int)nv;
  B.groups_draw = b->d_gdraw; B.groups_shadow = b->d_gshadow; B.ngroups = BATCH_TABLE;
  B.bar = b->d_bar; B.nblocks = (uint32_t)(b->grid + b->phantom); B.spin_limit = b->spin_limit;
  if (b->mode == AXR_BATCH_PERSISTENT) {
    void *args[] = {&B};
    const void *kern = b->shade_nrm ? (const void *)k_batch<true> : (const void *)k_batch<false>;
    CK(cudaLaunchCooperativeKernel(kern, dim3(b->grid), dim3(128), args, 0, s));
  } else {
    // phased: clear, setup | opaque raster -> tiled opaque | (fork) alpha
    // raster -> (after the coarse units) tiled alpha | (join) fallback, shade
    int sms = c->sms;
    kb_clear<<<sms * 8, 256, 0, s>>>(B);
    kb_setup<<<sms * 8, 256, 0, s>>>(B);
    CK(cudaEventRecord(b->ev_fork, s));
    CK(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    kb_raster<false><<<sms * 8, 128, 0, s>>>(B);
    CK(cudaEventRecord(b->ev_coarse, s));
    kb_raster<true><<<sms * 6, 128, 0, b->side>>>(B);
    CK(cudaStreamWaitEvent(b->side, b->ev_coarse, 0));
    kb_tiled<true><<<sms * 6, 128, 0, b->side>>>(B);
    CK(cudaEventRecord(b->ev_join, b->side));
    kb_tiled<false><<<sms * 8, 128, 0, s>>>(B);
    CK(cudaStreamWaitEvent(s, b->ev_join, 0));
    kb_fallback<<<sms * 4, 128, 0, s>>>(B);
    if (b->shade_nrm) kb_shade<true><<<sms * 4, 256, 0, s>>>(B);
    else kb_shade<false><<<sms * 4, 256, 0, s>>>(B);
    CK(cudaGetLastError());
  }
  for (size_t k = 0; k < nv; k++)
    CK(cudaMemcpyAsync(b->h_ctrs + k * CTR_N, b->buf[k].ctr, sizeof(uint32_t) * CTR_N, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(b->h_bar, b->d_bar, sizeof(uint32_t) * BAR_WORDS, cudaMemcpyDeviceToHost, s));
  return 0;
}

int batch_build_graph(axr_batch *b) {
  axr_ctx *c = b->c;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  b->graph = false;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int rc = batch_enqueue(b);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc || e != cudaSuccess || !g) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    return 0;   // not capturable here: render with direct launches
  }
  if (cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess) b->graph = true;
  else cudaGetLastError();
  cudaGraphDestroy(g);
  return 0;
}

// Checks the last render's counters; grows a view's unit queue after an
// overflow (that render was completed by the fallback path).
int batch_settle(axr_batch *b) {
  if (!b->pending) return 0;
  CK(cudaEventSynchronize(b->done));
  b->pending = false;
  if (b->h_bar[2]) return fail(AXR_ECUDA, "batch grid barrier timed out");
  bool rebuild = false;
  for (size_t k = 0; k < b->desc.size(); k++) {
    uint32_t *h = b->h_ctrs + k * CTR_N;
    if (h[CTR_LIMIT]) return fail(AXR_ECUDA, "a raster loop of batch view %zu reached its safety limit", k);
    if (b->desc[k].kind == AXR_VIEW_SHADED && h[CTR_OVERFLOW]) {
      axr_batch::Buf &x = b->buf[k];
      uint64_t need = (uint64_t)h[CTR_UNITS_RESERVED] + h[CTR_UNITS_RESERVED] / 4 + 1024;
      if (need > 0x7fffffffull) need = 0x7fffffffull;
      cudaFree(x.units);
      x.units = nullptr;
      b->bytes -= (int64_t)sizeof(uint2) * x.cap_units;
      x.cap_units = 0;
      if (!dalloc(&x.units, sizeof(uint2) * need, b->bytes)) return fail(AXR_ENOMEM, "batch unit queue");
      x.cap_units = (uint32_t)need;
      rebuild = true;
    }
  }
  if (rebuild && b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; b->graph = false; }
  return 0;
}

}  // namespace

extern "C" {

int axr_batch_create(axr_ctx *c, const axr_view_desc *views, int nviews, axr_batch **out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out) return fail(AXR_EINVAL, "out is null");
  *out = nullptr;
  if ((rc = batch_check_views(c, views, nviews))) return rc;
  if (c->groups.empty()) return fail(AXR_ESTATE, "add texture groups before creating a batch");
  if ((rc = sync_all(c))) return rc;
  axr_batch *b = new axr_batch();
  b->c = c;
  b->desc.assign(views, views + nviews);
  uint32_t units0 = 1u << 20;
  if (const char *e = getenv("AXR_UNIT_QUEUE")) {
    long v = atol(e);
    if (v >= 1 && v <= (1L << 30)) units0 = (uint32_t)v;
  }
  size_t ng = BATCH_TABLE;
  b->goff.assign(nviews, 0);
  bool ok = cudaMalloc(&b->d_views, sizeof(BatchView) * nviews) == cudaSuccess &&
            cudaMallocHost(&b->h_views, sizeof(BatchView) * nviews) == cudaSuccess &&
            cudaMalloc(&b->d_gdraw, sizeof(GroupDev) * ng) == cudaSuccess &&
            cudaMalloc(&b->d_gshadow, sizeof(GroupDev) * ng) == cudaSuccess &&
            cudaMallocHost(&b->h_gdraw, sizeof(GroupDev) * ng) == cudaSuccess &&
            cudaMallocHost(&b->h_gshadow, sizeof(GroupDev) * ng) == cudaSuccess &&
            cudaMalloc(&b->d_bar, sizeof(uint32_t) * BAR_WORDS) == cudaSuccess &&
            cudaMallocHost(&b->h_bar, sizeof(uint32_t) * BAR_WORDS) == cudaSuccess &&
            cudaMallocHost(&b->h_ctrs, sizeof(uint32_t) * CTR_N * nviews) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->read_done, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_coarse, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess;
  if (!ok) rc = fail(AXR_ENOMEM, "batch tables");
  b->bytes += (int64_t)(sizeof(BatchView) * nviews + 2 * sizeof(GroupDev) * ng + sizeof(uint32_t) * BAR_WORDS);
  if (!rc) rc = batch_alloc(b, units0);
  if (!rc) {
    // the grid must be co-resident for either shade variant of the kernel
    int per_sm = 0, per_sm2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<true>, 128, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_batch<false>, 128, 0) != cudaSuccess ||
        std::min(per_sm, per_sm2) < 1)
      rc = fail(AXR_ECUDA, "batch kernel occupancy");
    per_sm = std::min(per_sm, per_sm2);
    b->per_sm_max = per_sm;
    b->grid = per_sm * c->sms;
  }
  if (rc) {
    axr_batch_destroy(b);
    return rc;
  }
  memset(b->h_bar, 0, sizeof(uint32_t) * BAR_WORDS);
  memset(b->h_ctrs, 0, sizeof(uint32_t) * CTR_N * nviews);
  *out = b;
  return 0;
}

int axr_batch_set_views(axr_batch *b, const axr_view_desc *views, int nviews) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  int rc = batch_check_views(b->c, views, nviews);
  if (rc) return rc;
  if (nviews != (int)b->desc.size()) return fail(AXR_EINVAL, "batch has %zu views", b->desc.size());
  for (int k = 0; k < nviews; k++) {
    bool was_depth = b->desc[k].kind == AXR_VIEW_DEPTH, is_depth = views[k].kind == AXR_VIEW_DEPTH;
    if (was_depth != is_depth || views[k].w != b->desc[k].w || (!is_depth && views[k].h != b->desc[k].h))
      return fail(AXR_EINVAL, "view %d changes kind or size; create a new batch", k);
  }
  b->desc.assign(views, views + nviews);
  return 0;
}

int axr_batch_render(axr_batch *b, const int32_t *flags, const int32_t *alpha_index, const uint8_t *cast, int ngroups) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  axr_ctx *c = b->c;
  int rc = check_ctx(c);
  if (rc) return rc;
  if (ngroups != (int)c->groups.size()) return fail(AXR_EINVAL, "render with %d groups, handle has %zu", ngroups,
                                                    c->groups.size());
  if ((uint32_t)std::max(c->total_tris, 1) > b->cap_list) return fail(AXR_ESTATE, "groups were added after the batch was created");
  if ((rc = batch_settle(b))) return rc;       // the previous render has left the pinned tables
  for (auto &v : b->desc) {
    if (v.kind != AXR_VIEW_SHADED || v.ncascades > 0 || !flags) continue;
    int gf, gn;
    view_range(c, v, gf, gn);
    for (int g = gf; g < gf + gn; g++)
      if (flags[g] & F_SHADOW) return fail(AXR_ESTATE, "shadow materials in a shaded view without cascades");
  }
  // material tables: shaded views use their range's groups, depth views the
  // casters of their range; one segment per distinct range, rebased so that
  // triangle ids count from the range's first triangle
  GroupDev tab[MAX_GROUPS];
  if ((rc = group_table(c, flags, alpha_index, nullptr, false, ngroups, tab))) return rc;
  memset(b->h_gdraw, 0, sizeof(GroupDev) * BATCH_TABLE);
  memset(b->h_gshadow, 0, sizeof(GroupDev) * BATCH_TABLE);
  std::vector<std::pair<int, int>> segs;
  std::vector<int> seg_off;
  int used = 0;
  for (size_t k = 0; k < b->desc.size(); k++) {
    int gf, gn;
    view_range(c, b->desc[k], gf, gn);
    size_t j = 0;
    while (j < segs.size() && segs[j] != std::make_pair(gf, gn)) j++;
    if (j == segs.size()) {
      if (used + gn > BATCH_TABLE)
        return fail(AXR_EINVAL, "the batch's views use more than %d group-table entries", BATCH_TABLE);
      segs.push_back({gf, gn});
      seg_off.push_back(used);
      int base = c->groups[gf].tri_base;
      for (int g = 0; g < gn; g++) {
        GroupDev d = tab[gf + g];
        d.tri_base -= base;
        b->h_gdraw[used + g] = d;
        d.flags &= F_ALPHA;
        d.enabled = cast ? (cast[gf + g] ? 1 : 0) : 1;
        b->h_gshadow[used + g] = d;
      }
      used += gn;
    }
    b->goff[k] = seg_off[j];
  }
  batch_fill_views(b);
  // the shade variant: with the normal-mapped core only when a shaded view
  // draws such a material (a change rebuilds the captured graph)
  bool nrm = false;
  for (auto &v : b->desc) {
    if (v.kind != AXR_VIEW_SHADED || !flags) continue;
    int gf, gn;
    view_range(c, v, gf, gn);
    for (int g = gf; g < gf + gn; g++) nrm = nrm || (flags[g] & F_NORMAL) != 0;
  }
  if (nrm != b->shade_nrm) {
    b->shade_nrm = nrm;
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  }
  // shaded views sampling the handle's own shadow maps wait for their writers
  for (auto &v : b->desc)
    for (int j = 0; j < v.ncascades; j++)
      if (v.cascades[j] < 0) CK(cudaStreamWaitEvent(c->stream, c->shadows[-1 - v.cascades[j]].ev_write, 0));
  // the framebuffers are free once the last render's read-back has left them
  if (b->reads) CK(cudaStreamWaitEvent(c->stream, b->read_done, 0));
  b->reads = false;
  if (!b->exec) {
    if ((rc = batch_build_graph(b))) return rc;
  }
  if (b->exec) {
    CK(cudaGraphLaunch(b->exec, c->stream));
  } else {
    if ((rc = batch_enqueue(b))) return rc;
  }
  b->launches++;
  c->launches++;
  // the handle's shadow maps this render sampled: it is their last reader
  for (auto &v : b->desc)
    for (int j = 0; j < v.ncascades; j++)
      if (v.kind == AXR_VIEW_SHADED && v.cascades[j] < 0) CK(cudaEventRecord(c->shadows[-1 - v.cascades[j]].ev_read, c->stream));
  CK(cudaEventRecord(b->done, c->stream));
  b->pending = true;
  return 0;
}

int axr_batch_get_frame(axr_batch *b, int view, uint16_t *r, uint16_t *g, uint16_t *bb, float *depth) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  axr_ctx *c = b->c;
  int rc = check_ctx(c);
  if (rc) return rc;
  if (view < 0 || view >= (int)b->desc.size()) return fail(AXR_EINVAL, "view %d", view);
  const axr_view_desc &v = b->desc[view];
  axr_batch::Buf &x = b->buf[view];
  if (v.kind != AXR_VIEW_DEPTH) {
    size_t n = (size_t)v.w * v.h;
    if (r) CK(cudaMemcpyAsync(r, x.ro, n * 2, cudaMemcpyDeviceToHost, c->stream));
    if (g) CK(cudaMemcpyAsync(g, x.go, n * 2, cudaMemcpyDeviceToHost, c->stream));
    if (bb) CK(cudaMemcpyAsync(bb, x.bo, n * 2, cudaMemcpyDeviceToHost, c->stream));
    if (depth) CK(cudaMemcpyAsync(depth, x.db, n * 4, cudaMemcpyDeviceToHost, c->stream));
  } else if (depth) {
    CK(cudaMemcpyAsync(depth, x.map, sizeof(float) * (size_t)v.w * v.w, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return batch_settle(b);
}

int axr_batch_get_ids(axr_batch *b, int view, int32_t *tri_id, uint8_t *cov) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  axr_ctx *c = b->c;
  int rc = check_ctx(c);
  if (rc) return rc;
  if (view < 0 || view >= (int)b->desc.size() || b->desc[view].kind != AXR_VIEW_SHADED)
    return fail(AXR_EINVAL, "view %d is not a shaded view", view);
  if ((rc = batch_settle(b))) return rc;
  size_t n = (size_t)b->desc[view].w * b->desc[view].h;
  int32_t *dt = nullptr;
  uint8_t *dc = nullptr;
  if (cudaMalloc(&dt, n * 4) != cudaSuccess || cudaMalloc(&dc, n) != cudaSuccess) {
    cudaFree(dt);
    return fail(AXR_ENOMEM, "id buffers");
  }
  k_ids<<<grid_for(c, (long)n, 256, 8), 256, 0, c->stream>>>(b->buf[view].keys, (int)n, dt, dc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && tri_id) e = cudaMemcpyAsync(tri_id, dt, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && cov) e = cudaMemcpyAsync(cov, dc, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dt);
  cudaFree(dc);
  if (e != cudaSuccess) return fail(AXR_ECUDA, "batch ids: %s", cudaGetErrorString(e));
  return 0;
}

int axr_batch_read_async(axr_batch *b, int view, uint16_t *r, uint16_t *g, uint16_t *bb, float *depth) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  int rc = check_ctx(b->c);
  if (rc) return rc;
  if (view < 0 || view >= (int)b->desc.size() || b->desc[view].kind != AXR_VIEW_SHADED)
    return fail(AXR_EINVAL, "view %d is not a shaded view of the last render", view);
  const axr_view_desc &v = b->desc[view];
  axr_batch::Buf &x = b->buf[view];
  size_t n = (size_t)v.w * v.h;
  CK(cudaStreamWaitEvent(b->cs, b->done, 0));
  if (r) CK(cudaMemcpyAsync(r, x.ro, n * 2, cudaMemcpyDeviceToHost, b->cs));
  if (g) CK(cudaMemcpyAsync(g, x.go, n * 2, cudaMemcpyDeviceToHost, b->cs));
  if (bb) CK(cudaMemcpyAsync(bb, x.bo, n * 2, cudaMemcpyDeviceToHost, b->cs));
  if (depth) CK(cudaMemcpyAsync(depth, x.db, n * 4, cudaMemcpyDeviceToHost, b->cs));
  CK(cudaEventRecord(b->read_done, b->cs));
  b->reads = true;
  return 0;
}

int axr_batch_query(axr_batch *b) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  if (b->pending) {
    cudaError_t e = cudaEventQuery(b->done);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return fail(AXR_ECUDA, "batch query: %s", cudaGetErrorString(e));
  }
  if (b->reads) {
    cudaError_t e = cudaEventQuery(b->read_done);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return fail(AXR_ECUDA, "batch read-back: %s", cudaGetErrorString(e));
  }
  int rc = batch_settle(b);
  return rc ? rc : 1;
}

int axr_batch_phase_times(axr_batch *b, float ms[5]) {
  if (!b || !ms) return fail(AXR_EINVAL, "null batch or output");
  int rc = batch_settle(b);
  if (rc) return rc;
  const uint64_t *t = reinterpret_cast<const uint64_t *>(b->h_bar + 4);
  for (int k = 0; k < 5; k++) ms[k] = t[k + 1] >= t[k] ? (float)((t[k + 1] - t[k]) * 1e-6) : 0.f;
  return 0;
}

int axr_batch_bytes(axr_batch *b, int64_t *bytes) {
  if (!b || !bytes) return fail(AXR_EINVAL, "null batch or output");
  *bytes = b->bytes;
  return 0;
}

int axr_batch_stats(axr_batch *b, int64_t *renders, int *graph, int *grid) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  if (renders) *renders = b->launches;
  if (graph) *graph = b->graph ? 1 : 0;
  if (grid) *grid = b->grid;
  return 0;
}

int axr_batch_set_tuning(axr_batch *b, int blocks_per_sm, int min_chunk) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  if (blocks_per_sm < 1 || blocks_per_sm > b->per_sm_max)
    return fail(AXR_EINVAL, "blocks per SM %d outside [1, %d]", blocks_per_sm, b->per_sm_max);
  if (min_chunk < 1 || min_chunk > 256) return fail(AXR_EINVAL, "chunk rows %d outside [1, 256]", min_chunk);
  int rc = batch_settle(b);
  if (rc) return rc;
  CK(cudaStreamSynchronize(b->c->stream));
  b->grid = blocks_per_sm * b->c->sms;
  b->min_chunk = min_chunk;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; b->graph = false; }
  return 0;
}

int axr_batch_set_mode(axr_batch *b, int mode) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  if (mode != AXR_BATCH_PERSISTENT && mode != AXR_BATCH_PHASED) return fail(AXR_EINVAL, "batch mode %d", mode);
  int rc = batch_settle(b);
  if (rc) return rc;
  CK(cudaStreamSynchronize(b->c->stream));
  b->mode = mode;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; b->graph = false; }
  return 0;
}

int axr_batch_inject_barrier_stall(axr_batch *b, int phantom_blocks, long long spin_limit) {
  if (!b) return fail(AXR_EINVAL, "null batch");
  if (phantom_blocks < 0 || phantom_blocks > 1024) return fail(AXR_EINVAL, "phantom blocks %d", phantom_blocks);
  if (spin_limit < 1 || spin_limit > BARRIER_SPIN_LIMIT) return fail(AXR_EINVAL, "spin limit %lld", spin_limit);
  int rc = batch_settle(b);
  if (rc) return rc;
  CK(cudaStreamSynchronize(b->c->stream));
  b->phantom = phantom_blocks;
  b->spin_limit = (long)spin_limit;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; b->graph = false; }
  return 0;
}

int axr_set_shadow_mode(axr_ctx *c, int mode, int slice) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  if (mode < 0 || mode > 2) return fail(AXR_EINVAL, "shadow mode %d outside [0, 2]", mode);
  if (slice != 0 && (slice < 32 || slice > (1 << 20)))
    return fail(AXR_EINVAL, "shadow slice %d outside [32, 2^20] (0 keeps it)", slice);
  c->shadow_mode = mode;
  if (slice) c->shadow_slice = slice;
  return 0;
}

int axr_set_tuning(axr_ctx *c, int min_chunk) {
  if (!c) return fail(AXR_EINVAL, "null handle");
  if (min_chunk < 1 || min_chunk > 256) return fail(AXR_EINVAL, "chunk rows %d outside [1, 256]", min_chunk);
  c->min_chunk = min_chunk;
  return 0;
}

int axr_batch_destroy(axr_batch *b) {
  if (!b) return 0;
  if (b->c) cudaStreamSynchronize(b->c->stream);
  if (b->cs) { cudaStreamSynchronize(b->cs); cudaStreamDestroy(b->cs); }
  if (b->side) { cudaStreamSynchronize(b->side); cudaStreamDestroy(b->side); }
  if (b->read_done) cudaEventDestroy(b->read_done);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_coarse) cudaEventDestroy(b->ev_coarse);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  batch_free_buffers(b);
  cudaFree(b->d_views); cudaFree(b->d_gdraw); cudaFree(b->d_gshadow); cudaFree(b->d_bar);
  if (b->h_views) cudaFreeHost(b->h_views);
  if (b->h_gdraw) cudaFreeHost(b->h_gdraw);
  if (b->h_gshadow) cudaFreeHost(b->h_gshadow);
  if (b->h_bar) cudaFreeHost(b->h_bar);
  if (b->h_ctrs) cudaFreeHost(b->h_ctrs);
  if (b->done) cudaEventDestroy(b->done);
  delete b;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Shadow depth pass without device allocation.
//
// Some callers cannot call cudaMalloc/cudaFree while they render: an engine
// that hands all device memory to its own allocator, or a frame loop that
// must not hit the implicit device synchronisation those calls can cause
// while other streams are busy.  axr_shadow_map_noalloc serves them: the
// caller passes device pointers for the triangles and the depth map, and the
// only scratch (the list of accepted triangles and two work counters) lives
// in the file-scope array below, which every GPU that loads this library
// holds until the process exits.
// ---------------------------------------------------------------------------

namespace {

constexpr uint32_t NOALLOC_MAX_TRIS = 1u << 20;     // 4 MiB of triangle list per GPU
constexpr int NOALLOC_MAX_DIM = 16384;
// Each caster is one work item whose rows lie in the map plus the setup's
// 120-texel guard bands (trisetupOrtho.c), so no raster loop reaches the
// safety cap, which this entry point could not report (it returns before
// the GPU runs).
static_assert(NOALLOC_MAX_DIM + 240 < LOOP_LIMIT, "a caster's rows stay below the loop cap");
constexpr uint32_t NOALLOC_WORDS = NOALLOC_MAX_TRIS + CTR_N;
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_WORDS];

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocSlot {
  unsigned long long ctx_id;   // the context the address was resolved in
  uint32_t *ptr;               // device address of the array there
};
NoallocSlot g_noalloc[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;
bool g_ctx_fns_looked_up = false;

// One caster group, passed by value (no device-side table).
__global__ void __launch_bounds__(256) k_shadow_setup_noalloc(GroupDev G, ShadowParams S) {
  __shared__ GroupDev sg[1];
  if (threadIdx.x == 0) sg[0] = G;
  __syncthreads();
  int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < S.total_tris; base += gridDim.x * blockDim.x) {
    int t = base + threadIdx.x;
    bool ok, alpha;
    int rows, g, ix[3], iy[3];
    float z[3];
    shadow_classify(sg, S, t, ok, alpha, rows, g, ix, iy, z);
    shadow_append(S, t, ok, alpha, rows, lane);   // S.items is null: no row chunks
  }
}

template <bool ALPHA>
__global__ void __launch_bounds__(128, ALPHA ? 6 : 8) k_shadow_raster_noalloc(GroupDev G, ShadowParams S) {
  __shared__ GroupDev sg[1];
  __shared__ ShadowQ<ALPHA> qs[4];
  if (threadIdx.x == 0) sg[0] = G;
  __syncthreads();
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  shadow_warp_loop<ALPHA>(S, sg, qs[w], lane, ALPHA ? CTR_SH_LIST_A : CTR_SH_LIST, ALPHA ? CTR_SH_WORK_A : CTR_SH_WORK);
}

// The process-unique id of the context current on this thread (binding the
// device's primary context first if none is), through the driver's
// cuCtxGetCurrent / cuCtxGetId, which only read host state.  Returns false
// when the driver does not provide them.
bool current_ctx_id(int dev, unsigned long long *id) {
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_ctx_fns_looked_up) {
      g_ctx_fns_looked_up = true;
      void *f1 = nullptr, *f2 = nullptr;
      cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
      cudaError_t e1 = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1);
      cudaError_t e2 = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2);
      if (e1 == cudaSuccess && e2 == cudaSuccess && q1 == cudaDriverEntryPointSuccess &&
          q2 == cudaDriverEntryPointSuccess && f1 && f2) {
        g_ctx_current = (PFN_cuCtxGetCurrent_v4000)f1;
        g_ctx_id = (PFN_cuCtxGetId_v12000)f2;
      }
      if (e1 != cudaSuccess || e2 != cudaSuccess) cudaGetLastError();   // the failed lookup's error is not the caller's
    }
  }
  if (!g_ctx_current || !g_ctx_id) return false;
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS) return false;
  if (!ctx) {
    if (cudaSetDevice(dev) != cudaSuccess || g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  }
  return g_ctx_id(ctx, id) == CUDA_SUCCESS;
}

// Resolves the device address of g_noalloc_scratch in the current context
// (the host-side name is only a stand-in for it).  The address is cached per
// device together with the context's id and looked up again only when the
// context changes: after cudaDeviceReset the runtime loads the module into a
// new context, where the array may sit elsewhere.  Without the driver's
// context id it is looked up on every call.
int noalloc_scratch(uint32_t **out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(AXR_EINVAL, "device %d beyond %d", dev, NOALLOC_MAX_DEVICES);
  unsigned long long id = 0;
  bool have_id = current_ctx_id(dev, &id);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocSlot &sl = g_noalloc[dev];
  if (have_id && sl.ptr && sl.ctx_id == id) {
    *out = sl.ptr;
    return 0;
  }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return fail(AXR_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
  sl.ptr = have_id ? (uint32_t *)p : nullptr;   // without a context id a cached copy cannot be checked
  sl.ctx_id = id;
  *out = (uint32_t *)p;
  return 0;
}

}  // namespace

extern "C" int axr_shadow_map_noalloc(const float *xyz, const float *uv, const uint8_t *alpha_mask, int alpha_side,
                                      int ntris, const float pos[3], const float vm[9], float scale, float bias,
                                      float *map, int dim, void *stream) {
  if (!xyz || !pos || !vm || !map) return fail(AXR_EINVAL, "null argument");
  if (ntris < 0 || (uint32_t)ntris > NOALLOC_MAX_TRIS)
    return fail(AXR_EINVAL, "axr_shadow_map_noalloc takes at most %u triangles per call, got %d", NOALLOC_MAX_TRIS,
                ntris);
  if (dim < 4 || dim > NOALLOC_MAX_DIM)
    return fail(AXR_EINVAL, "shadow map size %d outside [4, %d]", dim, NOALLOC_MAX_DIM);
  if (alpha_mask && (!uv || !is_pow2(alpha_side)))
    return fail(AXR_EINVAL, "alpha casters need uv and a power-of-two mask side (got %d)", alpha_side);
  uint32_t *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  if (ntris == 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  GroupDev G;
  memset(&G, 0, sizeof G);
  G.xyz = xyz; G.uv = uv; G.ntris = ntris; G.tri_base = 0; G.enabled = 1;
  if (alpha_mask) { G.flags = F_ALPHA; G.amask = alpha_mask; G.alen = alpha_side; }
  ShadowParams S;
  memset(&S, 0, sizeof S);
  S.groups = nullptr; S.ngroups = 1; S.total_tris = ntris;
  S.sh.map = map; S.sh.dim = dim; S.sh.scale = scale;
  memcpy(S.sh.pos, pos, sizeof S.sh.pos);
  memcpy(S.sh.vv, vm, sizeof S.sh.vv);
  S.map = map; S.bias = bias;
  S.list = scratch;
  S.cap_list = NOALLOC_MAX_TRIS;
  S.ctr = scratch + NOALLOC_MAX_TRIS;
  // the counters keep the previous call's values: start them at zero
  CK(cudaMemsetAsync(S.ctr, 0, sizeof(uint32_t) * CTR_N, s));
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long g = ((long)ntris + 255) / 256;
  if (g > (long)sms * 16) g = (long)sms * 16;
  k_shadow_setup_noalloc<<<(int)std::max(g, 1L), 256, 0, s>>>(G, S);
  if (alpha_mask) k_shadow_raster_noalloc<true><<<sms * 6, 128, 0, s>>>(G, S);
  else k_shadow_raster_noalloc<false><<<sms * 8, 128, 0, s>>>(G, S);
  CK(cudaGetLastError());
  return 0;
}
