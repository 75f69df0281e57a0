// ref_harness.cpp -- host side of oracle/_ref (TEST INFRASTRUCTURE ONLY).
//
// Restates the host orchestration of the reference's CLDraw
// (PyOpenCL27C/Ops0.py:93-910, drawAll at :471-648; shadowMap in
// PyOpenCL27C/Ops.py:1089-1141) with the reference's device buffer layouts
// (float3 as 16 bytes, SP/ZZ/TIA/TIB/TNA/TNB/TOA/TOB/IBUF/NBUF/AL), and runs
// the reference's own kernels (compiled by build_ref.py) one work-item at a
// time.  Serial mode (nthreads == 1) runs work-groups in order and work-items
// in id order, which is the canonical semantics the oracle restates; the only
// adjustment is that a tile's local depth copy is loaded before the tile's
// first triangle, and that the bin count the tile kernel resets at its end is
// seen by all of its work-items.  Threaded mode runs one work-group per
// OpenMP thread (used only for timing).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>
#include <omp.h>
#include "ref_shim.h"

namespace cl_shim {
thread_local int g_group[2];
thread_local int g_local[2];
thread_local int g_global[2];
thread_local void (*g_barrier)() = nullptr;

namespace ref_trisetup {
void setup(float3 *XYZ, float3 *VN, int *TIA, int *TIB, int *TNA, int *TNB, float2 *XY, float *ZZ,
           float *Vpos, float3 *VV, const float sScale, const int wF, const int hF, const float cAX,
           const float cAY, const int lenP);
}
namespace ref_trisetup_cull {
void setup(float3 *XYZ, float3 *VN, int *TIA, int *TIB, int *TNA, int *TNB, float2 *XY, float *ZZ,
           float *Vpos, float3 *VV, const float sScale, const int wF, const int hF, const float cAX,
           const float cAY, const int lenP);
}
namespace ref_trisetup_ortho {
void setup(float3 *XYZ, int *TI, int *TN, int2 *XY, float *ZZ, float *Vpos, float3 *VV, const float shBias,
           const float sScale, const int wF, const int hF, const float cAX, const float cAY, const int lenP);
}
namespace ref_gather {
void setup(int *TI, int *TN, int *TO, int *AL, const int tn, const int numBlocks);
}
namespace ref_coarse {
void draw(int *TO, int *F, int *FN, float2 *P, int wF, int hF, int lenP);
}
namespace ref_draw {
void draw(int *TO, int *TN, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, ushort *TR, ushort *TG, ushort *TB,
          const int lenT, const int wF, const int hF);
void drawSmall(int *TO, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, ushort *TR, ushort *TG,
               ushort *TB, const int lenT, const int wF, const int hF, const int lenP);
float *local_ZBuf();
}
// Shaders_src/av_draw_normmap_mip.c expanded by the reference's AVSL generator
namespace ref_draw_mip {
void draw(int *TO, int *TN, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int numMip, uchar3 *NM,
          float *Vpos, float3 *LInt, float3 *LDir, float *SD, const int wS, const float sScale, float3 *SV,
          float *SPos, const float mipBias, const int wF, const int hF);
void drawSmall(int *TO, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int numMip,
               uchar3 *NM, float *Vpos, float3 *LInt, float3 *LDir, float *SD, const int wS, const float sScale,
               float3 *SV, float *SPos, const float mipBias, const int wF, const int hF, const int lenP);
float *local_ZBuf();
}
// Shaders_src/av_draw_normmap.c and av_draw_normmap_alpha.c, expanded likewise
namespace ref_draw_nrm {
void draw(int *TO, int *TN, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int lenT, uchar3 *NM,
          float roughness, char isMetal, float *Vpos, float3 *LInt, float3 *LDir, float *SD, const int wS,
          const float sScale, float3 *SV, float *SPos, const int wF, const int hF);
void drawSmall(int *TO, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int lenT, uchar3 *NM,
               float roughness, char isMetal, float *Vpos, float3 *LInt, float3 *LDir, float *SD, const int wS,
               const float sScale, float3 *SV, float *SPos, const int wF, const int hF, const int lenP);
float *local_ZBuf();
}
namespace ref_draw_nrm_alpha {
void draw(int *TO, int *TN, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int lenT, bool *TA,
          uchar3 *NM, float roughness, char isMetal, float *Vpos, float3 *LInt, float3 *LDir, float *SD,
          const int wS, const float sScale, float3 *SV, float *SPos, const int wF, const int hF);
void drawSmall(int *TO, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, ushort *TR, ushort *TG, ushort *TB, const int lenT, bool *TA,
               uchar3 *NM, float roughness, char isMetal, float *Vpos, float3 *LInt, float3 *LDir, float *SD,
               const int wS, const float sScale, float3 *SV, float *SPos, const int wF, const int hF,
               const int lenP);
float *local_ZBuf();
}
namespace ref_draw_alpha {
void draw(int *TO, int *TN, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, ushort *TR, ushort *TG, ushort *TB,
          const int lenT, bool *TA, const int wF, const int hF);
void drawSmall(int *TO, ushort *Ro, ushort *Go, ushort *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, ushort *TR, ushort *TG,
               ushort *TB, const int lenT, bool *TA, const int wF, const int hF, const int lenP);
float *local_ZBuf();
}
namespace ref_drawmin {
void draw(int *TO, float *F, int2 *P, float *Z, int wF, int hF, int lenP);
}
namespace ref_drawmin_alpha {
void draw(int *TO, float *F, int2 *P, float *Z, float2 *UV, bool *TA, int lenT, int wF, int hF, int lenP);
}
namespace ref_clearzb {
void clearFrame(float *F, const int wF, const int hF, const int BS, const int lenP);
}
namespace ref_gamma {
void g(ushort *Ro, ushort *Go, ushort *Bo, const float exposure, const int wF, const int hF, const int BS,
       const int stepW, const int stepH);
}
namespace ref_drawmulti {
void draw(int *TO, int *TN, sat_u16 *Ro, sat_u16 *Go, sat_u16 *Bo, float *F, float2 *P, float *Z, float2 *UV,
          float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, sat_u16 *TR, sat_u16 *TG, sat_u16 *TB,
          const int lenT, sat_u16 *TR2, sat_u16 *TG2, sat_u16 *TB2, const int lenT2, sat_u16 *TR3, sat_u16 *TG3,
          sat_u16 *TB3, const int lenT3, sat_u16 *TR4, sat_u16 *TG4, sat_u16 *TB4, const int lenT4, const int wF,
          const int hF);
void drawSmall(int *TO, sat_u16 *Ro, sat_u16 *Go, sat_u16 *Bo, float *F, float2 *P, float *Z, float2 *UV,
               float3 *I, float3 *N, float3 *PXYZ, float3 *LInt, float3 *LDir, sat_u16 *TR, sat_u16 *TG,
               sat_u16 *TB, const int lenT, sat_u16 *TR2, sat_u16 *TG2, sat_u16 *TB2, const int lenT2,
               sat_u16 *TR3, sat_u16 *TG3, sat_u16 *TB3, const int lenT3, sat_u16 *TR4, sat_u16 *TG4,
               sat_u16 *TB4, const int lenT4, const int wF, const int hF, const int lenP);
float *local_ZBuf();
}
namespace ref_ssao {
void ao(ushort *Ro, ushort *Go, ushort *Bo, float *F, const float sScale, float *R, const int wF, const int hF,
        const int BS);
}
namespace ref_dof {
void dof(ushort *Ro, ushort *Go, ushort *Bo, ushort *R2, ushort *G2, ushort *B2, float *F, const float focus,
         const int wF, const int hF, const int BS);
}
namespace ref_blur {
void blurH(ushort *r2, ushort *g2, ushort *b2, ushort *Rt, ushort *Gt, ushort *Bt, ushort *Ro, ushort *Go, ushort *Bo,
           int wF, int hF, const int BS, int stepW, float stepH);
}
namespace ref_blur2 {
void blurV(ushort *Ro, ushort *Go, ushort *Bo, ushort *Rt, ushort *Gt, ushort *Bt, ushort *r2, ushort *g2, ushort *b2,
           int wF, int hF, const int BS, int stepW, float stepH);
}
namespace ref_vert {
void transform(float3 *XYZ, float3 *VN, float3 *OldR, float3 *RR, float *O, const int lStart, const int lEnd);
void Ttranslate(float3 *XYZ, float *O, const int lStart, const int lEnd);
void vertL(float3 *XYZ, float3 *VN, float3 *I, float3 *LInt, float3 *LDir, float3 *PInt, float3 *PPos,
           float3 *SInt, float3 *SDir, float3 *SPos, const float ambLight, const char lenD, const short lenP,
           const int lenS, const int lenV);
}
}  // namespace cl_shim

using namespace cl_shim;

static const int BS = 128;      // BLOCK_SIZE = TILE_BUF (Ops0.py:19-21)
static const int TILE_BUF = 128;

namespace {

struct Group {
  int V = 0, T = 0;
  std::vector<float3> xyz, vn, li;
  std::vector<float2> uv, sp;
  std::vector<float> zz;
  std::vector<int> tia, tib, tna, tnb, toa, tob;
  std::vector<ushort> tr, tg, tb;
  int tex_size = 0;
  // the normal-mapped materials: the normal map (one texel per texel of the
  // texture or chain), roughness and metal switch, and the mipBias
  std::vector<uchar3> nm;
  float roughness = 0;
  int is_metal = 0;
  float mip_bias = 0;
};

struct Shadow {
  std::vector<float> map;
  int dim = 0;
  float scale = 1;
  float pos[3] = {0, 0, 0};
  float3 vec[3];
};

struct Ctx {
  int W, H, WC, HC;
  std::vector<Group> groups;
  std::vector<std::vector<uint8_t>> alphas;
  std::vector<int> alpha_len;
  std::vector<ushort> ro, go, bo;
  std::vector<float> db;
  std::vector<int> ibuf, nbuf, al;
  float vpos[3] = {0, 0, 0};
  float3 vmat[3];
  float sscale = 1, cax = 1, cay = 1;
  float3 lint[1], ldir[1];
  Shadow shadows[8];
  int overflow = 0;
  int mip_kernels = 0;   // mip groups (flags bit 0) drawn by ref_draw_mip
  int normal_shadow = -1; // the cascade the normal-mapped materials sample (-1: none)
};

// the shadow arguments of the normal-mapped materials (getShadow, Ops.py:621-622)
struct NormalShadow {
  float *SD;
  int wS;
  float scale;
  float3 *SV;
  float *SPos;
};
float g_no_shadow_map[16] = {65535, 65535, 65535, 65535, 65535, 65535, 65535, 65535,
                             65535, 65535, 65535, 65535, 65535, 65535, 65535, 65535};
float3 g_no_shadow_vec[3];
float g_no_shadow_pos[3] = {0, 0, 0};
NormalShadow normal_shadow(Ctx *c) {
  if (c->normal_shadow >= 0 && c->normal_shadow < 8 && !c->shadows[c->normal_shadow].map.empty()) {
    Shadow &s = c->shadows[c->normal_shadow];
    return {s.map.data(), s.dim / 2, s.scale, s.vec, s.pos};
  }
  return {g_no_shadow_map, 2, 1.0f, g_no_shadow_vec, g_no_shadow_pos};   // no tap can lie in [2, 2)
}

// run kernel `fn(bx, tx)` over a 1-D grid of `ng` groups of BS items
template <class F>
void grid1(int ng, int nthreads, F fn) {
  if (nthreads <= 1) {
    for (int bx = 0; bx < ng; bx++) {
      g_group[0] = bx; g_group[1] = 0;
      for (int tx = 0; tx < BS; tx++) {
        g_local[0] = tx; g_local[1] = 0;
        fn(bx, tx);
      }
    }
  } else {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int bx = 0; bx < ng; bx++) {
      g_group[0] = bx; g_group[1] = 0;
      for (int tx = 0; tx < BS; tx++) {
        g_local[0] = tx; g_local[1] = 0;
        fn(bx, tx);
      }
    }
  }
}

float3 f3(const float *p) { return make_float3(p[0], p[1], p[2]); }

// a barrier across the threads of one launch (one thread per work-item)
struct LaunchBarrier {
  std::mutex m;
  std::condition_variable cv;
  int n = 0, waiting = 0;
  long gen = 0;
  void wait() {
    std::unique_lock<std::mutex> lk(m);
    long g = gen;
    if (++waiting == n) {
      waiting = 0;
      gen++;
      cv.notify_all();
    } else {
      cv.wait(lk, [&] { return gen != g; });
    }
  }
};
LaunchBarrier *g_launch_barrier = nullptr;
void launch_barrier_wait() { g_launch_barrier->wait(); }

// runs fn(bx, by, tx, ty) for every work-item of an (sx x sy) x (tx x ty)
// launch, one thread each, with barrier() ordering the whole launch
template <class F>
void launch_threads(int gx, int gy, int lx, int ly, F fn) {
  LaunchBarrier b;
  b.n = gx * gy * lx * ly;
  g_launch_barrier = &b;
  std::vector<std::thread> th;
  for (int by = 0; by < gy; by++)
    for (int bx = 0; bx < gx; bx++)
      for (int ty = 0; ty < ly; ty++)
        for (int tx = 0; tx < lx; tx++)
          th.emplace_back([=] {
            g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
            g_barrier = launch_barrier_wait;
            fn();
            g_barrier = nullptr;
          });
  for (auto &t : th) t.join();
  g_launch_barrier = nullptr;
}

sat_u16 *su(std::vector<ushort> &v) { return reinterpret_cast<sat_u16 *>(v.data()); }

// the 4-way blend material (Ops0.py:533-545, 604-617): this group's texture
// and the next three groups'
struct Multi {
  sat_u16 *t[4][3];
  int len[4];
};
Multi multi_textures(Ctx *c, int tn) {
  Multi m;
  for (int k = 0; k < 4; k++) {
    Group &G = c->groups[tn + k];
    m.t[k][0] = su(G.tr); m.t[k][1] = su(G.tg); m.t[k][2] = su(G.tb);
    m.len[k] = G.tex_size;
  }
  return m;
}

std::vector<float3> f3s(const float *p, int n) {
  std::vector<float3> v(n > 0 ? n : 1, make_float3(0, 0, 0));   // the reference binds a 4-byte buffer when empty
  for (int i = 0; i < n; i++) v[i] = f3(p + 3 * (size_t)i);
  return v;
}

// 1-D launch of `ng` groups of BS work-items with global ids set
template <class F>
void grid1_global(int ng, F fn) {
  for (int bx = 0; bx < ng; bx++) {
    g_group[0] = bx; g_group[1] = 0;
    for (int tx = 0; tx < BS; tx++) {
      g_local[0] = tx; g_local[1] = 0;
      g_global[0] = bx * BS + tx; g_global[1] = 0;
      fn();
    }
  }
}

}  // namespace

extern "C" {

void *ref_create(int w, int h) {
  Ctx *c = new Ctx();
  c->W = w; c->H = h; c->WC = w / 16; c->HC = h / 16;
  c->ro.assign((size_t)w * h, 1); c->go.assign((size_t)w * h, 1); c->bo.assign((size_t)w * h, 1);
  c->db.assign((size_t)w * h, 65535.f);
  c->ibuf.assign((size_t)c->WC * c->HC * TILE_BUF + TILE_BUF * 64, -1);
  c->nbuf.assign((size_t)c->WC * c->HC, 0);
  c->al.assign(64, 0);
  return c;
}

void ref_destroy(void *h) { delete (Ctx *)h; }

// CLDraw.addTextureGroup (Ops0.py:276-322) plus the LI buffer vertLight fills
int ref_add_group(void *h, const float *xyz, const float *uv, const float *vn, const float *li, int ntris,
                  const uint16_t *r, const uint16_t *g, const uint16_t *b, long ntexels, int tex_size) {
  Ctx *c = (Ctx *)h;
  Group G;
  G.T = ntris; G.V = ntris * 3;
  G.xyz.resize(G.V); G.vn.resize(G.V); G.li.resize(G.V); G.uv.resize(G.V);
  for (int v = 0; v < G.V; v++) {
    G.xyz[v] = f3(xyz + 3 * (size_t)v);
    G.vn[v] = f3(vn + 3 * (size_t)v);
    G.li[v] = f3(li + 3 * (size_t)v);
    G.uv[v] = make_float2(uv[2 * (size_t)v], uv[2 * (size_t)v + 1]);
  }
  G.sp.assign(G.V, make_float2(0, 0));
  G.zz.assign(G.V, 0);
  int gs = G.T / BS + 1;
  G.tia.assign((size_t)gs * BS, 0); G.tib.assign((size_t)gs * BS, 0);
  G.tna.assign(gs, 0); G.tnb.assign(gs, 0);
  G.toa.assign((size_t)gs * BS, 0); G.tob.assign((size_t)gs * BS, 0);
  G.tr.assign(r, r + ntexels); G.tg.assign(g, g + ntexels); G.tb.assign(b, b + ntexels);
  G.tex_size = tex_size;
  c->groups.push_back(std::move(G));
  return (int)c->groups.size() - 1;
}

int ref_add_alpha(void *h, const uint8_t *mask, int len) {
  Ctx *c = (Ctx *)h;
  c->alphas.emplace_back(mask, mask + (size_t)len * len);
  c->alpha_len.push_back(len);
  return (int)c->alphas.size() - 1;
}

// Draws the mip groups with the reference's normal-mapped mip material
// (on != 0), each with its mipBias and a flat normal map (128, 128, 255).
// Its shadow lookup `sampleShadow` is defined nowhere in the reference; the
// build gives it a stand-in returning 0, which is exact for the pin's use:
// with a zero light intensity the shadow term and the specular term vanish.
int ref_set_mip_kernels(void *h, int on, const float *bias, int n) {
  Ctx *c = (Ctx *)h;
  if (n != (int)c->groups.size()) return -1;
  c->mip_kernels = on;
  for (int i = 0; i < n; i++) {
    Group &G = c->groups[i];
    G.mip_bias = bias ? bias[i] : 0.f;
    if (G.nm.empty()) {
      uchar3 flat;
      flat.x = 128; flat.y = 128; flat.z = 255; flat.pad_ = 0;
      G.nm.assign(G.tr.size(), flat);
    }
  }
  return 0;
}

// CLDraw.addNrmMap + a normal-mapped material on group g: the normal map as
// RGBA bytes (one texel per texel of the group's texture or chain), the
// material's roughness (its "normal" pair's second value) and metal switch,
// and its mipBias (the normal-mapped mip material).  The cascade the
// materials sample is set with ref_set_normal_shadow.
int ref_set_normal(void *h, int g, const uint8_t *rgba, long ntexels, float roughness, int is_metal,
                   float mip_bias) {
  Ctx *c = (Ctx *)h;
  if (g < 0 || g >= (int)c->groups.size() || ntexels < (long)c->groups[g].tr.size()) return -1;
  Group &G = c->groups[g];
  G.nm.resize(ntexels);
  for (long i = 0; i < ntexels; i++) {
    G.nm[i].x = rgba[4 * i]; G.nm[i].y = rgba[4 * i + 1]; G.nm[i].z = rgba[4 * i + 2]; G.nm[i].pad_ = rgba[4 * i + 3];
  }
  G.roughness = roughness;
  G.is_metal = is_metal;
  G.mip_bias = mip_bias;
  return 0;
}

void ref_set_normal_shadow(void *h, int i) { ((Ctx *)h)->normal_shadow = i; }

void ref_set_view(void *h, const float *pos, const float *vv, float sscale, float cax, float cay) {
  Ctx *c = (Ctx *)h;
  for (int i = 0; i < 3; i++) c->vpos[i] = pos[i];
  for (int i = 0; i < 3; i++) c->vmat[i] = f3(vv + 3 * i);
  c->sscale = sscale; c->cax = cax; c->cay = cay;
}

void ref_set_light(void *h, const float *lint, const float *ldir) {
  Ctx *c = (Ctx *)h;
  c->lint[0] = f3(lint);
  c->ldir[0] = f3(ldir);
}

// clearZBuffer: clearzb.clearFrame over a 2x2 grid of 2x2 work-items (Ops0.py:650-653)
void ref_clear_zbuffer(void *h) {
  Ctx *c = (Ctx *)h;
  const int s = 2, t = 2;
  for (int by = 0; by < s; by++)
    for (int bx = 0; bx < s; bx++)
      for (int ty = 0; ty < t; ty++)
        for (int tx = 0; tx < t; tx++) {
          g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
          ref_clearzb::clearFrame(c->db.data(), c->W, c->H, t, s * t);
        }
}

void ref_set_depth(void *h, const float *db) {
  Ctx *c = (Ctx *)h;
  memcpy(c->db.data(), db, sizeof(float) * c->db.size());
}

// CLDraw.drawAll (Ops0.py:471-648): flags bit 1 = alpha, bit 3 = cull
int ref_draw_all(void *h, const int *flags, const int *alpha_index, const uint8_t *mask, int n, int nthreads) {
  Ctx *c = (Ctx *)h;
  int ng = (int)c->groups.size();
  if (n != ng) return -1;
  c->overflow = 0;
  std::vector<int> gsn(ng, 0);
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    Group &G = c->groups[tn];
    int gs = G.T / BS + 1;
    gsn[tn] = gs;
    bool cull = (flags[tn] & 8) != 0;
    grid1(gs, nthreads, [&](int, int) {
      if (cull)
        ref_trisetup_cull::setup(G.xyz.data(), G.vn.data(), G.tia.data(), G.tib.data(), G.tna.data(),
                                 G.tnb.data(), G.sp.data(), G.zz.data(), c->vpos, c->vmat, c->sscale, c->W,
                                 c->H, c->cax, c->cay, G.T);
      else
        ref_trisetup::setup(G.xyz.data(), G.vn.data(), G.tia.data(), G.tib.data(), G.tna.data(), G.tnb.data(),
                            G.sp.data(), G.zz.data(), c->vpos, c->vmat, c->sscale, c->W, c->H, c->cax, c->cay,
                            G.T);
    });
  }
  // small
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    Group &G = c->groups[tn];
    grid1(gsn[tn], 1, [&](int, int) {
      ref_gather::setup(G.tia.data(), G.tna.data(), G.toa.data(), c->al.data(), tn, gsn[tn]);
    });
  }
  std::vector<int> newSize(c->al.begin(), c->al.end());
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    Group &G = c->groups[tn];
    int ns = newSize[tn] / BS + 1;
    if (newSize[tn] <= 0) continue;
    bool alpha = (flags[tn] & 2) != 0;
    bool multi = !alpha && (flags[tn] & 16) != 0;
    if (multi && tn + 3 >= ng) return -3;
    bool *TA = alpha ? (bool *)c->alphas[alpha_index[tn]].data() : nullptr;
    grid1(ns, nthreads, [&](int, int) {
      if (multi) {
        Multi m = multi_textures(c, tn);
        ref_drawmulti::drawSmall(G.toa.data(), su(c->ro), su(c->go), su(c->bo), c->db.data(), G.sp.data(),
                                 G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), c->lint, c->ldir,
                                 m.t[0][0], m.t[0][1], m.t[0][2], m.len[0], m.t[1][0], m.t[1][1], m.t[1][2], m.len[1],
                                 m.t[2][0], m.t[2][1], m.t[2][2], m.len[2], m.t[3][0], m.t[3][1], m.t[3][2], m.len[3],
                                 c->W, c->H, newSize[tn]);
      } else if (flags[tn] & 32) {   // av_draw_normmap(_alpha, _mip).c
        NormalShadow ns = normal_shadow(c);
        if (alpha)
          ref_draw_nrm_alpha::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(),
                                        G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(),
                                        G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, TA, G.nm.data(),
                                        G.roughness, (char)G.is_metal, c->vpos, c->lint, c->ldir, ns.SD, ns.wS,
                                        ns.scale, ns.SV, ns.SPos, c->W, c->H, newSize[tn]);
        else if (flags[tn] & 1)
          ref_draw_mip::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(), G.sp.data(),
                                  G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), G.tr.data(),
                                  G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(), c->vpos, c->lint, c->ldir,
                                  ns.SD, ns.wS, ns.scale, ns.SV, ns.SPos, G.mip_bias, c->W, c->H, newSize[tn]);
        else
          ref_draw_nrm::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(), G.sp.data(),
                                  G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), G.tr.data(),
                                  G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(), G.roughness, (char)G.is_metal,
                                  c->vpos, c->lint, c->ldir, ns.SD, ns.wS, ns.scale, ns.SV, ns.SPos, c->W, c->H,
                                  newSize[tn]);
      } else if (!alpha && c->mip_kernels && (flags[tn] & 1)) {
        float sd[4] = {0, 0, 0, 0};
        ref_draw_mip::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(), G.sp.data(),
                                G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), G.tr.data(),
                                G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(), c->vpos, c->lint, c->ldir, sd, 1,
                                1.0f, c->vmat, c->vpos, G.mip_bias, c->W, c->H, newSize[tn]);
      } else if (alpha)
        ref_draw_alpha::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(),
                                  G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(),
                                  c->lint, c->ldir, G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, TA, c->W,
                                  c->H, newSize[tn]);
      else
        ref_draw::drawSmall(G.toa.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(), G.sp.data(),
                            G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), c->lint, c->ldir,
                            G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, c->W, c->H, newSize[tn]);
    });
  }
  // large
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    Group &G = c->groups[tn];
    grid1(gsn[tn], 1, [&](int, int) {
      ref_gather::setup(G.tib.data(), G.tnb.data(), G.tob.data(), c->al.data(), tn, gsn[tn]);
    });
  }
  newSize.assign(c->al.begin(), c->al.end());
  for (int tn = 0; tn < ng; tn++) {
    if (mask && mask[tn]) continue;
    Group &G = c->groups[tn];
    if (newSize[tn] <= 0) continue;
    int ns = newSize[tn] / BS + 1;
    grid1(ns, nthreads, [&](int, int) {
      ref_coarse::draw(G.tob.data(), c->ibuf.data(), c->nbuf.data(), G.sp.data(), c->WC, c->HC, newSize[tn]);
    });
    for (int t = 0; t < c->WC * c->HC; t++)
      if (c->nbuf[t] > TILE_BUF) c->overflow = 1;
    if (c->overflow) return -2;  // the reference's bins overflow: result undefined
    bool alpha = (flags[tn] & 2) != 0;
    bool multi = !alpha && (flags[tn] & 16) != 0;
    if (multi && tn + 3 >= ng) return -3;
    bool *TA = alpha ? (bool *)c->alphas[alpha_index[tn]].data() : nullptr;
    int ntiles = c->WC * c->HC;
    auto tile = [&](int bx) {
      bool nrm = !multi && (flags[tn] & 32);
      bool mipk = !alpha && !multi && (flags[tn] & 1) && (c->mip_kernels || nrm);
      float *zb = multi ? ref_drawmulti::local_ZBuf() : (nrm && alpha) ? ref_draw_nrm_alpha::local_ZBuf()
                  : mipk ? ref_draw_mip::local_ZBuf() : nrm ? ref_draw_nrm::local_ZBuf()
                  : alpha ? ref_draw_alpha::local_ZBuf() : ref_draw::local_ZBuf();
      NormalShadow ns = normal_shadow(c);
      int tileX = bx % c->WC, tileY = bx / c->WC;
      for (int r = 0; r < 16; r++)
        for (int i = 0; i < 16; i++) zb[r * 16 + i] = c->db[(size_t)c->W * (tileY * 16 + r) + tileX * 16 + i];
      int nb = c->nbuf[bx];
      g_group[0] = bx; g_group[1] = 0;
      for (int tx = 0; tx < BS; tx++) {
        c->nbuf[bx] = nb;
        g_local[0] = tx; g_local[1] = 0;
        if (multi) {
          Multi m = multi_textures(c, tn);
          ref_drawmulti::draw(c->ibuf.data(), c->nbuf.data(), su(c->ro), su(c->go), su(c->bo), c->db.data(),
                              G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), c->lint,
                              c->ldir, m.t[0][0], m.t[0][1], m.t[0][2], m.len[0], m.t[1][0], m.t[1][1], m.t[1][2],
                              m.len[1], m.t[2][0], m.t[2][1], m.t[2][2], m.len[2], m.t[3][0], m.t[3][1], m.t[3][2],
                              m.len[3], c->W, c->H);
        } else if (nrm && alpha) {
          ref_draw_nrm_alpha::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(),
                                   c->db.data(), G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(),
                                   G.xyz.data(), G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, TA, G.nm.data(),
                                   G.roughness, (char)G.is_metal, c->vpos, c->lint, c->ldir, ns.SD, ns.wS, ns.scale,
                                   ns.SV, ns.SPos, c->W, c->H);
        } else if (mipk && nrm) {
          ref_draw_mip::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(),
                             c->db.data(), G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(),
                             G.xyz.data(), G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(), c->vpos,
                             c->lint, c->ldir, ns.SD, ns.wS, ns.scale, ns.SV, ns.SPos, G.mip_bias, c->W, c->H);
        } else if (nrm) {
          ref_draw_nrm::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(),
                             c->db.data(), G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(),
                             G.xyz.data(), G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(),
                             G.roughness, (char)G.is_metal, c->vpos, c->lint, c->ldir, ns.SD, ns.wS, ns.scale,
                             ns.SV, ns.SPos, c->W, c->H);
        } else if (mipk) {
          float sd[4] = {0, 0, 0, 0};
          ref_draw_mip::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(),
                             c->db.data(), G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(),
                             G.xyz.data(), G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, G.nm.data(), c->vpos,
                             c->lint, c->ldir, sd, 1, 1.0f, c->vmat, c->vpos, G.mip_bias, c->W, c->H);
        } else if (alpha)
          ref_draw_alpha::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(),
                               c->db.data(), G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(),
                               G.xyz.data(), c->lint, c->ldir, G.tr.data(), G.tg.data(), G.tb.data(),
                               G.tex_size, TA, c->W, c->H);
        else
          ref_draw::draw(c->ibuf.data(), c->nbuf.data(), c->ro.data(), c->go.data(), c->bo.data(), c->db.data(),
                         G.sp.data(), G.zz.data(), G.uv.data(), G.li.data(), G.vn.data(), G.xyz.data(), c->lint,
                         c->ldir, G.tr.data(), G.tg.data(), G.tb.data(), G.tex_size, c->W, c->H);
      }
      c->nbuf[bx] = 0;  // what work-item 0 leaves behind (Templates.py:188)
    };
    if (nthreads <= 1) {
      for (int bx = 0; bx < ntiles; bx++) tile(bx);
    } else {
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
      for (int bx = 0; bx < ntiles; bx++) tile(bx);
    }
  }
  return 0;
}

void ref_get_frame(void *h, uint16_t *r, uint16_t *g, uint16_t *b, float *db) {
  Ctx *c = (Ctx *)h;
  size_t n = (size_t)c->W * c->H;
  memcpy(r, c->ro.data(), n * 2); memcpy(g, c->go.data(), n * 2); memcpy(b, c->bo.data(), n * 2);
  memcpy(db, c->db.data(), n * 4);
}

void ref_set_frame(void *h, const uint16_t *r, const uint16_t *g, const uint16_t *b) {
  Ctx *c = (Ctx *)h;
  size_t n = (size_t)c->W * c->H;
  memcpy(c->ro.data(), r, n * 2); memcpy(c->go.data(), g, n * 2); memcpy(c->bo.data(), b, n * 2);
}

// addShadowMap / placeShadowMap / clearShadowMap (Ops.py:1031-1087)
int ref_add_shadow_map(void *h, int i, int size, float scale) {
  Ctx *c = (Ctx *)h;
  if (i < 0 || i >= 8) return -1;
  Shadow &s = c->shadows[i];
  s.map.assign((size_t)size * size, 65535.f);
  s.dim = size; s.scale = scale;
  return 0;
}

void ref_place_shadow_map(void *h, int i, const float *pos, const float *vv) {
  Ctx *c = (Ctx *)h;
  Shadow &s = c->shadows[i];
  for (int k = 0; k < 3; k++) s.pos[k] = pos[k];
  for (int k = 0; k < 3; k++) s.vec[k] = f3(vv + 3 * k);
}

void ref_clear_shadow_map(void *h, int i) {
  Ctx *c = (Ctx *)h;
  Shadow &s = c->shadows[i];
  const int sg = 4, t = 4;
  for (int by = 0; by < sg; by++)
    for (int bx = 0; bx < sg; bx++)
      for (int ty = 0; ty < t; ty++)
        for (int tx = 0; tx < t; tx++) {
          g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
          ref_clearzb::clearFrame(s.map.data(), s.dim, s.dim, t, sg * t);
        }
}

// CLDraw.shadowMap (Ops.py:1089-1141)
int ref_shadow_map(void *h, int i, const uint8_t *cast, const int *flags, const int *alpha_index, int n,
                   float bias, int nthreads) {
  Ctx *c = (Ctx *)h;
  Shadow &s = c->shadows[i];
  int ng = (int)c->groups.size();
  if (n != ng) return -1;
  std::vector<int> tsn, gsn;
  for (int tn = 0; tn < ng; tn++) {
    if (!cast[tn]) continue;
    Group &G = c->groups[tn];
    int gs = G.T / BS + 1;
    tsn.push_back(tn); gsn.push_back(gs);
    grid1(gs, nthreads, [&](int, int) {
      ref_trisetup_ortho::setup(G.xyz.data(), G.tia.data(), G.tna.data(), (int2 *)G.sp.data(), G.zz.data(),
                                s.pos, s.vec, bias, s.scale, s.dim, s.dim, c->cax, c->cay, G.T);
    });
  }
  for (size_t k = 0; k < tsn.size(); k++) {
    Group &G = c->groups[tsn[k]];
    int gs = gsn[k];
    int tn = tsn[k];
    grid1(gs, 1, [&](int, int) { ref_gather::setup(G.tia.data(), G.tna.data(), G.toa.data(), c->al.data(), tn, gs); });
  }
  std::vector<int> newSize(c->al.begin(), c->al.end());
  for (size_t k = 0; k < tsn.size(); k++) {
    int tn = tsn[k];
    Group &G = c->groups[tn];
    if (newSize[tn] <= 0) continue;
    int ns = newSize[tn] / BS + 1;
    bool alpha = (flags[tn] & 2) != 0;
    grid1(ns, nthreads, [&](int, int) {
      if (!alpha)
        ref_drawmin::draw(G.toa.data(), s.map.data(), (int2 *)G.sp.data(), G.zz.data(), s.dim, s.dim, newSize[tn]);
      else
        ref_drawmin_alpha::draw(G.toa.data(), s.map.data(), (int2 *)G.sp.data(), G.zz.data(), G.uv.data(),
                                (bool *)c->alphas[alpha_index[tn]].data(), c->alpha_len[alpha_index[tn]], s.dim,
                                s.dim, newSize[tn]);
    });
  }
  return 0;
}

void ref_get_shadow_map(void *h, int i, float *out) {
  Ctx *c = (Ctx *)h;
  memcpy(out, c->shadows[i].map.data(), sizeof(float) * c->shadows[i].map.size());
}

// CLDraw.gamma (Ops0.py:654-660): 4x4 groups of 4x4 items
void ref_gamma(void *h, float ex) {
  Ctx *c = (Ctx *)h;
  const int s = 4, t = 4;
  int stepH = (c->H + s * t - 1) / (s * t);
  for (int by = 0; by < s; by++)
    for (int bx = 0; bx < s; bx++)
      for (int ty = 0; ty < t; ty++)
        for (int tx = 0; tx < t; tx++) {
          g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
          ref_gamma::g(c->ro.data(), c->go.data(), c->bo.data(), ex, c->W, c->H, t, s * t, stepH);
        }
}

int ref_overflow(void *h) { return ((Ctx *)h)->overflow; }

// CLDraw.rotate (Ops.py:481-497): vert.transform over vertices [start, end)
// of group g, with OldR = oldRM and RR = rotMat transposed.
int ref_transform(void *h, int g, const float *old_rm, const float *rot_mat, const float *origin, int start, int end) {
  Ctx *c = (Ctx *)h;
  if (g < 0 || g >= (int)c->groups.size()) return -1;
  Group &G = c->groups[g];
  if (start < 0 || end < start || end > G.V) return -1;
  float3 oldr[3], rr[3];
  for (int i = 0; i < 3; i++) {
    oldr[i] = f3(old_rm + 3 * i);
    rr[i] = make_float3(rot_mat[i], rot_mat[3 + i], rot_mat[6 + i]);
  }
  float o[3] = {origin[0], origin[1], origin[2]};
  grid1_global((end - start) / BS + 1, [&] {
    ref_vert::transform(G.xyz.data(), G.vn.data(), oldr, rr, o, start, end);
  });
  return 0;
}

// CLDraw.translate (Ops.py:499-508): vert.Ttranslate over [start, end)
int ref_translate(void *h, int g, const float *coords, int start, int end) {
  Ctx *c = (Ctx *)h;
  if (g < 0 || g >= (int)c->groups.size()) return -1;
  Group &G = c->groups[g];
  if (start < 0 || end < start || end > G.V) return -1;
  float o[3] = {coords[0], coords[1], coords[2]};
  grid1_global((end - start) / BS + 1, [&] { ref_vert::Ttranslate(G.xyz.data(), o, start, end); });
  return 0;
}

// CLDraw.vertLight (Ops.py:552-612): vert.vertL over every masked group
int ref_vert_light(void *h, const uint8_t *mask, int n, const float *dir_int, const float *dir_dir, int nd,
                   const float *pint, const float *ppos, int np, const float *sint, const float *sdir,
                   const float *spos, int ns, float amb) {
  Ctx *c = (Ctx *)h;
  if (n != (int)c->groups.size()) return -1;
  std::vector<float3> di = f3s(dir_int, nd), dd = f3s(dir_dir, nd), pi = f3s(pint, np), pp = f3s(ppos, np),
                      si = f3s(sint, ns), sd = f3s(sdir, ns), sp = f3s(spos, ns);
  for (int g = 0; g < n; g++) {
    if (!mask[g]) continue;
    Group &G = c->groups[g];
    int lenV = G.V;
    grid1(lenV / BS + 1, 1, [&](int, int) {
      ref_vert::vertL(G.xyz.data(), G.vn.data(), G.li.data(), di.data(), dd.data(), pi.data(), pp.data(), si.data(),
                      sd.data(), sp.data(), amb, (char)nd, (short)np, ns, lenV);
    });
  }
  return 0;
}

// the vertex buffers of group g, packed as 3 floats per vertex
int ref_get_geometry(void *h, int g, float *xyz, float *vn, float *li) {
  Ctx *c = (Ctx *)h;
  if (g < 0 || g >= (int)c->groups.size()) return -1;
  const Group &G = c->groups[g];
  for (int v = 0; v < G.V; v++) {
    const float3 *src[3] = {&G.xyz[v], &G.vn[v], &G.li[v]};
    float *dst[3] = {xyz, vn, li};
    for (int k = 0; k < 3; k++)
      if (dst[k]) {
        dst[k][3 * (size_t)v] = src[k]->x;
        dst[k][3 * (size_t)v + 1] = src[k]->y;
        dst[k][3 * (size_t)v + 2] = src[k]->z;
      }
  }
  return 0;
}

// CLDraw.ssao (Ops.py:973-983): (H/16) x (W/16) work-groups of 16 x 16 over
// the frame in place.  The kernel reads the depth one row past the buffer on
// the last row when H is a multiple of 16; that row holds 65535 here.
void ref_ssao(void *h, const float *rnd) {
  Ctx *c = (Ctx *)h;
  std::vector<float> F(c->db);
  F.resize((size_t)c->W * (c->H + 1), 65535.f);
  std::vector<float> R(rnd, rnd + 48);
  const int s = 16;
  for (int bx = 0; bx < c->H / s; bx++)
    for (int by = 0; by < c->W / s; by++)
      for (int tx = 0; tx < s; tx++)
        for (int ty = 0; ty < s; ty++) {
          g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
          ref_ssao::ao(c->ro.data(), c->go.data(), c->bo.data(), F.data(), c->sscale, R.data(), c->W, c->H, s);
        }
}

// CLDraw.dof (Ops.py:985-995): the gather into SSRO/SSGO/SSBO, then copied
// back to the frame
void ref_dof(void *h, float focus) {
  Ctx *c = (Ctx *)h;
  std::vector<ushort> r2(c->ro), g2(c->go), b2(c->bo);
  const int s = 16;
  for (int bx = 0; bx < c->H / s; bx++)
    for (int by = 0; by < c->W / s; by++)
      for (int tx = 0; tx < s; tx++)
        for (int ty = 0; ty < s; ty++) {
          g_group[0] = bx; g_group[1] = by; g_local[0] = tx; g_local[1] = ty;
          ref_dof::dof(c->ro.data(), c->go.data(), c->bo.data(), r2.data(), g2.data(), b2.data(), c->db.data(),
                       focus, c->W, c->H, s);
        }
  c->ro = r2; c->go = g2; c->bo = b2;
}

// CLDraw.blur (Ops.py:1009-1020): blurH then blurV, 4 x 4 work-groups of
// 4 x 4, stepW 16, stepH ceil(H/16); each launch runs one thread per
// work-item so that its barrier orders the whole launch.  The half-size
// buffers start at 0 and carry 8 zero rows past their end (blurV reads
// that far below its last row).
void ref_bloom(void *h) {
  Ctx *c = (Ctx *)h;
  size_t hn = (size_t)(c->W / 2) * (c->H / 2 + 8);
  std::vector<ushort> r2(hn, 0), g2(hn, 0), b2(hn, 0), r3(hn, 0), g3(hn, 0), b3(hn, 0);
  const int s = 4, t = 4;
  float stepH = ceilf((float)c->H / (float)(s * t));
  launch_threads(s, s, t, t, [&] {
    ref_blur::blurH(c->ro.data(), c->go.data(), c->bo.data(), r2.data(), g2.data(), b2.data(), r3.data(), g3.data(),
                    b3.data(), c->W, c->H, t, s * t, stepH);
  });
  launch_threads(s, s, t, t, [&] {
    ref_blur2::blurV(r2.data(), g2.data(), b2.data(), r3.data(), g3.data(), b3.data(), c->ro.data(), c->go.data(),
                     c->bo.data(), c->W, c->H, t, s * t, stepH);
  });
}

}  // extern "C"
