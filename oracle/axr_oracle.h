/*
 * axr_oracle.h -- CPU oracle for the AXI Visualizer rasterizer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py call it.  The
 * product path (axi_visualizer_b200 + libaxr.so) never links or calls it.
 *
 * It restates, in plain C with IEEE single-precision arithmetic and no FMA
 * contraction, the reference's OpenCL kernels for the path:
 *   PyOpenCL27C/Pipe/trisetup.c, trisetup_cull.c, trisetupOrtho.c, coarse.c,
 *   PyOpenCL27C/Shaders_src/Templates.py (tiled `draw` and direct `drawSmall`),
 *   PyOpenCL27C/Shaders_src/av_draw_base.c, av_draw_alpha.c,
 *   av_draw_normmap_mip.c (mip selection + trilinear), av_alpha_max.c
 *   (double-cascade 5-tap shadow), PyOpenCL27C/Shaders/drawmin.c,
 *   drawminalpha.c, clearzb.c, Post/gamma.c
 * and the host orchestration of PyOpenCL27C/Ops0.py:471-648 (drawAll) and
 * PyOpenCL27C/Ops.py:1089-1141 (shadowMap).
 *
 * Serial semantics (the reference's GPU kernels race; this is the canonical
 * order that a work-item-serial OpenCL runtime gives, with each tile's local
 * depth copy loaded before its first triangle):
 *   small pass (materials in order, triangles in index order, bottom half
 *   then top half) and then, per material, the large pass (tile bins filled
 *   by the coarse binner in triangle order).  A fragment that passes
 *   `depth >= tz` overwrites depth and colour, so ties go to the later one.
 * Bins are unbounded (the reference's 128-entry bins overflow silently).
 *
 * Parity of this restatement is pinned against the reference's own OpenCL C
 * kernels compiled for the CPU (oracle/build_ref.py -> oracle/_ref) on seeded
 * scenes, and against golden fixtures generated from them (tests/golden).
 */
#ifndef AXR_ORACLE_H
#define AXR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* material flags, parsed from the reference's material strings
 * (PyOpenCL27C/VertObjects.py:142-151, Ops.py:737-740,772-805) */
#define ORC_MIP    1
#define ORC_ALPHA  2
#define ORC_SHADOW 4
#define ORC_CULL   8
#define ORC_MULTI 16   /* av_draw_multi.c: blend with the next three groups' textures */
#define ORC_NORMAL 32  /* av_draw_normmap.c (+ _alpha.c with ORC_ALPHA, _mip.c with ORC_MIP) */

typedef struct orc_group {
  int ntris;
  const float *xyz;  /* [ntris*3][3] vertex positions            */
  const float *vn;   /* [ntris*3][3] vertex normals              */
  const float *uv;   /* [ntris*3][2] texture coordinates         */
  const float *li;   /* [ntris*3][3] per-vertex light `I`        */
  const uint16_t *tr, *tg, *tb; /* texture planes; mip chains smallest level first */
  int tex_size;      /* lenT (texels per side), or numMip = log2(side) for mip */
  int flags;         /* ORC_* */
  int alpha_index;   /* which alpha mask the alpha test samples */
  float mip_bias;
  /* normal-mapped materials: RGBA normal map with one texel per texel of the
   * texture (or chain), roughness (the "normal" pair's second value), metal */
  const uint8_t *nm;
  float roughness;
  int is_metal;
} orc_group;

typedef struct orc_alpha {
  const uint8_t *mask; /* [len*len] booleans */
  int len;
} orc_alpha;

typedef struct orc_shadow {
  float *map;        /* [dim*dim] f32 depth */
  int dim;
  float scale;
  float pos[3];
  float vv[9];       /* rows: depth axis, x axis, y axis (Utils.viewMat) */
} orc_shadow;

typedef struct orc_frame {
  int w, h;
  float pos[3];
  float vv[9];       /* rows: view vector, horizontal, vertical */
  float sscale, cax, cay;
  float lint[3], ldir[3];
  float amb;         /* ambLight (shadowed fraction) */
  uint16_t *ro, *go, *bo;
  float *db;
  int32_t *tri_id;   /* [h*w] global triangle id of the visible fragment, -1 none */
  uint8_t *cov;      /* [h*w] 1 where this drawAll wrote a fragment */
} orc_frame;

/* One CLDraw.drawAll: mask[g] != 0 skips group g (Ops0.py:482-485).
 * shadows[0..nshadow) are the cascades the `shadow` materials sample
 * (drawAll's shadowIds); the normal-mapped materials sample shadows[0].
 * nthreads > 1 runs the OpenMP build (same result). */
int orc_draw_all(orc_frame *f, const orc_group *g, int ng, const uint8_t *mask,
                 const orc_alpha *alphas, int nalpha,
                 const orc_shadow *shadows, int nshadow, int nthreads);

/* One CLDraw.shadowMap: cast[g] != 0 selects casters; alpha materials use the
 * alpha-tested depth kernel (Ops.py:1089-1141). */
int orc_shadow_map(orc_shadow *s, const orc_group *g, int ng, const uint8_t *cast,
                   const orc_alpha *alphas, int nalpha, float bias, int nthreads);

/* clearzb.c: fills the [0, w/lenP*lenP) x [0, h/lenP*lenP) region with 65535 */
void orc_clear_depth(float *f, int w, int h, int lenP);

/* Post/gamma.c on the three u16 planes, in place */
void orc_gamma(uint16_t *r, uint16_t *g, uint16_t *b, int w, int h, float exposure);

/* Exposes the per-triangle setup (trisetup.c / trisetup_cull.c) for tests:
 * cls[t] = 0 rejected, 1 small, 2 large; sp [ntris*3][2]; zz [ntris*3]. */
void orc_setup_persp(const orc_group *g, const orc_frame *f, uint8_t *cls,
                     float *sp, float *zz);

/* coarse.c: number of (triangle, tile) bin entries the large triangles of
 * group g produce, and the per-tile counts (tile_counts [W/16*H/16]). */
long orc_coarse_counts(const orc_group *g, const orc_frame *f, int32_t *tile_counts);

/* Correctly rounded log2 used by the mip selection, exposed for tests. */
float orc_log2f(float x);

/* Post/ssao.c in place on the colour planes: 16 depth samples per pixel of
 * the w/16*16 x h/16*16 region around its reconstructed position, from the
 * random table rnd[32]; a depth read one row past the buffer (the last row
 * when h is a multiple of 16) reads 65535. */
void orc_ssao(uint16_t *r, uint16_t *g, uint16_t *b, const float *db, int w, int h, float sscale,
              const float *rnd);

/* Post/dof.c: depth-of-field gather of the w/16*16 x h/16*16 region into
 * (r2, g2, b2) (the reference writes SSRO/SSGO/SSBO and copies them back). */
void orc_dof(const uint16_t *r, const uint16_t *g, const uint16_t *b, const float *db, int w, int h,
             float focus, uint16_t *r2, uint16_t *g2, uint16_t *b2);

/* Post/blur.c + Post/blur2.c (CLDraw.blur, Ops.py:1009-1020): the bloom,
 * in place on the colour planes.  Each kernel's phases run one after the
 * other over the whole image (the reference's barrier orders only one
 * work-group; the intended order is the global one).  Half-resolution rows
 * that no phase writes, and the rows the vertical blur reads past its
 * buffer, read 0. */
void orc_bloom(uint16_t *r, uint16_t *g, uint16_t *b, int w, int h);

/* Vertex stage (Pipe/vert.c) on packed vertex arrays (3 floats a vertex).
 * orc_transform: vertices [start, end) move to rot^T-rows . (old . (p - o)) + o
 * and their normals to rot^T-rows . (old . n) (CLDraw.rotate).
 * orc_translate: vertices [start, end) move by c (CLDraw.translate).
 * orc_vert_light: li of nv vertices from directional lights 1..nd-1, np point
 * and ns spot lights, floored at amb (CLDraw.vertLight). */
void orc_transform(float *xyz, float *vn, const float old_rm[9], const float rot_mat[9],
                   const float origin[3], int start, int end);
void orc_translate(float *xyz, const float c[3], int start, int end);
void orc_vert_light(const float *xyz, const float *vn, float *li, int nv,
                    const float *dir_int, const float *dir_dir, int nd,
                    const float *pint, const float *ppos, int np,
                    const float *sint, const float *sdir, const float *spos, int ns, float amb);

#ifdef __cplusplus
}
#endif
#endif
