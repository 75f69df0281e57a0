/*
 * axr.h -- C ABI of libaxr.so, the B200 (sm_100a) implementation of the
 * AXI Visualizer rasterizer hot path: tiled scanline rasterization with
 * depth test, perspective-correct textured shading (bilinear / trilinear
 * mip, alpha test, double-cascade shadow lookup) and the shadow-map depth
 * pass.
 *
 * The entry points replace the methods of the reference's draw runtime,
 * class CLDraw in PyOpenCL27C/Ops.py (and Ops0.py), which the engine holds
 * as ThreeDBackend.draw (PyOpenCL27C/Compute.py:182-187).  Each declaration
 * cites the method it stands in for.  Plain pointers and sizes only; host
 * pointers are borrowed for the duration of the call.
 *
 * Errors: every function returns 0 on success and a negative AXR_E* code on
 * failure; axr_last_error() gives a message for the calling thread.  A
 * handle is not thread-safe; separate handles may be used from separate
 * threads.  All work of one handle runs in order on its own CUDA stream.
 */
#ifndef AXR_H
#define AXR_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AXR_OK 0
#define AXR_EINVAL -1   /* bad argument */
#define AXR_ECUDA -2    /* CUDA runtime error */
#define AXR_ENOMEM -3   /* device allocation failed */
#define AXR_EOVERFLOW -4 /* a work queue overflowed; the call was not completed */
#define AXR_ESTATE -5   /* call out of order (e.g. shading with no shadow map) */

/* material flags: the substrings CLDraw.drawAll tests in the material
 * strings (Ops.py:737-740,772-805; VertObjects.py:142-151) */
#define AXR_MIP 1     /* "mip": trilinear mip chain, tex_size = log2(side) */
#define AXR_ALPHA 2   /* "alpha": bilinear boolean alpha test before depth */
#define AXR_SHADOW 4  /* "shadow": double-cascade 5-tap shadow lookup */
#define AXR_CULL 8    /* "cull": back-face rejection (trisetup_cull.c:49-54) */
#define AXR_MULTI 16  /* "multi": 4-way blend with the next three groups' textures
                         (av_draw_multi.c; Ops0.py:533-545); needs a single-level
                         texture and groups g+1..g+3 with >= side^2 texels; no mip or
                         shadow lookup; ignored on AXR_ALPHA groups */

typedef struct axr_ctx axr_ctx;

/* Message of the last failed call on this thread ("" if none). */
const char *axr_last_error(void);

/* CLDraw.__init__(size_sky, max_uv, w, h, max_particles) (Ops.py:127-229):
 * framebuffers of w x h (w a multiple of 16; the tile grid is w/16 x h/16,
 * Ops.py:131-132) on CUDA device `device`. */
int axr_create(int w, int h, int device, axr_ctx **out);

/* Releases every device buffer of the handle (the reference never frees). */
int axr_destroy(axr_ctx *ctx);

/* CLDraw.setScaleCull(s, cx, cy) (Ops.py:231-233) */
int axr_set_scale_cull(axr_ctx *ctx, float sscale, float cax, float cay);

/* CLDraw.addTextureGroup(xyz, uv, vn, r, g, b, mip) (Ops.py:331-378):
 * ntris triangles as 3*ntris vertices: xyz [3*ntris][3], uv [3*ntris][2],
 * vn [3*ntris][3]; texture planes r, g, b of `ntexels` uint16 each (one
 * side*side level, or the full mip chain smallest level first when
 * mip_side > 0, Utils.createMips).  tex_size is the reference's texSize:
 * side, or log2(side) for mip.  Returns the group id in *out_id.  A group
 * holds at most 715,827,881 triangles, so that its vertex indices fit the
 * int vertex ranges of axr_transform / axr_translate / axr_vert_light; a
 * handle holds fewer than 2^30 - 1 in all. */
int axr_add_texture_group(axr_ctx *ctx, const float *xyz, const float *uv, const float *vn, int ntris,
                          const uint16_t *r, const uint16_t *g, const uint16_t *b, long ntexels,
                          int mip_side, int *out_id);

/* Per-vertex light `I` of a group ([3*ntris][3]); CLDraw.vertLight fills the
 * same LI buffer on the device (Ops.py:552-612, vert.c:38-87).  Groups start
 * with I = 0. */
int axr_set_vert_light(axr_ctx *ctx, int group, const float *li);

/* CLDraw.vertLight(mask, dirI, dirD, pointI, pointP, spotI, spotD, spotP)
 * (Ops.py:552-612, vert.c:38-88): for every group whose mask entry is
 * non-zero, on the device,
 *   I = max(sum_{i>=1} max(0, dot(n, dir_i) + 0.5) * 0.66 * dint_i
 *         + sum_points [dot(n, x - p) > 0] dot(n, u) / (1 + |x - p|^2) * pint
 *         + sum_spots [dot(sdir, x - p) > 0 and dot(n, x - p) > 0]
 *               dot(n, u) * dot(u, sdir) / (1.5 + |x - p|^2) * sint,  amb)
 * with u = (x - p) / |x - p| (light 0 is the per-pixel primary light).
 * Light arrays are [count][3]; at most 127 directional and 32767 point
 * lights (the reference passes the counts as char and short).  Queued on
 * the handle's stream; the light arrays are copied before the call returns. */
int axr_vert_light(axr_ctx *ctx, const uint8_t *mask, int ngroups, const float *dir_int, const float *dir_dir,
                   int ndirs, const float *point_int, const float *point_pos, int npoints, const float *spot_int,
                   const float *spot_dir, const float *spot_pos, int nspots, float amb);

/* CLDraw.rotate(oldRM, rotMat, origin, cStart, cEnd, tn) (Ops.py:481-497,
 * vert.c:3-28): vertices [v_start, v_end) of a group (v_end < 0: to the end)
 * move to rotMat^T . (oldRM . (p - origin)) + origin, and their normals to
 * rotMat^T . (oldRM . n).  old_rm and rot_mat are row-major 3x3.  Queued on
 * the handle's stream; shadow passes queued later see the new geometry and
 * shadow passes in flight finish reading the old one first. */
int axr_transform(axr_ctx *ctx, int group, const float *old_rm, const float *rot_mat, const float *origin,
                  int v_start, int v_end);

/* CLDraw.translate(coords, cStart, cEnd, tn) (Ops.py:499-508, vert.c:29-36):
 * vertices [v_start, v_end) of a group move by coords; ordered as
 * axr_transform. */
int axr_translate(axr_ctx *ctx, int group, const float *coords, int v_start, int v_end);

/* The mipBias of a group's trilinear level selection
 * (av_draw_normmap_mip.c:20,43: fmip = clamp(|log2 dt| / 2 + mipBias, 0,
 * numMip - 1)), which the reference passes per draw as the value of a dict
 * material's "mip" entry (Ops.py:687).  It stays with the group for every
 * later drawAll and batch render; 0 until set.  A bias that is not a finite
 * number is refused. */
int axr_set_mip_bias(axr_ctx *ctx, int group, float bias);

/* New: copies a group's vertex arrays to the host ([3*ntris][3] each; any
 * pointer may be NULL) after the work queued before it on the handle's
 * stream.  The reference keeps them in device buffers (Ops.py:618-620). */
int axr_get_vertices(axr_ctx *ctx, int group, float *xyz, float *vn, float *li);

/* CLDraw.copyTo(tn, vp, vn, cstart) (Ops.py:448-452): overwrite vertices
 * [3*tri_start, 3*(tri_start+ntris)) of a group. */
int axr_copy_to(axr_ctx *ctx, int group, const float *xyz, const float *vn, int tri_start, int ntris);

/* CLDraw.addTexAlpha(a) (Ops.py:454-456): boolean alpha mask side x side. */
int axr_add_tex_alpha(axr_ctx *ctx, const uint8_t *mask, int side, int *out_id);

/* CLDraw.addNrmMap(rgb, name) (Ops.py:299-302): a normal map of ntexels
 * texels as RGBA bytes (the reference's align34 layout; A unused), one
 * texel per texel of the textures it is used with (a full chain, smallest
 * level first, for the mip variant).  Returns its id. */
int axr_add_normal_map(axr_ctx *ctx, const uint8_t *rgba, long ntexels, int *out_id);

/* The normal-mapped materials of group `group` (material flag 32, the
 * reference's dict material {"normal": (name, roughness), "metal": ...},
 * Ops.py:669-699, 772-805): its normal map (-1: none), roughness and metal
 * switch.  A drawAll of the material needs a normal map with at least as
 * many texels as the group's texture.  It combines with alpha
 * (av_draw_normmap_alpha.c) or mip (av_draw_normmap_mip.c, whose
 * arguments carry no roughness or metal), not both; its sampleShadow,
 * which the reference defines nowhere, counts the five taps of the draw's
 * first cascade (0.2 each). */
int axr_set_normal_material(axr_ctx *ctx, int group, int map, float roughness, int metal);

/* CLDraw.setPrimaryLight(dirI, dirD) (Ops.py:1143-1151) */
int axr_set_primary_light(axr_ctx *ctx, const float dir_int[3], const float dir_dir[3]);

/* CLDraw.setPos(vc) / setVM(vM) (Ops.py:475-479): camera position and
 * view basis rows [view vector, horizontal, vertical]. */
int axr_set_pos(axr_ctx *ctx, const float pos[3]);
int axr_set_vm(axr_ctx *ctx, const float vm[9]);

/* Asynchronous read-back of the frame (colour planes and/or depth; NULL
 * skips a plane) for frame loops: the frame is copied on the device into one
 * of two staging slots, ordered before the next frame's writes, then to the
 * host on a copy stream while later frames render.  Host buffers should be
 * pinned (pageable ones make the copy synchronous).  *ticket names the read;
 * axr_wait_frame blocks until it is on the host, axr_frame_done polls (1 =
 * done).  A third read waits for the first, whose slot it reuses, so keep
 * at most two reads in flight per set of host buffers.  New (the reference's
 * getFrame is synchronous). */
int axr_read_frame_async(axr_ctx *ctx, uint16_t *r, uint16_t *g, uint16_t *b, float *depth, int64_t *ticket);
int axr_wait_frame(axr_ctx *ctx, int64_t ticket);

/* The same for a display client: the frame mapped by Post/gamma.c's formula
 * with `exposure` (as axr_gamma, but the planes stay unchanged) and packed
 * on the device as interleaved 8-bit RGB into rgb [h][w][3] (3 bytes per
 * pixel instead of 10).  Same ring, tickets and rules as above.  New. */
int axr_read_frame_rgb8_async(axr_ctx *ctx, float exposure, uint8_t *rgb, int64_t *ticket);
int axr_frame_done(axr_ctx *ctx, int64_t ticket);

/* CLDraw.clearZBuffer() (Ops0.py:650-653, clearzb.c): depth := 65535 on the
 * [0, w/4*4) x [0, h/4*4) region the reference's 4x4 work-items cover. */
int axr_clear_zbuffer(axr_ctx *ctx);

/* Colour half of the current reference's clearZBuffer (Ops.py:939-946, which
 * also fills the colour planes with the sky colour): every pixel of the
 * colour planes := (r, g, b), each in [0, 65535]. */
int axr_clear_color(axr_ctx *ctx, int r, int g, int b);

/* CLDraw.drawAll(shaders, mask, shadowIds) (Ops0.py:471-648, Ops.py:716-937):
 * flags[g] (AXR_*), alpha_index[g] (alpha mask of alpha groups; may be
 * NULL = 0), mask[g] != 0 skips group g (may be NULL).  shadow_ids lists
 * the shadow maps (cascades, at most 2) that AXR_SHADOW groups sample. */
int axr_draw_all(axr_ctx *ctx, const int32_t *flags, const int32_t *alpha_index, const uint8_t *mask, int ngroups,
                 const int32_t *shadow_ids, int nshadow);

/* CLDraw.getFrame() (Ops.py:1224-1230): copies the three uint16 colour
 * planes and the float depth ([h][w] each) into host buffers; any pointer
 * may be NULL to skip that plane.  Synchronises the handle's stream. */
int axr_get_frame(axr_ctx *ctx, uint16_t *r, uint16_t *g, uint16_t *b, float *depth);

/* Visibility of the last drawAll (new outputs, not in the reference):
 * tri_id = global triangle id (group base + index) of the visible fragment,
 * -1 where drawAll wrote nothing; coverage = 1 where it wrote.  Either
 * pointer may be NULL. */
int axr_get_ids(axr_ctx *ctx, int32_t *tri_id, uint8_t *coverage);

/* Uploads host depth/colour (tests and resume). Any pointer may be NULL. */
int axr_set_frame(axr_ctx *ctx, const uint16_t *r, const uint16_t *g, const uint16_t *b, const float *depth);

/* CLDraw.gamma(ex) (Ops0.py:654-660, Post/gamma.c) on the colour planes. */
int axr_gamma(axr_ctx *ctx, float exposure);

/* CLDraw.ssao() (Ops.py:973-983, Post/ssao.c): screen-space ambient
 * occlusion in place on the colour planes of the w/16*16 x h/16*16 region,
 * from the depth buffer and a random table (rnd[0..31] are read; the
 * reference draws 48 uniform floats once).  A depth read one row past the
 * buffer (the kernel's neighbour on the last row when h is a multiple of 16)
 * reads 65535.  Queued on the handle's stream. */
int axr_ssao(axr_ctx *ctx, const float *rnd, int n);

/* CLDraw.dof(focus) (Ops.py:985-995, Post/dof.c): depth-of-field gather of
 * the w/16*16 x h/16*16 region (circle of confusion 4|d - focus|/focus/d,
 * at most 4 pixels) replacing its colour; the rows below the region keep
 * their colour.  Queued on the handle's stream. */
int axr_dof(axr_ctx *ctx, float focus);

/* CLDraw.blur() (Ops.py:1009-1020, Post/blur.c + Post/blur2.c): the bloom,
 * in place on the colour planes.  A half-resolution bright pass, a 19-tap
 * horizontal and a 19-tap vertical blur, then the bilinear upsample added
 * to the frame; each pass covers the whole image before the next.  Rows of
 * the half-resolution planes that no pass writes, and the 8 rows the
 * vertical blur reads past them, read 0.  Queued on the handle's stream. */
int axr_bloom(axr_ctx *ctx);

/* CLDraw.addShadowMap(i, size, scale, ambLight) (Ops.py:1048-1070) */
int axr_add_shadow_map(axr_ctx *ctx, int i, int size, float scale, float amb_light);

/* CLDraw.placeShadowMap(i, pos, facing, ambLight) (Ops.py:1078-1087): vm are
 * the rows of Utils.viewMat(*facing). amb_light < 0 keeps the current one. */
int axr_place_shadow_map(axr_ctx *ctx, int i, const float pos[3], const float vm[9], float amb_light);

/* CLDraw.clearShadowMap(i) (Ops.py:1022-1028): 65535 over the 16x16 blocks. */
int axr_clear_shadow_map(axr_ctx *ctx, int i);

/* CLDraw.shadowMap(i, whichCast, shaders, bias) (Ops.py:1089-1141):
 * ortho setup (trisetupOrtho.c) and depth-min raster (drawmin.c, or the
 * alpha-tested drawminalpha.c for AXR_ALPHA groups) of every group with
 * cast[g] != 0. */
int axr_shadow_map(axr_ctx *ctx, int i, const uint8_t *cast, const int32_t *flags, const int32_t *alpha_index,
                   int ngroups, float bias);

/* CLDraw.getSHM(i) (Ops.py:1218-1222): copies the size x size depth map. */
int axr_get_shadow_map(axr_ctx *ctx, int i, float *out);

/* Blocks until all work queued on the handle has finished. */
int axr_sync(axr_ctx *ctx);

/* The handle's CUDA stream (a cudaStream_t), so callers can time or order
 * work against it (e.g. torch.cuda.ExternalStream). */
int axr_get_stream(axr_ctx *ctx, void **stream);

/* Device pointers of the framebuffers ([h][w]; keys are the 64-bit
 * depth/order visibility words of the last drawAll) for zero-copy users. */
int axr_frame_device_ptrs(axr_ctx *ctx, void **r, void **g, void **b, void **depth, void **keys);

/* Launch statistics of the last drawAll: number of kernels launched and
 * work-queue sizes (small triangles, large triangles, tile units). */
int axr_last_stats(axr_ctx *ctx, int64_t *kernels, int64_t *n_small, int64_t *n_large, int64_t *n_units);

/* Work-queue sizes of the last drawAll by kind (new; waits for the
 * handle's work): out[0..n) of, in order, opaque and alpha-tested small
 * triangles, large triangles, and opaque and alpha-tested tile units. */
int axr_last_queues(axr_ctx *ctx, int64_t *out, int n);

/* Number of kernels the handle has launched since axr_create. */
int axr_launch_count(axr_ctx *ctx, int64_t *total);

/* Per-kernel timing (tracing): when enabled, every kernel launch is
 * bracketed by CUDA events on the handle's stream; axr_kernel_times reports,
 * per kernel name, the summed device time (ms) and the launch count since
 * timing was enabled.  names receives up to `max` NUL-terminated names of
 * name_len bytes each. Both calls synchronise the stream. */
int axr_set_kernel_timing(axr_ctx *ctx, int enable);
int axr_kernel_times(axr_ctx *ctx, int max, char *names, int name_len, double *total_ms, int64_t *launches, int *n);

/* ------------------------------------------------------------------------
 * Batched multi-view rendering (no counterpart in the reference, which draws
 * one view per drawAll).  A batch holds views of uneven size over the
 * handle's scene: shaded perspective views (main view, cubemap faces) and
 * depth-only orthographic views (shadow cascades, which the shaded views of
 * the same batch sample).  One render runs every view in one cooperative
 * persistent kernel, replayed from a captured CUDA graph; each view's result
 * is bit-identical to rendering it alone with drawAll/shadowMap.
 * ------------------------------------------------------------------------ */
#define AXR_VIEW_SHADED 0
#define AXR_VIEW_DEPTH 1
#define AXR_VIEW_SKIP 2    /* a shaded view's slot that this render leaves untouched */

typedef struct axr_view_desc {
  int kind;          /* AXR_VIEW_SHADED or AXR_VIEW_DEPTH */
  int w, h;          /* shaded: framebuffer (w a multiple of 16); depth: map side w (h unused) */
  float pos[3];      /* camera position */
  float vm[9];       /* basis rows (view, horizontal, vertical) / Utils.viewMat rows */
  float scale;       /* shaded: sScale; depth: orthographic scale */
  float cax, cay;    /* shaded: cull bounds (setScaleCull) */
  float bias;        /* depth: shBias of shadowMap */
  int cascades[2];   /* shaded: batch indices of the depth views it samples, or -1-i for
                        the handle's shadow map i (rendered by axr_shadow_map) */
  int ncascades;
  int group_first;   /* the view draws groups [group_first, group_first + group_count) */
  int group_count;   /* 0 = every group of the handle.  Triangle ids count from the
                        range's first triangle, so a scene kept as a group range of a
                        shared handle renders exactly as in a handle of its own */
  int clear_color;   /* shaded: 1 = colour planes := bg before drawing (as axr_clear_color)
                        and depth outside the clearzb region := 0 (a new buffer's value),
                        so the result does not depend on what the slot held before */
  int bg[3];
} axr_view_desc;

typedef struct axr_batch axr_batch;

/* Creates a batch of views over the handle's current groups (add groups
 * first).  Allocates the views' framebuffers, maps and work queues. */
int axr_batch_create(axr_ctx *ctx, const axr_view_desc *views, int nviews, axr_batch **out);

/* New cameras (same sizes; a shaded slot may switch between AXR_VIEW_SHADED and
 * AXR_VIEW_SKIP) for the next render. */
int axr_batch_set_views(axr_batch *b, const axr_view_desc *views, int nviews);

/* Renders every view: depth views clear and draw the casters (cast[g] != 0,
 * NULL = all) of their group range, shaded views clear and draw their group
 * range with flags[g] and alpha_index[g] (as axr_draw_all); AXR_VIEW_SKIP
 * slots are left as they are.  Asynchronous on the handle's stream: renders
 * of several batches of one handle queue behind each other on the GPU while
 * the host prepares the next. */
int axr_batch_render(axr_batch *b, const int32_t *flags, const int32_t *alpha_index, const uint8_t *cast,
                     int ngroups);

/* Copies a view's result: colour planes + depth of a shaded view, or the
 * depth map of a depth view (into `depth`).  Synchronises. */
int axr_batch_get_frame(axr_batch *b, int view, uint16_t *r, uint16_t *g, uint16_t *bb, float *depth);

/* Triangle id / coverage of a shaded view of the last render. */
int axr_batch_get_ids(axr_batch *b, int view, int32_t *tri_id, uint8_t *coverage);

/* Queues the copy of a shaded view's colour planes (and depth, if not NULL)
 * of the last render into host memory (pinned for an asynchronous copy) on
 * the batch's copy stream, behind the render; does not block.  The data is
 * there once axr_batch_query returns 1. */
int axr_batch_read_async(axr_batch *b, int view, uint16_t *r, uint16_t *g, uint16_t *bb, float *depth);

/* 1 if the last render and the reads queued after it have finished and the
 * render's work counters were checked, 0 if still running (does not block),
 * negative on an error of that render. */
int axr_batch_query(axr_batch *b);

/* Durations in ms of the five phases of the last render (clear, setup,
 * coarse + small triangles + depth maps, tiled large triangles, shading), from
 * the GPU's global timer at the grid barriers; waits for the render. */
int axr_batch_phase_times(axr_batch *b, float ms[5]);

/* Device memory held by the batch (framebuffers, maps, work queues, tables). */
int axr_batch_bytes(axr_batch *b, int64_t *bytes);

/* Number of renders, whether renders replay a captured graph (1) or launch
 * directly (0), and the persistent grid size in blocks. */
int axr_batch_stats(axr_batch *b, int64_t *renders, int *graph, int *grid);

/* Tuning knobs (picked by axi_visualizer_b200/autotune.py): persistent grid
 * size in blocks per SM (1..occupancy limit) and the minimum number of rows
 * per small-triangle work item.  Results do not depend on them. */
int axr_batch_set_tuning(axr_batch *b, int blocks_per_sm, int min_chunk);

/* How a render runs: AXR_BATCH_PERSISTENT (default) = one cooperative
 * persistent kernel whose phases are separated by grid barriers (fewest
 * launches: best for many small views); AXR_BATCH_PHASED = the same phases
 * as separate kernels in the captured graph, each at its own occupancy, the
 * alpha-tested rasterizers on a parallel branch (best for heavy views;
 * axr_batch_phase_times then reports zeros).  Results do not depend on it. */
#define AXR_BATCH_PERSISTENT 0
#define AXR_BATCH_PHASED 1
int axr_batch_set_mode(axr_batch *b, int mode);

/* Fault injection for tests of failure detection (persistent form): the next
 * renders' grid barriers wait for phantom_blocks blocks that are never
 * launched, and every waiting block gives up after spin_limit polls (at most
 * the default, about 2^26), so the render ends with the error "batch grid
 * barrier timed out" instead of hanging.  (0, 67108864) restores normal
 * renders.  No GPU fault is involved. */
int axr_batch_inject_barrier_stall(axr_batch *b, int phantom_blocks, long long spin_limit);
int axr_set_tuning(axr_ctx *ctx, int min_chunk);

/* How CLDraw.shadowMap (Ops.py:1089-1141) draws the casters: 0 (the
 * default) = one work item per caster row chunk with global atomics; 2 and 1
 * = for maps of side <= 8192, the tiled pass -- casters binned to 32 x
 * 32-texel tiles, each tile's minimum taken in shared memory, casters, spans
 * and texels that cannot lower the tile skipped before the exact depth --
 * with each tile's units taken front first (2) or as binned (1).  `slice`
 * (32 .. 2^20, 0 keeps the current value, 512 at first) is the number of a
 * tile's units per block: a tile of n units is drawn by ceil(n / slice)
 * blocks.  The maps are identical in every mode. */
int axr_set_shadow_mode(axr_ctx *ctx, int mode, int slice);

/* Queue sizes of shadow map i's passes (new, like axr_last_stats; waits for
 * the handle's work): out[0..n) of, in order, the tiled passes that
 * overflowed their unit queue (each was drawn per caster in the same
 * launches, and the queue grew), the units the last pass needed, the
 * queue's capacity, and the last pass's opaque and alpha-tested casters. */
int axr_shadow_stats(axr_ctx *ctx, int i, int64_t *out, int n);

int axr_batch_destroy(axr_batch *b);

/* Shadow-map depth pass that allocates no device memory.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc/cudaFree
 * while rendering (an engine whose own allocator owns all device memory, or
 * a frame loop that must not take the implicit device synchronisation those
 * calls can cause).  Same arithmetic as axr_shadow_map for one group of
 * casters: ortho setup (trisetupOrtho.c) and depth-min raster (drawmin.c,
 * or drawminalpha.c when alpha_mask is given).
 *
 * All pointers except pos/vm are DEVICE pointers on the current device:
 * xyz [3*ntris][3]; uv [3*ntris][2] and alpha_mask [alpha_side^2] only for
 * alpha-tested casters (else NULL); map [dim][dim] is updated in place (the
 * caller clears it, e.g. to 65535).  Work is queued on `stream` (NULL = the
 * default stream); the call does not synchronise.
 *
 * Limits: at most 1,048,576 triangles per call (larger counts are rejected
 * with AXR_EINVAL); dim in [4, 16384].  Scratch: a fixed 4 MiB array inside
 * the library, held by every GPU that loads it until the process exits.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress); make the first call on each device before any
 * stream capture.  Every call shares the array, so calls that overlap on the
 * GPU (concurrent streams, or several host threads) race and give wrong
 * maps: serialise them.  It returns before the GPU runs, so unlike
 * axr_shadow_map it reports no device-side condition: the raster loops'
 * safety cap (65,536 rounds) cannot trip here, since each caster is one
 * work item of at most dim + 240 rows (16,624 for the largest map). */
int axr_shadow_map_noalloc(const float *xyz, const float *uv, const uint8_t *alpha_mask, int alpha_side, int ntris,
                           const float pos[3], const float vm[9], float scale, float bias, float *map, int dim,
                           void *stream);

#ifdef __cplusplus
}
#endif
#endif
