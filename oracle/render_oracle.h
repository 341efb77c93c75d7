/*
 * CPU oracle of the headless frame (aq_renderer_draw) — TEST INFRASTRUCTURE
 * ONLY.  The library never links, loads or calls it.
 *
 * A plain-C restatement of one frame of the reference's renderer, drawn the
 * way GL draws it: primitive by primitive in submission order, each fragment
 * depth-tested and blended into the framebuffer as it arrives (main.cu:111-145,
 * Fluid/Fluid_3D_FLIP.cu:396-430, the .cu files of Rendering/Renderer3D and the shaders
 * under resources/Shaders/).  The CUDA frame instead walks per-tile lists of
 * primitives pixel by pixel; both follow the same fixed-function rules
 * (render_oracle.c, top comment), so their images agree byte for byte except
 * where expf differs between the two math libraries.
 *
 * The shading functions are pinned against the reference's own GLSL, compiled
 * as C++ against the reference's vendored glm (oracle/shade_harness.cpp),
 * through tests/golden/ref_shade.npz.  The fixed-function stages have no
 * reference source (the GL driver does them): those are unpinned.
 */
#ifndef AQ_RENDER_ORACLE_H
#define AQ_RENDER_ORACLE_H

#include <stdint.h>

#include "../include/aquarius_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One frame into rgba (W*H*4 bytes, row 0 at the bottom).  phase (may be
 * NULL) receives the phase-thickness texture (W*H*4 floats).  sky: six
 * face*face RGB8 faces (posx, negx, posy, negy, posz, negz) or NULL; logo:
 * lw*lh RGB8 or NULL.  Returns 0, or -1 on a bad argument. */
int orc_render_frame(const aq_draw_command* dc, const float* points, int32_t n_points, const float* mesh,
                     int64_t n_vertices, const uint8_t* sky, int32_t face, const uint8_t* logo, int32_t lw,
                     int32_t lh, uint8_t* rgba, float* phase);

/* rayTraceEnvironment (resources/Shaders/RayTraceEnvironment.glsl:117-178). */
void orc_trace_environment(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo,
                           int32_t lw, int32_t lh, const float origin[3], const float dir[3], float out[4]);

/* FluidMeshRenderer_fs.glsl main() for one fragment with the given varyings
 * and phase-thickness texel (the value texture() returns, before * 0.1). */
void orc_shade_mesh(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo,
                    int32_t lw, int32_t lh, const float frag_pos[3], const float frag_normal[3],
                    const float texel[4], float out[4]);

/* The texture samplers: cube map (linear, clamp to edge) and 2D (linear,
 * clamp to edge); RGB in out[0..2], out[3] = 1. */
void orc_sample_cube(const uint8_t* sky, int32_t face, const float dir[3], float out[4]);
void orc_sample_2d(const uint8_t* img, int32_t w, int32_t h, float s, float t, float out[4]);

/* aq_draw_command_default restated (camera.h + glm::lookAt/perspective in
 * float, as glm computes them). */
void orc_draw_command_default(aq_draw_command* dc, int32_t width, int32_t height, float domain_size,
                              int32_t size_y);

#ifdef __cplusplus
}
#endif

#endif /* AQ_RENDER_ORACLE_H */
