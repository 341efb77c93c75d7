// The reference's fragment shaders compiled as C++ — TEST INFRASTRUCTURE
// ONLY (the shading pin of the headless frame).
//
// resources/Shaders/RayTraceEnvironment.glsl, FluidMeshRenderer_fs.glsl and
// Container_face_fs.glsl, translated mechanically by glsl_to_cpp.py into
// oracle/_ref/shade/*.inc at build time (oracle/Makefile target ``shade``)
// and compiled against glsl_shim.hpp.  Each entry point sets the shader's
// uniforms and varyings the way FluidMeshRenderer::draw / Container::drawFace
// do (Rendering/Renderer3D/FluidMeshRenderer.cu:56-126, Container.cu:71-120,
// Rendering/Shader.cpp:130-152) and runs the shader's main() or
// rayTraceEnvironment().  tests/golden/make_golden.py records their outputs
// as fixtures for the oracle's shading functions.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <iostream>

#include "../include/aquarius_b200.h"
#include "glsl_shim.hpp"

// The reference's Camera (Rendering/Renderer3D/camera.h) on its vendored glm;
// its own includes are made here first so that they stay global.
#include <vector>

#include <GL/glew.h>
#include <glm/glm.hpp>
#include <glm/gtc/matrix_transform.hpp>

namespace refcam {
using std::max;
using std::min;
#include "camera.h"
}  // namespace refcam

namespace fmr {
using namespace glsl_shim;
#define main shader_main
#include "RayTraceEnvironment.inc"
#include "FluidMeshRenderer_fs.inc"
#undef main
}  // namespace fmr

namespace cface {
using namespace glsl_shim;
#define main shader_main
#include "RayTraceEnvironment.inc"
#include "Container_face_fs.inc"
#undef main
}  // namespace cface

namespace {

glsl_shim::vec3 v3(const float* p) { return glsl_shim::vec3(p[0], p[1], p[2]); }

void out4(const glsl_shim::vec4& c, float* o) {
  o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
}

}  // namespace

extern "C" {

// main.cu:115-133 on the first frame: Camera(fluid->getCenter()),
// camera->getViewMatrix(), glm::perspective(camera->FOV, w/h, 0.1, 1000),
// camera->getActualPosition().
void aqshade_camera(int32_t width, int32_t height, float domain_size, float view[16], float projection[16],
                    float eye[3]) {
  std::streambuf* old = std::cout.rdbuf(nullptr);  // the constructor prints its vectors
  const float c = domain_size / 2;
  refcam::Camera cam(glm::vec3(c, c, c));
  std::cout.rdbuf(old);
  const glm::mat4 v = cam.getViewMatrix();
  const float ratio = (float)width / (float)height;
  const glm::mat4 p = glm::perspective(cam.FOV, ratio, 0.1f, 1000.0f);
  std::memcpy(view, &v[0][0], 16 * sizeof(float));
  std::memcpy(projection, &p[0][0], 16 * sizeof(float));
  const glm::vec3 e = cam.getActualPosition();
  eye[0] = e.x; eye[1] = e.y; eye[2] = e.z;
}

void aqshade_trace(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo, int32_t lw,
                   int32_t lh, const float origin[3], const float dir[3], float out[4]) {
  glsl_shim::samplerCube s;
  s.faces = sky;
  s.face = face;
  glsl_shim::sampler2D l;
  l.img = logo;
  l.w = lw;
  l.h = lh;
  out4(fmr::rayTraceEnvironment(v3(origin), v3(dir), dc->environment_mode, dc->cornell_box_size, dc->container_size,
                                v3(dc->light_position), s, l),
       out);
}

void aqshade_mesh(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo, int32_t lw,
                  int32_t lh, const float frag_pos[3], const float frag_normal[3], const float texel[4],
                  float out[4]) {
  using namespace fmr;
  fragPos = v3(frag_pos);
  fragNormal = v3(frag_normal);
  fragPosNDC = glsl_shim::vec3(0, 0, 0);
  cameraPosition = v3(dc->camera_position);
  lightPosition = v3(dc->light_position);
  containerSize = dc->container_size;
  cornellBoxSize = dc->cornell_box_size;
  environmentMode = dc->environment_mode;
  renderMode = dc->render_mode;
  skybox.faces = sky;
  skybox.face = face;
  oxLogo.img = logo;
  oxLogo.w = lw;
  oxLogo.h = lh;
  phaseThicknessTexture.value = texel;
  // FluidMeshRenderer::draw(drawCommand, multiphase, ...) from Fluid::draw
  const int m = dc->render_mode;
  usePhaseThicknessTexture = (m == AQ_RENDER_MULTIPHASE_MESH || (m >= AQ_RENDER_REFRACT_MESH && m <= AQ_RENDER_PHASE1_MESH)) ? 1 : 0;
  for (int i = 0; i < 4; ++i)
    phaseColors[i] = glsl_shim::vec4(dc->phase_colors[i][0], dc->phase_colors[i][1], dc->phase_colors[i][2],
                                     dc->phase_colors[i][3]);
  phaseCount = dc->phase_count;
  color = glsl_shim::vec4(0);
  shader_main();
  out4(color, out);
}

void aqshade_container(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo, int32_t lw,
                       int32_t lh, const float frag_pos[3], float out[4]) {
  using namespace cface;
  FragPos = v3(frag_pos);
  cameraPosition = v3(dc->camera_position);
  lightPosition = v3(dc->light_position);
  containerSize = dc->container_size;
  cornellBoxSize = dc->cornell_box_size;
  environmentMode = dc->environment_mode;
  skybox.faces = sky;
  skybox.face = face;
  oxLogo.img = logo;
  oxLogo.w = lw;
  oxLogo.h = lh;
  color = glsl_shim::vec4(0);
  shader_main();
  out4(color, out);
}

}  // extern "C"
