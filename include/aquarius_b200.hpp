// Header-only C++ wrapper over the C ABI (aquarius_b200.h) that mirrors the
// reference's plugin surface, so code written against
// Fluid_3D_FLIP::Fluid / FluidConfig (AmesingFlank/Aquarius) changes only its
// include and namespace:
//
//   reference                                      here
//   ShapeType, InitializationVolume, ConfigFLIP,    aquarius_b200::ShapeType, ...
//   FluidConfig  (Fluid/FluidConfig.cuh:16-97)       (same members, same defaults)
//   Fluid_3D_FLIP::Fluid::init(FluidConfig)          aquarius_b200::Fluid_3D_FLIP::Fluid::init
//   ::simulationStep(), ::physicalTime,              same names
//   ::getCenter(), ::getContainerSize()
//     (Fluid/Fluid.h:4-12, Fluid/Fluid_3D.cuh:7-12)
//   ::initInkRenderer(), ::inkParticleCount          same names; the ink then
//     (Fluid/Fluid_3D_FLIP.cu:676-709)                moves at the end of every
//                                                    step (the reference's
//                                                    commented-out :349-350)
//
//   DrawCommand (Rendering/DrawCommand.h:37-59)       aquarius_b200::DrawCommand
//   ::draw(const DrawCommand&)                       same name: the headless
//     (Fluid/Fluid_3D_FLIP.cu:396-430)                 frame (aq_fluid_draw) into
//                                                    an RGBA8 image owned by a
//                                                    Renderer instead of a GL
//                                                    framebuffer
//
// Differences: errors throw aquarius_b200::Error (the reference prints and
// exits); draw() renders into a device image (row 0 at the bottom, as
// glReadPixels returns it) that Renderer::downloadImage copies out, since no
// graphics API is used; the centre is returned as std::array<float,3>
// instead of glm::vec3.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "aquarius_b200.h"

namespace aquarius_b200 {

struct Error : std::runtime_error {
  aq_status status;
  Error(aq_status st, const std::string& what) : std::runtime_error(what), status(st) {}
};

inline void check(aq_status st, const char* call) {
  if (st != AQ_OK) throw Error(st, std::string(call) + ": " + aq_last_error());
}

struct float3_ {
  float x, y, z;
};

enum class ShapeType { Sphere, Square };  // Fluid/FluidConfig.cuh:16-18

struct InitializationVolume {  // Fluid/FluidConfig.cuh:20-38
  ShapeType shapeType = ShapeType::Square;
  float3_ boxMin{0, 0, 0};
  float3_ boxMax{1, 0.1875f, 1};
  float3_ ballCenter{0.5f, 0.75f, 0.5f};
  float ballRadius = 0.125f;
  int phase = 0;
  InitializationVolume() = default;
  explicit InitializationVolume(ShapeType type) : shapeType(type) {}
};

struct ConfigFLIP {  // Fluid/FluidConfig.cuh:41-50
  int sizeX = 50;
  int sizeY = 50;
  int sizeZ = 50;
  int pressureIterations = 100;
  int diffusionIterations = 100;
  float timestep = 0.033f;
  float FLIPcoeff = 0.95f;
  float particleJitter = 0.05f;
};

struct FluidConfig {  // Fluid/FluidConfig.cuh:68-97
  std::string method = "FLIP";
  std::vector<InitializationVolume> initialVolumes;
  float3_ gravity{0, -9.8f, 0};
  int phaseCount = 2;
  std::array<float, 4> phaseDensities{1, 1, 1, 1};
  float diffusionCoeff = 0.001f;
  ConfigFLIP FLIP;
  // Extensions (no reference counterpart); defaults reproduce the reference.
  float gridPhysicalSize = 10.f;
  unsigned seed = 1;
  aq_pressure_init pressureInit = AQ_PRESSURE_CARRY;
  aq_solve_mode solveMode = AQ_SOLVE_FIXED;
  float relResidual = 1e-4f;
  int maxIterations = 2000;
  int checkInterval = 40;
  int device = 0;
  void* stream = nullptr;

  FluidConfig() {
    initialVolumes.emplace_back(ShapeType::Square);
    initialVolumes.emplace_back(ShapeType::Sphere);
  }

  aq_config to_c() const {
    if (method != "FLIP") throw Error(AQ_ERR_INVALID_CONFIG, "only the FLIP method is implemented");
    if (initialVolumes.size() > AQ_MAX_VOLUMES) throw Error(AQ_ERR_INVALID_CONFIG, "too many volumes");
    aq_config c;
    check(aq_config_default(&c), "aq_config_default");
    c.volume_count = (int32_t)initialVolumes.size();
    for (size_t i = 0; i < initialVolumes.size(); ++i) {
      const InitializationVolume& v = initialVolumes[i];
      aq_volume& o = c.volumes[i];
      o.shape = v.shapeType == ShapeType::Sphere ? AQ_SHAPE_SPHERE : AQ_SHAPE_SQUARE;
      o.box_min[0] = v.boxMin.x; o.box_min[1] = v.boxMin.y; o.box_min[2] = v.boxMin.z;
      o.box_max[0] = v.boxMax.x; o.box_max[1] = v.boxMax.y; o.box_max[2] = v.boxMax.z;
      o.ball_center[0] = v.ballCenter.x; o.ball_center[1] = v.ballCenter.y; o.ball_center[2] = v.ballCenter.z;
      o.ball_radius = v.ballRadius;
      o.phase = v.phase;
    }
    c.gravity[0] = gravity.x; c.gravity[1] = gravity.y; c.gravity[2] = gravity.z;
    c.phase_count = phaseCount;
    for (int k = 0; k < 4; ++k) c.phase_densities[k] = phaseDensities[k];
    c.diffusion_coeff = diffusionCoeff;
    c.size_x = FLIP.sizeX; c.size_y = FLIP.sizeY; c.size_z = FLIP.sizeZ;
    c.pressure_iterations = FLIP.pressureIterations;
    c.diffusion_iterations = FLIP.diffusionIterations;
    c.timestep = FLIP.timestep;
    c.flip_coeff = FLIP.FLIPcoeff;
    c.particle_jitter = FLIP.particleJitter;
    c.domain_size = gridPhysicalSize;
    c.seed = seed;
    c.pressure_init = pressureInit;
    c.solve_mode = solveMode;
    c.rel_residual = relResidual;
    c.max_iterations = maxIterations;
    c.check_interval = checkInterval;
    c.device = device;
    c.stream = stream;
    return c;
  }
};

using DrawCommand = aq_draw_command;

// The frame target of draw(): the reference draws into the window's GL
// framebuffer; here an RGBA8 device image owned by the renderer, with the
// skybox and logo textures the reference loads from files set by the caller.
class Renderer {
 public:
  explicit Renderer(int device = 0, void* stream = nullptr) {
    check(aq_renderer_create(device, stream, &r_), "aq_renderer_create");
  }
  Renderer(const Renderer&) = delete;
  Renderer& operator=(const Renderer&) = delete;
  ~Renderer() {
    if (r_) aq_renderer_destroy(r_);
  }
  // Six face_size^2 RGB8 faces, posx negx posy negy posz negz (Skybox.cu:24-44).
  void setSkybox(const uint8_t* faces_rgb, int face_size) {
    check(aq_renderer_set_skybox(r_, faces_rgb, face_size), "aq_renderer_set_skybox");
  }
  void setLogo(const uint8_t* rgb, int width, int height) {
    check(aq_renderer_set_logo(r_, rgb, width, height), "aq_renderer_set_logo");
  }
  void synchronize() { check(aq_renderer_synchronize(r_), "aq_renderer_synchronize"); }
  // The last frame, W*H*4 bytes into host memory, row 0 at the bottom.
  void downloadImage(uint8_t* host) { check(aq_renderer_download_image(r_, host), "aq_renderer_download_image"); }
  aq_renderer* handle() const { return r_; }

 private:
  aq_renderer* r_ = nullptr;
};

// DrawCommand of main.cu's first frame for a fluid (camera, projection,
// light, container, render and environment modes).
inline DrawCommand defaultDrawCommand(int width, int height, float containerSize, int sizeY) {
  DrawCommand dc{};
  check(aq_draw_command_default(&dc, width, height, containerSize, sizeY), "aq_draw_command_default");
  return dc;
}

namespace Fluid_3D_FLIP {

class Fluid {
 public:
  Fluid() = default;
  explicit Fluid(const FluidConfig& config) { init(config); }
  Fluid(const Fluid&) = delete;
  Fluid& operator=(const Fluid&) = delete;
  ~Fluid() { release(); }

  // Fluid::init (Fluid/Fluid_3D_FLIP.cu:435-505)
  void init(const FluidConfig& config) {
    release();
    const aq_config c = config.to_c();
    check(aq_fluid_create(&c, &f_), "aq_fluid_create");
    config_ = config;
    physicalTime = 0;
  }
  // Fluid::simulationStep (Fluid/Fluid_3D_FLIP.cu:316-352); asynchronous
  void simulationStep() {
    check(aq_fluid_step(f_, 1), "aq_fluid_step");
    double t = 0;
    check(aq_fluid_time(f_, &t), "aq_fluid_time");
    physicalTime = (float)t;
  }
  // Fluid::draw (Fluid/Fluid_3D_FLIP.cu:396-430), headless: meshes the
  // particles (mesh modes), fills the point-sprite VBO and draws the frame
  // into the renderer's image, or into rgba (a device buffer of W*H*4 bytes).
  void draw(const DrawCommand& drawCommand, Renderer& renderer, uint8_t* rgba = nullptr) {
    check(aq_fluid_draw(f_, renderer.handle(), &drawCommand, rgba), "aq_fluid_draw");
  }
  // The reference's one-argument form: draws with a renderer the fluid owns
  // (created on the fluid's device and stream at the first draw).
  void draw(const DrawCommand& drawCommand) {
    if (!renderer_) {
      void* stream = nullptr;
      check(aq_fluid_stream(f_, &stream), "aq_fluid_stream");
      renderer_.reset(new Renderer(config_.device, stream));
    }
    draw(drawCommand, *renderer_);
  }
  // The renderer of the one-argument draw (nullptr before the first draw).
  Renderer* renderer() const { return renderer_.get(); }
  std::array<float, 3> getCenter() const {
    std::array<float, 3> c{};
    check(aq_fluid_container(f_, c.data(), nullptr), "aq_fluid_container");
    return c;
  }
  float getContainerSize() const {
    float s = 0;
    check(aq_fluid_container(f_, nullptr, &s), "aq_fluid_container");
    return s;
  }
  int particleCount() const {
    int32_t n = 0;
    check(aq_fluid_particle_count(f_, &n), "aq_fluid_particle_count");
    return n;
  }
  void synchronize() { check(aq_fluid_synchronize(f_), "aq_fluid_synchronize"); }
  // Fluid::initInkRenderer (Fluid/Fluid_3D_FLIP.cu:676-709), headless: seeds
  // the ink once; from then on every simulationStep ends with
  // transferToInkParticles + moveInkParticles(timestep).
  void initInkRenderer() {
    int32_t n = 0;
    check(aq_fluid_enable_ink(f_, &n), "aq_fluid_enable_ink");
    inkParticleCount = n;
  }
  // transferToInkParticles + moveInkParticles(timestep)
  // (Fluid/Fluid_3D_FLIP.cu:711-725) on the current grids, as one launch.
  void advanceInk() { check(aq_fluid_ink_advance(f_), "aq_fluid_ink_advance"); }
  // Ink positions / velocities as [3][inkParticleCount] planes (either may be NULL).
  void downloadInk(float* position, float* velocity) {
    check(aq_fluid_download_ink(f_, position, velocity), "aq_fluid_download_ink");
  }
  aq_fluid* handle() const { return f_; }
  const FluidConfig& config() const { return config_; }

  float physicalTime = 0;  // Fluid/Fluid.h:10
  int inkParticleCount = 0;  // Fluid/Fluid_3D_FLIP.cuh:106

 private:
  void release() {
    renderer_.reset();
    if (f_) aq_fluid_destroy(f_);
    f_ = nullptr;
  }
  aq_fluid* f_ = nullptr;
  FluidConfig config_;
  std::unique_ptr<Renderer> renderer_;
};

}  // namespace Fluid_3D_FLIP
}  // namespace aquarius_b200
