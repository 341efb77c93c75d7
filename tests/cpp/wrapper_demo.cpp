// Compiles the C++ wrapper the way a reference user would and runs the calls
// that need no GPU.  Without a device, init() throws aquarius_b200::Error with
// AQ_ERR_NO_DEVICE; with one, it steps a small scene.
#include <cstdio>

#include "aquarius_b200.hpp"

int main() {
  using namespace aquarius_b200;
  FluidConfig config;
  config.FLIP.sizeX = config.FLIP.sizeY = config.FLIP.sizeZ = 16;
  aq_config c = config.to_c();
  if (aq_config_validate(&c) != AQ_OK) return 2;
  Fluid_3D_FLIP::Fluid fluid;
  try {
    fluid.init(config);
  } catch (const Error& e) {
    std::printf("init: %s\n", e.what());
    return e.status == AQ_ERR_NO_DEVICE ? 0 : 3;
  }
  fluid.initInkRenderer();
  fluid.simulationStep();
  fluid.synchronize();
  std::vector<float> ink(3 * (size_t)fluid.inkParticleCount);
  fluid.downloadInk(ink.data(), nullptr);
  // Fluid::draw with main.cu's first-frame command, into the fluid's renderer
  const int W = 96, H = 64;
  DrawCommand dc = defaultDrawCommand(W, H, fluid.getContainerSize(), config.FLIP.sizeY);
  dc.environment_mode = AQ_ENV_CHESS_BOARD;  // procedural floor: lit without loaded textures
  fluid.draw(dc);
  std::vector<uint8_t> image((size_t)W * H * 4);
  fluid.renderer()->downloadImage(image.data());
  long lit = 0;
  for (size_t i = 0; i < image.size(); i += 4) lit += (image[i] | image[i + 1] | image[i + 2]) != 0;
  std::printf("particles %d ink %d time %.3f center %.1f size %.1f lit %ld\n", fluid.particleCount(),
              fluid.inkParticleCount, fluid.physicalTime, fluid.getCenter()[0], fluid.getContainerSize(), lit);
  return fluid.physicalTime > 0 && fluid.inkParticleCount > 0 && lit > 0 ? 0 : 4;
}
