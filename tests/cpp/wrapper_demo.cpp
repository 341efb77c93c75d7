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
  std::printf("particles %d ink %d time %.3f center %.1f size %.1f\n", fluid.particleCount(),
              fluid.inkParticleCount, fluid.physicalTime, fluid.getCenter()[0], fluid.getContainerSize());
  return fluid.physicalTime > 0 && fluid.inkParticleCount > 0 ? 0 : 4;
}
