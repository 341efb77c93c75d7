/* Headless stub of the reference's mesh renderer (constructed by init). */
#pragma once
#include "../../Common/GpuCommons.h"
#include "../DrawCommand.h"
#include "PointSprites.h"
#include <memory>
#include <vector>

struct FluidMeshRenderer {
  float* coordsDevice = nullptr;
  explicit FluidMeshRenderer(int) {}
  void draw(const DrawCommand&, bool = false, std::shared_ptr<PointSprites> = nullptr, float = 0,
            std::vector<float4> = {}) {}
};
