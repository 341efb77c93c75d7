/* Headless stub of the reference's point-sprite renderer: the FLIP path only
 * constructs it and, in draw(), hands it a VBO pointer.  No graphics. */
#pragma once
#include "../../Common/GpuCommons.h"
#include "../DrawCommand.h"
#include <memory>

struct PointSprites {
  int count = 0;
  int stride = 7;
  float* positionsDevice = nullptr;
  explicit PointSprites(int count_) : count(count_) {}
  void draw(const DrawCommand&, float, unsigned int) {}
};
