/* Headless stub of the reference's surface mesher: constructed by
 * Fluid::init and called from draw(); meshing is not part of the step. */
#pragma once
#include "../../Common/GpuCommons.h"

struct Mesher {
  int triangleCount = 0;
  Mesher(float3, float, int, int, int) {}
  template <typename Particle>
  void mesh(Particle*&, Particle*&, int*, int*, float*) {}
};
