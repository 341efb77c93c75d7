// Headless stand-in for GL/glew.h: the reference's camera.h includes it but
// uses nothing from it (test infrastructure only; oracle/shade_harness.cpp).
#pragma once
