/*
 * Headless stand-in for the reference's Common/GpuCommons.h, used only to
 * build the reference FLIP sources as a test oracle (oracle/_ref).
 * It keeps what the FLIP path uses from the original header: glm,
 * helper_math, thrust, Commons.h (divUp, random0to1) and the two error
 * macros.  It drops the GL/GLFW/interop includes.  The macros keep the
 * reference's cudaDeviceSynchronize() but record the first error instead of
 * calling exit(), so a failing call is reported to the caller.
 */
#ifndef AQUARIUS_GPUCOMMONS_H
#define AQUARIUS_GPUCOMMONS_H

#include <glm/glm.hpp>
#include <glm/gtc/matrix_transform.hpp>
#include <glm/gtc/type_ptr.hpp>

#include <string>
#include <iostream>
#include <stdexcept>
#include <stdio.h>
#include <helper_math.h>
#include <device_launch_parameters.h>
#include <stdarg.h>
#include <functional>
#include <memory>
#include <vector>

#include <thrust/functional.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>
#include <thrust/execution_policy.h>
#include "Commons.h"

extern cudaError_t aqref_first_error;

inline void aqref_record(cudaError_t err, const char* what, const char* file, int line) {
  if (err != cudaSuccess && aqref_first_error == cudaSuccess) {
    aqref_first_error = err;
    fprintf(stderr, "reference CUDA error: %s (%s) in %s at line %d\n", cudaGetErrorString(err), what, file, line);
  }
}

#define HANDLE_ERROR(err) \
  cudaDeviceSynchronize(); \
  aqref_record((err), "call", __FILE__, __LINE__)

#define CHECK_CUDA_ERROR(msg) \
  do { cudaDeviceSynchronize(); aqref_record(cudaGetLastError(), (msg), __FILE__, __LINE__); } while (0)

inline void printGLError() {}

// The reference sizes the device printf FIFO when a Fluid is built
// (Fluid/Fluid_3D_FLIP.cu:489).  CUDA refuses that call once any kernel with
// printf has run in the process, which happens when a test builds a second
// reference Fluid after stepping a first one.  The FIFO only bounds buffered
// device printf output, never the simulation, so that refusal is not an
// error here; every other limit and error passes through.
inline cudaError_t aqref_device_set_limit(cudaLimit limit, size_t value) {
  const cudaError_t e = cudaDeviceSetLimit(limit, value);
  if (e == cudaErrorInvalidValue && limit == cudaLimitPrintfFifoSize) {
    (void)cudaGetLastError();
    return cudaSuccess;
  }
  return e;
}
#define cudaDeviceSetLimit aqref_device_set_limit

#endif
