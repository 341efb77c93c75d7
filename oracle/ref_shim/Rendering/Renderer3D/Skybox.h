/* Headless stub: included by the FLIP header, unused by the step. */
#ifndef CUBEMAPLEARN_SKYBOX_H
#define CUBEMAPLEARN_SKYBOX_H
struct Skybox {};
#endif
