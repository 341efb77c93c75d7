/* Headless stub: included by the FLIP header, unused by the step. */
#pragma once
struct Container {};
