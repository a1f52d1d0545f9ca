// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Force-included last when building oracle/_ref/libwfref_det.so: the
// reference's host-compiled code with its C-library elementary functions
// replaced by the renderer's deterministic ones (wf_math.h).  Everything else
// in the reference stays as written, so the only difference between
// libwfref.so and libwfref_det.so is the math library, and the CUDA kernels
// (which use wf_math.h) can be compared with libwfref_det.so bit for bit.
#pragma once
#include <math.h>
#include <stdlib.h>
#include <complex>
#include <random>
#include <thread>
#include <mutex>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include "../wavefront-path-tracer_b200/csrc/wf_math.h"
// sincosf (texture transforms, device_traversal.cuh:335): sine and cosine
// from the same functions as sinf/cosf below.
inline void wfref_det_sincosf(float x, float* s, float* c) {
    *s = wfm::sinf(x);
    *c = wfm::cosf(x);
}
#define sincosf wfref_det_sincosf
#define sinf wfm::sinf
#define cosf wfm::cosf
#define tanf wfm::tanf
#define atan2f wfm::atan2f
#define logf wfm::logf
#define expf wfm::expf
#define powf wfm::powf
#define sin wfm::sin
#define cos wfm::cos
