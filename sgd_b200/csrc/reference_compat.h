// The reference's C++ layer classes under their global-namespace names, for
// callers written against layers/A_B1.hh and utils/matrix_double.hh (for
// example SGD.cu:176-187 and Bilinear.cu:25-39 of the reference, which build
// a MatrixD, call A_B1::project / back_project and read the result): include
// this header in place of those two and link sgd_b200/libnetwork.so.
#pragma once

#include "b1_layer.h"
#include "matrix_double.h"

using MatrixD = sgd::MatrixD;
using A_B1 = sgd::A_B1;
