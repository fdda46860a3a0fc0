// The reference header Geometry/auxiliary.h, provided by this library's C++ shim (iternlm.hpp)
// so that a driver written against the reference compiles unchanged.
#pragma once
#include "iternlm.hpp"
