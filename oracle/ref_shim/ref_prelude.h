// Included ahead of every reference source compiled by oracle/ref_build.sh
// (TEST INFRASTRUCTURE ONLY).  The reference builds with its precompiled
// headers (SVO/include/pch.h and friends), which bring in <cfloat> and the
// float overloads its headers name as std::tanf / std::powf / std::ldexpf;
// GCC 13's libstdc++ declares those only in the global namespace.
#pragma once
#include <algorithm>
#include <any>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
namespace std {
using ::ldexpf;
using ::powf;
using ::tanf;
}  // namespace std
