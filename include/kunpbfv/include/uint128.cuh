// Drop-in for kunpBFV's include/uint128.cuh: a driver written for the reference
// (#include "include/uint128.cuh") compiles unmodified with -I <this repo>/include/kunpbfv
// and runs on libkbfv.so.
#pragma once
#include "../../kbfv_compat_global.hpp"
