// Drop-in for kunpBFV's include/BFVcontext.h: a driver written for the reference
// (#include "include/BFVcontext.h") compiles unmodified with -I <this repo>/include/kunpbfv
// and runs on libkbfv.so.
#pragma once
#include "../../kbfv_compat_global.hpp"
