// Include shim: tutorial/Base5prop.cuh includes "../kernel.cuh"; this
// forwards to the build-time truncated copy of the reference's
// header/kernel.cuh (oracle/_ref/kshim/header/kernel.cuh, -I before the
// reference tree).
#pragma once
#include "header/kernel.cuh"
