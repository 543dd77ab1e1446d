// Include shim: tutorial/Base5prop.cuh includes "../graph.h"; with
// -I oracle/ref_shim_gpu/inc that name resolves here, and this forwards to
// the reference's header/graph.h (found through -I <reference>).
#pragma once
#include "header/graph.h"
