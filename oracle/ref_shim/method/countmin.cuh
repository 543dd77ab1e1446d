// shim: CPUlp.cuh includes this CUDA header but uses nothing from it
#pragma once
