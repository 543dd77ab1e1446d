// shim: the reference CSR loader, header/graph.h
#pragma once
#include <climits>
#include "header/graph.h"
