// Umbrella header of the C++ front end (header-only, over librw_tree.so).
#pragma once

#include <cuda_runtime.h>

#include "rw_tree.h"
#include "redwood_tree/app_data.hpp"
#include "redwood_tree/cu_dispatcher.hpp"
#include "redwood_tree/cu_mem_resource.hpp"
#include "redwood_tree/engine.hpp"
