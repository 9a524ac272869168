// Project-written stand-in: the reference's CUDA files include <glm/vec4.hpp>.
#pragma once

#include "glm.hpp"
