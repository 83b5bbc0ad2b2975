// Stand-in for glm/gtc/matrix_transform.hpp: translate and scale live in
// ../glm.hpp (TEST INFRASTRUCTURE ONLY, see there).
#pragma once
#include "../glm.hpp"
