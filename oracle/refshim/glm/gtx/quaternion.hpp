// TEST INFRASTRUCTURE ONLY: the glm header path the reference includes; its contents are in
// kf_glm_subset.hpp.
#pragma once
#include <glm/kf_glm_subset.hpp>
