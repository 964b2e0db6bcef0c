// TEST INFRASTRUCTURE ONLY: the stb_image entry points that project/src/depth_map.cpp calls to
// read depth PNGs (stb is an empty submodule of the reference).  The harness hands frames to
// DepthMap::update(void*) from memory, so the file readers report failure.
#pragma once
#include <cstdlib>
static inline unsigned short* stbi_load_16(const char*, int*, int*, int*, int) { return nullptr; }
static inline void stbi_image_free(void* p) { std::free(p); }
