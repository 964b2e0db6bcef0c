// TEST INFRASTRUCTURE ONLY: stands in for the reference's project/src/window.h (an SDL/OpenGL
// window and Kinect sensor class) in the compute files that include it and use none of it
// (project/src/measurement.cuh:3).  The harness has no window: frames come from memory.
#pragma once
