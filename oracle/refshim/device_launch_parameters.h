// device_launch_parameters.h -- empty host stand-in (TEST INFRASTRUCTURE ONLY): the prelude supplies the CUDA
// types and qualifiers the reference rasterizer uses.
#pragma once
