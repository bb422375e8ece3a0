// Stand-in for the reference's utils/cuda/CUDAMacro.h (test infrastructure): host-only build.
#pragma once
#define _CUDA_GENERAL_CALL_
