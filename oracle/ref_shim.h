/*
 * ref_shim.h -- pre-included (nvcc --pre-include) when the reference's own
 * CUDA build is compiled for sm_100a into oracle/_ref/.  The reference uses the
 * pre-CUDA-9 warp shuffle __shfl_xor (src/GPU_kernels.cu:359,366-367,3075,3089),
 * which no longer exists; this maps it onto the full-warp synchronous form.
 * No reference source is modified or copied.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#define __shfl_xor(v, m) __shfl_xor_sync(0xffffffffu, (v), (m))
