/* ORACLE (test infrastructure): force-included when compiling the
 * unmodified reference sources for sm_100a. The reference was written for
 * sm_35 and calls the pre-Volta warp intrinsics __any/__shfl/__shfl_up/
 * __shfl_down (match/Match.cu:594, 937, 1003-1052, ...), which do not exist
 * for compute_70 and later. They are mapped here to their *_sync forms with
 * a full-warp mask, which is what the reference's whole-warp call sites mean.
 */
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#ifdef __cplusplus
#include <thrust/device_vector.h>
#include <thrust/scan.h>
#include <thrust/sort.h>
#endif
#ifdef __CUDACC__
#define __any(p) __any_sync(0xffffffffu, (p))
#define __shfl(v, ...) __shfl_sync(0xffffffffu, (v), __VA_ARGS__)
#define __shfl_up(v, ...) __shfl_up_sync(0xffffffffu, (v), __VA_ARGS__)
#define __shfl_down(v, ...) __shfl_down_sync(0xffffffffu, (v), __VA_ARGS__)
#endif
