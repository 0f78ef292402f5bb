// Test double of the CUDA driver header: the few types and entry points the
// engine's host runtime (harvest_cuda_b200/csrc/hv_runtime.h) names. The
// test program defines the functions and decides what each call returns.
#pragma once

typedef int CUresult;
typedef int CUdevice;
typedef struct FakeCudaContext* CUcontext;

#define CUDA_SUCCESS 0

CUresult cuInit(unsigned int flags);
CUresult cuDevicePrimaryCtxRetain(CUcontext* ctx, CUdevice device);
CUresult cuDevicePrimaryCtxRelease(CUdevice device);
CUresult cuCtxGetCurrent(CUcontext* ctx);
CUresult cuCtxSetCurrent(CUcontext ctx);
