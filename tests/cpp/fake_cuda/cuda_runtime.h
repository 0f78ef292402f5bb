// Test double of the CUDA runtime header: the types, constants and calls
// that the engine's host runtime (harvest_cuda_b200/csrc/hv_runtime.h) uses.
// Error codes keep the runtime's numeric values, so messages read the same.
// The test program defines the functions and decides what each call returns.
#pragma once
#include <cstddef>

#include "cuda.h"

enum cudaError {
  cudaSuccess = 0,
  cudaErrorMemoryAllocation = 2,
  cudaErrorInsufficientDriver = 35,
  cudaErrorNoDevice = 100,
};
typedef enum cudaError cudaError_t;

enum cudaDeviceAttr {
  cudaDevAttrMultiProcessorCount = 16,
  cudaDevAttrComputeCapabilityMajor = 75,
};

struct cudaDeviceProp {
  char name[256];
  int major;
  int minor;
};

enum cudaDriverEntryPointQueryResult {
  cudaDriverEntryPointSuccess = 0,
  cudaDriverEntryPointSymbolNotFound = 1,
};
#define cudaEnableDefault 0ULL

typedef struct FakeCudaStream* cudaStream_t;
typedef struct FakeCudaEvent* cudaEvent_t;

const char* cudaGetErrorName(cudaError_t error);
const char* cudaGetErrorString(cudaError_t error);
cudaError_t cudaGetLastError(void);
cudaError_t cudaGetDeviceCount(int* count);
cudaError_t cudaDeviceGetAttribute(int* value, enum cudaDeviceAttr attr, int device);
cudaError_t cudaGetDeviceProperties(struct cudaDeviceProp* prop, int device);
cudaError_t cudaGetDriverEntryPoint(const char* symbol, void** fn, unsigned long long flags,
                                    enum cudaDriverEntryPointQueryResult* status);
cudaError_t cudaMalloc(void** ptr, size_t bytes);
cudaError_t cudaFree(void* ptr);
cudaError_t cudaEventSynchronize(cudaEvent_t event);
cudaError_t cudaStreamSynchronize(cudaStream_t stream);
