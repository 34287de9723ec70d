// capi_plan.h -- the handle behind efmm_plan (internal header).
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include "plan.h"

struct efmm_plan {
  int device;
  cudaStream_t stream;
  std::unique_ptr<efmm::Plan> plan;
  cudaEvent_t user_ev[8];
};
