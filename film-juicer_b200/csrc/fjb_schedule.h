// fjb_schedule.h -- helpers shared by the boundary and the frame schedule.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/juicer_cuda_api.h"

namespace fjb {

void write_error(FjErrorBuffer* error, const std::string& text);
FjStatus ok_status();
FjStatus fail_status(uint32_t category, FjErrorBuffer* error, const std::string& text);
FjStatus cuda_status(cudaError_t e, FjErrorBuffer* error, const char* where);

} // namespace fjb
