// Shared pieces of the drop-in build: the reference's own class declarations
// (include/mshqc/*.h of mshqc, on the include path of this build) implemented
// on libmshqc_cuda.so.  One device context per process serves every class.
#pragma once

#include <stdexcept>
#include <string>

#include "../../include/mshqc_ao.h"
#include "../../include/mshqc_cd.h"

namespace mshqc_dropin {

// The process's context on the device named by MSHQC_DEVICE (default 0),
// created on first use; every failure of the C ABI becomes a
// std::runtime_error carrying the library's message.
mshqc_cd_ctx* context();
void check(int rc);
// MSHQC_CD_PRECISION=fp16x3 selects the mixed precision for the energies,
// anything else (the default) FP64.
int precision();
// Byte limit for amplitudes stored in results (MSHQC_T2_MAX_BYTES, default
// 8 GiB): the reference always stores t2; above the limit the drop-in
// leaves the tensors empty instead of exhausting host memory.
size_t t2_max_bytes();

}  // namespace mshqc_dropin
