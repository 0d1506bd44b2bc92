// Status strings and version of the C ABI.
#include <cuda_runtime.h>

#include "../../include/litho_b200.h"

extern "C" const char* litho_status_string(int status) {
  switch (status) {
    case LITHO_OK: return "ok";
    case LITHO_E_NULL: return "a required pointer is NULL";
    case LITHO_E_SIZE: return "a size or count is out of range";
    case LITHO_E_WORKSPACE: return "workspace is smaller than the *_workspace() size";
    case LITHO_E_BAND: return "band or coarse-grid geometry is inconsistent";
    case LITHO_E_UNSUPPORTED: return "request is valid but not served by this build";
    case LITHO_E_ALIGN: return "a pointer or offset is not aligned";
    case LITHO_E_DEVICE: return "no usable sm_100 device";
    case LITHO_E_SCRATCH:
      return "plan needs more scratch than the fixed no-allocation buffer holds; use litho_abbe() with a "
             "caller workspace or a smaller batch";
    case LITHO_E_TIMEOUT: return "a bounded device-side wait gave up";
  }
  if (status > 0) return cudaGetErrorString(static_cast<cudaError_t>(status));
  return "unknown status";
}

extern "C" int litho_version(void) { return 200; }

extern "C" int litho_abi_sizes(int32_t* out, int n) {
  const int32_t sz[] = {(int32_t)sizeof(LithoPupil), (int32_t)sizeof(LithoJob), (int32_t)sizeof(LithoItem),
                        (int32_t)sizeof(LithoNorm), (int32_t)sizeof(LithoAbbePlan),
                        (int32_t)sizeof(LithoMirror), (int32_t)sizeof(LithoUnevenGroup),
                        (int32_t)sizeof(LithoQueueTask)};
  const int k = (int)(sizeof(sz) / sizeof(sz[0]));
  for (int i = 0; i < n && i < k && out; ++i) out[i] = sz[i];
  return k;
}
