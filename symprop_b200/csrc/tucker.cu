// placeholder, replaced by the Tucker drivers
#include "tensor.cuh"
extern "C" int symprop_tucker(const symprop_tensor *, const symprop_config *, int, symprop_result *) {
  spb::set_last_error("not built yet");
  return SYMPROP_ERR_INVALID;
}
