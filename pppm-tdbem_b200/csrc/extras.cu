// Entry points whose implementation lands in later files of this library: the adjoint.
// Until then it reports PPPM_ERR_STATE with a message.
#include "handle.cuh"

extern "C" {

int pppm_adjoint(pppm_handle *, const float *, int, const float *, int, float *)
{
    pb::set_error("adjoint is not available in this build");
    return PPPM_ERR_STATE;
}
}
