// Entry points whose implementation lands in later files of this library: batched scenes
// and the adjoint.  Until then they report PPPM_ERR_STATE with a message.
#include "handle.cuh"

extern "C" {

int pppm_batch_create(pppm_handle **, int, pppm_batch **out)
{
    if (out)
        *out = nullptr;
    pb::set_error("batched scenes are not available in this build");
    return PPPM_ERR_STATE;
}

int pppm_batch_destroy(pppm_batch *) { return PPPM_OK; }

int pppm_batch_run(pppm_batch *, const float *const *, const int *, int)
{
    pb::set_error("batched scenes are not available in this build");
    return PPPM_ERR_STATE;
}

int pppm_adjoint(pppm_handle *, const float *, int, const float *, int, float *)
{
    pb::set_error("adjoint is not available in this build");
    return PPPM_ERR_STATE;
}
}
