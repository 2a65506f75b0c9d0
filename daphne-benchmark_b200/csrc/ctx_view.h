// Read-only view of a context's evaluation set-up (grid, constants, launch
// shape, stream), for entry points that live outside engine.cu.
#pragma once
#include <cuda_runtime.h>

#include "ndt_types.h"

struct ndt_ctx;

namespace ndt {

struct CtxEvalView {
    GridDev grid;
    double d1, d2;
    int compat;
    int precision;
    int variant;
    int sms;
    int device;
    cudaStream_t stream;
    bool have_map;
};

// Fills *v from the context; returns 0, or NDT_E_ARG for a null argument.
int ctx_eval_view(ndt_ctx *c, CtxEvalView *v);
// Records an error message on the context (ndt_last_error).
void ctx_set_error(ndt_ctx *c, const char *msg);

}  // namespace ndt
