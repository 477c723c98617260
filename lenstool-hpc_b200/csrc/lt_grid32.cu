/*
 * lt_grid32.cu -- FP32-compensated grid path (placeholder until the kernel lands).
 */
#include "lt_internal.h"

namespace lt {

lt_status prepare_catalog_extensions(lt_context *, lt_catalog *) { return LT_OK; }

int launch_fp32c(lt_context *ctx, const lt_catalog *, int, GridArgs &, void *)
{
    set_error(ctx, "FP32C precision is not available in this build");
    return (int)cudaErrorNotSupported;
}

void destroy_extensions(lt_context *) {}

} // namespace lt
