// Split-precision tcgen05 fit (placeholder until the tensor-core kernel lands).
#include "zola_internal.h"

namespace zola {

int launch_fit_split(zola_ctx* ctx, zola_psf*, WindowTables*, const float*, const double*, int,
                     const zola_fit_params*, double*, double*, double*, int*, int*, cudaStream_t) {
    ctx->err = "split-precision fit not built";
    return ZOLA_E_UNSUPPORTED;
}

}  // namespace zola
