// Device-side construction of the operator from the mesh (placeholder).
#include <cuda_runtime.h>

#include "ctx.h"

int setup_projectors_device(scd_ctx *c) { return set_error(c, SCD_NOT_READY, "device projectors not built yet"); }
int setup_nearzone_device(scd_ctx *c, int) { return set_error(c, SCD_NOT_READY, "device near zone not built yet"); }
int setup_vswf(scd_ctx *c, int, cd *) { return set_error(c, SCD_NOT_READY, "device VSWF not built yet"); }

extern "C" {
int scd_grid_from_mesh(int32_t, const double *, int32_t, const int32_t *, double, int32_t, scd_grid_desc *) { return SCD_NOT_READY; }
int scd_set_mesh(scd_ctx *c, int32_t, const double *, const int32_t *, const scd_c128 *) { return set_error(c, SCD_NOT_READY, "todo"); }
int scd_build_projectors(scd_ctx *c) { return setup_projectors_device(c); }
int scd_build_nearzone(scd_ctx *c, int32_t p) { return setup_nearzone_device(c, p); }
int scd_get_projectors(scd_ctx *c, scd_c128 *, scd_c128 *, scd_c128 *, scd_c128 *, int32_t *) { return set_error(c, SCD_NOT_READY, "todo"); }
int64_t scd_nearzone_count(scd_ctx *) { return -1; }
int scd_get_nearzone(scd_ctx *c, int64_t, scd_c128 *, int32_t *) { return set_error(c, SCD_NOT_READY, "todo"); }
int scd_vswf_rhs(scd_ctx *c, int32_t, scd_c128 *) { return set_error(c, SCD_NOT_READY, "todo"); }
}
