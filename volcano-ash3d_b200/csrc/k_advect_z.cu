// k_advect_z.cu -- the z sweep's instantiations (advect_z).  One
// translation unit per direction lets the three compile in parallel.
#include "k_advect.cuh"

namespace a3g {

int launch_advect_z(a3g_ctx *ctx) {
  int rc = refresh_dtv(ctx);
  if (rc) return rc;
  tbegin(ctx, A3G_K_ADVECT_Z);
  A3G_LIM_SWITCH(launch_dir_lim, 2, )
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}

}  // namespace a3g
