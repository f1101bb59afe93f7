// k_advect_y.cu -- the y sweep's instantiations (advect_y).  One
// translation unit per direction lets the three compile in parallel.  The y
// block kernel measured faster on B200 with the division fallback inlined
// (C2: 1.42 against 1.50 ms), unlike x and z.
#define A3G_DIV_FALLBACK_INLINE
#include "k_advect.cuh"

namespace a3g {

int launch_advect_y(a3g_ctx *ctx) {
  int rc = refresh_dtv(ctx);
  if (rc) return rc;
  tbegin(ctx, A3G_K_ADVECT_Y);
  A3G_LIM_SWITCH(launch_dir_lim, 1, )
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}

}  // namespace a3g
