// Instantiations of the generic functor stage for the built-in flux schemes
// (FP64; this translation unit is compiled with -fmad=false).
#include "fv_schemes.cuh"

namespace dn {

cudaError_t launch_scheme_stage(int scheme, const dn_stage_launch* L, const WallBC& wall)
{
  switch (scheme) {
    case DN_FLUX_AUSMPLUS:
    case DN_FLUX_AUSMPLUS_FUNCTOR: {
      SchemeFlux<AusmPlusScheme> op{AusmPlusScheme{}, wall};
      return launch_functor_stage(L, op);
    }
    case DN_FLUX_VANLEER: {
      SchemeFlux<VanLeerScheme> op{VanLeerScheme{}, wall};
      return launch_functor_stage(L, op);
    }
    case DN_FLUX_ROE: {
      SchemeFlux<RoeScheme> op{RoeScheme{}, wall};
      return launch_functor_stage(L, op);
    }
    default:
      return cudaErrorInvalidValue;
  }
}

} // namespace dn
