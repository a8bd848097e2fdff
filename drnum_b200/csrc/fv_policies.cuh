// Storage/arithmetic policies of the fused stage kernel.
#pragma once

#include <cstdint>

namespace dn {

// Plain FP64: stored, computed and updated in double, operation order of the
// reference CPU iterator.  The translation unit that instantiates it is built
// with -fmad=false so no multiply-add pair is contracted.
struct PolicyF64 {
  using Store = double;
  using Real = double;
  using FaceT = double;
  struct Params {
    double Ax, Ay, Az;   // face areas dy*dz, dx*dz, dx*dy (cartesianiterator.h:96-98)
    double pf;           // factor/dV (cartesianiterator.h:311)
  };
  static __device__ __forceinline__ double load(const Params&, int, double x) { return x; }
  static __device__ __forceinline__ double face(const Params&, int, double F) { return F; }
  static __device__ __forceinline__ double update(const Params& p, int, double un, double r, int&)
  {
    return un + p.pf*r;
  }
};

} // namespace dn
