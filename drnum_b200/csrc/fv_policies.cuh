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

// FP32 bulk with grid-quantised offsets.
//
// A patch stores per variable v an FP64 base B_v and a power-of-two quantum
// q_v; a cell holds the FP32 value o = (U - B_v)/q_v, which is always an
// integer with |o| < 2^24, so U = B_v + q_v*o is exact in FP64.  Arithmetic
// runs in FP32 on U = B_v + q_v*o.  Each face flux, scaled by factor/dV, is
// rounded once to an integer number of quanta; both cells of the face add the
// same integer with opposite sign and all sums of such integers are exact in
// FP32.  Hence the per-variable totals (mass, momenta, energy) over a
// periodic patch are conserved exactly, and their FP64 sums are exact and
// independent of the summation order.  The resolution of q_v is chosen as the
// FP32 spacing of the variable's magnitude scale, so it matches plain FP32
// storage.  A cell that would leave the exact range sets bit 1 of the error
// word (the value is still rounded to the nearest FP32).
struct PolicyF32Q {
  using Store = float;
  using Real = float;
  using FaceT = float;
  struct Params {
    float Ax, Ay, Az;
    float base[5];       // B_v rounded to FP32 (arithmetic only)
    float quantum[5];    // q_v
    float face_scale[5]; // (factor/dV)/q_v
  };
  static __device__ __forceinline__ float load(const Params& p, int v, float o)
  {
    return fmaf(p.quantum[v], o, p.base[v]);
  }
  // round to the nearest integer with ties to even; valid for every finite x
  // because x + copysign(1.5*2^23, x) has a magnitude of at least 2^23
  static __device__ __forceinline__ float round_int(float x)
  {
    const float m = copysignf(12582912.0f, x);
    return __fsub_rn(__fadd_rn(x, m), m);
  }
  static __device__ __forceinline__ float face(const Params& p, int v, float F)
  {
    return round_int(__fmul_rn(F, p.face_scale[v]));
  }
  static __device__ __forceinline__ float update(const Params&, int, float un, float r, int& bad)
  {
    const float o = __fadd_rn(un, r);
    if (!(fabsf(o) < 16777216.0f)) bad |= 1;
    return o;
  }
};

} // namespace dn
