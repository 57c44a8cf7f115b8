// Spectral operators of the k-space scheme, generated per point from 1D
// tables (shared by the column kernels).
#pragma once
#include "kernels.cuh"

namespace kwb {

// sin(x)/x and cos(x) from their Maclaurin series (Horner form) as
// polynomials in u = x^2, so callers holding |k|^2 need no square root.
// Accurate to FP32 rounding for |x| <= pi; larger arguments use sinf / cosf.
__device__ __forceinline__ float sinc_sq(float u) {
  if (u > 9.8696044f) {
    const float x = sqrtf(u);
    return sinf(x) / x;
  }
  // Horner over sum_{n=0}^{10} (-1)^n u^n / (2n+1)!
  float s = 1.9572941063391262e-20f;            //  1/21!
  s = fmaf(s, u, -8.2206352466243295e-18f);     // -1/19!
  s = fmaf(s, u, 2.8114572543455206e-15f);      //  1/17!
  s = fmaf(s, u, -7.6471637318198164e-13f);     // -1/15!
  s = fmaf(s, u, 1.6059043836821613e-10f);      //  1/13!
  s = fmaf(s, u, -2.5052108385441720e-08f);     // -1/11!
  s = fmaf(s, u, 2.7557319223985893e-06f);      //  1/9!
  s = fmaf(s, u, -1.9841269841269841e-04f);     // -1/7!
  s = fmaf(s, u, 8.3333333333333333e-03f);      //  1/5!
  s = fmaf(s, u, -1.6666666666666667e-01f);     // -1/3!
  s = fmaf(s, u, 1.0f);
  return s;
}

__device__ __forceinline__ float cos_sq(float u) {
  if (u > 9.8696044f) return cosf(sqrtf(u));
  float s = 4.1103176233121648e-19f;            //  1/20!
  s = fmaf(s, u, -1.5619206968586225e-16f);     // -1/18!
  s = fmaf(s, u, 4.7794773323873853e-14f);      //  1/16!
  s = fmaf(s, u, -1.1470745597729725e-11f);     // -1/14!
  s = fmaf(s, u, 2.0876756987868099e-09f);      //  1/12!
  s = fmaf(s, u, -2.7557319223985891e-07f);     // -1/10!
  s = fmaf(s, u, 2.4801587301587302e-05f);      //  1/8!
  s = fmaf(s, u, -1.3888888888888889e-03f);     // -1/6!
  s = fmaf(s, u, 4.1666666666666667e-02f);      //  1/4!
  s = fmaf(s, u, -0.5f);                        // -1/2!
  s = fmaf(s, u, 1.0f);
  return s;
}

__device__ __forceinline__ float sinc_series(float x) { return sinc_sq(x * x); }
__device__ __forceinline__ float cos_series(float x) { return cos_sq(x * x); }

__device__ __forceinline__ float2 eval_op(const SpecOp& op, const SpecTables& T, int dim, int ix,
                                          int iy, int iz) {
  float k2 = __ldg(T.k2[0] + ix) + __ldg(T.k2[1] + iy);
  if (dim == 3) k2 += __ldg(T.k2[2] + iz);
  const float k = sqrtf(k2);
  switch (op.kind) {
    case OP_GRAD_POS:
    case OP_GRAD_NEG: {
      // kappa = sinc(c_ref k dt / 2), sinc(x) = sin(x) / x (k-Wave/private/sinc.m:38-39)
      const float kap = sinc_series(T.cdt2 * k);
      const int id = op.axis == 0 ? ix : (op.axis == 1 ? iy : iz);
      const float2* tab = (op.kind == OP_GRAD_POS) ? T.ddk_pos[op.axis] : T.ddk_neg[op.axis];
      const float2 d = __ldg(tab + id);
      const float s = kap * T.scale;
      return make_float2(d.x * s, d.y * s);
    }
    case OP_NABLA1:
    case OP_NABLA2: {
      // k.^(y-2) / k.^(y-1) with the infinite value at k = 0 set to zero
      // (kspaceFirstOrder_createAbsorptionVariables.m:37-39, 49-51)
      const float e = (op.kind == OP_NABLA1) ? T.ym2 : T.ym1;
      float v;
      if (k == 0.f)
        v = (e == 0.f) ? 1.f : 0.f;
      else
        v = exp2f(e * log2f(k));
      return make_float2(v * T.scale, 0.f);
    }
    case OP_KAPPA:
      return make_float2(sinc_series(T.cdt2 * k) * T.scale, 0.f);
    case OP_SHIFT_NEG: {
      const int id = op.axis == 0 ? ix : (op.axis == 1 ? iy : iz);
      const float2 d = __ldg(T.shift_neg[op.axis] + id);
      return make_float2(d.x * T.scale, d.y * T.scale);
    }
    case OP_KAPPA_SHIFT_NEG: {
      const int id = op.axis == 0 ? ix : (op.axis == 1 ? iy : iz);
      const float2 d = __ldg(T.shift_neg[op.axis] + id);
      const float s = sinc_series(T.cdt2 * k) * T.scale;
      return make_float2(d.x * s, d.y * s);
    }
    case OP_SRC_KAPPA:
      return make_float2(cos_series(T.cdt2 * k) * T.scale, 0.f);
    default:
      return make_float2(T.scale, 0.f);
  }
}

}  // namespace kwb
