// GELU and its derivative for the encoder kernels, in FP32 for BF16 outputs.
//
// Phi(z) = (1 + erf(z / sqrt 2)) / 2 with erf from Abramowitz & Stegun 7.1.26,
// erf(x) = 1 - (a1 t + a2 t^2 + a3 t^3 + a4 t^4 + a5 t^5) e^{-x^2}, t = 1 / (1 + p x),
// x >= 0, |error| <= 1.5e-7 (far below the BF16 rounding of the stored values);
// e^{-x^2} with x = |z| / sqrt 2 is also e^{-z^2/2}, so phi(z) = e^{-z^2/2} / sqrt(2 pi)
// shares the exponential.
#pragma once

namespace umapb {

__device__ __forceinline__ void gauss_cdf_pdf(float z, float& cdf, float& pdf) {
  const float x = fabsf(z) * 0.70710678118654752f;
  const float t = __fdividef(1.0f, fmaf(0.3275911f, x, 1.0f));
  const float e = __expf(-x * x);
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
  const float erfx = 1.0f - poly * e;
  cdf = 0.5f * (1.0f + copysignf(erfx, z));
  pdf = 0.39894228040143268f * e;
}

__device__ __forceinline__ float gelu(float z) {
  float c, p;
  gauss_cdf_pdf(z, c, p);
  return z * c;
}

// d/dz [z Phi(z)] = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad(float z) {
  float c, p;
  gauss_cdf_pdf(z, c, p);
  return fmaf(z, p, c);
}

}  // namespace umapb
