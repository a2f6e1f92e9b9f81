// GLL derivative tables as compile-time constants, shared by the element
// kernels of the solver and of the kernel smoother.
#pragma once

#include <cuda_runtime.h>

namespace sem {

// D[i][l] = l_l'(xi_i) and DWt[i][l] = w_l D[l][i] for the GLL nodes
// (-1, -sqrt(3/7), 0, sqrt(3/7), 1): double-precision values rounded to
// float, identical to the host-built tables.  Only ever indexed with
// compile-time constants (fully unrolled loops), so they fold to immediates.

// Contraction term with a compile-time GLL coefficient: a zero coefficient
// (the interior diagonal D[i][i] = 0 of the GLL derivative matrix, and the
// matching entries of the weighted transpose) costs no instruction.
__device__ __forceinline__ float cfma(float c, float v, float a) {
  return c == 0.0f ? a : fmaf(c, v, a);
}

__device__ __forceinline__ float gD(int i, int l) {
  constexpr float t[25] = {
      -5.0f, 6.7565024887242409f, -2.6666666666666674f, 1.410164177942427f, -0.5f,
      -1.2409902530309822f, 0.0f, 1.7457431218879393f,
      -0.76376261582597327f, 0.25900974696901707f,
      0.37499999999999989f, -1.3365845776954535f, 0.0f, 1.3365845776954532f,
      -0.37499999999999989f,
      -0.25900974696901713f, 0.76376261582597349f, -1.7457431218879396f,
      0.0f, 1.2409902530309824f,
      0.5f, -1.4101641779424272f, 2.6666666666666674f, -6.75650248872424f, 5.0f};
  return t[i * 5 + l];
}
__device__ __forceinline__ float gDWt(int i, int l) {
  constexpr float t[25] = {
      -0.5f, -0.67565024887242353f, 0.26666666666666661f, -0.14101641779424265f,
      0.050000000000000003f,
      0.67565024887242409f, 0.0f, -0.95046014413898916f,
      0.41582631306080775f, -0.14101641779424273f,
      -0.26666666666666677f, 0.95046014413898916f, 0.0f, -0.95046014413898927f,
      0.26666666666666677f,
      0.1410164177942427f, -0.41582631306080764f, 0.95046014413898905f,
      0.0f, -0.67565024887242409f,
      -0.050000000000000003f, 0.14101641779424262f, -0.26666666666666661f,
      0.67565024887242375f, 0.5f};
  return t[i * 5 + l];
}
__device__ __forceinline__ float gW(int i) {
  constexpr float t[5] = {0.10000000000000001f, 0.5444444444444444f, 0.71111111111111114f,
                          0.5444444444444444f, 0.10000000000000001f};
  return t[i];
}

}  // namespace sem
