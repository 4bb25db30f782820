// Per-(face, frequency) term of the analytic triangle Fourier transform.
//
// For a triangle with vertex phases x_a, x_b, x_c (x_v = xi . v) the reference
// evaluates (deltamic/cpp/fourier3d_cuda_kernel.cu:238-278, render.py:97-103)
//
//   F = e_a/(ab*ca) + e_b/(bc*ab) + e_c/(ca*bc),   e_v = exp(-i x_v),
//   ab = x_b-x_a, bc = x_c-x_b, ca = x_a-x_c,
//
// with degenerate branches R1 (two differences within Seps: F = e^{-i mean}/2),
// R2 |ab|<=Seps, R3 |bc|<=Seps, R4 |ca|<=Seps (the close pair merged at its
// midpoint d: F = (i e_d + (e_d - e_o)/delta)/delta), else R5 above.
// F is minus the second divided difference of exp(-i x) at the three phases.
//
// This file evaluates the same function in FP32 without the cancellation of
// the R5 formula:
//  * phases of vertices come from 32-bit fixed point: with xi_d = m_d pi / L_d
//    (m_d = 2k_d - (n_d - 1) an integer) and U_d = round((v_d - lo_d)/L_d * 2^31),
//    the phase in turns is sum_d m_d U_d / 2^32 (mod 1), exact in uint32;
//  * phase differences come from edge vectors (never from differences of large
//    phases), in half units h = (x_q - x_p)/2;
//  * F = e_p * G(U, W) with p the vertex opposite the largest difference,
//    U = x_q - x_p, W = x_r - x_p and
//        G = -i (S(U) - S(W)) / (W - U),   S(t) = (1 - e^{-it})/(it)
//          = e^{-it/2} sinc(t/2),
//    sinc by Taylor polynomial for |t/2| < 1 and sin/rcp otherwise;
//  * when |W - U| < 1 the divided difference is summed as its Taylor series
//    G = sum_n (-i)^n h_n(U,W)/(n+2)!  (h_n complete homogeneous symmetric
//    polynomials), which is exact to < 1e-7 there;
//  * the reference's branch selection (R1..R4 at Seps = sqrt(FLT_EPSILON)) is
//    kept: in those branches the same merged-vertex / centroid values are formed.
//
// The header compiles for the host too (libm sin/cos instead of the MUFU
// approximations) so the math can be checked on a machine without a GPU.
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define DM_HD __host__ __device__ __forceinline__
#define DM_HD_NOINLINE __host__ __device__ __noinline__
#else
#define DM_HD static inline
#define DM_HD_NOINLINE static
#endif

namespace dm {

// Seps/2: the reference compares |ab| <= sqrt(FLT_EPSILON); differences here are
// held in half units.
constexpr float kSepsHalf = 1.72633492e-4f;
// Series for |W - U| < 1 (half units: largest |h| < 0.5).
constexpr float kSeriesHalf = 0.5f;
// Polynomial sinc / sinc' below this half-angle magnitude.
constexpr float kPolyX = 1.0f;
constexpr float kTwoPi = 6.28318530717958647692f;

struct c32 {
  float x, y;
};

DM_HD c32 cmul(c32 a, c32 b) { return c32{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }

DM_HD float bits_to_float(uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

DM_HD void sincos_fast(float a, float* s, float* c) {
#if defined(__CUDA_ARCH__)
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*s) : "f"(a));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*c) : "f"(a));
#else
  *s = sinf(a);
  *c = cosf(a);
#endif
}

DM_HD float rcp_fast(float a) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
#else
  return 1.0f / a;
#endif
}

// Fixed-point phase (turns * 2^32, mod 2^32) -> angle in [-pi, pi).  Adding half
// a turn and keeping the top 23 bits (rounded) as the mantissa of a float in
// [1, 2) gives turns + 0.5 (mod 1) without any integer->float conversion.
DM_HD float turns_to_angle(uint32_t s) {
  uint32_t b = (((s ^ 0x80000000u) + 0x100u) >> 9) | 0x3F800000u;
  return (bits_to_float(b) - 1.5f) * kTwoPi;
}

// Taylor series of sin(x)/x and its derivative in y = x^2 (|x| < 1: the first
// dropped terms are below 2e-9).
DM_HD float sinc_poly(float y) {
  return 1.0f + y * (-1.0f / 6.0f + y * (1.0f / 120.0f + y * (-1.0f / 5040.0f +
         y * (1.0f / 362880.0f + y * (-1.0f / 39916800.0f)))));
}
DM_HD float dsinc_poly_over_x(float y) {
  return -1.0f / 3.0f + y * (1.0f / 30.0f + y * (-1.0f / 840.0f +
         y * (1.0f / 45360.0f + y * (-1.0f / 3991680.0f))));
}

// Per-face geometry as the kernels hold it.
struct FaceGeom {
  uint32_t Ua[3], Ub[3], Uc[3];  // fixed-point vertex positions (turns per unit m, * 2^32)
  float hab[3], hbc[3];          // (v_b - v_a) * pi/(2 L_d), (v_c - v_b) * pi/(2 L_d)
};

// Per-frequency data: integer grid offsets and the same values as floats.
struct XiVal {
  int32_t mi[3];
  float mf[3];
};

DM_HD uint32_t fixed_phase(const int32_t mi[3], uint32_t U0, uint32_t U1, uint32_t U2) {
  return (uint32_t)mi[0] * U0 + (uint32_t)mi[1] * U1 + (uint32_t)mi[2] * U2;
}

// G(U, W) and (optionally) dG/dU, dG/dW via S, for |W - U| >= 1.
// Inputs in half units (hu = U/2, hw = W/2); derivatives are per full unit.
template <bool kGrad>
DM_HD void g_sinc(float hu, float hw, c32& G, c32& Gu, c32& Gw) {
  float su, cu, sw, cw;
  sincos_fast(hu, &su, &cu);
  sincos_fast(hw, &sw, &cw);
  const float yu = hu * hu, yw = hw * hw;
  const bool pu = fabsf(hu) < kPolyX, pw = fabsf(hw) < kPolyX;
  const float uc = pu ? 1.0f : hu;
  const float wc = pw ? 1.0f : hw;
  const float d2 = 2.0f * (hw - hu);  // W - U
  const float R = rcp_fast(uc * wc * d2);
  const float t = d2 * R;
  const float ru = wc * t, rw = uc * t;   // 1/hu, 1/hw (where used)
  const float rD = (uc * wc) * R;         // 1/(W - U)
  const float snu = pu ? sinc_poly(yu) : su * ru;
  const float snw = pw ? sinc_poly(yw) : sw * rw;
  const float Sur = cu * snu, Sui = -su * snu;
  const float Swr = cw * snw, Swi = -sw * snw;
  G.x = (Sui - Swi) * rD;
  G.y = (Swr - Sur) * rD;
  if (kGrad) {
    const float dsu = pu ? hu * dsinc_poly_over_x(yu) : (cu - snu) * ru;
    const float dsw = pw ? hw * dsinc_poly_over_x(yw) : (cw - snw) * rw;
    // S'(t) = e^{-it/2} (sinc'(t/2) - i sinc(t/2)) / 2
    const float Spur = 0.5f * (cu * dsu - su * snu), Spui = -0.5f * (cu * snu + su * dsu);
    const float Spwr = 0.5f * (cw * dsw - sw * snw), Spwi = -0.5f * (cw * snw + sw * dsw);
    // dG/dU = (G - i S'(U))/(W-U),  dG/dW = (i S'(W) - G)/(W-U)
    Gu.x = (G.x + Spui) * rD;
    Gu.y = (G.y - Spur) * rD;
    Gw.x = (-Spwi - G.x) * rD;
    Gw.y = (Spwr - G.y) * rD;
  }
}

// Taylor series of G = -g[0,U,W] for g = exp(-i t) in full units, |U|,|W| <= 1:
//   G      = sum_n (-i)^n h_n(U,W)   / (n+2)!
//   dG/dU  = -i sum_n (-i)^n h_n(U,U,W) / (n+3)!
//   dG/dW  = -i sum_n (-i)^n h_n(U,W,W) / (n+3)!
template <bool kGrad>
DM_HD void g_series(float U, float W, c32& G, c32& Gu, c32& Gw) {
  // 1/(n+2)! and 1/(n+3)! for n = 0..9
  const float f2[10] = {1.0f / 2, 1.0f / 6, 1.0f / 24, 1.0f / 120, 1.0f / 720, 1.0f / 5040,
                        1.0f / 40320, 1.0f / 362880, 1.0f / 3628800, 1.0f / 39916800};
  const float f3[10] = {1.0f / 6, 1.0f / 24, 1.0f / 120, 1.0f / 720, 1.0f / 5040, 1.0f / 40320,
                        1.0f / 362880, 1.0f / 3628800, 1.0f / 39916800, 1.0f / 479001600};
  float A = 1.0f, B = 1.0f, C = 1.0f, wp = 1.0f;
  float gr = 0.f, gi = 0.f, ur = 0.f, ui = 0.f, vr = 0.f, vi = 0.f;
#pragma unroll
  for (int n = 0; n < 10; ++n) {
    if (n > 0) {
      wp *= W;
      A = U * A + wp;          // h_n(U,W)
      B = U * B + A;           // h_n(U,U,W)
      C = W * C + A;           // h_n(U,W,W)
    }
    const float a = A * f2[n];
    switch (n & 3) {  // (-i)^n = 1, -i, -1, i
      case 0: gr += a; break;
      case 1: gi -= a; break;
      case 2: gr -= a; break;
      default: gi += a; break;
    }
    if (kGrad) {
      // -i (-i)^n = (-i)^{n+1}
      const float b = B * f3[n], c = C * f3[n];
      switch (n & 3) {
        case 0: ui -= b; vi -= c; break;   // -i
        case 1: ur -= b; vr -= c; break;   // -1
        case 2: ui += b; vi += c; break;   // i
        default: ur += b; vr += c; break;  // 1
      }
    }
  }
  G = c32{gr, gi};
  if (kGrad) {
    Gu = c32{ur, ui};
    Gw = c32{vr, vi};
  }
}

// Phase differences of a face at a frequency, in half units.
DM_HD void half_diffs(const float mf[3], const FaceGeom& g, float& hab, float& hbc, float& hca) {
  hab = mf[0] * g.hab[0] + mf[1] * g.hab[1] + mf[2] * g.hab[2];
  hbc = mf[0] * g.hbc[0] + mf[1] * g.hbc[1] + mf[2] * g.hbc[2];
  hca = -(hab + hbc);
}

// Fast path: generic branch (no difference within Seps, largest difference >= 1).
// Returns true when the pair needs the general evaluator instead (outputs are
// then meaningless).  On the fast path: E = exp(-i x_p), G and, if kGrad, dG/dU,
// dG/dW; piv = 0/1/2 for pivot a/b/c.
template <bool kGrad>
DM_HD bool pair_fast(const XiVal& xv, const FaceGeom& g, c32& E, c32& G, c32& Gu, c32& Gw,
                     int& piv) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  const float aab = fabsf(hab), abc = fabsf(hbc), aca = fabsf(hca);
  const float mn = fminf(aab, fminf(abc, aca));
  const float mx = fmaxf(aab, fmaxf(abc, aca));
  const bool special = (mn <= kSepsHalf) || (mx < kSeriesHalf);
  const bool pa = (abc >= aca) && (abc >= aab);
  const bool pb = !pa && (aca >= aab);
  piv = pa ? 0 : (pb ? 1 : 2);
  const float hu = pa ? hab : (pb ? hbc : hca);
  const float hw = pa ? -hca : (pb ? -hab : -hbc);
  const uint32_t P0 = pa ? g.Ua[0] : (pb ? g.Ub[0] : g.Uc[0]);
  const uint32_t P1 = pa ? g.Ua[1] : (pb ? g.Ub[1] : g.Uc[1]);
  const uint32_t P2 = pa ? g.Ua[2] : (pb ? g.Ub[2] : g.Uc[2]);
  const float th = turns_to_angle(fixed_phase(xv.mi, P0, P1, P2));
  float s, c;
  sincos_fast(th, &s, &c);
  E = c32{c, -s};
  g_sinc<kGrad>(hu, hw, G, Gu, Gw);
  return special;
}

// General evaluator for any configuration, following the reference's branch
// selection.  Returns F and the three partials dF/dx_a, dF/dx_b, dF/dx_c.
template <bool kGrad>
DM_HD_NOINLINE void pair_general(const XiVal& xv, const FaceGeom& g, c32& F, c32* dF) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  const float aab = fabsf(hab), abc = fabsf(hbc), aca = fabsf(hca);
  const bool sab = aab <= kSepsHalf, sbc = abc <= kSepsHalf, sca = aca <= kSepsHalf;
  const bool r1 = (sab && sbc) || (sbc && sca) || (sca && sab);
  int base;       // vertex whose fixed-point phase anchors E
  float delta;    // extra phase (full units) added to that vertex
  int mode;       // 0: R1, 1: R2, 2: R3, 3: R4, 4: R5
  float U = 0.f, W = 0.f;
  int piv = 0;
  if (r1) {
    mode = 0; base = 0; delta = (2.0f * hab - 2.0f * hca) * (1.0f / 3.0f);
  } else if (sab) {
    mode = 1; base = 0; delta = hab; W = -2.0f * hca - hab;      // x_c - (x_a+x_b)/2
  } else if (sbc) {
    mode = 2; base = 1; delta = hbc; W = -2.0f * hab - hbc;      // x_a - (x_b+x_c)/2
  } else if (sca) {
    mode = 3; base = 2; delta = hca; W = -2.0f * hbc - hca;      // x_b - (x_c+x_a)/2
  } else {
    mode = 4; delta = 0.f;
    const bool pa = (abc >= aca) && (abc >= aab);
    const bool pb = !pa && (aca >= aab);
    piv = pa ? 0 : (pb ? 1 : 2);
    base = piv;
    U = 2.0f * (pa ? hab : (pb ? hbc : hca));
    W = 2.0f * (pa ? -hca : (pb ? -hab : -hbc));
  }
  const uint32_t* Ub = base == 0 ? g.Ua : (base == 1 ? g.Ub : g.Uc);
  const float th = turns_to_angle(fixed_phase(xv.mi, Ub[0], Ub[1], Ub[2])) + delta;
  float s, c;
  sincos_fast(th, &s, &c);
  const c32 E{c, -s};
  c32 G, Gu{0.f, 0.f}, Gw{0.f, 0.f};
  if (mode == 0) {
    G = c32{0.5f, 0.f};
  } else if (fabsf(W - U) < 2.0f * kSeriesHalf) {
    g_series<kGrad>(U, W, G, Gu, Gw);
  } else {
    g_sinc<kGrad>(0.5f * U, 0.5f * W, G, Gu, Gw);
  }
  F = cmul(E, G);
  if (!kGrad) return;
  const c32 miF{F.y, -F.x};  // -i F
  if (mode == 0) {
    const c32 t{miF.x * (1.0f / 3.0f), miF.y * (1.0f / 3.0f)};
    dF[0] = t; dF[1] = t; dF[2] = t;
    return;
  }
  const c32 EGw = cmul(E, Gw);
  if (mode == 4) {
    const c32 EGu = cmul(E, Gu);
    const c32 dp{miF.x - EGu.x - EGw.x, miF.y - EGu.y - EGw.y};
    const int q = piv == 2 ? 0 : piv + 1;
    const int r = q == 2 ? 0 : q + 1;
    dF[piv] = dp; dF[q] = EGu; dF[r] = EGw;
    return;
  }
  // merged pair: the lone vertex o gets E dG/dW, each merged vertex half the rest
  const c32 half{0.5f * (miF.x - EGw.x), 0.5f * (miF.y - EGw.y)};
  const int o = mode == 1 ? 2 : (mode == 2 ? 0 : 1);
  for (int v = 0; v < 3; ++v) dF[v] = (v == o) ? EGw : half;
}

}  // namespace dm
