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
//  * when the largest difference is below 3.5 the term is expanded about the
//    centroid: F = e^{-i x_g} H(p2, p3) with d_v = x_v - x_g, p2 = sum d^2,
//    p3 = sum d^3 and H = sum_n (-i)^n h_n(d)/(n+2)! (h_n complete homogeneous
//    symmetric polynomials, reduced by the Newton identities to a polynomial in
//    p2, p3; coefficients in series_coeffs.cuh), exact to < 1e-8 there;
//  * the reference's branch selection (R1..R4 at Seps = sqrt(FLT_EPSILON)) is
//    kept: in those branches the phases are merged exactly as the reference
//    does (centroid, or midpoint of the close pair) and the same evaluators run.
//
// The header compiles for the host too (libm sin/cos instead of the MUFU
// approximations) so the math can be checked on a machine without a GPU.
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#include "series_coeffs.cuh"

#if defined(__CUDACC__)
#define DM_HD __host__ __device__ __forceinline__
#else
#define DM_HD static inline
#endif

namespace dm {

// Seps/2: the reference compares |ab| <= sqrt(FLT_EPSILON); differences here are
// held in half units.
constexpr float kSepsHalf = 1.72633492e-4f;
// Centroid series when the largest difference is below 3.5 (half units: 1.75);
// its short coefficient set when it is at most 1.5 (half units: 0.75).
constexpr float kSeriesHalf = 1.75f;
constexpr float kSeriesLoHalf = 0.75f;
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

// A frequency off the grid (an explicit xi list): m_d = xi_d L_d / pi is real,
// split into its nearest integer mi_d and the remainder fr_d (|fr_d| <= 1/2);
// mf_d = m_d as a float (for the phase differences).
struct XiValOff {
  int32_t mi[3];
  float mf[3];
  float fr[3];
};

DM_HD uint32_t fixed_phase(const int32_t mi[3], uint32_t U0, uint32_t U1, uint32_t U2) {
  return (uint32_t)mi[0] * U0 + (uint32_t)mi[1] * U1 + (uint32_t)mi[2] * U2;
}

DM_HD int32_t round_to_int(float x) {
#if defined(__CUDA_ARCH__)
  return __float2int_rn(x);
#else
  return (int32_t)lrintf(x);
#endif
}

// Vertex phase as an angle in [-pi, pi).  On the grid the phase in turns is
// sum_d mi_d U_d / 2^32 (mod 1), exact in uint32.  Off the grid (split phase)
// the remainder adds sum_d fr_d U_d / 2^32 turns, with U_d read as signed (the
// off-grid cell has lower corner 0 and |v_d| < L_d / 2, so |U_d| < 2^30): that
// term is below 3/8 of a turn and is formed in float, rounded back to 2^-32-turn
// units and added in uint32 before the turns become an angle.
DM_HD float vertex_angle(const XiVal& xv, uint32_t U0, uint32_t U1, uint32_t U2) {
  return turns_to_angle(fixed_phase(xv.mi, U0, U1, U2));
}
DM_HD float vertex_angle(const XiValOff& xv, uint32_t U0, uint32_t U1, uint32_t U2) {
  const float c = xv.fr[0] * (float)(int32_t)U0 + xv.fr[1] * (float)(int32_t)U1 +
                  xv.fr[2] * (float)(int32_t)U2;
  return turns_to_angle(fixed_phase(xv.mi, U0, U1, U2) + (uint32_t)round_to_int(c));
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

// ---------------------------------------------------------------------------
// Centroid series: H(p2, p3) and its partials in p2 and p3.

// First N coefficients of c (ascending) at x, and the derivative; N == 0 gives 0.
template <int N>
DM_HD void horner(const float* c, float x, float& v, float& dv) {
  if constexpr (N == 0) {
    v = 0.f;
    dv = 0.f;
  } else {
    v = c[N - 1];
    dv = 0.f;
#pragma unroll
    for (int k = N - 2; k >= 0; --k) {
      dv = dv * x + v;
      v = v * x + c[k];
    }
  }
}

// H = P0 + p3^2 P2 + p3^4 P4 + i p3 (Q1 + p3^2 Q3) (polynomials in p2) and, if
// kGrad, its partials in p2 and p3; parts of length 0 are left out.
template <bool kGrad, int N0, int N2, int N4, int M1, int M3>
DM_HD void centroid_H_set(const float* P0, const float* P2, const float* P4, const float* Q1,
                          const float* Q3, float p2, float p3, c32& H, c32& Hp2, c32& Hp3) {
  float a0, a0d, a2, a2d, a4, a4d, b1, b1d, b3, b3d;
  horner<N0>(P0, p2, a0, a0d);
  horner<N2>(P2, p2, a2, a2d);
  horner<N4>(P4, p2, a4, a4d);
  horner<M1>(Q1, p2, b1, b1d);
  horner<M3>(Q3, p2, b3, b3d);
  const float q = p3 * p3;
  if constexpr (N4 > 0) {
    H.x = a0 + q * (a2 + q * a4);
  } else {
    H.x = a0 + q * a2;
  }
  if constexpr (M3 > 0) {
    H.y = p3 * (b1 + q * b3);
  } else {
    H.y = p3 * b1;
  }
  if (kGrad) {
    if constexpr (N4 > 0) {
      Hp2.x = a0d + q * (a2d + q * a4d);
      Hp3.x = p3 * (2.0f * a2 + 4.0f * q * a4);
    } else {
      Hp2.x = a0d + q * a2d;
      Hp3.x = p3 * (2.0f * a2);
    }
    if constexpr (M3 > 0) {
      Hp2.y = p3 * (b1d + q * b3d);
      Hp3.y = b1 + 3.0f * q * b3;
    } else {
      Hp2.y = p3 * b1d;
      Hp3.y = b1;
    }
  }
}

// The whole series domain (kLo false: largest phase difference below 3.5), or the
// short set for largest differences up to 1.5 (same truncation error there).
template <bool kGrad, bool kLo = false>
DM_HD void centroid_H(float p2, float p3, c32& H, c32& Hp2, c32& Hp3) {
  if constexpr (kLo) {
    constexpr float P0[] = DM_SERIES_LO_P0;
    constexpr float P2[] = DM_SERIES_LO_P2;
    constexpr float P4[] = DM_SERIES_LO_P4;
    constexpr float Q1[] = DM_SERIES_LO_Q1;
    constexpr float Q3[] = DM_SERIES_LO_Q3;
    centroid_H_set<kGrad, DM_SERIES_LO_P0_N, DM_SERIES_LO_P2_N, DM_SERIES_LO_P4_N,
                   DM_SERIES_LO_Q1_N, DM_SERIES_LO_Q3_N>(P0, P2, P4, Q1, Q3, p2, p3, H, Hp2, Hp3);
  } else {
    constexpr float P0[] = DM_SERIES_P0;
    constexpr float P2[] = DM_SERIES_P2;
    constexpr float P4[] = DM_SERIES_P4;
    constexpr float Q1[] = DM_SERIES_Q1;
    constexpr float Q3[] = DM_SERIES_Q3;
    centroid_H_set<kGrad, DM_SERIES_P0_N, DM_SERIES_P2_N, DM_SERIES_P4_N, DM_SERIES_Q1_N,
                   DM_SERIES_Q3_N>(P0, P2, P4, Q1, Q3, p2, p3, H, Hp2, Hp3);
  }
}

// Phase differences of a face at a frequency, in half units.
DM_HD void half_diffs(const float mf[3], const FaceGeom& g, float& hab, float& hbc, float& hca) {
  hab = mf[0] * g.hab[0] + mf[1] * g.hab[1] + mf[2] * g.hab[2];
  hbc = mf[0] * g.hbc[0] + mf[1] * g.hbc[1] + mf[2] * g.hbc[2];
  hca = -(hab + hbc);
}

DM_HD c32 expmi(float angle) {
  float s, c;
  sincos_fast(angle, &s, &c);
  return c32{c, -s};
}

// Centroid path.  Vertex phases x'_v = x_v + off[v] with half differences
// (hab, hbc, hca) of the x'.  Outputs E = exp(-i x'_g), H and, if kGrad, the
// centroid deviations d[3] and the partials Hp2, Hp3; F = E H.
template <bool kGrad, bool kLo = false, class XV>
DM_HD void eval_series(const XV& xv, const FaceGeom& g, float hab, float hca, float off_a,
                       c32& E, c32& H, c32& Hp2, c32& Hp3, float d[3], float& p2) {
  // d_a = (ca - ab) / 3, d_b = d_a + ab, d_c = d_a - ca for the full differences
  // ab = 2 hab, ca = 2 hca (the doubling is exact, so these are the same floats)
  const float da = (hca - hab) * (2.0f / 3.0f);
  const float db = fmaf(2.0f, hab, da);
  const float dc = fmaf(-2.0f, hca, da);
  p2 = da * da + db * db + dc * dc;
  const float p3 = 3.0f * da * db * dc;  // sum d^3 when sum d = 0
  E = expmi(vertex_angle(xv, g.Ua[0], g.Ua[1], g.Ua[2]) + (off_a - da));
  centroid_H<kGrad, kLo>(p2, p3, H, Hp2, Hp3);
  d[0] = da;
  d[1] = db;
  d[2] = dc;
}

// Pivot path (largest difference >= 3.5).  Outputs E = exp(-i x'_p), G and, if
// kGrad, dG/dU and dG/dW; F = E G; piv = 0/1/2 for pivot a/b/c.
template <bool kGrad, class XV>
DM_HD void eval_pivot(const XV& xv, const FaceGeom& g, float hab, float hbc, float hca,
                      const float off[3], c32& E, c32& G, c32& Gu, c32& Gw, int& piv) {
  const float aab = fabsf(hab), abc = fabsf(hbc), aca = fabsf(hca);
  const bool pa = (abc >= aca) && (abc >= aab);
  const bool pb = !pa && (aca >= aab);
  piv = pa ? 0 : (pb ? 1 : 2);
  const float hu = pa ? hab : (pb ? hbc : hca);
  const float hw = pa ? -hca : (pb ? -hab : -hbc);
  const uint32_t P0 = pa ? g.Ua[0] : (pb ? g.Ub[0] : g.Uc[0]);
  const uint32_t P1 = pa ? g.Ua[1] : (pb ? g.Ub[1] : g.Uc[1]);
  const uint32_t P2 = pa ? g.Ua[2] : (pb ? g.Ub[2] : g.Uc[2]);
  const float o = pa ? off[0] : (pb ? off[1] : off[2]);
  E = expmi(vertex_angle(xv, P0, P1, P2) + o);
  g_sinc<kGrad>(hu, hw, G, Gu, Gw);
}

// F and dF/dx_{a,b,c} for vertex phases x_v + off[v] (no degenerate branch).
template <bool kGrad, class XV>
DM_HD void eval_any(const XV& xv, const FaceGeom& g, float hab, float hbc, float hca,
                    const float off[3], c32& F, c32* dF) {
  const float amax = fmaxf(fabsf(hab), fmaxf(fabsf(hbc), fabsf(hca)));
  if (amax < kSeriesHalf) {
    c32 E, H, Hp2, Hp3;
    float d[3], p2;
    eval_series<kGrad>(xv, g, hab, hca, off[0], E, H, Hp2, Hp3, d, p2);
    F = cmul(E, H);
    if (kGrad) {
      const c32 EHp2 = cmul(E, Hp2), EHp3 = cmul(E, Hp3);
      for (int v = 0; v < 3; ++v) {
        const float a = 2.0f * d[v], b = 3.0f * d[v] * d[v] - p2;
        dF[v] = c32{F.y * (1.0f / 3.0f) + a * EHp2.x + b * EHp3.x,
                    -F.x * (1.0f / 3.0f) + a * EHp2.y + b * EHp3.y};
      }
    }
  } else {
    c32 E, G, Gu, Gw;
    int piv;
    eval_pivot<kGrad>(xv, g, hab, hbc, hca, off, E, G, Gu, Gw, piv);
    F = cmul(E, G);
    if (kGrad) {
      const c32 EGu = cmul(E, Gu), EGw = cmul(E, Gw);
      const int q = piv == 2 ? 0 : piv + 1;
      const int r = q == 2 ? 0 : q + 1;
      dF[piv] = c32{F.y - EGu.x - EGw.x, -F.x - EGu.y - EGw.y};
      dF[q] = EGu;
      dF[r] = EGw;
    }
  }
}

// Degenerate frequencies of the reference (a phase difference within Seps):
// R1 collapses the three phases to their centroid, R2/R3/R4 merge the close pair
// at its midpoint (fourier3d_cuda_kernel.cu:250-271, render.py:77-102); the
// merged vertices share the derivative of the merged phase equally.
template <bool kGrad, class XV>
DM_HD void pair_degenerate(const XV& xv, const FaceGeom& g, float hab, float hbc, float hca,
                           c32& F, c32* dF) {
  const bool sab = fabsf(hab) <= kSepsHalf, sbc = fabsf(hbc) <= kSepsHalf,
             sca = fabsf(hca) <= kSepsHalf;
  const bool r1 = (sab && sbc) || (sbc && sca) || (sca && sab);
  float off[3] = {0.f, 0.f, 0.f};
  int mode;
  if (r1) {
    mode = 0;
    off[0] = (2.0f * hab - 2.0f * hca) * (1.0f / 3.0f);
    off[1] = off[0] - 2.0f * hab;
    off[2] = off[0] + 2.0f * hca;
    hab = hbc = hca = 0.f;
  } else if (sab) {
    mode = 1;
    off[0] = hab;
    off[1] = -hab;
    hbc += 0.5f * hab;
    hca += 0.5f * hab;
    hab = 0.f;
  } else if (sbc) {
    mode = 2;
    off[1] = hbc;
    off[2] = -hbc;
    hab += 0.5f * hbc;
    hca += 0.5f * hbc;
    hbc = 0.f;
  } else {
    mode = 3;
    off[2] = hca;
    off[0] = -hca;
    hab += 0.5f * hca;
    hbc += 0.5f * hca;
    hca = 0.f;
  }
  c32 d3[3];
  eval_any<kGrad>(xv, g, hab, hbc, hca, off, F, d3);
  if (!kGrad) return;
  if (mode == 0) {
    const c32 m{(d3[0].x + d3[1].x + d3[2].x) * (1.0f / 3.0f),
                (d3[0].y + d3[1].y + d3[2].y) * (1.0f / 3.0f)};
    dF[0] = m; dF[1] = m; dF[2] = m;
    return;
  }
  // merged pair (i, j), lone vertex o
  const int i = mode == 1 ? 0 : (mode == 2 ? 1 : 2);
  const int j = i == 2 ? 0 : i + 1;
  const int o = j == 2 ? 0 : j + 1;
  const c32 m{0.5f * (d3[i].x + d3[j].x), 0.5f * (d3[i].y + d3[j].y)};
  dF[i] = m;
  dF[j] = m;
  dF[o] = d3[o];
}

// Classification shared by the kernels: 0 = centroid series, 1 = pivot,
// 2 = reference-degenerate branch.
DM_HD int pair_class(float hab, float hbc, float hca) {
  const float aab = fabsf(hab), abc = fabsf(hbc), aca = fabsf(hca);
  const float mn = fminf(aab, fminf(abc, aca));
  const float mx = fmaxf(aab, fmaxf(abc, aca));
  return mn <= kSepsHalf ? 2 : (mx < kSeriesHalf ? 0 : 1);
}

// Any pair: F and (if kGrad) dF/dx_{a,b,c}.
template <bool kGrad, class XV>
DM_HD void pair_general(const XV& xv, const FaceGeom& g, c32& F, c32* dF) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  if (pair_class(hab, hbc, hca) == 2) {
    pair_degenerate<kGrad>(xv, g, hab, hbc, hca, F, dF);
  } else {
    const float off[3] = {0.f, 0.f, 0.f};
    eval_any<kGrad>(xv, g, hab, hbc, hca, off, F, dF);
  }
}

// Short series set for a pair whose largest half difference is at most
// kSeriesLoHalf.  On the GPU the choice is made for the converged lanes of the
// warp together (short set only if every one of them qualifies), so a warp does
// not run both sets.
DM_HD bool series_short(float hab, float hbc, float hca) {
  const bool lo = fmaxf(fabsf(hab), fmaxf(fabsf(hbc), fabsf(hca))) <= kSeriesLoHalf;
#if defined(__CUDA_ARCH__)
  return __all_sync(__activemask(), lo);
#else
  return lo;
#endif
}

// ---------------------------------------------------------------------------
// Per-pair work of the kernels (shared with the host test build).

// Forward: F on the series / pivot paths; returns false for a degenerate pair
// (F then undefined: the caller runs pair_degenerate for it).
template <class XV>
DM_HD bool pair_forward(const XV& xv, const FaceGeom& g, c32& F) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  const int cls = pair_class(hab, hbc, hca);
  if (cls == 2) return false;
  const float off[3] = {0.f, 0.f, 0.f};
  if (cls == 0) {
    c32 E, H, Hp2, Hp3;
    float d[3], p2;
    if (series_short(hab, hbc, hca))
      eval_series<false, true>(xv, g, hab, hca, 0.f, E, H, Hp2, Hp3, d, p2);
    else
      eval_series<false, false>(xv, g, hab, hca, 0.f, E, H, Hp2, Hp3, d, p2);
    F = cmul(E, H);
  } else {
    c32 E, G, Gu, Gw;
    int piv;
    eval_pivot<false>(xv, g, hab, hbc, hca, off, E, G, Gu, Gw, piv);
    F = cmul(E, G);
  }
  return true;
}

// Adjoint: z_v = Re(conj(g) dF/dx_v) and r = Re(conj(g) F) for cotangent g, and
// F itself if kF; returns false for a degenerate pair (outputs undefined).
template <bool kF, class XV>
DM_HD bool pair_adjoint_t(const XV& xv, const FaceGeom& g, float gre, float gim, float z[3],
                          float& r, c32& Fo) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  const int cls = pair_class(hab, hbc, hca);
  if (cls == 2) return false;
  if (cls == 0) {
    c32 E, H, Hp2, Hp3;
    float d[3], p2;
    if (series_short(hab, hbc, hca))
      eval_series<true, true>(xv, g, hab, hca, 0.f, E, H, Hp2, Hp3, d, p2);
    else
      eval_series<true, false>(xv, g, hab, hca, 0.f, E, H, Hp2, Hp3, d, p2);
    const float hx = gre * E.x + gim * E.y;  // h = conj(g) E
    const float hy = gre * E.y - gim * E.x;
    r = hx * H.x - hy * H.y;
    if (kF) Fo = cmul(E, H);
    const float zt3 = hx * H.y + hy * H.x;  // z_a + z_b + z_c (sum d = 0)
    const float zt = zt3 * (1.0f / 3.0f);
    const float r1 = 2.0f * (hx * Hp2.x - hy * Hp2.y);
    const float r2 = hx * Hp3.x - hy * Hp3.y;
    z[0] = zt + r1 * d[0] + r2 * (3.0f * d[0] * d[0] - p2);
    z[1] = zt + r1 * d[1] + r2 * (3.0f * d[1] * d[1] - p2);
    z[2] = (zt3 - z[0]) - z[1];
  } else {
    const float off[3] = {0.f, 0.f, 0.f};
    c32 E, G, Gu, Gw;
    int piv;
    eval_pivot<true>(xv, g, hab, hbc, hca, off, E, G, Gu, Gw, piv);
    const float hx = gre * E.x + gim * E.y;
    const float hy = gre * E.y - gim * E.x;
    r = hx * G.x - hy * G.y;
    if (kF) Fo = cmul(E, G);
    const float zt = hx * G.y + hy * G.x;  // Re(conj(g) (-i F))
    const float zu = hx * Gu.x - hy * Gu.y;
    const float zw = hx * Gw.x - hy * Gw.y;
    const float zp = zt - zu - zw;
    z[0] = piv == 0 ? zp : (piv == 1 ? zw : zu);
    z[1] = piv == 0 ? zu : (piv == 1 ? zp : zw);
    z[2] = piv == 0 ? zw : (piv == 1 ? zu : zp);
  }
  return true;
}

template <class XV>
DM_HD bool pair_adjoint(const XV& xv, const FaceGeom& g, float gre, float gim, float z[3],
                        float& r) {
  c32 unused;
  return pair_adjoint_t<false>(xv, g, gre, gim, z, r, unused);
}

// Adjoint of a degenerate pair (F returned as well).
template <class XV>
DM_HD void pair_adjoint_degenerate(const XV& xv, const FaceGeom& g, float gre, float gim,
                                   float z[3], float& r, c32& F) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  c32 dF[3];
  pair_degenerate<true>(xv, g, hab, hbc, hca, F, dF);
  r = gre * F.x + gim * F.y;
  for (int v = 0; v < 3; ++v) z[v] = gre * dF[v].x + gim * dF[v].y;
}
template <class XV>
DM_HD void pair_adjoint_degenerate(const XV& xv, const FaceGeom& g, float gre, float gim,
                                   float z[3], float& r) {
  c32 F;
  pair_adjoint_degenerate(xv, g, gre, gim, z, r, F);
}

// Forward of a degenerate pair.
template <class XV>
DM_HD c32 pair_forward_degenerate(const XV& xv, const FaceGeom& g) {
  float hab, hbc, hca;
  half_diffs(xv.mf, g, hab, hbc, hca);
  c32 F;
  pair_degenerate<false>(xv, g, hab, hbc, hca, F, nullptr);
  return F;
}

// ---------------------------------------------------------------------------
// Two pairs per instruction on the centroid-series path.
//
// sm_100 issues paired FP32 instructions (FFMA2 / FMUL2 / FADD2: two lanes' FP32
// operations, one per half of a 64-bit register pair, per instruction).  The
// meshFT kernels are issue-bound, so two pairs that take the series path with the
// same coefficient set -- two faces at one frequency (adjoint), or one face at two
// frequencies (forward) -- run their FP32 arithmetic packed: per component the
// same operations in the same order as the scalar functions above, with the
// integer phase and the MUFU sine / cosine still per pair.

struct v2 {
  float x, y;
};

DM_HD v2 B2(float s) { return v2{s, s}; }
DM_HD v2 neg2(v2 a) { return v2{-a.x, -a.y}; }
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
DM_HD v2 fma2(v2 a, v2 b, v2 c) {
  const float2 r = __ffma2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y), make_float2(c.x, c.y));
  return v2{r.x, r.y};
}
DM_HD v2 mul2(v2 a, v2 b) {
  const float2 r = __fmul2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return v2{r.x, r.y};
}
DM_HD v2 add2(v2 a, v2 b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return v2{r.x, r.y};
}
#else
DM_HD v2 fma2(v2 a, v2 b, v2 c) { return v2{fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y)}; }
DM_HD v2 mul2(v2 a, v2 b) { return v2{a.x * b.x, a.y * b.y}; }
DM_HD v2 add2(v2 a, v2 b) { return v2{a.x + b.x, a.y + b.y}; }
#endif
DM_HD v2 sub2(v2 a, v2 b) { return add2(a, neg2(b)); }

template <int N>
DM_HD void horner2(const float* c, v2 x, v2& v, v2& dv) {
  if constexpr (N == 0) {
    v = B2(0.f);
    dv = B2(0.f);
  } else {
    v = B2(c[N - 1]);
    dv = B2(0.f);
#pragma unroll
    for (int k = N - 2; k >= 0; --k) {
      dv = fma2(dv, x, v);
      v = fma2(v, x, B2(c[k]));
    }
  }
}

// centroid_H_set for two pairs: H = (Hx, Hy) and, if kGrad, its partials.
template <bool kGrad, int N0, int N2, int N4, int M1, int M3>
DM_HD void centroid_H_set2(const float* P0, const float* P2, const float* P4, const float* Q1,
                           const float* Q3, v2 p2, v2 p3, v2& Hx, v2& Hy, v2& Hp2x, v2& Hp2y,
                           v2& Hp3x, v2& Hp3y) {
  v2 a0, a0d, a2, a2d, a4, a4d, b1, b1d, b3, b3d;
  horner2<N0>(P0, p2, a0, a0d);
  horner2<N2>(P2, p2, a2, a2d);
  horner2<N4>(P4, p2, a4, a4d);
  horner2<M1>(Q1, p2, b1, b1d);
  horner2<M3>(Q3, p2, b3, b3d);
  const v2 q = mul2(p3, p3);
  if constexpr (N4 > 0) {
    Hx = fma2(q, fma2(q, a4, a2), a0);
  } else {
    Hx = fma2(q, a2, a0);
  }
  if constexpr (M3 > 0) {
    Hy = mul2(p3, fma2(q, b3, b1));
  } else {
    Hy = mul2(p3, b1);
  }
  if (kGrad) {
    if constexpr (N4 > 0) {
      Hp2x = fma2(q, fma2(q, a4d, a2d), a0d);
      Hp3x = mul2(p3, fma2(mul2(B2(4.0f), q), a4, mul2(B2(2.0f), a2)));
    } else {
      Hp2x = fma2(q, a2d, a0d);
      Hp3x = mul2(p3, mul2(B2(2.0f), a2));
    }
    if constexpr (M3 > 0) {
      Hp2y = mul2(p3, fma2(q, b3d, b1d));
      Hp3y = fma2(mul2(B2(3.0f), q), b3, b1);
    } else {
      Hp2y = mul2(p3, b1d);
      Hp3y = b1;
    }
  }
}

template <bool kGrad, bool kLo>
DM_HD void centroid_H2(v2 p2, v2 p3, v2& Hx, v2& Hy, v2& Hp2x, v2& Hp2y, v2& Hp3x, v2& Hp3y) {
  if constexpr (kLo) {
    constexpr float P0[] = DM_SERIES_LO_P0;
    constexpr float P2[] = DM_SERIES_LO_P2;
    constexpr float P4[] = DM_SERIES_LO_P4;
    constexpr float Q1[] = DM_SERIES_LO_Q1;
    constexpr float Q3[] = DM_SERIES_LO_Q3;
    centroid_H_set2<kGrad, DM_SERIES_LO_P0_N, DM_SERIES_LO_P2_N, DM_SERIES_LO_P4_N,
                    DM_SERIES_LO_Q1_N, DM_SERIES_LO_Q3_N>(P0, P2, P4, Q1, Q3, p2, p3, Hx, Hy,
                                                          Hp2x, Hp2y, Hp3x, Hp3y);
  } else {
    constexpr float P0[] = DM_SERIES_P0;
    constexpr float P2[] = DM_SERIES_P2;
    constexpr float P4[] = DM_SERIES_P4;
    constexpr float Q1[] = DM_SERIES_Q1;
    constexpr float Q3[] = DM_SERIES_Q3;
    centroid_H_set2<kGrad, DM_SERIES_P0_N, DM_SERIES_P2_N, DM_SERIES_P4_N, DM_SERIES_Q1_N,
                    DM_SERIES_Q3_N>(P0, P2, P4, Q1, Q3, p2, p3, Hx, Hy, Hp2x, Hp2y, Hp3x,
                                    Hp3y);
  }
}

// Centroid deviations d_v, p2 and p3 of two pairs from their half differences.
DM_HD void series_dev2(v2 hab, v2 hca, v2 d[3], v2& p2, v2& p3) {
  d[0] = mul2(sub2(hca, hab), B2(2.0f / 3.0f));
  d[1] = fma2(B2(2.0f), hab, d[0]);
  d[2] = fma2(B2(-2.0f), hca, d[0]);
  p2 = fma2(d[2], d[2], fma2(d[1], d[1], mul2(d[0], d[0])));
  p3 = mul2(mul2(B2(3.0f), d[0]), mul2(d[1], d[2]));
}

// Both pairs in the series domain (no degenerate difference, largest below 3.5)?
DM_HD bool series_pair2(v2 hab, v2 hbc, v2 hca) {
  return pair_class(hab.x, hbc.x, hca.x) == 0 && pair_class(hab.y, hbc.y, hca.y) == 0;
}

// Short coefficient set for both pairs (and, on the GPU, every converged lane).
DM_HD bool series_short2(v2 hab, v2 hbc, v2 hca) {
  const float m0 = fmaxf(fabsf(hab.x), fmaxf(fabsf(hbc.x), fabsf(hca.x)));
  const float m1 = fmaxf(fabsf(hab.y), fmaxf(fabsf(hbc.y), fabsf(hca.y)));
  const bool lo = fmaxf(m0, m1) <= kSeriesLoHalf;
#if defined(__CUDA_ARCH__)
  return __all_sync(__activemask(), lo);
#else
  return lo;
#endif
}

// Adjoint of two faces (vertex-a positions Ua0, Ua1) at one frequency on the
// series path: z_v = Re(conj(g) dF/dx_v) and r = Re(conj(g) F), lane x for the
// first face, y for the second (pair_adjoint_t's series branch).
template <bool kLo, class XV>
DM_HD void adjoint_series2(const XV& xv, const uint32_t Ua0[3], const uint32_t Ua1[3], v2 hab,
                           v2 hca, float gre, float gim, v2 z[3], v2& r) {
  v2 d[3], p2, p3;
  series_dev2(hab, hca, d, p2, p3);
  float s0, c0, s1, c1;
  sincos_fast(vertex_angle(xv, Ua0[0], Ua0[1], Ua0[2]) - d[0].x, &s0, &c0);
  sincos_fast(vertex_angle(xv, Ua1[0], Ua1[1], Ua1[2]) - d[0].y, &s1, &c1);
  const v2 Ex{c0, c1}, Ey{-s0, -s1};
  v2 Hx, Hy, Hp2x, Hp2y, Hp3x, Hp3y;
  centroid_H2<true, kLo>(p2, p3, Hx, Hy, Hp2x, Hp2y, Hp3x, Hp3y);
  const v2 hx = fma2(B2(gre), Ex, mul2(B2(gim), Ey));        // h = conj(g) E
  const v2 hy = fma2(B2(gre), Ey, mul2(B2(-gim), Ex));
  r = fma2(hx, Hx, mul2(neg2(hy), Hy));
  const v2 zt3 = fma2(hx, Hy, mul2(hy, Hx));  // z_a + z_b + z_c
  const v2 zt = mul2(zt3, B2(1.0f / 3.0f));
  const v2 r1 = mul2(B2(2.0f), fma2(hx, Hp2x, mul2(neg2(hy), Hp2y)));
  const v2 r2 = fma2(hx, Hp3x, mul2(neg2(hy), Hp3y));
#pragma unroll
  for (int v = 0; v < 2; ++v)
    z[v] = fma2(r2, fma2(mul2(B2(3.0f), d[v]), d[v], neg2(p2)), fma2(r1, d[v], zt));
  z[2] = sub2(sub2(zt3, z[0]), z[1]);
}

// Forward of one face (vertex-a position Ua) at two frequencies on the series
// path: F = (Fx, Fy) per lane (pair_forward's series branch).
template <bool kLo, class XV>
DM_HD void forward_series2(const XV& x0, const XV& x1, const uint32_t Ua[3], v2 hab, v2 hca,
                           v2& Fx, v2& Fy) {
  v2 d[3], p2, p3;
  series_dev2(hab, hca, d, p2, p3);
  float s0, c0, s1, c1;
  sincos_fast(vertex_angle(x0, Ua[0], Ua[1], Ua[2]) - d[0].x, &s0, &c0);
  sincos_fast(vertex_angle(x1, Ua[0], Ua[1], Ua[2]) - d[0].y, &s1, &c1);
  const v2 Ex{c0, c1}, Ey{-s0, -s1};
  v2 Hx, Hy, u0, u1, u2, u3;
  centroid_H2<false, kLo>(p2, p3, Hx, Hy, u0, u1, u2, u3);
  Fx = fma2(Ex, Hx, mul2(neg2(Ey), Hy));
  Fy = fma2(Ex, Hy, mul2(Ey, Hx));
}

}  // namespace dm
