// Host build of the kernel pair math (deltamic_b200/csrc/pair_math.cuh) for CPU
// tests: the same per-pair functions the CUDA kernels call (pair_forward,
// pair_adjoint and their degenerate-branch variants), with libm sin/cos in place
// of the MUFU approximations.  Built by tests/test_pairmath_host.py with g++.
#include <cmath>
#include <cstdint>

#include "../deltamic_b200/csrc/pair_math.cuh"

using namespace dm;

static FaceGeom make_geom(const double* va, const double* vb, const double* vc,
                          const double* lo, const double* len) {
  FaceGeom g;
  const double* v[3] = {va, vb, vc};
  uint32_t* U[3] = {g.Ua, g.Ub, g.Uc};
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < 3; ++d) {
      double t = (v[k][d] - lo[d]) / len[d] * 2147483648.0;
      U[k][d] = (uint32_t)(int64_t)std::llrint(t);
    }
  for (int d = 0; d < 3; ++d) {
    double s = M_PI / (2.0 * len[d]);
    g.hab[d] = (float)((vb[d] - va[d]) * s);
    g.hbc[d] = (float)((vc[d] - vb[d]) * s);
  }
  return g;
}

extern "C" {

// For each (frequency i, face k): F (forward path), z[3] = Re(conj(g_i) dF/dx_v)
// and r = Re(conj(g_i) F) (adjoint path), and the pair class (0 series, 1 pivot,
// 2 degenerate).  verts[nv*3] double, faces[nt*3] int64, m[nxi*3] int32,
// g[nxi*2] float (re, im); outputs sized nxi*nt (F: *2, z: *3).
void dm_host_pairs(const double* verts, const int64_t* faces, int64_t nt, const int32_t* m,
                   int64_t nxi, const float* gc, const double* lo, const double* len, float* F,
                   float* z, float* r, uint8_t* cls) {
  for (int64_t k = 0; k < nt; ++k) {
    const FaceGeom g = make_geom(verts + 3 * faces[3 * k], verts + 3 * faces[3 * k + 1],
                                 verts + 3 * faces[3 * k + 2], lo, len);
    for (int64_t i = 0; i < nxi; ++i) {
      XiVal xv;
      for (int d = 0; d < 3; ++d) {
        xv.mi[d] = m[3 * i + d];
        xv.mf[d] = (float)m[3 * i + d];
      }
      const int64_t o = i * nt + k;
      float hab, hbc, hca;
      half_diffs(xv.mf, g, hab, hbc, hca);
      cls[o] = (uint8_t)pair_class(hab, hbc, hca);
      c32 Fv;
      if (!pair_forward(xv, g, Fv)) Fv = pair_forward_degenerate(xv, g);
      F[2 * o] = Fv.x;
      F[2 * o + 1] = Fv.y;
      float zz[3], rr;
      if (!pair_adjoint(xv, g, gc[2 * i], gc[2 * i + 1], zz, rr))
        pair_adjoint_degenerate(xv, g, gc[2 * i], gc[2 * i + 1], zz, rr);
      for (int v = 0; v < 3; ++v) z[3 * o + v] = zz[v];
      r[o] = rr;
    }
  }
}

// The same outputs for frequencies off the grid (explicit xi list): the cell has
// lower corner 0 and lengths len[3] (the device takes 2.5 max|v_d|), each xi
// becomes m = xi L / pi split into its nearest integer and the remainder, as the
// list kernels' record builder does.  xi[nxi*3] double.
void dm_host_pairs_off(const double* verts, const int64_t* faces, int64_t nt, const double* xi,
                       int64_t nxi, const float* gc, const double* len, float* F, float* z,
                       float* r, uint8_t* cls) {
  const double lo[3] = {0.0, 0.0, 0.0};
  for (int64_t k = 0; k < nt; ++k) {
    const FaceGeom g = make_geom(verts + 3 * faces[3 * k], verts + 3 * faces[3 * k + 1],
                                 verts + 3 * faces[3 * k + 2], lo, len);
    for (int64_t i = 0; i < nxi; ++i) {
      XiValOff xv;
      for (int d = 0; d < 3; ++d) {
        const double m = xi[3 * i + d] * len[d] / M_PI;
        const double mi = std::rint(m);
        xv.mi[d] = (int32_t)mi;
        xv.mf[d] = (float)m;
        xv.fr[d] = (float)(m - mi);
      }
      const int64_t o = i * nt + k;
      float hab, hbc, hca;
      half_diffs(xv.mf, g, hab, hbc, hca);
      cls[o] = (uint8_t)pair_class(hab, hbc, hca);
      c32 Fv;
      if (!pair_forward(xv, g, Fv)) Fv = pair_forward_degenerate(xv, g);
      F[2 * o] = Fv.x;
      F[2 * o + 1] = Fv.y;
      float zz[3], rr;
      if (!pair_adjoint(xv, g, gc[2 * i], gc[2 * i + 1], zz, rr))
        pair_adjoint_degenerate(xv, g, gc[2 * i], gc[2 * i + 1], zz, rr);
      for (int v = 0; v < 3; ++v) z[3 * o + v] = zz[v];
      r[o] = rr;
    }
  }
}

// Packed two-pair series path against the scalar one: for faces (2j, 2j+1) at
// each grid frequency (adjoint_series2) and for frequencies (2i, 2i+1) at each
// face (forward_series2), where both pairs are series pairs; other entries are
// left untouched (the caller fills them with the scalar results).
void dm_host_series2(const double* verts, const int64_t* faces, int64_t nt, const int32_t* m,
                     int64_t nxi, const float* gc, const double* lo, const double* len, float* z,
                     float* r, float* F) {
  for (int64_t i = 0; i < nxi; ++i) {
    XiVal xv;
    for (int d = 0; d < 3; ++d) {
      xv.mi[d] = m[3 * i + d];
      xv.mf[d] = (float)m[3 * i + d];
    }
    for (int64_t k = 0; k + 1 < nt; k += 2) {
      const FaceGeom g0 = make_geom(verts + 3 * faces[3 * k], verts + 3 * faces[3 * k + 1],
                                    verts + 3 * faces[3 * k + 2], lo, len);
      const FaceGeom g1 = make_geom(verts + 3 * faces[3 * k + 3], verts + 3 * faces[3 * k + 4],
                                    verts + 3 * faces[3 * k + 5], lo, len);
      float a0, b0, c0, a1, b1, c1;
      half_diffs(xv.mf, g0, a0, b0, c0);
      half_diffs(xv.mf, g1, a1, b1, c1);
      const v2 hab{a0, a1}, hbc{b0, b1}, hca{c0, c1};
      if (!series_pair2(hab, hbc, hca)) continue;
      v2 zz[3], rr;
      if (series_short2(hab, hbc, hca))
        adjoint_series2<true>(xv, g0.Ua, g1.Ua, hab, hca, gc[2 * i], gc[2 * i + 1], zz, rr);
      else
        adjoint_series2<false>(xv, g0.Ua, g1.Ua, hab, hca, gc[2 * i], gc[2 * i + 1], zz, rr);
      const int64_t o0 = i * nt + k, o1 = o0 + 1;
      for (int v = 0; v < 3; ++v) {
        z[3 * o0 + v] = zz[v].x;
        z[3 * o1 + v] = zz[v].y;
      }
      r[o0] = rr.x;
      r[o1] = rr.y;
    }
  }
  for (int64_t k = 0; k < nt; ++k) {
    const FaceGeom g = make_geom(verts + 3 * faces[3 * k], verts + 3 * faces[3 * k + 1],
                                 verts + 3 * faces[3 * k + 2], lo, len);
    for (int64_t i = 0; i + 1 < nxi; i += 2) {
      XiVal x0, x1;
      for (int d = 0; d < 3; ++d) {
        x0.mi[d] = m[3 * i + d];
        x0.mf[d] = (float)m[3 * i + d];
        x1.mi[d] = m[3 * i + 3 + d];
        x1.mf[d] = (float)m[3 * i + 3 + d];
      }
      float a0, b0, c0, a1, b1, c1;
      half_diffs(x0.mf, g, a0, b0, c0);
      half_diffs(x1.mf, g, a1, b1, c1);
      const v2 hab{a0, a1}, hbc{b0, b1}, hca{c0, c1};
      if (!series_pair2(hab, hbc, hca)) continue;
      v2 Fx, Fy;
      if (series_short2(hab, hbc, hca))
        forward_series2<true>(x0, x1, g.Ua, hab, hca, Fx, Fy);
      else
        forward_series2<false>(x0, x1, g.Ua, hab, hca, Fx, Fy);
      const int64_t o0 = i * nt + k, o1 = (i + 1) * nt + k;
      F[2 * o0] = Fx.x;
      F[2 * o0 + 1] = Fy.x;
      F[2 * o1] = Fx.y;
      F[2 * o1 + 1] = Fy.y;
    }
  }
}

}  // extern "C"
