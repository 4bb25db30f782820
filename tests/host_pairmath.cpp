// Host build of the kernel pair math (deltamic_b200/csrc/pair_math.cuh) for CPU
// tests: the same formulas the CUDA kernels run, with libm sin/cos in place of
// the MUFU approximations.  Built by tests/test_pairmath_host.py with g++.
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

// For each (face k, frequency m) pair: F and dF/dx_{a,b,c} (complex, interleaved
// re/im) and whether the fast path flagged it special.
// verts[nv*3] double, faces[nt*3] int64, m[nxi*3] int32; outputs sized nxi*nt.
void dm_host_pairs(const double* verts, const int64_t* faces, int64_t nt, const int32_t* m,
                   int64_t nxi, const double* lo, const double* len, float* F, float* dF,
                   uint8_t* special, int use_fast) {
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
      c32 E, G, Gu, Gw, Fv, d3[3];
      int piv;
      bool sp = pair_fast<true>(xv, g, E, G, Gu, Gw, piv);
      special[o] = sp ? 1 : 0;
      if (use_fast && !sp) {
        Fv = cmul(E, G);
        const c32 miF{Fv.y, -Fv.x};
        const c32 EGu = cmul(E, Gu), EGw = cmul(E, Gw);
        const int q = piv == 2 ? 0 : piv + 1, r = q == 2 ? 0 : q + 1;
        d3[piv] = c32{miF.x - EGu.x - EGw.x, miF.y - EGu.y - EGw.y};
        d3[q] = EGu;
        d3[r] = EGw;
      } else {
        pair_general<true>(xv, g, Fv, d3);
      }
      F[2 * o] = Fv.x;
      F[2 * o + 1] = Fv.y;
      for (int v = 0; v < 3; ++v) {
        dF[6 * o + 2 * v] = d3[v].x;
        dF[6 * o + 2 * v + 1] = d3[v].y;
      }
    }
  }
}

}  // extern "C"
