// Generated by gen_series.py (do not edit): centroid-series coefficients,
// terms n <= 14, monomials below 1e-09 for D <= 3.5 dropped.
// Ascending powers of p2.
#pragma once
#define DM_SERIES_P0_N 7
#define DM_SERIES_P0 {5.000000000e-01f, -2.083333333e-02f, 3.472222222e-04f, -3.100198413e-06f, 1.722332451e-08f, -6.523986559e-11f, 1.792304000e-13f}
#define DM_SERIES_P2_N 5
#define DM_SERIES_P2 {-2.755731922e-06f, 4.592886537e-08f, -3.479459498e-10f, 1.593159111e-12f, -4.978622221e-15f}
#define DM_SERIES_P4_N 1
#define DM_SERIES_P4 {1.416141432e-13f}
#define DM_SERIES_Q1_N 6
#define DM_SERIES_Q1 {2.777777778e-03f, -6.613756614e-05f, 6.889329806e-07f, -4.175351398e-09f, 1.672817066e-11f, -4.779477332e-14f}
#define DM_SERIES_Q3_N 3
#define DM_SERIES_Q3 {-9.278558661e-10f, 1.189558803e-11f, -7.080707159e-14f}
