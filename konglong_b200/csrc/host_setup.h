// host_setup.h - host-side table construction of the B200 RTM engine.
#pragma once
#include <vector>

namespace rtm {
// order-2*ne central-difference weights: c1[0..ne] (c1[0] = 0), c2[0..ne]
void fd_weights(int ne, double *c1, double *c2);
// compact FD factors of one axis: bm [n][5], bl [n][4], am [12][5]; isgn 1 or 2;
// rdiag [n] = 1 / pivot (FP64 division, then rounded)
void cfd_plan(int n, double d, int isgn, std::vector<float> &bm, std::vector<float> &bl, std::vector<float> &am,
              std::vector<float> *rdiag = nullptr);
// per-layer PML recursion constants [w][6] (scale 1, then scale `scaler`)
void pml_profile(int w, double d, double dt, double vmax, double eps, double scaler, std::vector<float> &co);
// FFTWR2R first derivative of one axis as a row-major n x n line matrix
// (out_t = sum_u D[t][u] x_u), isign +1 (cosine in, sine out) or -1
void r2r_line_matrix(int n, float d, int isign, std::vector<float> &D);
void r2c_line_matrix(int n, float d, int isign, std::vector<float> &D);
// Util::CompactOrmsbySpreadCoeff + edge taper; returns the first grid index
int spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, int ntaper, float *coeff);
}  // namespace rtm
