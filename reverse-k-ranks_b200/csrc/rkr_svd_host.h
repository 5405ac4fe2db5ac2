// rkr_svd_host.h -- the host half of the SVD transform (rkr_host.cpp), shared by rkr_svd_build and
// the device build of rkr_index_svd_build (rkr_svd.cu).
#pragma once
#include <vector>

namespace rkr {
// From the Gram matrix G = user^T user ([d][d], full; overwritten): the singular values s
// (descending), their right singular vectors Es ([d][d], column k for s[k]), transfer_item
// ([d][d]: transfer_item[r][c] = s_r * Es[c][r]) and check_dim for sigma_ratio (SVD.hpp:62-124,
// 214-226).
void svd_from_gram(std::vector<double> &G, int d, float sigma_ratio, float *transfer_item, std::vector<double> &Es,
                   std::vector<float> &s, int *check_dim);
}  // namespace rkr
