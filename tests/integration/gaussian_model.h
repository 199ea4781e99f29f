// Project-written stand-in for OmniGS include/gaussian_model.h, for the drop-in link test only.
// include/gaussian_rasterizer.h includes it but src/gaussian_rasterizer.cpp uses nothing from it;
// the real header pulls in Sophus, simple-knn and tinyply, which this test does not need.
#pragma once

#include <torch/torch.h>
