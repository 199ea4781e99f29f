// Project-written stand-in for OmniGS include/camera.h, for the drop-in link test only.
//
// The reference's GaussianRasterizationSettings (include/gaussian_rasterizer.h:36-49) names
// Camera::CameraModelType; src/gaussian_rasterizer.cpp casts it to int (:67, :84).  This header
// supplies just that enumeration with the reference's values (include/camera.h:54-58), so the
// reference's unmodified autograd layer compiles without OpenCV.
#pragma once

#include <torch/torch.h>

class Camera {
 public:
  enum CameraModelType { INVALID = 0, PINHOLE = 1, FISHEYE = 2, LONLAT = 3 };
};
