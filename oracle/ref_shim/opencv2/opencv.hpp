// Test infrastructure only (the reference comparator build).
// Empty stand-in for <opencv2/opencv.hpp>: the reference's device headers
// include it but the depth-path kernels use nothing from OpenCV, and the
// OpenCV C++ headers are not installed in this image.
#pragma once
