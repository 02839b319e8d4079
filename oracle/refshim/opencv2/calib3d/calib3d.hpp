// opencv2/calib3d/calib3d.hpp -- host stand-in (TEST INFRASTRUCTURE): everything lives in opencv2/opencv.hpp.
#include "../opencv.hpp"
