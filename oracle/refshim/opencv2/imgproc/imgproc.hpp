// opencv2/imgproc/imgproc.hpp -- host stand-in (TEST INFRASTRUCTURE): everything lives in opencv2/opencv.hpp.
#include "../opencv.hpp"
