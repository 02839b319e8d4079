// opencv2/core/core.hpp -- host stand-in (TEST INFRASTRUCTURE): everything lives in opencv2/opencv.hpp.
#include "../opencv.hpp"
