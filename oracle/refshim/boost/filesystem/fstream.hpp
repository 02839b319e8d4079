// boost/filesystem/fstream.hpp -- host stand-in (TEST INFRASTRUCTURE): see boost/filesystem.hpp.
#include "../filesystem.hpp"
