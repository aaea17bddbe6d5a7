// Stand-in for Boost.Filesystem's path header (see boost/filesystem.hpp).
#pragma once

#include "../filesystem.hpp"
