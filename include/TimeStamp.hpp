// Phase time stamp: (phase name, seconds), the same type as the reference's
// TimeStamp.hpp:7 so plugins and harnesses written against it compile here.
#pragma once

#include <string>
#include <utility>
#include <vector>

using TimeStamp = std::pair<std::string, double>;
