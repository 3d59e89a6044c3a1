#pragma once
#include <random>
namespace boost { namespace random { typedef std::mt19937 mt19937; } }
