#pragma once
#include <random>
namespace boost { namespace random { template <class I = int> using uniform_int_distribution = std::uniform_int_distribution<I>; } }
