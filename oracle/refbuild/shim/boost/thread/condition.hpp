// std stand-in for boost::condition (a condition variable usable with any lock).
#pragma once
#include <condition_variable>
namespace boost { typedef std::condition_variable_any condition; }
