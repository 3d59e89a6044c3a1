#pragma once
#include <chrono>
namespace boost { namespace chrono { using std::chrono::system_clock; template <class R, class P = std::ratio<1>> using duration = std::chrono::duration<R, P>; using std::chrono::duration_cast; } }
