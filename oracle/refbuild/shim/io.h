#pragma once
#include <unistd.h>
inline int _access(const char* p, int m) { return access(p, m); }
